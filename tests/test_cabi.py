"""CPU: the C-ABI library loads and exports every symbol include/cvqpg.h declares (no GPU calls)."""
import ctypes
import os
import re

import pytest

from conftest import REPO

HEADER = os.path.join(REPO, "include", "cvqpg.h")


def declared_in_header():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"CVQPG_API\s+[\w\s\*]+?\b(cvqpg_\w+)\s*\(", text)))


def test_header_and_binding_agree():
    from complex_valued_quadratic_phase_gaussian_b200 import _lib
    assert declared_in_header() == _lib.declared_symbols()


def test_library_exports_every_declared_symbol():
    from complex_valued_quadratic_phase_gaussian_b200 import _lib
    from complex_valued_quadratic_phase_gaussian_b200.build import build as build_lib
    build_lib()
    handle = ctypes.CDLL(_lib.LIB_PATH)
    missing = [s for s in declared_in_header() if not hasattr(handle, s)]
    assert not missing, missing


def test_host_only_queries():
    from complex_valued_quadratic_phase_gaussian_b200 import _lib
    lib = _lib.lib()
    assert lib.cvqpg_status_string(0) == b"ok"
    assert lib.cvqpg_version() >= 100
    n = _lib.size_query(lib.cvqpg_render_workspace_size, 1000, 64, 64, 5000)
    assert n > 1000 * 64
    assert lib.cvqpg_render_num_lists(0, 1920, 1080) == 120 * 68
    assert lib.cvqpg_render_num_lists(1, 1920, 1080) == 30 * 17
    assert lib.cvqpg_render_num_lists(2, 1920, 1080) == 1
    with pytest.raises(RuntimeError):
        _lib.size_query(lib.cvqpg_render_workspace_size, -1, 64, 64, 10)
