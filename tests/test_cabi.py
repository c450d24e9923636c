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


def test_blasm_host_queries():
    import ctypes as ct
    from complex_valued_quadratic_phase_gaussian_b200 import _lib
    from complex_valued_quadratic_phase_gaussian_b200.propagator import BlasmParams
    lib = _lib.lib()
    p = BlasmParams()
    p.channels, p.planes, p.height, p.width, p.pad_height, p.pad_width = 3, 3, 1080, 1920, 1408, 2240
    p.pixel_pitch = 3.74e-6
    for i, wl in enumerate((639e-9, 515e-9, 473e-9)):
        p.wavelengths[i] = wl
    for i, z in enumerate((5e-4, 1e-3, 1.5e-3)):
        p.distances[i] = z
    t = _lib.size_query(lib.cvqpg_blasm_tables_size, ct.byref(p))
    w = _lib.size_query(lib.cvqpg_blasm_workspace_size, ct.byref(p))
    assert 0 < t < 1 << 20
    # row-pass intermediate (C x 2pW x pH) + kept column output (P x C x H x 2pW), complex64
    assert w >= 8 * (3 * 4480 * 1408 + 9 * 1080 * 4480)
    p.height = 1081  # odd sizes are rejected
    with pytest.raises(RuntimeError):
        _lib.size_query(lib.cvqpg_blasm_workspace_size, ct.byref(p))
