"""CPU: host helpers of bench.py that shape its JSON line (no GPU, no timing)."""
import importlib.util
import os

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(REPO, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_profiled_traffic_comes_from_the_workloads_own_profile(bench):
    """The roofline's `traffic` is read from the committed ncu summary of the same workload: the
    1080p summaries give the column adjoint's bytes, and a workload without a capture gives None
    rather than another workload's bytes."""
    t = bench.profiled_traffic("adjoint_columns")
    assert t is not None and 3e8 < t < 6e8  # 464.5 MB compulsory per 1080p launch
    assert bench.profiled_traffic("adjoint_columns", "rgb1080") == t
    assert bench.profiled_traffic("adjoint_columns", "gray256") is None
    assert bench.profiled_traffic("no_such_stage") is None


def test_stage_bytes_of_the_headline_grid(bench):
    """Compulsory bytes per launch that the roofline divides by the stage time (complex64 = 8 B)."""
    from complex_valued_quadratic_phase_gaussian_b200.fit import FitConfig
    cfg = FitConfig(img_size=(1920, 1080), num_gaussians=96000, wavelengths=[639e-9, 515e-9, 473e-9],
                    pixel_pitch=3.74e-6, num_planes=3, d_val=1e-3, volume_depth=1e-3)
    b = bench.stage_bytes(cfg)
    # adjoint columns: Bt read 3 x 3 x 1080 x 4480 x 8 B + Ab written 3 x 1080 x 4480 x 8 B
    assert b["adjoint_columns"] == 9 * 1080 * 4480 * 8 + 3 * 1080 * 4480 * 8
    # forward columns: A read 3 x 1408 x 4480 x 8 B + the kept rows of B written
    assert b["blasm_columns"] == 3 * 1408 * 4480 * 8 + 9 * 1080 * 4480 * 8
