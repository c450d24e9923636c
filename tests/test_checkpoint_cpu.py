"""CPU: the checkpoint format and the POH oracle against the reference's own code
(tests/golden/make_golden.py: checkpoint, dpac).

* A checkpoint the reference's Gaussians2D.save_gaussians wrote (model_2d_gaussian_rgb.py:155-167)
  reads back here with the same values and image size.
* A checkpoint this library's save_gaussians writes has the reference file's keys, dtypes and
  shapes, and the reference's Gaussians2D.load_gaussians (:169-180) loaded exactly its values.
* The DPAC oracle (oracle/poh.py) reproduces the reference's 8-bit POH levels
  (export_poh.py:110-119, 175-180): at least 99.9 % identical, the rest one level apart.
"""
import os

import numpy as np
import torch

from conftest import GOLDEN
from oracle import poh as opoh

RAW = ("means_2d", "pre_act_scales", "pre_act_rotation", "colours", "pre_act_phase", "pre_act_opacities",
       "curvature")


def test_reads_reference_checkpoint(golden):
    from complex_valued_quadratic_phase_gaussian_b200.fit import read_gaussians
    g = golden("checkpoint")
    raw, size = read_gaussians(os.path.join(GOLDEN, "checkpoint_ref.pth"))
    assert size == (int(g["W"]), int(g["H"]))
    for k in RAW:
        np.testing.assert_array_equal(raw[k].numpy(), g[f"ref_{k}"])


def test_written_checkpoint_matches_reference_format(golden, tmp_path):
    from complex_valued_quadratic_phase_gaussian_b200.fit import read_gaussians, save_gaussians
    g = golden("checkpoint")
    path = str(tmp_path / "ours.pth")
    save_gaussians({k: g[f"ours_{k}"] for k in RAW}, (int(g["W"]), int(g["H"])), path)
    mine = torch.load(path, map_location="cpu")
    ref = torch.load(os.path.join(GOLDEN, "checkpoint_ref.pth"), map_location="cpu")
    assert set(mine) == set(ref)
    assert type(mine["img_size"]) is type(ref["img_size"]) and tuple(mine["img_size"]) == tuple(ref["img_size"])
    for k in RAW:
        assert mine[k].dtype == ref[k].dtype and mine[k].shape == ref[k].shape and mine[k].device == ref[k].device
        np.testing.assert_array_equal(mine[k].numpy(), g[f"ours_{k}"])
        np.testing.assert_array_equal(g[f"loaded_{k}"], g[f"ours_{k}"])  # what the reference's loader read
    raw, size = read_gaussians(path)
    assert size == (int(g["W"]), int(g["H"]))


def test_dpac_oracle_matches_reference(golden):
    g = golden("dpac")
    pH, pW = (int(v) for v in g["pad"])
    got = opoh.dpac_levels(g["field"], pH, pW)
    ref = g["levels"]
    assert got.shape == ref.shape
    diff = (got.astype(np.int64) - ref.astype(np.int64)) % 256
    diff = np.minimum(diff, 256 - diff)
    assert np.mean(diff == 0) >= 0.999 and diff.max() <= 1
