"""GPU: multi-plane defocus targets (cvqpg_targets_synthesize) against the reference loss and the oracle.

Gates: plane index exact; targets within 1e-5 relative L2 of the reference's
get_targets() (float32 2D correlation vs separable float32 passes) and of the
float64 oracle. The golden puts one plane only where the image is zero, so the
reference's "masked image sums to zero" rule (its term is dropped) is checked.
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import loss as oloss

pytestmark = pytest.mark.gpu


def test_targets_match_reference_get_targets(golden):
    from complex_valued_quadratic_phase_gaussian_b200.scenes import multiplane_targets_device
    g = golden("targets_rgb")
    t, q = multiplane_targets_device(g["image"], g["depth"], int(g["P"]))
    torch.cuda.synchronize()
    assert np.array_equal(q.cpu().numpy(), g["plane"])
    assert rel_l2(t.cpu().numpy(), g["targets"]) < 1e-5
    assert float(t[:, :, :, :6].abs().max()) == 0.0  # the dropped plane


@pytest.mark.parametrize("P,split", [(3, 1.0), (2, 0.5), (5, 1.0)])
def test_targets_match_oracle(P, split):
    from complex_valued_quadratic_phase_gaussian_b200.scenes import multiplane_targets_device, rgb_blobs
    img, depth = rgb_blobs(80, 120, seed=P, num_blobs=50)
    t, q = multiplane_targets_device(img, depth, P, split_ratio=split)
    ref, qref = oloss.defocus_targets(img, depth, P, split_ratio=split)
    torch.cuda.synchronize()
    assert np.array_equal(q.cpu().numpy(), qref)
    assert rel_l2(t.cpu().numpy(), ref) < 1e-5
