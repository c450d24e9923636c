"""CPU: the counter-based target-noise generator of the oracle.

Philox4x32-10 is pinned to the known-answer vectors published with the
algorithm (J. K. Salmon et al., "Parallel Random Numbers: As Easy as 1, 2, 3",
SC 2011; Random123 distribution); the kernels' generator is compared with this
one through the noisy loss on the GPU.
"""
import numpy as np

from oracle import loss as oloss


def test_philox4x32_10_known_answers():
    cases = [((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
             ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
             ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
              (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]
    for ctr, key, want in cases:
        got = tuple(int(v) for v in oloss.philox4x32_10(*ctr, *key))
        assert got == want


def test_plane_noise_layout_and_moments():
    shape = (2, 3, 37, 41)
    z = oloss.plane_noise(shape, 11, 5)
    assert z.shape == shape and z.dtype == np.float32
    assert np.array_equal(z, oloss.plane_noise(shape, 11, 5))
    assert not np.array_equal(z, oloss.plane_noise(shape, 11, 6))
    assert not np.array_equal(z, oloss.plane_noise(shape, 12, 5))
    # rows 4q..4q+3 of a column come from one counter, in lane order
    P, C, H, W = shape
    n4 = oloss.normals4_at(11, 5, np.array([(1 * C + 2) * ((H + 3) // 4) * W + 3 * W + 7], dtype=np.uint64))[0]
    assert np.array_equal(z[1, 2, 12:16, 7], n4)
    big = oloss.plane_noise((1, 1, 512, 512), 3, 0).ravel().astype(np.float64)
    assert abs(big.mean()) < 0.01 and abs(big.std() - 1.0) < 0.01
