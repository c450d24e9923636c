"""CPU: pin the pad/clamp/BLASM oracle to the reference propagator (with the restated odak functions)."""
import numpy as np
import pytest

from conftest import rel_l2
from oracle import blasm as ob

CASES = ["propagate_rgb", "propagate_gray_bandlimit"]


def _args(g):
    return (int(g["pH"]), int(g["pW"]), list(g["wavelengths"]), list(g["distances"]), float(g["pitch"]))


@pytest.mark.parametrize("name", CASES)
def test_oracle_intensity_matches_reference(golden, name):
    g = golden(name)
    pH, pW, wl, dist, dx = _args(g)
    V = ob.chain_forward(g["field"].astype(np.complex128), pH, pW, wl, dist, dx, aperture_radius=float(g["aperture"]))
    assert rel_l2(np.abs(V) ** 2, g["I_crop"]) < 2e-5
    Vfull = ob.chain_forward(g["field"].astype(np.complex128), pH, pW, wl, dist, dx, out_hw=(pH, pW),
                             aperture_radius=float(g["aperture"]))
    assert rel_l2(np.abs(Vfull) ** 2, g["I_full"]) < 2e-5


@pytest.mark.parametrize("name", CASES)
def test_oracle_gradient_matches_reference_autograd(golden, name):
    g = golden(name)
    pH, pW, wl, dist, dx = _args(g)
    field = g["field"].astype(np.complex128)
    V = ob.chain_forward(field, pH, pW, wl, dist, dx, aperture_radius=float(g["aperture"]))
    gV = 2.0 * V * g["wts"]  # d(sum w |V|^2)/dV in the torch convention
    gf = ob.chain_backward(field, gV, pH, pW, wl, dist, dx, aperture_radius=float(g["aperture"]))
    assert rel_l2(gf, g["grad_field"]) < 2e-4
    assert gf[0, 3, 5] == 0


def test_propagate_adjoint_identity():
    rng = np.random.default_rng(0)
    C, pH, pW, oh, ow = 3, 20, 24, 12, 14
    x = rng.normal(size=(C, pH, pW)) + 1j * rng.normal(size=(C, pH, pW))
    y = rng.normal(size=(2, C, oh, ow)) + 1j * rng.normal(size=(2, C, oh, ow))
    wl, dist = [639e-9, 515e-9, 473e-9], [1e-3, 2e-3]
    lhs = np.vdot(y, ob.propagate(x, wl, dist, 8e-6, (oh, ow), aperture_radius=15))
    rhs = np.vdot(ob.propagate_adjoint(y, (pH, pW), wl, dist, 8e-6, aperture_radius=15), x)
    assert abs(lhs - rhs) < 1e-10 * abs(lhs)
