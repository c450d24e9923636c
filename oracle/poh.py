"""Oracle: DPAC phase-only hologram encoding (export_poh.py:110-119, 175-194), numpy.

Test infrastructure only (see oracle/__init__.py). The padded field is the
oracle's soft window pad + amplitude clamp (oracle/blasm.py); phase, DPAC and
the 8-bit quantisation follow the reference in float32 (torch.angle % 2pi,
arccos of the clamped amplitude, checkerboard of -/+, % 2pi, round half to
even of poh / 2pi * 256, mod 256).
"""
import numpy as np

from . import blasm as ob


def dpac_levels(field, pH, pW):
    padded = ob.clamp_amplitude(ob.soft_window_pad(np.asarray(field, dtype=np.complex128), pH, pW))
    padded = padded.astype(np.complex64)
    two_pi = np.float32(2 * np.pi)
    phase = np.mod(np.angle(padded).astype(np.float32), two_pi)
    amp = np.clip(np.abs(padded).astype(np.float32), 0, 1)
    offset = np.arccos(amp).astype(np.float32)
    lo, hi = phase - offset, phase + offset
    y = np.arange(pH)[:, None]
    x = np.arange(pW)[None, :]
    poh = np.where(((y + x) % 2 == 0)[None], lo, hi).astype(np.float32)
    poh = np.mod(poh, two_pi)
    return (np.rint(poh / two_pi * np.float32(256)).astype(np.int64) % 256).astype(np.uint8)
