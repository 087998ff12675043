"""The host plan of the generic 2D kernels, checked on the CPU.

The forward kernel enumerates, per (view, block of 32 bins), the cells of the
block's strip record; the back kernel evaluates each cell's bins inside its
tile's window.  Both are correct only if every cell whose footprint meets a
block is a candidate of that block, and every cell's footprint lies inside its
tile's window (a cell wholly off the detector, whose clamped range the
reference still evaluates at an edge bin, has footprint exactly 0 there).
The ranges here are computed independently: the reference's
rule (pixel corners at +-reach through the view's index-space matrix pmi,
floored and clamped; layers/A_B0.cu:158-195, layers/A_B1.cu:100-151), in FP64
from the oracle's pmi.  The snapped 45-degree views take their ranges from the
reference's singular-matrix rule, not from the geometry, and are left out (the
kernels evaluate the footprint from the true geometry there, which is zero
outside the geometric strip).
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle
from sgd_b200 import _lib

BLOCK, TI, TJ = 32, 8, 32


def plan_grid(nx, ny, nu, x0, dx, y0, dy, ri, rj, du, lsd, lso, ang):
    L = _lib.lib()
    f = L.sgd_fan2d_plan
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 9 + [ctypes.c_void_p] * 3
    np_ = len(ang)
    nblk = -(-nu // BLOCK)
    ti, tj = -(-nx // TI), -(-ny // TJ)
    strips = np.zeros((np_, nblk, 8), dtype=np.float32)
    twin = np.zeros((ti * tj, np_, 2), dtype=np.int32)
    a = np.ascontiguousarray(ang, dtype=np.float64)
    w = f(nx, ny, np_, nu, x0, dx, y0, dy, ri, rj, du, lsd, lso, a.ctypes.data, strips.ctypes.data,
          twin.ctypes.data)
    assert w > 0, _lib.last_error()
    return strips, twin, w


def plan(reach, nx, ny, nu, dx, dy, du, lsd, lso, ang):
    """Pixel grid centred on the isocentre, ranges from the corners at +-reach."""
    return plan_grid(nx, ny, nu, -0.5 * (nx - 1) * dx, dx, -0.5 * (ny - 1) * dy, dy, reach, reach, du, lsd, lso, ang)


def ranges(pmi, reach, nx, ny, nu):
    """(lo, hi, out) per pixel (ix, iy) of one view, the reference's rule."""
    ix, iy = np.meshgrid(np.arange(nx, dtype=np.float64), np.arange(ny, dtype=np.float64), indexing="ij")
    pm = pmi.astype(np.float64)
    us = []
    for sx in (-reach, reach):
        for sy in (-reach, reach):
            x, y = ix + sx, iy + sy
            us.append((pm[0] * x + pm[3] + pm[1] * y) / (pm[8] * x + pm[11] + pm[9] * y))
    us = np.stack(us)
    umin, umax = us.min(0), us.max(0)
    lo = np.clip(np.floor(umin), 0, nu - 1).astype(int)
    hi = np.clip(np.floor(umax), 0, nu - 1).astype(int)
    return lo, hi, (umax < 0) | (umin >= nu)


def candidates(rec, nx, ny):
    """Cells the forward kernel visits for one strip record (its FP32 arithmetic)."""
    f32 = np.float32
    jmaj = rec[0] > 0.5
    nmin = nx if jmaj else ny
    mask = np.zeros((nx, ny), dtype=bool)
    for m in range(int(rec[6]), int(rec[7]) + 1):
        na = f32(rec[2]) * f32(m) + f32(rec[1])
        nb = f32(rec[4]) * f32(m) + f32(rec[3])
        lo = max(0, int(np.ceil(f32(min(na, nb)) - f32(rec[5]))))
        hi = min(nmin - 1, int(np.floor(f32(max(na, nb)) + f32(rec[5]))))
        if hi < lo:
            continue
        if jmaj:
            mask[lo:hi + 1, m] = True
        else:
            mask[m, lo:hi + 1] = True
    return mask


CASES = {
    # nx, ny, nu, dx, dy, du, lsd, lso, views (subset of the full circle)
    "small": (40, 28, 70, 1.0, 1.0, 1.0, 300.0, 150.0, 2 * np.pi * np.arange(24) / 24),
    "aniso": (33, 47, 90, 0.8, 1.1, 1.3, 500.0, 260.0, 2 * np.pi * (np.arange(20) + 0.37) / 20),
    "fan512": (512, 512, 736, 0.5, 0.5, 1.0, 1085.6, 595.0, 2 * np.pi * np.arange(0, 720, 37) / 720),
}


@pytest.mark.parametrize("reach", [0.5, 1.0])
@pytest.mark.parametrize("case", sorted(CASES))
def test_plan_covers_every_range(case, reach):
    nx, ny, nu, dx, dy, du, lsd, lso, ang = CASES[case]
    strips, twin, wcap = plan(reach, nx, ny, nu, dx, dy, du, lsd, lso, ang)
    geo = oracle.geometry(nx, ny, 1, nu, 1, dx, dy, 1.0, du, 1.0, lsd, lso, ang)
    tj = -(-ny // TJ)
    tile = (np.arange(nx)[:, None] // TI) * tj + (np.arange(ny)[None, :] // TJ)
    checked = 0
    for p in range(len(ang)):
        puv = geo["puv"][p]
        if abs(np.float32(puv[0]) - np.float32(puv[1])) < 1e-7:
            continue  # snapped 45-degree view: the reference's singular range rule
        lo, hi, out = ranges(geo["pmi"][p], reach, nx, ny, nu)
        live = ~out
        # back: every range inside its tile's window
        w = twin[tile, p]
        ok = (~live) | ((lo >= w[..., 0]) & (hi <= w[..., 1]))
        assert ok.all(), f"view {p}: {np.count_nonzero(~ok)} ranges outside their tile windows"
        assert (w[..., 1] - w[..., 0] + 1).max() <= wcap
        # forward: every cell meeting a block is among its candidates
        for k in range(strips.shape[1]):
            u0, u1 = k * BLOCK, min(nu, (k + 1) * BLOCK) - 1
            need = live & (hi >= u0) & (lo <= u1)
            if not need.any():
                continue
            cand = candidates(strips[p, k], nx, ny)
            miss = need & ~cand
            assert not miss.any(), f"view {p} block {k}: {np.count_nonzero(miss)} cells missing from the strip"
            # the strip is not much wider than needed
            assert cand.sum() <= 1.6 * need.sum() + 8 * max(nx, ny)
            checked += 1
    assert checked > 0
