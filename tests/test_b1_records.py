"""The B1 footprint records the kernels read, built by the library's host code
(sgd_b1_bin_records) and evaluated here on the CPU: the closed-form footprint
of each (pixel, view, bin), summed into a forward projection, against the
FP64 replica of the reference formula (layers/A_B1.cu:182-202,
layers/spline_conv.hh:295-405).  This checks the record layout and every
constant of the closed form without a GPU; the kernels' own arithmetic on
the same records is checked on the GPU (tests/test_b1_gpu.py)."""
import ctypes

import numpy as np
import pytest

from geometry_cases import fan_case, rel_l2
from sgd_b200.phantom import ellipse_phantom

KCONV_EPS = 1e-7  # the reference's footprint threshold (layers/A_B1.cu:203)


def records(nx, ny, nu, dx, dy, du, lsd, lso, ang, dz=None, drho=None):
    """(np, nu, 16) float32 records, fields in the order of the C layout."""
    from sgd_b200 import _lib
    L = _lib.lib()
    dp = ctypes.POINTER(ctypes.c_double)
    f = L.sgd_b1_bin_records
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 5 + [dp, dp, dp, ctypes.c_void_p]
    npv = len(ang)
    out = np.zeros(npv * nu * 16, dtype=np.float32)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) if a is not None else None for a in (ang, dz, drho)]
    ptrs = [a.ctypes.data_as(dp) if a is not None else None for a in arrs]
    assert f(nx, ny, npv, nu, dx, dy, du, lsd, lso, *ptrs, out.ctypes.data) == 0, _lib.last_error()
    # [view][chunk][bin][4] -> [view][bin][chunk*4 + k]
    return out.reshape(npv, 4, nu, 4).transpose(0, 2, 1, 3).reshape(npv, nu, 16)


def G(y, r):
    """Odd extension of the cumulative profile, y in units of the half-width
    a, from the record's constants (FP64 evaluation of the FP32 constants)."""
    beta, opb, nk3, k4 = r[..., 6], r[..., 8], r[..., 10], r[..., 12]
    ay = np.abs(y)
    w = np.maximum(beta - ay, 0.0)
    s_in = ay - 0.5 * ay * ay + nk3 + k4 * w ** 4
    p = np.maximum(opb - ay, 0.0)
    q = np.maximum(1.0 - ay, 0.0)
    s_out = 0.5 + k4 * (q ** 4 + w ** 4 - 0.5 * p ** 4)
    return np.copysign(np.where(1.0 - ay >= beta, s_in, s_out), y)


def forward_from_records(rec, x, nx, ny, dx, dy):
    i = np.arange(nx, dtype=np.float64)[None, :, None]
    j = np.arange(ny, dtype=np.float64)[None, None, :]
    img = x.reshape(nx, ny)                                   # host layout x[i*ny + j]
    out = np.empty(rec.shape[:2])
    for p in range(rec.shape[0]):                             # one view at a time
        r = rec[p].astype(np.float64)[:, None, None, :]       # (nu, 1, 1, 16)
        ya = i * r[..., 0] + (j * r[..., 2] + r[..., 4])
        yb = i * r[..., 1] + (j * r[..., 3] + r[..., 5])
        conv = (G(yb, r) - G(ya, r)) / (yb - ya) * r[..., 14]
        conv = np.where(conv > KCONV_EPS, conv, 0.0)
        out[p] = (dx * dy) * np.einsum("uij,ij->u", conv, img)
    return out.ravel()


@pytest.mark.parametrize("case", ["tiny", "rect", "snap", "wide"])
def test_records_reproduce_the_reference_formula(oracle_mod, case):
    nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case(case)
    ang = ang[:: max(1, len(ang) // 12)]                      # at most about a dozen views
    rec = records(nx, ny, nu, dx, dy, du, lsd, lso, ang)
    x = ellipse_phantom(nx, ny, dx, dy, seed=5).ravel()
    b_ref, _ = oracle_mod.b1_forward(x, nx, ny, nu, dx, dy, du, lsd, lso, ang)
    assert rel_l2(forward_from_records(rec, x, nx, ny, dx, dy), b_ref) < 5e-6


def test_records_with_source_offsets(oracle_mod):
    """drho moves the source along its axis (utils/geo.cu:248-251); dz does
    not enter a 2D footprint."""
    nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case("rect")
    ang = ang[::3]
    rng = np.random.default_rng(9)
    dz, drho = rng.uniform(-5, 5, len(ang)), rng.uniform(-8, 8, len(ang))
    rec = records(nx, ny, nu, dx, dy, du, lsd, lso, ang, dz, drho)
    x = ellipse_phantom(nx, ny, dx, dy, seed=6).ravel()
    b_ref, _ = oracle_mod.b1_forward(x, nx, ny, nu, dx, dy, du, lsd, lso, ang, dz, drho)
    assert rel_l2(forward_from_records(rec, x, nx, ny, dx, dy), b_ref) < 5e-6
    assert np.array_equal(rec, records(nx, ny, nu, dx, dy, du, lsd, lso, ang, None, drho))


def test_record_fields_are_consistent():
    nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case("rect")
    r = records(nx, ny, nu, dx, dy, du, lsd, lso, ang).astype(np.float64)
    for k in (6, 8, 10, 12):                                  # stored operand pairs
        assert np.array_equal(r[..., k], r[..., k + 1])
    beta, a = r[..., 6], r[..., 15]
    assert np.all(beta <= 1) and np.all(beta >= 0) and np.all(a > 0)
    assert np.allclose(r[..., 8], 1 + beta, rtol=1e-6)
    assert np.allclose(r[..., 10], -beta * beta / 12, rtol=1e-6, atol=1e-12)
    assert np.allclose(r[..., 14], 1 / a, rtol=1e-6)
    nz = beta * a > 1e-7
    assert np.allclose(r[..., 12][nz], 1 / (12 * beta[nz] ** 2), rtol=1e-6)
    assert np.all(r[..., 12][~nz] == 0)
    # a and b = beta a are the pixel's half-widths across the central ray:
    # a^2 + b^2 lies between min(dx, dy)^2 and max(dx, dy)^2
    s = a * a * (1 + beta * beta)
    assert np.all(s >= min(dx, dy) ** 2 * (1 - 1e-6)) and np.all(s <= max(dx, dy) ** 2 * (1 + 1e-6))


def test_records_reject_bad_geometry():
    from sgd_b200 import _lib
    with pytest.raises(AssertionError, match="lso < lsd"):
        records(8, 8, 12, 1.0, 1.0, 1.0, 10.0, 20.0, np.zeros(4))
    assert "lso < lsd" in _lib.last_error()
