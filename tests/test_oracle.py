"""The CPU oracle (test infrastructure) against its own invariants and against
the golden vectors of the reference library (tests/golden/)."""
import os

import numpy as np
import pytest

from conftest import ROOT
from geometry_cases import fan_case, rel_l2
from sgd_b200.phantom import ellipse_phantom, ellipse_chords, random_ellipses


def test_geometry_snaps_45_degree_views(oracle_mod):
    nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case("snap")
    g = oracle_mod.geometry(nx, ny, 1, nu, 1, dx, dy, 1, du, 1, lsd, lso, ang + 3e-8)
    # utils/geo.cu:254-257: within 1e-7 of an odd multiple of 45 degrees the angle is snapped
    puv = g["puv"][:4]
    assert np.allclose(np.abs(puv[:, 0]), np.abs(puv[:, 1]), atol=1e-12)
    # views 1 and 3 (3pi/4, 7pi/4 -> -pi/4) have puv.x == puv.y: the singular path
    assert abs(g["puv"][1, 0] - g["puv"][1, 1]) < 1e-12 and abs(g["puv"][3, 0] - g["puv"][3, 1]) < 1e-12


def test_geometry_maps_bin_centres(oracle_mod):
    nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case("rect")
    g = oracle_mod.geometry(nx, ny, 1, nu, 1, dx, dy, 1, du, 1, lsd, lso, ang)
    for p in range(len(ang)):
        if abs(g["puv"][p, 0] - g["puv"][p, 1]) < 1e-7:
            continue
        pm = g["pm"][p].reshape(3, 4)
        for u in (0, nu // 2, nu - 1):
            # a point on the ray through bin centre u maps to u + 1/2
            c = g["dtv"][p] + g["puv"][p] * (u - nu / 2 + 0.5)
            X = g["src"][p] + 0.37 * (c - g["src"][p])
            h = pm @ np.append(X, 1.0)
            assert abs(h[0] / h[2] - (u + 0.5)) < 1e-9


@pytest.mark.parametrize("case", ["small", "rect", "snap", "wide"])
def test_oracle_b1_adjoint_fp64(oracle_mod, case):
    nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case(case)
    rng = np.random.default_rng(1234)
    x = rng.standard_normal(nx * ny)
    y = rng.standard_normal(len(ang) * nu)
    ax, _ = oracle_mod.b1_forward(x, nx, ny, nu, dx, dy, du, lsd, lso, ang)
    aty = oracle_mod.b1_backward(y, nx, ny, nu, dx, dy, du, lsd, lso, ang)
    assert abs(ax @ y - x @ aty) / abs(ax @ y) < 1e-12


def test_oracle_b1_fp32_emulation_close_to_fp64(oracle_mod):
    nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case("small")
    x = ellipse_phantom(nx, ny, dx, dy, seed=0).ravel()
    b64, c64 = oracle_mod.b1_forward(x, nx, ny, nu, dx, dy, du, lsd, lso, ang, precision=0)
    b32, c32 = oracle_mod.b1_forward(x, nx, ny, nu, dx, dy, du, lsd, lso, ang, precision=1)
    assert c64 == c32
    assert rel_l2(b32, b64) < 5e-6


def test_oracle_b1_matches_analytic_line_integrals(oracle_mod):
    # the B1 projection of a point-sampled smooth phantom approaches the exact
    # line integrals as the pixel shrinks (model error, not rounding)
    nx = ny = 256
    dx = dy = 0.5
    nu, du, LSD, lso = 64, 1.0, 1085.6, 595.0
    ang = np.array([0.2, 1.3])
    radius = 0.5 * nx * dx
    ell = random_ellipses(3, 4, radius)
    ell[:, 2:4] = np.maximum(ell[:, 2:4], 0.3 * radius)  # large, smooth-ish ellipses
    from sgd_b200.phantom import sample_ellipses, pixel_centres
    X, Y = pixel_centres(nx, ny, dx, dy)
    img = sample_ellipses(ell, X, Y)
    b, _ = oracle_mod.b1_forward(img.ravel(), nx, ny, nu, dx, dy, du, LSD, lso, ang)
    g = oracle_mod.geometry(nx, ny, 1, nu, 1, dx, dy, 1, du, 1, LSD, lso, ang)
    exact = []
    for p in range(len(ang)):
        c = g["dtv"][p][:2] + np.outer(np.arange(nu) - nu / 2 + 0.5, g["puv"][p][:2])
        s = np.broadcast_to(g["src"][p][:2], c.shape)
        exact.append(ellipse_chords(ell, s[:, 0], s[:, 1], c[:, 0], c[:, 1]))
    exact = np.concatenate(exact)
    assert rel_l2(b, exact) < 0.05


GOLDEN = os.path.join(ROOT, "tests", "golden")


def _golden_files():
    return sorted(f for f in os.listdir(GOLDEN) if f.endswith(".npz")) if os.path.isdir(GOLDEN) else []


@pytest.mark.parametrize("fname", _golden_files())
def test_oracle_matches_reference_golden(oracle_mod, fname):
    """Golden vectors written by the reference library built from its own
    sources and run on a B200 (tests/golden/make_golden.py)."""
    z = np.load(os.path.join(GOLDEN, fname))
    kind = str(z["kind"])
    if kind.startswith("hex_"):
        mode = kind[4:]
        nl, nc, nu = (int(v) for v in z["sizes"])
        dt, du, lsd, lso = (float(v) for v in z["params"])
        b, cnt = oracle_mod.hex_forward(mode, z["x"], nl, nc, nu, dt, du, lsd, lso, z["angles"])
        # the reference computes in FP32 (and steps bin centres in FP32); the
        # replica in FP64 from the same FP32 inputs
        assert rel_l2(b, z["b"]) < 5e-5
        assert cnt == int(z["count"])
        xt = oracle_mod.hex_backward(mode, z["y"], nl, nc, nu, dt, du, lsd, lso, z["angles"])
        assert rel_l2(xt, z["xt"]) < 5e-5
        return
    nx, ny, nu = (int(v) for v in z["sizes"])
    dx, dy, du, lsd, lso = (float(v) for v in z["params"])
    ang = z["angles"]
    fwd = getattr(oracle_mod, f"{kind}_forward")
    bwd = getattr(oracle_mod, f"{kind}_backward")
    b, cnt = fwd(z["x"], nx, ny, nu, dx, dy, du, lsd, lso, ang)
    assert rel_l2(b, z["b"]) < float(z["tol"])
    assert cnt == int(z["count"])
    xt = bwd(z["y"], nx, ny, nu, dx, dy, du, lsd, lso, ang)
    assert rel_l2(xt, z["xt"]) < float(z["tol"])


@pytest.mark.parametrize("case", ["c2", "snap", "rect"])
def test_product_pmi_bit_identical_to_oracle(oracle_mod, case):
    """The library's projection matrices (host code) equal the restatement of
    utils/geo.cu bit for bit: the separable-footprint and 3D kernels take
    their visited bins from floors of pmi projections."""
    import ctypes
    from sgd_b200 import _lib
    nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case(case)
    ang = np.ascontiguousarray(ang, dtype=np.float64)
    L = _lib.lib()
    pm = np.zeros((len(ang), 12))
    pmi = np.zeros((len(ang), 12), dtype=np.float32)
    dp = ctypes.POINTER(ctypes.c_double)
    assert L.sgd_geometry_pmi(nx, ny, 1, len(ang), nu, 1, ctypes.c_double(dx), ctypes.c_double(dy),
                              ctypes.c_double(1.0), ctypes.c_double(du), ctypes.c_double(1.0), ctypes.c_double(lsd),
                              ctypes.c_double(lso), ang.ctypes.data_as(dp), None, None, pm.ctypes.data_as(dp),
                              pmi.ctypes.data_as(ctypes.POINTER(ctypes.c_float))) == 0
    g = oracle_mod.geometry(nx, ny, 1, nu, 1, dx, dy, 1, du, 1, lsd, lso, ang)
    assert np.array_equal(pm, g["pm"])
    assert np.array_equal(pmi, g["pmi"])
