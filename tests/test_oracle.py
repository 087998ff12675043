"""The CPU oracle (test infrastructure) against its own invariants and against
the golden vectors of the reference library (tests/golden/)."""
import os

import numpy as np
import pytest

from conftest import ROOT
from geometry_cases import cone_case, fan_case, rel_l2
from sgd_b200.phantom import ellipse_chords, ellipse_phantom, ellipsoid_phantom, random_ellipses


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
    if kind.startswith("matgen_"):
        import scipy.sparse
        import scipy.sparse.linalg
        npv, nu, nx, ny = (int(v) for v in z["sizes"])
        dx, dy, du, lsd, lso = (float(v) for v in z["params"])
        shape = (npv * nu, nx * ny)
        r, c, v = oracle_mod.matrix_generation(kind[7:], npv, nu, nx, ny, dx, dy, du, lsd, lso, precision=1)
        M = scipy.sparse.csr_matrix((v, (r, c)), shape=shape)
        R = scipy.sparse.csr_matrix((z["vals"], (z["rows"], z["cols"])), shape=shape)
        assert scipy.sparse.linalg.norm(M - R) / scipy.sparse.linalg.norm(R) < 1e-5
        assert abs(M.nnz - R.nnz) <= 2e-3 * R.nnz
        return
    if kind in ("b1_3d", "sf3d"):
        g = tuple(int(v) for v in z["sizes"]) + tuple(float(v) for v in z["params"]) + (z["angles"],)
        if kind == "b1_3d":
            b, cnt = oracle_mod.b1_3d_forward(z["x"], *g)
            assert rel_l2(b, z["b"]) < 5e-5
            assert abs(cnt - int(z["count"])) <= 1e-4 * cnt + 3
            return
        # FP32 reference against the FP64 replica of its formulas
        assert rel_l2(oracle_mod.sf3d_forward(z["x"], *g), z["b"]) < 2e-5
        assert rel_l2(oracle_mod.sf3d_forward(z["x"], *g, trap=True), z["b_tt"]) < 2e-5
        assert rel_l2(oracle_mod.sf3d_backward(z["y"], *g), z["xt"]) < 2e-5
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


@pytest.mark.parametrize("case", ["fan512", "snap", "rect"])
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


@pytest.mark.parametrize("trap", [False, True])
def test_sf3d_corrected_oracle_is_adjoint(oracle_mod, trap):
    g = cone_case("tallz")
    nx, ny, nz, nu, nv = g[:5]
    rng = np.random.default_rng(3)
    x = rng.standard_normal(nx * ny * nz)
    y = rng.standard_normal(len(g[-1]) * nu * nv)
    lhs = np.dot(oracle_mod.sf3d_forward(x, *g, mode=1, trap=trap), y)
    rhs = np.dot(x, oracle_mod.sf3d_backward(y, *g, mode=1, trap=trap))
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


def test_sf3d_reference_forward_sees_support_only(oracle_mod):
    """layers/SF_projector.cu:190-221 never multiplies the footprint by the
    voxel value: the replica's reference mode depends on the support only."""
    g = cone_case("tallz")
    nx, ny, nz = g[:3]
    x = np.random.default_rng(4).random(nx * ny * nz) * (np.arange(nx * ny * nz) % 3 != 0)
    b = oracle_mod.sf3d_forward(x, *g)
    assert np.array_equal(b, oracle_mod.sf3d_forward((x != 0).astype(float), *g))
    assert not np.array_equal(b, oracle_mod.sf3d_forward(x, *g, mode=1))


# ---- exact FP64 projectors (the model-error references) --------------------

@pytest.mark.parametrize("kind", ["b0", "b1"])
def test_exact_matrix_line_integrals(oracle_mod, kind):
    """Exact matrix times the point-sampled ellipse phantom approaches the
    analytic ellipse line integrals as the pixels shrink."""
    nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case("snap")
    M = oracle_mod.exact_fan2d_matrix(kind, nx, ny, nu, dx, dy, du, lsd, lso, ang)
    assert M.shape == (len(ang) * nu, nx * ny) and np.all(M >= 0)
    # a single pixel's projections sum over bins to about its area / du (B0)
    # or the hat's integral dx dy / du (B1), magnified onto the detector
    col = M[:, (nx // 2) * ny + ny // 2].reshape(len(ang), nu).sum(axis=1)
    mag = lsd / lso
    assert np.allclose(col * du / mag, dx * dy, rtol=2e-2)


@pytest.mark.parametrize("kind", ["b0", "b1"])
@pytest.mark.parametrize("case", ["tiny", "snap"])
def test_formula_replica_model_error_vs_exact(oracle_mod, kind, case):
    """The reference formulas (replicated in FP64) against the exact
    bin-averaged line integrals of the same basis: the model error of the
    footprint approximations, stated per basis."""
    nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case(case)
    x = ellipse_phantom(nx, ny, dx, dy, seed=3).ravel()
    M = oracle_mod.exact_fan2d_matrix(kind, nx, ny, nu, dx, dy, du, lsd, lso, ang)
    b, _ = getattr(oracle_mod, f"{kind}_forward")(x, nx, ny, nu, dx, dy, du, lsd, lso, ang)
    err = rel_l2(b, M @ x)
    assert err < {"b0": 1e-3, "b1": 5e-4}[kind]


@pytest.mark.parametrize("case", ["tiny", "snap"])
def test_sf_model_error_vs_exact_pixel_indicator(oracle_mod, case):
    """A_SF approximates the pixel indicator's projection (trapezoid
    footprint): its FP64 replica against the exact bin-averaged chords."""
    nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case(case)
    x = ellipse_phantom(nx, ny, dx, dy, seed=3).ravel()
    M = oracle_mod.exact_fan2d_matrix("b0", nx, ny, nu, dx, dy, du, lsd, lso, ang)
    b, _ = oracle_mod.sf_forward(x, nx, ny, nu, dx, dy, du, lsd, lso, ang)
    assert rel_l2(b, M @ x) < 1e-3


def test_exact_hex_matrix_carries_the_hexagon_area(oracle_mod):
    """Nearly parallel rays (source 50 m away): a site's bin-averaged chords
    summed over the bins times the bin width at the site give the area of
    the regular hexagon of circumradius dt, (3 sqrt 3 / 2) dt^2."""
    nl, nc, nu, dt, du = 5, 4, 80, 2.0, 0.25
    lsd, lso = 1.0e5, 5.0e4
    ang = np.array([0.0, 0.37, np.pi / 6, 1.9])
    M = oracle_mod.exact_hex_matrix(nl, nc, nu, dt, du, lsd, lso, ang)
    site = 1 * nl + 2  # ic = 1, il = 2 (an even row)
    col = M[:, site].reshape(len(ang), nu).sum(axis=1)
    area = 1.5 * np.sqrt(3.0) * dt * dt
    # the site sits 1.7 mm off the isocentre: its magnification differs from
    # lsd / lso by ~4e-5 depending on the view
    assert np.allclose(col * du * lso / lsd, area, rtol=1e-4)
    assert not M[:, (nc - 1) * nl + 1].any()  # odd rows hold nc - 1 sites


def test_h0_model_error_vs_exact_hexagon(oracle_mod):
    """H0's value is three times the hexagon indicator's chord (the sum of
    the three unit-integral rhombus splines scaled by the hexagon area,
    layers/A_H0.cu:245); with the true hexagon bounds its FP64 replica sits
    within 1e-4 of the exact bin-averaged chords, while the reference's
    bounds (at the 0.5 dt row pitch, layers/A_H0.cu:556) lose mass away from
    the centre row."""
    nl, nc, nu, dt, du, lsd, lso = 16, 12, 60, 2.0, 1.5, 1085.6, 595.0
    ang = np.array([0.3, 1.1, np.pi / 4, 2.5])
    M = oracle_mod.exact_hex_matrix(nl, nc, nu, dt, du, lsd, lso, ang)
    x = np.random.default_rng(0).random(nc * nl)
    exact = 3.0 * (M @ x)
    b, _ = oracle_mod.hex_forward("h0c", x, nl, nc, nu, dt, du, lsd, lso, ang)
    assert rel_l2(b, exact) < 1e-4
    b_ref, _ = oracle_mod.hex_forward("h0", x, nl, nc, nu, dt, du, lsd, lso, ang)
    assert rel_l2(b_ref, exact) > 0.1


def test_exact_hl_matrix_carries_the_hat_integral(oracle_mod):
    """Nearly parallel rays: a site's bin-averaged line integrals of the
    Courant hat summed over the bins times the bin width at the site give
    the hat's integral, (sqrt 3 / 2) dt^2 (the triangular lattice's cell)."""
    nl, nc, nu, dt, du = 5, 4, 80, 2.0, 0.25
    lsd, lso = 1.0e5, 5.0e4
    ang = np.array([0.0, 0.37, np.pi / 6, 1.9])
    M = oracle_mod.exact_hl_matrix(nl, nc, nu, dt, du, lsd, lso, ang)
    col = M[:, 1 * nl + 2].reshape(len(ang), nu).sum(axis=1)
    # the site sits 1.7 mm off the isocentre (magnification off by ~4e-5)
    assert np.allclose(col * du * lso / lsd, 0.5 * np.sqrt(3.0) * dt * dt, rtol=1e-4)


def test_hl_model_error_vs_exact_linear_element(oracle_mod):
    """Hl's formula (the X-ray of the three-direction box spline convolved
    with the bin's width, layers/A_Hl.cu:21-46) against the exact bin-averaged
    line integrals of the Courant hat: the model error of its bin blur."""
    nl, nc, nu, dt, du, lsd, lso = 24, 12, 60, 2.0, 1.5, 1085.6, 595.0
    ang = np.array([0.3, 1.1, np.pi / 4, 2.5])
    M = oracle_mod.exact_hl_matrix(nl, nc, nu, dt, du, lsd, lso, ang)
    x = np.random.default_rng(0).random(nc * nl)
    b, _ = oracle_mod.hex_forward("hl", x, nl, nc, nu, dt, du, lsd, lso, ang)
    assert rel_l2(b, M @ x) < 5e-5


def test_sf3d_corrected_against_voxel_chords(oracle_mod):
    """The corrected SF_projector forward (FP64 replica) against the voxel
    indicator's chord lengths averaged over the detector cells (the Simpson
    restatement of Ref_project_Simpson, adaptive): unit scale for 2 mm voxels
    (the reference's amplitude would give half), model error below 1e-3."""
    nx, ny, nz, nu, nv, dx, dy, dz, du, dv, lsd, lso, ang = cone_case("small")
    ang = ang[:3] + 0.013
    x = ellipsoid_phantom(nx, ny, nz, dx, dy, dz, seed=0).ravel()
    g = (nx, ny, nz, nu, nv, dx, dy, dz, du, dv, lsd, lso, ang)
    r = oracle_mod.ref_simpson_3d(x, *g, adaptive=True)
    b = oracle_mod.sf3d_forward(x, *g, mode=1)
    alpha = float(b @ r) / float(r @ r)
    assert abs(alpha - 1.0) < 2e-3
    assert rel_l2(b, r) < 2e-3


@pytest.mark.parametrize("voxel", [(2.0, 1.6, 2.0), (2.0, 2.0, 1.5), (1.5, 2.5, 2.0)])
def test_sf3d_corrected_against_voxel_chords_non_cubic(oracle_mod, voxel):
    """As above on non-cubic voxels: the corrected amplitude (the voxel's
    volume over the squared source distance, times the normalised trapezoid
    and rectangle) keeps unit scale for any voxel shape."""
    nx, ny, nz, nu, nv, _, _, _, du, dv, lsd, lso, ang = cone_case("small")
    dx, dy, dz = voxel
    ang = ang[:3] + 0.013
    x = ellipsoid_phantom(nx, ny, nz, dx, dy, dz, seed=0).ravel()
    g = (nx, ny, nz, nu, nv, dx, dy, dz, du, dv, lsd, lso, ang)
    r = oracle_mod.ref_simpson_3d(x, *g, adaptive=True)
    b = oracle_mod.sf3d_forward(x, *g, mode=1)
    assert abs(float(b @ r) / float(r @ r) - 1.0) < 4e-3
    assert rel_l2(b, r) < 4e-3


def test_chord_simpson_3d(oracle_mod):
    """Ref_project_Simpson restated: a uniform odd-sized cube seen along +x
    carries its length on the central cell (the nine samples avoid voxel
    faces); a row of voxels with an edge on the central ray covers a quarter
    of the central cell, which the adaptive rule resolves and the reference's
    fixed 3 x 3 rule does not (its centre sample lies on the edge)."""
    from geometry_cases import LSD, LSO
    n, d = 15, 2.0
    g = (n, n, n, 24, 24, d, d, d, 3.0, 3.0, LSD, LSO, np.array([0.0]))
    for adaptive in (False, True):
        b = oracle_mod.ref_simpson_3d(np.ones(n ** 3), *g, adaptive=adaptive).reshape(24, 24)
        assert abs(b[12, 12] - n * d) / (n * d) < 1e-3
    g = cone_case("tiny")
    nx, ny, nz, nu, nv = g[:5]
    x = np.zeros((nz, ny, nx))
    x[nz // 2, ny // 2, :] = 1
    b = oracle_mod.ref_simpson_3d(x.ravel(), *g, adaptive=True, max_depth=6).reshape(len(g[-1]), nv, nu)
    assert abs(b[0, nv // 2, nu // 2] - nx * g[5] / 4) / (nx * g[5] / 4) < 1e-2
    b3 = oracle_mod.ref_simpson_3d(x.ravel(), *g).reshape(len(g[-1]), nv, nu)
    assert b3[0, nv // 2, nu // 2] > 2 * b[0, nv // 2, nu // 2]


QUAD = os.path.join(GOLDEN, "quad")


def _quad_files():
    return sorted(f for f in os.listdir(QUAD) if f.endswith(".npz")) if os.path.isdir(QUAD) else []


@pytest.mark.parametrize("fname", _quad_files())
def test_exact_oracle_matches_reference_quad(oracle_mod, fname):
    """The exact FP64 matrices against the reference's own exact projectors
    (python/matrix_gen/A_B0_ref_project.py, A_B1_ref_project.py: scipy quad
    per bin, run unmodified by tests/golden/quad/make_quad_golden.py).

    B0 (chord through the pixel square) agrees for any pixel shape.  The B1
    script returns the bilinear element's line integral divided by the pixel
    area dx*dy (the reference's CUDA kernel multiplies it in,
    layers/A_B1.cu:201, and so do the FP64 replica and this oracle), and it
    gives each side's pitch the other side's blur (A_B1_ref_project.py:39-40,
    vx = dx sin(theta) with theta measured from the y axis), which only shows
    when dx != dy: these fixtures keep square pixels, where the two agree once
    scaled by dx*dy."""
    z = np.load(os.path.join(QUAD, fname))
    kind = str(z["kind"])
    nx, ny, npv, nu = (int(v) for v in z["sizes"])
    dx, dy, du, lsd, lso = (float(v) for v in z["params"])
    ang = np.linspace(0, 2 * np.pi, npv, endpoint=False)
    Q = np.zeros((npv * nu, nx * ny))
    Q[z["rows"], z["cols"]] = z["vals"]
    E = oracle_mod.exact_fan2d_matrix(kind, nx, ny, nu, dx, dy, du, lsd, lso, ang)
    scale = dx * dy if kind == "b1" else 1.0
    assert rel_l2(E, scale * Q) < 1e-6
    # every entry the quadrature keeps, to its absolute tolerance (1.49e-8)
    assert np.abs(E - scale * Q).max() < 5e-6 * np.abs(E).max()
    if kind == "b1" and dx != 1.0:
        assert abs(rel_l2(E, Q) - abs(dx * dy - 1.0)) < 1e-6  # E = dx*dy Q: the missing factor, exactly


def test_formula_model_errors_against_reference_quad_on_non_square_pixels(oracle_mod):
    """The reference's B0 and A_SF formulas (FP64 replicas) against the
    reference's own exact pixel-indicator projector on 1.0 x 0.8 mm pixels
    (tests/golden/quad/quad_b0_aniso.npz).  B0 keeps its model error; A_SF's
    amplitude dx / max(|sin t|, |cos t|) (layers/A_SF.cu:177, :316) is the
    pixel's chord along the ray only for square pixels and is 15 % off here,
    while the chord min(dx / |sin t|, dy / |cos t|) brings it back to the
    square-pixel model error."""
    z = np.load(os.path.join(QUAD, "quad_b0_aniso.npz"))
    nx, ny, npv, nu = (int(v) for v in z["sizes"])
    dx, dy, du, lsd, lso = (float(v) for v in z["params"])
    assert dx != dy
    ang = np.linspace(0, 2 * np.pi, npv, endpoint=False)
    Q = np.zeros((npv * nu, nx * ny))
    Q[z["rows"], z["cols"]] = z["vals"]
    x = ellipse_phantom(nx, ny, dx, dy, seed=3).ravel()
    y = Q @ x
    b0, _ = oracle_mod.b0_forward(x, nx, ny, nu, dx, dy, du, lsd, lso, ang)
    assert rel_l2(b0, y) < 1e-3
    sf, _ = oracle_mod.sf_forward(x, nx, ny, nu, dx, dy, du, lsd, lso, ang)
    assert rel_l2(sf, y) > 0.1
    chord, _ = oracle_mod.sf_forward(x, nx, ny, nu, dx, dy, du, lsd, lso, ang, chord=True)
    assert rel_l2(chord, y) < 2e-3


@pytest.mark.parametrize("voxel,dv", [(1.0, 0.75), (2.0, 1.5), (2.0, 3.0)])
def test_b1_3d_scale_is_the_row_height_at_the_isocentre(oracle_mod, voxel, dv):
    """A uniform cube's central rays against their path lengths (adaptive
    Simpson voxel chords).  The reference's A_B1_3D forward (FP64 replica)
    normalises each voxel's axial trapezoid to unit area
    (layers/A_B1_3D.cu:210), so a detector row receives a fraction of the
    voxel instead of a density per mm: its value is the line integral times
    the row height projected to the isocentre, dv * lso / lsd, whatever the
    voxel size.  The corrected SF_projector carries the line integral."""
    from geometry_cases import LSD, LSO
    n, nd = 16, 24
    ang = np.array([0.3])
    g = (n, n, n, nd, nd, voxel, voxel, voxel, 1.5, dv, LSD, LSO, ang)
    x = np.ones(n ** 3)
    r = oracle_mod.ref_simpson_3d(x, *g, adaptive=True).reshape(nd, nd)
    b, _ = oracle_mod.b1_3d_forward(x, *g)
    s = oracle_mod.sf3d_forward(x, *g, mode=1).reshape(nd, nd)
    c = (slice(nd // 2 - 2, nd // 2 + 2), slice(nd // 2 - 2, nd // 2 + 2))
    ratio = b.reshape(nd, nd)[c] / r[c]
    assert np.all(np.abs(ratio / (dv * LSO / LSD) - 1.0) < 1e-2)
    assert np.all(np.abs(s[c] / r[c] - 1.0) < 5e-3)
