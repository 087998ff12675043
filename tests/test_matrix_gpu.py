"""System matrices built on the GPU: the layers' own matrices against their
projection kernels, and the reference's generators (pixel_matrix_generation,
bilinear_matrix_generation) against the reference library and the CPU replica."""
import numpy as np
import pytest
import scipy.sparse
import scipy.sparse.linalg

from geometry_cases import fan_case, hex_case, rel_l2
from sgd_b200.phantom import ellipse_phantom

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

# (kind, np, nu, nx, ny, dx, dy, du, lsd, lso): the golden-vector cases and a
# larger one
GEN_CASES = {
    "b1_small": ("b1", 8, 40, 24, 24, 2.0, 2.0, 2.0, 1085.6, 595.0),
    "b0_small": ("b0", 8, 40, 24, 24, 2.0, 2.0, 2.0, 1085.6, 595.0),
    "b1_rect": ("b1", 6, 32, 20, 14, 1.5, 2.5, 1.7, 900.0, 500.0),
    "b0_rect": ("b0", 6, 32, 20, 14, 1.5, 2.5, 1.7, 900.0, 500.0),
    "b1_mid": ("b1", 90, 184, 128, 128, 1.0, 1.0, 1.0, 1085.6, 595.0),
}


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")


def _coo(rows, cols, vals, shape):
    return scipy.sparse.csr_matrix((vals, (np.asarray(rows, np.int64), np.asarray(cols, np.int64))), shape=shape)


def _compare(A, B):
    """(relative Frobenius distance, relative nnz difference)."""
    d = scipy.sparse.linalg.norm(A - B) / scipy.sparse.linalg.norm(B)
    return d, abs(A.nnz - B.nnz) / B.nnz


@pytest.mark.parametrize("kind,case", [("b1", "small"), ("b1", "rect"), ("b1", "snap"), ("SF", "small"),
                                       ("SF", "snap"), ("b0", "small"), ("b0", "rect")])
def test_layer_matrix_reproduces_projector(kind, case):
    from sgd_b200 import operators as ops
    cls = {"b1": ops.A_B1_operator, "SF": ops.A_SF_operator, "b0": ops.A_B0_operator}[kind]
    nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case(case)
    A = cls(nx, ny, len(ang), nu, dx, dy, du, lsd, lso, ang)
    M = A.matrix()
    assert M.shape == A.shape and M.nnz > 0 and M.has_sorted_indices
    x = ellipse_phantom(nx, ny, dx, dy, seed=2).ravel()
    assert rel_l2(M @ x, A.matvec(x)) < 1e-6
    y = np.random.default_rng(3).random(A.shape[0])
    assert rel_l2(M.T @ y, A.rmatvec(y)) < 1e-6


@pytest.mark.parametrize("mode,case", [("h0c", "small"), ("hl", "small"), ("h0", "small")])
def test_hex_layer_matrix_reproduces_forward(mode, case):
    from sgd_b200 import operators as ops
    nl, nc, nu, dt, du, lsd, lso, ang = hex_case(case)
    if mode == "hl":
        A = ops.A_Hl_operator(nl, nc, len(ang), nu, dt, du, lsd, lso, ang)
    else:
        A = ops.A_H0_operator(nl, nc, len(ang), nu, dt, du, lsd, lso, ang, exact_bounds=(mode == "h0c"))
    M = A.matrix()
    x = np.random.default_rng(4).random(A.shape[1])
    assert rel_l2(M @ x, A.matvec(x)) < 1e-6
    if mode != "h0":  # the reference H0 backward is not the transpose of its forward
        y = np.random.default_rng(5).random(A.shape[0])
        assert rel_l2(M.T @ y, A.rmatvec(y)) < 1e-6


@pytest.mark.parametrize("name", ["b1_small", "b0_small", "b1_rect", "b0_rect"])
def test_generator_matches_reference_library(name):
    import reflib
    from sgd_b200.operators import matrix_generation
    if not reflib.available():
        pytest.fail("reference library oracle/_ref/libnetwork.so not built (make -C oracle ref)")
    kind, npv, nu, nx, ny, dx, dy, du, lsd, lso = GEN_CASES[name]
    shape = (npv * nu, nx * ny)
    n_ref, t_ref = reflib.matrix_generation(kind, npv, nu, nx, ny, dx, dy, du, lsd, lso, 400000)
    n, t = matrix_generation(kind, nx, ny, npv, nu, dx, dy, du, lsd, lso)
    R = _coo(t_ref[:n_ref, 0], t_ref[:n_ref, 1], t_ref[:n_ref, 2], shape)
    M = _coo(t[:n, 0], t[:n, 1], t[:n, 2], shape)
    d, dn = _compare(M, R)
    # both FP32: entries at the support edges (tiny, rounding-dominated) may
    # exist in one and not the other; the values agree to the reference's own
    # FP32 rounding
    assert d < 1e-5 and dn < 1e-2
    x = np.random.default_rng(0).random(shape[1])
    assert rel_l2(M @ x, R @ x) < 1e-5
    # row-major order, columns ascending within rows, as the reference writes them
    key = t[:n, 0] * shape[1] + t[:n, 1]
    assert np.all(np.diff(key) > 0)


@pytest.mark.parametrize("name", ["b1_small", "b0_rect", "b1_mid"])
def test_generator_matches_cpu_replica(oracle_mod, name):
    from sgd_b200.operators import generate_matrix
    kind, npv, nu, nx, ny, dx, dy, du, lsd, lso = GEN_CASES[name]
    shape = (npv * nu, nx * ny)
    r, c, v = oracle_mod.matrix_generation(kind, npv, nu, nx, ny, dx, dy, du, lsd, lso, precision=0)
    M, R = generate_matrix(kind, nx, ny, npv, nu, dx, dy, du, lsd, lso), _coo(r, c, v, shape)
    d, dn = _compare(M, R)
    # FP32 against FP64: the generator's shifted windows reach the profile's
    # tails, where G(x2) - G(x1) cancels in FP32 (the reference's own FP32
    # values sit at the same distance)
    assert d < 5e-5 and dn < 1e-2
    x = np.random.default_rng(0).random(shape[1])
    assert rel_l2(M @ x, R @ x) < 1e-5


def test_generator_buffer_too_small_reports_error():
    from sgd_b200 import _lib
    from sgd_b200.operators import matrix_generation
    with pytest.raises(_lib.ProjectorError, match="holds"):
        matrix_generation("b1", 24, 24, 8, 40, 2.0, 2.0, 2.0, 1085.6, 595.0, buffer_size=100)


def test_b1_generator_window_differs_from_projector():
    """bilinear_matrix_generation integrates each footprint over a window
    shifted from the bin (layers/A_B1.cu:411-415): its matrix times dx*dy is
    not the forward projector, unlike pixel_matrix_generation's."""
    from sgd_b200 import operators as ops
    npv, nu, nx, ny, d, du, lsd, lso = 16, 48, 32, 32, 2.0, 2.0, 1085.6, 595.0
    ang = 2 * np.pi * np.arange(npv) / npv
    x = ellipse_phantom(nx, ny, d, d, seed=6).ravel()
    for kind, cls, lo, hi in (("b0", ops.A_B0_operator, 0.0, 1e-4), ("b1", ops.A_B1_operator, 1e-2, 1.0)):
        M = ops.generate_matrix(kind, nx, ny, npv, nu, d, d, du, lsd, lso)
        A = cls(nx, ny, npv, nu, d, d, du, lsd, lso, ang)
        assert lo <= rel_l2(M @ x * d * d, A.matvec(x)) < hi


def test_matrix_operators_match_generated_matrix(tmp_path):
    from sgd_b200 import operators as ops
    nx, ny, npv, nu, d, du, lsd, lso = 24, 24, 8, 40, 2.0, 2.0, 1085.6, 595.0
    A = ops.A_B0_operator_matrix(nx, ny, npv, nu, d, d, du, lsd, lso, directory=str(tmp_path))
    M = ops.generate_matrix("b0", nx, ny, npv, nu, d, d, du, lsd, lso)
    scipy.sparse.save_npz(tmp_path / f"A_B1_sparse_{nx}_{ny}_{npv}_{nu}.npz", 2 * M)
    B = ops.A_B1_operator_matrix(nx, ny, npv, nu, d, d, du, lsd, lso, directory=str(tmp_path))
    x = np.random.default_rng(7).random(nx * ny)
    assert rel_l2(A.matvec(x), M @ x) < 1e-15
    assert rel_l2(B.matvec(x), 2 * (M @ x)) < 1e-15
    y = np.random.default_rng(8).random(npv * nu)
    assert rel_l2(A.rmatvec(y), M.T @ y) < 1e-15
