"""B0 in parallel-beam geometry (the 128^2, 180-view, 185-bin workload and
smaller cases) against the exact FP64 oracle, adjoint, and the long-source fan
surrogate."""
import numpy as np
import pytest

from geometry_cases import rel_l2
from sgd_b200.phantom import ellipse_phantom

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")


CASES = {
    "par128": (128, 128, 185, 1.0, 1.0, 1.0, np.pi * np.arange(180) / 180),
    "rect": (40, 27, 61, 1.3, 0.8, 0.9, np.array([0.0, 0.2, np.pi / 4, 1.9, 3 * np.pi / 4, 2.8])),
}


def make(case):
    from sgd_b200.operators import A_B0_parallel_operator
    nx, ny, nu, dx, dy, du, ang = CASES[case]
    return A_B0_parallel_operator(nx, ny, len(ang), nu, dx, dy, du, ang), (nx, ny, nu, dx, dy, du, ang)


@pytest.mark.parametrize("case", ["par128", "rect"])
def test_matches_exact_fp64_oracle(oracle_mod, case):
    """For parallel rays the 3-direction box spline is the exact bin-averaged
    line integral of the pixel indicator, so the only error is FP32."""
    A, (nx, ny, nu, dx, dy, du, ang) = make(case)
    if case == "par128":
        ang = ang[::15]  # 12 of the 180 views keep the dense oracle small
        from sgd_b200.operators import A_B0_parallel_operator
        A = A_B0_parallel_operator(nx, ny, len(ang), nu, dx, dy, du, ang)
    M = oracle_mod.exact_parallel_matrix("b0", nx, ny, nu, dx, dy, du, ang)
    x = ellipse_phantom(nx, ny, dx, dy, seed=4).ravel()
    assert rel_l2(A.matvec(x), M @ x) < 1e-5
    y = np.random.default_rng(2).random(A.shape[0])
    assert rel_l2(A.rmatvec(y), M.T @ y) < 1e-5


@pytest.mark.parametrize("case", ["par128", "rect"])
def test_adjoint_dot_product(case):
    A, _ = make(case)
    rng = np.random.default_rng(1234)
    x = rng.standard_normal(A.shape[1])
    y = rng.standard_normal(A.shape[0])
    lhs, rhs = float(np.dot(A.matvec(x), y)), float(np.dot(x, A.rmatvec(y)))
    assert abs(lhs - rhs) / abs(lhs) < 1e-6


def test_long_source_fan_surrogate_approaches_parallel():
    """The reference has only fan geometry: its B0 with the source 10^4 pixels
    away and the detector at the isocentre differs from the parallel layer by
    the residual ray divergence only."""
    from sgd_b200.operators import A_B0_operator
    A, (nx, ny, nu, dx, dy, du, ang) = make("par128")
    lso = 1e4 * dx
    F = A_B0_operator(nx, ny, len(ang), nu, dx, dy, du, lso + 1e-3, lso, ang)
    x = ellipse_phantom(nx, ny, dx, dy, seed=5).ravel()
    assert rel_l2(F.matvec(x), A.matvec(x)) < 2e-2


def test_matrix_and_device_entry():
    A, (nx, ny, nu, dx, dy, du, ang) = make("rect")
    M = A.matrix()
    x = ellipse_phantom(nx, ny, dx, dy, seed=6).ravel()
    assert rel_l2(M @ x, A.matvec(x)) < 1e-6
