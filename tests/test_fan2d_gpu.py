"""Generic 2D fan-beam projectors (A_SF, ...) on the GPU: parity with the FP64
oracle replica and with the reference library, dot-product adjoint test."""
import numpy as np
import pytest

from geometry_cases import fan_case, rel_l2
from sgd_b200.phantom import ellipse_phantom

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL_PHANTOM = 1e-5
TOL_ADJOINT = 1e-6
# Against the FP64 replica.  B0 reproduces the reference's FP32 arithmetic,
# including its FP32 stepping of the bin centre (layers/A_B0.cu:202), so it
# sits from the FP64 replica where the reference itself sits (up to ~2e-5 on
# these cases); its parity bar is the reference library, at TOL_PHANTOM.
TOL_ORACLE = {"SF": 1e-5, "b0": 5e-5}

KINDS = {
    # kind: (operator class name, oracle prefix, reference-library prefix)
    "SF": ("A_SF_operator", "sf", "SF"),
    "b0": ("A_B0_operator", "b0", "b0"),
}


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")


def make_op(kind, case):
    import sgd_b200.operators as ops
    nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case(case)
    cls = getattr(ops, KINDS[kind][0])
    return cls(nx, ny, len(ang), nu, dx, dy, du, lsd, lso, ang), (nx, ny, nu, dx, dy, du, lsd, lso, ang)


@pytest.mark.parametrize("kind", list(KINDS))
@pytest.mark.parametrize("case", ["tiny", "small", "rect", "snap", "wide", "fan512"])
def test_matches_fp64_oracle(oracle_mod, kind, case):
    A, g = make_op(kind, case)
    nx, ny, nu, dx, dy, du, lsd, lso, ang = g
    fwd = getattr(oracle_mod, KINDS[kind][1] + "_forward")
    bwd = getattr(oracle_mod, KINDS[kind][1] + "_backward")
    x = ellipse_phantom(nx, ny, dx, dy, seed=0).ravel()
    b_ref, _ = fwd(x, *g)
    assert rel_l2(A.matvec(x), b_ref) < TOL_ORACLE[kind]
    assert rel_l2(A.rmatvec(b_ref), bwd(b_ref, *g)) < TOL_ORACLE[kind]


@pytest.mark.parametrize("kind", list(KINDS))
@pytest.mark.parametrize("case", ["small", "rect", "snap", "fan512"])
def test_adjoint_dot_product(kind, case):
    A, g = make_op(kind, case)
    nx, ny, nu = g[0], g[1], g[2]
    rng = np.random.default_rng(1234)
    x = rng.standard_normal(nx * ny)
    y = rng.standard_normal(len(g[-1]) * nu)
    lhs = float(np.dot(A.matvec(x), y))
    rhs = float(np.dot(x, A.rmatvec(y)))
    assert abs(lhs - rhs) / abs(lhs) < TOL_ADJOINT


@pytest.mark.parametrize("kind", list(KINDS))
@pytest.mark.parametrize("case", ["small", "snap", "fan512"])
def test_matches_reference_library(kind, case):
    import reflib
    if not reflib.available():
        pytest.fail("reference library oracle/_ref/libnetwork.so not built (make -C oracle ref)")
    A, g = make_op(kind, case)
    nx, ny, nu, dx, dy, du, lsd, lso, ang = g
    R = reflib.RefFan2D(KINDS[kind][2], nx, ny, nu, dx, dy, du, lsd, lso, ang)
    x = ellipse_phantom(nx, ny, dx, dy, seed=5).ravel()
    b_ref, cnt = R.forward(x)
    assert rel_l2(A.matvec(x), b_ref) < TOL_PHANTOM
    assert rel_l2(A.rmatvec(b_ref), R.backward(b_ref)) < TOL_PHANTOM
    assert A.conv_count == cnt or abs(A.conv_count - cnt) <= 1e-4 * cnt + 2


@pytest.mark.parametrize("kind", list(KINDS))
def test_device_api_matches_host_api(kind):
    from sgd_b200.torch_ops import FanProjector
    A, g = make_op(kind, "small")
    nx, ny, nu, dx, dy, du, lsd, lso, ang = g
    P = FanProjector(kind, nx, ny, nu, dx, dy, du, lsd, lso, ang)
    x = ellipse_phantom(nx, ny, dx, dy, seed=2)
    bd = P.forward(torch.tensor(x, dtype=torch.float32, device="cuda"))
    assert rel_l2(bd.cpu().numpy().ravel(), A.matvec(x.ravel())) < 1e-6
    yd = P.backward(bd)
    assert rel_l2(yd.cpu().numpy().ravel(), A.rmatvec(bd.cpu().numpy().ravel().astype(np.float64))) < 1e-6
