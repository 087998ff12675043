"""The B1 reference-rounding mode (sgd_b1ref_*, A_B1_operator(...,
reference_rounding=True)) on the GPU: parity with the reference layer built
from its own sources (layers/A_B1.cu) on phantom and Gaussian inputs, with and
without per-view offsets; the dot-product adjoint test; its distance from the
FP64 replica (the reference's own FP32 rounding, of the order of 1e-5);
device and host entry points; determinism."""
import numpy as np
import pytest

from geometry_cases import fan_case, rel_l2
from sgd_b200.phantom import ellipse_phantom

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL_PARITY = 1e-5      # rel-L2 to the reference library, every input
TOL_ADJOINT = 1e-6     # |<Ax,y> - <x,A^T y>| / |<Ax,y>|, FP64 dot products
TOL_REPLICA = 5e-5     # to the FP64 replica: the reference's own FP32 rounding sits ~1e-5 - 3e-5 away


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")


def ops(case, **kw):
    from sgd_b200.operators import A_B1_operator
    nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case(case)
    return A_B1_operator(nx, ny, len(ang), nu, dx, dy, du, lsd, lso, ang, reference_rounding=True, **kw)


def ref(case, **kw):
    import reflib
    if not reflib.available():
        pytest.fail("reference library oracle/_ref/libnetwork.so not built (make -C oracle ref)")
    nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case(case)
    return reflib.RefFan2D("b1", nx, ny, nu, dx, dy, du, lsd, lso, ang, **kw)


@pytest.mark.parametrize("case", ["tiny", "small", "snap", "wide", "fan512"])
def test_b1ref_matches_reference_library(case):
    nx, ny, nu, dx, dy, *_ = fan_case(case)
    A, R = ops(case), ref(case)
    x = ellipse_phantom(nx, ny, dx, dy, seed=7).ravel()
    b_ref, cnt = R.forward(x)
    assert rel_l2(A.matvec(x), b_ref) < TOL_PARITY
    assert rel_l2(A.rmatvec(b_ref), R.backward(b_ref)) < TOL_PARITY
    assert A.conv_count == cnt


@pytest.mark.parametrize("case", ["small", "fan512"])
def test_b1ref_gaussian_matches_reference_library(case):
    A, R = ops(case), ref(case)
    rng = np.random.default_rng(1234)
    x = rng.standard_normal(A.shape[1])
    y = rng.standard_normal(A.shape[0])
    assert rel_l2(A.matvec(x), R.forward(x)[0]) < TOL_PARITY
    assert rel_l2(A.rmatvec(y), R.backward(y)) < TOL_PARITY


def test_b1ref_offsets_match_reference_library():
    rng = np.random.default_rng(0)
    nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case("small")
    dz, drho = rng.uniform(-3.0, 3.0, len(ang)), rng.uniform(-8.0, 8.0, len(ang))
    A, R = ops("small", dz=dz, drho=drho), ref("small", dz=dz, drho=drho)
    x = ellipse_phantom(nx, ny, dx, dy, seed=8).ravel()
    b_ref, _ = R.forward(x)
    assert rel_l2(A.matvec(x), b_ref) < TOL_PARITY
    assert rel_l2(A.rmatvec(b_ref), R.backward(b_ref)) < TOL_PARITY


@pytest.mark.parametrize("case", ["small", "rect", "snap", "wide", "fan512"])
def test_b1ref_adjoint_dot_product(case):
    A = ops(case)
    rng = np.random.default_rng(1234)
    x = rng.standard_normal(A.shape[1])
    y = rng.standard_normal(A.shape[0])
    lhs = float(np.dot(A.matvec(x), y))
    rhs = float(np.dot(x, A.rmatvec(y)))
    assert abs(lhs - rhs) / abs(lhs) < TOL_ADJOINT


@pytest.mark.parametrize("case", ["small", "rect", "fan512"])
def test_b1ref_near_fp64_replica(oracle_mod, case):
    nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case(case)
    A = ops(case)
    x = ellipse_phantom(nx, ny, dx, dy, seed=9).ravel()
    b64, cnt = oracle_mod.b1_forward(x, nx, ny, nu, dx, dy, du, lsd, lso, ang)
    assert rel_l2(A.matvec(x), b64) < TOL_REPLICA
    assert rel_l2(A.rmatvec(b64), oracle_mod.b1_backward(b64, nx, ny, nu, dx, dy, du, lsd, lso, ang)) < TOL_REPLICA
    assert abs(A.conv_count - cnt) <= 1e-4 * cnt + 2


def test_b1ref_device_matches_host_and_is_deterministic():
    from sgd_b200.torch_ops import FanProjector
    nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case("small")
    A = ops("small")
    P = FanProjector("b1ref", nx, ny, nu, dx, dy, du, lsd, lso, ang)
    x = ellipse_phantom(nx, ny, dx, dy, seed=2)
    xd = torch.tensor(x, dtype=torch.float32, device="cuda")
    bd = P.forward(xd)
    assert np.array_equal(bd.cpu().numpy().ravel(), A.matvec(x.ravel()).astype(np.float32))
    assert torch.equal(P.forward(xd), bd)
    yd = P.backward(bd)
    assert torch.equal(P.backward(bd), yd)
    assert np.array_equal(yd.cpu().numpy().ravel(),
                          A.rmatvec(bd.cpu().numpy().ravel().astype(np.float64)).astype(np.float32))
