"""torch.autograd through every projector kind: the gradient of <A x, y> is
the hand-written back projection A^T y, the gradient through the back
projection is the forward, and each pair used for autograd passes the
dot-product adjoint test."""
import numpy as np
import pytest

from geometry_cases import cone_case, fan_case, hex_case

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")


def projector(kind):
    from sgd_b200 import torch_ops as T
    if kind in ("b1", "SF", "b0"):
        nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case("small")
        return T.FanProjector(kind, nx, ny, nu, dx, dy, du, lsd, lso, ang)
    if kind == "b0_parallel":
        return T.ParallelB0Projector(48, 40, 70, 1.0, 1.2, 1.0, np.pi * np.arange(30) / 30)
    if kind in ("h0c", "hl"):
        nl, nc, nu, dt, du, lsd, lso, ang = hex_case("small")
        return T.HexProjector(nl, nc, nu, dt, du, lsd, lso, ang, mode=kind)
    if kind in ("b1_3d", "sf3d"):
        nx, ny, nz, nu, nv, dx, dy, dz, du, dv, lsd, lso, ang = cone_case("small")
        return T.ConeProjector(kind, nx, ny, nz, nu, nv, dx, dy, dz, du, dv, lsd, lso, ang, exact=True)
    raise KeyError(kind)


KINDS = ["b1", "SF", "b0", "b0_parallel", "h0c", "hl", "b1_3d", "sf3d"]


@pytest.mark.parametrize("kind", KINDS)
def test_gradients_are_the_other_projector(kind):
    from sgd_b200.torch_ops import back_project, project
    P = projector(kind)
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn(P.image_shape, device="cuda", generator=g, requires_grad=True)
    y = torch.randn(P.sino_shape, device="cuda", generator=g)
    (project(x, P) * y).sum().backward()
    assert torch.equal(x.grad, P.backward(y.contiguous()))  # the back kernels gather: deterministic
    s = y.clone().requires_grad_(True)
    w = torch.randn(P.image_shape, device="cuda", generator=g)
    (back_project(s, P) * w).sum().backward()
    # the generic forward kernels sum with atomics: equal up to summation order
    fw = P.forward(w.contiguous()).double()
    assert float((s.grad.double() - fw).norm() / fw.norm()) < 1e-6
    # the pair is an adjoint pair (FP64 dot products) on N(0, 1) vectors of
    # seed 1234
    rng = np.random.default_rng(1234)
    x = torch.tensor(rng.standard_normal(P.image_shape), dtype=torch.float32, device="cuda")
    y = torch.tensor(rng.standard_normal(P.sino_shape), dtype=torch.float32, device="cuda")
    ax = P.forward(x).double()
    aty = P.backward(y).double()
    lhs = float((ax * y.double()).sum())
    rhs = float((x.double() * aty).sum())
    assert abs(lhs - rhs) / abs(lhs) < 1e-6


def test_batched_leading_dimension():
    from sgd_b200.torch_ops import project
    P = projector("b1")
    x = torch.randn((3,) + P.image_shape, device="cuda")
    out = project(x, P)
    assert out.shape == (3,) + P.sino_shape
    assert torch.equal(out[1], P.forward(x[1].contiguous()))
