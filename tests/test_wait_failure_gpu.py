"""The back projectors' bounded-wait failure path, taken on purpose.

Every back-projection kernel stages its view chunks into shared memory with
bulk asynchronous copies and waits for them on an mbarrier a bounded number of
polls.  Setting that bound to 0 (sgd_*_set_wait_limit) makes every first wait
give up at once: the kernel must still wait, with the full bound, for the
copies it issued, leave its tiles unwritten, and raise the device flag that
the status call reports as -1 with a message; the context stays usable and
the next call with the default bound gives the same bits as before.  Nothing
here faults or hangs a GPU: the copies complete, only the wait is cut short.
"""
import numpy as np
import pytest

from geometry_cases import cone_case, fan_case
from sgd_b200 import _lib

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

DEFAULT_POLLS = 1 << 22
SENTINEL = 12345.0


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")


def _sino(P, seed=3):
    g = torch.Generator(device="cuda").manual_seed(seed)
    return torch.rand(P.sino_shape, device="cuda", generator=g)


@pytest.mark.parametrize("kind", ["b1", "SF", "b1ref"])
def test_back_projection_wait_failure_is_reported_and_recoverable(kind):
    from sgd_b200.torch_ops import FanProjector
    L = _lib.lib()
    nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case("small")
    P = FanProjector(kind, nx, ny, nu, dx, dy, du, lsd, lso, ang)
    set_limit = L.sgd_b1_set_wait_limit if kind == "b1" else L.sgd_proj2d_set_wait_limit
    status = L.sgd_b1_status if kind == "b1" else L.sgd_proj2d_status
    y = _sino(P)
    good = P.backward(y).clone()
    assert status(P.handle) == 0
    out = torch.full(P.image_shape, SENTINEL, device="cuda")
    try:
        assert set_limit(P.handle, 0) == 0
        P.backward(y, out=out)
        assert status(P.handle) == -1
        assert "wait" in _lib.last_error()
    finally:
        assert set_limit(P.handle, DEFAULT_POLLS) == 0
    # every tile left unwritten
    assert torch.all(out == SENTINEL)
    assert status(P.handle) == 0  # the flag was cleared by the read
    again = P.backward(y)
    assert status(P.handle) == 0
    assert torch.equal(again, good)


def test_batch_back_projection_wait_failure_is_reported_and_recoverable():
    from sgd_b200.batch import B1Batch
    L = _lib.lib()
    # (nx, ny, nu, dx, dy, du, lsd, lso, angles) per slice
    B = B1Batch([(64, 64, 96, 1.0, 1.0, 1.0, 1085.6, 595.0, 2 * np.pi * np.arange(90) / 90),
                 (48, 48, 72, 1.0, 1.0, 1.0, 1085.6, 595.0, 2 * np.pi * np.arange(60) / 60)])
    g = torch.Generator(device="cuda").manual_seed(5)
    sino = torch.rand(B.sinogram_arena().shape, device="cuda", generator=g)
    good = B.image_arena()
    B.backward(sino, good)
    torch.cuda.synchronize()
    B.status()
    out = torch.full(good.shape, SENTINEL, device="cuda")
    try:
        assert L.sgd_b1_batch_set_wait_limit(B.handle, 0) == 0
        B.backward(sino, out)
        torch.cuda.synchronize()
        with pytest.raises(_lib.ProjectorError, match="bounded wait"):
            B.status()
    finally:
        assert L.sgd_b1_batch_set_wait_limit(B.handle, DEFAULT_POLLS) == 0
    assert torch.all(out == SENTINEL)
    again = B.image_arena()
    B.backward(sino, again)
    torch.cuda.synchronize()
    B.status()
    assert torch.equal(again, good)


@pytest.mark.parametrize("kind", ["b1_3d", "sf3d"])
def test_cone_back_projection_wait_failure_is_reported_and_recoverable(kind):
    """The cone-beam back projectors (exact-transpose pairs): a CTA that gives
    up on its staged view leaves its voxels unwritten and raises the flag."""
    from sgd_b200.torch_ops import ConeProjector
    L = _lib.lib()
    nx, ny, nz, nu, nv, dx, dy, dz, du, dv, lsd, lso, ang = cone_case("small")
    P = ConeProjector(kind, nx, ny, nz, nu, nv, dx, dy, dz, du, dv, lsd, lso, ang)
    set_limit = getattr(L, f"sgd_{kind}_set_wait_limit")
    status = getattr(L, f"sgd_{kind}_status")
    y = _sino(P)
    good = P.backward(y).clone()
    assert status(P.handle) == 0
    out = torch.full(P.image_shape, SENTINEL, device="cuda")
    try:
        assert set_limit(P.handle, 0) == 0
        P.backward(y, out=out)
        assert status(P.handle) == -1
        assert "wait" in _lib.last_error()
    finally:
        assert set_limit(P.handle, DEFAULT_POLLS) == 0
    assert torch.all(out == SENTINEL)
    assert status(P.handle) == 0
    again = P.backward(y)
    assert status(P.handle) == 0
    assert torch.equal(again, good)
