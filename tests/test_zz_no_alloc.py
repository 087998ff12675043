"""sgd_b1_forward_noalloc: the B1 forward projection for callers that cannot
allocate device memory while they run (code under another framework's memory
pool, or a real-time loop where cudaMalloc's implicit synchronisation is not
allowed).  It keeps its scratch in a fixed 4 MiB array in the library instead
of allocating.  This file is collected last so that a run stopping at the
first failure has already run every other test."""
import ctypes

import numpy as np
import pytest

from geometry_cases import fan_case, rel_l2
from sgd_b200.phantom import ellipse_phantom

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-5  # the projector tests' parity tolerance


def _entry():
    from sgd_b200 import _lib
    return _lib.lib().sgd_b1_forward_noalloc


def test_noalloc_forward_matches_allocating_entry_point_twice():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required")
    from sgd_b200.torch_ops import FanProjector
    f = _entry()
    nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case("small")
    P = FanProjector("b1", nx, ny, nu, dx, dy, du, lsd, lso, ang)
    stream = torch.cuda.current_stream().cuda_stream
    for seed in (0, 1):  # two calls in a row: the shared scratch keeps the last call's contents
        img = torch.tensor(ellipse_phantom(nx, ny, dx, dy, seed=seed), dtype=torch.float32, device="cuda")
        ref = P.forward(img)  # the existing entry point, sgd_b1_forward_dev
        out = torch.full_like(ref, float("nan"))
        assert f(P.handle, ctypes.c_void_p(img.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                 ctypes.c_void_p(stream)) == 0
        torch.cuda.synchronize()
        o, r = out.cpu().numpy(), ref.cpu().numpy()
        assert np.all(np.isfinite(o))
        assert rel_l2(o, r) < TOL


def test_noalloc_call_allocates_nothing():
    """After the first call (which looks up the scratch array's address), a
    call changes no device allocation: the free device memory is the same
    before and after it, and the call still gives the projection."""
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required")
    from sgd_b200.torch_ops import FanProjector
    f = _entry()
    nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case("small")
    P = FanProjector("b1", nx, ny, nu, dx, dy, du, lsd, lso, ang)
    img = torch.tensor(ellipse_phantom(nx, ny, dx, dy, seed=2), dtype=torch.float32, device="cuda")
    out = torch.zeros(P.sino_shape, dtype=torch.float32, device="cuda")
    ref = P.forward(img)

    def call():
        s = torch.cuda.current_stream().cuda_stream
        return f(P.handle, ctypes.c_void_p(img.data_ptr()), ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(s))

    assert call() == 0  # first call: address lookup
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    assert call() == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert rel_l2(out.cpu().numpy(), ref.cpu().numpy()) < TOL


def test_noalloc_rejects_images_beyond_its_scratch():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required")
    from sgd_b200 import _lib
    from sgd_b200.torch_ops import FanProjector
    f = _entry()
    nx, ny = 1025, 1024  # one column over the 1024 x 1024 limit
    P = FanProjector("b1", nx, ny, 64, 0.25, 0.25, 8.0, 1085.6, 595.0, np.array([0.0, 1.0]))
    img = torch.zeros((nx, ny), dtype=torch.float32, device="cuda")
    out = torch.zeros(P.sino_shape, dtype=torch.float32, device="cuda")
    rc = f(P.handle, ctypes.c_void_p(img.data_ptr()), ctypes.c_void_p(out.data_ptr()),
           ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == -1
    assert "exceeds" in _lib.last_error()
