"""The 32-channel 3x3 convolution on the tensor cores (sgd_b200/csrc/
conv_tc.cu: tcgen05 MMAs, FP32 activations as three BF16 terms, BF16
weights, FP32 accumulation in tensor memory) against the FP64 oracle and the
FP32 direct-convolution kernel.  The products are exact in both kernels;
the tensor cores' FP32 accumulation rounds with fewer guard bits than an FMA
chain (1.3e-6 rel-L2 from FP64 measured against 3e-7 for the direct
kernel), so the bar here is 5e-6."""
import numpy as np
import pytest

from oracle import cnn_oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")


TOL = 5e-6


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


def _run(fn, X, W16, B, n, h, w, relu):
    from sgd_b200 import _lib
    from sgd_b200.cnn import _stream
    out = torch.full((n, 32, h, w), float("nan"), device="cuda")
    _lib.check(fn(X.data_ptr(), W16.data_ptr(), B.data_ptr(), out.data_ptr(), n, 32, 32, h, w, relu, _stream()),
               "conv")
    torch.cuda.synchronize()
    return out


# one partial tile, exact tiles, a partial second tile, a single row and column
@pytest.mark.parametrize("n,h,w", [(2, 16, 16), (2, 9, 128), (1, 5, 200), (3, 1, 37), (1, 40, 1), (2, 33, 257)])
@pytest.mark.parametrize("relu", [0, 1])
def test_tensor_core_conv_matches_fp64_oracle_and_fp32_kernel(n, h, w, relu):
    from sgd_b200 import _lib
    from sgd_b200.cnn import _declare
    L = _lib.lib()
    _declare(L)
    rng = np.random.default_rng(n * 1000 + h * 10 + w + relu)
    x = rng.standard_normal((n, 32, h, w)).astype(np.float32)
    wt = (rng.standard_normal((32, 32, 3, 3)) * 0.2).astype(np.float32)
    b = rng.standard_normal(32).astype(np.float32)
    X = torch.tensor(x, device="cuda")
    W16 = torch.tensor(wt, device="cuda").to(torch.bfloat16)
    B = torch.tensor(b, device="cuda")
    tc = _run(L.sgd_conv3x3_forward_tc, X, W16, B, n, h, w, relu)
    _lib.check(L.sgd_conv3x3_tc_status(), "tensor-core conv status")
    fp32 = _run(L.sgd_conv3x3_forward, X, W16, B, n, h, w, relu)
    wq = W16.float().cpu().numpy().astype(np.float64)
    ref = cnn_oracle.conv3x3(x.astype(np.float64), wq, b.astype(np.float64))
    if relu:
        ref = np.maximum(ref, 0.0)
    t = tc.cpu().numpy()
    assert np.all(np.isfinite(t))
    assert rel(t, ref) < TOL
    assert rel(t, fp32.cpu().numpy()) < TOL


def test_tensor_core_conv_rejects_other_channel_counts():
    from sgd_b200 import _lib
    from sgd_b200.cnn import _declare, _stream
    L = _lib.lib()
    _declare(L)
    X = torch.zeros((1, 16, 8, 8), device="cuda")
    W16 = torch.zeros((32, 16, 3, 3), device="cuda", dtype=torch.bfloat16)
    out = torch.zeros((1, 32, 8, 8), device="cuda")
    rc = L.sgd_conv3x3_forward_tc(X.data_ptr(), W16.data_ptr(), None, out.data_ptr(), 1, 16, 32, 8, 8, 0, _stream())
    assert rc == -1
    assert "32 input and 32 output channels" in _lib.last_error()


def test_network_forward_on_tensor_cores_matches_direct_kernels():
    """The warm-start network with its 32-channel layers on the tensor cores
    gives the output of the same network on the FP32 direct kernels."""
    from sgd_b200.cnn import WarmStartCNN
    rng = np.random.default_rng(5)
    nets = [WarmStartCNN(channels=(1, 32, 32, 32, 1), seed=2, tensor_cores=tc) for tc in (True, False)]
    for w in nets[0].w32:
        w.copy_(torch.tensor((rng.standard_normal(tuple(w.shape)) * 0.1).astype(np.float32)))
    for a, b in zip(nets[1].w32, nets[0].w32):
        a.copy_(b)
    for net in nets:
        net.w16 = [w.to(torch.bfloat16) for w in net.w32]
    x = torch.tensor(rng.standard_normal((2, 1, 40, 150)).astype(np.float32), device="cuda")
    y_tc, y_fp32 = (net.forward(x) for net in nets)
    torch.cuda.synchronize()
    assert rel(y_tc.cpu().numpy(), y_fp32.cpu().numpy()) < TOL
