"""Warm-start CNN kernels (sgd_b200/csrc/cnn.cu) against the FP64 CPU oracle:
convolution forward, input and weight gradients, the whole network's
parameter gradients, and a training loop that lowers the loss."""
import numpy as np
import pytest

from oracle import cnn_oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")


def bf16_round(a):
    return torch.tensor(a, dtype=torch.float32).to(torch.bfloat16).to(torch.float32).numpy().astype(np.float64)


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


@pytest.mark.parametrize("ci,co,h,w", [(1, 32, 19, 23), (32, 32, 16, 16), (32, 32, 37, 45), (16, 32, 9, 70),
                                       (32, 1, 33, 17), (3, 5, 8, 40)])
def test_conv_forward_and_gradients(ci, co, h, w):
    from sgd_b200 import _lib
    from sgd_b200.cnn import _declare, _stream
    L = _lib.lib()
    _declare(L)
    rng = np.random.default_rng(ci * 100 + co)
    x = rng.standard_normal((2, ci, h, w)).astype(np.float32)
    wt = (rng.standard_normal((co, ci, 3, 3)) * 0.2).astype(np.float32)
    b = rng.standard_normal(co).astype(np.float32)
    wq = bf16_round(wt)  # the kernels read BF16 weights
    X = torch.tensor(x, device="cuda")
    W16 = torch.tensor(wt, device="cuda").to(torch.bfloat16)
    B = torch.tensor(b, device="cuda")
    out = torch.empty((2, co, h, w), device="cuda")
    _lib.check(L.sgd_conv3x3_forward(X.data_ptr(), W16.data_ptr(), B.data_ptr(), out.data_ptr(), 2, ci, co, h, w, 0,
                                     _stream()), "fwd")
    ref = cnn_oracle.conv3x3(x.astype(np.float64), wq, b.astype(np.float64))
    assert rel(out.cpu().numpy(), ref) < 1e-6
    g = rng.standard_normal((2, co, h, w)).astype(np.float32)
    G = torch.tensor(g, device="cuda")
    gin = torch.empty_like(X)
    scratch = torch.empty(ci * co * 9, dtype=torch.bfloat16, device="cuda")
    _lib.check(L.sgd_conv3x3_backward_data(G.data_ptr(), W16.data_ptr(), scratch.data_ptr(), gin.data_ptr(), 2, ci,
                                           co, h, w, _stream()), "bwd data")
    gw = torch.zeros((co, ci, 3, 3), device="cuda")
    gb = torch.zeros(co, device="cuda")
    _lib.check(L.sgd_conv3x3_backward_weight(X.data_ptr(), G.data_ptr(), gw.data_ptr(), gb.data_ptr(), 2, ci, co, h,
                                             w, _stream()), "bwd weight")
    rgx, rgw, rgb = cnn_oracle.conv3x3_grads(x.astype(np.float64), wq, g.astype(np.float64))
    assert rel(gin.cpu().numpy(), rgx) < 1e-6
    assert rel(gw.cpu().numpy(), rgw) < 1e-5
    assert rel(gb.cpu().numpy(), rgb) < 1e-5


def test_network_gradients_match_oracle_and_finite_differences():
    from sgd_b200.cnn import WarmStartCNN
    net = WarmStartCNN(channels=(1, 8, 8, 1), seed=3)
    rng = np.random.default_rng(0)
    for w in net.w32:  # a non-trivial last layer
        w.copy_(torch.tensor((rng.standard_normal(tuple(w.shape)) * 0.3).astype(np.float32)))
    net.w16 = [w.to(torch.bfloat16) for w in net.w32]
    for b in net.b:
        b.copy_(torch.tensor((rng.standard_normal(b.numel()) * 0.1).astype(np.float32)))
    x = rng.standard_normal((2, 1, 12, 10)).astype(np.float32)
    gy = rng.standard_normal((2, 1, 12, 10)).astype(np.float32)
    y = net.forward(torch.tensor(x, device="cuda"), keep=True)
    grads = net.backward(torch.tensor(gy, device="cuda"))
    ws = [bf16_round(w.cpu().numpy()) for w in net.w32]
    bs = [b.cpu().numpy().astype(np.float64) for b in net.b]
    yref, _ = cnn_oracle.network(x.astype(np.float64), ws, bs)
    assert rel(y.cpu().numpy(), yref) < 1e-6
    gws, gbs = cnn_oracle.network_grads(x.astype(np.float64), ws, bs, gy.astype(np.float64))
    for k in range(len(ws)):
        assert rel(grads[k].cpu().numpy(), gws[k]) < 1e-5
        assert rel(grads[len(ws) + k].cpu().numpy(), gbs[k]) < 1e-5
    # central differences of the FP64 oracle on one weight (step 1e-3)
    k, idx = 1, (2, 3, 1, 1)
    wp = [w.copy() for w in ws]
    wm = [w.copy() for w in ws]
    wp[k][idx] += 1e-3
    wm[k][idx] -= 1e-3
    fd = (np.sum(gy * cnn_oracle.network(x.astype(np.float64), wp, bs)[0]) -
          np.sum(gy * cnn_oracle.network(x.astype(np.float64), wm, bs)[0])) / 2e-3
    assert abs(fd - float(grads[k][idx])) < 1e-3 * max(1.0, abs(fd))


def test_training_lowers_the_loss():
    from sgd_b200.cnn import WarmStartCNN
    rng = np.random.default_rng(1)
    # denoising toy task: spatially smooth targets (5x5 box-filtered noise) plus white noise
    z = rng.standard_normal((16, 1, 28, 28))
    t = (sum(z[:, :, a:a + 24, b:b + 24] for a in range(5) for b in range(5)) / 5.0).astype(np.float32)
    x = t + 0.5 * rng.standard_normal(t.shape).astype(np.float32)
    net = WarmStartCNN(channels=(1, 16, 16, 1), seed=0)
    X, T = torch.tensor(x, device="cuda"), torch.tensor(t, device="cuda")
    first = float(net.train_step(X, T, lr=3e-3))
    for _ in range(150):
        last = float(net.train_step(X, T, lr=3e-3))
    assert last < 0.7 * first
