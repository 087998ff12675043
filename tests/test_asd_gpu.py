"""ASD-POCS on the GPU (plain, and with the CNN warm start), and the phantom
sinogram simulator."""
import numpy as np
import pytest

from geometry_cases import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")


def test_simulator_matches_analytic_chords(oracle_mod):
    """Noise-free simulated sinogram = bin-averaged closed-form ellipse chords
    (numpy FP64) on the reference's geometry."""
    from sgd_b200.asd import Geometry, simulate
    from sgd_b200.phantom import ellipse_chords
    geo = Geometry(64, 12)
    _, sino, ell = simulate(geo, [5, 6], i0=0.0, sub=4)
    g = oracle_mod.geometry(geo.n, geo.n, 1, geo.nu, 1, geo.d, geo.d, 1, geo.du, 1, geo.lsd, geo.lso, geo.angles)
    for k in range(2):
        ref = np.zeros((geo.views, geo.nu))
        for p in range(geo.views):
            src, dtv, puv = g["src"][p], g["dtv"][p], g["puv"][p]
            for s in range(4):
                t = np.arange(geo.nu) - 0.5 * geo.nu + (s + 0.5) / 4
                q = dtv[None, :2] + t[:, None] * puv[None, :2]
                ref[p] += ellipse_chords(ell[k], src[0], src[1], q[:, 0], q[:, 1]) / 4
        assert rel_l2(sino[k].double().cpu().numpy(), ref) < 1e-6


def test_poisson_noise_level():
    from sgd_b200.asd import Geometry, simulate
    geo = Geometry(64, 12)
    _, clean, _ = simulate(geo, [1], i0=0.0)
    _, noisy, _ = simulate(geo, [1], i0=1e5, noise_seed=3)
    d = (noisy - clean).double()
    # b = 100 ln(I0/N): var(b) ~ 1e4 / (I0 e^{-L/100})
    pred = (1e4 / (1e5 * torch.exp(-clean.double() / 100))).mean().sqrt()
    assert 0.7 < float(d.std() / pred) < 1.3


def test_asd_pocs_reduces_error_and_images_are_independent():
    from sgd_b200.asd import ASDPOCS, Geometry, rmse, simulate
    geo = Geometry(64, 30)
    truth, sino, _ = simulate(geo, [0, 1, 2], i0=0.0)
    s = ASDPOCS(geo, 3, nonneg=False)  # the ellipse family has negative densities
    s.set_data(sino, hist_cap=30)
    e0 = rmse(s.images(), truth)
    s.run(30)
    torch.cuda.synchronize()
    s.status()
    e1 = rmse(s.images(), truth)
    assert torch.all(e1 < 0.6 * e0)
    h = s.history(30)
    assert np.all(h[5:, :, 0] < h[0, :, 0])  # data residual falls
    x3 = s.images().clone()
    one = ASDPOCS(geo, 1, nonneg=False)
    one.set_data(sino[1:2])
    one.run(30)
    torch.cuda.synchronize()
    assert rel_l2(one.images()[0].double().cpu().numpy(), x3[1].double().cpu().numpy()) < 1e-4


def test_learned_warm_start_beats_plain():
    """Train on plain-ASD-POCS pairs of small phantoms; the warm-started run
    reaches plain's final error in fewer than half of plain's iterations."""
    from sgd_b200.asd import ASDPOCS, Geometry, learned_run, make_pairs, plain_curve, simulate, train
    from sgd_b200.cnn import WarmStartCNN
    geo = Geometry(64, 40)
    iters, k_in = 60, 3
    xs, ts = make_pairs(geo, list(range(100, 356)), iters, k_in, count=64)
    net = WarmStartCNN(channels=(1, 16, 16, 16, 16, 1), seed=0)
    losses = train(net, xs, ts, epochs=15, batch=16, lr=2e-3)
    assert losses[-1] < 0.9 * losses[0]
    truth, sino, _ = simulate(geo, list(range(16)), noise_seed=77)
    s = ASDPOCS(geo, 16, nonneg=False)
    plain = plain_curve(s, sino, truth, iters, every=3)
    target = plain[-1][2]
    it_l, ms_l, curve = learned_run(s, net, sino, truth, k_in, target, iters)
    torch.cuda.synchronize()
    s.status()
    assert curve[-1][2] <= target
    assert k_in + it_l < iters / 2


def test_positivity_constraint():
    from sgd_b200.asd import ASDPOCS, Geometry, simulate
    geo = Geometry(64, 30)
    _, sino, _ = simulate(geo, [0, 1], i0=0.0)
    s = ASDPOCS(geo, 2, nonneg=True)
    s.set_data(sino)
    s.run(5)
    torch.cuda.synchronize()
    s.status()
    # TV descent after the projection may push a few values marginally below 0
    assert float(s.images().min()) > -0.05
