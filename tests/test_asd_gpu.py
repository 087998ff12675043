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
    """Train on plain-ASD-POCS pairs of small phantoms (targets: plain run to
    its convergence rule); on new phantoms the warm-started run reaches
    plain's converged RMSE (FP64 pixel-averaged truth) in at most a third of
    plain's GPU time."""
    from sgd_b200.asd import ASDPOCS, Geometry, learned_run, make_pairs, plain_converged, simulate, train
    from sgd_b200.cnn import WarmStartCNN
    geo = Geometry(64, 40)
    k_in = 3
    s = ASDPOCS(geo, 16, nonneg=False)
    ctruth, csino, _ = simulate(geo, list(range(500, 516)), noise_seed=55, truth="average")
    K, _, _, _ = plain_converged(s, csino, ctruth, 300)
    xs, ts = make_pairs(geo, list(range(100, 356)), K, k_in, count=64)
    net = WarmStartCNN(channels=(1, 16, 16, 16, 16, 1), seed=0)
    losses = train(net, xs, ts, epochs=15, batch=16, lr=2e-3)
    assert losses[-1] < 0.9 * losses[0]
    truth, sino, _ = simulate(geo, list(range(16)), noise_seed=77, truth="average")
    net.forward(torch.zeros((16, 1, 64, 64), device="cuda"))  # kernels initialised once, as deployed
    it_p, ms_p, target, _ = plain_converged(s, sino, truth, 300)
    it_l, ms_l, curve = learned_run(s, net, sino, truth, k_in, target, 300)
    torch.cuda.synchronize()
    s.status()
    assert curve[-1][2] <= target
    assert ms_l <= ms_p / 3, (it_p, ms_p, k_in, it_l, ms_l)


def _tv_grad(x):
    """Gradient of the isotropic TV, FP64, as tv_grad_kernel forms it (Sidky
    and Pan 2008 eq. 11, eps = 1e-8, replicated edges; x[i, j])."""
    P = np.pad(x, 1, mode="edge")
    c = P[1:-1, 1:-1]
    eps = 1e-8
    a1, a2 = c - P[:-2, 1:-1], c - P[1:-1, :-2]
    g = (a1 + a2) / np.sqrt(eps + a1 * a1 + a2 * a2)
    xi = P[2:, 1:-1]
    b1, b2 = xi - c, xi - P[2:, :-2]
    g -= b1 / np.sqrt(eps + b1 * b1 + b2 * b2)
    xj = P[1:-1, 2:]
    c1, c2 = xj - c, xj - P[:-2, 2:]
    g -= c1 / np.sqrt(eps + c1 * c1 + c2 * c2)
    return g


def _asd_reference(A, b, x, iters, beta=1.0, beta_red=0.995, alpha=0.002, alpha_red=0.95, r_max=0.94, eps=0.0,
                   ng=20):
    """ASD-POCS iterations in NumPy FP64 on the system matrix A, the steps of
    sgd_b200/csrc/asd_pocs.cu: SART with R = A 1, C = A^T 1; ng normalised TV
    descent steps of length dtvg (0 in the first iteration, alpha |dx_SART|
    after it); dtvg shrinks by alpha_red when the TV change exceeds r_max
    times the SART change; beta shrinks by beta_red.  Returns x and the
    (|Ax - b|, |dx_SART|, |dx_TV|) of each iteration."""
    n = int(round(np.sqrt(A.shape[1])))
    R = A @ np.ones(A.shape[1])
    C = A.T @ np.ones(A.shape[0])
    dtvg, hist = 0.0, []
    for it in range(iters):
        res = b - A @ x
        dd = np.linalg.norm(res)
        r = np.where(R > 1e-6, res / np.where(R > 1e-6, R, 1.0), 0.0)
        g = A.T @ r
        xp = x
        x = x + np.where(C > 1e-6, beta * g / np.where(C > 1e-6, C, 1.0), 0.0)
        dp = np.linalg.norm(x - xp)
        xres = x.copy()
        for _ in range(ng):
            gt = _tv_grad(x.reshape(n, n)).ravel()
            nrm = np.linalg.norm(gt)
            if nrm > 0:
                x = x - dtvg * gt / nrm
        dg = np.linalg.norm(x - xres)
        if it == 0:
            dtvg = alpha * dp
        if dg > r_max * dp and dd > eps:
            dtvg *= alpha_red
        beta *= beta_red
        hist.append((dd, dp, dg))
    return x, np.array(hist)


def test_asd_pocs_matches_fp64_restatement(oracle_mod):
    """The GPU solver on a 32^2 fan-beam slice against the same iterations in
    NumPy FP64 on the oracle's B1 system matrix (the FP64 replica of
    layers/A_B1.cu, which the GPU projector matches to ~5e-7).

    Two iterations (one TV descent) agree to 1e-4.  Later iterations drift
    apart by the TV gradient's own conditioning: with eps = 1e-8 its terms
    a / sqrt(eps + a^2) turn an FP32 rounding of x (~6e-8 at |x| ~ 1) into a
    relative change of ~ulp / sqrt(eps) ~ 6e-4.  The same restatement with
    only its TV gradient rounded to FP32 differs from the FP64 one by 2.5e-4
    after three iterations and 6.3e-4 after four, so four iterations are held
    to 2e-3 (and the TV step lengths, which the same rounding moves by 1e-3,
    to 5e-3)."""
    from sgd_b200.asd import ASDPOCS, Geometry, simulate
    geo = Geometry(32, 24)
    n, _, nu, dx, dy, du, lsd, lso, ang = geo.slice()
    truth, sino, _ = simulate(geo, [5], i0=0.0)
    A = oracle_mod.b1_matrix(n, n, nu, dx, dy, du, lsd, lso, ang, np.arange(len(ang)))
    b = sino[0].double().cpu().numpy().ravel()
    # (iterations, image tolerance, tolerance of the TV step lengths)
    for iters, tol, tol_tv in ((2, 1e-4, 1e-3), (4, 2e-3, 5e-3)):
        s = ASDPOCS(geo, 1, nonneg=False)
        s.set_data(sino, hist_cap=iters)
        s.run(iters)
        torch.cuda.synchronize()
        s.status()
        x_gpu = s.images()[0].double().cpu().numpy().ravel()
        x_ref, h_ref = _asd_reference(A, b, np.zeros(n * n), iters)
        assert rel_l2(x_gpu, x_ref) < tol, iters
        h = s.history(iters)[:, 0, :].astype(np.float64)
        assert np.allclose(h[:, 0], h_ref[:, 0], rtol=1e-4) and np.allclose(h[:, 1], h_ref[:, 1], rtol=1e-4)
        assert np.allclose(h[1:, 2], h_ref[1:, 2], rtol=tol_tv) and h[0, 2] == 0.0


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
