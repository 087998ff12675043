"""ASD-POCS reconstruction on the GPU, plain and with the CNN warm start.

The reference's optimizer/asd_pocs.cu is empty; this module drives the
library's ASD-POCS (``sgd_asd_*``: SART step, positivity, adaptive TV descent,
every scalar on the device, one CUDA graph per iteration) over a batch of
fan-beam B1 slices, and the seeded phantom simulator (``sgd_ellipse_sinograms``:
closed-form ellipse line integrals averaged over the bin, Poisson counts,
b = 100 ln(I0 / counts) as python/FORBILD.py:355-390).

Learned warm start: plain ASD-POCS run for ``k_in`` iterations gives the
network's input; the network (sgd_b200.cnn.WarmStartCNN) is trained to map it
to the converged plain reconstruction; reconstruction then continues with
ASD-POCS from the network's output.  Plain ASD-POCS remains the fallback.

    python -m sgd_b200.asd [--images 64] [--train 2000] [--iters 100]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import time

import numpy as np
import torch

from . import _lib
from .batch import B1Batch
from .phantom import ellipse_phantom, ellipse_phantom_average, random_ellipses

_vp = ctypes.c_void_p
LSD, LSO = 1085.6, 595.0


def _declare(L):
    if getattr(L, "_asd_declared", False):
        return
    i, f, d = ctypes.c_int, ctypes.c_float, ctypes.c_double
    L.sgd_asd_create.restype = _vp
    L.sgd_asd_create.argtypes = [_vp, f, f, f, f, f, f, i, i]
    L.sgd_asd_destroy.restype = None
    L.sgd_asd_destroy.argtypes = [_vp]
    L.sgd_asd_bind.restype = i
    L.sgd_asd_bind.argtypes = [_vp, _vp, _vp, _vp, _vp, i]
    L.sgd_asd_reset.restype = i
    L.sgd_asd_reset.argtypes = [_vp]
    L.sgd_asd_run.restype = i
    L.sgd_asd_run.argtypes = [_vp, i, _vp]
    L.sgd_asd_history.restype = i
    L.sgd_asd_history.argtypes = [_vp, _vp, i]
    L.sgd_ellipse_sinograms.restype = i
    L.sgd_ellipse_sinograms.argtypes = [_vp, i, i, i, i, d, d, d, _vp, i, d, ctypes.c_ulonglong, _vp, _vp]
    L._asd_declared = True


class Geometry:
    """A square fan-beam slice: n x n pixels over a 256 mm field, `views`
    angles over 2 pi, ceil(1.44 n) bins of 512/n mm (1 mm at n = 512, the
    headline slice): the fan covers the field's circumscribed circle
    (1.44 * 512 mm * SOD / SDD = 404 mm > 362 mm) at every n, so the data are
    not truncated."""

    def __init__(self, n=256, views=120, lsd=LSD, lso=LSO):
        self.n, self.views, self.lsd, self.lso = n, views, lsd, lso
        self.d = 256.0 / n
        self.nu = math.ceil(1.44 * n)
        self.du = 512.0 / n
        self.angles = 2 * np.pi * np.arange(views) / views

    def slice(self):
        return (self.n, self.n, self.nu, self.d, self.d, self.du, self.lsd, self.lso, self.angles)


def simulate(geo, seeds, i0=1e5, sub=8, noise_seed=0, truth="points"):
    """(truth (N, n, n) on the device, sinograms (N, views, nu) float32 on the
    device, ellipses (N, 10, 6)).  truth="points": the phantom sampled at
    pixel centres, FP32; truth="average": the phantom averaged over each
    pixel in FP64 (ellipse_phantom_average), the reconstruction experiment's
    ground truth."""
    L = _lib.lib()
    _declare(L)
    radius = 0.5 * geo.n * geo.d
    ell = np.ascontiguousarray(np.stack([random_ellipses(s, 10, radius) for s in seeds]), dtype=np.float64)
    sino = torch.empty((len(seeds), geo.views, geo.nu), dtype=torch.float32, device="cuda")
    ang = np.ascontiguousarray(geo.angles, dtype=np.float64)
    _lib.check(L.sgd_ellipse_sinograms(ell.ctypes.data, 10, len(seeds), geo.views, geo.nu, geo.du, geo.lsd, geo.lso,
                                       ang.ctypes.data, sub, float(i0), int(noise_seed), sino.data_ptr(),
                                       torch.cuda.current_stream().cuda_stream), "sgd_ellipse_sinograms")
    if truth == "average":
        t = np.stack([ellipse_phantom_average(geo.n, geo.n, geo.d, geo.d, seed=s) for s in seeds])
        return torch.tensor(t, dtype=torch.float64, device="cuda"), sino, ell
    t = np.stack([ellipse_phantom(geo.n, geo.n, geo.d, geo.d, seed=s) for s in seeds]).astype(np.float32)
    return torch.tensor(t, device="cuda"), sino, ell


class ASDPOCS:
    """ASD-POCS over `count` slices of one geometry.  The TV step per descent
    step is alpha * |dx_SART| (alpha = 0.002: twenty steps then move the
    image by 4% of the SART change, so the data step leads; Sidky and Pan's
    alpha = 0.2 applies to a full ART sweep, a much larger change than one
    SART step).  ``nonneg`` projects onto x >= 0 after each SART step (the
    classical constraint for attenuation images; the seeded ellipse family
    has negative densities, so its experiments turn it off)."""

    def __init__(self, geo, count, beta=1.0, beta_red=0.995, alpha=0.002, alpha_red=0.95, r_max=0.94, eps=0.0,
                 ng=20, nonneg=True):
        self.L = _lib.lib()
        _declare(self.L)
        self.geo, self.count = geo, count
        self.batch = B1Batch([geo.slice()] * count)
        self.h = self.L.sgd_asd_create(self.batch.handle, beta, beta_red, alpha, alpha_red, r_max, eps, ng,
                                       int(bool(nonneg)))
        if not self.h:
            raise _lib.ProjectorError(f"sgd_asd_create: {_lib.last_error()}")
        self.x = self.batch.image_arena()
        self.b = self.batch.sinogram_arena()
        self._bound = False
        self.hist_cap = 0

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.L.sgd_asd_destroy(h)
            self.h = None

    def images(self):
        return self.x.view(self.count, self.geo.n, self.geo.n)

    def set_data(self, sino, x0=None, hist_cap=0):
        """Data (count, views, nu) and the starting image (zeros by default);
        resets the adaptive state."""
        self.b.copy_(sino.reshape(-1))
        if x0 is None:
            self.x.zero_()
        else:
            self.x.copy_(x0.reshape(-1))
        torch.cuda.synchronize()
        if not self._bound or hist_cap != self.hist_cap:
            n = np.full(self.count, self.geo.n, dtype=np.int32)
            _lib.check(self.L.sgd_asd_bind(self.h, self.x.data_ptr(), self.b.data_ptr(), n.ctypes.data, n.ctypes.data,
                                           hist_cap), "sgd_asd_bind")
            self._bound = True
            self.hist_cap = hist_cap
        else:
            _lib.check(self.L.sgd_asd_reset(self.h), "sgd_asd_reset")

    def run(self, iters):
        _lib.check(self.L.sgd_asd_run(self.h, iters, torch.cuda.current_stream().cuda_stream), "sgd_asd_run")

    def history(self, iters):
        """(iters, count, 3): |Ax - b| entering each SART step, |dx_SART|, |dx_TV|."""
        out = np.zeros((iters, self.count, 3), dtype=np.float32)
        _lib.check(self.L.sgd_asd_history(self.h, out.ctypes.data, iters), "sgd_asd_history")
        return out

    def status(self):
        self.batch.status()


def rmse(x, truth):
    """Per-image RMSE against the phantom, FP64."""
    d = (x.double() - truth.double()).reshape(x.shape[0], -1)
    return torch.sqrt((d * d).mean(dim=1))


def timed(fn):
    """GPU milliseconds of fn() by CUDA events on the current stream."""
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def plain_curve(solver, sino, truth, iters, every=5, info=None):
    """(iterations, GPU ms of the iterations alone, mean RMSE) after each block
    of `every` iterations; the RMSE evaluation is outside the timed region.
    With info a dict, info["residual"] = mean |Ax - b| entering each
    iteration's SART step."""
    solver.set_data(sino, hist_cap=iters if info is not None else 0)
    curve, ms, done = [], 0.0, 0
    while done < iters:
        k = min(every, iters - done)
        ms += timed(lambda: solver.run(k))
        done += k
        curve.append((done, ms, float(rmse(solver.images(), truth).mean())))
    if info is not None:
        info["residual"] = [float(r) for r in solver.history(iters)[:, :, 0].mean(axis=1)]
    return curve


def plain_converged(solver, sino, truth, max_iters, every=5, window=10, tol=1e-3):
    """Plain ASD-POCS until its mean RMSE has changed by less than `tol`
    (relative) over the last `window` iterations, checked every `every`
    iterations (window a multiple of every), or `max_iters`: (iterations, GPU
    ms of the iterations alone, mean RMSE, curve).  The rule fixes "plain's
    final RMSE" by the method's own convergence instead of an arbitrary
    iteration count."""
    solver.set_data(sino)
    curve, ms, done = [(0, 0.0, float(rmse(solver.images(), truth).mean()))], 0.0, 0
    back = window // every
    while done < max_iters:
        ms += timed(lambda: solver.run(every))
        done += every
        curve.append((done, ms, float(rmse(solver.images(), truth).mean())))
        if len(curve) > back and abs(curve[-1][2] - curve[-1 - back][2]) < tol * curve[-1][2]:
            break
    return done, ms, curve[-1][2], curve


def make_pairs(geo, seeds, iters, k_in, count=64, noise_seed=0, nonneg=False):
    """Training pairs from plain ASD-POCS for the phantoms `seeds`, `count` at
    a time: (iterate after k_in iterations, iterate after `iters`)."""
    solver = ASDPOCS(geo, count, nonneg=nonneg)
    xs, ts = [], []
    for s0 in range(0, len(seeds), count):
        chunk = list(seeds[s0:s0 + count])
        while len(chunk) < count:
            chunk.append(chunk[-1])
        _, sino, _ = simulate(geo, chunk, noise_seed=noise_seed + s0)
        solver.set_data(sino)
        solver.run(k_in)
        xs.append(solver.images().clone())
        solver.run(iters - k_in)
        ts.append(solver.images().clone())
    solver.status()
    n = len(seeds)
    return torch.cat(xs)[:n], torch.cat(ts)[:n]


def train(net, x, t, epochs=10, batch=16, lr=1e-3, seed=0, lr_final=None, checkpoint=None):
    """Mean per-sample loss per epoch.  With lr_final the step size follows a
    cosine from lr down to lr_final over the epochs.

    checkpoint: a file path.  After every epoch the network's state (weights,
    Adam moments and step), the shuffling generator's state and the losses so
    far are written there; if the file exists when train() starts, training
    resumes after its last epoch and continues exactly as the uninterrupted
    run would (same batches, same step sizes); a checkpoint of a run with
    other epochs, sample count, batch, seed or step sizes is refused.  The
    loss of an epoch is the mean over the samples it trained on."""
    gen = torch.Generator().manual_seed(seed)
    n = x.shape[0]
    losses = []
    lr0 = lr
    start = 0
    if checkpoint is not None and os.path.exists(checkpoint):
        ck = torch.load(checkpoint, map_location="cpu", weights_only=True)
        if (ck["epochs"] != epochs or ck["n"] != n or ck["batch"] != batch or ck["seed"] != seed
                or ck.get("lr") != lr0 or ck.get("lr_final") != lr_final):
            raise ValueError(f"checkpoint {checkpoint} was written by another training run")
        net.load_state_dict(ck["net"])
        gen.set_state(ck["generator"])
        losses = list(ck["losses"])
        start = ck["epoch"]
    for ep in range(start, epochs):
        if lr_final is not None and epochs > 1:
            lr = lr_final + 0.5 * (lr0 - lr_final) * (1.0 + math.cos(math.pi * ep / (epochs - 1)))
        perm = torch.randperm(n, generator=gen)
        tot = 0.0
        used = n - n % batch  # the last n % batch samples of the permutation sit out this epoch
        for k in range(0, used, batch):
            idx = perm[k:k + batch].to(x.device)
            loss = net.train_step(x[idx].unsqueeze(1), t[idx].unsqueeze(1), lr=lr)
            tot += float(loss)
        losses.append(tot / max(used, 1))
        if checkpoint is not None:
            tmp = checkpoint + ".tmp"
            torch.save({"epoch": ep + 1, "epochs": epochs, "n": n, "batch": batch, "seed": seed, "lr": lr0,
                        "lr_final": lr_final, "net": net.state_dict(), "generator": gen.get_state(),
                        "losses": losses}, tmp)
            os.replace(tmp, checkpoint)
    return losses


def learned_run(solver, net, sino, truth, k_in, target, max_iters, every=1, info=None):
    """k_in plain iterations, the network, then ASD-POCS until the mean RMSE
    reaches `target`: (iterations after the network, GPU ms, curve); the
    network's own GPU ms goes to info["net_ms"] and the mean |Ax - b|
    entering each later SART step to info["residual"] when info is a dict."""
    solver.set_data(sino)
    ms = timed(lambda: solver.run(k_in))
    x = solver.images().unsqueeze(1).clone()
    out = {}
    ms_net = timed(lambda: out.setdefault("y", net.forward(x)))
    ms += ms_net
    solver.set_data(sino, x0=out["y"], hist_cap=max_iters if info is not None else 0)
    curve = [(0, ms, float(rmse(solver.images(), truth).mean()))]
    if info is not None:
        info["net_ms"] = ms_net
    done = 0
    while done < max_iters and curve[-1][2] > target:
        ms += timed(lambda: solver.run(every))
        done += every
        curve.append((done, ms, float(rmse(solver.images(), truth).mean())))
    if info is not None and done:
        info["residual"] = [float(r) for r in solver.history(done)[:, :, 0].mean(axis=1)]
    return done, ms, curve


def experiment(n=256, views=120, images=64, train_pairs=2000, k_in=5, epochs=40, batch=16, lr=1e-3, lr_final=1e-4,
               max_iters=1000, checkpoint=None, log=None):
    """Learned warm start against plain ASD-POCS (64 fan-beam phantoms 256^2,
    120 views, Poisson I0 = 1e5 by default).  Plain runs to the convergence
    rule of plain_converged on a calibration batch: its iteration count K
    makes the training targets (plain after K iterations) of `train_pairs`
    seeded phantoms, whose inputs are plain after k_in.  On the evaluation
    batch plain runs to the same rule; its RMSE there, against the FP64
    pixel-averaged phantoms, is the target, and the learned run (k_in plain
    iterations, the network, then ASD-POCS) stops on reaching it.  GPU times
    are CUDA-event times of the iterations and the network.  Returns a dict."""
    from .cnn import WarmStartCNN
    say = log or (lambda *a: None)
    geo = Geometry(n, views)
    # calibration batch: plain's iterations to convergence
    ctruth, csino, _ = simulate(geo, list(range(5000, 5000 + images)), noise_seed=555, truth="average")
    solver = ASDPOCS(geo, images, nonneg=False)
    K, _, _, _ = plain_converged(solver, csino, ctruth, max_iters)
    say(f"calibration: plain converges after {K} iterations")
    t0 = time.perf_counter()
    xs, ts = make_pairs(geo, list(range(1000, 1000 + train_pairs)), K, k_in)
    t_pairs = time.perf_counter() - t0
    net = WarmStartCNN(seed=0)
    t0 = time.perf_counter()
    losses = train(net, xs, ts, epochs=epochs, batch=batch, lr=lr, lr_final=lr_final, checkpoint=checkpoint)
    t_train = time.perf_counter() - t0
    say(f"pairs {t_pairs:.1f} s, training {t_train:.1f} s")
    del xs, ts
    truth, sino, _ = simulate(geo, list(range(images)), noise_seed=999, truth="average")
    # one untimed pass of the network at the reconstruction's shape: a
    # deployed network is loaded and its kernels initialised once
    net.forward(torch.zeros((images, 1, n, n), device="cuda"))
    torch.cuda.synchronize()
    it_p, ms_p, target, curve_p = plain_converged(solver, sino, truth, max_iters)
    solver.set_data(sino, hist_cap=it_p)
    solver.run(it_p)
    res_p = [float(r) for r in solver.history(it_p)[:, :, 0].mean(axis=1)]
    info = {}
    it_l, ms_l, curve_l = learned_run(solver, net, sino, truth, k_in, target, max_iters, info=info)
    solver.status()
    return {
        "workload": f"{images} fan-beam phantoms {n}^2 at {geo.d} mm, {views} views, {geo.nu} bins at {geo.du} mm, "
                    f"SOD {LSO} mm, SDD {LSD} mm, Poisson I0=1e5; plain ASD-POCS to convergence vs the CNN warm "
                    f"start after {k_in} plain iterations",
        "rmse_truth": "FP64 pixel averages of the ellipse phantoms (8 x 8 samples per pixel), FP64 RMSE",
        "convergence_rule": "mean RMSE changed by < 1e-3 (relative) over 10 iterations, checked every 5",
        "calibration_iters": K,
        "calibration_converged": K < max_iters,
        "plain": {"iters": it_p, "converged": it_p < max_iters, "gpu_ms": ms_p, "rmse": target, "curve": curve_p,
                  "data_residual": res_p},
        "learned": {"plain_iters_before_net": k_in, "iters_after_net": it_l, "gpu_ms": ms_l,
                    "net_ms": info["net_ms"], "data_residual": info.get("residual", []), "rmse": curve_l[-1][2],
                    "curve": curve_l, "reached": curve_l[-1][2] <= target},
        "time_ratio": ms_l / ms_p,
        "training": {"pairs": train_pairs, "target_iters": K, "epochs": epochs, "loss": losses, "pairs_s": t_pairs,
                     "train_s": t_train},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--views", type=int, default=120)
    ap.add_argument("--images", type=int, default=64)
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--k-in", type=int, default=5)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--lr-final", type=float, default=1e-4)
    ap.add_argument("--max-iters", type=int, default=400)
    ap.add_argument("--checkpoint", default=None,
                    help="file for per-epoch training checkpoints; an existing one is resumed")
    args = ap.parse_args()
    line = experiment(args.n, args.views, args.images, args.train, args.k_in, args.epochs, args.batch, args.lr,
                      args.lr_final, args.max_iters, args.checkpoint, log=lambda m: print(m, flush=True))
    print(json.dumps(line))


if __name__ == "__main__":
    main()
