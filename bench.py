#!/usr/bin/env python
"""Throughput of the B1 bilinear fan-beam projector pair (forward + adjoint).

Workload: 512 x 512 image at 0.5 mm of a seeded random-ellipse phantom,
720 views over [0, 2 pi), 736 bins at 1.0 mm, source-isocentre 595 mm,
source-detector 1085.6 mm.  One step = one forward projection and one back
projection (A x, A^T y).  Metric: fwd+adj voxel-view updates per second,
2 * nx * ny * np per step, summed over all ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`--impl reference` times the reference's CPU path for this operator (its
sparse system matrix applied as python/operators/operators.py:31-49 does) on
a bounded sample of views, the same CSR product on every host core
(torch.sparse_csr, MKL), W warm-up and K timed steps as our arm; the
single-threaded scipy figure (the reference's own call) is reported beside
it.  Our arm's line also carries, measured after its timed region, the same
CPU path (`cpu_baseline`) and the reference's own CUDA layer built from its
sources (`reference_gpu`).
Each rank of a multi-GPU run projects its own phantom (independent replicas,
weak scaling); there is no collective on the data path.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX = NY = 512
DX = DY = 0.5
NP, NU, DU = 720, 736, 1.0
LSD, LSO = 1085.6, 595.0
ANGLES = 2 * np.pi * np.arange(NP) / NP
METRIC = "fwd+adj voxel-view updates/s (B1 fan beam)"
UNIT = "voxel-view updates/s"
CONFIG = {
    "workload": "B1 bilinear fan-beam forward + adjoint, 512x512 @0.5mm, 720 views over 2pi, 736 bins @1mm, "
                "SOD 595 mm, SDD 1085.6 mm, seeded 10-ellipse phantom",
    "nx": NX, "ny": NY, "views": NP, "bins": NU,
    "l2": "flushed between steps (256 MiB write outside the timed events)",
}
FLUSH_BYTES = 256 << 20


def max_over_ranks(x, world, device):
    """The largest of every rank's x (all ranks call it, in the same order):
    a multi-rank time is the slowest rank's."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _families():
    """name -> (description, constructor of a sgd_b200.torch_ops projector,
    voxel-views per direction, seeded input maker)."""
    HEX_ANG = 2 * np.pi * np.arange(360) / 360

    def fan(kind):
        from sgd_b200.torch_ops import FanProjector
        return FanProjector(kind, NX, NY, NU, DX, DY, DU, LSD, LSO, ANGLES)

    def par():
        from sgd_b200.torch_ops import ParallelB0Projector
        return ParallelB0Projector(128, 128, 185, 1.0, 1.0, 1.0, np.pi * np.arange(180) / 180)

    def hexp(mode, nl, nc, dt):
        from sgd_b200.torch_ops import HexProjector
        return HexProjector(nl, nc, NU, dt, DU, LSD, LSO, HEX_ANG, mode=mode)

    def cone(kind, n=256, views=360, nd=384, d=1.0, dd=1.5):
        from sgd_b200.torch_ops import ConeProjector
        ang = 2 * np.pi * np.arange(views) / views
        return ConeProjector(kind, n, n, n, nd, nd, d, d, d, dd, dd, LSD, LSO, ang)

    return {
        "sf_fan512": ("A_SF separable footprint fan beam, 512x512 @0.5mm, 720 views, 736 bins @1mm",
                  lambda: fan("SF"), NX * NY * NP),
        "b1ref_fan512": ("A_B1 in the reference layer's FP32 rounding, fan beam, 512x512 @0.5mm, 720 views, "
                         "736 bins @1mm", lambda: fan("b1ref"), NX * NY * NP),
        "b0_fan512": ("A_B0 pixel basis fan beam, 512x512 @0.5mm, 720 views, 736 bins @1mm",
                  lambda: fan("b0"), NX * NY * NP),
        "b0_parallel128": ("B0 parallel beam, 128x128 @1mm, 180 views over pi, 185 bins @1mm",
                           par, 128 * 128 * 180),
        "h0_hex2e18": ("H0 hexagonal lattice (true hexagon bounds), 550 rows x 477 sites, dt 0.62 mm, 360 views, "
                  "736 bins @1mm", lambda: hexp("h0c", 550, 477, 0.62), 550 * 477 * 360),
        "hl_hex2e18": ("Hl hexagonal lattice, 953 rows x 275 sites, dt 1.075 mm, 360 views, 736 bins @1mm",
                  lambda: hexp("hl", 953, 275, 1.075), 953 * 275 * 360),
        "b1_3d_cone256": ("A_B1_3D cone beam (exact-transpose pair), 256^3 @1mm, 360 views, 384x384 @1.5mm",
                     lambda: cone("b1_3d"), 256 ** 3 * 360),
        "sf3d_cone256": ("SF_projector cone beam (corrected pair), 256^3 @1mm, 360 views, 384x384 @1.5mm",
                    lambda: cone("sf3d"), 256 ** 3 * 360),
        "b1_3d_small": ("A_B1_3D cone beam, the 256^3 cone geometry at half resolution for profiling: 128^3 @2mm, "
                        "180 views, 192x192 @3mm", lambda: cone("b1_3d", 128, 180, 192, 2.0, 3.0), 128 ** 3 * 180),
        "sf3d_small": ("SF_projector cone beam (corrected pair), the 256^3 cone geometry at half resolution for "
                       "profiling: 128^3 @2mm, 180 views, 192x192 @3mm",
                       lambda: cone("sf3d", 128, 180, 192, 2.0, 3.0), 128 ** 3 * 180),
    }


FAMILIES = ("sf_fan512", "b1ref_fan512", "b0_fan512", "b0_parallel128", "h0_hex2e18", "hl_hex2e18", "b1_3d_cone256", "sf3d_cone256", "b1_3d_small",
            "sf3d_small")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["fan512", "batch48", "asd_c5", "cnn_conv32"] + sorted(FAMILIES),
                    default="fan512",
                    help="fan512: the headline single-slice workload; batch48: 48 uneven slices in one "
                         "graph-replayed persistent launch per direction; asd_c5: learned vs plain ASD-POCS "
                         "(several minutes: pair generation and training included); cnn_conv32: the CNN's "
                         "32-channel convolution on the tensor cores; the others: the other "
                         "projector families at their configurations (device-resident fwd+adj)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# reference arm / CPU baseline: scipy CSR SpMV on a bounded sample of views
# ---------------------------------------------------------------------------
class quiet_stdout:
    """Sends what native code writes to stdout (the reference library prints
    its launch shapes) to stderr, so that stdout carries the JSON line only."""

    def __enter__(self):
        import ctypes
        self._libc = ctypes.CDLL(None)
        sys.stdout.flush()
        self._libc.fflush(None)
        self._saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        self._libc.fflush(None)
        os.dup2(self._saved, 1)
        os.close(self._saved)
        return False


def reference_matrix_rows(n_views):
    """Rows of the B1 system matrix for `n_views` uniformly spaced views, as
    the reference's own generator builds them (bilinear_matrix_generation,
    layers/A_B1.cu:545-593, from oracle/_ref/libnetwork.so, built from its
    sources; it runs on the GPU, one dense view at a time), as scipy CSR; None
    without that library or a GPU, or when the call fails.  Its angles 2 pi p /
    n_views are the headline's views p * 720 / n_views."""
    import ctypes
    import scipy.sparse as sp
    import torch
    path = os.path.join(ROOT, "oracle", "_ref", "libnetwork.so")
    if not os.path.exists(path) or NP % n_views or not torch.cuda.is_available():
        return None
    L = ctypes.CDLL(path)
    f = L.bilinear_matrix_generation
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 5 + [ctypes.c_void_p, ctypes.c_int]
    # room for 10 entries per pixel-view (the footprint has about 3.4): the
    # generator aborts the process on a full buffer (assert)
    cap = n_views * NX * NY * 10
    buf = np.empty(3 * cap)
    with quiet_stdout():
        n = f(n_views, NU, NX, NY, DX, DY, DU, LSD, LSO, buf.ctypes.data, cap)
    if n <= 0:
        return None
    t = buf[:3 * n].reshape(n, 3)
    return sp.csr_matrix((t[:, 2], (t[:, 0].astype(np.int64), t[:, 1].astype(np.int64))),
                         shape=(n_views * NU, NX * NY))


class CpuSpmv:
    """The reference's CPU path for this operator: its sparse system matrix
    applied as python/operators/operators.py:45-49 does (A @ x, A.T @ y), on
    the rows of `n_views` evenly spaced views (a bounded sample).  The entries
    come from the reference's own generator where its library was built
    (kind "reference"), else from the oracle's FP64 replica of
    layers/A_B1.cu (kind "port").  Built once."""

    def __init__(self, n_views=12):
        import torch
        from sgd_b200.phantom import ellipse_phantom
        self.views = np.arange(0, NP, NP // n_views)[:n_views]
        self.A = reference_matrix_rows(n_views)
        self.kind = "reference"
        if self.A is None:
            from oracle import oracle
            self.A = oracle.b1_matrix(NX, NY, NU, DX, DY, DU, LSD, LSO, ANGLES, self.views)
            self.kind = "port"
        self.AT = self.A.T.tocsr()
        self.x = ellipse_phantom(NX, NY, DX, DY, seed=0).ravel()
        self.y = self.A @ self.x
        self.units = 2.0 * NX * NY * len(self.views)
        self.threads = os.cpu_count() or 1
        torch.set_num_threads(self.threads)

        def csr(M):
            return torch.sparse_csr_tensor(torch.from_numpy(M.indptr.astype(np.int64)),
                                           torch.from_numpy(M.indices.astype(np.int64)), torch.from_numpy(M.data),
                                           size=M.shape)

        self.At, self.ATt = csr(self.A), csr(self.AT)
        self.xt, self.yt = torch.from_numpy(self.x), torch.from_numpy(self.y)
        self.At @ self.xt  # first call initialises the sparse backend

    def step_threads(self):
        """Seconds of one A@x + A.T@y on every host core (torch CSR, MKL)."""
        t0 = time.perf_counter()
        self.At @ self.xt
        self.ATt @ self.yt
        return time.perf_counter() - t0

    def step_scipy(self):
        """Seconds of one A@x + A.T@y in scipy (single-threaded, the reference's own call)."""
        t0 = time.perf_counter()
        self.A @ self.x
        self.AT @ self.y
        return time.perf_counter() - t0

    def desc(self, v1, vn):
        src = ("the reference's own bilinear_matrix_generation (oracle/_ref, built from layers/A_B1.cu)"
               if self.kind == "reference" else "the FP64 replica of layers/A_B1.cu")
        return (f"CSR SpMV A@x and A.T@y (python/operators/operators.py:45-49 path), FP64, rows of {len(self.views)} "
                f"of {NP} views (nnz {self.A.nnz}), entries from {src}; "
                f"scipy 1 thread {v1:.3e}/s, torch CSR (MKL) {self.threads} threads {vn:.3e}/s")


def cpu_spmv_sample(n_views=12, reps=3):
    """Best-of-`reps` updates/s of the sampled CPU path, single-threaded and on
    every host core; the faster is the value."""
    t_all = time.perf_counter()
    S = CpuSpmv(n_views)
    best1 = min(S.step_scipy() for _ in range(reps))
    bestn = min(S.step_threads() for _ in range(reps))
    v1, vn = S.units / best1, S.units / bestn
    spent = time.perf_counter() - t_all
    if vn >= v1:
        return {"value": vn, "cores": S.threads, "single_thread": v1, "desc": S.desc(v1, vn), "spent": spent,
                "kind": S.kind}
    return {"value": v1, "cores": 1, "single_thread": v1, "desc": S.desc(v1, vn), "spent": spent, "kind": S.kind}


def run_reference(args, rank, world):
    """The reference arm: the reference's CPU path (CpuSpmv) on the host cores,
    W warm-up and exactly K timed steps, each one A@x + A.T@y of the sample."""
    if rank != 0:
        return
    S = CpuSpmv()
    for _ in range(args.warmup):
        S.step_threads()
    times = [S.step_threads() for _ in range(args.steps)]
    single = S.units / min(S.step_scipy() for _ in range(3))
    value = S.units / statistics.median(times)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": CONFIG, "parallelism": f"host threads x{S.threads}",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": S.threads, "kind": S.kind,
                         "sample": S.desc(single, value), "single_thread_value": single},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def reference_gpu_layer():
    """The reference's own B1 CUDA layer (layers/A_B1.cu built from its sources
    into oracle/_ref/libnetwork.so) on the headline geometry, on this GPU,
    outside the timed region: its kernels alone (A_B1::project /
    back_project on resident device buffers, per-view launches) and its C ABI
    end to end (b1_forward_projection + b1_backward_projection on FP64 host
    arrays).  None when the library was not built."""
    import ctypes
    lib_path = os.path.join(ROOT, "oracle", "_ref", "libnetwork.so")
    if not os.path.exists(lib_path):
        return None
    L = ctypes.CDLL(lib_path)
    dp = ctypes.POINTER(ctypes.c_double)
    L.b1_init.restype = ctypes.c_void_p
    L.b1_init.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 5 + [dp] * 3
    L.b1_forward_projection.restype = ctypes.c_int
    L.b1_forward_projection.argtypes = [dp, dp, ctypes.c_void_p]
    L.b1_backward_projection.restype = None
    L.b1_backward_projection.argtypes = [dp, dp, ctypes.c_void_p]
    L.ref_b1_kernel_ms.restype = ctypes.c_float
    L.ref_b1_kernel_ms.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    ang = np.ascontiguousarray(ANGLES, dtype=np.float64)
    from sgd_b200.phantom import ellipse_phantom
    x = np.ascontiguousarray(ellipse_phantom(NX, NY, DX, DY, seed=0).ravel(), dtype=np.float64)
    y = np.zeros(NP * NU)
    xt = np.zeros(NX * NY)
    reps = 2
    with quiet_stdout():
        h = L.b1_init(NX, NY, NP, NU, DX, DY, DU, LSD, LSO, ang.ctypes.data_as(dp), None, None)
        back = ctypes.c_float(0.0)
        fwd = L.ref_b1_kernel_ms(h, 3, ctypes.byref(back))
        L.b1_forward_projection(y.ctypes.data_as(dp), x.ctypes.data_as(dp), h)
        t0 = time.perf_counter()
        for _ in range(reps):
            L.b1_forward_projection(y.ctypes.data_as(dp), x.ctypes.data_as(dp), h)
            L.b1_backward_projection(y.ctypes.data_as(dp), xt.ctypes.data_as(dp), h)
        abi_ms = (time.perf_counter() - t0) / reps * 1e3
    units = 2.0 * NX * NY * NP
    return {"kernels_fwd_ms": fwd, "kernels_bwd_ms": back.value,
            "kernels_updates_per_s": units / ((fwd + back.value) * 1e-3),
            "c_abi_ms_per_step": abi_ms, "c_abi_updates_per_s": units / (abi_ms * 1e-3),
            "source": "oracle/_ref/libnetwork.so: the reference's layers/A_B1.cu built from its own sources "
                      "(its per-view launches and FP64 atomics), timed on this GPU outside the timed region; "
                      "kernels: CUDA events around A_B1::project / back_project (3 calls each); C ABI: "
                      "b1_forward_projection + b1_backward_projection on FP64 host arrays (2 pairs, wall clock)"}


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", uuid, f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        self.file.flush()
        self.file.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for row in self.file.read().strip().splitlines():
            parts = [p.strip() for p in row.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.file.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def load_op_counts():
    with open(os.path.join(ROOT, "sgd_b200", "op_counts.json")) as f:
        return json.load(f)


def load_traffic():
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return {}
    with open(p) as f:
        return json.load(f)


def fp32_peak(dev, stream):
    """FP32 FMA throughput (FLOP/s, FMA = 2) of this GPU now, from the library's
    probe kernel: the roofline denominator (MEASURED_PEAKS has no FP32 entry)."""
    import ctypes
    import torch
    from sgd_b200 import _lib
    L = _lib.lib()
    L.sgd_fp32_fma_rate.restype = ctypes.c_double
    L.sgd_fp32_fma_rate.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    nsm = torch.cuda.get_device_properties(dev).multi_processor_count
    scratch = torch.empty(nsm * 64, dtype=torch.float32, device=dev)
    return max(L.sgd_fp32_fma_rate(scratch.data_ptr(), nsm * 8 * 4, 4096, stream.cuda_stream) for _ in range(3))


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from sgd_b200.operators import A_B1_operator
    from sgd_b200.phantom import ellipse_phantom
    from sgd_b200.torch_ops import FanProjector
    from sgd_b200 import _lib

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    P = FanProjector("b1", NX, NY, NU, DX, DY, DU, LSD, LSO, ANGLES)
    x_host = ellipse_phantom(NX, NY, DX, DY, seed=rank)
    img = torch.tensor(x_host, dtype=torch.float32, device=dev)
    sino = torch.empty((NP, NU), dtype=torch.float32, device=dev)
    back = torch.empty((NX, NY), dtype=torch.float32, device=dev)
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        P.forward(img, out=sino)
        P.backward(sino, out=back)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)

    K = args.steps
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(K)]
    uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    sampler = ClockSampler(uuid)
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    t_wall = time.perf_counter()
    for k in range(K):
        flush.fill_(float(k))
        ev[k][0].record(stream)
        P.forward(img, out=sino)
        ev[k][1].record(stream)
        P.backward(sino, out=back)
        ev[k][2].record(stream)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    wall = time.perf_counter() - t_wall
    clocks = sampler.stop()
    fwd_ms = [ev[k][0].elapsed_time(ev[k][1]) for k in range(K)]
    bwd_ms = [ev[k][1].elapsed_time(ev[k][2]) for k in range(K)]
    step_ms = sum(f + b for f, b in zip(fwd_ms, bwd_ms)) / K
    step_ms = max_over_ranks(step_ms, world, dev)
    units = 2.0 * NX * NY * NP
    value = world * units / (step_ms * 1e-3)

    # end-to-end through the reference-facing C ABI with host FP64 buffers
    A = A_B1_operator(NX, NY, NP, NU, DX, DY, DU, LSD, LSO, ANGLES)
    xh = x_host.ravel().astype(np.float64)
    yh = A.matvec(xh)
    A.rmatvec(yh)
    ke = min(K, 20)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(ke):
        yh = A.matvec(xh)
        A.rmatvec(yh)
    e2e_s = (time.perf_counter() - t0) / ke
    e2e_value = world * units / max_over_ranks(e2e_s, world, dev)

    if rank != 0:
        return

    # roofline of the dominant kernel: algorithmic FLOPs of the reference
    # formula per launch over its measured duration, against the FP32 FMA
    # rate measured on this GPU now
    ops = load_op_counts()["b1_fan512"]
    V = NX * NY * NP
    E = P.conv_count
    flops = ops["range_flops_per_pixel_view"] * V + ops["flops_per_evaluation"] * E
    fwd_avg, bwd_avg = statistics.mean(fwd_ms), statistics.mean(bwd_ms)
    dom, dom_ms = ("b1_back_kernel", bwd_avg) if bwd_avg >= fwd_avg else ("b1_forward_kernel", fwd_avg)
    peak = fp32_peak(dev, stream)
    achieved = flops / (dom_ms * 1e-3)
    traffic = load_traffic().get(dom)
    roofline = {
        "bound": "fp32", "kernel": dom, "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "TFLOP/s",
        "frac": achieved / peak, "traffic": traffic,
        "peak_source": "measured now: FP32 FMA probe kernel (sgd_fp32_fma_rate), same clocks",
        "flops_per_launch": flops,
        "flops_model": f"{ops['range_flops_per_pixel_view']:.1f} x pixel-views + "
                       f"{ops['flops_per_evaluation']:.1f} x footprint evaluations ({E})",
        "fwd_ms": fwd_avg, "bwd_ms": bwd_avg,
    }

    # baselines, after the timed region, one GPU only: the reference's CPU
    # path and the reference's own CUDA layer
    cpu = ref_gpu = None
    if world == 1:
        r = cpu_spmv_sample(reps=3)
        cpu = {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": r["kind"], "sample": r["desc"],
               "single_thread_value": r["single_thread"], "seconds": round(r["spent"], 2)}
        ref_gpu = reference_gpu_layer()

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "config": CONFIG, "parallelism": f"replicas x{world}",
        "roofline": roofline, "cpu_baseline": cpu, "reference_gpu": ref_gpu,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 4 * (NX * NY + NP * NU),
                "d2h_bytes_per_step": 4 * (NP * NU + NX * NY),
                "path": "A_B1_operator.matvec/rmatvec -> b1_forward_projection / b1_backward_projection, FP64 numpy"},
        "gpu_launches": 3 * K,
        "clocks": clocks,
        "wall_s": wall,
    }
    print(json.dumps(line), flush=True)


def run_batch48(args, rank, world, local_rank):
    """48 uneven slices (sides 256/384/512, 360/540/720 views, ceil(1.44 N)
    bins) forward + adjoint per step, replayed from one CUDA graph."""
    import torch
    from sgd_b200.batch import B1Batch, uneven_slices
    from sgd_b200.phantom import ellipse_phantom

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    slices = uneven_slices(seed=rank)
    B = B1Batch(slices)
    fw, vc, loaded = B.tune()
    img = B.image_arena()
    for k, v in enumerate(B.images(img)):
        s = slices[k]
        v.copy_(torch.tensor(ellipse_phantom(s[0], s[1], s[3], s[4], seed=k), dtype=torch.float32))
    sino, back = B.sinogram_arena(), B.image_arena()
    B.capture(img, sino, sino, back)
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        B.replay()
    torch.cuda.synchronize(dev)
    K = args.steps
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(K)]
    uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    sampler = ClockSampler(uuid)
    time.sleep(0.3)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    for k in range(K):
        flush.fill_(float(k))
        ev[k][0].record(stream)
        B.replay()
        ev[k][1].record(stream)
    torch.cuda.synchronize(dev)
    clocks = sampler.stop()
    B.status()
    step_ms = sum(e[0].elapsed_time(e[1]) for e in ev) / K
    step_ms = max_over_ranks(step_ms, world, dev)
    units = 2.0 * sum(s[0] * s[1] * len(s[8]) for s in slices)
    if rank != 0:
        return
    line = {
        "metric": "fwd+adj voxel-view updates/s (B1 fan beam, 48-slice uneven batch)",
        "value": world * units / (step_ms * 1e-3), "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "48 fan-beam slices, N ~ U{256,384,512} at 256/N mm, views ~ U{360,540,720}, "
                               "ceil(1.44 N) bins at 1 mm, SOD 595 mm, SDD 1085.6 mm, seeded ellipse phantoms; "
                               "forward then adjoint, one CUDA graph (2 persistent launches + transpose)",
                   "voxel_views": units / 2, "variant": {"fw": fw, "vc": vc, "from_cache": loaded},
                   "l2": "flushed between steps (256 MiB write outside the timed events)"},
        "gpu_launches": 3 * K, "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def run_family(args, rank, world, local_rank):
    """Device-resident forward + adjoint of one of the other projector
    families (FAMILIES), timed like the headline workload."""
    import torch
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    desc, make, vv = _families()[args.workload]
    P = make()
    g = torch.Generator(device=dev).manual_seed(rank)
    x = torch.rand(P.image_shape, device=dev, generator=g)
    y = torch.empty(P.sino_shape, device=dev)
    b = torch.empty(P.image_shape, device=dev)
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        P.forward(x, out=y)
        P.backward(y, out=b)
    torch.cuda.synchronize(dev)
    K = args.steps
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(K)]
    sampler = ClockSampler("GPU-" + str(torch.cuda.get_device_properties(dev).uuid))
    time.sleep(0.3)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    for k in range(K):
        flush.fill_(float(k))
        ev[k][0].record(stream)
        P.forward(x, out=y)
        ev[k][1].record(stream)
        P.backward(y, out=b)
        ev[k][2].record(stream)
    torch.cuda.synchronize(dev)
    clocks = sampler.stop()
    fwd = statistics.mean(e[0].elapsed_time(e[1]) for e in ev)
    bwd = statistics.mean(e[1].elapsed_time(e[2]) for e in ev)
    step_ms = max_over_ranks(fwd + bwd, world, dev)
    if rank != 0:
        return
    roofline = None
    ops = load_op_counts().get(args.workload)
    if ops and "flops_per_cell_view" in ops:
        # the reference formula's FLOPs per launch (both directions evaluate
        # every visited (cell, bin) pair once) over the slower direction's time
        flops = ops["flops_per_cell_view"] * vv
        dom, dom_ms = ("back", bwd) if bwd >= fwd else ("forward", fwd)
        peak = fp32_peak(dev, stream)
        roofline = {"bound": "fp32", "kernel": f"{P.kernels[dom]}", "achieved": flops / (dom_ms * 1e-3) / 1e12,
                    "peak": peak / 1e12, "unit": "TFLOP/s", "frac": flops / (dom_ms * 1e-3) / peak,
                    "traffic": load_traffic().get(f"{args.workload}:{dom}"),
                    "peak_source": "measured now: FP32 FMA probe kernel (sgd_fp32_fma_rate), same clocks",
                    "flops_per_launch": flops, "flops_model": f"{ops['flops_per_cell_view']:.1f} x cell-views "
                    f"({ops['source']})", "fwd_ms": fwd, "bwd_ms": bwd,
                    "fwd_plus_adj_frac": 2 * flops / ((fwd + bwd) * 1e-3) / peak}
    line = {
        "metric": f"fwd+adj voxel-view updates/s ({args.workload})", "value": world * 2.0 * vv / (step_ms * 1e-3),
        "unit": UNIT, "n_gpus": world, "steps": K, "warmup": args.warmup, "ms_per_step": step_ms,
        "fwd_ms": fwd, "bwd_ms": bwd, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (uniform random image)",
        "config": {"workload": desc, "voxel_views": vv,
                   "l2": "flushed between steps (256 MiB write outside the timed events)"},
        "roofline": roofline, "gpu_launches": P.launches_per_step * K, "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def run_conv32(args, rank, world, local_rank):
    """The warm-start CNN's 32-to-32-channel 3x3 convolution (its three middle
    layers) on 64 images of 256^2: the tensor-core kernel
    (sgd_conv3x3_forward_tc: tcgen05 MMAs, FP32 activations as three BF16
    terms) and the FP32 direct kernel beside it, device-resident, L2 flushed
    between steps.  Roofline: DRAM bytes (the activations read and written
    once) over the measured HBM copy bandwidth, and the tensor FLOPs of the
    three passes over the measured BF16 GEMM peak."""
    import torch
    from sgd_b200.cnn import _declare, _stream
    from sgd_b200 import _lib
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    L = _lib.lib()
    _declare(L)
    n, h, w = 64, 256, 256
    g = torch.Generator(device=dev).manual_seed(rank)
    X = torch.randn((n, 32, h, w), device=dev, generator=g)
    W16 = (torch.randn((32, 32, 3, 3), device=dev, generator=g) * 0.2).to(torch.bfloat16)
    B = torch.randn(32, device=dev, generator=g)
    out_tc, out_fp = torch.empty_like(X), torch.empty_like(X)

    def tc():
        _lib.check(L.sgd_conv3x3_forward_tc(X.data_ptr(), W16.data_ptr(), B.data_ptr(), out_tc.data_ptr(), n, 32, 32,
                                            h, w, 1, _stream()), "conv tc")

    def fp():
        _lib.check(L.sgd_conv3x3_forward(X.data_ptr(), W16.data_ptr(), B.data_ptr(), out_fp.data_ptr(), n, 32, 32, h,
                                         w, 1, _stream()), "conv fp32")

    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        tc()
        fp()
    torch.cuda.synchronize(dev)
    K = args.steps
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(K)]
    uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    sampler = ClockSampler(uuid)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    for k in range(K):
        flush.fill_(float(k))
        ev[k][0].record(stream)
        tc()
        ev[k][1].record(stream)
        flush.fill_(float(k) + 0.5)
        ev[k][2].record(stream)
        fp()
        ev[k][3].record(stream)
    torch.cuda.synchronize(dev)
    clocks = sampler.stop()
    _lib.check(L.sgd_conv3x3_tc_status(), "conv tc status")
    tc_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in ev)
    fp_times = [e[2].elapsed_time(e[3]) for e in ev]
    step_ms = max_over_ranks(tc_ms, world, dev)
    if rank != 0:
        return
    pixels = n * h * w
    bytes_ = 2 * pixels * 32 * 4
    flops = 3 * 2.0 * pixels * 32 * 288
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    bf16 = peaks.get("bf16_tflops", 1590.0)
    rel = float((out_tc - out_fp).double().norm() / out_fp.double().norm())
    line = {
        "metric": "32-channel 3x3 convolution pixels/s (warm-start CNN middle layer, tensor cores)",
        "value": world * pixels / (step_ms * 1e-3), "unit": "pixels/s", "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16x3 operands, f32 accumulation", "data": "synthetic (normal activations)",
        "config": {"workload": "3x3 conv 32->32 channels, ReLU, 64 images 256x256, NCHW FP32",
                   "l2": "flushed between kernels (256 MiB write outside the timed events)"},
        "fp32_direct_ms": statistics.mean(fp_times),
        "rel_l2_tc_vs_fp32": rel,
        "roofline": {"bound": "hbm", "kernel": "conv3x3_c32_tc_kernel", "achieved": bytes_ / (tc_ms * 1e-3) / 1e9,
                     "peak": hbm, "unit": "GB/s", "frac": bytes_ / (tc_ms * 1e-3) / 1e9 / hbm,
                     "traffic": load_traffic().get("cnn_conv32:conv3x3_c32_tc_kernel"), "tensor_tflops": flops / (tc_ms * 1e-3) / 1e12, "tensor_peak": bf16,
                     "tensor_frac": flops / (tc_ms * 1e-3) / 1e12 / bf16,
                     "peak_source": "MEASURED_PEAKS.json (hbm_gbs, bf16_tflops)" if peaks else "fallback"},
        "gpu_launches": K, "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def run_asd(args, rank, world, local_rank):
    """Learned warm start vs plain ASD-POCS (64 fan-beam
    phantoms 256^2, 120 views, Poisson I0 = 1e5, the 5-layer 32-channel CNN
    trained on 2000 plain-ASD-POCS pairs by the library's kernels).  The
    value is the learned run's GPU time to plain's converged RMSE over
    plain's GPU time to convergence (lower is better; target <= 1/3)."""
    import torch
    from sgd_b200.asd import experiment
    torch.cuda.set_device(local_rank)
    r = experiment(log=(lambda m: print(m, file=sys.stderr, flush=True)) if rank == 0 else None)
    if rank != 0:
        return
    line = {
        "metric": "learned / plain ASD-POCS GPU time to plain's converged RMSE", "value": r["time_ratio"],
        "unit": "ratio", "n_gpus": world, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded ellipse phantoms, Poisson noise)",
        "config": {"workload": r["workload"], "rmse_truth": r["rmse_truth"], "convergence_rule": r["convergence_rule"]},
        "plain": {k: r["plain"][k] for k in ("iters", "converged", "gpu_ms", "rmse")},
        "learned": {k: r["learned"][k] for k in ("plain_iters_before_net", "iters_after_net", "gpu_ms", "net_ms",
                                                  "rmse", "reached")},
        "data_residual": {"plain_last": r["plain"]["data_residual"][-1],
                          "learned_last": (r["learned"]["data_residual"] or [None])[-1]},
        "training": {k: r["training"][k] for k in ("pairs", "target_iters", "epochs", "pairs_s", "train_s")},
        "calibration_converged": r["calibration_converged"],
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.workload == "batch48":
            run_batch48(args, rank, world, local_rank)
        elif args.workload == "asd_c5":
            run_asd(args, rank, world, local_rank)
        elif args.workload == "cnn_conv32":
            run_conv32(args, rank, world, local_rank)
        elif args.workload in FAMILIES:
            run_family(args, rank, world, local_rank)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
