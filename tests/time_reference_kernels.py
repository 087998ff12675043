"""Times the reference's own CUDA projector kernels (oracle/_ref/libnetwork.so,
built from the reference's sources) beside this library's, on the same GPU
and the headline geometry (512x512 @0.5 mm, 720 views over 2 pi, 736 bins @1 mm,
SOD 595 mm, SDD 1085.6 mm).  Test infrastructure: a measurement of the
reference, not part of the product.

    python tests/time_reference_kernels.py [--reps 5]

Per projector kind (b1, SF, b0) one JSON line: kernel-only milliseconds per
direction for both (device-resident buffers; the reference's through the
layer's project/back_project, its per-view launches included) and the
end-to-end milliseconds of one forward + one backward through the FP64 host
C ABI (host copies and conversions included).  With --e2e-only h0,hl,b1_3d
the hexagonal (about 2^18 sites, 360 views) and cone-beam (256^3, 360 views,
384^2 detector) layers are compared end to end through the same C ABI, in
the reference's own modes.  With --matrix the system-matrix generators
(bilinear_matrix_generation, pixel_matrix_generation) are timed on both
libraries at 128^2 x 180 views and 256^2 x 90 views."""
import argparse
import ctypes
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [HERE, os.path.dirname(HERE)]

import reflib  # noqa: E402

NX = NY = 512
DX = DY = 0.5
NP, NU, DU = 720, 736, 1.0
LSD, LSO = 1085.6, 595.0
ANGLES = 2 * np.pi * np.arange(NP) / NP


def ours(kind, reps):
    import torch
    from sgd_b200 import operators as ops
    from sgd_b200.phantom import ellipse_phantom
    from sgd_b200.torch_ops import FanProjector
    P = FanProjector(kind, NX, NY, NU, DX, DY, DU, LSD, LSO, ANGLES)
    x = torch.tensor(ellipse_phantom(NX, NY, DX, DY, seed=0), dtype=torch.float32, device="cuda")
    y = P.forward(x)
    b = P.backward(y)
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    e[0].record()
    for _ in range(reps):
        P.forward(x, out=y)
    e[1].record()
    for _ in range(reps):
        P.backward(y, out=b)
    e[2].record()
    torch.cuda.synchronize()
    cls = {"b1": ops.A_B1_operator, "SF": ops.A_SF_operator, "b0": ops.A_B0_operator}[kind]
    A = cls(NX, NY, NP, NU, DX, DY, DU, LSD, LSO, ANGLES)
    xh = ellipse_phantom(NX, NY, DX, DY, seed=0).ravel()
    A.rmatvec(A.matvec(xh))
    t0 = time.perf_counter()
    for _ in range(reps):
        A.rmatvec(A.matvec(xh))
    e2e = (time.perf_counter() - t0) / reps * 1e3
    return e[0].elapsed_time(e[1]) / reps, e[1].elapsed_time(e[2]) / reps, e2e


def reference(kind, reps):
    from sgd_b200.phantom import ellipse_phantom
    L = reflib.lib()
    R = reflib.RefFan2D(kind, NX, NY, NU, DX, DY, DU, LSD, LSO, ANGLES)
    fn = getattr(L, f"ref_{kind.lower()}_kernel_ms")
    fn.restype = ctypes.c_float
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    back = ctypes.c_float(0.0)
    fwd = fn(R.h, reps, ctypes.byref(back))
    xh = ellipse_phantom(NX, NY, DX, DY, seed=0).ravel()
    yh, _ = R.forward(xh)
    R.backward(yh)
    t0 = time.perf_counter()
    for _ in range(reps):
        yh, _ = R.forward(xh)
        R.backward(yh)
    e2e = (time.perf_counter() - t0) / reps * 1e3
    return fwd, back.value, e2e


def e2e_pair(kind, reps):
    """(reference ms, ours ms) of one forward + one backward through the C ABI."""
    from sgd_b200 import operators as ops
    rng = np.random.default_rng(0)
    if kind in ("h0", "hl"):
        nl, nc, dt = (550, 477, 0.62) if kind == "h0" else (953, 275, 1.075)
        ang = 2 * np.pi * np.arange(360) / 360
        R = reflib.RefHex(kind, nl, nc, NU, dt, DU, LSD, LSO, ang)
        cls = ops.A_H0_operator if kind == "h0" else ops.A_Hl_operator
        A = cls(nl, nc, len(ang), NU, dt, DU, LSD, LSO, ang)
        x = rng.random(nl * nc)
    else:
        n, ang = 256, 2 * np.pi * np.arange(360) / 360
        R = reflib.RefCone(n, n, n, 384, 384, 1.0, 1.0, 1.0, 1.5, 1.5, LSD, LSO, ang)
        A = ops.A_B1_3D_operator(n, n, n, len(ang), 384, 384, 1.0, 1.0, 1.0, 1.5, 1.5, LSD, LSO, ang)
        x = rng.random(n ** 3)

    def run(f, b):
        y = f(x)
        y = y[0] if isinstance(y, tuple) else y
        b(y)

    run(R.forward, R.backward)
    t0 = time.perf_counter()
    for _ in range(reps):
        run(R.forward, R.backward)
    tr = (time.perf_counter() - t0) / reps * 1e3
    run(A.matvec, A.rmatvec)
    t0 = time.perf_counter()
    for _ in range(reps):
        run(A.matvec, A.rmatvec)
    to = (time.perf_counter() - t0) / reps * 1e3
    return tr, to


def matrix_pair(kind, n, views):
    """(reference s, ours s, nnz) of one call of the generator at n^2 pixels of
    (256/n) mm, `views` views, ceil(1.44 n) bins of (512/n) mm."""
    from sgd_b200.operators import matrix_generation
    d, nu, du = 256.0 / n, int(np.ceil(1.44 * n)), 512.0 / n
    cap = int(5 * n * n * views)
    t0 = time.perf_counter()
    nr, _ = reflib.matrix_generation(kind, views, nu, n, n, d, d, du, LSD, LSO, cap)
    tr = time.perf_counter() - t0
    matrix_generation(kind, n, n, views, nu, d, d, du, LSD, LSO, buffer_size=cap)  # first call: setup
    t0 = time.perf_counter()
    no, _ = matrix_generation(kind, n, n, views, nu, d, d, du, LSD, LSO, buffer_size=cap)
    to = time.perf_counter() - t0
    return tr, to, nr, no


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--matrix", action="store_true")
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--kinds", default="b1,SF,b0")
    ap.add_argument("--e2e-only", default="")
    args = ap.parse_args()
    if not reflib.available():
        print(json.dumps({"unavailable": "oracle/_ref/libnetwork.so not built (make -C oracle ref)"}))
        return
    units = 2.0 * NX * NY * NP
    for kind in [k for k in args.kinds.split(",") if k]:
        rf, rb, re = reference(kind, args.reps)
        of, ob, oe = ours(kind, args.reps)
        print(json.dumps({
            "kind": kind, "geometry": "512x512 @0.5mm, 720 views, 736 bins @1mm, SOD 595, SDD 1085.6",
            "reference_ms": {"fwd": rf, "back": rb, "e2e_fwd_back": re},
            "ours_ms": {"fwd": of, "back": ob, "e2e_fwd_back": oe},
            "kernel_speedup": (rf + rb) / (of + ob), "e2e_speedup": re / oe,
            "ours_updates_per_s": units / ((of + ob) * 1e-3),
            "reference_updates_per_s": units / ((rf + rb) * 1e-3),
        }), flush=True)
    for kind in [k for k in args.e2e_only.split(",") if k]:
        tr, to = e2e_pair(kind, max(1, args.reps // 2))
        print(json.dumps({"kind": kind, "reference_e2e_fwd_back_ms": tr, "ours_e2e_fwd_back_ms": to,
                          "e2e_speedup": tr / to, "modes": "the reference's own (H0 bounds, A_B1_3D pair as "
                          "the reference: its backward returns zeros, timed all the same)"}), flush=True)
    if args.matrix:
        for kind in ("b1", "b0"):
            for n, views in ((128, 180), (256, 90)):
                tr, to, nr, no = matrix_pair(kind, n, views)
                print(json.dumps({"generator": kind, "pixels": n, "views": views, "reference_s": tr, "ours_s": to,
                                  "speedup": tr / to, "nnz_reference": nr, "nnz_ours": no}), flush=True)


if __name__ == "__main__":
    main()
