"""Writes the golden vectors of tests/golden/ by running the reference projector
library built from its own sources (oracle/_ref/libnetwork.so) on a GPU.

    python tests/golden/make_golden.py OUTDIR

Each fixture holds the geometry, a seeded phantom x, the reference's forward
b = A x and footprint count, a second sinogram y (forward of another phantom)
and the reference's back projection xt = A^T y.  The CPU oracle is checked
against them by tests/test_oracle.py.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import reflib  # noqa: E402
from geometry_cases import cone_case, fan_case, hex_case  # noqa: E402
from sgd_b200.phantom import ellipse_phantom, ellipsoid_phantom, hex_phantom  # noqa: E402

CASES = {
    "b1_tiny": ("b1", "tiny"),
    "b1_snap": ("b1", "snap"),
    "b1_wide": ("b1", "wide"),
    "sf_tiny": ("SF", "tiny"),
    "sf_snap": ("SF", "snap"),
    "sf_wide": ("SF", "wide"),
    "b0_tiny": ("b0", "tiny"),
    "b0_snap": ("b0", "snap"),
    "b0_wide": ("b0", "wide"),
}


HEX_CASES = {
    "hex_h0_small": ("h0", "small", 1.5),
    "hex_hl_small": ("hl", "small", 0.5),
}


# cone-beam fixtures: A_B1_3D forward (its C backward returns zeros), and the
# SF layer's forward (SF-TR and SF-TT) and back projection
CONE_CASES = {
    "b1_3d_tiny": ("b1_3d", "tiny"),
    "sf3d_tiny": ("sf3d", "tiny"),
    "sf3d_tallz": ("sf3d", "tallz"),
}


# matrix generators: (kind, np, nu, nx, ny, dx, dy, du, lsd, lso)
MATRIX_CASES = {
    "matgen_b1_small": ("b1", 8, 40, 24, 24, 2.0, 2.0, 2.0, 1085.6, 595.0),
    "matgen_b0_small": ("b0", 8, 40, 24, 24, 2.0, 2.0, 2.0, 1085.6, 595.0),
    "matgen_b1_rect": ("b1", 6, 32, 20, 14, 1.5, 2.5, 1.7, 900.0, 500.0),
}


def main(out):
    os.makedirs(out, exist_ok=True)
    for name, (kind, npv, nu, nx, ny, dx, dy, du, lsd, lso) in MATRIX_CASES.items():
        n, spmat = reflib.matrix_generation(kind, npv, nu, nx, ny, dx, dy, du, lsd, lso, 400000)
        t = spmat[:n]
        np.savez_compressed(os.path.join(out, f"{name}.npz"), kind="matgen_" + kind,
                            sizes=np.array([npv, nu, nx, ny]), params=np.array([dx, dy, du, lsd, lso]),
                            rows=t[:, 0].astype(np.int64), cols=t[:, 1].astype(np.int32), vals=t[:, 2])
        print(name, "nnz", n)
    for name, (kind, case) in CONE_CASES.items():
        g = cone_case(case)
        nx, ny, nz, nu, nv, dx, dy, dz, du, dv, lsd, lso, ang = g
        x = ellipsoid_phantom(nx, ny, nz, dx, dy, dz, seed=11).ravel()
        extra = {}
        if kind == "b1_3d":
            R = reflib.RefCone(*g)
            b, cnt = R.forward(x)
            extra = dict(count=cnt)
        else:
            R = reflib.RefSF3D(*g)
            b = R.forward(x)
            y = np.random.default_rng(12).random(len(ang) * nu * nv)
            extra = dict(b_tt=R.forward(x, trap=True), y=y, xt=R.backward(y))
        np.savez_compressed(os.path.join(out, f"{name}.npz"), kind=kind, sizes=np.array([nx, ny, nz, nu, nv]),
                            params=np.array([dx, dy, dz, du, dv, lsd, lso]), angles=ang, x=x, b=b, tol=1e-5,
                            **extra)
        print(name, "norm b", np.linalg.norm(b))
    for name, (kind, case, pitch) in HEX_CASES.items():
        nl, nc, nu, dt, du, lsd, lso, ang = hex_case(case)
        R = reflib.RefHex(kind, nl, nc, nu, dt, du, lsd, lso, ang)
        x = hex_phantom(nl, nc, dt, pitch * dt, seed=11).ravel()
        b, cnt = R.forward(x)
        y, _ = R.forward(hex_phantom(nl, nc, dt, pitch * dt, seed=12).ravel())
        xt = R.backward(y)
        np.savez_compressed(os.path.join(out, f"{name}.npz"), kind="hex_" + kind, sizes=np.array([nl, nc, nu]),
                            params=np.array([dt, du, lsd, lso]), angles=ang, x=x, b=b, count=cnt, y=y, xt=xt,
                            tol=1e-5)
        print(name, "count", cnt, "norm b", np.linalg.norm(b))
    for name, (kind, case) in CASES.items():
        nx, ny, nu, dx, dy, du, lsd, lso, ang = fan_case(case)
        R = reflib.RefFan2D(kind, nx, ny, nu, dx, dy, du, lsd, lso, ang)
        x = ellipse_phantom(nx, ny, dx, dy, seed=11).ravel()
        b, cnt = R.forward(x)
        y, _ = R.forward(ellipse_phantom(nx, ny, dx, dy, seed=12).ravel())
        xt = R.backward(y)
        np.savez_compressed(os.path.join(out, f"{name}.npz"), kind=kind.lower(), sizes=np.array([nx, ny, nu]),
                            params=np.array([dx, dy, du, lsd, lso]), angles=ang, x=x, b=b, count=cnt, y=y,
                            xt=xt, tol=1e-5)
        print(name, "count", cnt, "norm b", np.linalg.norm(b))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
