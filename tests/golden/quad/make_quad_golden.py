"""Writes the quad golden matrices of tests/golden/quad/ by running the
reference's own exact projectors, python/matrix_gen/A_B0_ref_project.py and
A_B1_ref_project.py (scipy `quad` over each bin of the bin-averaged line
integral, numba-compiled integrands), unmodified, from the reference tree.

    python tests/golden/quad/make_quad_golden.py [REFERENCE_ROOT] [OUTDIR]

REFERENCE_ROOT defaults to $SGD_REFERENCE, else the reference checkout beside
the repository (read only; Python writes no bytecode there).  Each fixture holds the geometry and the reference's COO
triplets (row p*nu + u, column ix*ny + iy, value); views are the scripts'
own linspace(0, 2 pi, np, endpoint=False).  tests/test_oracle.py checks the
CPU oracle's exact matrices (oracle_exact_fan2d_matrix) against them.
"""
import contextlib
import io
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# (basis, nx, ny, np, nu, dx, dy, du, lsd, lso): small fan geometries the
# quadrature finishes in about a second
CASES = {
    "quad_b0_aniso": ("b0", 12, 10, 5, 24, 1.0, 0.8, 1.1, 60.0, 30.0),
    "quad_b1_unit": ("b1", 12, 10, 5, 24, 1.0, 1.0, 1.1, 60.0, 30.0),
    "quad_b1_iso08": ("b1", 12, 10, 5, 24, 0.8, 0.8, 1.1, 60.0, 30.0),
}


def main(ref_root, out):
    sys.dont_write_bytecode = True
    py = os.path.join(ref_root, "python")
    sys.path[:0] = [py, os.path.join(py, "matrix_gen")]
    import A_B0_ref_project
    import A_B1_ref_project
    scripts = {"b0": A_B0_ref_project, "b1": A_B1_ref_project}
    os.makedirs(out, exist_ok=True)
    for name, (kind, nx, ny, npv, nu, dx, dy, du, lsd, lso) in CASES.items():
        with contextlib.redirect_stdout(io.StringIO()):  # the B1 script prints every pixel
            t = scripts[kind].get_projection_matrix(nx, ny, npv, nu, dx, dy, du, lsd, lso)
        np.savez_compressed(os.path.join(out, f"{name}.npz"), kind=kind, sizes=np.array([nx, ny, npv, nu]),
                            params=np.array([dx, dy, du, lsd, lso]), rows=t[0].astype(np.int64),
                            cols=t[1].astype(np.int64), vals=t[2])
        print(name, "entries", t.shape[1])


if __name__ == "__main__":
    default_ref = os.environ.get("SGD_REFERENCE",
                                 os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(HERE))), "..",
                                              "reference"))
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.normpath(default_ref),
         sys.argv[2] if len(sys.argv) > 2 else HERE)
