"""Freezes the algorithmic work of the reference's projector formulas, counted
by the oracle's FLOP-counting scalar over a sample of views, into
sgd_b200/op_counts.json (read by bench.py for the roofline).

    python oracle/make_op_counts.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from oracle import oracle  # noqa: E402

OUT = os.path.join(os.path.dirname(HERE), "sgd_b200", "op_counts.json")


def main():
    out = {}
    ang = 2 * np.pi * np.arange(720) / 720
    r, f, e = oracle.b1_flops(512, 512, 736, 0.5, 0.5, 1.0, 1085.6, 595.0, ang, nviews=24)
    out["b1_fan512"] = {
        "geometry": "B1 fan 512x512 @0.5mm, 720 views, 736 bins @1mm, SOD 595, SDD 1085.6",
        "range_flops_per_pixel_view": r,
        "flops_per_evaluation": f,
        "evaluations_per_pixel_view": e,
        "source": "oracle/sgd_oracle.cpp oracle_b1_flops: +,-,*,/,sqrt of layers/A_B1.cu:96-206 "
                  "and layers/spline_conv.hh:295-405 counted on the path taken, 24 views",
    }
    per_view = "FLOPs per cell-view of the reference formula (bin range, per-cell terms, every bin visited)"
    fan = 2 * np.pi * np.arange(720) / 720
    hexa = 2 * np.pi * np.arange(360) / 360
    par = np.pi * np.arange(180) / 180
    rows = {
        "sf_fan512": ("sf", 512, 512, 736, 0.5, 0.5, 1.0, 1085.6, 595.0, fan,
                      "layers/A_SF.cu:96-225 (atan2/sin/cos per pixel-view not counted)"),
        "b0_fan512": ("b0", 512, 512, 736, 0.5, 0.5, 1.0, 1085.6, 595.0, fan, "layers/A_B0.cu:140-229"),
        # the reference has no parallel geometry: its B0 formula on a fan with
        # the source 1e4 pixels away stands in for the count
        "b0_parallel128": ("b0", 128, 128, 185, 1.0, 1.0, 1.0, 2e4, 1e4, par,
                           "layers/A_B0.cu:140-229 on a distant-source fan (no parallel geometry in the reference)"),
        "h0_hex2e18": ("h0", 550, 477, 736, 0.62, 0.62, 1.0, 1085.6, 595.0, hexa,
                       "layers/A_H0.cu:84-256 (six-vertex bound 6 x 9)"),
        "hl_hex2e18": ("hl", 953, 275, 736, 1.075, 1.075, 1.0, 1085.6, 595.0, hexa,
                       "layers/A_Hl.cu:21-46, :84-156, :168-266"),
    }
    for name, (kind, a, b, nu, dx, dy, du, lsd, lso, ang, src) in rows.items():
        f, nb = oracle.fan2d_flops(kind, a, b, nu, dx, dy, du, lsd, lso, ang, nviews=24)
        out[name] = {"flops_per_cell_view": f, "bins_per_cell_view": nb, "model": per_view,
                     "source": f"oracle/sgd_oracle.cpp oracle_fan2d_flops: {src}, 24 views"}
    # the B1 reference-rounding mode evaluates the B1 formula
    b1 = out["b1_fan512"]
    out["b1ref_fan512"] = {
        "flops_per_cell_view": b1["range_flops_per_pixel_view"]
        + b1["flops_per_evaluation"] * b1["evaluations_per_pixel_view"],
        "bins_per_cell_view": b1["evaluations_per_pixel_view"], "model": per_view,
        "source": "the b1_fan512 counts (layers/A_B1.cu:96-206)"}
    # the cone-beam forward formulas at the 256^3 workload (and its half-size
    # profiling case): every 4th column of voxels (all rows), 4 views
    cones = {
        "b1_3d_cone256": ("b1_3d", 256, 360, 384, 1.0, 1.5, "layers/A_B1_3D.cu:82-312"),
        "sf3d_cone256": ("sf3d", 256, 360, 384, 1.0, 1.5,
                         "layers/SF_projector.cu:81-234, amplitude and in-detector bins of the corrected pair"),
        "b1_3d_small": ("b1_3d", 128, 180, 192, 2.0, 3.0, "layers/A_B1_3D.cu:82-312"),
        "sf3d_small": ("sf3d", 128, 180, 192, 2.0, 3.0,
                       "layers/SF_projector.cu:81-234, amplitude and in-detector bins of the corrected pair"),
    }
    for name, (kind, n, views, nd, d, dd, src) in cones.items():
        ang = 2 * np.pi * np.arange(views) / views
        f, nb = oracle.cone_flops(kind, n, nd, d, dd, 1085.6, 595.0, ang, nviews=4, stride=4)
        out[name] = {"flops_per_cell_view": f, "bins_per_cell_view": nb,
                     "model": "FLOPs per voxel-view of the reference forward formula (bin ranges, per-voxel "
                              "terms, every (u, v) bin visited)",
                     "source": f"oracle/sgd_oracle.cpp oracle_cone_flops: {src}, 4 views, every 4th voxel column"}
    with open(OUT, "w") as fh:
        json.dump(out, fh, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
