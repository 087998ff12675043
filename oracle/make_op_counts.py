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
    with open(OUT, "w") as fh:
        json.dump(out, fh, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
