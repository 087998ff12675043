"""The algorithmic work frozen in sgd_b200/op_counts.json (the roofline
numerators of bench.py) is what the oracle's FLOP-counting scalar gives for
the reference formulas: recount the cone-beam entries (a few seconds) and
check every entry's fields."""
import json
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
COUNTS = json.load(open(os.path.join(ROOT, "sgd_b200", "op_counts.json")))


@pytest.mark.parametrize("name,kind", [("b1_3d_cone256", "b1_3d"), ("sf3d_cone256", "sf3d")])
def test_cone_counts_are_the_oracle_recount(oracle_mod, name, kind):
    ang = 2 * np.pi * np.arange(360) / 360
    f, nb = oracle_mod.cone_flops(kind, 256, 384, 1.0, 1.5, 1085.6, 595.0, ang, nviews=4, stride=4)
    assert COUNTS[name]["flops_per_cell_view"] == f
    assert COUNTS[name]["bins_per_cell_view"] == nb


def test_every_family_has_a_count():
    for name in ("b1_fan512", "sf_fan512", "b0_fan512", "b0_parallel128", "h0_hex2e18", "hl_hex2e18",
                 "b1ref_fan512", "b1_3d_cone256", "sf3d_cone256", "b1_3d_small", "sf3d_small"):
        e = COUNTS[name]
        per = e.get("flops_per_cell_view", e.get("flops_per_evaluation"))
        assert per and per > 0, name
        assert "source" in e and ("oracle" in e["source"] or "b1_fan512" in e["source"]), name
