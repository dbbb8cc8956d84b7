"""The pointwise work table of the roofline model (profiles/pointwise_flops.json)
against a fresh count with the op-counting scalar (tests/count_pointwise_flops.py)
on a degree-1 block: the per-point volume and face counts and the CG iteration's
split into points, DOFs and elements."""
from __future__ import annotations

import json
import os

import pytest

from count_pointwise_flops import count

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("riemann,key", [(1, "ismail_roe"), (0, "roe")])
def test_pointwise_table_matches_a_fresh_count(riemann, key):
    with open(os.path.join(ROOT, "profiles", "pointwise_flops.json")) as f:
        table = json.load(f)[key]
    c = count(riemann, 1)
    assert c["volume"] == table["volume_flops_per_point"]
    assert c["volume_specials"] == table["volume_specials_per_point"]
    assert c["face"] == table["face_flops_per_point"]
    assert c["face_specials"] == table["face_specials_per_point"]
    want = (table["cg_flops_per_iteration_per_point"] * c["M"] ** 3
            + table["cg_flops_per_iteration_per_dof"] * c["K"] ** 3
            + table["cg_flops_per_iteration_per_element"])
    assert c["cg_iteration"] == pytest.approx(want, abs=1e-6)
