"""The oracle's four-player sweeps against the reference's own kernels.

tests/golden/ref_mw_river.npz holds the regrets, strategy sums and root
counterfactual values that the reference's kernel_4way_forward_sweep /
kernel_4way_evaluate_terminals / kernel_4way_backward_cfr_plus
(src/postflop/multiway_4way_engine.cu:41-257) produced on a B200 for a seeded
ICM river subgame (made by tests/golden/make_ref_mw_golden.py).  The oracle's
CFR+ in the reference semantics must reproduce them: regrets and strategy
sums within 1e-4 of their largest entry, root counterfactual values within
1e-4 of the pot (the ranges are normalised, so the opponents' mass product is
at most 1)."""
import os

import numpy as np
import pytest

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_mw_river.npz")


def load_fixture():
    if not os.path.isfile(FIX):
        pytest.skip("tests/golden/ref_mw_river.npz not generated")
    z = np.load(FIX)
    sub = {"nodes": z["nodes"], "rows": tuple(int(x) for x in z["rows"]), "board": z["board"], "combos": z["combos"],
           "ranges": [z["ranges"][p] for p in range(4)], "bubble": z["bubble"], "pot": float(z["pot"])}
    want = {int(it): {"R": [z[f"it{it}_R{p}"] for p in range(4)], "S": [z[f"it{it}_S{p}"] for p in range(4)],
                      "cfv": z[f"it{it}_cfv"]} for it in z["iters"]}
    return sub, want


def compare(sub, want, got):
    for k in ("R", "S"):
        for p in range(4):
            scale = max(1e-12, float(np.abs(want[k][p]).max()))
            assert np.abs(want[k][p] - got[k][p]).max() <= 1e-4 * scale, (k, p)
    assert np.abs(want["cfv"] - got["cfv"]).max() <= 1e-4 * sub["pot"]


def test_fixture_is_a_nontrivial_solve():
    sub, want = load_fixture()
    assert len(sub["combos"]) == 400 and max(sub["nodes"]["num_actions"]) <= 3
    for w in want.values():
        assert all(np.abs(w["R"][p]).max() > 0 for p in range(4)) and np.abs(w["cfv"]).max() > 0


@pytest.mark.parametrize("iters", [1, 4])
def test_oracle_matches_reference_kernels(orc, iters):
    sub, want = load_fixture()
    got = orc.mw_solve(sub, iters, algo=0, semantics=1, avg_power=1.0)
    compare(sub, want[iters], got)
