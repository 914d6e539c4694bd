"""The oracle's heads-up sweeps against the reference's own kernels.

tests/golden/ref_hu_river.npz holds the regrets, strategy sums and root
counterfactual values that the reference's kernel_forward_sweep /
kernel_evaluate_terminals / kernel_backward_sweep
(src/postflop/honest_multistreet_solver.cu:88-249) produced on a B200 for a
seeded river subgame (made by tests/golden/make_ref_hu_golden.py).  The
oracle's CFR+ in the reference semantics, with simultaneous updates and linear
averaging, must reproduce them: regrets and strategy sums within 1e-4 of their
largest entry, counterfactual values within 1e-4 of the pot per unit of
opponent mass (the reference sums showdowns in FP32, the oracle in FP64)."""
import os

import numpy as np
import pytest

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_hu_river.npz")


def load_fixture():
    if not os.path.isfile(FIX):
        pytest.skip("tests/golden/ref_hu_river.npz not generated")
    z = np.load(FIX)
    sub = {"nodes": z["nodes"], "rows": tuple(int(x) for x in z["rows"]), "board": z["board"],
           "combos0": z["combos"], "combos1": z["combos"].copy(), "range0": z["range0"], "range1": z["range1"],
           "pot": float(z["pot"])}
    want = {int(it): {k: z[f"it{it}_{k}"] for k in ("R0", "R1", "S0", "S1", "cfv0", "cfv1")} for it in z["iters"]}
    return sub, want


def compare(sub, want, got):
    for key in ("R0", "R1", "S0", "S1"):
        scale = max(1e-12, float(np.abs(want[key]).max()))
        assert np.abs(want[key] - got[key]).max() <= 1e-4 * scale, key
    for q in (0, 1):
        mass = float(np.sum(sub[f"range{1 - q}"]))
        assert np.abs(want[f"cfv{q}"] - got[f"cfv{q}"]).max() <= 1e-4 * sub["pot"] * mass, q


def test_fixture_is_a_nontrivial_solve():
    sub, want = load_fixture()
    assert len(sub["combos0"]) == 700 and max(sub["nodes"]["num_actions"]) <= 3
    for w in want.values():
        assert np.abs(w["R0"]).max() > 0 and np.abs(w["S1"]).max() > 0 and np.abs(w["cfv0"]).max() > 0


@pytest.mark.parametrize("iters", [1, 4])
def test_oracle_matches_reference_kernels(orc, iters):
    sub, want = load_fixture()
    got = orc.cfr_solve(sub, iters, algo=0, semantics=1, alternate=0, avg_power=1.0)
    compare(sub, want[iters], got)
