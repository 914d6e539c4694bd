"""The preflop DCFR chain against the reference's own loop kernels.

tests/golden/ref_pf_dcfr.npz holds the strategy sums and last strategies that
the reference's kernel_update_dynamic_reaches / kernel_cosolve_100_board_matrices /
kernel_build_closed_preflop_cfvs / kernel_dcfr_step
(src/preflop/preflop_grid_generator.cu:228-421), built with its own
--use_fast_math, produced on a B200 after preflop_gen's 500 iterations (made by
tests/golden/make_ref_pf_golden.py).  Its inputs are the reference-mode all-in
and class matrices whose hashes tests/golden/preflop_ref.json pins, and that
file's strategy sums are the oracle's (which the GPU chain matches bit for
bit).  The two must agree: each node's sums within 1e-4 of its largest sum,
the normalised average strategies within 1e-4, and the 15-hand table
preflop_gen prints (3 decimals) identical.  They are not bit-identical: the
reference's fast-math divisions round differently from IEEE division."""
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NODES = {"btn_root": (0, 3), "bb_def": (3, 6), "btn_vs_3b": (6, 8), "bb_vs_jam": (8, 10)}
INDICES = [0, 1, 2, 3, 4, 5, 6, 12, 13, 17, 72, 85, 91, 104, 168]


@pytest.fixture(scope="module")
def both():
    f = os.path.join(GOLD, "ref_pf_dcfr.npz")
    if not os.path.isfile(f):
        pytest.skip("tests/golden/ref_pf_dcfr.npz not generated")
    z = np.load(f)
    g = json.load(open(os.path.join(GOLD, "preflop_ref.json")))
    return z, g


def test_same_inputs_and_schedule(both):
    z, g = both
    assert str(z["allin_f32_sha256"]) == g["allin_f32_sha256"]
    assert str(z["class_mats_sha256"]) == g["class_mats_sha256"]
    assert int(z["iters"]) == g["dcfr_iters"] == 500
    assert (float(z["stack_bb"]), float(z["bubble"]), float(z["dead_pot"])) == pytest.approx(
        (g["stack_bb"], g["bubble"], g["dead_pot"]))


@pytest.mark.parametrize("node", list(NODES))
def test_strategy_sums_match_reference_loop(both, node):
    z, g = both
    a, b = NODES[node]
    ref = z["sums"].astype(np.float64)[a:b, :169]
    orc = np.asarray(g["sums"], np.float64)[a:b, :169]
    assert np.abs(ref - orc).max() <= 1e-4 * np.abs(orc).max()
    pr = ref / np.maximum(ref.sum(0), 1e-30)
    po = orc / np.maximum(orc.sum(0), 1e-30)
    assert np.abs(pr - po).max() <= 1e-4


def test_printed_table_is_identical(both):
    z, g = both

    def table(s):
        out = []
        for c in INDICES:   # preflop_grid_generator.cu:640-652
            btn = s[0:3, c] / (s[0:3, c].sum() + np.float32(1e-7))
            bb = s[3:6, c] / (s[3:6, c].sum() + np.float32(1e-7))
            out.append(" ".join(f"{x:.3f}" for x in list(btn) + list(bb)))
        return out
    assert table(z["sums"]) == table(np.asarray(g["sums"], np.float32))
