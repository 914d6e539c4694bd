"""The checker's restatement of the batched river workload (oracle/pyworkload.py)
draws the same subgames as the product's generator: same boards, supports,
weights and trees, node for node.  bench.py's CPU legs build their subgames
with it, so the CPU baseline never loads the product library."""
import numpy as np
import pytest

import pyworkload


def _same_tree(a, b):
    assert a.dtype.names == b.dtype.names
    for k in a.dtype.names:
        assert np.array_equal(a[k], b[k]), k


def test_batched_workload_matches_the_product_generator(wl):
    mine = pyworkload.river_batch(n=300, seed=2)
    theirs = wl.river_batch(n=300, seed=2)
    for g, h in zip(mine, theirs):
        assert g["board"] == h["board"] and g["pot"] == h["pot"]
        assert tuple(g["rows"]) == tuple(h["rows"])
        _same_tree(g["nodes"], h["nodes"])
        for p in (0, 1):
            assert np.array_equal(g[f"combos{p}"], h[f"combos{p}"])
            assert np.array_equal(g[f"range{p}"], h[f"range{p}"])


@pytest.mark.parametrize("sizes,cap,pot,stack", [
    ([0.5, 1.0], 1, 100.0, 200.0), ([0.33, 0.75, 1.5], 2, 60.0, 470.0), ([0.25, 0.6, 1.1, 2.0], 3, 30.2, 362.4),
    ([1.9], 3, 187.3, 93.6), ([0.7, 1.3], 2, 20.0, 10.0), ([0.5], 1, 100.0, 0.0)])
def test_river_tree_matches_the_product_builder(mtt, sizes, cap, pot, stack):
    nodes, rows = pyworkload.river_tree(pot, stack, sizes, raise_cap=cap)
    ref, rrows, _ = mtt.build_tree(pot, stack, sizes, raise_cap=cap)
    assert tuple(rows) == tuple(rrows)
    _same_tree(nodes, ref)


def test_live_combos(mtt):
    rng = np.random.default_rng(0)
    for _ in range(20):
        board = [int(c) for c in rng.choice(52, size=5, replace=False)]
        assert np.array_equal(pyworkload.live_combos(board), mtt.live_combos(board))
