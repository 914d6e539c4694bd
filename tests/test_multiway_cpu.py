"""Host parts of the four-player path: Malmuth-Harville ICM (FP64) against the
oracle's direct enumeration of finishing orders, bubble factors, and the
four-player tree builder."""
import importlib

import numpy as np
import pytest


@pytest.fixture(scope="module")
def mw():
    return importlib.import_module("mtt-gpu-solver_b200.multiway")


@pytest.mark.parametrize("n,m,seed", [(8, 3, 0), (6, 3, 1), (9, 4, 2), (3, 2, 3), (10, 5, 4)])
def test_icm_equity_matches_enumeration(mw, orc, n, m, seed):
    rng = np.random.default_rng(seed)
    stacks = rng.lognormal(np.log(20.0), 0.5, size=n)
    pay = np.sort(rng.random(m))[::-1]
    pay = pay / pay.sum()
    e = mw.icm_equity(stacks, pay)
    assert np.allclose(e, orc.icm_equity(stacks, pay), rtol=1e-12, atol=1e-15)
    assert abs(e.sum() - pay.sum()) < 1e-12          # every paid place is given out
    order = np.argsort(stacks)
    assert (np.diff(e[order]) >= -1e-15).all()        # more chips, more equity


def test_icm_single_payout_is_chip_share(mw):
    st = np.array([10.0, 30.0, 60.0])
    assert np.allclose(mw.icm_equity(st, [1.0]), st / st.sum())


def test_bubble_factors(mw):
    stacks = np.array([10, 20, 30, 40, 5, 15, 25, 35], float)
    bf = mw.bubble_factors(stacks, [0.5, 0.3, 0.2], [0, 1, 2, 3])
    assert bf.shape == (4, 4)
    off = bf[~np.eye(4, dtype=bool)]
    assert (off > 1.0).all()                          # ICM: losing hurts more than winning helps
    for k in range(4):
        assert abs(bf[k, k] - np.mean(np.delete(bf[k], k))) < 1e-12
    # winner-take-all is chip EV
    assert np.allclose(mw.bubble_factors(stacks, [1.0], [0, 1, 2, 3]), 1.0)


def test_four_player_tree(mw):
    nodes, rows, depth = mw.build_tree(4.0, [20, 20, 20, 20], [0.5, 1.0], 1.0, 1)
    assert len(nodes) == 677 and rows == (169, 169, 169, 169)
    t = nodes["type"]
    assert (nodes["num_actions"][t == 0] <= 3).all()
    assert np.allclose(nodes["pot_size"], nodes["committed"].sum(axis=1), rtol=1e-6)
    for i in np.nonzero(t == 0)[0]:
        c0, na = nodes["children_offset"][i], nodes["num_actions"][i]
        assert c0 > i and c0 + na <= len(nodes)
    fm = nodes["active_mask"][t == 1]
    assert all(bin(int(m)).count("1") == 1 for m in fm)
    sm = nodes["active_mask"][t == 2]
    assert all(bin(int(m)).count("1") >= 2 for m in sm)
    # short stacks cap the bets (no side pots): fewer nodes, still valid
    n2, r2, _ = mw.build_tree(4.0, [3, 20, 20, 20], [0.5, 1.0], 1.0, 1)
    assert 0 < len(n2) < 677
