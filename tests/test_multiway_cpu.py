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


def test_config4_tree_size(wl):
    """The four-player configuration: bets {50%, 100%}, one pot-sized raise
    size re-raised up to twice, at seed 4's stacks."""
    sub = wl.multiway_icm(seed=4)
    assert len(sub["nodes"]) == 1585 and len(sub["combos"]) == 1081


def _no_removal_values(orc, sub, node, reach):
    """Ties split, opponents' full masses (no card removal), for comparison."""
    nd = sub["nodes"][node]
    board = list(sub["board"])
    cards = np.array([(a, b) for a in range(52) for b in range(a + 1, 52)], np.uint8)[sub["combos"].astype(np.int64)]
    sc = orc.eval7(np.array([board + list(c) for c in cards], np.uint8)).astype(np.int64)
    H = len(sc)
    W = np.array([r.sum() for r in reach], np.float64)
    L = np.array([[reach[o][sc < sc[h]].sum() for h in range(H)] for o in range(4)])
    E = np.array([[reach[o][sc == sc[h]].sum() for h in range(H)] for o in range(4)])
    bf = np.asarray(sub["bubble"], np.float64).reshape(4, 4)
    am, pot, c = int(nd["active_mask"]), float(nd["pot_size"]), nd["committed"].astype(np.float64)
    out = np.zeros((4, H))
    for p in range(4):
        opp = [o for o in range(4) if o != p]
        others = np.prod(W[opp])
        for h in range(H):
            if nd["type"] == 1:
                w = (am & -am).bit_length() - 1
                out[p, h] = ((pot - c[p]) if p == w else -bf[p, w] * c[p]) * others
            elif not (am >> p) & 1:
                out[p, h] = -bf[p, p] * c[p] * others
            else:
                act = [o for o in opp if (am >> o) & 1]
                ina = np.prod([W[o] for o in opp if not (am >> o) & 1])
                share = 0.0
                for T in range(1 << len(act)):
                    pr = np.prod([E[o, h] if (T >> i) & 1 else L[o, h] for i, o in enumerate(act)])
                    share += pr * (pot / (1 + bin(T).count("1")) - c[p])
                LE = np.prod([L[o, h] + E[o, h] for o in act])
                out[p, h] = (share - bf[p, p] * c[p] * (np.prod(W[act]) - LE)) * ina
    return out


@pytest.mark.parametrize("seed", [7, 8])
def test_card_removal_moves_terminals_toward_the_exact_game(wl, orc, seed):
    """At small sizes, the correct semantics' terminal values (each opponent's
    mass counted over the hands that share no card with the hero) against
    the exact four-player showdown over disjoint hands, and the same payoffs
    with no card removal.  Removing the hero's cards roughly halves the mean
    error; what remains is the opponents' overlaps with one another (about a
    quarter of random opponent triples share a card), which the
    independent-opponents model keeps."""
    sub = wl.multiway_icm(seed=seed, n_hands=26)
    rng = np.random.default_rng(seed)
    reach = [rng.dirichlet(np.full(26, 0.5)).astype(np.float32) for _ in range(4)]
    t = sub["nodes"]["type"]
    am = sub["nodes"]["active_mask"]
    picks = [int(np.where(t == 1)[0][0])]
    for k in (4, 3, 2):
        idx = np.where((t == 2) & (np.array([bin(int(x)).count("1") for x in am]) == k))[0]
        if len(idx):
            picks.append(int(idx[0]))
    for node in picks:
        exact = orc.mw_terminal(sub, node, reach, exact=True)
        cr = orc.mw_terminal(sub, node, reach, semantics=0).astype(np.float64)
        nr = _no_removal_values(orc, sub, node, reach)
        e_cr, e_nr = float(np.abs(cr - exact).max()), float(np.abs(nr - exact).max())
        m_cr, m_nr = float(np.abs(cr - exact).mean()), float(np.abs(nr - exact).mean())
        assert e_cr < 0.85 * e_nr and m_cr < 0.65 * m_nr, (node, e_cr, e_nr, m_cr, m_nr)
