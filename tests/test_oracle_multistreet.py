"""The oracle's nested chance layers (flop subgames: 49 turn cards, then the
river run out), on the CPU: properties the exact game has.  A flop subgame
whose every turn and river card is dealt must agree with the same game
written as a sum over boards, and its FP64 best response must bound the
average strategies' values."""
import numpy as np


def _flop_sub(wl):
    return wl.flop_runout(seed=8, n_hands=24, stack=100.0, bet_sizes=(1.0,), raise_cap=0)


def test_flop_best_response_bounds_values_and_zero_sum(wl, orc):
    sub = _flop_sub(wl)
    o = orc.cfr_solve(sub, 20, alternate=1, avg_power=2.0)
    br0, br1, ev0, ev1, z, expl = orc.best_response(sub, o["S0"], o["S1"])
    assert br0 >= ev0 - 1e-9 and br1 >= ev1 - 1e-9
    assert abs(ev0 + ev1) <= 1e-9 * sub["pot"] * max(z, 1.0)     # the correct game is zero-sum
    assert expl >= 0.0


def test_flop_exploitability_falls_with_iterations(wl, orc):
    sub = _flop_sub(wl)
    e = []
    for iters in (2, 40):
        o = orc.cfr_solve(sub, iters, alternate=1, avg_power=2.0)
        e.append(orc.best_response(sub, o["S0"], o["S1"])[5])
    assert e[1] < 0.5 * e[0], e


def test_flop_check_down_equals_the_mean_over_runouts(mtt, wl, orc):
    """A flop tree with no chips behind: both players check, the turn and the
    river are dealt, and the hands show down.  Its root values must be the
    showdown values averaged over every (turn, river) runout that avoids both
    hands, computed here pair by pair from the oracle's evaluator."""
    sub = _flop_sub(wl)
    nodes, rows, _ = mtt.build_tree(100.0, 0.0, [1.0], raise_cap=0, allin=False, street=3, board=sub["board"])
    g = dict(sub, nodes=nodes, rows=rows)
    o = orc.cfr_solve(g, 1, alternate=0)
    board = [int(c) for c in g["board"]]
    cards = np.array([(a, c) for a in range(52) for c in range(a + 1, 52)], np.int64)
    c0, c1 = cards[g["combos0"].astype(np.int64)], cards[g["combos1"].astype(np.int64)]
    r1 = g["range1"].astype(np.float64)
    deck = [c for c in range(52) if c not in board]
    want = np.zeros(len(c0))
    for i, h in enumerate(c0):
        for j, v in enumerate(c1):
            if set(h) & set(v):
                continue
            rest = [c for c in deck if c not in h and c not in v]
            runs = np.array([(t, r) for t in rest for r in rest if r != t], np.uint8)
            base = np.tile(np.array(board, np.uint8), (len(runs), 1))
            s0 = orc.eval7(np.concatenate([base, runs, np.tile(np.array(h, np.uint8), (len(runs), 1))], axis=1))
            s1 = orc.eval7(np.concatenate([base, runs, np.tile(np.array(v, np.uint8), (len(runs), 1))], axis=1))
            want[i] += r1[j] * float(np.mean(np.where(s0 > s1, 50.0, np.where(s0 < s1, -50.0, 0.0))))
    assert np.allclose(o["cfv0"], want, rtol=1e-5, atol=1e-4)
