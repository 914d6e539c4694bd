"""Per-hand parity with the oracle at the benchmarked sizes.

The other solver tests compare with the oracle on 24-120 hands.  The kernels
have size-dependent paths those cases never reach: scan chunks of 13 positions
(3 H up to 3,328 with 256 threads) on river boards and 15 on turn boards, the
power-of-two fixed-point scale of large opponent masses, 256-hand warp items,
shared-memory plans of the largest tables and 16-terminal groups.  Here the
batched solver and the oracle (orc_cfr_solve + orc_best_response, dense
O(H^2) FP64 showdowns) run the same seeded inputs at full size:

  * the plain river subgame: uniform ranges over all 1,081 live combos, pot
    100, stack 200, bets {50%, 100%} + all-in, one raise;
  * two batched uneven subgames with 1,081-combo supports on both sides,
    lognormal(0, 1) weights, 3 and 4 bet sizes from U[25%, 200%] and raise
    cap 3 (the largest trees of the batched configuration);
  * a turn subgame with all 1,128 live combos and Dirichlet(0.3) weights, one
    bet size, the river dealt as a chance layer;
  * the four-player ICM river over all 1,081 live combos.

Both semantics run: MTT_SEM_CORRECT and the reference's
(honest_multistreet_solver.cu:88-249, multiway_4way_engine.cu:41-257), which
tests/golden/ref_hu_river.npz and ref_mw_river.npz pin to the reference's own
kernels at 700 and 400 combos.

Tolerances (the solver tests' own):
  * counterfactual values within 1e-4 of pot x opponent mass (heads-up) or of
    the pot (four players, normalised ranges);
  * regrets and strategy sums within 1e-4 of their largest entry;
  * the FP64 best response of the GPU's strategy sums within 1e-9 (relative
    and absolute) of the oracle's best response on the same sums.
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _compare_hu(sub, o, g):
    for key in ("R0", "R1", "S0", "S1"):
        a, b = o[key], g[key]
        scale = max(1e-12, float(np.abs(a).max()))
        d = float(np.abs(a - b).max())
        assert d <= TOL * scale, (key, d, scale)
    for q in (0, 1):
        mass = float(np.sum(sub[f"range{1 - q}"]))
        d = float(np.abs(o[f"cfv{q}"] - g[f"cfv{q}"]).max())
        assert d <= TOL * sub["pot"] * mass, (q, d, sub["pot"] * mass)


def _solve_batch(mtt, subs, sched, **kw):
    b = mtt.RiverBatch(subs)
    b.set_schedule(*sched)
    b.solve(mtt.solve_params(**kw))
    res = b.results()
    reads = [b.read(i) for i in range(len(subs))]
    b.close()
    return res, reads


def _uneven_full_support(mtt, wl, seed):
    """Two batched-configuration subgames forced to 1,081-combo supports:
    3 and 4 bet sizes, raise cap 3, pot and SPR drawn as the workload does."""
    rng = np.random.default_rng(seed)
    subs = []
    for nsz in (3, 4):
        board = wl.draw_board(rng)
        live = mtt.live_combos(board)
        assert len(live) == 1081
        sizes = np.sort(rng.uniform(0.25, 2.0, size=nsz)).round(3)
        pot = float(np.round(rng.uniform(20.0, 200.0), 1))
        spr = float(np.round(rng.uniform(4.0, 12.0), 2))      # deep enough for every raise level
        nodes, rows, _ = mtt.build_tree(pot, float(np.round(pot * spr, 1)), list(sizes), raise_cap=3)
        g = {"nodes": nodes, "rows": rows, "board": board, "pot": pot}
        for p in (0, 1):
            g[f"combos{p}"] = live.copy()
            g[f"range{p}"] = rng.lognormal(0.0, 1.0, size=len(live)).astype(np.float32)
        subs.append(g)
    return subs


SCHEDULES = [(128, 128, 16), (256, 256, 16)]   # (CTA threads, hands per warp item, terminals per CTA)


@pytest.mark.parametrize("sched", SCHEDULES)
@pytest.mark.parametrize("sem,alternate", [(0, 1), (1, 0)])
@pytest.mark.parametrize("iters", [1, 4])
def test_river_uniform_1081_vs_oracle(mtt, wl, orc, cuda, iters, sem, alternate, sched):
    sub = wl.river_uniform(seed=0)
    assert len(sub["combos0"]) == 1081
    res, reads = _solve_batch(mtt, [sub], sched, iters=iters, semantics=sem, alternate=alternate,
                              avg_power=2.0 if alternate else 1.0, threads=sched[0])
    o = orc.cfr_solve(sub, iters, semantics=sem, alternate=alternate, avg_power=2.0 if alternate else 1.0)
    _compare_hu(sub, o, reads[0])
    br = orc.best_response(sub, reads[0]["S0"], reads[0]["S1"])
    assert np.allclose(res[0], br, rtol=1e-9, atol=1e-9), (res[0], br)


@pytest.mark.parametrize("sched", SCHEDULES)
@pytest.mark.parametrize("sem", [0, 1])
@pytest.mark.parametrize("iters", [1, 4])
def test_uneven_batch_full_supports_vs_oracle(mtt, wl, orc, cuda, iters, sem, sched):
    subs = _uneven_full_support(mtt, wl, seed=20)
    assert max(len(g["nodes"]) for g in subs) > 800
    res, reads = _solve_batch(mtt, subs, sched, iters=iters, semantics=sem, alternate=1, avg_power=2.0,
                              threads=sched[0])
    for i, g in enumerate(subs):
        o = orc.cfr_solve(g, iters, semantics=sem, alternate=1, avg_power=2.0)
        _compare_hu(g, o, reads[i])
        br = orc.best_response(g, reads[i]["S0"], reads[i]["S1"])
        assert np.allclose(res[i], br, rtol=1e-9, atol=1e-9), (i, res[i], br)


@pytest.mark.parametrize("sem", [0, 1])
@pytest.mark.parametrize("iters", [1, 2])
def test_turn_full_range_vs_oracle(mtt, orc, cuda, iters, sem):
    rng = np.random.default_rng(33)
    board = [int(c) for c in rng.choice(52, size=4, replace=False)]
    nodes, rows, _ = mtt.build_tree(60.0, 120.0, [0.75], raise_cap=1, street=4, board=board)
    live = mtt.live_combos(board)
    assert len(live) == 1128
    sub = {"nodes": nodes, "rows": rows, "board": board, "pot": 60.0}
    for p in (0, 1):
        w = rng.dirichlet(np.full(1326, 0.3))[live.astype(np.int64)]
        sub[f"combos{p}"] = live.copy()
        sub[f"range{p}"] = (w / w.sum()).astype(np.float32)
    res, reads = _solve_batch(mtt, [sub], (256, 256, 16), iters=iters, semantics=sem, alternate=1, avg_power=2.0,
                              threads=256)
    o = orc.cfr_solve(sub, iters, semantics=sem, alternate=1, avg_power=2.0)
    _compare_hu(sub, o, reads[0])
    br = orc.best_response(sub, reads[0]["S0"], reads[0]["S1"])
    assert np.allclose(res[0], br, rtol=1e-8, atol=1e-9), (res[0], br)


@pytest.mark.parametrize("sem", [0, 1])
@pytest.mark.parametrize("iters", [1, 4])
def test_multiway_icm_1081_vs_oracle(mtt, wl, orc, cuda, iters, sem):
    mw = importlib.import_module("mtt-gpu-solver_b200.multiway")
    sub = wl.multiway_icm(seed=4)
    assert len(sub["combos"]) == 1081
    b = mw.MultiwayBatch([sub])
    b.solve(mtt.solve_params(iters=iters, semantics=sem))
    g = b.read(0)
    vals = b.values()[0]
    b.close()
    o = orc.mw_solve(sub, iters, semantics=sem)
    for p in range(4):
        for k in ("R", "S"):
            a, c = o[k][p], g[k][p]
            scale = max(1e-12, float(np.abs(a).max()))
            assert np.abs(a - c).max() <= TOL * scale, (k, p)
    assert np.abs(o["cfv"] - g["cfv"]).max() <= TOL * sub["pot"]
    assert np.allclose(vals, o["values"], atol=TOL * sub["pot"])
