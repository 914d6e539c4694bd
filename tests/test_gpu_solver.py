"""Batched CFR solver on the GPU vs the CPU oracle.

The oracle restates the reference sweeps (honest_multistreet_solver.cu:88-249)
with dense O(H^2) showdowns accumulated in FP64; the GPU uses rank-order
prefix scans in FP32.  Tolerances (all written here):
  * counterfactual values: 1e-4 of the pot per unit of opponent range mass;
  * regrets and strategy sums: 1e-4 relative to the largest entry;
  * the FP64 best response: 1e-9 on identical strategy sums.
Strict comparisons use few iterations: regret matching's uniform fallback
(sum of positive regrets <= 1e-7, honest_multistreet_solver.cu:117) and the
CFR+ clip are discontinuous, so FP32 rounding differences between two valid
summation orders can later pick different branches for indifferent hands.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_POT = 1e-4


def _solve_gpu(mtt, subs, **kw):
    b = mtt.RiverBatch(subs)
    p = mtt.solve_params(**kw)
    b.solve(p)
    res = b.results()
    reads = [b.read(i) for i in range(len(subs))]
    b.close()
    return res, reads


def _compare(sub, orc_out, gpu_out):
    pot = sub["pot"]
    for key in ("R0", "R1", "S0", "S1"):
        a, g = orc_out[key], gpu_out[key]
        scale = max(1e-12, float(np.abs(a).max()))
        assert np.abs(a - g).max() <= 1e-4 * scale, key
    for q in (0, 1):
        mass = float(np.sum(sub[f"range{1 - q}"]))
        d = np.abs(orc_out[f"cfv{q}"] - gpu_out[f"cfv{q}"]).max()
        assert d <= TOL_POT * pot * mass, (q, d, pot * mass)


@pytest.mark.parametrize("alternate", [0, 1])
@pytest.mark.parametrize("algo,sem", [(0, 0), (1, 0), (0, 1), (1, 1)])
@pytest.mark.parametrize("iters", [1, 4])
def test_river_vs_oracle(mtt, wl, orc, cuda, iters, algo, sem, alternate):
    sub = wl.river_uniform(seed=3, n_hands=80)
    res, reads = _solve_gpu(mtt, [sub], iters=iters, algo=algo, semantics=sem, alternate=alternate, threads=128)
    o = orc.cfr_solve(sub, iters, algo=algo, semantics=sem, alternate=alternate)
    _compare(sub, o, reads[0])
    br = orc.best_response(sub, reads[0]["S0"], reads[0]["S1"])
    assert np.allclose(res[0], br, rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("alternate", [0, 1])
def test_uneven_batch_vs_oracle(mtt, wl, orc, cuda, alternate):
    subs = wl.river_batch(n=6, seed=11, min_support=40, max_support=90, max_sizes=3)
    res, reads = _solve_gpu(mtt, subs, iters=3, alternate=alternate, threads=64)
    for i, g in enumerate(subs):
        o = orc.cfr_solve(g, 3, alternate=alternate)
        _compare(g, o, reads[i])
        br = orc.best_response(g, reads[i]["S0"], reads[i]["S1"])
        assert np.allclose(res[i], br, rtol=1e-9, atol=1e-9)


def test_longer_solve_tracks_oracle(mtt, wl, orc, cuda):
    """After 60 alternating CFR+ iterations both sides agree on exploitability
    and root EV to 1e-4 of the pot."""
    subs = wl.river_batch(n=4, seed=17, min_support=60, max_support=120, max_sizes=2)
    res, reads = _solve_gpu(mtt, subs, iters=60, threads=256)
    for i, g in enumerate(subs):
        o = orc.cfr_solve(g, 60, alternate=1)
        br = orc.best_response(g, o["S0"], o["S1"])
        assert abs(res[i][5] - br[5]) <= 1e-4, (res[i][5], br[5])
        assert abs(res[i][2] - br[2]) <= 1e-4 * g["pot"]


@pytest.mark.parametrize("threads", [64, 256])
def test_results_do_not_depend_on_cta_size(mtt, wl, cuda, threads):
    subs = wl.river_batch(n=3, seed=5, min_support=100, max_support=300)
    base_res, base = _solve_gpu(mtt, subs, iters=20, threads=128)
    res, reads = _solve_gpu(mtt, subs, iters=20, threads=threads)
    for a, b in zip(base, reads):
        for k in a:
            assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(base_res, res)


def test_graph_replay_matches_direct(mtt, wl, cuda):
    import torch
    subs = wl.river_batch(n=4, seed=9, min_support=50, max_support=200)
    b = mtt.RiverBatch(subs)
    p = mtt.solve_params(iters=40, threads=128)
    b.solve(p)
    r1 = b.results(); s1 = b.read(2)
    b.solve(p, graph=True)
    b.solve(p, graph=True)
    torch.cuda.synchronize()
    r2 = b.results(); s2 = b.read(2)
    b.close()
    assert np.array_equal(r1, r2)
    assert np.array_equal(s1["S0"], s2["S0"]) and np.array_equal(s1["R1"], s2["R1"])


@pytest.mark.parametrize("algo,sem,alternate", [(0, 0, 1), (1, 0, 1), (0, 1, 0)])
def test_turn_subgame_with_river_chance_vs_oracle(mtt, orc, cuda, algo, sem, alternate):
    rng = np.random.default_rng(21)
    board = [int(c) for c in rng.choice(52, size=4, replace=False)]
    nodes, rows, _ = mtt.build_tree(60, 100, [0.75], raise_cap=1, street=4, board=board)
    live = mtt.live_combos(board)
    c0 = np.sort(rng.choice(live, size=40, replace=False)).astype(np.uint16)
    c1 = np.sort(rng.choice(live, size=36, replace=False)).astype(np.uint16)
    sub = {"nodes": nodes, "rows": rows, "board": board, "combos0": c0, "combos1": c1,
           "range0": rng.dirichlet(np.full(40, 0.3)).astype(np.float32),
           "range1": rng.dirichlet(np.full(36, 0.3)).astype(np.float32), "pot": 60.0}
    res, reads = _solve_gpu(mtt, [sub], iters=3, algo=algo, semantics=sem, alternate=alternate, threads=128)
    o = orc.cfr_solve(sub, 3, algo=algo, semantics=sem, alternate=alternate)
    _compare(sub, o, reads[0])
    br = orc.best_response(sub, reads[0]["S0"], reads[0]["S1"])
    assert np.allclose(res[0], br, rtol=1e-8, atol=1e-9)


def test_config0_converges_below_0p1_percent(mtt, wl, cuda):
    sub = wl.river_uniform(seed=0)
    res, _ = _solve_gpu(mtt, [sub], iters=1000, threads=256)
    br0, br1, ev0, ev1, Z, expl = res[0]
    assert abs(ev0 + ev1) < 1e-6 * sub["pot"]          # zero-sum
    assert br0 >= ev0 - 1e-9 and br1 >= ev1 - 1e-9      # a best response is at least the average's value
    assert expl <= 1e-3


def test_config2_sample_reaches_the_gate(mtt, wl, cuda):
    """1,000 alternating CFR+ iterations, then subgames above 0.1% of the pot
    continue in 500-iteration chunks until every one passes."""
    subs = wl.river_batch(n=64, seed=2)
    b = mtt.RiverBatch(subs)
    b.solve(mtt.solve_params(iters=1000, threads=256, avg_power=2.0, target_expl=1e-3, max_iters=4000,
                             chunk_iters=500))
    res = b.results()
    its = b.iterations()
    b.close()
    expl = res[:, 5]
    assert np.isfinite(res).all()
    assert (res[:, 0] >= res[:, 2] - 1e-9).all() and (res[:, 1] >= res[:, 3] - 1e-9).all()
    assert (expl <= 1e-3).all(), np.sort(expl)[-5:]
    assert (its >= 1000).all() and (its[expl > 0] <= 4000).all()


def test_continuation_matches_a_longer_solve(mtt, wl, cuda):
    """A subgame continued by the gate ends exactly where an uninterrupted
    solve of the same length ends."""
    subs = wl.river_batch(n=6, seed=4, min_support=80, max_support=200)
    b = mtt.RiverBatch(subs)
    b.solve(mtt.solve_params(iters=40, threads=128, target_expl=1e-9, max_iters=60, chunk_iters=20))
    its = b.iterations()
    cont = [b.read(i) for i in range(len(subs))]
    b.close()
    assert (its == 60).all()
    res, ref = _solve_gpu(mtt, subs, iters=60, threads=128)
    for a_, r_ in zip(cont, ref):
        for k in ("R0", "R1", "S0", "S1"):
            assert np.array_equal(a_[k], r_[k]), k


def test_config1_abstraction_small_ranges_vs_oracle(mtt, wl, orc, cuda):
    """The turn+river tree of the DCFR workload (bets 33/75/150% + all-in,
    2 raises on both streets, 104k nodes) with 24-combo ranges: DCFR
    (1.5, 0, 2) against the oracle."""
    sub = wl.turn_dcfr(seed=1, n_hands=24)
    res, reads = _solve_gpu(mtt, [sub], iters=3, algo=1, alpha=1.5, beta=0.0, gamma=2.0, threads=256)
    o = orc.cfr_solve(sub, 3, algo=1, alpha=1.5, beta=0.0, gamma=2.0, alternate=1)
    _compare(sub, o, reads[0])


def test_config1_full_solve(mtt, wl, cuda):
    """The full turn+river DCFR workload (1,128 live combos per player):
    exploitability falls with the iterations and ends small."""
    sub = wl.turn_dcfr(seed=1)
    b = mtt.RiverBatch([sub])
    b.solve(mtt.solve_params(iters=50, algo=1, alpha=1.5, beta=0.0, gamma=2.0, threads=256), graph=True)
    e50 = b.results()[0, 5]
    b.solve(mtt.solve_params(iters=500, algo=1, alpha=1.5, beta=0.0, gamma=2.0, threads=256), graph=True)
    r = b.results()[0]
    b.close()
    assert np.isfinite(r).all()
    assert r[5] < e50 and r[5] < 5e-3, (e50, r[5])


def test_kernel_profile_reports_each_kernel_class(mtt, wl, cuda):
    subs = wl.river_batch(n=8, seed=21, min_support=60, max_support=200, max_sizes=2)
    b = mtt.RiverBatch(subs)
    p = mtt.solve_params(iters=3, alternate=True, threads=128)
    prof = b.kernel_profile(p, iters=3)
    for k in ("k_fwd", "k_term", "k_bwd"):
        assert prof[k]["ms"] > 0.0 and prof[k]["bytes"] > 0.0, (k, prof[k])
    # the profiled iterations are ordinary ones: a solve afterwards is unaffected
    b.solve(p)
    r1 = b.results()
    b2 = mtt.RiverBatch(subs)
    b2.solve(p)
    assert np.array_equal(r1, b2.results())
    b.close()
    b2.close()


@pytest.mark.parametrize("algo,sem,alternate", [(0, 0, 1), (1, 0, 1), (0, 1, 0), (0, 0, 0)])
def test_flop_subgame_turn_chance_and_river_runout_vs_oracle(mtt, wl, orc, cuda, algo, sem, alternate):
    """Two chance layers (49 turn cards, then 48 river cards run out to
    showdowns): table variants per (turn, river) board and chance divisors
    per node, against the oracle's dense showdowns."""
    sub = wl.flop_runout(seed=8, n_hands=36, stack=100.0, bet_sizes=(1.0,), raise_cap=0)
    kinds = np.bincount(sub["nodes"]["type"], minlength=4)
    assert kinds[3] > 49                     # turn chance nodes and the river chance nodes below them
    res, reads = _solve_gpu(mtt, [sub], iters=3, algo=algo, semantics=sem, alternate=alternate, threads=128)
    o = orc.cfr_solve(sub, 3, algo=algo, semantics=sem, alternate=alternate)
    _compare(sub, o, reads[0])
    br = orc.best_response(sub, reads[0]["S0"], reads[0]["S1"])
    assert np.allclose(res[0], br, rtol=1e-8, atol=1e-9)


def test_flop_subgame_full_ranges_converges(mtt, wl, cuda):
    """Full flop ranges (1,176 live combos), 2 bet sizes + all-in, one raise:
    exploitability falls with iterations, and graph replay equals direct
    launches."""
    sub = wl.flop_runout(seed=9)
    expl = []
    for iters in (20, 200):
        res, _ = _solve_gpu(mtt, [sub], iters=iters, alternate=True, avg_power=2.0)
        assert np.isfinite(res).all()
        expl.append(res[0][5])
    assert expl[1] < 0.5 * expl[0] and expl[1] < 0.02, expl
    b = mtt.RiverBatch([sub])
    p = mtt.solve_params(iters=10, alternate=True)
    b.solve(p, graph=True)
    r1 = b.results()
    b.solve(p, graph=False)
    assert np.array_equal(r1, b.results())
    b.close()


def test_batches_reuse_pool_memory_and_trim(mtt, wl, cuda):
    """A batch created where a destroyed one was (pool memory kept) solves
    the same; trimming returns the memory and later batches still work."""
    subs = wl.river_batch(n=12, seed=31, min_support=60, max_support=300, max_sizes=2)
    p = mtt.solve_params(iters=20, alternate=True, threads=128)
    out = []
    for k in range(3):
        b = mtt.RiverBatch(subs)
        b.solve(p, graph=True)
        out.append(b.results())
        b.close()
        if k == 1:
            mtt.trim_pool()
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[0], out[2])


@pytest.mark.parametrize("hpw,chunk", [(256, 16), (128, 3), (256, 1)])
def test_results_do_not_depend_on_the_schedule(mtt, wl, cuda, hpw, chunk):
    """Hands per sweep warp item and terminals per CTA change only the launch
    shape: every value is bit-identical to the default schedule."""
    subs = wl.river_batch(n=8, seed=41, min_support=150, max_support=700, max_sizes=3)
    p = mtt.solve_params(iters=12, alternate=True, threads=128)
    out = []
    for sched in ((128, 16), (hpw, chunk)):
        b = mtt.RiverBatch(subs)
        b.set_schedule(128, *sched)
        assert b.schedule() == {"threads": 128, "hands_per_warp": sched[0], "term_chunk": sched[1]}
        b.solve(p, graph=True)
        out.append((b.results(), [b.read(i) for i in range(len(subs))]))
        b.close()
    assert np.array_equal(out[0][0], out[1][0])
    for a_, b_ in zip(out[0][1], out[1][1]):
        for k in a_:
            assert np.array_equal(a_[k], b_[k]), k


def test_autotune_picks_a_schedule(mtt, wl, cuda):
    subs = wl.river_batch(n=16, seed=42, min_support=100, max_support=400, max_sizes=2)
    b = mtt.RiverBatch(subs)
    p = mtt.solve_params(iters=10, alternate=True)
    t = b.autotune(p)
    s = b.schedule()
    assert t in (64, 128, 256) and s["threads"] == t
    assert s["hands_per_warp"] in (128, 256) and s["term_chunk"] in (8, 16)
    p.threads = t
    b.solve(p, graph=True)
    r1 = b.results()
    b.set_schedule(128, 128, 16)
    b.solve(p, graph=True)
    assert np.array_equal(r1, b.results())
    b.close()


def test_destroy_waits_for_its_own_solve_and_frees_for_the_next_batch(mtt, wl, cuda):
    """mtt_batch_destroy waits on the streams the batch ran on, not on the
    device: a batch destroyed right after its solve was queued on a
    non-blocking stream must not hand its memory to the next batch while the
    solve still runs.  The next batch (created from the pool right away)
    solves to the same bits as a batch created on a quiet device."""
    import torch
    subs = wl.river_batch(n=64, seed=5, min_support=200, max_support=700)
    p = mtt.solve_params(iters=30, threads=128)
    ref = mtt.RiverBatch(subs[32:])
    ref.solve(p, graph=True)
    want = ref.results()
    want_s = ref.read(3)
    ref.close()
    side = torch.cuda.Stream()
    a = mtt.RiverBatch(subs[:32])
    with torch.cuda.stream(side):
        a.solve(p, stream=side, graph=True)
    a.close()                           # no synchronisation by the caller
    b = mtt.RiverBatch(subs[32:])       # reuses the pool's memory
    b.solve(p, graph=True)
    got = b.results()
    got_s = b.read(3)
    b.close()
    assert np.array_equal(want, got)
    assert np.array_equal(want_s["R0"], got_s["R0"]) and np.array_equal(want_s["S1"], got_s["S1"])
