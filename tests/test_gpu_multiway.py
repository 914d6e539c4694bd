"""Four-player GPU solver vs the oracle (multiway_4way_engine.cu:41-257).

Tolerances (written here): regrets and strategy sums within 1e-4 of the
largest entry; root counterfactual values within 1e-4 of the pot (ranges are
normalised, so the opponents' mass product is 1); average-strategy values
within 1e-4 of the pot."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mw():
    return importlib.import_module("mtt-gpu-solver_b200.multiway")


def _solve(mw, mtt, sub, iters, graph=False, **kw):
    b = mw.MultiwayBatch([sub])
    b.solve(mtt.solve_params(iters=iters, **kw), graph=graph)
    out = b.read(0)
    out["values"] = b.values()[0]
    b.close()
    return out


@pytest.mark.parametrize("iters", [1, 5])
@pytest.mark.parametrize("algo", [0, 1])
@pytest.mark.parametrize("sem", [0, 1])
def test_multiway_vs_oracle(mw, mtt, wl, orc, cuda, iters, algo, sem):
    sub = wl.multiway_icm(seed=7, n_hands=64)
    g = _solve(mw, mtt, sub, iters, algo=algo, semantics=sem)
    o = orc.mw_solve(sub, iters, algo=algo, semantics=sem)
    for p in range(4):
        for k in ("R", "S"):
            a, b = o[k][p], g[k][p]
            scale = max(1e-12, float(np.abs(a).max()))
            assert np.abs(a - b).max() <= 1e-4 * scale, (k, p)
    assert np.abs(o["cfv"] - g["cfv"]).max() <= 1e-4 * sub["pot"]
    assert np.allclose(g["values"], o["values"], atol=1e-4 * sub["pot"])


def test_multiway_graph_replay_matches_direct(mw, mtt, wl, cuda):
    sub = wl.multiway_icm(seed=8, n_hands=120)
    a = _solve(mw, mtt, sub, 30, graph=False)
    b = _solve(mw, mtt, sub, 30, graph=True)
    for p in range(4):
        assert np.array_equal(a["R"][p], b["R"][p]) and np.array_equal(a["S"][p], b["S"][p])


def test_multiway_batch_of_uneven_subgames(mw, mtt, wl, orc, cuda):
    subs = [wl.multiway_icm(seed=s, n_hands=n) for s, n in ((11, 40), (12, 90), (13, 17))]
    b = mw.MultiwayBatch(subs)
    b.solve(mtt.solve_params(iters=4))
    vals = b.values()
    for i, sub in enumerate(subs):
        g = b.read(i)
        o = orc.mw_solve(sub, 4)
        for p in range(4):
            scale = max(1e-12, float(np.abs(o["R"][p]).max()))
            assert np.abs(o["R"][p] - g["R"][p]).max() <= 1e-4 * scale
        assert np.allclose(vals[i], o["values"], atol=1e-4 * sub["pot"])
    b.close()


def test_config4_full_range_solve(mw, mtt, wl, cuda):
    """The four-player ICM river at full size (1,081 live combos, 1,585 nodes),
    200 iterations: finite values, and regret matching moved away from uniform."""
    sub = wl.multiway_icm(seed=4)
    assert len(sub["nodes"]) == 1585 and len(sub["combos"]) == 1081
    g = _solve(mw, mtt, sub, 200, graph=True)
    assert np.isfinite(g["values"]).all()
    assert all(np.isfinite(s).all() and (s >= 0).all() for s in g["S"])
    assert max(float(s.max()) for s in g["S"]) > 0
