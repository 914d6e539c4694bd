"""Depth-limited turn solving: leaf nodes valued per river card inside the
solver's iteration (check-down by the fixed-point showdown scan, plus the
leaf network's correction), measured against the full turn + river solve.

Tolerances (all written here):
  * leaf values with check-down alone against the host aggregation of the
    O(H^2) check-down kernel's values per river card: 1e-5 of the pot per
    unit of opponent reach mass (FP32 sums in different orders);
  * graph replay against direct launches: bit-identical.
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dl():
    return importlib.import_module("mtt-gpu-solver_b200.depthlimit")


def _host_leaf_values(m, ln, spot, g, reach, k, div=44.0):
    """Per-player leaf values at node k from the per-river check-down values."""
    combos = spot["combos"].astype(np.int64)
    H = len(combos)
    cards = np.array([(a, c) for a in range(52) for c in range(a + 1, 52)], np.int64)[combos]
    pot = float(g["nodes"][k]["pot_size"])
    rivers = [c for c in range(52) if c not in spot["board"]]
    meta, M = [], []
    for c in rivers:
        blk = (cards[:, 0] == c) | (cards[:, 1] == c)
        full = []
        for p in range(2):
            f = np.zeros(1326)
            f[combos] = reach[k, p * H:(p + 1) * H].astype(np.float64) * ~blk
            full.append(f)
        M.append([full[0].sum(), full[1].sum()])
        meta.append({"board": list(spot["board"]) + [c], "range0": full[0], "range1": full[1]})
    CD = ln.checkdown_values(meta).astype(np.float64)
    M = np.asarray(M)
    out = []
    for q in range(2):
        v = np.zeros(H)
        for j, c in enumerate(rivers):
            ok = ~((cards[:, 0] == c) | (cards[:, 1] == c))
            v += np.where(ok, M[j, 1 - q] * CD[j, q * 1326 + combos], 0.0)
        out.append(v * pot / div)
    return out, M


@pytest.mark.parametrize("sem,div", [(0, 44.0), (1, 46.0)])
def test_checkdown_leaf_values_match_host_aggregation(mtt, dl, cuda, sem, div):
    ln = importlib.import_module("mtt-gpu-solver_b200.leafnet")
    spot = dl.turn_spot(seed=3)
    g = dl.subgame(spot, True)
    b = mtt.RiverBatch([g])
    b.set_leafnet(None)
    b.solve(mtt.solve_params(iters=1, exploitability=False, alternate=False, semantics=sem), graph=False)
    reach, cfv = b.read_vectors(0, len(g["nodes"]))
    b.close()
    H = len(spot["combos"])
    leaves = np.nonzero(g["nodes"]["type"] == mtt.NODE_LEAF)[0]
    assert len(leaves) == 5
    for k in leaves:
        want, M = _host_leaf_values(mtt, ln, spot, g, reach, k, div)
        pot = float(g["nodes"][k]["pot_size"])
        for q in range(2):
            tol = 1e-5 * pot * max(M[:, 1 - q].max(), 1e-30)
            assert np.abs(cfv[k, q * H:(q + 1) * H] - want[q]).max() <= tol, (k, q)


def test_network_leaves_graph_equals_direct_and_zero_network_is_checkdown(mtt, dl, cuda):
    ln = importlib.import_module("mtt-gpu-solver_b200.leafnet")
    spot = dl.turn_spot(seed=4)
    net = ln.LeafNet(batch_cap=512, seed=3, zero_output=True)   # output layer zero: corrections are 0
    a = dl.solve(spot, True, net=net, iters=40, graph=True)
    b = dl.solve(spot, True, net=net, iters=40, graph=False)
    c = dl.solve(spot, True, net=None, iters=40, graph=True)
    for k in ("cfv0", "cfv1", "strategy0"):
        assert np.array_equal(a[k], b[k]), k
        assert np.array_equal(a[k], c[k]), k
    net.close()


def test_leaf_batch_rejects_unset_leaves_and_best_response(mtt, dl, cuda):
    spot = dl.turn_spot(seed=5)
    b = mtt.RiverBatch([dl.subgame(spot, True)])
    with pytest.raises(mtt.MttError):
        b.solve(mtt.solve_params(iters=2, exploitability=False))      # leaf values undefined
    b.set_leafnet(None)
    with pytest.raises(mtt.MttError):
        b.solve(mtt.solve_params(iters=2, exploitability=True))       # no best response through leaves
    b.close()
    full = mtt.RiverBatch([dl.subgame(spot, False)])
    with pytest.raises(mtt.MttError):
        full.set_leafnet(None)                                         # a batch without leaves
    full.close()


def test_depth_limited_solve_against_the_full_solve(mtt, dl, cuda):
    """The network is trained on leaf samples from full solves of 64 seeded
    spots (the distribution the depth-limited solve queries), then measured
    at the leaves of three held-out spots against their full solve, next to
    check-down leaves, and the depth-limited solves are compared with the
    full solve at the turn root.  The numbers are printed; the assertions
    bound them."""
    import time
    import torch
    X, T, W, meta = dl.leaf_training_set(64, seed=100, iters=300)
    net = dl.train_on(X, T, W, meta, epochs=3)
    leaf = [dl.leaf_errors_in_situ(dl.turn_spot(seed=s), net, iters=300) for s in (0, 1, 2)]
    e_net = float(np.mean([e["net"] for e in leaf]))
    e_cd = float(np.mean([e["checkdown"] for e in leaf]))
    spot = dl.turn_spot(seed=0)
    times, res = {}, {}
    for name, kw in (("full", {"limited": False}), ("net", {"limited": True, "net": net}),
                     ("checkdown", {"limited": True, "net": None})):
        dl.solve(spot, iters=20, **kw)                               # warm-up (graph capture)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res[name] = dl.solve(spot, iters=300, **kw)
        torch.cuda.synchronize()
        times[name] = time.perf_counter() - t0
    err = {k: dl.errors(spot, res[k], res["full"]) for k in ("net", "checkdown")}
    print(f"depth-limited: leaf MAE at the spots' leaves (pot units) net {e_net:.4f} vs check-down {e_cd:.4f}; "
          f"root value error net {err['net']['value']:.4f} check-down {err['checkdown']['value']:.4f}; "
          f"300 iterations full {times['full']:.3f} s, net {times['net']:.3f} s, check-down {times['checkdown']:.3f} s")
    assert e_net < e_cd
    assert err["net"]["value"] < 0.1 and err["checkdown"]["value"] < 0.1
    net.close()
