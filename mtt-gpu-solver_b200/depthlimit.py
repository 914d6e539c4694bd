"""Depth-limited turn solving with the leaf network (no reference counterpart).

A turn subgame is built twice from the same spot:
- full: every turn betting round that closes with chips behind deals the
  river (48 cards) and plays a river round with the same sizes.  This is the
  fallback, and the reference for the depth-limited solve's error.
- depth-limited (river_leaves): those rounds end in a NODE_LEAF.  Its river
  values come from the leaf network, per river card, on both players' current
  reach.  The solver evaluates it inside every pass of every iteration
  (mtt_batch_set_leafnet).

The network is trained on river subgames the batched solver generates, with
the same bet sizes and raise cap as the spot's river rounds.  Their stacks
are the chips behind / pot ratios of the spot's leaves.  The network predicts
the residual over check-down values.  Check-down leaves, i.e. the same solve
with no network, are the method the network is compared with.
"""
import numpy as np

from . import RiverBatch, build_tree, live_combos, solve_params
from . import leafnet as ln
from .workloads import draw_board


def turn_spot(seed=0, pot=100.0, stack=150.0, bet_sizes=(0.5, 1.0), raise_cap=1, alpha=0.3):
    """A heads-up turn spot:
    - a seeded 4-card board;
    - each player's range is Dirichlet(alpha) over the 1,326 combos, with
      board-blocked combos removed;
    - pot, stack, bet sizes (+ all-in) and raise cap shared by both streets."""
    rng = np.random.default_rng(seed)
    board = draw_board(rng, 4)
    live = live_combos(board)
    spot = {"board": board, "pot": float(pot), "stack": float(stack), "bet_sizes": list(bet_sizes),
            "raise_cap": int(raise_cap), "combos": live}
    for p in (0, 1):
        w = rng.dirichlet(np.full(1326, alpha))[live.astype(np.int64)]
        spot[f"range{p}"] = (w / w.sum()).astype(np.float32)
    return spot


def subgame(spot, limited):
    """The spot's turn subgame (dict for RiverBatch): full, or depth-limited."""
    nodes, rows, _ = build_tree(spot["pot"], spot["stack"], spot["bet_sizes"], raise_cap=spot["raise_cap"], street=4,
                                board=spot["board"], river_leaves=limited)
    g = {"nodes": nodes, "rows": rows, "board": spot["board"], "pot": spot["pot"]}
    for p in (0, 1):
        g[f"combos{p}"] = spot["combos"]
        g[f"range{p}"] = spot[f"range{p}"]
    return g


def leaf_sprs(spot):
    """Chips behind / pot at each of the spot's depth-limit leaves (sorted, unique)."""
    from . import NODE_LEAF
    nodes = subgame(spot, True)["nodes"]
    leaf = nodes[nodes["type"] == NODE_LEAF]
    return sorted({round(float(r) / float(pt), 6) for r, pt in zip(leaf["reserved"], leaf["pot_size"])})


def train_leaf_net(sprs, n_train=16384, seed=5, iters=150, epochs=3, lr=1e-4, batch=512, cap=2048, net_seed=1,
                   n_val=0, stream=None):
    """The leaf network, trained as a residual over check-down values on
    n_train solver-generated river subgames (leafnet.river_training_set with
    stacks at `sprs` times the pot).  With n_val > 0, also returns held-out
    mean absolute errors in pot units: {"net": check-down + network,
    "checkdown": check-down alone}."""
    import torch
    X, T, W, meta = ln.river_training_set(n_train + n_val, seed=seed, iters=iters, batch=4096, spr=tuple(sprs),
                                          stream=stream)
    CD = ln.checkdown_values(meta)
    dev = torch.device("cuda")
    put = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    Xt, Rt, Wt = put(X[:n_train]), put(T[:n_train] - CD[:n_train]), put(W[:n_train])
    net = ln.LeafNet(batch_cap=max(cap, ((n_val + 7) // 8) * 8), seed=net_seed, zero_output=True)
    rng = np.random.default_rng(seed + 1)
    for _ in range(epochs):
        perm = torch.from_numpy(rng.permutation(n_train)).to(dev)
        for k in range(0, n_train - batch + 1, batch):
            idx = perm[k:k + batch]
            net.train_step(Xt[idx].contiguous(), Rt[idx].contiguous(), Wt[idx].contiguous(), lr=lr, want_loss=False)
    net.check()
    if n_val <= 0:
        return net
    Xv, Tv, Wv, CDv = X[n_train:], T[n_train:], W[n_train:], CD[n_train:]
    pred = CDv + net.forward(put(Xv)).cpu().numpy()
    live = Wv > 0
    return net, {"net": float(np.abs(pred - Tv)[live].mean()), "checkdown": float(np.abs(CDv - Tv)[live].mean())}


def solve(spot, limited, net=None, residual=True, iters=300, graph=True):
    """Alternating CFR+ (quadratic averaging) on the spot's turn subgame.
    Returns the root counterfactual values of both players (last iterate,
    over the spot's combos) and player 0's average root strategy [actions, H]."""
    g = subgame(spot, limited)
    b = RiverBatch([g])
    if limited:
        b.set_leafnet(net, residual=residual)
    b.solve(solve_params(iters=iters, exploitability=not limited, alternate=True, avg_power=2.0), graph=graph)
    r = b.read(0)
    b.close()
    na = int(g["nodes"][0]["num_actions"])
    s0 = np.asarray(r["S0"][:na], np.float64)
    tot = s0.sum(axis=0, keepdims=True)
    strat = np.where(tot > 0, s0 / np.where(tot > 0, tot, 1.0), 1.0 / na)
    return {"cfv0": np.asarray(r["cfv0"], np.float64), "cfv1": np.asarray(r["cfv1"], np.float64),
            "strategy0": strat}


def errors(spot, approx, full):
    """Depth-limited solve vs the full solve, in pot units:
    - "value": the range-weighted mean absolute difference of both players'
      root values (opponent ranges sum to 1);
    - "strategy": the range-weighted total-variation distance of player 0's
      average root strategy."""
    pot = spot["pot"]
    r0, r1 = spot["range0"].astype(np.float64), spot["range1"].astype(np.float64)
    dv = 0.5 * (float(np.dot(r0, np.abs(approx["cfv0"] - full["cfv0"]))) +
                float(np.dot(r1, np.abs(approx["cfv1"] - full["cfv1"])))) / pot
    ds = float(np.dot(r0, 0.5 * np.abs(approx["strategy0"] - full["strategy0"]).sum(axis=0)))
    return {"value": dv, "strategy": ds}


def leaf_errors_in_situ(spot, net, iters=300, residual=True):
    """The leaf estimates measured at the spot's own leaves against the full
    solve.  The full turn + river subgame is solved (alternating CFR+,
    `iters`).  At every river chance node that closes a turn round with chips
    behind (a depth-limit leaf of the limited tree), both players' final
    reach is taken.  Each player's leaf value is predicted from that reach,
    with the same per-river aggregation the solver's leaf kernels use, by
    check-down alone and by check-down + the network.  Both predictions are
    compared with the full solve's value at that node.
    Returns {"net": e, "checkdown": e}: e is the reach-weighted mean absolute
    error in pot units, with the opponent's reach mass at the leaf scaled to 1."""
    import torch
    from . import NODE_CHANCE, NODE_DECISION
    g = subgame(spot, False)
    nodes = g["nodes"]
    b = RiverBatch([g])
    b.solve(solve_params(iters=iters, exploitability=False, alternate=True, avg_power=2.0), graph=True)
    reach, cfv = b.read_vectors(0, len(nodes))
    b.close()
    board = [int(c) for c in spot["board"]]
    rivers = [c for c in range(52) if c not in board]
    combos = spot["combos"].astype(np.int64)
    H = len(combos)
    cards = np.array([(a, c) for a in range(52) for c in range(a + 1, 52)], np.int64)[combos]
    num = {"net": 0.0, "checkdown": 0.0}
    den = 0.0
    for k in np.nonzero(nodes["type"] == NODE_CHANCE)[0]:
        first = int(nodes[k]["children_offset"])
        if nodes[first]["type"] != NODE_DECISION:
            continue                      # an all-in deal: showdowns follow, no leaf
        pot = float(nodes[k]["pot_size"])
        # chips behind: the stack less what this player added beyond half the starting pot
        spr = (spot["stack"] - (float(nodes[k]["committed"][0]) - spot["pot"] / 2)) / pot
        X, meta, M = [], [], []
        for c in rivers:
            blk = (cards[:, 0] == c) | (cards[:, 1] == c)
            full = []
            for p in range(2):
                r = reach[k, p * H:(p + 1) * H].astype(np.float64) * ~blk
                f = np.zeros(1326)
                f[combos] = r
                full.append(f)
            M.append([full[0].sum(), full[1].sum()])
            X.append(ln.features(board + [c], full[0], full[1], 100.0, 100.0 * spr))
            meta.append({"board": board + [c], "range0": full[0], "range1": full[1]})
        M = np.asarray(M)
        CD = ln.checkdown_values(meta).astype(np.float64)
        Y = net.forward(torch.from_numpy(np.stack(X)).cuda()).cpu().numpy().astype(np.float64)
        est = {"checkdown": CD, "net": CD + Y if residual else Y}
        for q in range(2):
            o = 1 - q
            mass_o = reach[k, o * H:(o + 1) * H].astype(np.float64).sum()
            w = reach[k, q * H:(q + 1) * H].astype(np.float64)
            if mass_o <= 0.0 or w.sum() <= 0.0:
                continue
            truth = cfv[k, q * H:(q + 1) * H].astype(np.float64)
            for name, y in est.items():
                v = np.zeros(H)
                for j, c in enumerate(rivers):
                    ok = ~((cards[:, 0] == c) | (cards[:, 1] == c))
                    v += np.where(ok, M[j, o] * y[j, q * 1326 + combos], 0.0)
                v *= pot / 44.0
                num[name] += float(np.dot(w, np.abs(v - truth))) / (pot * mass_o)
            den += float(w.sum())
    return {name: num[name] / den for name in num}


def leaf_training_set(n_spots, seed=100, iters=300, spot_kw=None):
    """Training samples from the distribution the depth-limited solve queries:
    full turn + river solves of n_spots seeded spots (alternating CFR+,
    `iters`, batched).  Every river root below a leaf-closing chance node
    gives one sample:
    - features: both players' reach there (the river card's combos removed by
      the deal), board and chips behind / pot, as leafnet.features builds them;
    - targets: each player's value there divided by pot x the opponent's reach
      mass (ranges summing to 1);
    - weights: 1 on the spot's combos.
    Returns (X, T, W, meta) like leafnet.river_training_set."""
    from . import NODE_CHANCE, NODE_DECISION
    spot_kw = spot_kw or {}
    spots = [turn_spot(seed=seed + i, **spot_kw) for i in range(n_spots)]
    subs = [subgame(s, False) for s in spots]
    b = RiverBatch(subs)
    b.solve(solve_params(iters=iters, exploitability=False, alternate=True, avg_power=2.0), graph=True)
    X, T, W, meta = [], [], [], []
    for i, (sp, g) in enumerate(zip(spots, subs)):
        nodes = g["nodes"]
        reach, cfv = b.read_vectors(i, len(nodes))
        combos = sp["combos"].astype(np.int64)
        H = len(combos)
        board = [int(c) for c in sp["board"]]
        for k in np.nonzero(nodes["type"] == NODE_CHANCE)[0]:
            first = int(nodes[k]["children_offset"])
            if nodes[first]["type"] != NODE_DECISION:
                continue
            pot = float(nodes[k]["pot_size"])
            spr = (sp["stack"] - (float(nodes[k]["committed"][0]) - sp["pot"] / 2)) / pot
            for a in range(int(nodes[k]["num_actions"])):
                ch = first + a
                c = int(nodes[ch]["turn_idx"])
                full = [np.zeros(1326), np.zeros(1326)]
                t = np.zeros(2652, np.float32)
                w = np.zeros(2652, np.float32)
                mass = [float(reach[ch, p * H:(p + 1) * H].astype(np.float64).sum()) for p in range(2)]
                if min(mass) <= 0.0:
                    continue
                for p in range(2):
                    full[p][combos] = reach[ch, p * H:(p + 1) * H]
                for p in range(2):
                    t[p * 1326 + combos] = cfv[ch, p * H:(p + 1) * H] / (pot * mass[1 - p])
                    w[p * 1326 + combos] = 1.0
                pc = _pairs(combos)
                blk = (pc[:, 0] == c) | (pc[:, 1] == c)     # combos the river card removes
                for p in range(2):
                    w[p * 1326 + combos[blk]] = 0.0
                    t[p * 1326 + combos[blk]] = 0.0
                X.append(ln.features(board + [c], full[0], full[1], 100.0, 100.0 * spr))
                T.append(t)
                W.append(w)
                meta.append({"board": board + [c], "range0": full[0], "range1": full[1]})
    b.close()
    return np.stack(X), np.stack(T), np.stack(W), meta


_PAIRS = np.array([(a, c) for a in range(52) for c in range(a + 1, 52)], np.int64)


def _pairs(combos):
    return _PAIRS[np.asarray(combos, np.int64)]


def train_on(X, T, W, meta, epochs=3, lr=1e-4, batch=512, cap=2048, net_seed=1, seed=7):
    """A residual leaf network trained on (X, T, W, meta) samples."""
    import torch
    CD = ln.checkdown_values(meta)
    dev = torch.device("cuda")
    put = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    n = len(X)
    Xt, Rt, Wt = put(X), put(T - CD), put(W)
    net = ln.LeafNet(batch_cap=cap, seed=net_seed, zero_output=True)
    rng = np.random.default_rng(seed)
    for _ in range(epochs):
        perm = torch.from_numpy(rng.permutation(n)).to(dev)
        for k in range(0, n - batch + 1, batch):
            idx = perm[k:k + batch]
            net.train_step(Xt[idx].contiguous(), Rt[idx].contiguous(), Wt[idx].contiguous(), lr=lr, want_loss=False)
    net.check()
    return net


def _checkdown_rows(boards, r0, r1, stream=None):
    """Check-down values [n, 2652] (pot units, as leafnet.checkdown_values)
    of n rows given as 5-card boards [n, 5] and full 1,326-combo reaches
    [n, 1326] (normalised here over each board's live combos)."""
    import ctypes
    import torch
    from ._lib import check, lib
    n = len(boards)
    out = torch.empty((n, ln.OUT), dtype=torch.float32, device="cuda")
    if n == 0:
        return out.cpu().numpy()
    rs = []
    for r in (r0, r1):
        tot = r.sum(axis=1, keepdims=True)
        rs.append(np.where(tot > 0, r / np.where(tot > 0, tot, 1.0), r).astype(np.float32))
    db = torch.from_numpy(np.ascontiguousarray(boards, np.uint8)).cuda()
    d0, d1 = torch.from_numpy(rs[0]).cuda(), torch.from_numpy(rs[1]).cuda()
    st = None if stream is None else ctypes.c_void_p(stream.cuda_stream)
    check("mtt_checkdown_values", lib().mtt_checkdown_values(
        ctypes.c_void_p(db.data_ptr()), ctypes.c_void_p(d0.data_ptr()), ctypes.c_void_p(d1.data_ptr()), n,
        ctypes.c_void_p(out.data_ptr()), st))
    return out.cpu().numpy()


def leaf_training_data(n_spots, seed=100, iters=300, batch_spots=128, spot_kw=None):
    """leaf_training_set at scale: the same samples (one per river root below
    a leaf-closing chance node of n_spots full turn + river solves), solved
    batch_spots spots at a time and extracted with array operations, with the
    check-down basis computed per batch.  Returns (X [n, 2706], R [n, 2652],
    W [n, 2652]): features, residual targets (target - check-down) and
    weights, float32."""
    from . import NODE_CHANCE, NODE_DECISION
    spot_kw = spot_kw or {}
    Xs, Rs, Ws = [], [], []
    for s0 in range(0, n_spots, batch_spots):
        spots = [turn_spot(seed=seed + i, **spot_kw) for i in range(s0, min(n_spots, s0 + batch_spots))]
        subs = [subgame(s, False) for s in spots]
        b = RiverBatch(subs)
        b.solve(solve_params(iters=iters, exploitability=False, alternate=True, avg_power=2.0), graph=True)
        boards, r0s, r1s, xs, ts, ws = [], [], [], [], [], []
        for i, (sp, g) in enumerate(zip(spots, subs)):
            nodes = g["nodes"]
            reach, cfv = b.read_vectors(i, len(nodes))
            combos = sp["combos"].astype(np.int64)
            H = len(combos)
            board = [int(c) for c in sp["board"]]
            cc = _PAIRS[combos]
            for k in np.nonzero(nodes["type"] == NODE_CHANCE)[0]:
                first = int(nodes[k]["children_offset"])
                if nodes[first]["type"] != NODE_DECISION:
                    continue
                pot = float(nodes[k]["pot_size"])
                spr = (sp["stack"] - (float(nodes[k]["committed"][0]) - sp["pot"] / 2)) / pot
                ch = first + np.arange(int(nodes[k]["num_actions"]))
                cards = nodes[ch]["turn_idx"].astype(np.int64)                        # river card per child
                blk = (cc[None, :, 0] == cards[:, None]) | (cc[None, :, 1] == cards[:, None])   # [R, H]
                rp = [reach[ch, p * H:(p + 1) * H].astype(np.float64) * ~blk for p in range(2)]
                mass = [r.sum(axis=1) for r in rp]
                ok = (mass[0] > 0) & (mass[1] > 0)
                if not ok.any():
                    continue
                R = int(ok.sum())
                x = np.zeros((R, ln.IN), np.float32)
                t = np.zeros((R, ln.OUT), np.float32)
                w = np.zeros((R, ln.OUT), np.float32)
                full = [np.zeros((R, 1326)), np.zeros((R, 1326))]
                for p in range(2):
                    full[p][:, combos] = rp[p][ok]
                    x[:, p * 1326 + combos] = (rp[p][ok] / mass[p][ok, None] * 1081.0).astype(np.float32)
                    v = cfv[ch[ok], p * H:(p + 1) * H].astype(np.float64) / (pot * mass[1 - p][ok, None])
                    t[:, p * 1326 + combos] = np.where(blk[ok], 0.0, v).astype(np.float32)
                    w[:, p * 1326 + combos] = (~blk[ok]).astype(np.float32)
                for c in board:
                    x[:, 2652 + c] = 1.0
                x[np.arange(R), 2652 + cards[ok]] = 1.0
                x[:, 2704] = 1.0
                x[:, 2705] = spr
                bd = np.empty((R, 5), np.uint8)
                bd[:, :4] = board
                bd[:, 4] = cards[ok]
                boards.append(bd)
                r0s.append(full[0])
                r1s.append(full[1])
                xs.append(x)
                ts.append(t)
                ws.append(w)
        b.close()
        if not xs:
            continue
        CD = _checkdown_rows(np.concatenate(boards), np.concatenate(r0s), np.concatenate(r1s))
        Xs.append(np.concatenate(xs))
        Rs.append(np.concatenate(ts) - CD)
        Ws.append(np.concatenate(ws))
    return np.concatenate(Xs), np.concatenate(Rs), np.concatenate(Ws)


def train_residual(X, R, W, epochs=4, lr=1e-4, batch=512, cap=2048, net_seed=1, seed=7):
    """A residual leaf network trained on (features, residual targets,
    weights) rows, as train_on does from leaf_training_set's output."""
    import torch
    dev = torch.device("cuda")
    Xt, Rt, Wt = (torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (X, R, W))
    net = ln.LeafNet(batch_cap=cap, seed=net_seed, zero_output=True)
    rng = np.random.default_rng(seed)
    n = len(X)
    for _ in range(epochs):
        perm = torch.from_numpy(rng.permutation(n)).to(dev)
        for k in range(0, n - batch + 1, batch):
            idx = perm[k:k + batch]
            net.train_step(Xt[idx].contiguous(), Rt[idx].contiguous(), Wt[idx].contiguous(), lr=lr, want_loss=False)
    net.check()
    return net


def evaluate(net, seeds, iters=300):
    """The depth-limited solve against the full turn + river solve on held-out
    spots: per spot, the root value error (pot units, errors()) and the solve
    time (one solve call, as solve() runs it) of network leaves, check-down
    leaves and the full tree, and the leaf MAE at the spot's leaves
    (leaf_errors_in_situ).  Returns a dict of per-spot lists and means."""
    import time
    import torch
    out = {"root_error": {"net": [], "checkdown": []}, "leaf_mae": {"net": [], "checkdown": []},
           "solve_s": {"full": [], "net": [], "checkdown": []}}
    for sd in seeds:
        spot = turn_spot(seed=sd)
        res = {}
        for name, kw in (("full", {"limited": False}), ("net", {"limited": True, "net": net}),
                         ("checkdown", {"limited": True, "net": None})):
            solve(spot, iters=10, **kw)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res[name] = solve(spot, iters=iters, **kw)
            torch.cuda.synchronize()
            out["solve_s"][name].append(time.perf_counter() - t0)
        for name in ("net", "checkdown"):
            out["root_error"][name].append(errors(spot, res[name], res["full"])["value"])
        le = leaf_errors_in_situ(spot, net, iters=iters)
        for name in ("net", "checkdown"):
            out["leaf_mae"][name].append(le[name])
    out["mean"] = {k: {n: float(np.mean(v)) for n, v in d.items()} for k, d in out.items() if k != "mean"}
    return out


if __name__ == "__main__":
    import argparse
    import json
    import time
    import torch
    ap = argparse.ArgumentParser(description="train the leaf network on solver-generated leaf samples and measure "
                                             "depth-limited turn solving against the full solve")
    ap.add_argument("--spots", type=int, default=1024, help="training spots (about 200 samples each)")
    ap.add_argument("--held-out", type=int, default=8)
    ap.add_argument("--epochs", type=int, default=4)
    ap.add_argument("--iters", type=int, default=300)
    a = ap.parse_args()
    t0 = time.perf_counter()
    X, R, W = leaf_training_data(a.spots, seed=100, iters=a.iters)
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    t0 = time.perf_counter()
    net = train_residual(X, R, W, epochs=a.epochs)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    ev = evaluate(net, seeds=list(range(a.held_out)), iters=a.iters)
    print(json.dumps({"train_samples": int(len(X)), "train_spots": a.spots, "data_s": t_data, "train_s": t_train,
                      "epochs": a.epochs, "held_out_spots": a.held_out, **ev}))
    net.close()
