"""The batched river workload, restated for the CPU checker (numpy only).

TEST INFRASTRUCTURE ONLY: bench.py's CPU legs use it to build the subgames the
oracle solves without loading the product library, and a CPU test checks that
it draws exactly the subgames mtt-gpu-solver_b200.workloads.river_batch draws
(same generator calls in the same order, the same trees node for node).

* river_tree: the heads-up river betting tree in the reference's FlatNode
  layout (honest_multistreet_solver.cu:16-21), breadth-first with contiguous
  children, every amount rounded to float32 after each operation as the C
  builder computes it.  Action order at a decision node: [fold] [check|call]
  bets or raises by amount ascending, all-in last; amounts within 1e-5 of the
  stack are all-in; equal amounts are offered once.
* river_batch: the batched uneven river configuration (4,096 subgames by
  default): per subgame a seeded 5-card board, 1-4 bet sizes from U[25%,
  200%] pot, raise cap 1-3, pot U[20, 200], SPR U[0.5, 12], and for each
  player a support of 200-1,081 live combos with lognormal(0, 1) weights.
"""
from collections import deque

import numpy as np

NODE_DTYPE = np.dtype([
    ("type", "u1"), ("player", "u1"), ("num_actions", "u1"), ("active_mask", "u1"),
    ("children_offset", "<i4"), ("infoset_offset", "<i4"), ("turn_idx", "<i2"), ("depth", "<i2"),
    ("pot_size", "<f4"), ("committed", "<f4", (2,)), ("reserved", "<f4"),
])
DECISION, FOLD, SHOWDOWN = 0, 1, 2
F32 = np.float32
ALLIN_TOL = F32(1e-5)

_CC = [(a, b) for a in range(52) for b in range(a + 1, 52)]


def live_combos(board):
    bm = 0
    for c in board:
        bm |= 1 << int(c)
    return np.array([i for i, (a, b) in enumerate(_CC) if not ((bm >> a) & 1 or (bm >> b) & 1)], dtype=np.uint16)


def _reaches(amount, rem):
    return amount >= F32(rem * F32(F32(1.0) - ALLIN_TOL))


def river_tree(pot, stack, bet_sizes, raise_cap=1, allin=True):
    """(nodes, (rows0, rows1)) of a river subgame: both players start with
    half of `pot` committed and `stack` behind; raises reuse the bet sizes."""
    pot, stack = F32(pot), F32(stack)
    sizes = [F32(b) for b in bet_sizes]
    nodes = []

    def make(depth):
        nodes.append({"type": 0, "player": 0, "num_actions": 0, "active_mask": 0, "children_offset": 0,
                      "infoset_offset": 0, "turn_idx": -1, "depth": depth, "pot_size": F32(0),
                      "committed": [F32(0), F32(0)]})
        return len(nodes) - 1

    rows = [0, 0]
    half = F32(F32(0.5) * pot)
    q = deque([(make(0), {"c": [half, half], "rem": [stack, stack], "to_act": 0, "raises": 0, "bet_open": False})])
    while q:
        me, s = q.popleft()
        nd = nodes[me]
        nd["pot_size"] = F32(s["c"][0] + s["c"][1])
        nd["committed"] = [s["c"][0], s["c"][1]]
        p = s["to_act"]
        o = 1 - p
        to_call = F32(s["c"][o] - s["c"][p])
        rem_p, rem_o = s["rem"][p], s["rem"][o]
        tot = F32(s["c"][0] + s["c"][1])
        acts = []
        if to_call > 0:
            acts += [(0, F32(0)), (1, to_call)]
            if s["raises"] < raise_cap and not _reaches(to_call, rem_p) and rem_o > 0:
                amts = []
                for r in sizes:
                    a = F32(to_call + F32(r * F32(tot + to_call)))
                    amts.append(rem_p if _reaches(a, rem_p) else a)
                if allin:
                    amts.append(rem_p)
                acts += [(2, a) for a in sorted(set(amts))]
        else:
            acts.append((1, F32(0)))
            if rem_p > 0:
                amts = []
                for b in sizes:
                    a = F32(b * tot)
                    amts.append(rem_p if _reaches(a, rem_p) else a)
                if allin:
                    amts.append(rem_p)
                acts += [(2, a) for a in sorted(set(amts))]
        nd.update(type=DECISION, player=p, num_actions=len(acts), infoset_offset=rows[p])
        rows[p] += len(acts)
        first = len(nodes)
        nd["children_offset"] = first
        for _ in acts:
            make(nd["depth"] + 1)
        for k, (kind, amount) in enumerate(acts):
            ch = nodes[first + k]
            if kind == 0:
                ch.update(type=FOLD, player=p, active_mask=1 << o, pot_size=tot, committed=list(s["c"]))
                continue
            ns = {"c": list(s["c"]), "rem": list(s["rem"]), "to_act": s["to_act"], "raises": s["raises"],
                  "bet_open": s["bet_open"]}
            closes = False
            if kind == 1:
                if to_call > 0:
                    ns["c"][p] = s["c"][o]
                    ns["rem"][p] = F32(0) if _reaches(to_call, rem_p) else F32(rem_p - to_call)
                    closes = True
                elif p == 1:
                    closes = True
                else:
                    ns["to_act"] = o
            else:
                ns["c"][p] = F32(s["c"][p] + amount)
                ns["rem"][p] = F32(0) if amount == rem_p else F32(rem_p - amount)
                if s["bet_open"]:
                    ns["raises"] += 1
                ns["bet_open"] = True
                ns["to_act"] = o
            if not closes:
                q.append((first + k, ns))
                continue
            ch.update(type=SHOWDOWN, active_mask=3, pot_size=F32(ns["c"][0] + ns["c"][1]), committed=list(ns["c"]))
    out = np.zeros(len(nodes), NODE_DTYPE)
    for i, nd in enumerate(nodes):
        for k in ("type", "player", "num_actions", "active_mask", "children_offset", "infoset_offset", "turn_idx",
                  "depth", "pot_size"):
            out[i][k] = nd[k]
        out[i]["committed"] = nd["committed"]
    return out, (rows[0], rows[1])


def river_batch(n=4096, seed=2, min_support=200, max_support=1081, max_sizes=4):
    """The batched uneven river subgames, drawn as the product's generator
    draws them (numpy PCG64, the same calls in the same order)."""
    rng = np.random.default_rng(seed)
    cache = {}
    subs = []
    for _ in range(n):
        board = [int(c) for c in rng.choice(52, size=5, replace=False)]
        live = live_combos(board)
        nsz = int(rng.integers(1, max_sizes + 1))
        sizes = np.sort(rng.uniform(0.25, 2.0, size=nsz)).round(3)
        cap = int(rng.integers(1, 4))
        pot = float(np.round(rng.uniform(20.0, 200.0), 1))
        spr = float(np.round(rng.uniform(0.5, 12.0), 2))
        stack = float(np.round(pot * spr, 1))
        key = (pot, stack, tuple(float(s) for s in sizes), cap)
        if key not in cache:
            cache[key] = river_tree(pot, stack, sizes, raise_cap=cap)
        nodes, rows = cache[key]
        g = {"nodes": nodes, "rows": rows, "board": board, "pot": pot}
        for p in (0, 1):
            k = int(rng.integers(min_support, min(max_support, len(live)) + 1))
            sup = np.sort(rng.choice(live, size=k, replace=False)).astype(np.uint16)
            w = rng.lognormal(0.0, 1.0, size=k).astype(np.float32)
            g[f"combos{p}"] = sup
            g[f"range{p}"] = w
        subs.append(g)
    return subs
