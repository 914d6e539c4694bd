"""Four-player river solving with ICM loss multipliers (C ABI wrappers).

    mw = importlib.import_module("mtt-gpu-solver_b200.multiway")
    nodes, rows, depth = mw.build_tree(pot=4.0, stacks=[20, 20, 20, 20], bet_sizes=[0.5, 1.0], raise_size=1.0)
    bf = mw.bubble_factors(stacks8, [0.5, 0.3, 0.2], seats=[0, 1, 2, 3])   # FP64 Malmuth-Harville
    batch = mw.MultiwayBatch([{"nodes": nodes, "rows": rows, "board": board, "combos": live,
                               "ranges": [r0, r1, r2, r3], "bubble": bf}])
    batch.solve(params, graph=True); values = batch.values()
"""
import ctypes

import numpy as np

from ._lib import MW_NODE_DTYPE, MwSpec, MwSubgame, check, lib


def _stream(s):
    if s is None:
        return None
    return ctypes.c_void_p(s.cuda_stream if hasattr(s, "cuda_stream") else int(s))


def build_tree(pot, stacks, bet_sizes=(0.5, 1.0), raise_size=1.0, raise_cap=1):
    """4-player single-street tree (MW_NODE_DTYPE array), rows per player, max depth."""
    sp = MwSpec()
    sp.pot = float(pot)
    for p in range(4):
        sp.stacks[p] = float(stacks[p])
    sp.n_bet_sizes = len(bet_sizes)
    for k, b in enumerate(bet_sizes):
        sp.bet_sizes[k] = float(b)
    sp.raise_size = float(raise_size)
    sp.raise_cap = int(raise_cap)
    n = ctypes.c_int32()
    rows = (ctypes.c_int32 * 4)()
    depth = ctypes.c_int32()
    check("mtt_mw_tree_build", lib().mtt_mw_tree_build(ctypes.byref(sp), None, 0, ctypes.byref(n), rows,
                                                       ctypes.byref(depth)))
    nodes = np.zeros(n.value, dtype=MW_NODE_DTYPE)
    check("mtt_mw_tree_build", lib().mtt_mw_tree_build(ctypes.byref(sp), nodes.ctypes.data, n.value,
                                                       ctypes.byref(n), rows, ctypes.byref(depth)))
    return nodes, tuple(int(r) for r in rows), depth.value


def icm_equity(stacks, payouts):
    st = np.ascontiguousarray(stacks, np.float64)
    pay = np.ascontiguousarray(payouts, np.float64)
    out = np.zeros(len(st), np.float64)
    check("mtt_icm_equity", lib().mtt_icm_equity(st.ctypes.data, len(st), pay.ctypes.data, len(pay), out.ctypes.data))
    return out


def bubble_factors(stacks, payouts, seats):
    st = np.ascontiguousarray(stacks, np.float64)
    pay = np.ascontiguousarray(payouts, np.float64)
    se = np.ascontiguousarray(seats, np.int32)
    out = np.zeros(len(se) * len(se), np.float64)
    check("mtt_icm_bubble_factors", lib().mtt_icm_bubble_factors(st.ctypes.data, len(st), pay.ctypes.data, len(pay),
                                                                 se.ctypes.data, len(se), out.ctypes.data))
    return out.reshape(len(se), len(se))


class MultiwayBatch:
    """Four-player river subgames resident on the current CUDA device.

    Each subgame: nodes (MW_NODE_DTYPE), rows (4), board (5 cards), combos
    (ascending ids, shared by the four players), ranges (4 arrays over
    combos), bubble (4x4 loss multipliers, default all ones)."""

    def __init__(self, subgames):
        arr = (MwSubgame * len(subgames))()
        keep = []
        for i, g in enumerate(subgames):
            nodes = np.ascontiguousarray(g["nodes"], dtype=MW_NODE_DTYPE)
            combos = np.ascontiguousarray(g["combos"], dtype=np.uint16)
            rg = [np.ascontiguousarray(r, dtype=np.float32) for r in g["ranges"]]
            keep += [nodes, combos] + rg
            s = arr[i]
            s.nodes = nodes.ctypes.data
            s.n_nodes = len(nodes)
            for p in range(4):
                s.rows[p] = int(g["rows"][p])
                s.ranges[p] = rg[p].ctypes.data
            for k, c in enumerate(g["board"]):
                s.board[k] = int(c)
            s.H = len(combos)
            s.combos = combos.ctypes.data
            bf = np.ones(16) if g.get("bubble") is None else np.asarray(g["bubble"], np.float64).reshape(16)
            for k in range(16):
                s.bubble[k] = float(bf[k])
        self.n = len(subgames)
        self.meta = [(tuple(int(r) for r in g["rows"]), len(g["combos"])) for g in subgames]
        h = ctypes.c_void_p()
        check("mtt_mw_batch_create", lib().mtt_mw_batch_create(arr, self.n, ctypes.byref(h)))
        self._h = h

    def solve(self, params, graph=False, stream=None):
        check("mtt_mw_batch_solve", lib().mtt_mw_batch_solve(self._h, ctypes.byref(params), int(bool(graph)),
                                                             _stream(stream)))

    def values(self, stream=None):
        """[n, 4] EV of each player's range (chips) under the average strategies."""
        out = np.zeros((self.n, 4), np.float64)
        check("mtt_mw_batch_values", lib().mtt_mw_batch_values(self._h, out.ctypes.data, _stream(stream)))
        return out

    def read(self, s):
        rows, H = self.meta[s]
        R = [np.zeros((rows[p], H), np.float32) for p in range(4)]
        S = [np.zeros((rows[p], H), np.float32) for p in range(4)]
        cfv = np.zeros((4, H), np.float32)
        pr = (ctypes.c_void_p * 4)(*[R[p].ctypes.data for p in range(4)])
        ps = (ctypes.c_void_p * 4)(*[S[p].ctypes.data for p in range(4)])
        check("mtt_mw_batch_read", lib().mtt_mw_batch_read(self._h, s, pr, ps, cfv.ctypes.data))
        return {"R": R, "S": S, "cfv": cfv}

    def close(self):
        if getattr(self, "_h", None):
            lib().mtt_mw_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
