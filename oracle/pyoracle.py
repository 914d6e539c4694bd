"""ctypes binding of the CPU oracle (oracle/libmtt_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU legs of bench.py, as the checker and the timed CPU baseline.  The product
(libmtt_b200.so and the mtt-gpu-solver_b200 package) never imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmtt_oracle.so")
_lib = None


def build():
    r = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return LIB_PATH


class Game(ctypes.Structure):
    _fields_ = [("nodes", ctypes.c_void_p), ("n_nodes", ctypes.c_int32), ("rows", ctypes.c_int32 * 2),
                ("board", ctypes.c_void_p), ("nboard", ctypes.c_int32), ("H", ctypes.c_int32 * 2),
                ("cards", ctypes.c_void_p * 2), ("range", ctypes.c_void_p * 2)]


class CfrParams(ctypes.Structure):
    _fields_ = [("iters", ctypes.c_int32), ("algo", ctypes.c_int32), ("alpha", ctypes.c_float),
                ("beta", ctypes.c_float), ("gamma", ctypes.c_float), ("semantics", ctypes.c_int32),
                ("alternate", ctypes.c_int32), ("avg_power", ctypes.c_float)]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.orc_score7.argtypes = [vp]; L.orc_score7.restype = ctypes.c_uint32
        L.orc_eval7_batch.argtypes = [vp, vp, ctypes.c_int64]
        L.orc_enumerate7.argtypes = [vp, vp]
        L.orc_gen_flops.argtypes = [vp]; L.orc_gen_flops.restype = ctypes.c_int
        L.orc_canonical_class.argtypes = [ctypes.c_int, ctypes.c_int]; L.orc_canonical_class.restype = ctypes.c_int
        L.orc_flop_ev.argtypes = [vp, vp, vp, vp, vp]
        L.orc_ev_dump.argtypes = [ctypes.c_int, ctypes.c_int, vp]
        L.orc_board_counts.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, vp, vp, vp]
        L.orc_cfr_solve.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp]; L.orc_cfr_solve.restype = ctypes.c_int
        L.orc_best_response.argtypes = [vp, vp, vp, vp]; L.orc_best_response.restype = ctypes.c_int
        L.orc_strategy_values.argtypes = [vp, vp, vp, vp, vp, vp]; L.orc_strategy_values.restype = ctypes.c_int
        L.orc_softmax_ev.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp]; L.orc_softmax_ev.restype = ctypes.c_int
        _lib = L
    return _lib


def eval7(cards7):
    c = np.ascontiguousarray(cards7, dtype=np.uint8)
    out = np.zeros(len(c), dtype=np.uint32)
    lib().orc_eval7_batch(c.ctypes.data, out.ctypes.data, len(c))
    return out


def enumerate7():
    hist = np.zeros(9, dtype=np.uint64)
    cs = ctypes.c_uint64()
    lib().orc_enumerate7(hist.ctypes.data, ctypes.byref(cs))
    return hist, cs.value


def gen_flops():
    out = np.zeros(1755 * 4, dtype=np.uint8)
    n = lib().orc_gen_flops(out.ctypes.data)
    return out.reshape(-1, 4)[:n]


def flop_ev(flop3, reach0=None, reach1=None):
    f = np.ascontiguousarray(flop3, dtype=np.uint8)
    e0 = np.zeros(1176, np.float32); e1 = np.zeros(1176, np.float32)
    r0 = np.ascontiguousarray(reach0, np.float32) if reach0 is not None else None
    r1 = np.ascontiguousarray(reach1, np.float32) if reach1 is not None else None
    lib().orc_flop_ev(f.ctypes.data, r0.ctypes.data if r0 is not None else None,
                      r1.ctypes.data if r1 is not None else None, e0.ctypes.data, e1.ctypes.data)
    return e0, e1


def ev_dump(f_begin, f_end):
    out = np.zeros((f_end - f_begin, 4, 2, 169), np.float32)
    lib().orc_ev_dump(f_begin, f_end, out.ctypes.data)
    return out


def board_counts(board, hands):
    b = np.ascontiguousarray(board, np.uint8)
    h = np.ascontiguousarray(hands, np.uint8)
    H = len(h)
    W = np.zeros((H, H), np.int32); T = np.zeros((H, H), np.int32); L = np.zeros((H, H), np.int32)
    lib().orc_board_counts(b.ctypes.data, len(b), h.ctypes.data, H, W.ctypes.data, T.ctypes.data, L.ctypes.data)
    return W, T, L


class _GameHolder:
    def __init__(self, sub):
        from numpy.lib import recfunctions  # noqa: F401  (numpy only)
        self.nodes = np.ascontiguousarray(sub["nodes"])
        self.board = np.ascontiguousarray(np.asarray(sub["board"], np.uint8))
        self.cards = [np.ascontiguousarray(_combo_cards(sub[f"combos{p}"])) for p in (0, 1)]
        self.range = [np.ascontiguousarray(sub[f"range{p}"], np.float32) for p in (0, 1)]
        g = Game()
        g.nodes = self.nodes.ctypes.data
        g.n_nodes = len(self.nodes)
        g.rows[0], g.rows[1] = int(sub["rows"][0]), int(sub["rows"][1])
        g.board = self.board.ctypes.data
        g.nboard = len(self.board)
        g.H[0], g.H[1] = len(self.range[0]), len(self.range[1])
        g.cards[0], g.cards[1] = self.cards[0].ctypes.data, self.cards[1].ctypes.data
        g.range[0], g.range[1] = self.range[0].ctypes.data, self.range[1].ctypes.data
        self.g = g
        self.rows = (g.rows[0], g.rows[1])
        self.H = (g.H[0], g.H[1])


_CC = np.array([(a, b) for a in range(52) for b in range(a + 1, 52)], dtype=np.uint8)


def _combo_cards(ids):
    return _CC[np.asarray(ids, dtype=np.int64)]


def cfr_solve(sub, iters, algo=0, alpha=1.5, beta=0.0, gamma=2.0, semantics=0, alternate=0, avg_power=1.0):
    gh = _GameHolder(sub)
    p = CfrParams(int(iters), int(algo), float(alpha), float(beta), float(gamma), int(semantics), int(alternate),
                  float(avg_power))
    R0 = np.zeros((gh.rows[0], gh.H[0]), np.float32); R1 = np.zeros((gh.rows[1], gh.H[1]), np.float32)
    S0 = np.zeros_like(R0); S1 = np.zeros_like(R1)
    c0 = np.zeros(gh.H[0], np.float32); c1 = np.zeros(gh.H[1], np.float32)
    st = lib().orc_cfr_solve(ctypes.byref(gh.g), ctypes.byref(p), R0.ctypes.data, R1.ctypes.data, S0.ctypes.data,
                             S1.ctypes.data, c0.ctypes.data, c1.ctypes.data)
    if st:
        raise RuntimeError(f"orc_cfr_solve status {st}")
    return {"R0": R0, "R1": R1, "S0": S0, "S1": S1, "cfv0": c0, "cfv1": c1}


def best_response(sub, S0, S1):
    gh = _GameHolder(sub)
    out = np.zeros(6, np.float64)
    s0 = np.ascontiguousarray(S0, np.float32); s1 = np.ascontiguousarray(S1, np.float32)
    st = lib().orc_best_response(ctypes.byref(gh.g), s0.ctypes.data, s1.ctypes.data, out.ctypes.data)
    if st:
        raise RuntimeError(f"orc_best_response status {st}")
    return out


def strategy_values(sub, sigma0, sigma1):
    gh = _GameHolder(sub)
    s0 = np.ascontiguousarray(sigma0, np.float32); s1 = np.ascontiguousarray(sigma1, np.float32)
    c0 = np.zeros(gh.H[0], np.float64); c1 = np.zeros(gh.H[1], np.float64)
    ev = ctypes.c_double()
    st = lib().orc_strategy_values(ctypes.byref(gh.g), s0.ctypes.data, s1.ctypes.data, c0.ctypes.data,
                                   c1.ctypes.data, ctypes.byref(ev))
    if st:
        raise RuntimeError(f"orc_strategy_values status {st}")
    return c0, c1, ev.value


def softmax_ev(sub, logits0, logits1, range0=None, range1=None):
    """EV0 (chips) and root CFVs when both players play softmax(logits_p)
    ([rows_p][H_p] float64), FP64 throughout."""
    gh = _GameHolder(sub)
    l0 = np.ascontiguousarray(logits0, np.float64); l1 = np.ascontiguousarray(logits1, np.float64)
    r0 = np.ascontiguousarray(sub["range0"] if range0 is None else range0, np.float64)
    r1 = np.ascontiguousarray(sub["range1"] if range1 is None else range1, np.float64)
    c0 = np.zeros(gh.H[0], np.float64); c1 = np.zeros(gh.H[1], np.float64)
    ev = ctypes.c_double()
    st = lib().orc_softmax_ev(ctypes.byref(gh.g), l0.ctypes.data, l1.ctypes.data, r0.ctypes.data, r1.ctypes.data,
                              ctypes.byref(ev), c0.ctypes.data, c1.ctypes.data)
    if st:
        raise RuntimeError(f"orc_softmax_ev status {st}")
    return ev.value, c0, c1


vp = ctypes.c_void_p


class MwGame(ctypes.Structure):
    _fields_ = [("nodes", ctypes.c_void_p), ("n_nodes", ctypes.c_int32), ("rows", ctypes.c_int32 * 4),
                ("board", ctypes.c_void_p), ("H", ctypes.c_int32), ("cards", ctypes.c_void_p),
                ("range", ctypes.c_void_p * 4), ("bubble", ctypes.c_float * 16)]


def mw_solve(sub, iters, algo=0, alpha=1.5, beta=0.0, gamma=2.0, semantics=0, avg_power=1.0):
    """Four-player oracle: dict with R, S (lists of [rows_p][H]), cfv [4][H], values [4]."""
    L = lib()
    if not getattr(L, "_mw_sig", False):
        L.orc_mw_solve.argtypes = [vp, vp, vp, vp, vp, vp]; L.orc_mw_solve.restype = ctypes.c_int
        L.orc_icm_equity.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, vp]; L.orc_icm_equity.restype = ctypes.c_int
        L._mw_sig = True
    nodes = np.ascontiguousarray(sub["nodes"])
    board = np.ascontiguousarray(np.asarray(sub["board"], np.uint8))
    cards = np.ascontiguousarray(_combo_cards(sub["combos"]))
    rg = [np.ascontiguousarray(r, np.float32) for r in sub["ranges"]]
    g = MwGame()
    g.nodes = nodes.ctypes.data
    g.n_nodes = len(nodes)
    for p in range(4):
        g.rows[p] = int(sub["rows"][p])
        g.range[p] = rg[p].ctypes.data
    g.board = board.ctypes.data
    g.H = len(cards)
    g.cards = cards.ctypes.data
    bf = np.ones(16) if sub.get("bubble") is None else np.asarray(sub["bubble"], np.float64).reshape(16)
    for k in range(16):
        g.bubble[k] = float(bf[k])
    H = len(cards)
    R = [np.zeros((int(sub["rows"][p]), H), np.float32) for p in range(4)]
    S = [np.zeros((int(sub["rows"][p]), H), np.float32) for p in range(4)]
    cfv = np.zeros((4, H), np.float32)
    vals = np.zeros(4, np.float64)
    pr = (ctypes.c_void_p * 4)(*[R[p].ctypes.data for p in range(4)])
    ps = (ctypes.c_void_p * 4)(*[S[p].ctypes.data for p in range(4)])
    prm = CfrParams(int(iters), int(algo), float(alpha), float(beta), float(gamma), int(semantics), 0,
                    float(avg_power))
    st = L.orc_mw_solve(ctypes.byref(g), ctypes.byref(prm), pr, ps, cfv.ctypes.data, vals.ctypes.data)
    if st:
        raise RuntimeError(f"orc_mw_solve status {st}")
    return {"R": R, "S": S, "cfv": cfv, "values": vals}


def _mw_game(sub):
    nodes = np.ascontiguousarray(sub["nodes"])
    board = np.ascontiguousarray(np.asarray(sub["board"], np.uint8))
    cards = np.ascontiguousarray(_combo_cards(sub["combos"]))
    g = MwGame()
    g.nodes = nodes.ctypes.data
    g.n_nodes = len(nodes)
    for p in range(4):
        g.rows[p] = int(sub["rows"][p])
    g.board = board.ctypes.data
    g.H = len(cards)
    g.cards = cards.ctypes.data
    bf = np.ones(16) if sub.get("bubble") is None else np.asarray(sub["bubble"], np.float64).reshape(16)
    for k in range(16):
        g.bubble[k] = float(bf[k])
    return g, (nodes, board, cards)


def mw_terminal(sub, node, reach, semantics=0, exact=False):
    """Values [4][H] of terminal `node` for per-player reach vectors
    reach[4][H]: the solver's terminal (semantics 0 correct, 1 reference) or,
    with exact=True, the exact showdown over disjoint hands (FP64, small H)."""
    L = lib()
    if not getattr(L, "_mwt_sig", False):
        L.orc_mw_terminal_values.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp]
        L.orc_mw_terminal_values.restype = ctypes.c_int
        L.orc_mw_exact_terminal.argtypes = [vp, ctypes.c_int, vp, vp]
        L.orc_mw_exact_terminal.restype = ctypes.c_int
        L._mwt_sig = True
    g, keep = _mw_game(sub)
    rg = [np.ascontiguousarray(r, np.float32) for r in reach]
    for p in range(4):
        g.range[p] = rg[p].ctypes.data
    pr = (ctypes.c_void_p * 4)(*[r.ctypes.data for r in rg])
    H = g.H
    if exact:
        out = np.zeros((4, H), np.float64)
        st = L.orc_mw_exact_terminal(ctypes.byref(g), int(node), pr, out.ctypes.data)
    else:
        out = np.zeros((4, H), np.float32)
        st = L.orc_mw_terminal_values(ctypes.byref(g), int(node), int(semantics), pr, out.ctypes.data)
    if st:
        raise RuntimeError(f"multiway terminal status {st}")
    return out


def icm_equity(stacks, payouts):
    L = lib()
    L.orc_icm_equity.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, vp]
    L.orc_icm_equity.restype = ctypes.c_int
    st = np.ascontiguousarray(stacks, np.float64)
    pay = np.ascontiguousarray(payouts, np.float64)
    out = np.zeros(len(st), np.float64)
    if L.orc_icm_equity(st.ctypes.data, len(st), pay.ctypes.data, len(pay), out.ctypes.data):
        raise RuntimeError("orc_icm_equity failed")
    return out


class PfParams(ctypes.Structure):
    _fields_ = [("iters", ctypes.c_int32), ("stack_bb", ctypes.c_float), ("bubble", ctypes.c_float),
                ("dead_pot", ctypes.c_float)]


def pf_allin(hc_begin=0, hc_end=169):
    L = lib()
    L.orc_pf_allin_matrix.argtypes = [ctypes.c_int, ctypes.c_int, vp, vp, vp]
    out = np.zeros(169 * 169, np.float32); w = np.zeros(169 * 169, np.int32); t = np.zeros(169 * 169, np.int32)
    L.orc_pf_allin_matrix(hc_begin, hc_end, out.ctypes.data, w.ctypes.data, t.ctypes.data)
    return out.reshape(169, 169), w.reshape(169, 169), t.reshape(169, 169)


def pf_flop_class(flop):
    L = lib()
    L.orc_pf_flop_class_matrix.argtypes = [vp, vp, vp]
    f = np.ascontiguousarray(flop, np.uint8)
    out = np.zeros(169 * 169, np.float32)
    L.orc_pf_flop_class_matrix(f.ctypes.data, out.ctypes.data, None)
    return out.reshape(169, 169)


def pf_dcfr(weights, class_mats, allin, iters=500, stack_bb=20.0, bubble=1.35, dead_pot=2.5):
    L = lib()
    L.orc_pf_dcfr.argtypes = [ctypes.c_int, vp, vp, vp, vp, vp, vp]
    L.orc_pf_dcfr.restype = ctypes.c_int
    w = np.ascontiguousarray(weights, np.float32)
    m = np.ascontiguousarray(class_mats, np.float32)
    a = np.ascontiguousarray(allin, np.float32)
    sums = np.zeros(10 * 192, np.float32); sig = np.zeros(10 * 192, np.float32)
    p = PfParams(int(iters), float(stack_bb), float(bubble), float(dead_pot))
    L.orc_pf_dcfr(len(w), w.ctypes.data, m.ctypes.data, a.ctypes.data, ctypes.byref(p), sums.ctypes.data,
                  sig.ctypes.data)
    return sums.reshape(10, 192), sig.reshape(10, 192)
