"""mtt-gpu-solver_b200 — B200 (sm_100a) rebuild of MTT-GPU-Solver's hot path.

Python mirror of the C ABI in include/mtt_b200.h.  Device buffers are torch
CUDA tensors; every call goes through libmtt_b200.so and raises MttError on a
non-zero status.  Import with importlib (the folder name has hyphens):

    mtt = importlib.import_module("mtt-gpu-solver_b200")
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import (ALGO_CFRPLUS, ALGO_DCFR, NODE_CHANCE, NODE_DECISION, NODE_DTYPE, NODE_FOLD, NODE_LEAF,
                   NODE_SHOWDOWN, SEM_CORRECT, SEM_REFERENCE, MttError, SolveParams, Subgame, TreeSpec,
                   check, lib)

__all__ = ["lib", "MttError", "NODE_DTYPE", "combo_id", "combo_cards", "live_combos", "build_tree",
           "eval7", "eval7_enumerate", "board_showdown_counts", "canonical_flops", "flop_ev", "ev_dump",
           "RiverBatch", "SolveParams"]


# ------------------------------------------------------------------ cards
def combo_id(c1, c2):
    """Lexicographic id (0..1325) of the unordered pair c1 != c2."""
    if c1 > c2:
        c1, c2 = c2, c1
    return c1 * 51 - (c1 * (c1 - 1)) // 2 + (c2 - c1 - 1)


_COMBO_CARDS = np.array([(a, b) for a in range(52) for b in range(a + 1, 52)], dtype=np.uint8)


def combo_cards(ids):
    return _COMBO_CARDS[np.asarray(ids)]


def live_combos(board):
    """Ascending combo ids that avoid the board cards."""
    bm = 0
    for c in board:
        bm |= 1 << int(c)
    ids = [i for i, (a, b) in enumerate(_COMBO_CARDS) if not ((bm >> int(a)) & 1 or (bm >> int(b)) & 1)]
    return np.array(ids, dtype=np.uint16)


# ------------------------------------------------------------------ trees
def make_spec(pot, stack, bet_sizes, raise_sizes=None, raise_cap=1, allin=True, street=5, river_leaves=False,
              river_runout=False):
    sp = TreeSpec()
    sp.pot = float(pot)
    sp.stack = float(stack)
    sp.n_bet_sizes = len(bet_sizes)
    for i, b in enumerate(bet_sizes):
        sp.bet_sizes[i] = float(b)
    rs = raise_sizes or []
    sp.n_raise_sizes = len(rs)
    for i, b in enumerate(rs):
        sp.raise_sizes[i] = float(b)
    sp.raise_cap = int(raise_cap)
    sp.allin = 1 if allin else 0
    sp.street = int(street)
    sp.river_leaves = 1 if river_leaves else 0
    sp.river_runout = 1 if river_runout else 0
    return sp


def build_tree(pot, stack, bet_sizes, raise_sizes=None, raise_cap=1, allin=True, street=5, board=None,
               river_leaves=False, river_runout=False):
    """Betting tree as a NODE_DTYPE array plus (rows0, rows1) and max depth.
    street 5: river; 4: turn (board of 4 cards); 3: flop (board of 3 cards,
    flop and turn betting, river run out).  river_leaves (turn trees): rounds
    that close with chips behind end in a NODE_LEAF valued by a leaf network
    instead of a river chance node.  river_runout (turn trees): the river is
    dealt straight to showdowns."""
    sp = make_spec(pot, stack, bet_sizes, raise_sizes, raise_cap, allin, street, river_leaves, river_runout)
    L = lib()
    n = ctypes.c_int32()
    rows = (ctypes.c_int32 * 2)()
    depth = ctypes.c_int32()
    if street in (3, 4) or board is not None:
        bd = np.ascontiguousarray(np.asarray(board if board is not None else [], dtype=np.uint8))
        check("mtt_tree_build_board", L.mtt_tree_build_board(ctypes.byref(sp), bd.ctypes.data, len(bd), None, 0,
                                                              ctypes.byref(n), rows, ctypes.byref(depth)))
        nodes = np.zeros(n.value, dtype=NODE_DTYPE)
        check("mtt_tree_build_board", L.mtt_tree_build_board(ctypes.byref(sp), bd.ctypes.data, len(bd),
                                                              nodes.ctypes.data, n.value, ctypes.byref(n), rows,
                                                              ctypes.byref(depth)))
    else:
        check("mtt_tree_build", L.mtt_tree_build(ctypes.byref(sp), None, 0, ctypes.byref(n), rows, ctypes.byref(depth)))
        nodes = np.zeros(n.value, dtype=NODE_DTYPE)
        check("mtt_tree_build", L.mtt_tree_build(ctypes.byref(sp), nodes.ctypes.data, n.value, ctypes.byref(n), rows,
                                                 ctypes.byref(depth)))
    return nodes, (rows[0], rows[1]), depth.value


def validate_tree(nodes, rows):
    r = (ctypes.c_int32 * 2)(*rows)
    return lib().mtt_tree_validate(np.ascontiguousarray(nodes).ctypes.data, len(nodes), r)


# ------------------------------------------------------------------ device helpers
def _stream(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _dev(t, dtype):
    import torch
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == dtype and t.is_contiguous()):
        raise TypeError(f"expected a contiguous CUDA tensor of {dtype}")
    return ctypes.c_void_p(t.data_ptr())


def eval7(cards7, out=None, stream=None):
    """uint8 [n, 7] CUDA tensor -> int32 [n] reference scores (uint32 bits)."""
    import torch
    n = cards7.shape[0]
    if out is None:
        out = torch.empty(n, dtype=torch.int32, device=cards7.device)
    check("mtt_eval7", lib().mtt_eval7(_dev(cards7, torch.uint8), _dev(out, torch.int32), n, _stream(stream)))
    return out


def eval7_enumerate(with_keys=False, stream=None):
    import torch
    hist = torch.zeros(9, dtype=torch.int64, device="cuda")
    cs = torch.zeros(1, dtype=torch.int64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    keys = torch.empty(65536, dtype=torch.int32, device="cuda") if with_keys else None
    check("mtt_eval7_enumerate", lib().mtt_eval7_enumerate(
        _dev(hist, torch.int64), _dev(cs, torch.int64), _dev(keys, torch.int32) if keys is not None else None,
        _dev(err, torch.int32), _stream(stream)))
    return hist, cs, keys, err


def board_showdown_counts(board, hands, stream=None):
    """board: uint8 [nb] CUDA; hands: uint8 [H, 2] CUDA -> (W, T, L) int32 [H, H] (hero-major)."""
    import torch
    H = hands.shape[0]
    W = torch.empty((H, H), dtype=torch.int32, device=hands.device)
    T = torch.empty_like(W)
    L_ = torch.empty_like(W)
    check("mtt_board_showdown_counts", lib().mtt_board_showdown_counts(
        _dev(board, torch.uint8), board.shape[0], _dev(hands, torch.uint8), H, _dev(W, torch.int32),
        _dev(T, torch.int32), _dev(L_, torch.int32), _stream(stream)))
    return W, T, L_


GEMM_RELU, GEMM_OUT_BF16, GEMM_MASK = 1, 2, 4


def gemm_bf16(A, B, bias=None, relu=False, out_bf16=False, mask=None, out=None, err=None, stream=None,
              workspace=None):
    """C = A @ B.T (+ bias, ReLU / ReLU-mask) on the tcgen05 tensor cores.
    A: bf16 CUDA [M, K], B: bf16 CUDA [N, K] (row-major, K contiguous, row
    strides multiples of 8); C: float32 or bf16 [M, N].  workspace: an
    optional float32 CUDA tensor that lets a product of few output tiles be
    split along K (mtt_gemm_bf16_ws)."""
    import torch
    M, K = A.shape
    N = B.shape[0]
    if out is None:
        out = torch.empty((M, N), dtype=torch.bfloat16 if out_bf16 else torch.float32, device=A.device)
    own_err = err is None
    if own_err:
        err = torch.zeros(1, dtype=torch.int32, device=A.device)
    flags = (GEMM_RELU if relu else 0) | (GEMM_OUT_BF16 if out_bf16 else 0) | (GEMM_MASK if mask is not None else 0)
    for t in (A, B):
        if t.dtype != torch.bfloat16 or not t.is_cuda or t.stride(1) != 1:
            raise TypeError("A and B must be bf16 CUDA matrices with unit column stride")
    args = (ctypes.c_void_p(A.data_ptr()), A.stride(0), ctypes.c_void_p(B.data_ptr()), B.stride(0),
            ctypes.c_void_p(out.data_ptr()), out.stride(0), M, N, K,
            _dev(bias, torch.float32) if bias is not None else None,
            ctypes.c_void_p(mask.data_ptr()) if mask is not None else None, mask.stride(0) if mask is not None else 0,
            flags, ctypes.c_void_p(err.data_ptr()))
    if workspace is None:
        check("mtt_gemm_bf16", lib().mtt_gemm_bf16(*args, _stream(stream)))
    else:
        if workspace.dtype != torch.float32 or not workspace.is_cuda or not workspace.is_contiguous():
            raise TypeError("workspace must be a contiguous float32 CUDA tensor")
        check("mtt_gemm_bf16_ws", lib().mtt_gemm_bf16_ws(*args, ctypes.c_void_p(workspace.data_ptr()),
                                                         workspace.numel(), _stream(stream)))
    if own_err:
        torch.cuda.current_stream().synchronize() if stream is None else None
        if int(err.item()):
            raise MttError("mtt_gemm_bf16", 4)
    return out


def canonical_flops():
    out = np.zeros(1755 * 4, dtype=np.uint8)
    n = ctypes.c_int32()
    check("mtt_canonical_flops", lib().mtt_canonical_flops(out.ctypes.data, len(out) // 4, ctypes.byref(n)))
    return out.reshape(-1, 4)[: n.value]


def flop_ev(flops3, reach0=None, reach1=None, stream=None):
    import torch
    n = flops3.shape[0]
    ev0 = torch.empty((n, 1176), dtype=torch.float32, device=flops3.device)
    ev1 = torch.empty_like(ev0)
    r0 = _dev(reach0, torch.float32) if reach0 is not None else None
    r1 = _dev(reach1, torch.float32) if reach1 is not None else None
    check("mtt_flop_ev", lib().mtt_flop_ev(_dev(flops3, torch.uint8), n, r0, r1, _dev(ev0, torch.float32),
                                           _dev(ev1, torch.float32), _stream(stream)))
    return ev0, ev1


def ev_dump(flops3, stream=None):
    """[n, 4, 2, 169] float32: the reference ev_dumper's per-flop output."""
    import torch
    n = flops3.shape[0]
    out = torch.empty((n, 4, 2, 169), dtype=torch.float32, device=flops3.device)
    check("mtt_ev_dump", lib().mtt_ev_dump(_dev(flops3, torch.uint8), n, _dev(out, torch.float32), _stream(stream)))
    return out


# ------------------------------------------------------------------ solving
def solve_params(iters=1000, algo=ALGO_CFRPLUS, alpha=1.5, beta=0.0, gamma=2.0, semantics=SEM_CORRECT,
                 threads=0, exploitability=True, alternate=True, avg_power=1.0, target_expl=0.0, max_iters=0,
                 chunk_iters=0):
    p = SolveParams()
    p.iters, p.algo, p.alpha, p.beta, p.gamma = int(iters), int(algo), float(alpha), float(beta), float(gamma)
    p.semantics, p.threads, p.exploitability = int(semantics), int(threads), 1 if exploitability else 0
    p.alternate = 1 if alternate else 0
    p.avg_power = float(avg_power)
    p.target_expl, p.max_iters, p.chunk_iters = float(target_expl), int(max_iters), int(chunk_iters)
    return p


def trim_pool():
    """Returns the device memory that destroyed batches left in the library's
    pool to the driver (the pool keeps it for the next batch otherwise)."""
    check("mtt_trim_pool", lib().mtt_trim_pool())


class RiverBatch:
    """A batch of heads-up subgames resident on the current CUDA device.

    Each subgame is a dict with keys nodes (NODE_DTYPE array), rows (2),
    board (5 or 4 cards), combos0/combos1 (ascending uint16 ids) and
    range0/range1 (float32 weights).
    """

    def __init__(self, subgames):
        self._keep = []
        arr = (Subgame * len(subgames))()
        for i, g in enumerate(subgames):
            nodes = np.ascontiguousarray(g["nodes"], dtype=NODE_DTYPE)
            c0 = np.ascontiguousarray(g["combos0"], dtype=np.uint16)
            c1 = np.ascontiguousarray(g["combos1"], dtype=np.uint16)
            r0 = np.ascontiguousarray(g["range0"], dtype=np.float32)
            r1 = np.ascontiguousarray(g["range1"], dtype=np.float32)
            self._keep += [nodes, c0, c1, r0, r1]
            s = arr[i]
            s.nodes = nodes.ctypes.data
            s.n_nodes = len(nodes)
            s.rows[0], s.rows[1] = int(g["rows"][0]), int(g["rows"][1])
            bd = list(g["board"])
            for k, c in enumerate(bd):
                s.board[k] = int(c)
            s.nboard = len(bd)
            s.H[0], s.H[1] = len(c0), len(c1)
            s.combos[0], s.combos[1] = c0.ctypes.data, c1.ctypes.data
            s.ranges[0], s.ranges[1] = r0.ctypes.data, r1.ctypes.data
        self.n = len(subgames)
        self.meta = [(int(g["rows"][0]), int(g["rows"][1]), len(g["combos0"]), len(g["combos1"]))
                     for g in subgames]
        self.combos = [(np.asarray(g["combos0"], np.int64), np.asarray(g["combos1"], np.int64)) for g in subgames]
        h = ctypes.c_void_p()
        check("mtt_batch_create", lib().mtt_batch_create(arr, len(subgames), ctypes.byref(h)))
        self._h = h
        self._keep = None   # the library copied everything

    def solve(self, params, stream=None, graph=False):
        fn = lib().mtt_batch_solve_graph if graph else lib().mtt_batch_solve
        check("mtt_batch_solve", fn(self._h, ctypes.byref(params), _stream(stream)))

    def results(self, stream=None):
        out = np.zeros((self.n, 6), dtype=np.float64)
        check("mtt_batch_results", lib().mtt_batch_results(self._h, out.ctypes.data, _stream(stream)))
        return out

    def iterations(self):
        out = np.zeros(self.n, dtype=np.int32)
        check("mtt_batch_iterations", lib().mtt_batch_iterations(self._h, out.ctypes.data))
        return out

    def read(self, s):
        rows0, rows1, H0, H1 = self.meta[s]
        R0 = np.zeros((rows0, H0), np.float32); R1 = np.zeros((rows1, H1), np.float32)
        S0 = np.zeros((rows0, H0), np.float32); S1 = np.zeros((rows1, H1), np.float32)
        c0 = np.zeros(H0, np.float32); c1 = np.zeros(H1, np.float32)
        check("mtt_batch_read", lib().mtt_batch_read(self._h, s, R0.ctypes.data, R1.ctypes.data, S0.ctypes.data,
                                                     S1.ctypes.data, c0.ctypes.data, c1.ctypes.data))
        return {"R0": R0, "R1": R1, "S0": S0, "S1": S1, "cfv0": c0, "cfv1": c1}

    def read_vectors(self, s, n_nodes):
        """Per-node reach and counterfactual values of subgame s: two
        [n_nodes, H0 + H1] arrays (player 0's hands first)."""
        rows0, rows1, H0, H1 = self.meta[s]
        reach = np.zeros((n_nodes, H0 + H1), np.float32)
        cfv = np.zeros((n_nodes, H0 + H1), np.float32)
        check("mtt_batch_read_vectors", lib().mtt_batch_read_vectors(self._h, s, reach.ctypes.data, cfv.ctypes.data))
        return reach, cfv

    def root_values(self, s):
        """FP64 root values of subgame s from the last best-response pass:
        (ev0, ev1, br0, br1), each over that player's combos."""
        rows0, rows1, H0, H1 = self.meta[s]
        out = [np.zeros(H0), np.zeros(H1), np.zeros(H0), np.zeros(H1)]
        check("mtt_batch_root_values", lib().mtt_batch_root_values(self._h, s, *[o.ctypes.data for o in out]))
        return tuple(out)

    def info(self):
        db = ctypes.c_int64()
        ib = ctypes.c_int64()
        check("mtt_batch_info", lib().mtt_batch_info(self._h, ctypes.byref(db), ctypes.byref(ib)))
        return {"device_bytes": db.value, "iter_bytes": ib.value}

    def layout(self):
        """Offsets of each subgame's rows blocks and packed ranges in the
        device layout (see mtt_batch_layout)."""
        rows_off = np.zeros((self.n, 2), np.int64)
        range_off = np.zeros(self.n, np.int64)
        tr, tg = ctypes.c_int64(), ctypes.c_int64()
        check("mtt_batch_layout", lib().mtt_batch_layout(self._h, rows_off.ctypes.data, range_off.ctypes.data,
                                                         ctypes.byref(tr), ctypes.byref(tg)))
        return {"rows_off": rows_off, "range_off": range_off, "total_rows": tr.value, "total_range": tg.value}

    def ev_grad(self, logits, ranges, stream=None):
        """EV of player 0 under softmax(logits) strategies and its gradients.
        logits: float32 CUDA [total_rows], ranges: float32 CUDA [total_range]
        (layout()).  Returns (ev [n], grad_ranges, grad_logits), CUDA float32."""
        import torch
        ev = torch.empty(self.n, dtype=torch.float32, device=logits.device)
        g_r = torch.empty_like(ranges)
        g_l = torch.empty_like(logits)
        check("mtt_batch_ev_grad", lib().mtt_batch_ev_grad(
            self._h, _dev(logits, torch.float32), _dev(ranges, torch.float32), _dev(ev, torch.float32),
            _dev(g_r, torch.float32), _dev(g_l, torch.float32), _stream(stream)))
        return ev, g_r, g_l

    def check(self, stream=None):
        """Waits for the stream; raises if a bounded device wait gave up."""
        check("mtt_batch_check", lib().mtt_batch_check(self._h, _stream(stream)))

    def launch_count(self):
        """Kernels launched for this batch so far (graph replays count every node)."""
        n = ctypes.c_int64()
        check("mtt_batch_launch_count", lib().mtt_batch_launch_count(self._h, ctypes.byref(n)))
        return n.value

    def set_leafnet(self, net=None, residual=True):
        """Values the batch's depth-limit leaves (NODE_LEAF) by the leaf
        network `net` (a leafnet.LeafNet whose batch capacity holds 48 rows
        per leaf), as a residual over the check-down values when `residual`;
        net=None values them by check-down alone.  The network must outlive
        the solves."""
        h = net._h if net is not None else None
        flags = 1 if (net is not None and residual) else 0
        check("mtt_batch_set_leafnet", lib().mtt_batch_set_leafnet(self._h, h, flags))
        self._leafnet = net

    def kernel_profile(self, params, iters=10, stream=None):
        """Per-iteration device time (ms) and compulsory bytes of the forward
        sweeps, terminal launches and backward sweeps, timed with CUDA events
        around each kernel class over `iters` iterations (restarts the solve)."""
        ms = np.zeros(3, dtype=np.float64)
        by = np.zeros(3, dtype=np.float64)
        check("mtt_batch_kernel_profile", lib().mtt_batch_kernel_profile(
            self._h, ctypes.byref(params), int(iters), ms.ctypes.data, by.ctypes.data, _stream(stream)))
        return {k: {"ms": float(ms[i]), "bytes": float(by[i])}
                for i, k in enumerate(("k_fwd", "k_term", "k_bwd"))}

    def set_schedule(self, threads=0, hands_per_warp=128, term_chunk=16):
        """Sweep CTA size (0 = default), hands per sweep warp item (128 or
        256) and terminals per terminal CTA at most (1..16)."""
        check("mtt_batch_set_schedule", lib().mtt_batch_set_schedule(self._h, int(threads), int(hands_per_warp),
                                                                     int(term_chunk)))

    def schedule(self):
        t, h, c = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        check("mtt_batch_schedule", lib().mtt_batch_schedule(self._h, ctypes.byref(t), ctypes.byref(h),
                                                             ctypes.byref(c)))
        return {"threads": t.value, "hands_per_warp": h.value, "term_chunk": c.value}

    def autotune(self, params, stream=None):
        t = ctypes.c_int32()
        check("mtt_batch_autotune", lib().mtt_batch_autotune(self._h, ctypes.byref(params), _stream(stream),
                                                             ctypes.byref(t)))
        return t.value

    def close(self):
        if getattr(self, "_h", None):
            lib().mtt_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
