"""The leaf network: an MLP (2,706 -> 3 x 1,024 ReLU -> 2,652) that predicts
both players' river counterfactual values, trained on the GPU by the
library's own tcgen05 GEMM forward and backward kernels (C ABI wrappers).

Features of a river subgame (features()): each player's range over the
1,326 combos normalised to sum 1 and scaled by the number of live combos,
the board as a 52-card one-hot, pot / 100 and stack / 100.  Targets: the
root counterfactual values of each combo divided by the pot (ranges summing
to 1), zero and weight 0 for combos that touch the board."""
import ctypes

import numpy as np

from . import combo_cards
from ._lib import check, lib

IN, HIDDEN, OUT = 2706, 1024, 2652


def _stream(s):
    if s is None:
        return None
    return ctypes.c_void_p(s.cuda_stream if hasattr(s, "cuda_stream") else int(s))


def features(board, range0_1326, range1_1326, pot, stack):
    """One feature row (float32 [2706]) from full 1,326-combo ranges."""
    x = np.zeros(IN, np.float32)
    live = np.ones(1326, bool)
    for c in board:
        live &= ~np.any(_CARDS == int(c), axis=1)
    n_live = int(live.sum())
    for p, r in enumerate((range0_1326, range1_1326)):
        r = np.asarray(r, np.float64) * live
        s = r.sum()
        x[p * 1326:(p + 1) * 1326] = (r / s * n_live if s > 0 else r).astype(np.float32)
    for c in board:
        x[2652 + int(c)] = 1.0
    x[2704] = pot / 100.0
    x[2705] = stack / 100.0
    return x


_CARDS = np.array([(a, b) for a in range(52) for b in range(a + 1, 52)], np.int64)


class LeafNet:
    def __init__(self, batch_cap=4096, seed=0, zero_output=False):
        h = ctypes.c_void_p()
        check("mtt_leafnet_create", lib().mtt_leafnet_create(int(batch_cap), int(seed), 1 if zero_output else 0,
                                                             ctypes.byref(h)))
        self._h = h
        self.cap = batch_cap

    @staticmethod
    def _ptr(t, n_cols):
        import torch
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()
                and t.dim() == 2 and t.shape[1] == n_cols):
            raise TypeError(f"expected a contiguous CUDA float32 [M, {n_cols}] tensor")
        return ctypes.c_void_p(t.data_ptr())

    def forward(self, x, stream=None):
        import torch
        y = torch.empty((x.shape[0], OUT), dtype=torch.float32, device=x.device)
        check("mtt_leafnet_forward", lib().mtt_leafnet_forward(self._h, self._ptr(x, IN), x.shape[0],
                                                               ctypes.c_void_p(y.data_ptr()), _stream(stream)))
        return y

    def gradients(self, x, t, w=None, stream=None):
        loss = ctypes.c_double()
        check("mtt_leafnet_gradients", lib().mtt_leafnet_gradients(
            self._h, self._ptr(x, IN), self._ptr(t, OUT), self._ptr(w, OUT) if w is not None else None, x.shape[0],
            ctypes.byref(loss), _stream(stream)))
        return loss.value

    def train_step(self, x, t, w=None, lr=1e-3, stream=None, want_loss=True):
        loss = ctypes.c_double()
        check("mtt_leafnet_train_step", lib().mtt_leafnet_train_step(
            self._h, self._ptr(x, IN), self._ptr(t, OUT), self._ptr(w, OUT) if w is not None else None, x.shape[0],
            float(lr), ctypes.byref(loss) if want_loss else None, _stream(stream)))
        return loss.value if want_loss else None

    def params(self, layer):
        shape = (ctypes.c_int32 * 2)()
        check("mtt_leafnet_params", lib().mtt_leafnet_params(self._h, layer, None, None, None, None, shape))
        o, i = shape[0], shape[1]
        w = np.zeros((o, i), np.float32); b = np.zeros(o, np.float32)
        gw = np.zeros((o, i), np.float32); gb = np.zeros(o, np.float32)
        check("mtt_leafnet_params", lib().mtt_leafnet_params(self._h, layer, w.ctypes.data, b.ctypes.data,
                                                             gw.ctypes.data, gb.ctypes.data, shape))
        return {"w": w, "b": b, "gw": gw, "gb": gb}

    def check(self):
        check("mtt_leafnet_check", lib().mtt_leafnet_check(self._h))

    def close(self):
        if getattr(self, "_h", None):
            lib().mtt_leafnet_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _live_mask(board):
    live = np.ones(1326, bool)
    for c in board:
        live &= ~np.any(_CARDS == int(c), axis=1)
    return live


def river_training_set(n, seed=0, iters=300, batch=2048, spr=(0.5, 1.0, 2.0, 3.0, 4.0), stream=None):
    """n solver-generated training samples.  Each is a river subgame on a
    seeded board with pot 100, stack 100 * SPR (SPR from `spr`), bets {50%,
    100%} + all-in and one raise, ranges Dirichlet(alpha) over the live
    combos (alpha ~ U[0.1, 1] per player), solved by the batched GPU solver
    (alternating CFR+, quadratic averaging, `iters` iterations); the targets
    are the FP64 root values of both players under the average strategies,
    divided by the pot.  Returns (X [n,2706], T [n,2652], W [n,2652], meta)."""
    from . import RiverBatch, build_tree, solve_params
    rng = np.random.default_rng(seed)
    trees = {s: build_tree(100.0, 100.0 * s, [0.5, 1.0], raise_cap=1) for s in spr}
    X = np.zeros((n, IN), np.float32)
    T = np.zeros((n, OUT), np.float32)
    W = np.zeros((n, OUT), np.float32)
    meta = []
    for b0 in range(0, n, batch):
        subs = []
        for _ in range(min(batch, n - b0)):
            board = [int(c) for c in rng.choice(52, size=5, replace=False)]
            live = np.nonzero(_live_mask(board))[0]
            s = float(rng.choice(spr))
            nodes, rows, _ = trees[s]
            g = {"nodes": nodes, "rows": rows, "board": board, "pot": 100.0, "stack": 100.0 * s}
            for p in range(2):
                w = rng.dirichlet(np.full(len(live), rng.uniform(0.1, 1.0)))
                g[f"combos{p}"] = live.astype(np.uint16)
                g[f"range{p}"] = (w / w.sum()).astype(np.float32)
            subs.append(g)
        rb = RiverBatch(subs)
        rb.solve(solve_params(iters=iters, exploitability=True, alternate=True, avg_power=2.0), graph=True,
                 stream=stream)
        for k, g in enumerate(subs):
            i = b0 + k
            ev0, ev1, _, _ = rb.root_values(k)
            full = [np.zeros(1326), np.zeros(1326)]
            for p, ev in enumerate((ev0, ev1)):
                c = g[f"combos{p}"].astype(np.int64)
                full[p][c] = g[f"range{p}"]
                T[i, p * 1326 + c] = (ev / g["pot"]).astype(np.float32)
                W[i, p * 1326 + c] = 1.0
            X[i] = features(g["board"], full[0], full[1], g["pot"], g["stack"])
            meta.append({"board": g["board"], "range0": full[0], "range1": full[1]})
        rb.close()
    return X, T, W, meta


def checkdown_values(meta, device="cuda", stream=None):
    """The leaf estimate without a network: both players check the river
    down.  Per combo, the showdown value against the opponent's range with
    card removal and split ties, in units of the pot (ranges summing to 1),
    from the batched GPU kernel (mtt_checkdown_values).  Returns [n, 2652]
    like the targets (0 for combos touching the board)."""
    import torch
    n = len(meta)
    boards = np.asarray([m["board"] for m in meta], np.uint8).reshape(n, 5)
    bm = np.bitwise_or.reduce(np.left_shift(np.uint64(1), boards.astype(np.uint64)), axis=1)      # [n]
    cm = np.left_shift(np.uint64(1), _CARDS[:, 0].astype(np.uint64)) | \
        np.left_shift(np.uint64(1), _CARDS[:, 1].astype(np.uint64))                               # [1326]
    live = (bm[:, None] & cm[None, :]) == 0
    r = []
    for p in range(2):
        v = np.stack([np.asarray(m[f"range{p}"], np.float64) for m in meta]) * live
        tot = v.sum(axis=1, keepdims=True)
        r.append(np.where(tot > 0, v / np.where(tot > 0, tot, 1.0), v).astype(np.float32))
    db = torch.from_numpy(boards).to(device)
    d0, d1 = torch.from_numpy(r[0]).to(device), torch.from_numpy(r[1]).to(device)
    out = torch.empty((n, OUT), dtype=torch.float32, device=device)
    check("mtt_checkdown_values", lib().mtt_checkdown_values(
        ctypes.c_void_p(db.data_ptr()), ctypes.c_void_p(d0.data_ptr()), ctypes.c_void_p(d1.data_ptr()), n,
        ctypes.c_void_p(out.data_ptr()), _stream(stream)))
    return out.cpu().numpy()


def checkdown_values_fp64(meta, batch=4096):
    """The same check-down values from the solver's FP64 terminal pass on a
    one-node showdown tree (slower: every board is packed on the host)."""
    from . import NODE_DTYPE, NODE_SHOWDOWN, RiverBatch, solve_params
    node = np.zeros(1, dtype=NODE_DTYPE)
    node[0]["type"] = NODE_SHOWDOWN
    node[0]["pot_size"] = 100.0
    node[0]["committed"] = [50.0, 50.0]
    node[0]["turn_idx"] = -1
    out = np.zeros((len(meta), OUT), np.float32)
    for b0 in range(0, len(meta), batch):
        subs = []
        for m in meta[b0:b0 + batch]:
            live = np.nonzero(_live_mask(m["board"]))[0]
            g = {"nodes": node, "rows": (0, 0), "board": m["board"], "pot": 100.0}
            for p in range(2):
                r = np.asarray(m[f"range{p}"], np.float64)[live]
                g[f"combos{p}"] = live.astype(np.uint16)
                g[f"range{p}"] = (r / r.sum()).astype(np.float32) if r.sum() > 0 else r.astype(np.float32)
            subs.append(g)
        rb = RiverBatch(subs)
        rb.solve(solve_params(iters=0, exploitability=True))
        for k, g in enumerate(subs):
            ev0, ev1, _, _ = rb.root_values(k)
            c = g["combos0"].astype(np.int64)
            out[b0 + k, c] = (ev0 / 100.0).astype(np.float32)
            out[b0 + k, 1326 + c] = (ev1 / 100.0).astype(np.float32)
        rb.close()
    return out


def gemm_timing(M=4096, N=1024, K=2752, reps=20, seed=0):
    """Device time of the leaf network's tcgen05 GEMM on one shape
    (C[M x N] fp32 = A[M x K] B[N x K]^T, bf16 operands), two ways, after a
    warm-up call, with CUDA events on the current stream:
    - per call: reps calls from Python, each launched by the library (host
      work between launches included);
    - graph: the same reps launches captured once in a CUDA graph and
      replayed (the kernels back to back).
    Returns {"call_ms", "graph_ms", "call_tflops", "graph_tflops"}."""
    import torch
    from . import gemm_bf16
    g = torch.Generator(device="cuda").manual_seed(seed)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    C = torch.empty(M, N, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")   # one error word, checked at the end
    gemm_bf16(A, B, out=C, err=err)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        gemm_bf16(A, B, out=C, err=err)
    e1.record()
    torch.cuda.synchronize()
    call_ms = e0.elapsed_time(e1) / reps
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        gemm_bf16(A, B, out=C, err=err, stream=s)
        torch.cuda.synchronize()
        with torch.cuda.graph(graph, stream=s):
            for _ in range(reps):
                gemm_bf16(A, B, out=C, err=err, stream=s)
    graph.replay()
    torch.cuda.synchronize()
    e0.record()
    graph.replay()
    e1.record()
    torch.cuda.synchronize()
    graph_ms = e0.elapsed_time(e1) / reps
    if int(err.item()):
        raise RuntimeError("a bounded wait in the GEMM gave up")
    fl = 2.0 * M * N * K
    return {"call_ms": call_ms, "graph_ms": graph_ms, "call_tflops": fl / (call_ms * 1e-3) / 1e12,
            "graph_tflops": fl / (graph_ms * 1e-3) / 1e12}


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser(description="time the leaf network's GEMM on one shape")
    ap.add_argument("--shape", type=int, nargs=3, default=[4096, 1024, 2752], metavar=("M", "N", "K"))
    ap.add_argument("--reps", type=int, default=20)
    a = ap.parse_args()
    t = gemm_timing(*a.shape, reps=a.reps)
    print(f"gemm {a.shape[0]}x{a.shape[1]}x{a.shape[2]}: per call {t['call_ms']:.4f} ms ({t['call_tflops']:.1f} "
          f"TFLOP/s), graph-replayed {t['graph_ms']:.4f} ms ({t['graph_tflops']:.1f} TFLOP/s)")
