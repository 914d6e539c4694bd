"""Oracle for the flop-subset optimiser (non-negative orthogonal matching pursuit).

Test infrastructure only: the CUDA path (`mtt_subset_nnomp`) is checked against
these functions; nothing in the product imports this file.

Restates scripts/optimize_subset.py:
  - `flop_meta`            generate_1755_flops_meta            (optimize_subset.py:8-26)
  - `nnomp`                the selection loop and final weights (optimize_subset.py:29-50)
  - `subset_bin_bytes`     the mtt_subset.bin writer            (optimize_subset.py:52-56)
  - `subset_weights_text`  the mtt_subset_weights.txt writer    (optimize_subset.py:58-65)

The reference solves each non-negative least-squares subproblem with
scipy.optimize.nnls (scipy 1.18.1 in this image), a compiled implementation of
the classical active-set algorithm of Lawson and Hanson ("Solving Least Squares
Problems", SIAM 1995, ch. 23).  `nnls` below restates that published algorithm
in numpy, starting from x = 0 as scipy does, with each unconstrained
least-squares step solved by numpy's lstsq on the passive columns.  The
solution of a full-column-rank NNLS problem is unique, so two implementations
of the method differ by rounding only.
"""
import numpy as np

N_FEATURES = 4 * 2 * 169   # optimize_subset.py:6 (4 stack depths x 2 players x 169 classes)


def flop_meta():
    """The 1,755 canonical flops as (c1, c2, c3, orbit weight), card = rank * 4 + suit,
    in the dump's column order (optimize_subset.py:8-26)."""
    out = []
    for r in range(12, -1, -1):                           # trips
        out.append((4 * r, 4 * r + 1, 4 * r + 2, 4))
    for rp in range(12, -1, -1):                          # paired boards
        for rk in range(12, -1, -1):
            if rp != rk:
                out.append((4 * rp, 4 * rp + 1, 4 * rk, 12))
                out.append((4 * rp, 4 * rp + 1, 4 * rk + 2, 12))
    for r1 in range(12, 1, -1):                           # three ranks
        for r2 in range(r1 - 1, 0, -1):
            for r3 in range(r2 - 1, -1, -1):
                out += [(4 * r1, 4 * r2, 4 * r3, 4), (4 * r1, 4 * r2, 4 * r3 + 1, 12),
                        (4 * r1, 4 * r2 + 1, 4 * r3, 12), (4 * r1 + 1, 4 * r2, 4 * r3, 12),
                        (4 * r1, 4 * r2 + 1, 4 * r3 + 2, 24)]
    return out


def nnls(A, b, maxiter=None):
    """min ||A x - b|| subject to x >= 0 by Lawson-Hanson's active-set method.
    Returns (x, ||A x - b||).  Raises RuntimeError after maxiter (default 3 n)
    passive-set solves, as scipy.optimize.nnls does."""
    A = np.asarray(A, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    m, n = A.shape
    maxiter = maxiter or 3 * n
    x = np.zeros(n)
    passive = np.zeros(n, dtype=bool)
    tol = 10.0 * max(m, n) * np.finfo(np.float64).eps * max(1.0, np.abs(A).max())
    it = 0
    while True:
        w = A.T @ (b - A @ x)                  # dual: the gradient of -||Ax - b||^2 / 2
        cand = np.where(~passive & (w > tol))[0]
        if cand.size == 0:
            break
        passive[cand[np.argmax(w[cand])]] = True
        while True:
            it += 1
            if it > maxiter:
                raise RuntimeError("nnls: maximum number of iterations reached")
            P = np.where(passive)[0]
            z = np.zeros(n)
            z[P] = np.linalg.lstsq(A[:, P], b, rcond=None)[0]
            if np.all(z[P] > 0):
                x = z
                break
            # step from x towards z until the first passive weight reaches zero
            neg = P[z[P] <= 0]
            alpha = np.min(x[neg] / (x[neg] - z[neg]))
            x = x + alpha * (z - x)
            drop = passive & (x <= tol)
            x[drop] = 0.0
            passive &= ~drop
    return x, float(np.linalg.norm(A @ x - b))


def nnomp(dump, colw, nselect=100, trace=False):
    """Greedy non-negative OMP of optimize_subset.py:29-50.

    dump: [ncols][nfeat] f32 (mtt_ev_dump_1755.bin, one row per flop); colw: the
    flops' orbit weights.  Returns (indices, normalised FP64 weights); with
    trace=True also a dict of per-step diagnostics: the relative gap between
    the best and second-best correlation, and the smallest dual of a zero
    weight and positive weight of each subproblem (how far each step is from
    a tie or a degenerate active set)."""
    dump = np.asarray(dump, dtype=np.float32)
    ncols = dump.shape[0]
    A = dump.T                                          # [nfeat][ncols], optimize_subset.py:29
    colw = np.asarray(colw, dtype=np.float64)
    b = (A @ colw) / np.sum(colw)                       # :32, f32 matrix promoted to f64
    norms = np.linalg.norm(A, axis=0)                   # :36, computed in f32
    norms[norms == 0] = 1.0
    An = A / norms                                      # :38, f32
    sel, r = [], b.copy()
    gaps, duals, mins = [], [], []
    w = np.zeros(0)
    for _ in range(nselect):                            # :40-47
        c = An.T @ r
        c[sel] = -np.inf
        j = int(np.argmax(c))                           # first maximum, as np.argmax
        if trace:
            top = np.sort(c)[::-1]
            gaps.append(float((top[0] - top[1]) / abs(top[0])) if len(top) > 1 else np.inf)
        sel.append(j)
        As = A[:, sel].astype(np.float64)
        w, _ = nnls(As, b)
        r = b - As @ w
        if trace:
            d = As.T @ r
            scale = np.abs(As.T @ b).max()
            zero = w == 0
            duals.append(float(np.max(d[zero]) / scale) if zero.any() else -np.inf)
            mins.append(float(np.min(w[~zero]) / np.max(w)) if (~zero).any() else 0.0)
    # :49 solves the last subproblem again on the same inputs: the same weights
    wn = w * (ncols / np.sum(w))                        # :50
    if trace:
        return np.array(sel, dtype=np.int32), wn, {"gap": gaps, "zero_dual": duals, "min_weight": mins}
    return np.array(sel, dtype=np.int32), wn


def subset_bin_bytes(meta, idx, w):
    """mtt_subset.bin: u32 count, then per flop c1, c2, c3, 0 (u8) and the weight
    as f32 (optimize_subset.py:52-56), little-endian."""
    out = bytearray(np.uint32(len(idx)).astype("<u4").tobytes())
    for j, wj in zip(idx, w):
        c1, c2, c3, _ = meta[j]
        out += bytes((c1, c2, c3, 0)) + np.float32(wj).astype("<f4").tobytes()
    return bytes(out)


def subset_weights_text(meta, idx, w):
    """mtt_subset_weights.txt: one `<card><card><card>:<weight %.4f>` line per flop
    (optimize_subset.py:58-65)."""
    name = lambda c: "23456789TJQKA"[c // 4] + "cdhs"[c % 4]
    return "".join(f"{name(meta[j][0])}{name(meta[j][1])}{name(meta[j][2])}:{float(wj):.4f}\n"
                   for j, wj in zip(idx, w))
