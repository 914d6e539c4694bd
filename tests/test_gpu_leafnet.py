"""Leaf network on the GPU: gradients against the CPU oracle (numpy float64
with the GPU's BF16 rounding points), one Adam step, and learning.

Tolerances (written here): loss within 1e-4 relative; outputs within 1e-2
of the largest; per layer the weight and bias gradients within 2e-2 of the
oracle's in relative Frobenius norm.  The tensor cores accumulate in FP32 in
their own order, so a hidden unit whose sum sits next to a BF16 rounding
boundary can round one BF16 ulp away from the oracle's."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ln():
    return importlib.import_module("mtt-gpu-solver_b200.leafnet")


def _batch(rng, M):
    x = rng.standard_normal((M, 2706)).astype(np.float32) * 0.5
    t = rng.standard_normal((M, 2652)).astype(np.float32) * 0.3
    w = (rng.random((M, 2652)) > 0.2).astype(np.float32)
    return x, t, w


def test_gradients_match_oracle(ln, cuda):
    import torch
    import pymlp
    rng = np.random.default_rng(0)
    M = 64
    x, t, w = _batch(rng, M)
    net = ln.LeafNet(batch_cap=128, seed=3)
    dev = lambda a: torch.from_numpy(a).to(cuda)
    loss = net.gradients(dev(x), dev(t), dev(w))
    net.check()
    params = [net.params(l) for l in range(4)]
    oloss, oy, ograds = pymlp.gradients(params, x.astype(np.float64), t.astype(np.float64), w.astype(np.float64))
    assert abs(loss - oloss) <= 1e-4 * abs(oloss)
    y = net.forward(dev(x)).cpu().numpy()
    # a hidden unit whose FP32 sum sits near a BF16 rounding boundary can round
    # one BF16 ulp apart (0.4%), which moves the outputs by up to ~1e-2
    assert np.abs(y - oy[:, :2652]).max() <= 1e-2 * np.abs(oy).max()
    for l in range(4):
        for k in ("gw", "gb"):
            a, b = params[l][k], ograds[l][k]
            rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
            assert rel <= 2e-2, (l, k, rel)
    net.close()


def test_adam_step_and_learning(ln, cuda):
    import torch
    rng = np.random.default_rng(1)
    M = 256
    x = rng.standard_normal((M, 2706)).astype(np.float32) * 0.5
    # a learnable target: a fixed random linear map of the first 64 features
    P = rng.standard_normal((64, 2652)).astype(np.float32) * 0.05
    t = (x[:, :64] @ P).astype(np.float32)
    net = ln.LeafNet(batch_cap=M, seed=4)
    dx, dt = torch.from_numpy(x).to(cuda), torch.from_numpy(t).to(cuda)
    w0 = net.params(1)["w"]
    first = net.train_step(dx, dt, lr=1e-3)
    w1 = net.params(1)
    # Adam's first step moves every live weight by lr * sign(g) (|m/sqrt(v)| = 1)
    moved = np.abs(w1["w"] - w0)
    live = np.abs(w1["gw"]) > 1e-6
    assert np.allclose(moved[live], 1e-3, rtol=2e-2)
    losses = [first]
    for _ in range(150):
        losses.append(net.train_step(dx, dt, lr=1e-3))
    net.check()
    assert losses[-1] < 0.2 * losses[0], (losses[0], losses[-1])
    net.close()


def test_trained_net_improves_on_check_down_leaves_and_beats_solving_time(ln, mtt, cuda):
    """Train on river values the batched solver generates, then measure on
    held-out subgames against their full river solve.  The method without
    the network estimates a leaf by checking the river down; the network
    learns the correction for river betting on top of it (its output layer
    starts at zero), so it must end below the check-down error, and the
    estimate must come far faster than solving the subgames it replaces."""
    import time
    import torch
    n_train, n_val = 16384, 2048
    t0 = time.perf_counter()
    X, T, W, meta = ln.river_training_set(n_train + n_val, seed=5, iters=150, batch=4096)
    solve_s = (time.perf_counter() - t0) / (n_train + n_val)
    t1 = time.perf_counter()
    CD = ln.checkdown_values(meta)
    cd_s = (time.perf_counter() - t1) / (n_train + n_val)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda)
    Xt, Rt, Wt = dev(X[:n_train]), dev(T[:n_train] - CD[:n_train]), dev(W[:n_train])
    Xv, Tv, Wv, CDv = X[n_train:], T[n_train:], W[n_train:], CD[n_train:]
    net = ln.LeafNet(batch_cap=n_val, seed=1, zero_output=True)
    rng = np.random.default_rng(0)
    first = last = None
    for epoch in range(3):
        perm = torch.from_numpy(rng.permutation(n_train)).to(cuda)
        for k in range(0, n_train, 512):
            idx = perm[k:k + 512]
            loss = net.train_step(Xt[idx].contiguous(), Rt[idx].contiguous(), Wt[idx].contiguous(), lr=1e-4)
            first = loss if first is None else first
            last = loss
    net.check()
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    pred = CDv + net.forward(dev(Xv)).cpu().numpy()
    infer_s = (time.perf_counter() - t2) / n_val
    live = Wv > 0
    mae_net = float(np.abs(pred - Tv)[live].mean())
    mae_cd = float(np.abs(CDv - Tv)[live].mean())
    mae_zero = float(np.abs(Tv)[live].mean())
    print(f"leaf net: train loss {first:.5f} -> {last:.5f}; held-out MAE (pot units) check-down + net {mae_net:.4f}, "
          f"check-down {mae_cd:.4f}, zero {mae_zero:.4f}; {solve_s * 1e3:.3f} ms/solve vs "
          f"{(infer_s + cd_s) * 1e3:.3f} ms/estimate ({cd_s * 1e3:.3f} check-down + {infer_s * 1e3:.4f} network)")
    assert last < first
    assert mae_net < mae_cd < mae_zero
    assert (infer_s + cd_s) * 5 < solve_s
    net.close()


def test_checkdown_kernel_matches_the_solver_terminal_pass(ln, mtt, cuda):
    """The batched check-down kernel against the same values from the
    solver's FP64 showdown terminal on a one-node tree (FP32 sums: 1e-5)."""
    rng = np.random.default_rng(3)
    meta = []
    for _ in range(24):
        board = [int(c) for c in rng.choice(52, 5, replace=False)]
        live = ln._live_mask(board)
        m = {"board": board}
        for p in range(2):
            w = rng.dirichlet(np.full(1326, rng.uniform(0.1, 1.0))) * live
            m[f"range{p}"] = w / w.sum()
        meta.append(m)
    a = ln.checkdown_values(meta)
    b = ln.checkdown_values_fp64(meta)
    assert np.abs(a - b).max() <= 1e-5
