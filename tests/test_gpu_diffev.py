"""Differentiable EV of softmax strategies: GPU adjoint sweep vs the FP64 oracle.

The oracle (orc_softmax_ev) evaluates EV0 in FP64 with dense showdowns; the
GPU runs one FP32 sweep.  Tolerances (all written here):
  * EV0 and dEV0/drange (the root counterfactual values): 1e-5 of the pot per
    unit of range mass, i.e. |d| <= 1e-5 * pot * mass0 * mass1 for EV0 and
    1e-5 * pot * (opponent mass) per hand for the CFVs;
  * dEV0/dlogits against FP64 central finite differences of the oracle with
    h = 1e-6: |g - fd| <= 1e-5 * pot * mass0 * mass1 + 1e-3 * |fd|.
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

H_FD = 1e-6


@pytest.fixture(scope="module")
def dev_mod():
    return importlib.import_module("mtt-gpu-solver_b200.diffev")


def _packed(sev, logits_list, cuda):
    import torch
    L = np.zeros(sev.total_rows, np.float32)
    Rg = np.zeros(sev.total_range, np.float32)
    for s, (l0, l1) in enumerate(logits_list):
        rows0, rows1, H0, H1 = sev.batch.meta[s]
        Hp = [(H0 + 3) // 4 * 4, (H1 + 3) // 4 * 4]
        for p, (l, rows, H) in enumerate(((l0, rows0, H0), (l1, rows1, H1))):
            o = int(sev.rows_off[s, p])
            blk = L[o:o + rows * Hp[p]].reshape(rows, Hp[p])
            blk[:, :H] = l
    return torch.from_numpy(L).to(cuda), Rg


def _ranges_packed(sev, subs, cuda):
    import torch
    Rg = np.zeros(sev.total_range, np.float32)
    for s, g in enumerate(subs):
        H0, H1 = len(g["combos0"]), len(g["combos1"])
        o = int(sev.range_off[s])
        Rg[o:o + H0] = g["range0"]
        Rg[o + (H0 + 3) // 4 * 4:o + (H0 + 3) // 4 * 4 + H1] = g["range1"]
    return torch.from_numpy(Rg).to(cuda)


def _run(dev_mod, subs, logits, cuda):
    sev = dev_mod.StrategyEV(subs)
    L, _ = _packed(sev, logits, cuda)
    R = _ranges_packed(sev, subs, cuda)
    ev, g_r, g_l = sev.batch.ev_grad(L, R)
    sev.batch.check()
    return sev, L, R, ev.cpu().numpy(), g_r.cpu().numpy(), g_l


def test_ev_and_range_gradients_match_oracle(dev_mod, wl, orc, cuda):
    subs, logits = wl.diff_boards(n=4, seed=31, n_hands=90)
    sev, L, R, ev, g_r, _ = _run(dev_mod, subs, logits, cuda)
    for s, g in enumerate(subs):
        l0, l1 = logits[s]
        oev, c0, c1 = orc.softmax_ev(g, l0.astype(np.float64), l1.astype(np.float64))
        m0, m1 = float(g["range0"].sum()), float(g["range1"].sum())
        assert abs(ev[s] - oev) <= 1e-5 * g["pot"] * m0 * m1, (ev[s], oev)
        H0, H1 = len(c0), len(c1)
        o = int(sev.range_off[s]); Hp0 = (H0 + 3) // 4 * 4
        assert np.abs(g_r[o:o + H0] - c0).max() <= 1e-5 * g["pot"] * m1
        assert np.abs(g_r[o + Hp0:o + Hp0 + H1] + c1).max() <= 1e-5 * g["pot"] * m0
    sev.close()


def test_logit_gradients_match_fp64_finite_differences(dev_mod, wl, orc, cuda):
    subs, logits = wl.diff_boards(n=2, seed=32, n_hands=70)
    sev, L, R, ev, g_r, g_l = _run(dev_mod, subs, logits, cuda)
    rng = np.random.default_rng(5)
    worst = 0.0
    for s, g in enumerate(subs):
        G = [x.cpu().numpy() for x in sev.unpack_rows(g_l, s)]
        l64 = [logits[s][0].astype(np.float64), logits[s][1].astype(np.float64)]
        m0, m1 = float(g["range0"].sum()), float(g["range1"].sum())
        for _ in range(12):
            p = int(rng.integers(0, 2))
            r_, h_ = int(rng.integers(0, l64[p].shape[0])), int(rng.integers(0, l64[p].shape[1]))
            lp = [x.copy() for x in l64]; lm = [x.copy() for x in l64]
            lp[p][r_, h_] += H_FD; lm[p][r_, h_] -= H_FD
            fd = (orc.softmax_ev(g, *lp)[0] - orc.softmax_ev(g, *lm)[0]) / (2 * H_FD)
            d = abs(G[p][r_, h_] - fd)
            assert d <= 1e-5 * g["pot"] * m0 * m1 + 1e-3 * abs(fd), (s, p, r_, h_, G[p][r_, h_], fd)
            worst = max(worst, d / max(abs(fd), 1e-12))
    sev.close()


def test_autograd_function_scales_gradients(dev_mod, wl, orc, cuda):
    import torch
    subs, logits = wl.diff_boards(n=3, seed=33, n_hands=60)
    sev = dev_mod.StrategyEV(subs)
    L, _ = _packed(sev, logits, cuda)
    L = L.clone().requires_grad_(True)
    r0 = torch.zeros((3, 1326), device=cuda)
    r1 = torch.zeros((3, 1326), device=cuda)
    for s, g in enumerate(subs):
        r0[s, torch.from_numpy(g["combos0"].astype(np.int64)).to(cuda)] = torch.from_numpy(g["range0"]).to(cuda)
        r1[s, torch.from_numpy(g["combos1"].astype(np.int64)).to(cuda)] = torch.from_numpy(g["range1"]).to(cuda)
    r0.requires_grad_(True)
    r1.requires_grad_(True)
    w = torch.tensor([0.5, -2.0, 1.25], device=cuda)
    ev = sev(L, sev.pack_ranges(r0, r1))
    (w * ev).sum().backward()
    _, g_r, g_l = sev.batch.ev_grad(L.detach(), sev.pack_ranges(r0.detach(), r1.detach()))
    for s, g in enumerate(subs):
        oev, c0, c1 = orc.softmax_ev(g, logits[s][0].astype(np.float64), logits[s][1].astype(np.float64))
        c0g = r0.grad[s, torch.from_numpy(g["combos0"].astype(np.int64)).to(cuda)].cpu().numpy()
        c1g = r1.grad[s, torch.from_numpy(g["combos1"].astype(np.int64)).to(cuda)].cpu().numpy()
        m0, m1 = float(g["range0"].sum()), float(g["range1"].sum())
        assert np.abs(c0g - float(w[s]) * c0).max() <= 1e-5 * g["pot"] * m1 * abs(float(w[s]))
        assert np.abs(c1g + float(w[s]) * c1).max() <= 1e-5 * g["pot"] * m0 * abs(float(w[s]))
        for p in range(2):
            a = sev.unpack_rows(L.grad, s)[p]
            b = sev.unpack_rows(g_l, s)[p] * w[s]
            assert torch.equal(a, b)
        # blocked combos get no gradient
        blocked = np.setdiff1d(np.arange(1326), g["combos0"])
        assert float(r0.grad[s, torch.from_numpy(blocked).to(cuda)].abs().max()) == 0.0
    sev.close()


def test_full_boards_relative_error(dev_mod, wl, orc, cuda):
    """Config-3 boards at full size (1,081 hands): logit and range gradients
    against FP64 central differences on sampled coordinates."""
    subs, logits = wl.diff_boards(n=3, seed=3)
    sev, L, R, ev, g_r, g_l = _run(dev_mod, subs, logits, cuda)
    rng = np.random.default_rng(9)
    for s, g in enumerate(subs):
        G = [x.cpu().numpy() for x in sev.unpack_rows(g_l, s)]
        l64 = [logits[s][0].astype(np.float64), logits[s][1].astype(np.float64)]
        oev, c0, c1 = orc.softmax_ev(g, *l64)
        assert abs(ev[s] - oev) <= 1e-5 * g["pot"]
        for _ in range(3):
            p = int(rng.integers(0, 2))
            r_, h_ = int(rng.integers(0, l64[p].shape[0])), int(rng.integers(0, l64[p].shape[1]))
            lp = [x.copy() for x in l64]; lm = [x.copy() for x in l64]
            lp[p][r_, h_] += H_FD; lm[p][r_, h_] -= H_FD
            fd = (orc.softmax_ev(g, *lp)[0] - orc.softmax_ev(g, *lm)[0]) / (2 * H_FD)
            assert abs(G[p][r_, h_] - fd) <= 1e-5 * g["pot"] + 1e-3 * abs(fd)
    sev.close()
