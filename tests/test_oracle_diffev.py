"""CPU checks of the differentiable-EV oracle (orc_softmax_ev): the identities
the GPU adjoint relies on hold in FP64.  EV0 is bilinear in the two ranges,
so dEV0/drange0 = cfv0 and dEV0/drange1 = -cfv1 (zero-sum payoffs); a central
difference (h = 1e-6) must reproduce them to 1e-7 of the pot."""
import numpy as np


def _case(wl):
    subs, logits = wl.diff_boards(n=1, seed=41, n_hands=50)
    g = subs[0]
    return g, logits[0][0].astype(np.float64), logits[0][1].astype(np.float64)


def test_zero_sum_identity(wl, orc):
    g, l0, l1 = _case(wl)
    ev, c0, c1 = orc.softmax_ev(g, l0, l1)
    r0, r1 = g["range0"].astype(np.float64), g["range1"].astype(np.float64)
    assert abs(ev - float(r0 @ c0)) < 1e-12
    assert abs(ev + float(r1 @ c1)) < 1e-9 * g["pot"]


def test_range_gradients_are_the_counterfactual_values(wl, orc):
    g, l0, l1 = _case(wl)
    ev, c0, c1 = orc.softmax_ev(g, l0, l1)
    r0, r1 = g["range0"].astype(np.float64), g["range1"].astype(np.float64)
    h = 1e-6
    for k in (0, 7, 31):
        rp, rm = r0.copy(), r0.copy(); rp[k] += h; rm[k] -= h
        fd = (orc.softmax_ev(g, l0, l1, rp, r1)[0] - orc.softmax_ev(g, l0, l1, rm, r1)[0]) / (2 * h)
        assert abs(fd - c0[k]) < 1e-7 * g["pot"]
        rp, rm = r1.copy(), r1.copy(); rp[k] += h; rm[k] -= h
        fd = (orc.softmax_ev(g, l0, l1, r0, rp)[0] - orc.softmax_ev(g, l0, l1, r0, rm)[0]) / (2 * h)
        assert abs(fd + c1[k]) < 1e-7 * g["pot"]


def test_uniform_logits_give_uniform_strategy_values(wl, orc):
    """Equal logits are the uniform strategy: the same values as the
    behaviour-probability oracle with sigma = 1/A."""
    g, l0, l1 = _case(wl)
    z0, z1 = np.zeros_like(l0), np.zeros_like(l1)
    ev, c0, c1 = orc.softmax_ev(g, z0, z1)
    s0 = np.zeros(l0.shape, np.float32); s1 = np.zeros(l1.shape, np.float32)
    for nd in g["nodes"]:
        if nd["type"] == 0:
            A, r = int(nd["num_actions"]), int(nd["infoset_offset"])
            (s0 if nd["player"] == 0 else s1)[r:r + A] = 1.0 / A
    u0, u1, _ = orc.strategy_values(g, s0, s1)
    assert np.allclose(c0, u0, atol=1e-6) and np.allclose(c1, u1, atol=1e-6)
