"""Preflop anchor chain on the GPU vs the oracle (reference mode).

Integer counts and the order-fixed float results (equities, class averages)
must match bit for bit; the DCFR chain uses the same IEEE operations in the
same order as the oracle (no contractions), so it is compared bit for bit
too.  Full-size results are compared with tests/golden/preflop_ref.json,
made by tests/golden/make_preflop_golden.py from the oracle."""
import hashlib
import importlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def pf():
    return importlib.import_module("mtt-gpu-solver_b200.preflop")


@pytest.fixture(scope="module")
def subset(pf):
    return pf.read_subset(os.path.join(GOLD, "mtt_subset.bin"))


def test_allin_counts_match_oracle_rows(pf, orc, cuda):
    out, w, t = pf.allin_matrix(pf.REFERENCE, counts=True)
    w, t, out = w.cpu().numpy(), t.cpu().numpy(), out.cpu().numpy()
    for hb in (0, 12, 23, 24, 90, 91, 168):     # pairs, the class_to_cards boundary (24), offsuit
        o_out, o_w, o_t = orc.pf_allin(hb, hb + 1)
        assert np.array_equal(w[hb], o_w[hb]) and np.array_equal(t[hb], o_t[hb]), hb
        assert np.array_equal(out[hb].view(np.uint32), o_out[hb].view(np.uint32)), hb


def test_flop_class_matrices_match_oracle(pf, orc, subset, cuda):
    flops, _ = subset
    mats = pf.flop_class_matrices(flops[:2], pf.REFERENCE).cpu().numpy()
    for i in range(2):
        o = orc.pf_flop_class(flops[i])
        assert np.array_equal(mats[i].view(np.uint32), o.view(np.uint32)), i


def test_dcfr_chain_matches_oracle(pf, orc, subset, cuda):
    import torch
    flops, w = subset
    allin = pf.allin_matrix(pf.REFERENCE)
    mats = pf.flop_class_matrices(flops[:3], pf.REFERENCE)
    sums, sig = pf.dcfr(w[:3], mats, allin, iters=40)
    o_sums, o_sig = orc.pf_dcfr(w[:3], mats.cpu().numpy(), allin.cpu().numpy(), iters=40)
    torch.cuda.synchronize()
    assert np.array_equal(sums.cpu().numpy()[:, :169], o_sums[:, :169])
    assert np.array_equal(sig.cpu().numpy()[:, :169], o_sig[:, :169])


@pytest.mark.skipif(not os.path.exists(os.path.join(GOLD, "preflop_ref.json")), reason="no preflop fixture")
def test_full_chain_matches_golden(pf, subset, cuda):
    """All 100 subset flops and 500 DCFR iterations, as preflop_gen runs them."""
    import torch
    g = json.load(open(os.path.join(GOLD, "preflop_ref.json")))
    flops, w = subset
    out, wi, ti = pf.allin_matrix(pf.REFERENCE, counts=True)
    cnt = wi.cpu().numpy().astype("<i4").tobytes() + ti.cpu().numpy().astype("<i4").tobytes()
    assert hashlib.sha256(cnt).hexdigest() == g["allin_counts_sha256"]
    mats = pf.flop_class_matrices(flops, pf.REFERENCE)
    m = mats.cpu().numpy()
    per = [hashlib.sha256(m[i].astype("<f4").tobytes()).hexdigest() for i in range(len(m))]
    bad = [i for i, (a, b) in enumerate(zip(per, g["class_mat_sha256"])) if a != b]
    assert not bad, bad[:10]
    sums, _ = pf.dcfr(w, mats, out, iters=g["dcfr_iters"], stack_bb=g["stack_bb"], bubble=g["bubble"],
                      dead_pot=g["dead_pot"])
    torch.cuda.synchronize()
    assert np.array_equal(sums.cpu().numpy(), np.asarray(g["sums"], np.float32))


def test_correct_mode_sanity(pf, subset, cuda):
    """Correct mode: valid cards and no replacement give a consistent all-in
    matrix (E[h][v] + E[v][h] = 1 within Monte-Carlo noise; AA vs KK near
    82%), and flop matrices over all flop-compatible combos."""
    a = pf.allin_matrix(pf.CORRECT).cpu().numpy()
    off = ~np.eye(169, dtype=bool)
    assert np.abs((a + a.T - 1.0)[off]).max() < 0.06
    assert 0.78 < a[0, 1] < 0.86
    flops, _ = subset
    m = pf.flop_class_matrices(flops[:1], pf.CORRECT).cpu().numpy()[0]
    assert np.isfinite(m).all() and (m >= 0).all() and (m <= 1).all()
