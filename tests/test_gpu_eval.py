"""GPU evaluator, showdown counts and dumper chain vs the oracle and the
reference's shipped dump.  Integer outputs must match bit for bit."""
import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STD_HIST = [23294460, 58627800, 31433400, 6461620, 6180020, 4047644, 3473184, 224848, 41584]


def _random_hands(rng, n):
    return np.stack([rng.choice(52, size=7, replace=False) for _ in range(n)]).astype(np.uint8)


@pytest.mark.parametrize("n,offset", [(200_000, 0), (200_000 + 333, 0), (5_000, 1), (1, 0), (1023, 0)])
def test_eval7_matches_oracle(mtt, orc, cuda, n, offset):
    import torch
    rng = np.random.default_rng(n + offset)
    hands = _random_hands(rng, n)
    buf = torch.zeros(n * 7 + offset, dtype=torch.uint8, device=cuda)
    buf[offset:] = torch.from_numpy(hands.reshape(-1)).to(cuda)
    dev = buf[offset:].view(n, 7)   # offset 1: unaligned start takes the plain-load path
    got = mtt.eval7(dev.contiguous() if offset == 0 else dev).cpu().numpy().view(np.uint32)
    exp = orc.eval7(hands)
    assert np.array_equal(got, exp)


def test_eval7_empty(mtt, cuda):
    import torch
    out = mtt.eval7(torch.zeros((0, 7), dtype=torch.uint8, device=cuda))
    assert out.numel() == 0


def test_enumerate_all_hands_checksum_and_key_order(mtt, orc, cuda):
    hist, cs, keys, err = mtt.eval7_enumerate(with_keys=True)
    assert hist.cpu().tolist() == STD_HIST
    ohist, ocs = orc.enumerate7()
    assert int(cs.cpu().numpy().view(np.uint64)[0]) == ocs
    assert int(err.item()) == 0
    k = keys.cpu().numpy().view(np.uint32)
    used = np.nonzero(k != 0xFFFFFFFF)[0]
    assert len(used) == 3069                      # distinct reference scores
    assert (np.diff(k[used].astype(np.int64)) > 0).all()   # the 16-bit key is monotone in the score
    assert used.min() > 0 and used.max() < 0xFFFF


def _all_hands():
    return np.array([(a, b) for a in range(52) for b in range(a + 1, 52)], np.uint8)


@pytest.mark.parametrize("nboard,H,seed", [(5, 1326, 0), (4, 1326, 1), (4, 300, 7), (3, 120, 2), (3, 1, 3)])
def test_board_showdown_counts_match_oracle(mtt, orc, cuda, nboard, H, seed):
    import torch
    rng = np.random.default_rng(seed)
    board = rng.choice(52, size=nboard, replace=False).astype(np.uint8)
    hands = _all_hands()
    if H < 1326:
        hands = hands[np.sort(rng.choice(1326, size=H, replace=False))]
    W, T, L = mtt.board_showdown_counts(torch.from_numpy(board).to(cuda), torch.from_numpy(hands).to(cuda))
    oW, oT, oL = orc.board_counts(board, hands)
    assert np.array_equal(W.cpu().numpy(), oW)
    assert np.array_equal(T.cpu().numpy(), oT)
    assert np.array_equal(L.cpu().numpy(), oL)
    # antisymmetry of a head-to-head: i beats j <=> j loses to i
    assert np.array_equal(W.cpu().numpy(), L.cpu().numpy().T)


@pytest.mark.parametrize("fidx", [0, 20, 400, 1754])
def test_flop_ev_bit_exact_vs_oracle(mtt, orc, cuda, fidx):
    import torch
    flops = orc.gen_flops()
    f3 = np.ascontiguousarray(flops[fidx:fidx + 1, :3])
    ev0, ev1 = mtt.flop_ev(torch.from_numpy(f3).to(cuda))
    o0, o1 = orc.flop_ev(f3[0])
    assert np.array_equal(ev0.cpu().numpy()[0].view(np.uint32), o0.view(np.uint32))
    assert np.array_equal(ev1.cpu().numpy()[0].view(np.uint32), o1.view(np.uint32))
    # non-uniform reach too
    rng = np.random.default_rng(fidx)
    r0 = rng.random(1176).astype(np.float32); r1 = rng.random(1176).astype(np.float32)
    ev0, ev1 = mtt.flop_ev(torch.from_numpy(f3).to(cuda), torch.from_numpy(r0).to(cuda), torch.from_numpy(r1).to(cuda))
    o0, o1 = orc.flop_ev(f3[0], r0, r1)
    assert np.array_equal(ev0.cpu().numpy()[0].view(np.uint32), o0.view(np.uint32))
    assert np.array_equal(ev1.cpu().numpy()[0].view(np.uint32), o1.view(np.uint32))


def test_ev_dump_slices_bit_exact_vs_reference_file(mtt, orc, golden, cuda):
    import torch
    meta, sl = golden
    flops = orc.gen_flops()
    f3 = np.ascontiguousarray(flops[meta["slice_flops"], :3])
    out = mtt.ev_dump(torch.from_numpy(f3).to(cuda)).cpu().numpy()
    assert np.array_equal(out.view(np.uint32), sl.view(np.uint32))


def test_full_ev_dump_regenerates_reference_file(mtt, golden, cuda):
    import torch
    meta, _ = golden
    flops = mtt.canonical_flops()
    out = mtt.ev_dump(torch.from_numpy(np.ascontiguousarray(flops[:, :3])).to(cuda)).cpu().numpy()
    raw = np.ascontiguousarray(out, dtype="<f4").tobytes()
    assert len(raw) == meta["ev_dump_bytes"]
    assert hashlib.sha256(raw).hexdigest() == meta["ev_dump_sha256"]
