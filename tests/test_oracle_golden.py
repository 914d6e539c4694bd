"""The CPU oracle against the reference's own known answers (no GPU).

The reference ships one end-to-end golden vector for the hot path,
data/mtt_ev_dump_1755.bin; tests/golden holds 21 flop slices of it.  The
oracle must reproduce them bit for bit, which pins the evaluator
(mtt_ev_dumper.cu:53-83), the flop EV kernel (:85-116) and the host
aggregation (:141-168).
"""
import numpy as np
import pytest

# Standard 7-card category counts (the reference evaluator gets the categories right).
STD_HIST = [23294460, 58627800, 31433400, 6461620, 6180020, 4047644, 3473184, 224848, 41584]


def test_flop_list_matches_reference_layout(orc, golden):
    flops = orc.gen_flops()
    assert flops.shape == (1755, 4)
    assert int(flops[:, 3].astype(np.int64).sum()) == 22100   # C(52,3) orbit weights
    assert len({tuple(f[:3]) for f in flops}) == 1755
    assert tuple(flops[0]) == (48, 49, 50, 4)                  # AcAdAh first


@pytest.mark.parametrize("k", [0, 4, 9, 13, 20])
def test_oracle_reproduces_golden_dump_slice(orc, golden, k):
    meta, sl = golden
    f = meta["slice_flops"][k]
    out = orc.ev_dump(f, f + 1)[0]
    assert out.view(np.uint32).tolist() == sl[k].view(np.uint32).tolist()


def test_evaluator_category_histogram(orc):
    hist, cs = orc.enumerate7()
    assert hist.tolist() == STD_HIST
    assert int(hist.sum()) == 133784560


def test_evaluator_reference_quirks(orc):
    def s(cards):
        return int(orc.eval7(np.array([cards], np.uint8))[0])
    c = lambda r, su: r * 4 + su
    # one pair: kickers ignored (AA-K-Q-J vs AA-K-Q-T tie)
    a = s([c(12, 0), c(12, 1), c(11, 2), c(10, 3), c(9, 0), c(2, 1), c(0, 2)])
    b = s([c(12, 2), c(12, 3), c(11, 0), c(10, 1), c(8, 2), c(2, 3), c(0, 0)])
    assert a == b == (1 << 24) | (12 << 12)
    # high card compares the full 7-rank mask
    hc = s([c(12, 0), c(10, 1), c(8, 2), c(6, 3), c(4, 0), c(2, 1), c(0, 2)])
    assert hc == (1 << 12) | (1 << 10) | (1 << 8) | (1 << 6) | (1 << 4) | (1 << 2) | 1
    # wheel straight
    assert s([c(12, 0), c(0, 1), c(1, 2), c(2, 3), c(3, 0), c(8, 1), c(10, 2)]) == (4 << 24) | 3
    # full house with two trips uses the second trips
    fh = s([c(12, 0), c(12, 1), c(12, 2), c(5, 0), c(5, 1), c(5, 2), c(9, 3)])
    assert fh == (6 << 24) | (12 << 4) | 5


def test_board_counts_known_pair(orc):
    c = lambda r, su: r * 4 + su
    board = np.array([c(12, 0), c(11, 1), c(2, 2), c(5, 3)], np.uint8)   # Ac Kd 4h 7s
    hands = np.array([[c(12, 1), c(12, 2)], [c(0, 0), c(0, 1)], [c(12, 1), c(3, 0)]], np.uint8)
    W, T, L = orc.board_counts(board, hands)
    assert W[0, 1] + T[0, 1] + L[0, 1] == 44           # 48 live rivers - 4 hole cards
    assert W[0, 1] == 44 and L[1, 0] == 44              # trip aces vs 22: deuces never catch up
    assert W[0, 2] == 0 and T[0, 2] == 0 and L[0, 2] == 0   # shared card Ad: conflicting pair
