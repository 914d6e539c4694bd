"""mtt_board_showdown_counts_noalloc (static device scratch) against
mtt_board_showdown_counts (stream-ordered allocation), both called through the
C ABI.  Counts are integers, so the two must agree bit for bit, on two calls
in a row.  Collected last so that it also runs after every other GPU test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MTT_OK, MTT_ERR_UNSUPPORTED = 0, 6


def _counts(lib, fn, board, hands, stream):
    import torch
    H = hands.shape[0]
    out = [torch.full((H, H), -7, dtype=torch.int32, device=hands.device) for _ in range(3)]
    st = getattr(lib, fn)(ctypes.c_void_p(board.data_ptr()), board.shape[0], ctypes.c_void_p(hands.data_ptr()), H,
                          *(ctypes.c_void_p(t.data_ptr()) for t in out), ctypes.c_void_p(stream.cuda_stream))
    return st, out


@pytest.mark.parametrize("nboard,H,seed", [(5, 1326, 0), (4, 1326, 1), (4, 333, 5), (3, 384, 2), (3, 70, 9)])
def test_noalloc_counts_equal_allocating_counts(mtt, cuda, nboard, H, seed):
    import torch
    from importlib import import_module
    lib = import_module("mtt-gpu-solver_b200._lib").lib()
    rng = np.random.default_rng(seed)
    board = rng.choice(52, size=nboard, replace=False).astype(np.uint8)
    all_hands = np.array([(a, b) for a in range(52) for b in range(a + 1, 52)], np.uint8)
    hands = all_hands[np.sort(rng.choice(1326, size=H, replace=False))]
    d_board = torch.from_numpy(board).to(cuda)
    d_hands = torch.from_numpy(np.ascontiguousarray(hands)).to(cuda)
    stream = torch.cuda.current_stream()
    st, ref = _counts(lib, "mtt_board_showdown_counts", d_board, d_hands, stream)
    assert st == MTT_OK
    for _ in range(2):
        st, got = _counts(lib, "mtt_board_showdown_counts_noalloc", d_board, d_hands, stream)
        assert st == MTT_OK
        torch.cuda.synchronize()
        for a, b in zip(ref, got):
            assert torch.equal(a, b)


def test_noalloc_counts_reject_sizes_over_the_limit(mtt, cuda):
    import torch
    from importlib import import_module
    lib = import_module("mtt-gpu-solver_b200._lib").lib()
    d_board = torch.tensor([0, 5, 10], dtype=torch.uint8, device=cuda)
    all_hands = np.array([(a, b) for a in range(52) for b in range(a + 1, 52)], np.uint8)
    d_hands = torch.from_numpy(np.ascontiguousarray(all_hands[:385])).to(cuda)
    st, out = _counts(lib, "mtt_board_showdown_counts_noalloc", d_board, d_hands, torch.cuda.current_stream())
    assert st == MTT_ERR_UNSUPPORTED
    torch.cuda.synchronize()
    assert all(bool((t == -7).all()) for t in out)     # nothing was written
