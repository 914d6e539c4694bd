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


_RESET_SCRIPT = r'''
import ctypes, importlib, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
lib = importlib.import_module("mtt-gpu-solver_b200._lib").lib()
rt = ctypes.CDLL("libcudart.so.12")          # the runtime the library itself loaded
vp = ctypes.c_void_p

def dev_buf(nbytes):
    p = vp()
    assert rt.cudaMalloc(ctypes.byref(p), ctypes.c_size_t(nbytes)) == 0
    return p

def counts(fn, board, hands):
    H = len(hands)
    db, dh = dev_buf(len(board)), dev_buf(hands.nbytes)
    assert rt.cudaMemcpy(db, board.ctypes.data, ctypes.c_size_t(len(board)), 1) == 0
    assert rt.cudaMemcpy(dh, hands.ctypes.data, ctypes.c_size_t(hands.nbytes), 1) == 0
    outs = [dev_buf(4 * H * H) for _ in range(3)]
    st = getattr(lib, fn)(db, len(board), dh, H, *outs, None)
    assert st == 0, (fn, st)
    assert rt.cudaDeviceSynchronize() == 0
    res = []
    for o in outs:
        a = np.zeros((H, H), np.int32)
        assert rt.cudaMemcpy(a.ctypes.data, o, ctypes.c_size_t(a.nbytes), 2) == 0
        res.append(a)
        rt.cudaFree(o)
    rt.cudaFree(db); rt.cudaFree(dh)
    return res

rng = np.random.default_rng(4)
board = rng.choice(52, size=4, replace=False).astype(np.uint8)
allh = np.array([(a, b) for a in range(52) for b in range(a + 1, 52)], np.uint8)
hands = np.ascontiguousarray(allh[np.sort(rng.choice(1326, size=500, replace=False))])
want = counts("mtt_board_showdown_counts", board, hands)
for a, b in zip(want, counts("mtt_board_showdown_counts_noalloc", board, hands)):
    assert np.array_equal(a, b)
assert rt.cudaDeviceReset() == 0              # ends this process's own context only
for _ in range(2):
    for a, b in zip(want, counts("mtt_board_showdown_counts_noalloc", board, hands)):
        assert np.array_equal(a, b)
print("reset ok")
'''


def test_noalloc_counts_after_device_reset(cuda, tmp_path):
    """In a fresh process (it resets its own context): the counts agree with
    the allocating entry point before and after cudaDeviceReset, because the
    scratch address is looked up again in the new context."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    script = tmp_path / "reset_check.py"
    script.write_text(_RESET_SCRIPT)
    r = subprocess.run([sys.executable, str(script), root], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "reset ok" in r.stdout, r.stdout + r.stderr
