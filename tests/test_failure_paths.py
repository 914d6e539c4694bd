"""Failure detection without a GPU fault.

* Bounded device waits (GPU): mtt_selftest_bounded_wait makes one CTA wait on
  an mbarrier that nothing arrives on and no copy targets, with a 2 ms limit.
  The call must return MTT_ERR_TIMEOUT, and the device must stay usable: the
  same wait with an arrival, an evaluator batch and a small solve succeed
  afterwards.
* File errors (CPU): the preflop driver's subset reader
  (preflop_grid_generator.cu:446-459) and the subset optimiser's dump reader
  return MTT_ERR_IO / a non-zero exit on missing, truncated and corrupt files,
  and never read past the data.
"""
import ctypes
import os
import struct
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _status(mtt, name):
    return getattr(mtt._lib, name)


@pytest.mark.gpu
def test_bounded_wait_times_out_and_device_stays_usable(mtt, orc, wl, cuda):
    import torch
    L = mtt.lib()
    timeout = _status(mtt, "MTT_ERR_TIMEOUT")
    assert L.mtt_selftest_bounded_wait(0, 2000, None) == timeout
    assert L.mtt_selftest_bounded_wait(1, 2000, None) == 0
    assert L.mtt_selftest_bounded_wait(0, 2000, None) == timeout     # repeatable
    assert L.mtt_selftest_bounded_wait(0, 0, None) == _status(mtt, "MTT_ERR_INVALID")
    # the context is intact: an evaluator batch and a solve still agree with the oracle
    rng = np.random.default_rng(1)
    hands = np.stack([rng.choice(52, size=7, replace=False) for _ in range(1000)]).astype(np.uint8)
    got = mtt.eval7(torch.from_numpy(hands).to(cuda)).cpu().numpy().view(np.uint32)
    assert np.array_equal(got, orc.eval7(hands))
    sub = wl.river_uniform(seed=3, n_hands=80)
    b = mtt.RiverBatch([sub])
    b.solve(mtt.solve_params(iters=1, threads=128))
    b.check()
    r = b.read(0)
    b.close()
    o = orc.cfr_solve(sub, 1, alternate=1)
    for k in ("R0", "R1", "S0", "S1"):
        assert np.abs(o[k] - r[k]).max() <= 1e-4 * max(1e-12, float(np.abs(o[k]).max())), k


def _read_subset(mtt, path, capacity=200):
    L = mtt.lib()
    n = ctypes.c_int32(-1)
    flops = np.zeros(3 * capacity, np.uint8)
    w = np.zeros(capacity, np.float32)
    st = L.mtt_pf_read_subset(path.encode() if path else None, flops.ctypes.data, w.ctypes.data, capacity,
                              ctypes.byref(n))
    return st, n.value, flops, w


def _write_subset(path, recs, count=None):
    with open(path, "wb") as f:
        f.write(struct.pack("<I", len(recs) if count is None else count))
        for (a, b, c), wt in recs:
            f.write(bytes([a, b, c, 0]) + struct.pack("<f", wt))


def test_subset_reader_reports_io_errors(mtt, tmp_path):
    io_err = _status(mtt, "MTT_ERR_IO")
    recs = [((51, 46, 23), 3.5), ((0, 1, 20), 1.25), ((4, 8, 12), 0.5)]
    good = str(tmp_path / "good.bin")
    _write_subset(good, recs)
    st, n, flops, w = _read_subset(mtt, good)
    assert st == 0 and n == 3
    assert list(flops[:9]) == [51, 46, 23, 0, 1, 20, 4, 8, 12]
    assert np.allclose(w[:3], [3.5, 1.25, 0.5])
    # missing file
    assert _read_subset(mtt, str(tmp_path / "absent.bin"))[0] == io_err
    # shorter than its count header
    short = str(tmp_path / "short.bin")
    _write_subset(short, recs, count=10)
    assert _read_subset(mtt, short)[0] == io_err
    # cut inside a record
    cut = str(tmp_path / "cut.bin")
    data = open(good, "rb").read()
    open(cut, "wb").write(data[:4 + 8 + 5])
    assert _read_subset(mtt, cut)[0] == io_err
    # cut inside the count header
    open(cut, "wb").write(data[:2])
    assert _read_subset(mtt, cut)[0] == io_err
    # empty file
    open(cut, "wb").write(b"")
    assert _read_subset(mtt, cut)[0] == io_err
    # a card outside 0..51
    bad = str(tmp_path / "bad.bin")
    _write_subset(bad, [((51, 46, 23), 1.0), ((0, 60, 20), 1.0)])
    assert _read_subset(mtt, bad)[0] == io_err
    # an absurd count
    huge = str(tmp_path / "huge.bin")
    _write_subset(huge, recs, count=0xFFFFFFF0)
    assert _read_subset(mtt, huge)[0] == io_err
    # more records than the caller's capacity: invalid argument, not an overrun
    assert _read_subset(mtt, good, capacity=2)[0] == _status(mtt, "MTT_ERR_INVALID")


def test_subset_optimizer_rejects_a_truncated_dump(tmp_path):
    exe = os.path.join(ROOT, "mtt-gpu-solver_b200", "bin", "subset_optimizer")
    if not os.path.isfile(exe):
        pytest.skip("drivers not built")
    dump = tmp_path / "mtt_ev_dump_1755.bin"
    dump.write_bytes(np.zeros(1755 * 1352 - 7, np.float32).tobytes())    # 7 floats short
    r = subprocess.run([exe, "--dump", str(dump)], cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "cannot read" in r.stderr
    assert not (tmp_path / "mtt_subset.bin").exists()
    r = subprocess.run([exe, "--dump", str(tmp_path / "absent.bin")], cwd=tmp_path, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode != 0 and not (tmp_path / "mtt_subset.bin").exists()
