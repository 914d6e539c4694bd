"""The flop-subset optimiser on the GPU (mtt_subset_nnomp) against the oracle
(oracle/pysubset.py) and against the reference's shipped subset files.

Selections must be identical; FP64 weights agree to 1e-9 of the largest
weight (the device solves the normal equations from the previous step's
weights, the oracle least squares from zero: rounding differs, the solution
does not); zero weights must be exactly zero in both.  Each synthetic case's
oracle run is checked to be far from a tie first, so the comparison is
well posed."""
import hashlib
import importlib
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import pysubset

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def sub():
    return importlib.import_module("mtt-gpu-solver_b200.subset")


def _synth(ncols, nfeat, seed, zero_col=False):
    rng = np.random.default_rng(seed)
    basis = rng.standard_normal((8, nfeat))
    cols = (rng.random((ncols, 8)) @ basis + 0.5 * rng.standard_normal((ncols, nfeat))).astype(np.float32)
    if zero_col:
        cols[ncols // 3] = 0.0
    colw = rng.integers(1, 25, ncols).astype(np.float64)
    return cols, colw


# (ncols, nfeat, nselect, seed, zero column): float4 and scalar feature paths,
# the largest subproblem (128 columns), every column selected, one step
CASES = [(400, 96, 40, 0, False), (333, 130, 30, 1, True), (600, 260, 60, 2, False), (300, 200, 128, 3, False),
         (16, 40, 16, 4, False), (50, 7, 1, 5, False)]


@pytest.mark.parametrize("ncols,nfeat,nselect,seed,zero_col", CASES)
def test_nnomp_matches_oracle(sub, cuda, ncols, nfeat, nselect, seed, zero_col):
    import torch
    cols, colw = _synth(ncols, nfeat, seed, zero_col)
    oi, ow, tr = pysubset.nnomp(cols, colw, nselect, trace=True)
    assert min(tr["gap"]) > 1e-6 and max(tr["zero_dual"]) < -1e-9
    gi, gw = sub.nnomp(torch.from_numpy(cols).to(cuda), colw, nselect)
    assert np.array_equal(gi, oi)
    assert np.array_equal(gw == 0, ow == 0)
    assert np.abs(gw - ow).max() <= 1e-9 * ow.max()


def test_nnomp_is_deterministic(sub, cuda):
    import torch
    cols, colw = _synth(600, 260, 2)
    c = torch.from_numpy(cols).to(cuda)
    a = sub.nnomp(c, colw, 60)
    b = sub.nnomp(c, colw, 60)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1].view(np.uint64), b[1].view(np.uint64))


def test_nnomp_rejects_more_selections_than_columns(mtt, sub, cuda):
    import torch
    cols, colw = _synth(10, 8, 0)
    with pytest.raises(mtt.MttError):
        sub.nnomp(torch.from_numpy(cols).to(cuda), colw, 11)


def test_regenerated_dump_gives_the_shipped_subset(mtt, sub, cuda, tmp_path):
    # ev_dump on every canonical flop (bit-exact with the shipped dump), then
    # NN-OMP on the device, then the reference's file formats
    meta = json.load(open(os.path.join(GOLDEN, "golden.json")))
    fx = json.load(open(os.path.join(GOLDEN, "subset_nnomp.json")))
    flops, w, idx = sub.optimize(None, 100)
    assert idx.tolist() == fx["indices"]
    want = np.array(fx["weights"])
    assert np.array_equal(w == 0, want == 0)
    assert np.abs(w - want).max() <= 1e-9 * want.max()
    b, t = str(tmp_path / "mtt_subset.bin"), str(tmp_path / "mtt_subset_weights.txt")
    sub.write(b, t, flops, w)
    assert open(b, "rb").read() == open(os.path.join(GOLDEN, "mtt_subset.bin"), "rb").read()
    assert hashlib.sha256(open(t, "rb").read()).hexdigest() == meta["subset_weights_sha256"]


def test_subset_module_cli_reads_a_dump_file(mtt, sub, cuda, tmp_path):
    import torch
    meta = json.load(open(os.path.join(GOLDEN, "golden.json")))
    f3 = torch.from_numpy(np.ascontiguousarray(mtt.canonical_flops()[:, :3])).to(cuda)
    dump = mtt.ev_dump(f3).cpu().numpy()
    dump.astype("<f4").tofile(tmp_path / "mtt_ev_dump_1755.bin")
    assert sub.main(["--dump", str(tmp_path / "mtt_ev_dump_1755.bin"), "--out-dir", str(tmp_path)]) == 0
    assert hashlib.sha256((tmp_path / "mtt_subset.bin").read_bytes()).hexdigest() == meta["subset_sha256"]


def test_subset_module_runs_as_a_script(cuda, tmp_path):
    # python -m <package>.subset --regenerate: the device dump, then the selection
    meta = json.load(open(os.path.join(GOLDEN, "golden.json")))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-m", "mtt-gpu-solver_b200.subset", "--regenerate", "--out-dir", str(tmp_path)],
                       capture_output=True, text=True, timeout=600, cwd=root)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Subset generated: 100 flops saved to mtt_subset.bin" in r.stdout
    assert hashlib.sha256((tmp_path / "mtt_subset.bin").read_bytes()).hexdigest() == meta["subset_sha256"]
    txt = (tmp_path / "mtt_subset_weights.txt").read_bytes()
    assert hashlib.sha256(txt).hexdigest() == meta["subset_weights_sha256"]
