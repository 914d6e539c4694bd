"""CPU tests of the flop-subset optimiser's oracle, its golden fixture and the host side of its C ABI.

The oracle (oracle/pysubset.py) restates scripts/optimize_subset.py with its
own Lawson-Hanson NNLS; it is pinned here against scipy.optimize.nnls (the
reference's solver) and against the reference's shipped mtt_subset.bin /
mtt_subset_weights.txt through tests/golden/subset_nnomp.json.
"""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

import pysubset

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def fixture():
    return json.load(open(os.path.join(GOLDEN, "subset_nnomp.json")))


@pytest.fixture(scope="module")
def shipped():
    return json.load(open(os.path.join(GOLDEN, "golden.json")))


def test_nnls_known_answers():
    # the two examples of scipy.optimize.nnls's documentation
    x, rn = pysubset.nnls(np.array([[1.0, 0], [1, 0], [0, 1]]), np.array([2.0, 1, 1]))
    assert np.allclose(x, [1.5, 1.0], rtol=0, atol=1e-14) and abs(rn - 0.5 ** 0.5) < 1e-14
    x, rn = pysubset.nnls(np.array([[1.0, 0], [1, 0], [0, 1]]), np.array([-1.0, -1, -1]))
    assert np.array_equal(x, [0.0, 0.0]) and abs(rn - 3 ** 0.5) < 1e-14


@pytest.mark.parametrize("seed", range(6))
def test_nnls_matches_scipy(seed):
    from scipy.optimize import nnls as scipy_nnls
    rng = np.random.default_rng(seed)
    for _ in range(10):
        m, n = int(rng.integers(4, 70)), int(rng.integers(1, 35))
        A = rng.standard_normal((m, n))
        b = rng.standard_normal(m)
        x1, r1 = pysubset.nnls(A, b)
        x2, r2 = scipy_nnls(A, b)
        assert np.array_equal(x1 == 0, x2 == 0)
        assert np.abs(x1 - x2).max() <= 1e-10 * max(1.0, np.abs(x2).max())
        assert abs(r1 - r2) <= 1e-10 * max(1.0, r2)


def test_flop_meta_matches_canonical_flops(mtt):
    # the dump's column order: mtt_canonical_flops (host only) and the script's list agree
    assert np.array_equal(mtt.canonical_flops(), np.array(pysubset.flop_meta(), dtype=np.uint8))


def test_fixture_reproduces_shipped_files(fixture, shipped):
    meta = pysubset.flop_meta()
    idx, w = np.array(fixture["indices"]), np.array(fixture["weights"])
    raw = pysubset.subset_bin_bytes(meta, idx, w)
    assert raw == open(os.path.join(GOLDEN, "mtt_subset.bin"), "rb").read()
    assert hashlib.sha256(raw).hexdigest() == shipped["subset_sha256"] == fixture["subset_sha256"]
    txt = pysubset.subset_weights_text(meta, idx, w).encode()
    assert hashlib.sha256(txt).hexdigest() == shipped["subset_weights_sha256"]
    assert len(idx) == len(set(idx.tolist())) == 100
    assert abs(w.sum() - 1755.0) < 1e-9 and (w >= 0).all() and (w == 0).sum() == 5


def test_fixture_is_far_from_ties(fixture):
    # every selection and every active set of the shipped run is decided by a
    # margin far above FP64 (and FP32-feature) rounding
    assert min(fixture["step_gap"]) > 1e-5
    assert max(fixture["step_zero_dual"]) < -1e-6
    assert min(fixture["step_min_weight"]) > 1e-4


def test_c_writer_matches_reference_format(mtt, fixture, shipped, tmp_path):
    sub = __import__("importlib").import_module("mtt-gpu-solver_b200.subset")
    cf = mtt.canonical_flops()
    idx = np.array(fixture["indices"])
    b, t = str(tmp_path / "s.bin"), str(tmp_path / "s.txt")
    sub.write(b, t, cf[idx, :3], np.array(fixture["weights"]))
    assert hashlib.sha256(open(b, "rb").read()).hexdigest() == shipped["subset_sha256"]
    assert hashlib.sha256(open(t, "rb").read()).hexdigest() == shipped["subset_weights_sha256"]
    # the preflop reader takes it back
    pf = __import__("importlib").import_module("mtt-gpu-solver_b200.preflop")
    flops, wf = pf.read_subset(b)
    assert np.array_equal(flops, cf[idx, :3]) and np.array_equal(wf, np.float32(fixture["weights"]))


def test_c_writer_rejects_bad_cards(mtt, tmp_path):
    lib = mtt._lib.lib()
    f = np.array([[0, 1, 52]], np.uint8)
    w = np.ones(1)
    assert lib.mtt_subset_write(str(tmp_path / "x.bin").encode(), None, f.ctypes.data, w.ctypes.data, 1) == 1
    assert lib.mtt_subset_write(None, None, None, None, -1) == 1


def test_nnomp_abi_rejects_bad_arguments(mtt):
    # validated before any device work, so no GPU is needed
    lib = mtt._lib.lib()
    buf = np.zeros(64, np.float64)
    p = ctypes.c_void_p(buf.ctypes.data)
    assert lib.mtt_subset_nnomp(None, 10, 4, p, 2, p, p, None) == 1
    assert lib.mtt_subset_nnomp(p, 10, 4, p, 11, p, p, None) == 1      # more selections than columns
    assert lib.mtt_subset_nnomp(p, 500, 4, p, 129, p, p, None) == 1    # above MTT_SUBSET_MAX_SELECT
    assert lib.mtt_subset_nnomp(p, 10, 0, p, 2, p, p, None) == 1


def test_oracle_nnomp_greedy_and_kkt():
    # a small synthetic problem: each pick is the best normalised correlation
    # with the residual of the previous fit, and the last fit meets the NNLS
    # optimality conditions
    rng = np.random.default_rng(3)
    ncols, nfeat, k = 90, 40, 12
    basis = rng.standard_normal((6, nfeat))
    dump = (rng.random((ncols, 6)) @ basis + 0.3 * rng.standard_normal((ncols, nfeat))).astype(np.float32)
    colw = rng.integers(1, 5, ncols).astype(np.float64)
    idx, w = pysubset.nnomp(dump, colw, k)
    A = dump.T.astype(np.float64)
    b = A @ colw / colw.sum()
    sel, r = [], b.copy()
    for j in idx:
        c = (A.T @ r) / np.linalg.norm(A, axis=0)
        c[sel] = -np.inf
        assert int(np.argmax(c)) == j
        sel.append(int(j))
        x, _ = pysubset.nnls(A[:, sel], b)
        r = b - A[:, sel] @ x
    dual = A[:, sel].T @ r
    assert (x >= 0).all()
    assert np.abs(dual[x > 0]).max() < 1e-8 * np.abs(A[:, sel].T @ b).max()
    assert (dual[x == 0] <= 1e-8 * np.abs(A[:, sel].T @ b).max()).all()
    assert np.allclose(w, x * ncols / x.sum(), rtol=1e-14, atol=0)


def test_subset_module_finds_its_package_when_run_as_a_script():
    # `python -m <package>.subset` runs the file as a script; its package lookup
    # must still return the package.  A fresh interpreter runs the module the
    # way -m does (no GPU needed to check that).
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import runpy; g = runpy.run_module('mtt-gpu-solver_b200.subset', run_name='__script__'); "
            "print(g['_pkg']().__name__, hasattr(g['_pkg'](), 'canonical_flops'))")
    r = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.split() == ["mtt-gpu-solver_b200", "True"]


def test_c_writer_matches_python_formatting_on_any_weights(mtt, tmp_path):
    # the drop-in writer formats like the reference script for any weight: %.4f
    # of the exact binary value (round half to even there) and f32 rounding
    sub = __import__("importlib").import_module("mtt-gpu-solver_b200.subset")
    rng = np.random.default_rng(5)
    meta = pysubset.flop_meta()
    idx = rng.choice(1755, 200, replace=False)
    w = np.concatenate([rng.lognormal(0.0, 2.0, 180),
                        [0.0, 5e-5, 1.5e-4, 2.5e-4, 0.00015, 0.99995, 1755.0, 1e-12, 123.45675, 3.4e38,
                         0.125, 0.0625, 1.00005, 2.00005, 7e-5, 9.99995, 0.5, 17.55, 1e-45, 6.1e-5]])
    cf = np.array(meta, dtype=np.uint8)
    b, t = str(tmp_path / "w.bin"), str(tmp_path / "w.txt")
    sub.write(b, t, cf[idx, :3], w)
    assert open(b, "rb").read() == pysubset.subset_bin_bytes(meta, idx, w)
    assert open(t).read() == pysubset.subset_weights_text(meta, idx, w)


def test_fixture_fit_reproduces_published_r2(fixture):
    # the reference's README.md:7 publishes R^2 = 0.999984 for this selection's fit
    assert round(fixture["fit_r2"], 6) == 0.999984


@pytest.mark.parametrize("seed", [11, 12, 13])
def test_oracle_nnomp_matches_the_loop_with_scipy_nnls(seed):
    # the same greedy loop with the reference's solver (scipy.optimize.nnls) in
    # place of the oracle's own Lawson-Hanson: same selections, same weights
    from scipy.optimize import nnls as scipy_nnls
    rng = np.random.default_rng(seed)
    ncols, nfeat, k = 200, 60, 25
    basis = rng.standard_normal((8, nfeat))
    dump = (rng.random((ncols, 8)) @ basis + 0.4 * rng.standard_normal((ncols, nfeat))).astype(np.float32)
    colw = rng.integers(1, 25, ncols).astype(np.float64)
    idx, w = pysubset.nnomp(dump, colw, k)
    A = dump.T
    b = (A @ colw) / colw.sum()
    An = A / np.linalg.norm(A, axis=0)
    sel, r = [], b.copy()
    for _ in range(k):
        c = An.T @ r
        c[sel] = -np.inf
        sel.append(int(np.argmax(c)))
        x, _ = scipy_nnls(A[:, sel], b)
        r = b - A[:, sel] @ x
    assert idx.tolist() == sel
    ws = x * (ncols / x.sum())
    assert np.array_equal(w == 0, ws == 0)
    assert np.abs(w - ws).max() <= 1e-9 * ws.max()
