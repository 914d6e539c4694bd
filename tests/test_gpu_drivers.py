"""The command-line drivers on the GPU, against the library API on the same
inputs: ev_dumper's file bit for bit, preflop_gen's printed table, hu_solver's
printed values and exploitability, multiway_solver's run; ev_dumper then
subset_optimizer reproduce the reference's shipped subset files."""
import hashlib
import json
import os
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "mtt-gpu-solver_b200", "bin")


@pytest.fixture(scope="module", autouse=True)
def _drivers_built():
    """Builds the drivers when a checkout has only the library."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("mtt_build", os.path.join(ROOT, "mtt-gpu-solver_b200", "build.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    b.build_drivers(quiet=True)


def _run(args, cwd=None):
    r = subprocess.run([os.path.join(BIN, args[0])] + args[1:], capture_output=True, text=True, timeout=600, cwd=cwd)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def test_ev_dumper_writes_the_dump_slices(mtt, cuda, tmp_path):
    import torch
    out = _run(["ev_dumper", "--limit", "5"], cwd=tmp_path)
    assert "Successfully exported mtt_ev_dump_1755.bin" in out
    got = np.fromfile(tmp_path / "mtt_ev_dump_1755.bin", dtype="<f4")
    flops = np.ascontiguousarray(mtt.canonical_flops()[:5, :3])
    want = mtt.ev_dump(torch.from_numpy(flops).to(cuda)).cpu().numpy().ravel()
    assert got.shape == want.shape and np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_preflop_gen_prints_the_python_drivers_table(mtt, cuda):
    import importlib
    pf = importlib.import_module("mtt-gpu-solver_b200.preflop")
    subset = os.path.join(ROOT, "tests", "golden", "mtt_subset.bin")
    out = _run(["preflop_gen", "--subset", subset, "--iters", "40"])
    rows = [l.split() for l in out.splitlines() if l[:4].strip() in pf.NAMES and len(l.split()) == 7]
    flops, w = pf.read_subset(subset)
    sums, _ = pf.dcfr(w, pf.flop_class_matrices(flops, pf.REFERENCE), pf.allin_matrix(pf.REFERENCE), iters=40)
    want = pf.strategy_table(sums)
    assert len(rows) == 15
    for r, t in zip(rows, want):
        assert r[0] == t[0] and [f"{x:.3f}" for x in t[1:]] == r[1:], (r, t)


def test_hu_solver_matches_the_batch_api(mtt, wl, cuda):
    board = [51, 46, 23, 8, 2]
    out = _run(["hu_solver", "--config", "0", "--board", ",".join(map(str, board)), "--iters", "300"])
    vals = {k: float(v) for k, v in re.findall(r"(EV0|EV1|BR0|BR1) (-?[0-9.]+)", out)}
    expl = float(re.search(r"exploitability ([0-9.]+) % pot", out).group(1))
    nodes, rows, _ = mtt.build_tree(100.0, 200.0, [0.5, 1.0], raise_cap=1)
    live = mtt.live_combos(board)
    u = np.full(len(live), 1.0 / len(live), np.float32)
    sub = {"nodes": nodes, "rows": rows, "board": board, "combos0": live, "combos1": live, "range0": u, "range1": u,
           "pot": 100.0}
    b = mtt.RiverBatch([sub])
    b.solve(mtt.solve_params(iters=300, alternate=True, avg_power=2.0), graph=True)
    res = b.results()[0]
    b.close()
    for k, i in (("BR0", 0), ("BR1", 1), ("EV0", 2), ("EV1", 3)):
        assert abs(vals[k] - res[i]) <= 1e-5, (k, vals[k], res[i])
    assert abs(expl - res[5] * 100) <= 1e-3 and expl < 1.0


def test_hu_solver_flop_subgame_and_multiway_solver_run(mtt, cuda):
    out = _run(["hu_solver", "--street", "3", "--pot", "100", "--stack", "100", "--bets", "1.0", "--raise-cap", "0",
                "--iters", "40"])
    assert float(re.search(r"exploitability ([0-9.]+) % pot", out).group(1)) < 100.0
    out = _run(["multiway_solver", "--iters", "20"])
    evs = [float(x) for x in re.findall(r"EV (-?[0-9.]+) bb", out)]
    assert len(evs) == 4 and all(np.isfinite(evs))


def test_ev_dumper_then_subset_optimizer_reproduce_the_shipped_subset(tmp_path):
    # the reference's pipeline: ev_dumper writes the dump, optimize_subset.py
    # turns it into mtt_subset.bin and mtt_subset_weights.txt
    meta = json.load(open(os.path.join(ROOT, "tests", "golden", "golden.json")))
    _run(["ev_dumper"], cwd=tmp_path)
    dump = (tmp_path / "mtt_ev_dump_1755.bin").read_bytes()
    assert hashlib.sha256(dump).hexdigest() == meta["ev_dump_sha256"]
    out = _run(["subset_optimizer"], cwd=tmp_path)
    assert "Subset generated: 100 flops saved to mtt_subset.bin" in out
    assert hashlib.sha256((tmp_path / "mtt_subset.bin").read_bytes()).hexdigest() == meta["subset_sha256"]
    txt = (tmp_path / "mtt_subset_weights.txt").read_bytes()
    assert hashlib.sha256(txt).hexdigest() == meta["subset_weights_sha256"]
