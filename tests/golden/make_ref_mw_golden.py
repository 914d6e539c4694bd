"""Regenerate tests/golden/ref_mw_river.npz: the reference's own four-player
CFR+ kernels on an ICM river subgame, as a known answer for the multiway engine.

oracle/_ref/ref_mw_sweeps (built by `make -C oracle ref` from the reference's
src/postflop/multiway_4way_engine.cu) runs kernel_4way_forward_sweep /
kernel_4way_evaluate_terminals / kernel_4way_backward_cfr_plus (:41-257) for 1
and 4 iterations on a seeded subgame:
  - the four-player ICM river of the multiway configuration (stacks, payouts
    50/30/20 over eight seats, Malmuth-Harville bubble factors, Dirichlet(0.3)
    ranges) with 400 seeded live combos;
  - its tree with one pot-sized bet and one pot-sized raise: the reference's
    arrays hold at most three actions per node (MAX_POST_ACTIONS, :15).
The hands' 7-card scores come from the oracle's evaluator (bit-exact with the
reference's, pinned by the shipped dump); the reference's four-player file has
none.  The kernels' semantics are this build's MTT_SEM_REFERENCE with linear
strategy averaging.  The regrets, strategy sums and root counterfactual values
are stored in the oracle's row layout (R_p[row][hand]).

Run on a machine with a GPU, after `make -C oracle ref`:
    python tests/golden/make_ref_mw_golden.py [--out tests/golden/ref_mw_river.npz]
"""
import argparse
import importlib
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_mw_sweeps")
PAD = 1216
ITERS = (1, 4)


def subgame():
    wl = importlib.import_module("mtt-gpu-solver_b200.workloads")
    mw = importlib.import_module("mtt-gpu-solver_b200.multiway")
    sub = wl.multiway_icm(seed=31, n_hands=400)
    behind = [float(np.round(s - sub["pot"] / 4, 3)) for s in sub["stacks"][:4]]
    nodes, rows, _ = mw.build_tree(sub["pot"], behind, [1.0], 1.0, 1)
    assert int(np.max(nodes["num_actions"])) <= 3
    sub["nodes"], sub["rows"] = nodes, rows
    return sub


def scores(sub):
    import pyoracle
    cc = np.array([(a, b) for a in range(52) for b in range(a + 1, 52)], np.uint8)[np.asarray(sub["combos"], np.int64)]
    c7 = np.concatenate([np.tile(np.asarray(sub["board"], np.uint8), (len(cc), 1)), cc], axis=1)
    return np.asarray(pyoracle.eval7(np.ascontiguousarray(c7)), np.uint32)


def run_reference(sub, iters):
    """{R: [4], S: [4], cfv: [4][H]} of the reference kernels after iters iterations."""
    nodes = np.array(sub["nodes"], copy=True)
    dec = np.where(nodes["type"] == 0)[0]
    ref_nodes = nodes.copy()
    ref_nodes["infoset_offset"][dec] = np.arange(len(dec))
    H = len(sub["combos"])
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            f.write(np.array([len(nodes), H, iters, len(dec)], "<i4").tobytes())
            f.write(ref_nodes.tobytes())
            f.write(scores(sub).astype("<u4").tobytes())
            f.write(np.concatenate([np.asarray(r, "<f4") for r in sub["ranges"]]).tobytes())
            f.write(np.asarray(sub["bubble"], np.float64).reshape(16).astype("<f4").tobytes())
        subprocess.run([HARNESS, fin, fout], check=True, timeout=600)
        raw = np.fromfile(fout, "<f4")
    nR = len(dec) * 3 * PAD
    R, S, cfv = raw[:nR].reshape(-1, PAD), raw[nR:2 * nR].reshape(-1, PAD), raw[2 * nR:].reshape(4, PAD)
    rows = [int(x) for x in sub["rows"]]
    out = {"R": [np.zeros((rows[p], H), np.float32) for p in range(4)],
           "S": [np.zeros((rows[p], H), np.float32) for p in range(4)], "cfv": cfv[:, :H].copy()}
    for g, n in enumerate(dec):
        nd = nodes[n]
        p, o = int(nd["player"]), int(nd["infoset_offset"])
        for a in range(int(nd["num_actions"])):
            out["R"][p][o + a] = R[3 * g + a, :H]
            out["S"][p][o + a] = S[3 * g + a, :H]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "ref_mw_river.npz"))
    a = ap.parse_args()
    sub = subgame()
    arrays = {"nodes": sub["nodes"], "rows": np.asarray(sub["rows"], np.int32), "board": np.asarray(sub["board"], np.uint8),
              "combos": np.asarray(sub["combos"], np.uint16), "ranges": np.stack(sub["ranges"]).astype(np.float32),
              "bubble": np.asarray(sub["bubble"], np.float64).reshape(4, 4), "pot": np.float32(sub["pot"]),
              "iters": np.asarray(ITERS, np.int32)}
    for it in ITERS:
        out = run_reference(sub, it)
        for p in range(4):
            arrays[f"it{it}_R{p}"] = out["R"][p]
            arrays[f"it{it}_S{p}"] = out["S"][p]
        arrays[f"it{it}_cfv"] = out["cfv"]
    np.savez_compressed(a.out, **arrays)
    print("wrote", a.out, os.path.getsize(a.out), "bytes")


if __name__ == "__main__":
    main()
