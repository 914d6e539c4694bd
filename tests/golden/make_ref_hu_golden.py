"""Regenerate tests/golden/ref_hu_river.npz: the reference's own heads-up CFR+
kernels on a river subgame, as a known answer for the sweeps.

oracle/_ref/ref_hu_sweeps (built by `make -C oracle ref` from the reference's
src/postflop/honest_multistreet_solver.cu) runs kernel_forward_sweep /
kernel_evaluate_terminals / kernel_backward_sweep (:88-249) for 1 and 4
iterations on a seeded river subgame:
  - a river tree (pot 100, stack 200, a 75% pot bet plus all-in, one raise) in
    the reference's FlatNode layout: the reference's arrays hold at most three
    actions per node (MAX_ACTIONS, :12), so the river configuration's two bet
    sizes do not fit;
  - 700 seeded live combos for both players, all below combo 1,024 (the
    kernels sum a fold's opponent mass inside one 1,024-thread CTA), with
    different lognormal range weights per player.
The kernels' semantics are this build's MTT_SEM_REFERENCE with simultaneous
updates and linear strategy averaging.  The regrets, strategy sums and root
counterfactual values are stored in the oracle's row layout (R_p[row][hand]).

Run on a machine with a GPU, after `make -C oracle ref`:
    python tests/golden/make_ref_hu_golden.py [--out tests/golden/ref_hu_river.npz]
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
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_hu_sweeps")
PAD = 1216
ITERS = (1, 4)


def subgame():
    wl = importlib.import_module("mtt-gpu-solver_b200.workloads")
    sub = wl.river_uniform(seed=21, n_hands=700, bet_sizes=(0.75,))
    assert int(np.max(sub["nodes"]["num_actions"])) <= 3
    rng = np.random.default_rng(22)
    for p in (0, 1):
        w = rng.lognormal(0.0, 1.0, len(sub[f"combos{p}"])).astype(np.float32)
        sub[f"range{p}"] = (w / w.sum()).astype(np.float32)
    return sub


def run_reference(sub, iters):
    """(R0, R1, S0, S1, cfv0, cfv1) of the reference kernels after iters iterations."""
    nodes = np.array(sub["nodes"], copy=True)
    dec = np.where(nodes["type"] == 0)[0]
    gid = {int(n): g for g, n in enumerate(dec)}
    ref_nodes = nodes.copy()
    ref_nodes["infoset_offset"][dec] = np.arange(len(dec))
    ref_nodes["turn_idx"] = 0
    combos = np.asarray(sub["combos0"], np.int64)
    assert np.array_equal(combos, np.asarray(sub["combos1"], np.int64)) and len(combos) <= 1024
    cc = np.array([(a, b) for a in range(52) for b in range(a + 1, 52)], np.uint8)[combos]
    H = len(combos)
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            f.write(np.array([len(nodes), H, iters, len(dec)], "<i4").tobytes())
            f.write(ref_nodes.tobytes())
            f.write(cc.tobytes())
            f.write(np.asarray(sub["board"], np.uint8).tobytes())
            f.write(np.asarray(sub["range0"], "<f4").tobytes())
            f.write(np.asarray(sub["range1"], "<f4").tobytes())
        subprocess.run([HARNESS, fin, fout], check=True, timeout=600)
        raw = np.fromfile(fout, "<f4")
    nR = len(dec) * 3 * PAD
    R, S, cfv = raw[:nR].reshape(-1, PAD), raw[nR:2 * nR].reshape(-1, PAD), raw[2 * nR:].reshape(2, PAD)
    rows = [int(x) for x in sub["rows"]]
    out = {f"R{p}": np.zeros((rows[p], H), np.float32) for p in (0, 1)}
    out.update({f"S{p}": np.zeros((rows[p], H), np.float32) for p in (0, 1)})
    for n in dec:
        nd = nodes[n]
        p, o, g = int(nd["player"]), int(nd["infoset_offset"]), gid[int(n)]
        for a in range(int(nd["num_actions"])):
            out[f"R{p}"][o + a] = R[3 * g + a, :H]
            out[f"S{p}"][o + a] = S[3 * g + a, :H]
    out["cfv0"], out["cfv1"] = cfv[0, :H].copy(), cfv[1, :H].copy()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "ref_hu_river.npz"))
    a = ap.parse_args()
    sub = subgame()
    arrays = {"nodes": sub["nodes"], "rows": np.asarray(sub["rows"], np.int32), "board": np.asarray(sub["board"], np.uint8),
              "combos": np.asarray(sub["combos0"], np.uint16), "range0": sub["range0"], "range1": sub["range1"],
              "pot": np.float32(sub["pot"]), "iters": np.asarray(ITERS, np.int32)}
    for it in ITERS:
        for k, v in run_reference(sub, it).items():
            arrays[f"it{it}_{k}"] = v
    np.savez_compressed(a.out, **arrays)
    print("wrote", a.out, os.path.getsize(a.out), "bytes")


if __name__ == "__main__":
    main()
