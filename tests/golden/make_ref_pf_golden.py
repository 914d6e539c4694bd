"""Regenerate tests/golden/ref_pf_dcfr.npz: the reference's own preflop DCFR
loop, as a known answer for the preflop chain's solve.

oracle/_ref/ref_pf_dcfr (built by `make -C oracle ref` from the reference's
src/preflop/preflop_grid_generator.cu with its own --use_fast_math) runs the
loop kernels of preflop_gen (:228-421, host loop :545-614) for 500 iterations
over the shipped flop subset (tests/golden/mtt_subset.bin), 20 bb stacks,
bubble factor 1.35 and 2.5 bb of dead money, as preflop_gen does.  Its inputs,
the all-in matrix and the 100 class-reduced flop matrices in reference mode,
come from this build's library; their SHA-256 must equal the ones in
tests/golden/preflop_ref.json, the oracle's pinned full-size results.  The
reference's own all-in kernel is not run (it writes past a local array when a
sampled hand repeats a card).

Run on a machine with a GPU, after `make -C oracle ref`:
    python tests/golden/make_ref_pf_golden.py [--out tests/golden/ref_pf_dcfr.npz]
"""
import argparse
import hashlib
import importlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_pf_dcfr")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "ref_pf_dcfr.npz"))
    a = ap.parse_args()
    pf = importlib.import_module("mtt-gpu-solver_b200.preflop")
    g = json.load(open(os.path.join(HERE, "preflop_ref.json")))
    subset_path = os.path.join(HERE, "mtt_subset.bin")
    flops, _ = pf.read_subset(subset_path)
    allin = pf.allin_matrix(pf.REFERENCE).cpu().numpy().astype("<f4")
    mats = pf.flop_class_matrices(flops, pf.REFERENCE).cpu().numpy().astype("<f4")
    assert hashlib.sha256(allin.tobytes()).hexdigest() == g["allin_f32_sha256"]
    assert hashlib.sha256(mats.tobytes()).hexdigest() == g["class_mats_sha256"]
    records = open(subset_path, "rb").read()[4:]            # c1, c2, c3, pad, f32 weight per flop
    assert len(records) == 8 * len(flops)
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            f.write(np.array([len(flops), g["dcfr_iters"]], "<i4").tobytes())
            f.write(np.array([g["stack_bb"], g["bubble"], g["dead_pot"]], "<f4").tobytes())
            f.write(records)
            f.write(mats.tobytes())
            f.write(allin.tobytes())
        subprocess.run([HARNESS, fin, fout], check=True, timeout=600)
        out = np.fromfile(fout, "<f4").reshape(2, 10, 192)
    np.savez_compressed(a.out, sums=out[0], sigma=out[1], iters=np.int32(g["dcfr_iters"]),
                        stack_bb=np.float32(g["stack_bb"]), bubble=np.float32(g["bubble"]),
                        dead_pot=np.float32(g["dead_pot"]), allin_f32_sha256=g["allin_f32_sha256"],
                        class_mats_sha256=g["class_mats_sha256"])
    ref = np.asarray(g["sums"], np.float32)
    print("wrote", a.out, "max |sums - oracle| / max:", float(np.abs(out[0] - ref).max() / np.abs(ref).max()))


if __name__ == "__main__":
    main()
