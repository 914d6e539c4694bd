"""Regenerate tests/golden/ref_pf_flop_mats.npz: the reference's own flop
matrices and their class reduction for the first three flops of the shipped
subset.

oracle/_ref/ref_pf_flop_mats (built by `make -C oracle ref` from the
reference's src/preflop/preflop_grid_generator.cu with its own
--use_fast_math) runs kernel_gen_100_flop_matrices and
kernel_reduce_combo_to_class_matrices (:128-223) on inputs built as
preflop_gen builds them: the first 1,176 combos, each class listing up to 12
of them in order.  Each combo's class comes from mtt_pf_combo_class (the
reference's numbering).  The fixture stores the reference's [3][169][169]
class matrices ([flop][villain][hero]).

Run on a machine with a GPU, after `make -C oracle ref`:
    python tests/golden/make_ref_pf_mats_golden.py [--out tests/golden/ref_pf_flop_mats.npz]
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
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_pf_flop_mats")
N_FLOPS = 3


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "ref_pf_flop_mats.npz"))
    a = ap.parse_args()
    pf = importlib.import_module("mtt-gpu-solver_b200.preflop")
    records = open(os.path.join(HERE, "mtt_subset.bin"), "rb").read()[4:4 + 8 * N_FLOPS]
    flops = np.frombuffer(records, np.uint8).reshape(N_FLOPS, 8)[:, :3].copy()
    combos = [(c1, c2) for c1 in range(52) for c2 in range(c1 + 1, 52)][:1176]
    cls = np.array([pf.lib().mtt_pf_combo_class(c1, c2) for c1, c2 in combos], "<i2")
    assert cls.min() >= 0 and cls.max() <= 168
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            f.write(np.array([N_FLOPS], "<i4").tobytes())
            f.write(records)
            f.write(cls.tobytes())
        subprocess.run([HARNESS, fin, fout], check=True, timeout=600)
        ref = np.fromfile(fout, "<f4").reshape(N_FLOPS, 169, 169)
    ours = pf.flop_class_matrices(flops, pf.REFERENCE).cpu().numpy()
    same = int(np.sum(ref.view(np.uint32) == ours.view(np.uint32)))
    np.savez_compressed(a.out, flops=flops, class_mats=ref)
    print("wrote", a.out, "bit-identical entries vs the library:", same, "of", ref.size,
          "max |diff|:", float(np.abs(ref - ours).max()))


if __name__ == "__main__":
    main()
