"""Regenerates tests/golden/preflop_ref.json: the CPU oracle's restatement of
the reference preflop chain (src/preflop/preflop_grid_generator.cu) in
reference mode over the shipped flop subset (tests/golden/mtt_subset.bin, a
copy of the reference's data/mtt_subset.bin): SHA-256 of the all-in win/tie
counts and of the 100 class-reduced flop matrices, and the strategy sums
after 500 DCFR iterations (stack 20 BB, bubble factor 1.35, dead pot 2.5 BB).

    python tests/golden/make_preflop_golden.py      (about 3 minutes on 8 cores)
"""
import hashlib
import json
import os
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import pyoracle  # noqa: E402


def main():
    raw = open(os.path.join(HERE, "mtt_subset.bin"), "rb").read()
    n = struct.unpack("<I", raw[:4])[0]
    flops = np.zeros((n, 3), np.uint8)
    w = np.zeros(n, np.float32)
    for i in range(n):
        rec = raw[4 + 8 * i: 12 + 8 * i]
        flops[i] = list(rec[:3])
        w[i] = struct.unpack("<f", rec[4:8])[0]
    allin, wins, ties = pyoracle.pf_allin()
    mats = np.stack([pyoracle.pf_flop_class(f) for f in flops])
    sums, sig = pyoracle.pf_dcfr(w, mats, allin, 500)
    out = {
        "subset_flops": int(n),
        "allin_counts_sha256": hashlib.sha256(wins.astype("<i4").tobytes() + ties.astype("<i4").tobytes()).hexdigest(),
        "allin_f32_sha256": hashlib.sha256(allin.astype("<f4").tobytes()).hexdigest(),
        "class_mats_sha256": hashlib.sha256(mats.astype("<f4").tobytes()).hexdigest(),
        "class_mat_sha256": [hashlib.sha256(m.astype("<f4").tobytes()).hexdigest() for m in mats],
        "dcfr_iters": 500, "stack_bb": 20.0, "bubble": 1.35, "dead_pot": 2.5,
        "sums": sums.astype(float).tolist(),
    }
    json.dump(out, open(os.path.join(HERE, "preflop_ref.json"), "w"))
    print("wrote preflop_ref.json")


if __name__ == "__main__":
    main()
