"""Regenerate tests/golden/subset_nnomp.json: the flop-subset optimiser's known answer.

The reference's scripts/optimize_subset.py turns data/mtt_ev_dump_1755.bin
into data/mtt_subset.bin and data/mtt_subset_weights.txt by greedy
non-negative orthogonal matching pursuit.  This script runs the oracle's
restatement of it (oracle/pysubset.py) on the shipped dump, checks that its
output files are byte-identical to the two shipped files, and records:

  - the 100 selected column indices in selection order and their FP64
    normalised weights (the shipped file holds the weights only as f32);
  - per step, how far the selection is from a tie (relative gap between the
    best and second-best correlation) and how far each least-squares
    subproblem is from a degenerate active set (the largest dual of a zero
    weight, and the smallest positive weight, both relative);
  - the coefficient of determination R^2 of the final fit against the target,
    the figure the reference's README.md:7 publishes (0.999984).

Run once where the reference is mounted:
    python tests/golden/make_subset_golden.py /path/to/MTT-GPU-Solver
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import pysubset  # noqa: E402


def main(ref_root):
    dump = np.fromfile(os.path.join(ref_root, "data", "mtt_ev_dump_1755.bin"), dtype="<f4")
    dump = dump.reshape(1755, pysubset.N_FEATURES)
    meta = pysubset.flop_meta()
    idx, w, tr = pysubset.nnomp(dump, [m[3] for m in meta], 100, trace=True)
    bin_bytes = pysubset.subset_bin_bytes(meta, idx, w)
    txt = pysubset.subset_weights_text(meta, idx, w)
    assert bin_bytes == open(os.path.join(ref_root, "data", "mtt_subset.bin"), "rb").read()
    assert txt == open(os.path.join(ref_root, "data", "mtt_subset_weights.txt")).read()
    A = dump.T.astype(np.float64)
    colw = np.array([m[3] for m in meta], np.float64)
    target = A @ colw / colw.sum()
    fit = A[:, idx] @ (w * (np.sum(pysubset.nnls(A[:, idx], target)[0]) / len(meta)))
    r2 = 1.0 - np.sum((target - fit) ** 2) / np.sum((target - target.mean()) ** 2)
    out = {
        "source": "oracle/pysubset.py on MTT-GPU-Solver data/mtt_ev_dump_1755.bin; "
                  "its outputs equal data/mtt_subset.bin and data/mtt_subset_weights.txt byte for byte",
        "indices": [int(i) for i in idx],
        "weights": [float(x) for x in w],
        "subset_sha256": hashlib.sha256(bin_bytes).hexdigest(),
        "weights_txt_sha256": hashlib.sha256(txt.encode()).hexdigest(),
        "step_gap": tr["gap"],
        "step_zero_dual": tr["zero_dual"],
        "step_min_weight": tr["min_weight"],
        "fit_r2": float(r2),
    }
    with open(os.path.join(HERE, "subset_nnomp.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(f"min gap {min(tr['gap']):.3g}, max zero dual {max(tr['zero_dual']):.3g}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MTT_REFERENCE", "."))
