"""Regenerate the golden fixtures in this folder from the reference's shipped data.

The reference (MTT-GPU-Solver) ships one end-to-end known answer for the hot
path: data/mtt_ev_dump_1755.bin, the f32 [1755 flops][4 scenarios][2 players]
[169 classes] output of its ev_dumper (src/tools/mtt_ev_dumper.cu:118-176).
This script copies a spread of per-flop slices of that file and the SHA-256 of
the whole file (so a full regeneration can be checked without the 9.5 MB
file), plus the 804-byte data/mtt_subset.bin input of preflop_gen
(src/preflop/preflop_grid_generator.cu:446-457) and the SHA-256 of
data/mtt_subset_weights.txt.

Run once where the reference is mounted:
    python tests/golden/make_golden.py /path/to/MTT-GPU-Solver
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# a spread over the three flop families of generate_all_1755_flops
# (trips 0-12, paired 13-324, unpaired 325-1754)
SLICE_FLOPS = [0, 1, 7, 12, 13, 14, 100, 201, 324, 325, 326, 327, 328, 329,
               600, 777, 1000, 1234, 1500, 1753, 1754]
FLOATS_PER_FLOP = 4 * 2 * 169


def main(ref_root):
    dump_path = os.path.join(ref_root, "data", "mtt_ev_dump_1755.bin")
    raw = open(dump_path, "rb").read()
    assert len(raw) == 1755 * FLOATS_PER_FLOP * 4, len(raw)
    dump = np.frombuffer(raw, dtype="<f4").reshape(1755, FLOATS_PER_FLOP)
    np.asarray(dump[SLICE_FLOPS], dtype="<f4").tofile(os.path.join(HERE, "ev_dump_slices.f32"))
    subset = open(os.path.join(ref_root, "data", "mtt_subset.bin"), "rb").read()
    open(os.path.join(HERE, "mtt_subset.bin"), "wb").write(subset)
    weights_txt = open(os.path.join(ref_root, "data", "mtt_subset_weights.txt"), "rb").read()
    meta = {
        "source": "MTT-GPU-Solver data/ (reference shipped outputs)",
        "ev_dump_sha256": hashlib.sha256(raw).hexdigest(),
        "ev_dump_bytes": len(raw),
        "slice_flops": SLICE_FLOPS,
        "slice_file": "ev_dump_slices.f32",
        "subset_sha256": hashlib.sha256(subset).hexdigest(),
        "subset_weights_sha256": hashlib.sha256(weights_txt).hexdigest(),
    }
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1)
        f.write("\n")
    print("wrote", len(SLICE_FLOPS), "flop slices;", meta["ev_dump_sha256"])


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MTT_REFERENCE")
    if not root:
        sys.exit("usage: make_golden.py REFERENCE_ROOT  (or set MTT_REFERENCE)")
    main(root)
