"""Drives the reference's own heads-up sweep kernels (oracle/_ref/ref_hu_sweeps).

TEST INFRASTRUCTURE ONLY: the fixture generator and bench.py's reference-kernel
leg use it.  oracle/_ref/ref_hu_sweeps is built by `make -C oracle ref
REF=<MTT-GPU-Solver checkout>` from the reference's
src/postflop/honest_multistreet_solver.cu (kernel_forward_sweep /
kernel_evaluate_terminals / kernel_backward_sweep, :88-249) and needs a GPU.

The kernels hold at most three actions per node (MAX_ACTIONS, :12) and sum a
fold's opponent mass inside one 1,024-thread CTA, so a subgame they run has at
most three actions per node and at most 1,024 hands, the same list for both
players (the harness checks both before any launch).
"""
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HARNESS = os.path.join(HERE, "_ref", "ref_hu_sweeps")
PAD = 1216
_CC = np.array([(a, b) for a in range(52) for b in range(a + 1, 52)], np.uint8)


def available():
    return os.path.isfile(HARNESS) and os.access(HARNESS, os.X_OK)


def _write_input(sub, iters, path):
    nodes = np.array(sub["nodes"], copy=True)
    dec = np.where(nodes["type"] == 0)[0]
    ref_nodes = nodes.copy()
    ref_nodes["infoset_offset"][dec] = np.arange(len(dec))    # one infoset per decision node
    ref_nodes["turn_idx"] = 0                                  # the one equity matrix
    combos = np.asarray(sub["combos0"], np.int64)
    if not np.array_equal(combos, np.asarray(sub["combos1"], np.int64)) or len(combos) > 1024:
        raise ValueError("the reference kernels need one hand list of at most 1,024 combos")
    if int(np.max(nodes["num_actions"])) > 3:
        raise ValueError("the reference kernels hold at most three actions per node")
    with open(path, "wb") as f:
        f.write(np.array([len(nodes), len(combos), iters, len(dec)], "<i4").tobytes())
        f.write(ref_nodes.tobytes())
        f.write(_CC[combos].tobytes())
        f.write(np.asarray(sub["board"], np.uint8).tobytes())
        f.write(np.asarray(sub["range0"], "<f4").tobytes())
        f.write(np.asarray(sub["range1"], "<f4").tobytes())
    return dec


def run(sub, iters, timing=False, timeout=600):
    """Runs the kernels for `iters` iterations.  Returns (R, S, cfv, dec,
    ms, launches): R and S [n_decision * 3][1216] and the root CFVs [2][1216]
    as the kernels leave them, the decision node of each infoset, and with
    timing=True the CUDA-event time of the iterations (after a warm-up) and
    the kernel launches they made."""
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        dec = _write_input(sub, iters, fin)
        cmd = [HARNESS, fin, fout] + (["time"] if timing else [])
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"ref_hu_sweeps failed ({r.returncode}): {r.stdout}{r.stderr}")
        raw = np.fromfile(fout, "<f4")
    ms, launches = None, None
    if timing:
        parts = r.stdout.split()
        ms, launches = float(parts[parts.index("iters_ms") + 1]), int(parts[parts.index("launches") + 1])
    nR = len(dec) * 3 * PAD
    return (raw[:nR].reshape(-1, PAD), raw[nR:2 * nR].reshape(-1, PAD), raw[2 * nR:].reshape(2, PAD), dec, ms,
            launches)
