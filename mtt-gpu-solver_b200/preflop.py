"""The preflop anchor chain (preflop_gen): all-in matrix, class-reduced flop
matrices over a flop subset, and DCFR over the closed BTN-vs-BB tree.

    python -m mtt-gpu-solver_b200.preflop [--subset PATH] [--mode reference|correct] [--iters N]

prints the reference's 15-hand strategy table (preflop_grid_generator.cu:616-653)
from the GPU path."""
import argparse
import ctypes
import importlib
import sys

import numpy as np

from ._lib import PfParams, check, lib

REFERENCE, CORRECT = 0, 1
NAMES = ["AA", "KK", "QQ", "JJ", "TT", "99", "88", "22", "AKs", "A5s", "T9s", "76s", "AKo", "QJo", "32o"]
INDICES = [0, 1, 2, 3, 4, 5, 6, 12, 13, 17, 72, 85, 91, 104, 168]
NODE_ROWS = {"btn_root": (0, 3), "bb_def": (3, 6), "btn_vs_3b": (6, 8), "bb_vs_jam": (8, 10)}


def _stream(s):
    if s is None:
        return None
    return ctypes.c_void_p(s.cuda_stream if hasattr(s, "cuda_stream") else int(s))


def read_subset(path=None):
    """(flops uint8 [n, 3], weights float32 [n]) of a flop-subset file."""
    n = ctypes.c_int32()
    p = path.encode() if path else None
    check("mtt_pf_read_subset", lib().mtt_pf_read_subset(p, None, None, 0, ctypes.byref(n)))
    flops = np.zeros((n.value, 3), np.uint8)
    w = np.zeros(n.value, np.float32)
    check("mtt_pf_read_subset", lib().mtt_pf_read_subset(p, flops.ctypes.data, w.ctypes.data, n.value, ctypes.byref(n)))
    return flops, w


def allin_matrix(mode=REFERENCE, counts=False, device="cuda", stream=None):
    import torch
    out = torch.empty((169, 169), dtype=torch.float32, device=device)
    w = torch.empty((169, 169), dtype=torch.int32, device=device) if counts else None
    t = torch.empty_like(w) if counts else None
    check("mtt_pf_allin_matrix", lib().mtt_pf_allin_matrix(
        mode, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(w.data_ptr()) if counts else None,
        ctypes.c_void_p(t.data_ptr()) if counts else None, _stream(stream)))
    return (out, w, t) if counts else out


def flop_class_matrices(flops, mode=REFERENCE, device="cuda", stream=None):
    """[n, 169, 169] class equity matrices, out[f][v][h]."""
    import torch
    f = torch.as_tensor(np.ascontiguousarray(flops, np.uint8)).to(device)
    out = torch.empty((f.shape[0], 169, 169), dtype=torch.float32, device=device)
    check("mtt_pf_flop_class_matrices", lib().mtt_pf_flop_class_matrices(
        mode, ctypes.c_void_p(f.data_ptr()), f.shape[0], ctypes.c_void_p(out.data_ptr()), _stream(stream)))
    return out


def dcfr(weights, class_mats, allin, iters=500, stack_bb=20.0, bubble=1.35, dead_pot=2.5, stream=None):
    """Strategy sums and last strategies [10, 192] of the closed preflop tree."""
    import torch
    w = torch.as_tensor(np.ascontiguousarray(weights, np.float32)).to(class_mats.device)
    sums = torch.empty((10, 192), dtype=torch.float32, device=class_mats.device)
    sig = torch.empty_like(sums)
    p = PfParams(int(iters), float(stack_bb), float(bubble), float(dead_pot))
    check("mtt_pf_dcfr", lib().mtt_pf_dcfr(
        ctypes.c_void_p(w.data_ptr()), ctypes.c_void_p(class_mats.contiguous().data_ptr()), class_mats.shape[0],
        ctypes.c_void_p(allin.contiguous().data_ptr()), ctypes.byref(p), ctypes.c_void_p(sums.data_ptr()),
        ctypes.c_void_p(sig.data_ptr()), _stream(stream)))
    return sums, sig


def strategy_table(sums):
    """Normalised average strategies of the BTN root and BB defence for the
    reference's 15 display hands, as the reference prints them (+1e-7)."""
    s = np.asarray(sums.cpu() if hasattr(sums, "cpu") else sums, np.float32)
    rows = []
    for name, c in zip(NAMES, INDICES):
        b = s[0:3, c]; d = s[3:6, c]
        b = b / (b.sum(dtype=np.float32) + np.float32(1e-7))
        d = d / (d.sum(dtype=np.float32) + np.float32(1e-7))
        rows.append((name, *b.tolist(), *d.tolist()))
    return rows


def main(argv=None):
    import torch
    ap = argparse.ArgumentParser(prog="preflop_gen")
    ap.add_argument("--subset", default=None, help="flop subset (default data/mtt_subset.bin, then ./mtt_subset.bin)")
    ap.add_argument("--mode", default="reference", choices=["reference", "correct"])
    ap.add_argument("--iters", type=int, default=500)
    ap.add_argument("--stack", type=float, default=20.0)
    ap.add_argument("--bubble", type=float, default=1.35)
    ap.add_argument("--dead", type=float, default=2.5)
    a = ap.parse_args(argv)
    mode = REFERENCE if a.mode == "reference" else CORRECT
    flops, w = read_subset(a.subset)
    allin = allin_matrix(mode)
    mats = flop_class_matrices(flops, mode)
    sums, _ = dcfr(w, mats, allin, a.iters, a.stack, a.bubble, a.dead)
    torch.cuda.synchronize()
    print(f"preflop DCFR: {len(flops)} flops, {a.iters} iterations, stack {a.stack:g} BB, bubble factor {a.bubble:g}, "
          f"dead pot {a.dead:g} BB ({a.mode} mode)")
    print(f"{'Hand':7s}{'BTN Fold':12s}{'BTN MinRaise':14s}{'BTN Jam':12s}{'BB Fold':12s}{'BB Defend':14s}BB 3B-Jam")
    for r in strategy_table(sums):
        print(f"{r[0]:7s}{r[1]:<12.3f}{r[2]:<14.3f}{r[3]:<12.3f}{r[4]:<12.3f}{r[5]:<14.3f}{r[6]:.3f}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
