"""The flop-subset optimiser (scripts/optimize_subset.py) on the GPU.

    python -m mtt-gpu-solver_b200.subset [--dump PATH | --regenerate] [--select N] [--out-dir DIR]

reads mtt_ev_dump_1755.bin (default ./mtt_ev_dump_1755.bin; --regenerate
computes it on the device with `ev_dump`), selects the flops by greedy
non-negative orthogonal matching pursuit (`mtt_subset_nnomp`) and writes
mtt_subset.bin and mtt_subset_weights.txt as the reference script does
(optimize_subset.py:52-65)."""
import argparse
import ctypes
import importlib
import os
import sys

import numpy as np

from ._lib import check, lib

N_FEATURES = 4 * 2 * 169   # per flop: 4 stack depths x 2 players x 169 classes


def _stream(s):
    if s is None:
        return None
    return ctypes.c_void_p(s.cuda_stream if hasattr(s, "cuda_stream") else int(s))


def _pkg():
    # the package, also when this file runs as `python -m <package>.subset`
    return importlib.import_module(__package__)


def nnomp(cols, colw, nselect=100, stream=None):
    """Greedy NN-OMP (optimize_subset.py:29-50) over the rows of `cols`.

    cols: contiguous CUDA float32 [ncols, nfeat], one row per candidate (the
    dump as [1755, 1352]); colw: ncols column weights (any array; FP64 on the
    device).  Returns (indices int32 [nselect] in selection order, weights
    float64 [nselect] scaled to sum to ncols)."""
    import torch
    if not (isinstance(cols, torch.Tensor) and cols.is_cuda and cols.dtype == torch.float32 and cols.dim() == 2
            and cols.is_contiguous()):
        raise TypeError("cols: expected a contiguous 2-D CUDA float32 tensor")
    ncols, nfeat = cols.shape
    w = torch.as_tensor(np.asarray(colw, dtype=np.float64)).to(cols.device)
    if w.numel() != ncols:
        raise ValueError("colw: one weight per row of cols")
    idx = torch.empty(nselect, dtype=torch.int32, device=cols.device)
    out = torch.empty(nselect, dtype=torch.float64, device=cols.device)
    st = _stream(stream) if stream is not None else ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    check("mtt_subset_nnomp", lib().mtt_subset_nnomp(
        ctypes.c_void_p(cols.data_ptr()), ncols, nfeat, ctypes.c_void_p(w.data_ptr()), int(nselect),
        ctypes.c_void_p(idx.data_ptr()), ctypes.c_void_p(out.data_ptr()), st))
    return idx.cpu().numpy(), out.cpu().numpy()


def optimize(dump=None, nselect=100, device="cuda"):
    """The reference script end to end: dump [1755, 1352] float32 (host array
    or CUDA tensor; None = regenerate it with `ev_dump`), the canonical flops'
    orbit weights, NN-OMP.  Returns (flops uint8 [n, 3], weights float64 [n],
    indices int32 [n])."""
    import torch
    mtt = _pkg()
    meta = mtt.canonical_flops()
    if dump is None:
        f3 = torch.from_numpy(np.ascontiguousarray(meta[:, :3])).to(device)
        cols = mtt.ev_dump(f3).reshape(len(meta), -1)
    elif isinstance(dump, torch.Tensor):
        cols = dump.to(device=device, dtype=torch.float32).reshape(len(meta), -1).contiguous()
    else:
        cols = torch.from_numpy(np.ascontiguousarray(np.asarray(dump, dtype=np.float32).reshape(len(meta), -1))).to(device)
    idx, w = nnomp(cols, meta[:, 3].astype(np.float64), nselect)
    return np.ascontiguousarray(meta[idx, :3]), w, idx


def write(bin_path, txt_path, flops3, weights):
    """mtt_subset.bin and mtt_subset_weights.txt (either path may be None)."""
    f = np.ascontiguousarray(flops3, dtype=np.uint8)
    w = np.ascontiguousarray(weights, dtype=np.float64)
    if f.shape != (len(w), 3):
        raise ValueError("flops3: [n, 3] cards, one row per weight")
    check("mtt_subset_write", lib().mtt_subset_write(
        bin_path.encode() if bin_path else None, txt_path.encode() if txt_path else None,
        f.ctypes.data, w.ctypes.data, len(w)))


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--dump", default="mtt_ev_dump_1755.bin")
    ap.add_argument("--regenerate", action="store_true", help="compute the dump on the device instead of reading it")
    ap.add_argument("--select", type=int, default=100)
    ap.add_argument("--out-dir", default=".")
    a = ap.parse_args(argv)
    dump = None
    if not a.regenerate:
        dump = np.fromfile(a.dump, dtype="<f4")
        if dump.size != 1755 * N_FEATURES:
            print(f"{a.dump}: expected {1755 * N_FEATURES} floats, found {dump.size}", file=sys.stderr)
            return 1
    flops, w, _ = optimize(dump, a.select)
    write(os.path.join(a.out_dir, "mtt_subset.bin"), os.path.join(a.out_dir, "mtt_subset_weights.txt"), flops, w)
    print(f"Subset generated: {len(w)} flops saved to mtt_subset.bin")
    return 0


if __name__ == "__main__":
    sys.exit(main())
