"""ctypes binding of libmtt_b200.so (the C ABI declared in include/mtt_b200.h).

The shared library is built in-tree by build.py; importing this module loads
it and fails loudly if it is missing.  There is no CPU fallback.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmtt_b200.so")

MTT_OK = 0
MTT_ERR_INVALID, MTT_ERR_CUDA, MTT_ERR_NOMEM, MTT_ERR_TIMEOUT, MTT_ERR_IO, MTT_ERR_UNSUPPORTED = 1, 2, 3, 4, 5, 6
STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of memory", 4: "timeout", 5: "io",
          6: "unsupported"}

NODE_DECISION, NODE_FOLD, NODE_SHOWDOWN, NODE_CHANCE, NODE_LEAF = 0, 1, 2, 3, 4
ALGO_CFRPLUS, ALGO_DCFR = 0, 1
SEM_CORRECT, SEM_REFERENCE = 0, 1

# mtt_node: the reference FlatNode layout (honest_multistreet_solver.cu:16-21), 32 bytes
NODE_DTYPE = np.dtype([
    ("type", "u1"), ("player", "u1"), ("num_actions", "u1"), ("active_mask", "u1"),
    ("children_offset", "<i4"), ("infoset_offset", "<i4"), ("turn_idx", "<i2"), ("depth", "<i2"),
    ("pot_size", "<f4"), ("committed", "<f4", (2,)), ("reserved", "<f4"),
])
assert NODE_DTYPE.itemsize == 32


class TreeSpec(ctypes.Structure):
    _fields_ = [("pot", ctypes.c_float), ("stack", ctypes.c_float),
                ("n_bet_sizes", ctypes.c_int32), ("bet_sizes", ctypes.c_float * 8),
                ("n_raise_sizes", ctypes.c_int32), ("raise_sizes", ctypes.c_float * 8),
                ("raise_cap", ctypes.c_int32), ("allin", ctypes.c_int32), ("street", ctypes.c_int32),
                ("river_leaves", ctypes.c_int32), ("river_runout", ctypes.c_int32)]


class SolveParams(ctypes.Structure):
    _fields_ = [("iters", ctypes.c_int32), ("algo", ctypes.c_int32), ("alpha", ctypes.c_float),
                ("beta", ctypes.c_float), ("gamma", ctypes.c_float), ("semantics", ctypes.c_int32),
                ("threads", ctypes.c_int32), ("exploitability", ctypes.c_int32), ("alternate", ctypes.c_int32),
                ("avg_power", ctypes.c_float), ("target_expl", ctypes.c_float), ("max_iters", ctypes.c_int32),
                ("chunk_iters", ctypes.c_int32)]


class Subgame(ctypes.Structure):
    _fields_ = [("nodes", ctypes.c_void_p), ("n_nodes", ctypes.c_int32), ("rows", ctypes.c_int32 * 2),
                ("board", ctypes.c_uint8 * 5), ("nboard", ctypes.c_int32), ("H", ctypes.c_int32 * 2),
                ("combos", ctypes.c_void_p * 2), ("ranges", ctypes.c_void_p * 2)]


MW_NODE_DTYPE = np.dtype([
    ("type", "u1"), ("player", "u1"), ("num_actions", "u1"), ("active_mask", "u1"),
    ("children_offset", "<i4"), ("infoset_offset", "<i4"), ("pot_size", "<f4"), ("committed", "<f4", (4,)),
])
assert MW_NODE_DTYPE.itemsize == 32


class MwSpec(ctypes.Structure):
    _fields_ = [("pot", ctypes.c_float), ("stacks", ctypes.c_float * 4), ("n_bet_sizes", ctypes.c_int32),
                ("bet_sizes", ctypes.c_float * 2), ("raise_size", ctypes.c_float), ("raise_cap", ctypes.c_int32)]


class MwSubgame(ctypes.Structure):
    _fields_ = [("nodes", ctypes.c_void_p), ("n_nodes", ctypes.c_int32), ("rows", ctypes.c_int32 * 4),
                ("board", ctypes.c_uint8 * 5), ("H", ctypes.c_int32), ("combos", ctypes.c_void_p),
                ("ranges", ctypes.c_void_p * 4), ("bubble", ctypes.c_float * 16)]


class PfParams(ctypes.Structure):
    _fields_ = [("iters", ctypes.c_int32), ("stack_bb", ctypes.c_float), ("bubble", ctypes.c_float),
                ("dead_pot", ctypes.c_float)]


class MttError(RuntimeError):
    def __init__(self, fn, status, cuda_err=0):
        super().__init__(f"{fn} failed: {STATUS.get(status, status)} (status {status}, cudaError {cuda_err})")
        self.status = status


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with python mtt-gpu-solver_b200/build.py")
    L = ctypes.CDLL(LIB_PATH)
    vp, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
    sig = {
        "mtt_status_string": ([ctypes.c_int], ctypes.c_char_p),
        "mtt_last_cuda_error": ([], ctypes.c_int),
        "mtt_version": ([], ctypes.c_char_p),
        "mtt_selftest_bounded_wait": ([i32, i32, vp], ctypes.c_int),
        "mtt_tree_build": ([vp, vp, i32, vp, vp, vp], ctypes.c_int),
        "mtt_tree_build_board": ([vp, vp, i32, vp, i32, vp, vp, vp], ctypes.c_int),
        "mtt_tree_validate": ([vp, i32, vp], ctypes.c_int),
        "mtt_eval7": ([vp, vp, i64, vp], ctypes.c_int),
        "mtt_eval7_enumerate": ([vp, vp, vp, vp, vp], ctypes.c_int),
        "mtt_board_showdown_counts": ([vp, i32, vp, i32, vp, vp, vp, vp], ctypes.c_int),
        "mtt_board_showdown_counts_noalloc": ([vp, i32, vp, i32, vp, vp, vp, vp], ctypes.c_int),
        "mtt_canonical_flops": ([vp, i32, vp], ctypes.c_int),
        "mtt_flop_ev": ([vp, i32, vp, vp, vp, vp, vp], ctypes.c_int),
        "mtt_ev_dump": ([vp, i32, vp, vp], ctypes.c_int),
        "mtt_batch_create": ([vp, i32, vp], ctypes.c_int),
        "mtt_batch_solve": ([vp, vp, vp], ctypes.c_int),
        "mtt_batch_solve_graph": ([vp, vp, vp], ctypes.c_int),
        "mtt_batch_results": ([vp, vp, vp], ctypes.c_int),
        "mtt_batch_read": ([vp, i32, vp, vp, vp, vp, vp, vp], ctypes.c_int),
        "mtt_batch_iterations": ([vp, vp], ctypes.c_int),
        "mtt_batch_read_vectors": ([vp, i32, vp, vp], ctypes.c_int),
        "mtt_batch_info": ([vp, vp, vp], ctypes.c_int),
        "mtt_batch_root_values": ([vp, i32, vp, vp, vp, vp], ctypes.c_int),
        "mtt_batch_launch_count": ([vp, vp], ctypes.c_int),
        "mtt_batch_kernel_profile": ([vp, vp, i32, vp, vp, vp], ctypes.c_int),
        "mtt_batch_set_leafnet": ([vp, vp, i32], ctypes.c_int),
        "mtt_trim_pool": ([], ctypes.c_int),
        "mtt_batch_set_schedule": ([vp, i32, i32, i32], ctypes.c_int),
        "mtt_batch_schedule": ([vp, vp, vp, vp], ctypes.c_int),
        "mtt_leafnet_capacity": ([vp, vp], ctypes.c_int),
        "mtt_batch_layout": ([vp, vp, vp, vp, vp], ctypes.c_int),
        "mtt_batch_ev_grad": ([vp, vp, vp, vp, vp, vp, vp], ctypes.c_int),
        "mtt_batch_check": ([vp, vp], ctypes.c_int),
        "mtt_gemm_bf16": ([vp, i32, vp, i32, vp, i32, i32, i32, i32, vp, vp, i32, i32, vp, vp], ctypes.c_int),
        "mtt_gemm_bf16_ws": ([vp, i32, vp, i32, vp, i32, i32, i32, i32, vp, vp, i32, i32, vp, vp, ctypes.c_int64, vp],
                             ctypes.c_int),
        "mtt_leafnet_create": ([i32, ctypes.c_uint64, i32, vp], ctypes.c_int),
        "mtt_leafnet_forward": ([vp, vp, i32, vp, vp], ctypes.c_int),
        "mtt_leafnet_gradients": ([vp, vp, vp, vp, i32, vp, vp], ctypes.c_int),
        "mtt_leafnet_train_step": ([vp, vp, vp, vp, i32, ctypes.c_float, vp, vp], ctypes.c_int),
        "mtt_leafnet_params": ([vp, i32, vp, vp, vp, vp, vp], ctypes.c_int),
        "mtt_leafnet_check": ([vp], ctypes.c_int),
        "mtt_leafnet_destroy": ([vp], ctypes.c_int),
        "mtt_checkdown_values": ([vp, vp, vp, i32, vp, vp], ctypes.c_int),
        "mtt_pf_allin_matrix": ([i32, vp, vp, vp, vp], ctypes.c_int),
        "mtt_pf_flop_class_matrices": ([i32, vp, i32, vp, vp], ctypes.c_int),
        "mtt_pf_dcfr": ([vp, vp, i32, vp, vp, vp, vp, vp], ctypes.c_int),
        "mtt_pf_read_subset": ([ctypes.c_char_p, vp, vp, i32, vp], ctypes.c_int),
        "mtt_pf_combo_class": ([i32, i32], ctypes.c_int),
        "mtt_subset_nnomp": ([vp, i32, i32, vp, i32, vp, vp, vp], ctypes.c_int),
        "mtt_subset_write": ([ctypes.c_char_p, ctypes.c_char_p, vp, vp, i32], ctypes.c_int),
        "mtt_icm_equity": ([vp, i32, vp, i32, vp], ctypes.c_int),
        "mtt_icm_bubble_factors": ([vp, i32, vp, i32, vp, i32, vp], ctypes.c_int),
        "mtt_mw_tree_build": ([vp, vp, i32, vp, vp, vp], ctypes.c_int),
        "mtt_mw_batch_create": ([vp, i32, vp], ctypes.c_int),
        "mtt_mw_batch_solve": ([vp, vp, i32, vp], ctypes.c_int),
        "mtt_mw_batch_values": ([vp, vp, vp], ctypes.c_int),
        "mtt_mw_batch_read": ([vp, i32, vp, vp, vp], ctypes.c_int),
        "mtt_mw_batch_destroy": ([vp], ctypes.c_int),
        "mtt_batch_autotune": ([vp, vp, vp, vp], ctypes.c_int),
        "mtt_batch_destroy": ([vp], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def check(fn, status):
    if status != MTT_OK:
        raise MttError(fn, status, lib().mtt_last_cuda_error())


def exported_symbols():
    """Names of the functions include/mtt_b200.h declares."""
    import re
    hdr = open(os.path.join(os.path.dirname(HERE), "include", "mtt_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(mtt_[a-z0-9_]+)\s*\(", hdr, re.M)))
