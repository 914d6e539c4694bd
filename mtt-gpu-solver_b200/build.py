"""Build libmtt_b200.so (the sm_100a kernels + C ABI) in-tree with nvcc.

    python mtt-gpu-solver_b200/build.py [--force] [--jobs N]

Objects go to mtt-gpu-solver_b200/_build/, the shared library next to this
file.  Sources are rebuilt only when they (or any header) changed.
"""
import argparse
import concurrent.futures
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmtt_b200.so")
NVCC = os.environ.get("NVCC", os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc"))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# The image's $CC/$CXX wrappers lack parts of the runtime; the system g++ is complete.
CCBIN = ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "-I" + os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def _stale(obj, src, hdr_mtime):
    return not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), hdr_mtime)


def compile_one(src, obj, extra):
    cmd = [NVCC] + CCBIN + ARCH + COMMON + extra + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC] + CCBIN + ARCH + COMMON + extra + ["-x", "c++", "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return src, r.returncode, r.stdout + r.stderr, " ".join(cmd)


def build(force=False, jobs=8, verbose_ptxas=False, quiet=False):
    os.makedirs(BUILD, exist_ok=True)
    hdr_mtime = max([os.path.getmtime(h) for h in headers()] + [0.0])
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    objs, todo = [], []
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or verbose_ptxas or _stale(obj, src, hdr_mtime):
            todo.append((src, obj))
    with concurrent.futures.ThreadPoolExecutor(max_workers=jobs) as ex:
        for src, rc, out, cmd in ex.map(lambda t: compile_one(t[0], t[1], extra), todo):
            if rc != 0:
                sys.stderr.write(f"[build] FAILED {cmd}\n{out}\n")
                raise RuntimeError(f"nvcc failed on {os.path.basename(src)}")
            if out.strip() and (verbose_ptxas or not quiet):
                sys.stderr.write(out)
    if todo or not os.path.exists(LIB):
        cmd = [NVCC] + CCBIN + ARCH + ["-shared", "-o", LIB + ".tmp"] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
        shutil.move(LIB + ".tmp", LIB)
    return LIB


DRIVERS = os.path.join(HERE, "drivers")
BIN = os.path.join(HERE, "bin")
CUDA_LIB = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "lib64")


def build_drivers(force=False, quiet=False):
    """The command-line drivers (ev_dumper, preflop_gen, hu_solver,
    multiway_solver): host C++ over the C ABI, linked to libmtt_b200.so next
    to them (rpath $ORIGIN/..) into bin/."""
    os.makedirs(BIN, exist_ok=True)
    deps = glob.glob(os.path.join(DRIVERS, "*.h")) + [os.path.join(ROOT, "include", "mtt_b200.h"), LIB]
    dep_mtime = max(os.path.getmtime(d) for d in deps if os.path.exists(d))
    built = []
    for src in sorted(glob.glob(os.path.join(DRIVERS, "*.cpp"))):
        exe = os.path.join(BIN, os.path.splitext(os.path.basename(src))[0])
        built.append(exe)
        if not force and os.path.exists(exe) and os.path.getmtime(exe) >= max(os.path.getmtime(src), dep_mtime):
            continue
        cmd = [NVCC] + CCBIN + ARCH + ["-O2", "-std=c++17", "-x", "c++", src, "-I" + os.path.join(ROOT, "include"),
                                "-I" + DRIVERS, "-L" + HERE, "-lmtt_b200", "-L" + CUDA_LIB, "-lcudart",
                                "-Xlinker", "--disable-new-dtags", "-Xlinker", "-rpath=$ORIGIN/..",
                                "-Xlinker", "-rpath=" + CUDA_LIB, "-o", exe + ".tmp"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(f"[build] FAILED {' '.join(cmd)}\n{r.stdout}{r.stderr}\n")
            raise RuntimeError(f"driver build failed: {os.path.basename(src)}")
        if (r.stdout + r.stderr).strip() and not quiet:
            sys.stderr.write(r.stdout + r.stderr)
        shutil.move(exe + ".tmp", exe)
    return built


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=8)
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v (registers, spills, smem)")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.jobs, verbose_ptxas=a.ptxas))
    for exe in build_drivers(force=a.force):
        print(exe)
