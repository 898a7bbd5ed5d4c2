"""Build libqsketch.so (the C ABI in include/qsketch_c.h) for sm_100a, in-tree.

    python qsketch_b200/build.py            # build if sources changed
    python qsketch_b200/build.py --force    # rebuild
    python qsketch_b200/build.py --verbose  # also print ptxas register/spill reports
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libqsketch.so")
SOURCES = ["qs_msws.cu", "qs_cm.cu", "qs_aux.cu", "qs_api.cu", "qs_noalloc.cu", "qs_mlp.cu", "qs_learned.cu",
           "qs_shard.cu", "qs_remove.cu"]
HEADERS = ["qs_common.cuh", "qs_device.cuh", "qs_kernels.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libqsketch.so")
    return exe


def _flags(verbose):
    f = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
                "-I", os.path.join(ROOT, "include"), "-I", CSRC]
    if verbose:
        f += ["-Xptxas", "-v"]
    return f


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "qsketch_c.h")]
    objs, jobs = [], []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            jobs.append([nvcc(), "-c", src, "-o", obj] + _flags(verbose))

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    failed = False
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for cmd, r in ex.map(run, jobs):
            out = (r.stdout or "") + (r.stderr or "")
            if r.returncode != 0:
                failed = True
                sys.stderr.write(out)
            elif verbose and out:
                sys.stderr.write(out)
    if failed:
        raise RuntimeError("nvcc failed building libqsketch.so")
    if force or jobs or _stale(LIB, objs):
        cmd = [nvcc(), "-shared", "-o", LIB] + objs + ARCH + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc link of libqsketch.so failed")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
