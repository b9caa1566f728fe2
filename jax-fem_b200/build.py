"""Build libjaxfem_b200.so (all CUDA kernels + the C ABI) for sm_100a, in-tree.

    python jax-fem_b200/build.py [--force] [--verbose]

Objects go to jax-fem_b200/_build/, the shared library to
jax-fem_b200/lib/libjaxfem_b200.so.  Sources compile in parallel; a source is
rebuilt when it or any header is newer than its object.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libjaxfem_b200.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "--extended-lambda",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden"]


def nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(src, obj, hdr_mtime):
    if not os.path.exists(obj):
        return True
    m = os.path.getmtime(obj)
    return os.path.getmtime(src) > m or hdr_mtime > m


def build(force=False, verbose=False, extra_flags=()):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    hdr_mtime = max([os.path.getmtime(h) for h in _headers()] + [0.0])
    cc = nvcc()
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        if force or _stale(s, o, hdr_mtime):
            lang = ["-x", "cu"] if s.endswith(".cu") else ["-x", "c++"]
            cmd = [cc, *ARCH, *NVCC_FLAGS, *extra_flags, "-I", INCLUDE, "-I", CSRC, *lang, "-c", s, "-o", o]
            jobs.append((s, cmd))

    def run(job):
        s, cmd = job
        if verbose:
            print(" ".join(cmd), flush=True)
        p = subprocess.run(cmd, capture_output=True, text=True)
        return s, p

    failed = []
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for s, p in ex.map(run, jobs):
            if verbose and (p.stdout or p.stderr):
                print(p.stdout + p.stderr)
            if p.returncode != 0:
                failed.append((s, p.stderr))
    if failed:
        for s, err in failed:
            sys.stderr.write(f"--- {s}\n{err}\n")
        raise RuntimeError(f"{len(failed)} source(s) failed to compile")
    if jobs or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [cc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("link failed:\n" + p.stderr)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
