"""Builds the sm_100a shared library konglong_b200/_rtm_b200.so in-tree.

Every CUDA source is compiled by nvcc for `-gencode arch=compute_100a,
code=sm_100a` with -lineinfo; the host set-up code is compiled by the same
nvcc as C++.  Objects go to konglong_b200/_build (git-ignored).  Rebuilds
only what changed (source or header newer than the object).
"""
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "_rtm_b200.so")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "--extended-lambda",
           "-Xcompiler", "-fPIC", "-Xptxas", "-warn-spills", "-I" + os.path.join(ROOT, "include")]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def _stale(obj, src, newest_header):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return os.path.getmtime(src) > t or newest_header > t


def build(verbose=False, extra_flags=()):
    os.makedirs(BUILD, exist_ok=True)
    srcs = _sources()
    newest_header = max((os.path.getmtime(h) for h in _headers()), default=0)
    cc = nvcc()
    jobs = []
    objs = []
    for s in srcs:
        obj = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(obj)
        if _stale(obj, s, newest_header):
            cmd = [cc] + ARCH + NVFLAGS + list(extra_flags) + ["-c", s, "-o", obj]
            if s.endswith(".cpp"):
                cmd = [cc, "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-x", "c++",
                       "-I" + os.path.join(ROOT, "include"), "-c", s, "-o", obj]
            jobs.append((s, cmd))

    def run(job):
        src, cmd = job
        if verbose:
            print(" ".join(cmd), flush=True)
        p = subprocess.run(cmd, capture_output=True, text=True)
        return src, p

    relink = bool(jobs) or not os.path.exists(LIB)
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for src, p in ex.map(run, jobs):
            out = (p.stdout + p.stderr).strip()
            if p.returncode != 0:
                raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n{out}")
            if out and verbose:
                print(out)
    if relink:
        cmd = [cc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lcufft", "-lcublas"]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("link failed:\n" + p.stdout + p.stderr)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
