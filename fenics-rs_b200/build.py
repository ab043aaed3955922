"""Build libfenics_cuda.so (sm_100a) in-tree with nvcc.

    python fenics-rs_b200/build.py [--force]

Each .cu under csrc/ compiles to an object with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3``; rhs.cu additionally
gets ``--fmad=false`` so its load-vector sums keep the reference's operation
order. The objects link into fenics_cuda/libfenics_cuda.so next to the Python
binding that loads it.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "fenics_cuda", "libfenics_cuda.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-I", INCLUDE, "-I", CSRC]
PER_FILE = {"rhs.cu": ["--fmad=false"]}


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_compiler() -> list[str]:
    # The image exports CXX pointing at a wrapper; nvcc needs a plain g++.
    gxx = "/usr/bin/g++"
    return ["-ccbin", gxx] if os.path.exists(gxx) else []


def sources() -> list[str]:
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    hdrs = _headers()
    jobs = []
    objs = []
    for src in sources():
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src[:-3] + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            cmd = [nvcc] + _host_compiler() + ARCH + COMMON + PER_FILE.get(src, []) + ["-c", s, "-o", o]
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r.stderr

    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
        for err in ex.map(run, jobs):
            if verbose and err:
                print(err, file=sys.stderr)
    if force or jobs or _stale(OUT, objs):
        cmd = [nvcc] + _host_compiler() + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart"]
        run(cmd)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
