"""Build recipe for the CUDA library (libkf.so, sm_100a) and its generated tables.

`python -m oglfusionkinectv2_b200.build` (or `build()`) regenerates the marching-cubes
tables header, compiles every csrc/*.cu for sm_100a with nvcc and links libkf.so beside
this file.  Objects are rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libkf.so")
ROOT = os.path.dirname(PKG)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
                     "-Xptxas", "-warn-spills", "-DKF_BUILDING_LIBRARY"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx() -> list[str]:
    # nvcc's host compiler: the system g++ (an alternative toolchain on CXX may lack parts
    # of the standard runtime the link needs)
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def gen_tables() -> None:
    r = subprocess.run([sys.executable, os.path.join(CSRC, "gen_mc_tables.py")],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("table generation failed:\n" + r.stdout + r.stderr)


def build(verbose: bool = False, ptxas_verbose: bool = False) -> str:
    gen_tables()
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + [
        os.path.join(ROOT, "include", "kf.h"),
        os.path.join(CSRC, "generated", "kf_mc_tables.inc")]
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    objs = []
    jobs = []
    for src in sources:
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if _newer(obj, [src] + headers) or ptxas_verbose:
            cmd = [nvcc] + _host_cxx() + NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_verbose else []) + [
                "-c", src, "-o", obj]
            jobs.append((src, cmd))

    def run(job):
        src, cmd = job
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, cmd, r

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for src, cmd, r in ex.map(run, jobs):
            if verbose or ptxas_verbose or r.returncode != 0:
                print(" ".join(cmd))
                print(r.stdout + r.stderr)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {os.path.basename(src)}")
    if _newer(LIB, objs):
        cmd = [nvcc] + _host_cxx() + ARCH + ["-shared", "-o", LIB + ".tmp"] + objs + ["-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        os.replace(LIB + ".tmp", LIB)
    return LIB


def build_oracle(verbose: bool = False) -> str:
    """Compile the FP64 CPU oracle (test infrastructure under oracle/)."""
    gen_tables()
    r = subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], capture_output=True, text=True)
    if verbose or r.returncode != 0:
        print(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed")
    return os.path.join(ROOT, "oracle", "liboracle_kf.so")


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, ptxas_verbose="--ptxas" in sys.argv))
