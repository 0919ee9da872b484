"""Build libphotonpy_b200.so (sm_100a) in-tree with nvcc.

    python -m photonpy_b200.csrc.build [--verbose] [--define NAME=VALUE ...] [--out PATH]

Output: photonpy_b200/lib/libphotonpy_b200.so. The library statically links the CUDA
runtime so that it does not depend on which libcudart other modules of the process load.
--define passes compile-time switches (for example PB200_LM_IEEE_CHOL=1, see fit_common.cuh)
and --out writes such a build elsewhere; PHOTONPY_B200_LIBRARY makes the package load it.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
LIB_DIR = os.path.join(PKG, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libphotonpy_b200.so")
OBJ_DIR = os.path.join(PKG, "_build")

UNITS = ["estimator.cu", "estim_queue.cu", "spot_detect.cu", "spot_queue.cu", "probes.cu", "k_xyibg.cu", "k_constsigma.cu", "k_sigma.cu", "k_sigmaxy.cu",
         "k_astig.cu", "k_spline.cu", "k_tilted.cu", "k_mixed.cu"]
HEADERS = ["host_internal.h", "spot_internal.h", "models.cuh", "fit_kernels.cuh", "fit_common.cuh", "gauss_fit.cuh", "launch.cuh", "mixed.cuh", "adjoint.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return [os.path.join(HERE, u) for u in UNITS] + [os.path.join(HERE, h) for h in HEADERS] + [
        os.path.join(ROOT, "include", "photonpy_b200.h")]


def up_to_date() -> bool:
    if not os.path.exists(LIB_PATH):
        return False
    t = os.path.getmtime(LIB_PATH)
    return all(os.path.getmtime(s) <= t for s in sources())


def build(force: bool = False, verbose: bool = False, defines=(), out: str | None = None) -> str:
    lib_path = os.path.abspath(out) if out else LIB_PATH
    obj_dir = OBJ_DIR if not out else os.path.join(os.path.dirname(lib_path), "_obj")
    if not force and not out and not defines and up_to_date():
        return LIB_PATH
    os.makedirs(os.path.dirname(lib_path), exist_ok=True)
    os.makedirs(obj_dir, exist_ok=True)
    common = ["-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-O3", "-I", os.path.join(ROOT, "include")]
    common += ["-D" + d for d in defines]
    if verbose:
        common += ["-Xptxas", "-v"]

    newest_header = max(os.path.getmtime(os.path.join(HERE, h)) for h in HEADERS)
    newest_header = max(newest_header, os.path.getmtime(os.path.join(ROOT, "include", "photonpy_b200.h")))

    def compile_unit(u):
        src = os.path.join(HERE, u)
        obj = os.path.join(obj_dir, os.path.splitext(u)[0] + ".o")
        cmd = [nvcc(), *common, "-c", src, "-o", obj]
        stamp = obj + ".cmd"
        # an object is reused when it is newer than its sources and was built with the same command
        if (not force and os.path.exists(obj) and os.path.exists(stamp) and open(stamp).read() == " ".join(cmd)
                and os.path.getmtime(obj) >= max(os.path.getmtime(src), newest_header)):
            return obj, ""
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode == 0:
            with open(stamp, "w") as f:
                f.write(" ".join(cmd))
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {u}:\n{r.stdout}\n{r.stderr}")
        return obj, r.stderr

    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(UNITS), os.cpu_count() or 1))) as ex:
        results = list(ex.map(compile_unit, UNITS))
    if verbose:
        for _, log in results:
            sys.stderr.write(log)
    tmp = lib_path + f".tmp{os.getpid()}"
    cmd = [nvcc(), "-shared", *ARCH, "-o", tmp, *[o for o, _ in results], "-cudart", "static", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, lib_path)
    return lib_path


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--define", action="append", default=[], help="NAME=VALUE compile-time switch")
    ap.add_argument("--out", default=None, help="library path (default: the package's lib/)")
    args = ap.parse_args()
    print(build(force=args.force, verbose=args.verbose, defines=args.define, out=args.out))
