"""Build the sm_100a shared library libamigo_b200.so in-tree.

    python -m amigo_b200.build            # incremental
    python -m amigo_b200.build --force    # rebuild everything

Every CUDA source is compiled by nvcc for `-gencode arch=compute_100a,
code=sm_100a` only; host sources are compiled by nvcc's host compiler.  The
result is amigo_b200/_lib/libamigo_b200.so, loaded by amigo_b200/_lib.py.
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
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libamigo_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
          "-Xcompiler", "-Wall", "-I" + os.path.join(ROOT, "include"),
          "--expt-relaxed-constexpr"]
# Per-file extra flags.  The IPM vector kernels must not contract a*b+c
# into fused multiply-adds, so their elementwise results match the CPU
# reference bit for bit.
EXTRA = {"ipm_kernels.cu": ["--fmad=false"], "ipm_scaling.cu": ["--fmad=false"],
         "batch_ctrl.cu": ["--fmad=false"]}

SOURCES = ["symbolic.cpp", "ldl_plan.cpp", "ldl_factor.cu", "ldl_solve.cu",
           "capi.cpp", "ipm_kernels.cu", "capi_ipm.cpp", "csr_kernels.cu",
           "fem_simp.cu", "cartpole.cu", "tc_kernels.cu", "ipm_scaling.cu",
           "batch_ctrl.cu"]


def nvcc():
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def _headers_mtime():
    ts = [os.path.getmtime(os.path.join(CSRC, f)) for f in os.listdir(CSRC)
          if f.endswith((".h", ".cuh"))]
    ts.append(os.path.getmtime(os.path.join(ROOT, "include", "amigo_b200.h")))
    ts.append(os.path.getmtime(os.path.abspath(__file__)))
    return max(ts)


def _compile(src, force, hdr_t, verbose):
    obj = os.path.join(BUILD, src + ".o")
    path = os.path.join(CSRC, src)
    if (not force and os.path.exists(obj)
            and os.path.getmtime(obj) >= max(os.path.getmtime(path), hdr_t)):
        return obj, None
    cmd = [nvcc()] + ARCH + COMMON + EXTRA.get(src, []) + ["-c", path, "-o", obj]
    if src.endswith(".cu") and verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return obj, (r.stdout + r.stderr) if verbose else None


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(OUT_DIR, exist_ok=True)
    hdr_t = _headers_mtime()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, force, hdr_t, verbose), SOURCES))
    objs = [o for o, _ in results]
    if verbose:
        for o, log in results:
            if log:
                print(log)
    if (force or not os.path.exists(LIB)
            or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs)):
        tmp = LIB + ".tmp"
        cmd = [nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed: %s\n%s" % (r.stdout, r.stderr))
        os.replace(tmp, LIB)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    sys.exit(main())
