"""Build the engine's shared library (liboco_b200.so) and host tools in-tree with nvcc.

    python -m ocotillo_b200.build [--force]

Every CUDA translation unit is compiled for sm_100a only.  The FP64 kernels are compiled
with -fmad=false and IEEE division/square root so that they reproduce the CPU oracle bit for
bit; host code is compiled without FMA contraction for the same reason.
"""
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "liboco_b200.so")
DRIVER = os.path.join(PKG, "flux_feautrier_b200")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
                 "-I", os.path.join(ROOT, "include"), "-I", CSRC]

# (source, extra flags)
UNITS = [
    ("kernels_fp64.cu", ["-fmad=false", "-prec-div=true", "-prec-sqrt=true"]),
    ("kernels_mixed.cu", []),
    ("kernels_repair.cu", ["-fmad=false", "-prec-div=true", "-prec-sqrt=true"]),
    ("kernels_mixed_pillars.cu", ["-fmad=false", "-prec-div=true", "-prec-sqrt=true"]),
    ("oco_api.cu", []),
    ("oco_noalloc.cu", []),
    ("oco_batch.cu", []),
    ("kernels_epilogue.cu", ["-fmad=false"]),
    ("kernels_inputs.cu", ["-fmad=false", "-prec-div=true", "-prec-sqrt=true"]),
    ("oco_server.cu", []),
]
HOST_UNITS = [("oco_deck.cpp", [])]

HEADERS = ["ocomath.h", "ocomath_tables.h", "oco_consts.h", "oco_internal.h", "oco_ctx.h", "mixed_core.h", "fp64_core.h", "disk_core.h",
           "batch_layout.h", "fortran_records.h"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build failed: {os.path.basename(cmd[-1])}")
    return r


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "oco.h")]
    objs = []
    for src, extra in UNITS:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        if force or _newer(obj, [path, __file__] + hdrs):
            cmd = [NVCC] + COMMON + extra + ["-c", "-o", obj, path]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            r = _run(cmd)
            if verbose:
                sys.stdout.write(r.stderr)
        objs.append(obj)
    for src, extra in HOST_UNITS:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(BUILD, src.replace(".cpp", ".o"))
        if force or _newer(obj, [path, __file__] + hdrs):
            _run([NVCC] + COMMON + extra + ["-x", "cu", "-c", "-o", obj, path])
        objs.append(obj)
    if force or _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart=static", "-o", LIB] + objs)
    drv = os.path.join(CSRC, "flux_feautrier_b200.cpp")
    if os.path.exists(drv) and (force or _newer(DRIVER, [drv, LIB])):
        _run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
              "-o", DRIVER, drv, f"-L{PKG}", "-loco_b200", "-Wl,-rpath,$ORIGIN"])
    return LIB


def clean():
    shutil.rmtree(BUILD, ignore_errors=True)
    for f in (LIB, DRIVER):
        if os.path.exists(f):
            os.remove(f)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
