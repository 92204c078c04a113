"""Build the CUDA library in-tree: smaug-all_b200/lib/libsmaug_b200.so.

nvcc cross-compiles for sm_100a (B200) on a machine without a GPU.  The stage
kernels are compiled twice: stage_exact.cu with -fmad=false (bit-reproducible
against the CPU oracle) and stage_fast.cu with FMA contraction.  stage_fast.cu
also flushes FP32 subnormals to zero (-ftz=true; FP64 arithmetic is not
affected): the mixed path's hyperviscosity coefficient is a ratio of
differences that is bounded by 5 in exact arithmetic, and subnormal operands
(the far tails of a wave running into a uniform region) break that bound.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parents[2]          # smaug-all_b200/
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libsmaug_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "nvcc")
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr"] + ARCH

UNITS = [
    ("stage_exact.cu", ["-fmad=false"]),
    ("stage_fast.cu", ["-fmad=true", "-ftz=true"]),
    ("batch_k2f.cu", ["-fmad=true", "-ftz=true"]),
    ("batch_k2d.cu", ["-fmad=true", "-ftz=true"]),
    ("batch_k3f.cu", ["-fmad=true", "-ftz=true"]),
    ("batch_k3d.cu", ["-fmad=true", "-ftz=true"]),
    ("smaug_capi.cu", []),
    ("smaug_batch.cu", []),
    ("smaug_vacio.cpp", ["-Xcompiler", "-ffp-contract=off"]),
]


HOST_DRIVER = PKG / "host" / "smaug_run.c"
HOST_EXE = LIBDIR / "smaug_run"


def build_host_driver() -> Path:
    """The C host driver (host/smaug_run.c), linked against the library; it
    sits beside the library and finds it through its run path."""
    cuda = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
    cmd = ["gcc", "-O2", "-std=c99", "-Wall", "-I", str(PKG.parent / "include"), "-I", str(cuda / "include"),
           str(HOST_DRIVER), "-L", str(LIBDIR), "-lsmaug_b200", "-L", str(cuda / "lib64"), "-lcudart",
           "-Wl,-rpath,$ORIGIN", "-o", str(HOST_EXE)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"host driver build failed:\n{' '.join(cmd)}\n{r.stderr[-4000:]}")
    return HOST_EXE


def sources():
    # this file too: its flags are part of what the library is built from
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp")) + sorted(CSRC.glob("*.cuh")) + sorted(
        CSRC.glob("*.inc")) + [
        PKG.parent / "include" / "smaug_b200.h", PKG.parent / "include" / "smaug_cukernels.h",
        Path(__file__).resolve(), HOST_DRIVER, REF_LOOP]


def up_to_date() -> bool:
    if not LIB.exists() or not HOST_EXE.exists() or not all((LIBDIR / e).exists() for _, _, e in COMPAT):
        return False
    t = LIB.stat().st_mtime
    return all(s.stat().st_mtime <= t for s in sources())


# The reference-compatible per-operator entry points (include/smaug_cukernels.h),
# one library per dimensionality, built without FMA contraction, and the
# reference-shaped host loop over each (host/ref_loop.c).
COMPAT = [(2, "libsmaug_cu2d.so", "smaug_ref_loop2d"), (3, "libsmaug_cu3d.so", "smaug_ref_loop3d")]
REF_LOOP = PKG / "host" / "ref_loop.c"


def compat_lib(ndim: int) -> Path:
    return LIBDIR / dict((d, lib) for d, lib, _ in COMPAT)[ndim]


def ref_loop_exe(ndim: int) -> Path:
    return LIBDIR / dict((d, exe) for d, _, exe in COMPAT)[ndim]


def build_compat(objdir: Path) -> None:
    def one(entry):
        D, lib, exe = entry
        obj = objdir / f"smaug_cucompat{D}d.o"
        cmd = [NVCC, *COMMON, "-fmad=false", f"-DSMAUG_CU_NDIM={D}", "-c", str(CSRC / "smaug_cucompat.cu"),
               "-o", str(obj)]
        steps = [cmd,
                 [NVCC, "-shared", *ARCH, "-o", str(LIBDIR / lib), str(obj), "-L", str(LIBDIR), "-lsmaug_b200",
                  "-lcudart", "-Xlinker", "-rpath=$ORIGIN"],
                 ["gcc", "-O2", "-std=c99", "-Wall", f"-DSMAUG_CU_NDIM={D}", "-I", str(PKG.parent / "include"),
                  str(REF_LOOP), "-L", str(LIBDIR), f"-l:{lib}", "-lsmaug_b200", "-Wl,-rpath,$ORIGIN", "-o",
                  str(LIBDIR / exe)]]
        for c in steps:
            r = subprocess.run(c, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"compat build failed:\n{' '.join(c)}\n{r.stderr[-6000:]}")

    with ThreadPoolExecutor(max_workers=len(COMPAT)) as ex:
        list(ex.map(one, COMPAT))


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and up_to_date():
        return LIB
    LIBDIR.mkdir(parents=True, exist_ok=True)
    objdir = LIBDIR / "obj"
    objdir.mkdir(exist_ok=True)

    def one(unit):
        src, extra = unit
        obj = objdir / (Path(src).stem + ".o")
        cmd = [NVCC, *COMMON, *extra, "-Xptxas", "-v", "-c", str(CSRC / src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{' '.join(cmd)}\n{r.stderr[-6000:]}")
        (objdir / (Path(src).stem + ".ptxas.txt")).write_text(r.stderr)
        if verbose:
            print(r.stderr)
        return obj

    with ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        objs = list(ex.map(one, UNITS))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [NVCC, "-shared", *ARCH, "-o", str(tmp), *map(str, objs), "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
    os.replace(tmp, LIB)
    build_host_driver()
    build_compat(objdir)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
