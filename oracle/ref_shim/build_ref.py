#!/usr/bin/env python3
"""Host build of the SMAUG reference's own CUDA sources -- test infrastructure.

Builds ``oracle/_ref/libsmaug_ref2d.so``, ``oracle/_ref/libsmaug_ref3d.so`` and
``oracle/_ref/libsmaug_ref2d_drv.so`` (2-D with the spicule model's momentum
driver) from the reference's unmodified-on-disk sources under
``<reference>/dev/smaug/src`` (read-only), so that the reference itself pins the
oracle and the GPU path.  Nothing is copied into the repository: every
generated file lands in ``oracle/_ref/`` (git-ignored, shipped with the other
built libraries).

Recipe (our own; the reference Makefile is not run):

1. ``MODID`` templating exactly as ``dev/smaug/src/Makefile:177-245`` does with
   ``sed 's/MODID/<id>/g'``: gradops.cu / dervfields.cu / usersource.cu /
   init_user.cu become ``include/<name>_<id>.cuh`` next to the sources.
2. ``kernel<<<nb, nt[, smem]>>>(args);`` becomes ``SHIM_LAUNCH(nb, nt, kernel(args));``
   (cuda_host_shim.h runs the grid serially; every hot-path kernel writes only
   its own cell).  The four shared-memory max reductions are replaced by
   ``shim_blockmax`` with identical block maxima.
3. Three source patches, each a documented deviation of the pin:
   P1 hyperdifvisc1r.cu:1235,1253 -- ``hyperdifvisc1r_parallel`` stores q through
      the unpadded encoder ``encode3`` into the padded array wtemp2 while other
      threads zero that array in the same launch (a data race whose only
      surviving effect is garbage in the right-hand pad column).  Patched to
      ``encode3p2``; the value is then rewritten by hyperdifvisc1ar anyway and
      the pad column keeps the 0 that the zeroing pass writes.
   P2 computedervfields.cu:1353 -- ``temp[index]=0.0`` with ``index``
      uninitialised (undefined behaviour) becomes ``temp[iindex]=0.0``; those
      entries are already 0 at that point.
   P4 boundary.cu -- the model file's cuboundary is renamed model_cuboundary
      and bc_dispatch.inc (ours) becomes cuboundary: periodic and contcd4
      still go to the model file, cont / fixed / symm / asymm to the
      per-direction helpers of gradops.cu (the shipped model files each
      implement a different subset of the boundary types).
   P3 boundary.cu -- models/boundary.cu.sedov3d (periodic, contcd4 and fixed
      ghosts, 2-D and 3-D; the file the Makefile's sedov3d target installs) is
      used for every model.  Its boundary0_per_parallel/boundary1_per_parallel
      (models/boundary.cu.sedov3d:650,727) reset ``kp=0`` after decoding the
      thread index, so in 3-D only the k=0 plane of the x/y ghosts is ever
      refreshed; the two ``kp=0;`` statements are removed.  (The src/ copy of
      boundary.cu belongs to the fluxtube model and never fills periodic x
      ghosts; models/boundary.cu.ot is 2-D only.)
4. ``g++ -O2 -ffp-contract=off -fPIC`` with ``-DUSE_SAC`` (2-D) or
   ``-DUSE_SAC_3D`` (3-D), linked with ref_driver.cpp into a shared library.

Usage: python oracle/ref_shim/build_ref.py [--reference DIR] [--jobs N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import re
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ORACLE = HERE.parent
OUT = ORACLE / "_ref"

# Sources on the single-step hot path (make_inputs:76-98 minus host I/O,
# the unused hyperdifvisc1.cu and the MPI layer); divb.cu runs when the
# driver switches divbon / divbfix on.
KERNEL_SOURCES = {
    # file: [(template source, MODID)] -- Makefile:177-245
    "hyperdifmomsource1.cu": [("gradops.cu", "hdm1")],
    "hyperdifmomsourcene1.cu": [("gradops.cu", "hdmne1")],
    "hyperdifesource1.cu": [("gradops.cu", "hde1")],
    "hyperdifbsource1.cu": [("gradops.cu", "hdb1")],
    "hyperdifbsourcene1.cu": [("gradops.cu", "hdbne1")],
    "hyperdifrhosource1.cu": [("gradops.cu", "hdr1")],
    "nushk1.cu": [("gradops.cu", "nshk")],
    "hyperdifvisc1l.cu": [("gradops.cu", "hdv1l")],
    "hyperdifvisc1r.cu": [("gradops.cu", "hdv1r")],
    "centdiff1.cu": [("gradops.cu", "cd1"), ("dervfields.cu", "cd1"), ("usersource.cu", "cd1")],
    "centdiff2.cu": [("gradops.cu", "cd2"), ("dervfields.cu", "cd2"), ("usersource.cu", "cd2")],
    "computedervfields.cu": [("gradops.cu", "cdf"), ("dervfields.cu", "cdf")],
    "boundary.cu": [("gradops.cu", "b")],
    "init.cu": [("gradops.cu", "i"), ("init_user.cu", "i")],
    "update.cu": [("gradops.cu", "u")],
    "advance.cu": [("gradops.cu", "adv"), ("dervfields.cu", "adv")],
    "divb.cu": [("gradops.cu", "db"), ("dervfields.cu", "db")],
}

REDUCTIONS = {
    # kernel name -> write block max back to temp[b]
    "newreduction0computemax_parallel": 0,
    "newreduction0computemaxviscr_parallel": 0,
    "newreduction0computemaxviscl_parallel": 0,
    "newreduction0computemaxdtvisc_parallel": 1,
}

EXTRA_FLAGS = os.environ.get("SMAUG_REF_EXTRA_FLAGS", "").split()

LAUNCH_RE = re.compile(r"(\w+)\s*<<<(.*?)>>>\s*\(([^;]*)\)\s*;", re.S)


def _split_cfg(cfg: str) -> list[str]:
    return [c.strip() for c in cfg.split(",")]


FUNC_RE = re.compile(r"^(int|real|double)\s+(\w+)\s*\([^;{]*\)\s*\{", re.M)


def _match_brace(text: str, open_pos: int) -> int:
    """Index of the brace closing text[open_pos] ('{'), skipping comments and literals."""
    depth, i, n = 0, open_pos, len(text)
    while i < n:
        c = text[i]
        if text.startswith("//", i):
            i = text.find("\n", i)
            i = n if i < 0 else i
            continue
        if text.startswith("/*", i):
            i = text.find("*/", i + 2)
            i = n if i < 0 else i + 2
            continue
        if c in "\"'":
            j = i + 1
            while j < n and text[j] != c:
                j += 2 if text[j] == "\\" else 1
            i = j + 1
            continue
        if c == "{":
            depth += 1
        elif c == "}":
            depth -= 1
            if depth == 0:
                return i
        i += 1
    raise RuntimeError("unbalanced braces")


def add_missing_returns(text: str) -> str:
    """Most reference host wrappers are declared `int` but end without a
    return statement (e.g. centdiff1.cu:820-852).  In C++ that is undefined
    behaviour which g++ -O2 turns into a fall-through into unrelated code, so
    every non-void top-level function gets a trailing `return 0;` (a no-op
    where the function already returns)."""
    out, last = [], 0
    for m in FUNC_RE.finditer(text):
        if m.start() < last:
            continue
        close = _match_brace(text, m.end() - 1)
        out.append(text[last:close])
        out.append("\n  return 0; /* added by build_ref.py */\n")
        last = close
    out.append(text[last:])
    return "".join(out)


def transform(text: str, fname: str) -> str:
    def repl(m: re.Match) -> str:
        kern, cfg, args = m.group(1), _split_cfg(m.group(2)), m.group(3)
        if kern in REDUCTIONS:
            a = [x.strip() for x in args.split(",")]
            # (out, temp, ndimp)
            return (f"shim_blockmax((int)({cfg[0]}), (int)({cfg[1]}), {a[0]}, {a[1]}, "
                    f"{a[2]}, {REDUCTIONS[kern]});")
        return f"SHIM_LAUNCH({cfg[0]}, {cfg[1]}, {kern}({args}));"

    out = LAUNCH_RE.sub(repl, add_missing_returns(text))
    out = re.sub(r"extern\s+__shared__\s+(\w+)\s+(\w+)\s*\[\s*\]\s*;", r"static \1 \2[4096];", out)
    if fname == "hyperdifvisc1r.cu":
        n0 = out.count("wtemp2[encode3_hdv1r(p,i+1,j+1,k")
        out = out.replace("wtemp2[encode3_hdv1r(p,i+1,j+1,k", "wtemp2[encode3p2_hdv1r(p,i+1,j+1,k")
        if n0 != 2:
            raise RuntimeError(f"P1 patch expected 2 sites in hyperdifvisc1r.cu, found {n0}")
    if fname == "boundary.cu":
        out, n0 = re.subn(r"^kp=0;", "/* kp=0; removed by build_ref.py (P3) */", out, flags=re.M)
        if n0 != 2:
            raise RuntimeError(f"P3 patch expected 2 sites in boundary.cu.sedov3d, found {n0}")
        # P4: the other boundary types through the gradops.cu helpers
        out, n0 = re.subn(r"^int\s+cuboundary\s*\(", "int model_cuboundary(", out, flags=re.M)
        if n0 != 1:
            raise RuntimeError(f"P4 expected one cuboundary in boundary.cu.sedov3d, found {n0}")
        out += '\n#include "bc_dispatch.inc"\n'
    if fname == "computedervfields.cu":
        n0 = out.count("temp[index]=0.0;")
        out = out.replace("temp[index]=0.0;", "temp[iindex]=0.0;")
        if n0 != 1:
            raise RuntimeError(f"P2 patch expected 1 site in computedervfields.cu, found {n0}")
    return out


# Model files the Makefile's `ot` / `sedov3d` targets copy into src/
# (Makefile:23-140); the shipped src/usersource.cu and src/init_user.cu belong
# to another model.
TEMPLATE_FILES = {
    2: {"usersource.cu": "../models/usersource.cu.default", "init_user.cu": "../models/init_user.cu.ot"},
    3: {"usersource.cu": "../models/usersource.cu.default", "init_user.cu": "../models/init_user.cu.sedov3d"},
}

# Library variants: name -> (ndim, model files replacing TEMPLATE_FILES, extra
# defines).  "2d_drv" is the 2-D build with the spicule model's momentum
# driver (models/usersource.cu.spicule1, compiled in by USE_USERSOURCE).
VARIANTS = {
    "2d": (2, {}, []),
    "3d": (3, {}, []),
    "2d_drv": (2, {"usersource.cu": "../models/usersource.cu.spicule1"}, ["-DUSE_USERSOURCE"]),
}


SOURCE_FILES = {"boundary.cu": "../models/boundary.cu.sedov3d"}


def generate(ref_src: Path, build: Path, ndim: int, models: dict | None = None) -> list[Path]:
    (build / "src").mkdir(parents=True, exist_ok=True)
    (build / "include").mkdir(parents=True, exist_ok=True)
    done = set()
    outs = []
    for fname, templates in KERNEL_SOURCES.items():
        for tmpl, modid in templates:
            stem = tmpl[:-3]
            dst = build / "include" / f"{stem}_{modid}.cuh"
            if dst in done:
                continue
            files = dict(TEMPLATE_FILES[ndim], **(models or {}))
            src_file = ref_src / files.get(tmpl, tmpl)
            body = add_missing_returns(src_file.read_text(errors="replace").replace("MODID", modid))
            dst.write_text(body)
            done.add(dst)
        text = (ref_src / SOURCE_FILES.get(fname, fname)).read_text(errors="replace")
        dst = build / "src" / (fname[:-3] + ".cpp")
        dst.write_text(transform(text, fname))
        outs.append(dst)
    return outs


def compile_one(args):
    cmd, obj = args
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed for {obj}:\n{' '.join(cmd)}\n{r.stderr[-4000:]}")
    return obj


def build(reference: Path, variants=("2d", "3d", "2d_drv"), jobs: int = 8) -> None:
    ref_src = reference / "dev" / "smaug" / "src"
    if not ref_src.is_dir():
        raise FileNotFoundError(f"reference sources not found: {ref_src}")
    shim = HERE / "cuda_host_shim.h"
    driver = HERE / "ref_driver.cpp"
    OUT.mkdir(parents=True, exist_ok=True)
    for v in variants:
        d, models, extra = VARIANTS[v]
        build_dir = OUT / f"build{v}"
        srcs = generate(ref_src, build_dir, d, models)
        defs = (["-DUSE_SAC"] if d == 2 else ["-DUSE_SAC_3D"]) + extra
        base = ["g++", "-x", "c++", "-std=c++14", "-O2", "-ffp-contract=off", "-fPIC",
                "-fno-strict-aliasing", "-w", "-include", str(shim),
                "-I", str(ref_src), "-I", str(HERE)] + defs + EXTRA_FLAGS
        jobs_list = []
        objs = []
        for s in srcs + [driver]:
            obj = build_dir / (s.stem + ".o")
            jobs_list.append((base + ["-c", str(s), "-o", str(obj)], obj))
            objs.append(obj)
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            list(ex.map(compile_one, jobs_list))
        lib = OUT / f"libsmaug_ref{v}.so"
        cmd = ["g++", "-shared", "-o", str(lib)] + [str(o) for o in objs] + ["-lm"] + EXTRA_FLAGS
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
        print(f"built {lib}")
    build_hydro(reference)


# The hydrostatic-background helpers of the reference's spicule model
# (models/initialisation_user.h.spicule1_mpi): inte() (326-343), the trapezoid
# rule of its pressure integral, and temp() (345-360), its tanh temperature
# profile.  The two functions are cut out of the model file as they stand and
# compiled with a minimal prelude of the types they use, behind two extern "C"
# wrappers, into oracle/_ref/libsmaug_ref_hydro.so.
HYDRO_MODEL = "../models/initialisation_user.h.spicule1_mpi"
HYDRO_FUNCS = (r"^real\s+inte\s*\(", r"^void\s+temp\s*\(")
HYDRO_PRELUDE = """#include <math.h>
typedef double real;
struct params { int n[3]; };
enum { pos1 = 0 };
/* positions of the first coordinate along dim 0, one row (the only use) */
#define encode3_uin(p, i, j, k, f) ((f) * (p)->n[0] + (i))
"""
HYDRO_WRAP = """
extern "C" double ref_inte(const double *col, int n, int i, double dx) {
  real **w = new real *[n];
  for (int k = 0; k < n; ++k) w[k] = const_cast<real *>(col + k);
  const double r = inte(w, n, i, 0, dx);
  delete[] w;
  return r;
}
extern "C" void ref_temp(const double *z, int n, double *T) {
  struct params p = {{n, 1, 1}};
  int ii[3] = {0, 0, 0};
  temp(nullptr, const_cast<real *>(z), ii, &p, T);
}
"""


def build_hydro(reference: Path) -> Path:
    src = (reference / "dev" / "smaug" / "src" / HYDRO_MODEL).resolve().read_text(errors="replace")
    parts = [HYDRO_PRELUDE]
    for pat in HYDRO_FUNCS:
        m = re.search(pat, src, re.M)
        if not m:
            raise RuntimeError(f"{pat} not found in {HYDRO_MODEL}")
        close = _match_brace(src, src.index("{", m.end() - 1))
        parts.append(src[m.start():close + 1] + "\n")
    parts.append(HYDRO_WRAP)
    d = OUT / "buildhydro"
    d.mkdir(parents=True, exist_ok=True)
    cpp = d / "hydro_ref.cpp"
    cpp.write_text("".join(parts))
    lib = OUT / "libsmaug_ref_hydro.so"
    cmd = ["g++", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-w", "-o", str(lib), str(cpp), "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"hydro build failed:\n{r.stderr[-4000:]}")
    print(f"built {lib}")
    return lib


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None,
                    help="reference source tree (default: $SMAUG_REFERENCE, else ../reference beside the repo)")
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 4)
    ap.add_argument("--variants", default=",".join(VARIANTS))
    a = ap.parse_args()
    if a.reference is None:
        sys.path.insert(0, str(HERE.parents[1]))
        from oracle.ref_shim import reference_root
        ref = reference_root()
        if ref is None:
            ap.error("reference sources not found: pass --reference or set SMAUG_REFERENCE")
    else:
        ref = Path(a.reference)
    build(ref, tuple(a.variants.split(",")), a.jobs)
    return 0


if __name__ == "__main__":
    sys.exit(main())
