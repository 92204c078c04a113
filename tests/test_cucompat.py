"""The reference-compatible per-operator entry points (include/
smaug_cukernels.h, libsmaug_cu2d.so / libsmaug_cu3d.so): the libraries export
every function the header declares, the header's struct layouts are those of
the reference's iotypes.h (checked where the reference sources are present),
and the reference-shaped host loop (host/ref_loop.c) links against them.
Runs without a GPU."""
from __future__ import annotations

import ctypes
import re
import subprocess
from pathlib import Path

import pytest

from oracle.ref_shim import reference_root
from smaug_b200.build import COMPAT, LIBDIR, compat_lib, ref_loop_exe

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "smaug_cukernels.h"


def declared():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*(\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_single_step_set():
    names = declared()
    for must in ["cuinit", "initgrid", "cuboundary", "cuupdate", "cucomputedervfields", "cucentdiff1", "cucentdiff2",
                 "cuadvance", "cugrav", "cucomputec", "cucomputemaxc", "cucomputemaxcourant", "cugetdtvisc1",
                 "cuhyperdifvisc1ir", "cuhyperdifvisc1r", "cuhyperdifvisc1l", "cuhyperdifrhosource1",
                 "cuhyperdifesource1", "cuhyperdifmomsource1", "cuhyperdifmomsourcene1", "cuhyperdifbsource1",
                 "cuhyperdifbsourcene1", "cusource", "cudivb"]:
        assert must in names, must


@pytest.mark.parametrize("ndim", [2, 3])
def test_libraries_export_every_declared_function(ndim):
    lib = ctypes.CDLL(str(compat_lib(ndim)))
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.parametrize("ndim", [2, 3])
def test_ref_loop_links(ndim):
    r = subprocess.run([str(ref_loop_exe(ndim))], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


_LAYOUT_MEMBERS = ["n", "ng", "npgp", "fullgridini", "hdmean", "xmax", "xmin", "nt", "it", "tmax", "qt", "boundu",
                   "boundl", "cmax", "maxcourant", "steeringenabled", "dt", "dx", "gamma", "mu", "eta", "g", "sodifon",
                   "rkon", "moddton", "divbon", "divbfix", "cfgsavefrequency", "hyperdifmom", "mode", "readini",
                   "courant", "maxviscoef", "dtdiffvisc", "chyp", "chyp3", "test", "boundtype", "gpid", "npe",
                   "noghost"]


def _layout(tmp_path, include: str, defines: list) -> list:
    src = tmp_path / "lay.c"
    body = "".join(f'  printf("%zu\\n", offsetof(struct params, {m}));\n' for m in _LAYOUT_MEMBERS)
    src.write_text(f"#include <stdio.h>\n#include <stddef.h>\n{include}\nint main(void){{\n"
                   '  printf("%zu\\n%zu\\n%zu\\n", sizeof(struct params), sizeof(struct state), sizeof(struct bparams));\n'
                   f"{body}  return 0;\n}}\n")
    exe = tmp_path / "lay"
    subprocess.run(["gcc", "-w", *defines, str(src), "-o", str(exe)], check=True)
    return subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()


@pytest.mark.skipif(reference_root() is None, reason="reference sources not present")
@pytest.mark.parametrize("ndim", [2, 3])
def test_struct_layouts_equal_reference(tmp_path, ndim):
    """struct params / state / bparams of smaug_cukernels.h have the sizes and
    member offsets of the reference's iotypes.h and iobparams.h."""
    inc = reference_root() / "dev" / "smaug" / "include"
    ref = _layout(tmp_path, '#include "iotypes.h"\n#include "iobparams.h"',
                  ["-I", str(inc), "-DUSE_SAC" if ndim == 2 else "-DUSE_SAC_3D"])
    ours = _layout(tmp_path, '#include "smaug_cukernels.h"', ["-I", str(HEADER.parent), f"-DSMAUG_CU_NDIM={ndim}"])
    assert ours == ref
