"""Build ``libfis_b200.so`` in-tree with nvcc for sm_100a.

    python -c "import fis.build as b; b.build()"

The library holds every CUDA kernel of the package and the C ABI of
``include/fis.h``.  It is compiled with ``-fmad=false`` on top of the
explicit ``__f*_rn`` intrinsics: no multiply-add of the step may be contracted
into an FMA, whose single rounding would differ from the reference's.
"""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = ROOT / "csrc"
INCLUDE = ROOT.parent / "include"
OUT = PKG / "libfis_b200.so"

SOURCES = ("fis_engine.cu", "fis_evspmv.cu", "fis_graded.cu", "fis_calibrate.cu")
ARCH = "-gencode=arch=compute_100a,code=sm_100a"


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise FileNotFoundError("nvcc not found")


def command(out=OUT, extra=()):
    return [nvcc(), ARCH, "-lineinfo", "-O3", "-fmad=false", "-std=c++17",
            "-I" + str(INCLUDE), "-I" + str(CSRC), "-shared", "-Xcompiler", "-fPIC",
            "-o", str(out), *extra, *[str(CSRC / s) for s in SOURCES]]


def stale(out=OUT):
    if not out.exists():
        return True
    t = out.stat().st_mtime
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + [INCLUDE / "fis.h"]
    return any(d.stat().st_mtime > t for d in deps)


def build(force=False, verbose=False, out=OUT, extra=()):
    """Compile if any source is newer than the library; return its path."""
    if not force and not stale(out):
        return out
    cmd = command(out, extra)
    if verbose:
        print(" ".join(cmd))
    tmp = out.with_suffix(".tmp.so")
    cmd[cmd.index("-o") + 1] = str(tmp)
    subprocess.run(cmd, check=True)
    os.replace(tmp, out)
    return out


if __name__ == "__main__":
    build(force=True, verbose=True)
