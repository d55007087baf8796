"""Build the sm_100a library ``lib/libocean_b200.so`` and the ``bin/ocean3d5_b200``
executable in-tree with nvcc (cross-compiles without a GPU).

FP contraction is disabled (``-fmad=false``, ``-ffp-contract=off``): the fp64
step is bit-for-bit equal to the reference's NumPy arithmetic only when every
multiply and add rounds separately. The 3D step kernels are compiled a second
time for the mixed-precision path (``-DOC_MIXED``: FP32 fields, contraction on).
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "lib"
BIN_DIR = PKG / "bin"
LIB = LIB_DIR / "libocean_b200.so"
EXE = BIN_DIR / "ocean3d5_b200"
# executables over the C ABI: (main source, binary)
MAINS = [("ocean3d5_main.cpp", EXE), ("helmholtz_bench_main.cpp", BIN_DIR / "helmholtz_bench_b200"),
         ("eos_bench_main.cpp", BIN_DIR / "eos_bench_b200")]
SOURCES = ["step_kernels.cu", "step2d_kernels.cu", "helmholtz.cu", "helm_refined.cu", "capi.cu", "mixed.cu", "adjoint.cu",
           "thomas_noalloc.cu", "standalone.cu", "protocol.cpp"]
# (source, object, flags replacing the fp64 contraction flags): the mixed-precision build of the 3D kernels
MIXED = [("step_kernels.cu", "step_kernels_mixed.o", ["-DOC_MIXED", "-Xcompiler", "-fPIC"])]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-Wno-deprecated-gpu-targets", "-O3", "-std=c++17", "-lineinfo", "--extended-lambda", f"-I{ROOT / 'include'}",
          f"-I{CSRC}"]
FLAGS = COMMON + ["-fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    deps = ([CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "ocean_b200.h"]
            + [CSRC / m for m, _ in MAINS])
    if not force and not _stale(LIB, deps) and not any(_stale(exe, deps) for _, exe in MAINS):
        return LIB
    LIB_DIR.mkdir(exist_ok=True)
    BIN_DIR.mkdir(exist_ok=True)
    obj_dir = PKG / "_build"
    obj_dir.mkdir(exist_ok=True)
    objs = []
    cc = nvcc()
    for src in SOURCES:
        obj = obj_dir / (Path(src).stem + ".o")
        cmd = [cc, *ARCH, *FLAGS, "-c", str(CSRC / src), "-o", str(obj)]
        if src.endswith(".cpp"):
            cmd = [cc, *FLAGS, "-x", "c++", "-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    for src, name, extra in MIXED:
        obj = obj_dir / name
        cmd = [cc, *ARCH, *COMMON, *extra, "-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run([cc, *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart"], check=True)
    os.replace(tmp, LIB)
    for main, exe in MAINS:
        subprocess.run([cc, *FLAGS, "-x", "c++", str(CSRC / main), "-o", str(exe), f"-L{LIB_DIR}",
                        "-locean_b200", "-Xlinker", "-rpath,$ORIGIN/../lib", "-lcudart"], check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
