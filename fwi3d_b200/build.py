"""Build the native parts of fwi3d_b200 in-tree.

  fwi3d_b200/lib/libfwi3d.so        the CUDA library behind include/fwi3d.h
  fwi3d_b200/bin/modeling.exe       drop-in mains (C++ over the C ABI) that
  fwi3d_b200/bin/migration.exe      read the reference's parameters.txt
  fwi3d_b200/bin/inversion.exe

Everything is compiled for sm_100a only.  Run `python -m fwi3d_b200.build`.
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
HOST = PKG / "host"
LIB_DIR = PKG / "lib"
BIN_DIR = PKG / "bin"
LIB = LIB_DIR / "libfwi3d.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-O3"]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found")
    return exe


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and (res.stdout or res.stderr):
        sys.stderr.write(res.stdout + res.stderr)


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def build_library(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> Path:
    LIB_DIR.mkdir(exist_ok=True)
    units = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    srcs = units + sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "fwi3d.h"]
    if force or ptxas_info or _stale(LIB, srcs):
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-shared", "-o", str(LIB), *map(str, units)]
        if ptxas_info:
            cmd.insert(1, "-Xptxas=-v")
        _run(cmd, verbose)
    return LIB


def build_mains(force: bool = False, verbose: bool = False) -> list[Path]:
    """C++ drop-in executables linked against libfwi3d.so (rpath $ORIGIN/../lib)."""
    BIN_DIR.mkdir(exist_ok=True)
    common = sorted(HOST.glob("*.cpp"))
    mains = [p for p in common if p.stem.endswith("_main")]
    libsrc = [p for p in common if p not in mains]
    hdrs = sorted(HOST.glob("*.hpp")) + [ROOT / "include" / "fwi3d.h", LIB]
    out = []
    for m in mains:
        exe = BIN_DIR / (m.stem.replace("_main", "") + ".exe")
        if force or _stale(exe, [m, *libsrc, *hdrs]):
            cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", f"-I{ROOT / 'include'}", f"-I{HOST}",
                   str(m), *map(str, libsrc), f"-L{LIB_DIR}", "-lfwi3d",
                   "-Wl,-rpath,$ORIGIN/../lib", "-o", str(exe)]
            _run(cmd, verbose)
        out.append(exe)
    return out


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_library(force=force, verbose=verbose)
    if HOST.exists() and any(HOST.glob("*_main.cpp")):
        build_mains(force=force, verbose=verbose)


if __name__ == "__main__":
    args = set(sys.argv[1:])
    if "--ptxas" in args:
        build_library(ptxas_info=True, verbose=True)
    else:
        build_all(force="--force" in args, verbose=True)
