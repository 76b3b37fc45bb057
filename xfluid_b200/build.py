"""Builds libxfp.so (the CUDA library behind include/xfp.h) in-tree for sm_100a.

    python -m xfluid_b200.build          # build if sources changed
    python -m xfluid_b200.build --force

nvcc compiles every .cu under xfluid_b200/csrc/ for
``-gencode arch=compute_100a,code=sm_100a`` with the system g++ as host
compiler (so the library shares the process's libstdc++).
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
LIB = PKG / "libxfp.so"
INCLUDE = ROOT / "include"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def host_cxx() -> str:
    return "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = sources() + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not _stale():
        return LIB
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    common = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-ccbin", host_cxx(), f"-I{INCLUDE}", f"-I{CSRC}", "--expt-relaxed-constexpr"]
    if verbose:
        common += ["-Xptxas", "-v"]
    objs = []
    procs = []
    for src in sources():
        obj = objdir / (src.stem + ".o")
        objs.append(obj)
        cmd = common + ["-c", str(src), "-o", str(obj)]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = False
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stderr.write(out.decode(errors="replace"))
        if p.returncode != 0:
            failed = True
    if failed:
        raise RuntimeError("nvcc failed")
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.check_call([nvcc(), *ARCH, "-shared", "-ccbin", host_cxx(), *map(str, objs), "-o", str(tmp),
                           "-lcudart"])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
