"""Builds the in-tree shared library gpugraph_b200/libmapgraph_b200.so.

Every CUDA source is compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``) with the CUDA runtime linked
statically, so the library does not depend on which libcudart the host process
(e.g. PyTorch) has loaded. Objects go to gpugraph_b200/_build/; only sources
whose inputs changed are recompiled.
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libmapgraph_b200.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-O3", f"-I{INCLUDE}", f"-I{CSRC}"]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-pthread", f"-I{INCLUDE}", f"-I{CSRC}"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted(list(CSRC.rglob("*.cu")) + list(CSRC.rglob("*.cpp")))


def _digest(src: Path, flags: list[str]) -> str:
    h = hashlib.sha256()
    h.update(" ".join(flags).encode())
    h.update(src.read_bytes())
    for hdr in sorted(list(CSRC.rglob("*.cuh")) + list(CSRC.rglob("*.h")) + list(INCLUDE.glob("*.h"))):
        h.update(hdr.read_bytes())
    return h.hexdigest()[:16]


def _compile(src: Path, verbose_ptxas: bool) -> Path:
    rel = src.relative_to(CSRC)
    obj = BUILD / (str(rel).replace(os.sep, "__") + ".o")
    if src.suffix == ".cu":
        flags = ARCH + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose_ptxas else [])
        cmd = [nvcc()] + flags + ["-c", str(src), "-o", str(obj)]
    else:
        flags = CXX_FLAGS
        cmd = [os.environ.get("CXX", "g++")] + flags + ["-c", str(src), "-o", str(obj)]
    stamp = obj.with_suffix(".stamp")
    dig = _digest(src, flags)
    if obj.exists() and stamp.exists() and stamp.read_text() == dig and not verbose_ptxas:
        return obj
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    if verbose_ptxas and res.stderr:
        sys.stderr.write(res.stderr)
    stamp.write_text(dig)
    return obj


def build(verbose_ptxas: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(16, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    tmp = LIB.with_suffix(".so.tmp")
    # --no-undefined: a kernel stub declared in one file and renamed in another
    # fails the build instead of the first dlopen
    cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", str(tmp)] + [str(o) for o in objs] + [
        "-Xcompiler", "-pthread", "-Xlinker", "--no-undefined", "-lrt", "-ldl"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose_ptxas="-v" in sys.argv))
