"""Build recipe of libnfb200.so (sm_100a) in-tree.

    python abacus-public_b200/build.py [-v] [--ptxas-v]

Each .cu under csrc/ is compiled with nvcc for sm_100a only and linked into
abacus-public_b200/lib/libnfb200.so.  The library is plain C ABI
(include/nf_capi.h); nothing here depends on torch.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libnfb200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-ftz=true", "-prec-div=true",
              "-prec-sqrt=true", "-fmad=true", "-Xcompiler", "-fPIC,-O2",
              f"-I{ROOT / 'include'}", f"-I{CSRC}"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise FileNotFoundError("nvcc not found")


def sources():
    return sorted(CSRC.glob("*.cu")) + sorted((CSRC / "host").glob("*.cpp")) \
        if (CSRC / "host").exists() else sorted(CSRC.glob("*.cu"))


def _stale(src: pathlib.Path, obj: pathlib.Path) -> bool:
    if not obj.exists():
        return True
    deps = [src] + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + \
        list((ROOT / "include").glob("*.h"))
    return any(d.stat().st_mtime > obj.stat().st_mtime for d in deps)


def compile_one(src: pathlib.Path, ptxas_v: bool, verbose: bool) -> pathlib.Path:
    obj = OBJ / (src.stem + ".o")
    if not _stale(src, obj):
        return obj
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd = [nvcc(), "-x", "cu"] + ARCH + NVCC_FLAGS + ["-c", str(src), "-o", str(obj)]
    if ptxas_v:
        cmd += ["-Xptxas", "-v"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    if ptxas_v or verbose:
        sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False, ptxas_v: bool = False) -> pathlib.Path:
    OBJ.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: compile_one(s, ptxas_v, verbose), srcs))
    if LIB.exists() and all(o.stat().st_mtime <= LIB.stat().st_mtime for o in objs):
        return LIB
    cmd = [nvcc()] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] + \
        ["-lcudart", "-lpthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-v", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    a = ap.parse_args()
    print(build(verbose=a.v, ptxas_v=a.ptxas_v))
