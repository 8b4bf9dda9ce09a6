"""Build the in-tree CUDA libraries for sm_100a.

The libraries are compiled with nvcc directly (no JIT cache); every kernel is sm_100a-only.
  libhappyray_b200.so       IEEE arithmetic (no fast-math, no FMA contraction): build and
                            traversal results are the oracle's, bit for bit.
  libhappyray_b200_fast.so  the same C-ABI with the traversal kernels (trace.cu, jobs.cu)
                            compiled with FMA contraction, approximate division, reciprocal
                            and square root, and flush-to-zero; every other file (grid build,
                            sort, host code) is the IEEE build's, so grids stay bit-exact and
                            ray results are within the floating-point tolerance of the ray
                            queries (ids equal except at ties, t, u, v within 1e-5 relative of
                            FP64) instead of bit-exact.  Opt-in (HAPPYRAY_B200_ARITH=fast, or
                            link it).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
OUT = PKG / "libhappyray_b200.so"
OUT_FAST = PKG / "libhappyray_b200_fast.so"
OBJDIR = PKG / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-lineinfo", "-O3", "-std=c++17",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-I", str(INCLUDE), "-I", str(CSRC),
]
FAST_FLAGS = [f for f in NVCC_FLAGS if f not in ("-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false")]
FAST_FLAGS = [f.replace("-ffp-contract=off", "-ffp-contract=fast") for f in FAST_FLAGS]
FAST_FLAGS += ["-fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=true"]
FAST_SOURCES = ("trace.cu", "jobs.cu")   # the traversal kernels of the fast build


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libhappyray_b200.so")
    return exe


def _sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _headers():
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))


def _stale(out: Path, deps) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, verbose: bool, extra, fast: bool = False) -> Path:
    obj = (OBJDIR / "fast" if fast else OBJDIR) / (src.name + ".o")
    if not _stale(obj, [src] + _headers()) and not extra:
        return obj
    cmd = [nvcc()] + (FAST_FLAGS if fast else NVCC_FLAGS) + list(extra) + ["-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr, file=sys.stderr)
    return obj


def build(verbose: bool = False, extra=(), fast: bool = False) -> Path:
    """Compile every .cu under csrc/ and link libhappyray_b200.so, or with fast the
    fast-arithmetic libhappyray_b200_fast.so (incremental)."""
    (OBJDIR / "fast" if fast else OBJDIR).mkdir(parents=True, exist_ok=True)
    out = OUT_FAST if fast else OUT
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose, extra, fast and s.name in FAST_SOURCES), srcs))
    if _stale(out, objs) or extra:
        tmp = out.with_suffix(".so.tmp")
        cmd = [nvcc()] + ARCH + ["-shared", "-o", str(tmp)] + [str(o) for o in objs] + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, out)
    return out


def build_all(verbose: bool = False) -> None:
    """Both libraries."""
    build(verbose)
    build(verbose, fast=True)


if __name__ == "__main__":
    v = "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    print(build(verbose=v, extra=extra, fast="--fast" in sys.argv))
