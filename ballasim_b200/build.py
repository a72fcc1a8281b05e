"""Builds the CUDA library of the package in place: ballasim_b200/_lib/libballasim_b200.so.

nvcc compiles every .cu source in csrc/ for sm_100a only (-gencode arch=compute_100a,code=sm_100a) with the
floating-point policy the bitwise contract needs: no fused multiply-add on the device (--fmad=false) or the
host (-ffp-contract=off), IEEE division and square root, no flush to zero. The CUDA runtime is linked
statically, so the library needs only the driver at run time. The host-only .cpp sources (the SHA-256 of the event files, which
uses the x86 SHA extensions) go through g++ with the same host policy. Run ``python -m ballasim_b200.build``.
"""
from __future__ import annotations

import os
import subprocess
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "_lib" / "libballasim_b200.so"
INCLUDE = HERE.parent / "include"

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "--fmad=false", "-ftz=false", "-prec-div=true", "-prec-sqrt=true",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
    "-I", str(INCLUDE),
]


def nvcc() -> str:
    cand = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    return cand if Path(cand).exists() else "nvcc"


CXX_FLAGS = ["-std=c++17", "-O3", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-I", str(INCLUDE)]


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _deps() -> list[Path]:
    return sources() + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))


def up_to_date() -> bool:
    return LIB.exists() and all(LIB.stat().st_mtime >= p.stat().st_mtime for p in _deps())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and up_to_date():
        return LIB
    obj_dir = HERE / "_lib" / "obj"
    obj_dir.mkdir(parents=True, exist_ok=True)

    def compile_one(src: Path) -> Path:
        out = obj_dir / (src.stem + src.suffix.replace(".", "_") + ".o")
        if src.suffix == ".cpp":
            cmd = [os.environ.get("CXX", "g++"), *CXX_FLAGS, "-c", str(src), "-o", str(out)]
        else:
            cmd = [nvcc(), *NVCC_FLAGS, "-c", str(src), "-o", str(out)]
        if verbose and src.suffix == ".cu":
            cmd.insert(1, "-Xptxas=-v")
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stderr}")
        if verbose:
            print(r.stderr)
        return out

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(compile_one, sources()))
    tmp = LIB.with_suffix(".tmp.so")
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-cudart", "static", "-o", str(tmp),
           *map(str, objs)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed:\n{r.stderr}")
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    import sys

    print(build(force=True, verbose="-v" in sys.argv))
