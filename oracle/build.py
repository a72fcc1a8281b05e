"""Build recipes of the oracle (test infrastructure only).

- ``build_port()``: the C restatement in oracle/port/ -> oracle/_build/liboracle.so (gcc, -ffp-contract=off).
- ``build_ref()``: the reference's own CPU sources, compiled where they lie with the reference's floating-point
  policy (cmake/FloatingPoint.cmake:8-26: -ffp-contract=off -fno-fast-math, -march=x86-64-v3) and linked with
  oracle/ref_harness.cpp into oracle/_ref/libballa_ref.so. It needs the reference tree: REFERENCE_ROOT, else a
  directory named ``reference`` beside this repository; where neither exists the prebuilt library is used as it
  is. No reference source is copied.

Run ``python -m oracle.build`` from the repository root, or call the functions.
"""
from __future__ import annotations

import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
PORT_SO = HERE / "_build" / "liboracle.so"
REF_SO = HERE / "_ref" / "libballa_ref.so"

# The reference's sources on the path (SensorModel and its maps/params; the host WindowEngine).
REF_SOURCES = [
    "src/sensor/params.cpp",
    "src/sensor/param_fields.cpp",
    "src/sensor/maps.cpp",
    "src/sensor/noise_tables.cpp",
    "src/sensor/thread_pool.cpp",
    "src/sensor/sensor_model.cpp",
    "src/sensor/resim.cpp",
    "src/engine/window.cpp",
    "src/engine/par_host.cpp",
    "src/export/raw_writer.cpp",
]
REF_FLAGS = ["-std=c++20", "-O3", "-DNDEBUG", "-ffp-contract=off", "-fno-fast-math", "-march=x86-64-v3", "-fPIC"]
PORT_FLAGS = ["-std=c11", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-Wall"]


def reference_root() -> Path:
    env = os.environ.get("REFERENCE_ROOT")
    return Path(env) if env else HERE.parent.parent / "reference"


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def _newer(out: Path, inputs: list[Path]) -> bool:
    return out.exists() and all(out.stat().st_mtime >= p.stat().st_mtime for p in inputs if p.exists())


def build_port(force: bool = False) -> Path:
    srcs = [HERE / "port" / "oracle.c", HERE / "port" / "oracle.h"]
    if not force and _newer(PORT_SO, srcs):
        return PORT_SO
    PORT_SO.parent.mkdir(parents=True, exist_ok=True)
    tmp = PORT_SO.with_suffix(".tmp.so")
    _run(["gcc", *PORT_FLAGS, "-shared", "-o", str(tmp), str(srcs[0]), "-lm"])
    tmp.replace(PORT_SO)
    return PORT_SO


def build_ref(force: bool = False) -> Path | None:
    """Compiles the reference harness; None when the reference tree is absent and nothing is prebuilt."""
    root = reference_root()
    if not (root / "src" / "sensor" / "pixel.h").exists():
        return REF_SO if REF_SO.exists() else None
    harness = HERE / "ref_harness.cpp"
    deps = [harness, HERE / "port" / "oracle.c", HERE / "port" / "oracle.h"] + [root / s for s in REF_SOURCES]
    if not force and _newer(REF_SO, deps):
        return REF_SO
    obj_dir = HERE / "_ref" / "obj"
    obj_dir.mkdir(parents=True, exist_ok=True)
    inc = ["-I", str(root / "src"), "-I", str(HERE)]
    jobs = []
    for s in REF_SOURCES:
        o = obj_dir / (s.replace("/", "_") + ".o")
        if force or not _newer(o, [root / s]):
            jobs.append(["g++", *REF_FLAGS, *inc, "-c", str(root / s), "-o", str(o)])
    jobs.append(["g++", *REF_FLAGS, *inc, "-c", str(harness), "-o", str(obj_dir / "ref_harness.o")])
    jobs.append(["gcc", *PORT_FLAGS, "-c", str(HERE / "port" / "oracle.c"), "-o", str(obj_dir / "oracle_port.o")])
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        list(ex.map(_run, jobs))
    objs = [str(obj_dir / (s.replace("/", "_") + ".o")) for s in REF_SOURCES]
    objs += [str(obj_dir / "ref_harness.o"), str(obj_dir / "oracle_port.o")]
    tmp = REF_SO.with_suffix(".tmp.so")
    _run(["g++", "-shared", "-o", str(tmp), *objs, "-lpthread", "-Wl,--no-undefined"])
    tmp.replace(REF_SO)
    shutil.rmtree(obj_dir, ignore_errors=True) if os.environ.get("ORACLE_CLEAN_OBJ") else None
    return REF_SO


if __name__ == "__main__":
    print(build_port(force=True))
    print(build_ref(force=True))
