"""Build the CUDA library ``libbt200.so`` in-tree for the B200 (sm_100a).

``python -m beamtracer_b200.build`` compiles every ``csrc/*.cu`` with nvcc into
``beamtracer_b200/libbt200.so``.  No multiply-add is contracted (``--fmad=false``): the
kernels round exactly as their expressions are written, as the reference's CPU kernels do
-- except ``trace_fast.cu``, the tracer built again with contracted multiply-adds.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIBRARY = HERE / "libbt200.so"
INCLUDE = HERE.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-warn-spills"]
#: Sources built with contracted multiply-adds (every other one rounds as it is written).
CONTRACTED = {"trace_fast.cu"}
OBJECTS = HERE / "_build"


def sources() -> list[Path]:
    """The CUDA sources of the library."""
    return sorted(CSRC.glob("*.cu"))


def _stale() -> bool:
    if not LIBRARY.exists():
        return True
    built = LIBRARY.stat().st_mtime
    inputs = [*sources(), *CSRC.glob("*.cuh"), *INCLUDE.glob("*.h")]
    return any(p.stat().st_mtime > built for p in inputs)


def nvcc() -> str:
    """The nvcc to build with."""
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(found).exists():
        raise RuntimeError("nvcc is not available: cannot build libbt200.so")
    return found


def _compile(source: Path, verbose: bool) -> Path:
    fmad = "--fmad=true" if source.name in CONTRACTED else "--fmad=false"
    out = OBJECTS / (source.stem + ".o")
    command = [nvcc(), *ARCH, *COMMON, fmad, f"-I{INCLUDE}", "-c", str(source), "-o", str(out)]
    if verbose:
        command.insert(1, "-Xptxas=-v")
    result = subprocess.run(command, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"nvcc failed on {source.name}:\n{result.stdout}\n{result.stderr}")
    if verbose:
        print(result.stdout, result.stderr, file=sys.stderr)
    return out


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the library if it is missing or older than its sources; return its path.
    Every source is compiled on its own (with its own multiply-add rule), in parallel,
    then linked."""
    from concurrent.futures import ThreadPoolExecutor

    if not force and not _stale():
        return LIBRARY
    OBJECTS.mkdir(exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        objects = list(pool.map(lambda src: _compile(src, verbose), sources()))
    tmp = LIBRARY.with_suffix(f".so.tmp{os.getpid()}")
    command = [nvcc(), *ARCH, "-shared", *map(str, objects), "-o", str(tmp)]
    result = subprocess.run(command, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"nvcc failed to link:\n{result.stdout}\n{result.stderr}")
    os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    print(build(force=True, verbose="-v" in sys.argv))
