"""Builds the C-ABI shared library libluce_render_b200.so in this package directory.

Every CUDA source is compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``);
host C++ goes through nvcc's host compiler. Objects land in ``_build/`` at the repository
root and are rebuilt when a source or header is newer than its object.

    python luce_render_b200/build.py   (the package itself does not load before the library exists)
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
CSRC = PACKAGE / "csrc"
BUILD = ROOT / "_build" / "luce_render_b200"
LIBRARY = PACKAGE / "libluce_render_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "-I", str(ROOT / "include")]
CUDA_FLAGS = ARCH + ["-lineinfo", "--expt-relaxed-constexpr", "-Xptxas", "-v"]
# The integrator's shading divides and takes square roots at the reference's own
# precision (Vulkan's GLSL allows 2.5 ulp for a division and computes sqrt from
# inversesqrt), not as IEEE-exact software sequences. Its traversal kernels live in
# trace.cu, which takes no such flag: -ftz would also flush the denormal results of the
# explicitly rounded intrinsics (__fmul_rn, __fsub_rn, ...) the watertight test decides
# hits with, so the integrator's hits would no longer be the ray queries' and the brute
# force's.
FILE_FLAGS = {"integrator.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"]}


def nvcc() -> str:
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(found).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build luce_render_b200")
    return found


def sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h")))


def _compile(src: Path, obj: Path) -> tuple[Path, str]:
    cmd = [nvcc(), *COMMON, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cu":
        cmd[1:1] = CUDA_FLAGS + FILE_FLAGS.get(src.name, [])
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"compiling {src.name} failed:\n{' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")
    return src, proc.stderr


def build(verbose: bool = False) -> Path:
    """Compiles what changed and links the library; returns its path."""
    BUILD.mkdir(parents=True, exist_ok=True)
    newest_header = max((h.stat().st_mtime for h in headers()), default=0.0)
    jobs = []
    objects = []
    for src in sources():
        obj = BUILD / (src.name + ".o")
        objects.append(obj)
        if not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, newest_header):
            jobs.append((src, obj))
    if jobs:
        workers = min(len(jobs), os.cpu_count() or 4)
        with concurrent.futures.ThreadPoolExecutor(workers) as pool:
            for src, log in pool.map(lambda j: _compile(*j), jobs):
                if verbose and log:
                    print(f"--- {src.name}\n{log}", file=sys.stderr)
    # Link when anything compiled, or an object is newer than the library (compiled by
    # another step since the last link).
    stale = not LIBRARY.exists() or any(o.stat().st_mtime > LIBRARY.stat().st_mtime for o in objects)
    if jobs or stale:
        tmp = LIBRARY.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objects), "-lpthread"]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"linking failed:\n{' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")
        os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
