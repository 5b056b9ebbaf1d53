"""Build liblaker_b200.so (sm_100a) in-tree with nvcc.

The library is a plain C ABI over the CUDA runtime (no torch symbols), so it
is compiled with one nvcc invocation instead of a torch extension build.  The
shared object lands next to this file so that it travels with the source tree.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
CSRC = PKG_DIR / "csrc"
INCLUDE = PKG_DIR.parent / "include"
LIB_NAME = "liblaker_b200.so"
LIB_PATH = PKG_DIR / LIB_NAME

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    """Return the nvcc executable (CUDA_HOME or /usr/local/cuda or PATH)."""
    for cand in (
        os.environ.get("CUDA_HOME", ""),
        "/usr/local/cuda",
    ):
        if cand:
            p = Path(cand) / "bin" / "nvcc"
            if p.exists():
                return str(p)
    found = shutil.which("nvcc")
    if not found:
        raise RuntimeError("nvcc not found: set CUDA_HOME or put nvcc on PATH")
    return found


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale() -> bool:
    if not LIB_PATH.exists():
        return True
    lib_mtime = LIB_PATH.stat().st_mtime
    deps = sources() + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h")) + [Path(__file__)]
    return any(p.stat().st_mtime > lib_mtime for p in deps)


def _compile_flags() -> list[str]:
    return [*ARCH_FLAGS, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
            "-Xcompiler", "-fPIC", f"-I{INCLUDE}"]


def _run(cmd: list[str], verbose: bool) -> subprocess.CompletedProcess:
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed ({proc.returncode}):\n{proc.stdout}\n{proc.stderr}")
    if verbose and (proc.stdout or proc.stderr):
        print(proc.stdout, proc.stderr, file=sys.stderr)
    return proc


def build(force: bool = False, verbose: bool = False, extra_flags: list[str] | None = None) -> Path:
    """Compile every CUDA source of the package into liblaker_b200.so.

    Each translation unit is compiled to an object file in parallel (no
    relocatable device code: every unit carries its own kernels), then the
    objects are linked into the shared library.
    """
    if not force and not _stale():
        return LIB_PATH
    flags = list(extra_flags or []) + _compile_flags()
    objdir = PKG_DIR / "_build"
    objdir.mkdir(exist_ok=True)
    nvcc = nvcc_path()
    jobs = []
    for src in sources():
        obj = objdir / (src.stem + ".o")
        jobs.append((obj, [nvcc, *flags, "-c", "-o", str(obj), str(src)]))
    workers = max(1, min(len(jobs), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=workers) as pool:
        for fut in [pool.submit(_run, cmd, verbose) for _, cmd in jobs]:
            fut.result()
    tmp = LIB_PATH.with_suffix(".so.tmp")
    _run([nvcc, *ARCH_FLAGS, "-shared", "-o", str(tmp), *[str(o) for o, _ in jobs]], verbose)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    flags = [a for a in sys.argv[1:] if a.startswith("-")]
    print(build(force=True, verbose=True, extra_flags=flags))
