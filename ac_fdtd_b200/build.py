"""Build the CUDA library in-tree: ``python -m ac_fdtd_b200.build``.

One shared object, ``libacfdtd_b200.so``, compiled by nvcc for sm_100a only. ``-fmad=false``
keeps every multiply and add separately rounded, which is what lets the sweeps reproduce the
NumPy reference bit for bit (the reference's C backend uses ``-ffp-contract=off`` for the same
reason, ac-fdtd ``src/ac_fdtd/c_backend.py:15-18,41``).
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
SOURCES = [PACKAGE / "csrc" / "acfdtd_b200.cu"]
TARGET = PACKAGE / "libacfdtd_b200.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC", "-shared",
    "-I", str(ROOT / "include"),
]


def nvcc() -> str:
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(found).exists():
        raise RuntimeError("nvcc not found; the CUDA library cannot be built")
    return found


def needs_build(target: Path = TARGET) -> bool:
    if not target.exists():
        return True
    newest = max(p.stat().st_mtime for p in SOURCES + [ROOT / "include" / "acfdtd_b200.h"])
    return target.stat().st_mtime < newest


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build():
        return TARGET
    tmp = TARGET.with_suffix(f".tmp{os.getpid()}.so")
    command = [nvcc(), *NVCC_FLAGS, *map(str, SOURCES), "-o", str(tmp)]
    if verbose:
        command.insert(1, "-Xptxas=-v")
    result = subprocess.run(command, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"nvcc failed:\n{' '.join(command)}\n{result.stdout}\n{result.stderr}")
    if verbose:
        sys.stderr.write(result.stderr)
    tmp.replace(TARGET)
    return TARGET


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
