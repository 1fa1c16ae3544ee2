"""Build libthermal_b200.so in-tree with nvcc for sm_100a.

    python -m pcb_analysis_b200.build [--force]

The library is written next to this file so that it travels with the source
tree; the Python facade loads it from there and fails loudly when it is
missing.
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
REPO_DIR = PACKAGE_DIR.parent
CSRC = PACKAGE_DIR / "csrc"
LIBRARY = PACKAGE_DIR / "libthermal_b200.so"
HEADER = REPO_DIR / "include" / "thermal_b200.h"
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for candidate in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if candidate and Path(candidate).exists():
            return candidate
    raise RuntimeError("nvcc not found; set NVCC or put the CUDA toolkit on PATH")


def sources() -> list[Path]:
    return (sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.inl")) + sorted(CSRC.glob("*.h"))
            + [HEADER])


def needs_build() -> bool:
    if not LIBRARY.exists():
        return True
    built = LIBRARY.stat().st_mtime
    return any(path.stat().st_mtime > built for path in sources())


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the library unless it is newer than every source file."""

    if not force and not needs_build():
        return LIBRARY
    cmd = [
        _nvcc(),
        *ARCH_FLAGS,
        "-lineinfo",
        "-O3",
        "-std=c++17",
        "-Xcompiler",
        "-fPIC,-O3",
        "-shared",
        "-o",
        str(LIBRARY),
        str(CSRC / "tb_system.cu"),
    ]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    tmp = LIBRARY.with_suffix(".so.tmp")
    cmd[cmd.index(str(LIBRARY))] = str(tmp)
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"nvcc failed ({result.returncode}):\n{' '.join(cmd)}\n{result.stdout}\n{result.stderr}")
    if verbose:
        sys.stderr.write(result.stderr)
    os.replace(tmp, LIBRARY)
    return LIBRARY


def main() -> None:
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("--force", action="store_true")
    parser.add_argument("--verbose", action="store_true")
    args = parser.parse_args()
    print(build(force=args.force, verbose=args.verbose))


if __name__ == "__main__":
    main()
