"""Build recipe for the in-tree CUDA library ``pyticc_b200/_lib/libticc_b200.so``.

One translation unit (``csrc/capi.cu`` includes every kernel header) compiled for
sm_100a only, with static cudart so the library has no runtime-version coupling to
the Python process.
"""

from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parent
SOURCE = ROOT / "csrc" / "capi.cu"
OUTPUT = ROOT / "_lib" / "libticc_b200.so"
NVCC_FLAGS = [
    "-gencode",
    "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-O3",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC",
    "-shared",
]


def sources() -> list[Path]:
    return sorted((ROOT / "csrc").glob("*.cu*")) + [ROOT.parent / "include" / "ticc_b200.h"]


def is_stale() -> bool:
    if not OUTPUT.exists():
        return True
    built = OUTPUT.stat().st_mtime
    return any(path.stat().st_mtime > built for path in sources())


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the library if any source is newer than it (or when forced)."""
    if not force and not is_stale():
        return OUTPUT
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    OUTPUT.parent.mkdir(parents=True, exist_ok=True)
    command = [nvcc, *NVCC_FLAGS, "-o", str(OUTPUT), str(SOURCE)]
    if verbose:
        command.insert(1, "-Xptxas=-v")
    result = subprocess.run(command, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"nvcc failed ({result.returncode}):\n{result.stderr}")
    if verbose:
        print(result.stderr)
    return OUTPUT


if __name__ == "__main__":
    print(build(force=True, verbose=True))
