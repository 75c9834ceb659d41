"""Compile libinterax_b200.so (the sm_100a kernels and their C ABI) with nvcc.

The tile and schedule constants (ix_tuning.h's IX_TUNE_* macros) come from tuning.json beside this file, written by
the autotuner (tune.py); compile_library() also takes explicit values, which is how the tuner builds its candidates.
"""
import json
import os
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "libinterax_b200.so"
TUNING = PKG / "tuning.json"
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-O2", "-diag-suppress", "177"]


def tuned_values():
    """The autotuner's chosen IX_TUNE_* values ({} when there is no tuning file)."""
    if not TUNING.exists():
        return {}
    return dict(json.loads(TUNING.read_text())["chosen"])


def _define(name, value):
    if isinstance(value, float):
        return f"-D{name}={value!r}f"
    return f"-D{name}={int(value)}"


def compile_command(out, values=None):
    values = tuned_values() if values is None else values
    nvcc = os.environ.get("NVCC", "nvcc")
    return [nvcc, *NVCC_FLAGS, *[_define(k, v) for k, v in sorted(values.items())], "-shared", "-o", str(out),
            str(CSRC / "ix_context.cu")]


def compile_library(out=LIB, values=None):
    subprocess.run(compile_command(out, values), check=True)


def sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + \
        ([TUNING] if TUNING.exists() else [])


def build():
    """Compile the library in place when it is missing or older than a source or the tuning file."""
    if not LIB.exists() or any(s.stat().st_mtime > LIB.stat().st_mtime for s in sources()):
        compile_library(LIB)
