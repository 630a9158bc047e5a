"""Builds the reference's own CUDA step kernels into oracle/_ref/libref_gpu.so.

TEST INFRASTRUCTURE ONLY.  The reference's GPU backend compiles three kernel
sources held as Python strings (lfm/core/backends/kernel_source.py:
EVOLUTION_REAL_KERNEL_SRC, EVOLUTION_COMPLEX_KERNEL_SRC, EVOLUTION_KERNEL_SRC)
with CuPy's RawKernel.  This recipe reads those strings from the reference
checkout, writes them to oracle/_ref/ref_kernels.cu, and compiles them with
ref_gpu_launch.cu (the launchers) for sm_100a with nvcc's defaults, as NVRTC
compiles them for CuPy (FMA contraction on, no fast math).  oracle/_ref/ is
not committed; it travels with the working tree to the GPU machine.

    python oracle/build_ref_gpu.py REFERENCE_ROOT

The checkout comes from the argument or, without one, from the
LFM_REFERENCE_ROOT environment variable.  Without a checkout it does nothing
and says so.
"""

from __future__ import annotations

import importlib.util
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
LIB = OUT / "libref_gpu.so"
NAMES = ("EVOLUTION_REAL_KERNEL_SRC", "EVOLUTION_COMPLEX_KERNEL_SRC", "EVOLUTION_KERNEL_SRC")


def _kernel_sources(ref_root: Path) -> str:
    src = ref_root / "lfm" / "core" / "backends" / "kernel_source.py"
    spec = importlib.util.spec_from_file_location("_lfm_reference_kernel_source", src)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    parts = [f"// {n}, from lfm/core/backends/kernel_source.py\n{getattr(mod, n)}" for n in NAMES]
    return "\n".join(parts)


def build(ref_root: Path | None = None, force: bool = False) -> Path | None:
    ref_root = ref_root or os.environ.get("LFM_REFERENCE_ROOT")
    launcher = HERE / "ref_gpu_launch.cu"
    if not ref_root:
        print("no reference checkout given (argument or LFM_REFERENCE_ROOT): "
              "reference GPU kernels not built")
        return LIB if LIB.exists() else None
    ref_root = Path(ref_root)
    if not (ref_root / "lfm" / "core" / "backends" / "kernel_source.py").exists():
        print(f"reference checkout not found at {ref_root}: reference GPU kernels not built")
        return LIB if LIB.exists() else None
    OUT.mkdir(exist_ok=True)
    kernels = OUT / "ref_kernels.cu"
    text = _kernel_sources(ref_root)
    if not force and LIB.exists() and kernels.exists() and kernels.read_text() == text and (
            LIB.stat().st_mtime >= launcher.stat().st_mtime):
        return LIB
    kernels.write_text(text)
    nvcc = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.check_call([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3",
                           "-std=c++17", "-Xcompiler", "-fPIC", "-shared", f"-I{OUT}",
                           str(launcher), "-o", str(tmp)])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(Path(sys.argv[1]) if len(sys.argv) > 1 else None, force=True))
