"""Build liblfm_b200.so from csrc/ with nvcc for sm_100a (in-tree).

``python -m lfm_b200.build`` (from the ``lfm-physics_b200`` folder) or
``lfm_b200.build.build_library()`` compiles every ``csrc/*.cu`` into
``lfm_b200/_native/liblfm_b200.so``.  The library links cuFFT dynamically
and finds it through an rpath to the CUDA toolkit and to the copy bundled
with PyTorch, whichever the process loaded first.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
SRC_ROOT = PKG.parent
CSRC = SRC_ROOT / "csrc"
INCLUDE = SRC_ROOT.parent / "include"
LIB_DIR = PKG / "_native"
LIB_PATH = LIB_DIR / "liblfm_b200.so"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: set NVCC or put the CUDA toolkit on PATH")


def _rpaths() -> list[str]:
    paths = ["/usr/local/cuda/lib64"]
    try:
        import importlib.util

        spec = importlib.util.find_spec("nvidia.cufft")
        if spec and spec.submodule_search_locations:
            paths.insert(0, str(Path(list(spec.submodule_search_locations)[0]) / "lib"))
    except Exception:  # noqa: BLE001 - optional
        pass
    return paths


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale() -> bool:
    if not LIB_PATH.exists():
        return True
    t = LIB_PATH.stat().st_mtime
    deps = list(CSRC.glob("*")) + list(INCLUDE.glob("*.h"))
    return any(p.stat().st_mtime > t for p in deps)


def build_library(force: bool = False, verbose: bool = False) -> Path:
    """Compile the CUDA library if it is missing or older than its sources."""
    if not force and not _stale():
        return LIB_PATH
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    objs = []
    build_dir = LIB_DIR / "obj"
    build_dir.mkdir(exist_ok=True)
    common = [
        _nvcc(), *ARCH_FLAGS, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
        f"-I{INCLUDE}", f"-I{CSRC}",
    ]
    if verbose:
        common.append("-Xptxas=-v")
    procs = []
    for src in sources():
        obj = build_dir / (src.stem + ".o")
        objs.append(obj)
        procs.append((src, subprocess.Popen(common + ["-c", str(src), "-o", str(obj)],
                                            stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if verbose or p.returncode:
            sys.stderr.write(out.decode(errors="replace"))
        if p.returncode:
            failed.append(src.name)
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    tmp = LIB_PATH.with_suffix(".so.tmp")
    link = [_nvcc(), *ARCH_FLAGS, "-shared", "-o", str(tmp), *map(str, objs), "-lcufft",
            "-L/usr/local/cuda/lib64"]
    for rp in _rpaths():
        link += ["-Xlinker", f"-rpath={rp}"]
    subprocess.check_call(link)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build_library(force="--force" in sys.argv, verbose="-v" in sys.argv))
