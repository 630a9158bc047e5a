"""bench.py's multi-GPU modes at world size 1 (one GPU): one lattice as slabs
(--mode slab) and the sharded batched sweep (--mode sweep) run and print a
well-formed line.  On N GPUs (torchrun) the same code runs one slab / one share
of the lattices per rank."""

from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]

pytestmark = pytest.mark.gpu


def _run(*args) -> dict:
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], cwd=ROOT,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "ms_per_step", "scaling", "config",
              "clocks", "gpu_launches"):
        assert k in line, k
    assert line["value"] > 0 and line["n_gpus"] == 1
    return line


def test_slab_mode_runs_one_lattice_as_slabs(cuda_device):
    line = _run("--mode", "slab", "--N", "128", "--steps", "6", "--warmup", "3")
    assert line["scaling"] == "strong"
    assert line["config"]["planes_per_rank"] == 128


def test_sweep_mode_runs_the_sharded_sweep(cuda_device):
    line = _run("--mode", "sweep", "--batch-lattices", "24", "--steps", "6", "--warmup", "3")
    assert line["scaling"] == "strong" and line["config"]["lattices"] == 24
