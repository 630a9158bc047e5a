"""Autotuner for the batched and the single-lattice fused step kernels.

Every tile shape computes the same bits (the march order inside a tile does
not change any cell's arithmetic), so tuning is purely a timing search:

* ``tune_batch`` -- block size cap, shared-memory stages, cells per work item
  and CTAs per SM of a :class:`~lfm_b200.batch.BatchedLattices`;
* ``tune_lattice`` -- vector width, rows per tile, stages and plane chunk of
  the fused kernel for one (level, N) (lfm_tune_set).

Each candidate is timed with CUDA events over a few steps after a warm-up
step, on the state the object holds (restored afterwards).  Winners are
cached in a JSON file (``LFM_B200_TUNE_CACHE`` or ``_native/tune_cache.json``
beside the library) keyed by device name and workload signature, so a later
run with the same lattices skips the search.
"""

from __future__ import annotations

import itertools
import json
import os
from pathlib import Path

from . import _lib
from .build import LIB_DIR


def cache_path() -> Path:
    return Path(os.environ.get("LFM_B200_TUNE_CACHE", LIB_DIR / "tune_cache.json"))


def _load_cache() -> dict:
    p = cache_path()
    try:
        return json.loads(p.read_text())
    except (OSError, ValueError):
        return {}


def _store(key: str, value) -> None:
    p = cache_path()
    data = _load_cache()
    data[key] = value
    try:
        p.parent.mkdir(parents=True, exist_ok=True)
        tmp = p.with_suffix(f".{os.getpid()}.tmp")  # ranks on one host may store at once
        tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
        tmp.replace(p)
    except OSError:
        pass  # a read-only install still tunes, it only forgets


def _device_name(device) -> str:
    import torch

    return torch.cuda.get_device_name(device)


def _time_ms(device, fn, steps: int) -> float:
    import torch

    fn(1)  # warm-up (and any lazy set-up)
    torch.cuda.synchronize(device)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    fn(steps)
    b.record()
    torch.cuda.synchronize(device)
    return a.elapsed_time(b) / steps


def _time_graph_ms(evolver, steps: int) -> float:
    """Device time per step of `steps` (even) resident steps replayed as one
    CUDA graph, so that host launch overhead does not hide small lattices'
    kernel time."""
    import torch

    steps += steps % 2
    evolver._step()  # first launch of this tile outside capture (and prev damped)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for _ in range(steps):
            evolver._step()
    g.replay()
    torch.cuda.synchronize(evolver.device)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    g.replay()
    b.record()
    torch.cuda.synchronize(evolver.device)
    return a.elapsed_time(b) / steps


# ------------------------------------------------------------------ batches
BATCH_CANDIDATES = [
    dict(threads=t, stages=s, item_cells=c)
    for t, s, c in itertools.product((128, 256, 512), (3, 4, 5), (16384, 32768, 65536, 131072))
]


def batch_signature(configs) -> str:
    """(N, level) histogram of a batch: the tile plan depends on nothing else."""
    hist: dict[tuple, int] = {}
    for c in configs:
        k = (int(c.grid_size), int(c.field_level))
        hist[k] = hist.get(k, 0) + 1
    return "batch:" + ",".join(f"{n}{'rc'[lv]}{cnt}" for (n, lv), cnt in sorted(hist.items()))


def tune_batch(batch, candidates=None, steps: int = 6, use_cache: bool = True) -> dict:
    """Pick the fastest tuning for `batch` and apply it; returns {"best", "trials"}."""
    key = f"{_device_name(batch.device)}|{batch_signature(batch.configs)}"
    if use_cache and candidates is None:
        hit = _load_cache().get(key)
        if hit is not None:
            batch.retune(hit["best"])
            return hit
    saved = batch._arena.clone()
    saved_state = (batch._cur, batch._damp, batch.step)
    trials = []
    try:
        for cand in candidates or BATCH_CANDIDATES:
            try:
                batch.retune(cand)
            except _lib.LfmError:
                continue  # e.g. more shared memory than a CTA may have
            ms = _time_ms(batch.device, lambda k: batch.evolve(k, use_graph=False), steps)
            trials.append({"tuning": dict(cand), "ms_per_step": ms})
    finally:
        batch._arena.copy_(saved)
        batch._cur, batch._damp, batch.step = saved_state
    if not trials:
        raise RuntimeError("no batch tuning candidate could be launched")
    best = min(trials, key=lambda t: t["ms_per_step"])
    batch.retune(best["tuning"])
    out = {"best": best["tuning"], "ms_per_step": best["ms_per_step"], "trials": trials}
    if candidates is None:
        _store(key, out)
    return out


# ------------------------------------------------------------------ one lattice
def lattice_candidates(level: int):
    """Vector width x rows per tile x stages x plane chunk (0 = the planner's
    wave-balanced chunk).  Small lattices are latency-bound: deep rings and
    short chunks (many CTAs, few planes each) pay there."""
    vecs = {0: (4, 2), 1: (2,), 2: (2, 1)}[level]
    return [dict(vec=v, tj=tj, stages=s, ic=ic)
            for v, tj, s, ic in itertools.product(vecs, (1, 2, 4, 8), (3, 4, 6),
                                                  (0, 4, 8, 16, 32, 64))]


def tune_lattice(evolver, candidates=None, steps: int = 20, use_cache: bool = True) -> dict:
    """Pick the fused kernel's tile for the evolver's (level, N) and pin it (lfm_tune_set)."""
    level, N = int(evolver._level), int(evolver.N)
    key = f"{_device_name(evolver.device)}|lattice:{level}:{N}"
    if use_cache and candidates is None:
        hit = _load_cache().get(key)
        if hit is not None:
            b = hit["best"]
            _lib.tune_set(level, N, b["tj"], b["stages"], b["ic"], b["vec"])
            return hit
    if evolver._mode != "resident":
        raise ValueError("tune_lattice needs an Evolver with buffers='resident'")
    slots = [t for t in (*evolver._pr, *evolver._chi,
                         *(evolver._pi if evolver._has_imag else ())) if t is not None]
    saved = [t.clone() for t in slots]
    saved_state = (evolver._cur, evolver._damp, evolver.step, evolver._use_buffer_A)
    prev_path = None
    trials = []
    _lib.set_step_path(_lib.PATH_FUSED)
    try:
        for cand in candidates or lattice_candidates(level):
            _lib.tune_set(level, N, cand["tj"], cand["stages"], cand["ic"], cand["vec"])
            evolver._graphs = {}
            try:
                ms = _time_graph_ms(evolver, steps)
            except _lib.LfmError:
                continue  # tile does not fit this N
            used = _lib.tune_get(level, N)
            trials.append({"tile": used, "ms_per_step": ms})
    finally:
        _lib.set_step_path(_lib.PATH_AUTO if prev_path is None else prev_path)
        for t, s in zip(slots, saved):
            t.copy_(s)
        evolver._cur, evolver._damp, evolver.step, evolver._use_buffer_A = saved_state
        evolver._graphs = {}
    if not trials:
        _lib.tune_set(level, N, 0, 0, 0, 0)
        raise RuntimeError(f"no fused tile fits level {level} N={N}")
    best = min(trials, key=lambda t: t["ms_per_step"])
    b = best["tile"]
    _lib.tune_set(level, N, b["tj"], b["stages"], b["ic"], b["vec"])
    out = {"best": {k: b[k] for k in ("vec", "tj", "stages", "ic")},
           "ms_per_step": best["ms_per_step"], "trials": trials}
    if candidates is None:
        _store(key, out)
    return out
