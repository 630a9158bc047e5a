#!/usr/bin/env python
"""Benchmark of the fused leapfrog step: REAL level, 512^3 lattice, float32.

One "step" is one leapfrog step (GOV-01 + GOV-02 over the 19-point
Laplacian, sponge, clamp) of the whole lattice.  The workload is the
throughput configuration: chi = 19 + U(-1e-3, 1e-3), 64 Gaussian packets
(amplitude U[2,6], sigma U[2,4]) inside the sponge-free sphere, E_prev = E;
synthetic, seeded.  Inputs (4 x 537 MB) are larger than L2, so no flush is
needed between steps.

Prints one JSON line (rank 0).  `value` is device-timed (CUDA events around
K steps on the launching stream, max over ranks) with the state resident in
HBM; `e2e` is the same metric through the public API (Evolver) with the
initial state copied from pinned host memory and the final fields copied
back inside the timed region.  --impl reference times the CPU oracle (the
bit-exact restatement of the reference NumPy path) on the host cores.

Multi-GPU (torchrun), --mode:
  replicas (default)  every rank evolves its own lattice (independent lattices,
                      no collective in the data path): weak scaling;
  slab                one lattice split along i, one slab per rank, the ghost
                      planes exchanged with NCCL point-to-point after every step
                      (overlapped with the interior planes): strong scaling;
  sweep               the batched-sweep lattices shared out over the ranks by cost,
                      one batched launch per step on each, no collective while
                      stepping: strong scaling.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
for _p in (ROOT, ROOT / "lfm-physics_b200"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

BYTES_PER_CELL = {"real": 24}          # algorithmic: read E, E_prev, chi, chi_prev; write E', chi'
METRIC = "GCell-updates/s"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--mode", choices=["replicas", "slab", "sweep"], default="replicas",
                    help="replicas: every rank evolves its own lattice (weak scaling, the "
                         "default); slab: one lattice split along i over the ranks with the "
                         "NCCL ghost exchange (strong scaling); sweep: the batched-sweep "
                         "lattices split over the ranks (strong scaling)")
    ap.add_argument("--N", type=int, default=512)
    ap.add_argument("--cpu-seconds", type=float, default=10.0,
                    help="approximate CPU time of the oracle baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-main", action="store_true",
                    help="skip the main leg (profiling runs of the other legs; no main value)")
    ap.add_argument("--no-compensated", action="store_true")
    ap.add_argument("--no-split", action="store_true", help="skip the split-chi leg")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batch-lattices", type=int, default=256)
    ap.add_argument("--batch-steps", type=int, default=200)
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--level", choices=["real", "complex"], default="real",
                    help="level of the main leg; complex (with the packets as both parts) is a "
                         "secondary workload and turns the e2e, compensated and CPU legs off")
    ap.add_argument("--batch-tuning", default="auto",
                    help="auto (the autotuner), default, or THREADS,STAGES,ITEM_CELLS")
    ap.add_argument("--adjoint-steps", type=int, default=500)
    ap.add_argument("--no-color", action="store_true")
    ap.add_argument("--color-N", type=int, default=256)
    ap.add_argument("--color-steps", type=int, default=100)
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:  # noqa: BLE001
            pass
    return FALLBACK_HBM_GBS, "fallback"


def workload_config(N: int, level: str) -> dict:
    """The workload keys both arms report (the reference arm's line names the same
    workload as this implementation's)."""
    return {"workload": f"{level.upper()} {N}^3 leapfrog step (GOV-01 + GOV-02, 19-point, "
                        "sponge), 64 packets, chi0 = 19 +- 1e-3",
            "N": N, "level": level.upper(), "buffers": "resident",
            "bytes_per_cell": 36 if level == "complex" else BYTES_PER_CELL["real"]}


def profiled_traffic(N: int, level: str = "real"):
    """DRAM bytes per launch of the step kernel from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    try:
        d = json.loads(p.read_text())
        e = d.get(f"{level}_{N}")
        return None if e is None else float(e["dram_bytes_per_launch"])
    except Exception:  # noqa: BLE001
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait(timeout=5)
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1])]
        mx = max((num(r[2]) for r in rows if num(r[2])), default=None)
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v == "Active"})
        sm_sorted = sorted(sm)
        med = sm_sorted[len(sm_sorted) // 2] if sm_sorted else None
        return {"sm_mhz": med, "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


def cpu_baseline(N: int, seconds: float, E, chi) -> dict:
    """The oracle (bit-exact restatement of the reference CPU path), all host threads,
    on slabs of the same lattice until about `seconds` of work."""
    import numpy as np

    from lfm_b200.config import gravity_only
    from lfm_b200.mask import boundary_mask
    from oracle import oracle as O

    threads = os.cpu_count() or 1
    O.set_threads(threads)
    cfg = gravity_only(N)
    n = N**3
    Ef = E.reshape(-1)
    chif = chi.reshape(-1)
    mask = boundary_mask(N, cfg.boundary_fraction)  # same bits as the reference mask
    outs = [np.empty(n, np.float32) for _ in range(4)]
    be = O.OracleBackend()
    planes = min(N, max(threads, 16))
    done_cells = 0
    t0 = time.perf_counter()
    i0 = 0
    while True:
        O.set_plane_range(i0, i0 + planes)
        be.step_real(Ef, Ef, chif, chif, mask, *outs, N, cfg.dt**2, cfg.kappa, cfg.lambda_self,
                     cfg.chi0, cfg.e0_sq)
        done_cells += planes * N * N
        i0 = (i0 + planes) % N
        if time.perf_counter() - t0 >= seconds:
            break
    el = time.perf_counter() - t0
    O.set_plane_range(0, -1)
    return {"value": done_cells / el / 1e9, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"oracle REAL step on {done_cells // (N * N)} planes of the {N}^3 lattice "
                      f"({el:.1f} s, {threads} threads of {os.cpu_count()})"}


def cpu_baseline_numpy(N: int, E, chi) -> dict:
    """The reference's CPU path as its NumPy whole-array operations (one core, as
    NumPy runs them): one REAL step of the whole lattice."""
    from lfm_b200.config import gravity_only
    from lfm_b200.mask import boundary_mask
    from oracle import oracle as O

    cfg = gravity_only(N)
    mask = boundary_mask(N, cfg.boundary_fraction)
    Ef, chif = E.reshape(-1), chi.reshape(-1)
    t0 = time.perf_counter()
    O.numpy_step_real(Ef, Ef, chif, chif, mask, N, cfg.dt**2, cfg.kappa, cfg.lambda_self,
                      cfg.chi0, cfg.e0_sq)
    el = time.perf_counter() - t0
    return {"value": N**3 / el / 1e9, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": f"one REAL step of the whole {N}^3 lattice with the reference's NumPy "
                      f"array operations (oracle.numpy_step_real, bit-exact to the reference; "
                      f"{el:.1f} s, single-threaded NumPy)"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    import numpy as np

    from lfm_b200.config import gravity_only
    from lfm_b200.mask import boundary_mask
    from lfm_b200.workloads import real_solitons
    from oracle import oracle as O

    N = args.N
    E, chi = real_solitons(N)
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    cfg = gravity_only(N)
    n = N**3
    bufs = [E.reshape(-1).copy(), E.reshape(-1).copy(), chi.reshape(-1).copy(),
            chi.reshape(-1).copy()]
    outs = [np.empty(n, np.float32) for _ in range(4)]
    mask = boundary_mask(N, cfg.boundary_fraction)
    be = O.OracleBackend()
    planes = min(N, threads)

    def step(i0):
        O.set_plane_range(i0, i0 + planes)
        be.step_real(*bufs, mask, *outs, N, cfg.dt**2, cfg.kappa, cfg.lambda_self, cfg.chi0,
                     cfg.e0_sq)

    # Each reference "step" is a slab of the lattice, sized from a calibration
    # step so that warm-up plus timed steps take about a minute of host time.
    t0 = time.perf_counter()
    step(0)
    rate = planes * N * N / max(time.perf_counter() - t0, 1e-6)
    budget = 60.0 / max(args.steps + args.warmup, 1)
    planes = int(max(1, min(N, rate * budget // (N * N))))

    for w in range(args.warmup):
        step((w * planes) % N)
    t0 = time.perf_counter()
    for s in range(args.steps):
        step((s * planes) % N)
    el = time.perf_counter() - t0
    O.set_plane_range(0, -1)
    cells = planes * N * N * args.steps
    value = cells / el / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": dict(workload_config(N, "real"), sample_planes_per_step=planes),
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "port",
                         "sample": f"{planes} planes of the {N}^3 lattice per step"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_batched(args, be, dev, rank, barrier, max_over_ranks, peak):
    """Batched sweep: `batch_lattices` lattices (N in {32..96}, REAL/COMPLEX mixed,
    one packet each) in one persistent launch per step, the whole
    step loop replayed as one CUDA graph, against the plain loop of
    single-lattice Evolvers over the same lattices on the same GPU."""
    import torch

    from lfm_b200 import Evolver, _lib
    from lfm_b200.batch import BatchedLattices
    from lfm_b200.workloads import sweep_lattices

    steps = args.batch_steps + (args.batch_steps % 2)
    L = sweep_lattices(args.batch_lattices, seed=5 + 1000 * rank)
    cfgs = [c for c, _, _ in L]
    cells = sum(c.grid_size**3 for c in cfgs)
    bytes_step = sum(c.grid_size**3 * (36 if int(c.field_level) else 24) for c in cfgs)
    stream = torch.cuda.current_stream(dev)

    def load(tgt, i, pr, pi):
        args_ = (i,) if isinstance(tgt, BatchedLattices) else ()
        tgt.set_psi_real(*args_, pr)
        if pi is not None:
            tgt.set_psi_imag(*args_, pi)

    def timed(fn):
        torch.cuda.synchronize(dev)
        barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        return max_over_ranks(a.elapsed_time(b))

    os.environ.setdefault("LFM_B200_TUNE_CACHE", str(Path(tempfile.gettempdir()) /
                                                     "lfm_b200_bench_tune.json"))
    if args.batch_tuning in ("auto", "default"):
        tuning = "auto" if args.batch_tuning == "auto" else None
        fixed = dict(threads=256, stages=5, item_cells=131072)  # the library's default
    else:
        t, s_, c_ = (int(x) for x in args.batch_tuning.split(","))
        tuning = fixed = dict(threads=t, stages=s_, item_cells=c_)
    B = BatchedLattices(cfgs, backend=be, tuning=tuning)
    tune = B.tune_report or {"best": fixed, "ms_per_step": None, "trials": []}
    B.graph_block = steps
    for i, (c, pr, pi) in enumerate(L):
        load(B, i, pr, pi)
    B.evolve(max(args.warmup, 3) | 1)  # odd: leaves the damped state, parity 1
    B.evolve(steps)                    # captures the whole-loop graph of this parity
    B.evolve(steps)                    # ... and of the other
    ms_b = timed(lambda: B.evolve(steps))
    status = _lib.device_status(clear=True)
    if status:
        raise RuntimeError(f"device status word {status} after the batched steps")
    info = B.info()
    del B

    evs = []
    for c, pr, pi in L:
        ev = Evolver(c, backend=be)
        load(ev, 0, pr, pi)
        ev.evolve(max(args.warmup, 3) | 1)
        ev.warm_graphs()
        evs.append(ev)

    def plain():
        for ev in evs:
            ev.evolve(steps)

    ms_p = timed(plain)
    del evs

    # The loop as the reference's sweep runs it (sweep.py:52-82): per value a fresh
    # simulation object, its state set from the host, the steps, the metrics at the end.
    def reference_semantics():
        for c, pr, pi in L:
            ev = Evolver(c, backend=be)
            load(ev, 0, pr, pi)
            ev.evolve(steps)
            ev.metrics()

    ms_r = timed(reference_semantics)
    vb = cells * steps / (ms_b / 1e3) / 1e9
    vp = cells * steps / (ms_p / 1e3) / 1e9
    ach = bytes_step * steps / (ms_b / 1e3) / 1e9
    return {"value": vb, "unit": METRIC, "ms": ms_b, "steps": steps,
            "lattices": len(cfgs), "cells": cells,
            "levels": {"real": sum(1 for c in cfgs if int(c.field_level) == 0),
                       "complex": sum(1 for c in cfgs if int(c.field_level) == 1)},
            "plain_loop": {"value": vp, "unit": METRIC, "ms": ms_p,
                           "how": "one Evolver per lattice, evolve(steps) each in turn "
                                  "(two-step CUDA graphs)"},
            "speedup_vs_plain_loop": ms_p / ms_b,
            "reference_semantics_loop": {
                "value": cells * steps / (ms_r / 1e3) / 1e9, "unit": METRIC, "ms": ms_r,
                "how": "per lattice: a new Evolver, its state from the host, evolve(steps), "
                       "metrics() (the reference sweep's per-value loop, sweep.py:52-82)"},
            "speedup_vs_reference_semantics_loop": ms_r / ms_b,
            "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak, "bytes_per_cell": "24 REAL / 36 COMPLEX"},
            "launch": info, "gpu_launches": steps,
            "autotune": {"best": tune["best"], "ms_per_step": tune["ms_per_step"],
                         "default_ms_per_step": next(
                             (t["ms_per_step"] for t in tune.get("trials", [])
                              if t["tuning"] == dict(threads=256, stages=5, item_cells=131072)),
                             None),
                         "trials": len(tune.get("trials", []))}}


def run_color(args, be, dev, world, barrier, max_over_ranks, peak):
    """COLOR step (full_physics, three complex colours, S_a solved every step) on two
    colour-charged packets 40 cells apart with chi = 19 +- 1e-3, device-timed over
    `color_steps` graph-replayed steps on every rank (its own lattice each).  The fused
    stencil kernel moves 84 B/cell (Psi_a, chi and their previous values in, new values
    out) plus 12 B/cell of S_a read and 12 B/cell of |Psi_a|^2 written for the next
    solve; the S_a solve is a 2-D R2C over (j, k), the fused pass along i (FFT, filter,
    inverse FFT) and a 2-D C2R for power-of-two N.
    The same lattice without the tube coupling (kappa_tube = 0, no S_a) is timed
    beside it to split the step."""
    import torch

    from lfm_b200 import Evolver, _lib
    from lfm_b200.config import full_physics
    from lfm_b200.workloads import color_packets

    N, steps = args.color_N, args.color_steps
    pr, pi, chi = color_packets(N)
    stream = torch.cuda.current_stream(dev)

    def timed(cfg):
        ev = Evolver(cfg, backend=be)
        ev.set_psi_real(pr)
        ev.set_psi_imag(pi)
        ev.set_chi(chi)
        ev.evolve(max(args.warmup, 4))
        ev.warm_graphs()
        torch.cuda.synchronize(dev)
        barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ev.evolve(steps)
        b.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        ms = max_over_ranks(a.elapsed_time(b)) / steps
        del ev
        torch.cuda.empty_cache()
        return ms

    ms = timed(full_physics(N))
    tile = _lib.tune_get(2, N)
    ms_no_sa = timed(full_physics(N, kappa_tube=0.0))
    status = _lib.device_status(clear=True)
    if status:
        raise RuntimeError(f"device status word {status} after the COLOR steps")
    cells = N**3
    stencil = 84 * cells / (ms_no_sa / 1e3) / 1e9  # without the tube coupling: no S_a read
    return {"workload": f"COLOR {N}^3 full_physics, two colour-charged packets 40 cells apart, "
                        "S_a every step",
            "value": world * cells / (ms / 1e3) / 1e9, "unit": METRIC, "ms_per_step": ms,
            "steps": steps, "tile": tile,
            "without_sa": {"ms_per_step": ms_no_sa,
                           "value": world * cells / (ms_no_sa / 1e3) / 1e9,
                           "roofline": {"bound": "hbm", "achieved": stencil, "peak": peak,
                                        "unit": "GB/s", "frac": stencil / peak,
                                        "bytes_per_cell": 84}},
            "sa_ms_per_step": ms - ms_no_sa}


def run_adjoint(args, be, dev, barrier, max_over_ranks):
    """Gradient of |chi_final - chi_target|^2 through `adjoint_steps` COMPLEX 96^3
    steps (gravity_em: lambda = 4/31, eps_w = 0.1) with respect to the
    amplitude, centre and phase of two packets and a per-cell chi offset; the
    target is a forward run from other packet parameters
    (lfm_b200.workloads.adjoint_packets, seed 6).
    Forward = the checkpointed forward pass, backward = recompute + adjoint."""
    import torch

    from lfm_b200 import Evolver
    from lfm_b200.adjoint import leapfrog, memory_bytes, soliton_state
    from lfm_b200.config import gravity_em
    from lfm_b200.workloads import adjoint_packets

    N, steps = 96, args.adjoint_steps
    cfg = gravity_em(N)
    (amp, cen, ph), pert, sigma = adjoint_packets(N)
    params = [t.to(dev).float() for t in (amp, cen, ph)]
    od = cfg.chi0 * cfg.dt  # packets rotating as Simulation.place_soliton starts them
    with torch.no_grad():
        st = soliton_state(N, *[t.to(dev).float() for t in pert], sigma, cfg.chi0, None, True,
                           omega_dt=od)
        target = leapfrog(cfg, st, steps, backend=be)[4].clone()
        st[4] = st[5] = torch.full((N, N, N), cfg.chi0, device=dev, dtype=torch.float64)
        target_split = leapfrog(cfg, st, steps, backend=be, split_chi=True)[4].clone()
    stream = torch.cuda.current_stream(dev)

    def one(timed: bool, split: bool = False):
        p = [t.clone().requires_grad_(True) for t in params]
        dchi = torch.zeros((N, N, N), device=dev, requires_grad=True,
                           dtype=torch.float64 if split else torch.float32)
        st = soliton_state(N, *p, sigma, cfg.chi0, None if split else dchi, True, omega_dt=od)
        if split:  # chi in float64: chi0 + hi + lo in the split-chi steps
            st[4] = st[5] = cfg.chi0 + dchi
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize(dev)
        barrier()
        ev[0].record(stream)
        out = leapfrog(cfg, st, steps, backend=be, split_chi=split)
        ev[1].record(stream)
        loss = ((out[4] - (target_split if split else target)) ** 2).sum()
        loss.backward()
        ev[2].record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        fwd = max_over_ranks(ev[0].elapsed_time(ev[1]))
        bwd = max_over_ranks(ev[1].elapsed_time(ev[2]))
        return fwd, bwd, float(loss.detach()), [float(q.grad.abs().max()) for q in p] + [
            float(dchi.grad.abs().max())]

    one(False)
    torch.cuda.reset_peak_memory_stats(dev)
    base = torch.cuda.memory_allocated(dev)
    fwd, bwd, loss, gmax = one(True)
    peak = torch.cuda.max_memory_allocated(dev) - base
    # the plain forward of the same steps (Evolver, two-step CUDA graphs)
    evp = Evolver(cfg, backend=be)
    evp.set_psi_real(st[0])
    evp.set_psi_imag(st[2])
    evp.evolve(5)
    evp.warm_graphs()
    torch.cuda.synchronize(dev)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    evp.evolve(steps)
    b.record(stream)
    torch.cuda.synchronize(dev)
    plain = max_over_ranks(a.elapsed_time(b))
    mem = memory_bytes(cfg, steps)
    one(False, split=True)
    sfwd, sbwd, sloss, _ = one(True, split=True)
    return {"workload": f"COMPLEX {N}^3 gravity_em, {steps} steps, two packets + per-cell "
                        "chi offset, loss |chi - chi_target|^2",
            "forward_ms": fwd, "backward_ms": bwd, "backward_over_forward": bwd / fwd,
            "backward_over_plain_forward": bwd / plain, "plain_forward_ms": plain,
            "loss": loss, "grad_max": dict(zip(("amplitude", "centre", "phase", "dchi"), gmax)),
            "checkpoints": mem["checkpoints"], "checkpoint_bytes": mem["checkpoint_bytes"],
            "segment_bytes": mem["segment_bytes"], "all_states_bytes": mem["all_states_bytes"],
            "peak_extra_bytes": peak,
            "split_chi": {"how": "leapfrog(split_chi=True): chi as chi0 + hi + lo in the forward "
                                 "and the recomputed segments, chi and the loss in float64",
                          "forward_ms": sfwd, "backward_ms": sbwd,
                          "backward_over_forward": sbwd / sfwd, "loss": sloss,
                          "checkpoint_bytes": memory_bytes(cfg, steps,
                                                           split_chi=True)["checkpoint_bytes"]}}


def run_b200(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    from lfm_b200 import B200Backend, Evolver, _lib
    from lfm_b200.config import gravity_only
    from lfm_b200.workloads import real_solitons

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=dev)
    N = args.N
    E, chi = real_solitons(N, seed_chi=1 + 1000 * rank, seed_solitons=2 + 1000 * rank)
    be = B200Backend(dev)
    complex_level = args.level == "complex"
    if complex_level:
        from lfm_b200.config import gravity_em

        args.no_e2e = args.no_compensated = args.no_split = args.no_cpu_baseline = True
        main_cfg = gravity_em(N)
    else:
        main_cfg = gravity_only(N)
    if not args.no_main:
        ev = Evolver(main_cfg, backend=be)
        ev.set_psi_real(E)
        if complex_level:
            ev.set_psi_imag(0.5 * E)
        ev.set_chi(chi)
        ev.evolve(max(args.warmup, 3))
        ev.warm_graphs()
        torch.cuda.synchronize(dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- device-timed, state resident in HBM -------------------------------
    stream = torch.cuda.current_stream(dev)
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    if not args.no_main:
        ev.evolve(args.steps)
    t_end.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    clock_info = clocks.stop()
    ms = max_over_ranks(t_start.elapsed_time(t_end))
    status = _lib.device_status(clear=True)
    if status:
        raise RuntimeError(f"device status word {status} after the timed steps")
    cells = N**3
    if args.no_main:  # profiling runs of the other legs only: no main figure
        ms = float("nan")
    value = world * cells * args.steps / (ms / 1e3) / 1e9
    ms_per_step = ms / args.steps
    cfg_used = _lib.tune_get(int(main_cfg.field_level), N)

    peak, peak_kind = measured_peaks()
    bpc = 36 if complex_level else BYTES_PER_CELL["real"]
    bytes_per_launch = bpc * cells
    achieved = bytes_per_launch / (ms_per_step / 1e3) / 1e9

    # ---- compensated float32 variant (Delta form, 32 B/cell) ---------------
    comp = None
    if not args.no_compensated:
        from lfm_b200.compensated import CompensatedEvolver

        evc = CompensatedEvolver(gravity_only(N), backend=be)
        evc.set_psi_real(E)
        evc.set_chi(chi)
        evc.evolve(max(args.warmup, 4))
        evc.warm_graphs()
        torch.cuda.synchronize(dev)
        barrier()
        ca = torch.cuda.Event(enable_timing=True)
        cb = torch.cuda.Event(enable_timing=True)
        ca.record(stream)
        evc.evolve(args.steps)
        cb.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        cms = max_over_ranks(ca.elapsed_time(cb)) / args.steps
        cach = 32 * cells / (cms / 1e3) / 1e9
        comp = {"value": world * cells / (cms / 1e3) / 1e9, "unit": METRIC, "ms_per_step": cms,
                "bytes_per_cell": 32,
                "roofline": {"bound": "hbm", "achieved": cach, "peak": peak, "unit": "GB/s",
                             "frac": cach / peak, "frac_at_24B": 24 * cells / (cms / 1e3) / 1e9 / peak},
                "tile": _lib.tune_get(0, N)}
        del evc

    # ---- split chi (chi0 + hi + lo, float64 chi arithmetic, 36 B/cell) ----
    split = None
    if not args.no_split:
        from lfm_b200.split import SplitChiEvolver

        evs = SplitChiEvolver(gravity_only(N), backend=be)
        evs.set_psi_real(E)
        evs.set_chi(chi)
        evs.evolve(max(args.warmup, 4))
        evs.warm_graphs()
        torch.cuda.synchronize(dev)
        barrier()
        sa_ = torch.cuda.Event(enable_timing=True)
        sb_ = torch.cuda.Event(enable_timing=True)
        sa_.record(stream)
        evs.evolve(args.steps)
        sb_.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        sms = max_over_ranks(sa_.elapsed_time(sb_)) / args.steps
        sach = 36 * cells / (sms / 1e3) / 1e9
        split = {"value": world * cells / (sms / 1e3) / 1e9, "unit": METRIC, "ms_per_step": sms,
                 "bytes_per_cell": 36,
                 "roofline": {"bound": "hbm", "achieved": sach, "peak": peak, "unit": "GB/s",
                              "frac": sach / peak},
                 "accuracy": "max-relative vs float64 after 1000 steps of the 64^3 REAL "
                             "workload: see profiles/accuracy.json (split_f32)"}
        del evs

    color = None
    if not args.no_color:
        color = run_color(args, be, dev, world, barrier, max_over_ranks, peak)

    adjoint = None
    if not args.no_adjoint:
        adjoint = run_adjoint(args, be, dev, barrier, max_over_ranks)

    batched = None
    if not args.no_batched:
        batched = run_batched(args, be, dev, rank, barrier, max_over_ranks, peak)

    # ---- end to end through the public API ---------------------------------
    e2e = None
    if not args.no_e2e:
        E_h = torch.from_numpy(E).pin_memory()
        chi_h = torch.from_numpy(chi).pin_memory()
        chi_out = torch.empty_like(chi_h).pin_memory()
        E_out = torch.empty_like(E_h).pin_memory()
        ev2 = Evolver(gravity_only(N), backend=be)
        ev2.set_psi_real(E_h)
        ev2.set_chi(chi_h)
        ev2.evolve(4)
        ev2.warm_graphs()  # capture both step graphs outside the timed region
        torch.cuda.synchronize(dev)
        barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ev2.set_psi_real(E_h)
        ev2.set_chi(chi_h)
        ev2.evolve(args.steps)
        ev2.get_chi(out=chi_out)
        ev2.get_psi_real(out=E_out)
        b.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        ms2 = max_over_ranks(a.elapsed_time(b))
        h2d = E_h.numel() * 4 + chi_h.numel() * 4
        d2h = chi_out.numel() * 4 + E_out.numel() * 4
        e2e = {"value": world * cells * args.steps / (ms2 / 1e3) / 1e9, "unit": METRIC,
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
               "job": f"set_psi_real + set_chi from pinned host, evolve({args.steps}), "
                      "get_chi + get_psi_real to pinned host",
               "ms": ms2}
        if not np.isfinite(chi_out.numpy()).all():
            raise RuntimeError("non-finite chi after the end-to-end run")
        del ev2

    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": dict(workload_config(N, args.level), **{
                   "l2": f"inputs {4 * bpc // 6 * cells / 1e9:.2f} GB"
                         + (" > L2, no flush" if 4 * bpc // 6 * cells > 126e6 else
                            " (within L2: profiling size only)"),
                   "parallelism": f"independent lattices x{world}", "tile": cfg_used}),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": profiled_traffic(N, args.level),
                     "algorithmic_bytes_per_launch": bytes_per_launch},
        "clocks": clock_info,
        "gpu_launches": args.steps,
    }
    if e2e is not None:
        line["e2e"] = e2e
    if comp is not None:
        line["compensated"] = comp
    if split is not None:
        line["split_chi"] = split
    if batched is not None:
        line["batched"] = batched
    if adjoint is not None:
        line["adjoint"] = adjoint
    if color is not None:
        line["color"] = color
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(N, args.cpu_seconds, E, chi)
        line["cpu_baseline_numpy"] = cpu_baseline_numpy(N, E, chi)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def _dist_setup():
    import torch
    import torch.distributed as dist

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    return rank, world, dev, barrier, max_over_ranks


def _common_line(args, value, ms, world, config, scaling, clock_info, launches):
    return {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": scaling, "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": config, "clocks": clock_info,
            "gpu_launches": launches}


def run_slab(args):
    """One REAL N^3 lattice split along i over the ranks (SlabEvolver)."""
    import torch
    import torch.distributed as dist

    from lfm_b200 import B200Backend, _lib
    from lfm_b200.config import gravity_only
    from lfm_b200.slab import SlabEvolver
    from lfm_b200.workloads import real_solitons

    rank, world, dev, barrier, max_over_ranks = _dist_setup()
    N = args.N
    E, chi = real_solitons(N)
    s = SlabEvolver(gravity_only(N), backend=B200Backend(dev))
    s.set_psi_real(E)
    s.set_chi(chi)
    s.evolve(max(args.warmup, 3))
    torch.cuda.synchronize(dev)
    stream = torch.cuda.current_stream(dev)
    clocks = ClockSampler(int(dev.index))
    barrier()
    clocks.start()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    s.evolve(args.steps)
    b.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    clock_info = clocks.stop()
    ms = max_over_ranks(a.elapsed_time(b))
    status = _lib.device_status(clear=True)
    if status:
        raise RuntimeError(f"device status word {status} after the slab steps")
    overlapped = world > 1 and s.n_local >= 3
    cfg = dict(workload_config(N, "real"), parallelism=f"slab x{world} along i",
               planes_per_rank=s.n_local, overlap=overlapped,
               exchange_bytes_per_rank_step=0 if world == 1 else 2 * 2 * N * N * 4,
               l2="inputs > L2, no flush")
    line = _common_line(args, N**3 * args.steps / (ms / 1e3) / 1e9, ms, world, cfg, "strong",
                        clock_info, args.steps * (3 if overlapped else 1))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_sweep_sharded(args):
    """The batched-sweep lattices shared out over the ranks by cost (lfm_b200.sweep.shard);
    each rank advances its share in one batched launch per step."""
    import torch
    import torch.distributed as dist

    from lfm_b200 import B200Backend, _lib
    from lfm_b200.batch import BatchedLattices
    from lfm_b200.sweep import shard
    from lfm_b200.workloads import sweep_lattices

    rank, world, dev, barrier, max_over_ranks = _dist_setup()
    L = sweep_lattices(args.batch_lattices, seed=5)
    parts = shard([c.grid_size**3 for c, _, _ in L], world)
    mine = [L[i] for i in parts[rank]]
    steps = args.steps + (args.steps % 2)
    B = BatchedLattices([c for c, _, _ in mine], backend=B200Backend(dev))
    B.graph_block = steps
    for i, (c, pr, pi) in enumerate(mine):
        B.set_psi_real(i, pr)
        if pi is not None:
            B.set_psi_imag(i, pi)
    B.evolve(max(args.warmup, 3) | 1)
    B.evolve(steps)
    B.evolve(steps)
    torch.cuda.synchronize(dev)
    stream = torch.cuda.current_stream(dev)
    clocks = ClockSampler(int(dev.index))
    barrier()
    clocks.start()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    B.evolve(steps)
    b.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    clock_info = clocks.stop()
    ms = max_over_ranks(a.elapsed_time(b))
    status = _lib.device_status(clear=True)
    if status:
        raise RuntimeError(f"device status word {status} after the sharded sweep")
    cells = sum(c.grid_size**3 for c, _, _ in L)
    cfg = {"workload": f"batched sweep: {len(L)} lattices, N in {{32..96}}, REAL/COMPLEX mixed",
           "lattices": len(L), "cells": cells, "parallelism": f"lattices sharded x{world}",
           "lattices_this_rank0": len(parts[0]), "l2": "every lattice stepped once per step"}
    line = _common_line(args, cells * steps / (ms / 1e3) / 1e9, ms, world, cfg, "strong",
                        clock_info, steps)
    line["steps"] = steps
    del B
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.mode == "slab":
        return run_slab(args)
    if args.mode == "sweep":
        return run_sweep_sharded(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
