"""Parameter sweeps (lfm/sweep.py:14-157) on the batched lattice kernel.

``sweep`` / ``sweep_2d`` take the reference's arguments and return its rows
(``{param: value, **metrics}``).  The reference builds one ``Simulation`` per
value and runs them one after another; here every run's initial state is
built on the device (packet placement, Poisson equilibration with
lfm_poisson_chi_f32), all REAL / COMPLEX lattices with N a multiple of 4 are
stepped together by :class:`~lfm_b200.batch.BatchedLattices` (one launch per
step for the whole sweep) and the rest by one :class:`~lfm_b200.Evolver`
each.  Per run, the reference's ``Simulation`` semantics are kept:

* ``soliton`` kwargs go to ``place_soliton`` (position defaults to the
  centre, amplitude / sigma to the config's ``e_amplitude`` / ``sigma``;
  lfm/simulation.py:495-625), the packet is added to every colour;
* the run equilibrates chi when asked to or when a packet was placed (the
  auto-equilibration of ``Simulation.run``, lfm/simulation.py:965-982);
* metrics are ``compute_metrics`` of the final state against the Psi
  snapshot ``run`` keeps (taken at the start and every ``report_interval``
  steps, lfm/simulation.py:1160-1184).

Under ``torch.distributed`` the runs are shared out across the ranks (each
rank takes a contiguous group balanced by N^3, no collective while
stepping) and the rows are gathered at the end, so every rank returns the
full list.
"""

from __future__ import annotations

import itertools
from copy import deepcopy
from typing import Any

import numpy as np

from .config import BoundaryType, FieldLevel

METRIC_KEYS = ("energy_kinetic", "energy_gradient", "energy_potential", "energy_total",
               "chi_min", "chi_max", "chi_mean", "chi_std", "well_fraction", "void_fraction",
               "n_clusters", "psi_sq_total")


def gaussian_soliton(N: int, position, amplitude: float, sigma: float, phase: float = 0.0):
    """amplitude exp(-r^2 / (2 sigma^2)) e^{i phase} on an N^3 grid, float32 as
    lfm/fields/soliton.py:49-59 evaluates it.  Returns (psi_r, psi_i)."""
    x = np.arange(N, dtype=np.float32)
    px, py, pz = position
    r2 = ((x - px) ** 2)[:, None, None] + ((x - py) ** 2)[None, :, None] \
        + ((x - pz) ** 2)[None, None, :]
    env = amplitude * np.exp(-r2 / (2.0 * sigma**2))
    return (env * np.cos(phase)).astype(np.float32), (env * np.sin(phase)).astype(np.float32)


def equilibrate_chi(backend, config, psi_r, psi_i=None, out=None):
    """chi from the Poisson equilibration of device fields (lfm_poisson_chi_f32).

    psi_r / psi_i: float32 device tensors, (N, N, N) or (3, N, N, N) at the
    COLOR level.  The frozen shell is reset to chi0 when the config's
    boundary type is FROZEN, as Simulation.equilibrate does.
    """
    import torch

    from . import _lib
    from .backend import _stream_handle

    N = int(config.grid_size)
    if out is None:
        out = torch.empty((N, N, N), dtype=torch.float32, device=psi_r.device)
    frozen = config.boundary_type == BoundaryType.FROZEN
    _lib.call("lfm_poisson_chi_f32", backend.context.handle, int(config.field_level),
              psi_r.data_ptr(), None if psi_i is None else psi_i.data_ptr(), N,
              float(config.chi0), float(config.kappa), float(config.e0_sq),
              float(config.boundary_fraction), int(frozen), out.data_ptr(),
              _stream_handle(backend.device))
    return out


def _initial_state(cfg, soliton, equilibrate, backend):
    """(psi_r, psi_i, chi) device tensors of a fresh Simulation after
    place_soliton / equilibrate."""
    import torch

    N = int(cfg.grid_size)
    level = FieldLevel(int(cfg.field_level))
    dev = backend.device
    shape = (3, N, N, N) if level == FieldLevel.COLOR else (N, N, N)
    pr = torch.zeros(shape, dtype=torch.float32, device=dev)
    pi = None if level == FieldLevel.REAL else torch.zeros(shape, dtype=torch.float32, device=dev)
    placed = soliton is not None
    if placed:
        kw = dict(soliton)
        pos = kw.pop("position", None)
        if pos is None:
            pos = (N // 2, N // 2, N // 2)
        if kw.pop("velocity", None) is not None:
            raise NotImplementedError("velocity-boosted packets are not supported in sweeps")
        amp = kw.pop("amplitude", None)
        sig = kw.pop("sigma", None)
        phase = kw.pop("phase", 0.0)
        if kw:
            raise TypeError(f"unexpected soliton arguments {sorted(kw)}")
        amp = cfg.e_amplitude if amp is None else amp
        sig = cfg.sigma if sig is None else sig
        r, i = gaussian_soliton(N, pos, amp, sig, phase)
        pr += torch.from_numpy(r).to(dev)  # broadcast over colours, as current + pr does
        if pi is not None:
            pi += torch.from_numpy(i).to(dev)
    if equilibrate or placed:
        chi = equilibrate_chi(backend, cfg, pr, pi)
    else:
        chi = torch.full((N, N, N), float(cfg.chi0), dtype=torch.float32, device=dev)
    return pr, pi, chi


def _snapshot_step(cfg, steps: int) -> int:
    """Step of the Psi snapshot run() leaves for metrics(): the last multiple of
    report_interval reached, or 0."""
    r = int(cfg.report_interval)
    if r <= 0 or steps < r:
        return 0
    return (steps // r) * r


def _metrics(backend, cfg, st: dict, prev_r, prev_i) -> dict:
    from .metrics import device_metrics, interior_mask, n_clusters

    N = int(cfg.grid_size)
    m = device_metrics(backend.context.handle, int(cfg.field_level), N,
                       st["psi_r"].contiguous(), prev_r.contiguous(),
                       None if st.get("psi_i") is None else st["psi_i"].contiguous(),
                       None if prev_i is None else prev_i.contiguous(), st["chi"].contiguous(),
                       cfg.dt, getattr(cfg, "c", 1.0), cfg.boundary_fraction)
    psi_sq = st["psi_r"].double() ** 2
    if st.get("psi_i") is not None:
        psi_sq = psi_sq + st["psi_i"].double() ** 2
    if psi_sq.dim() == 4:
        psi_sq = psi_sq.sum(0)
    m["n_clusters"] = float(n_clusters(psi_sq.cpu().numpy(),
                                       interior_mask(N, cfg.boundary_fraction)))
    return {k: m[k] for k in METRIC_KEYS}


def _batchable(cfg) -> bool:
    return (int(cfg.field_level) in (FieldLevel.REAL, FieldLevel.COMPLEX)
            and int(cfg.grid_size) % 4 == 0 and int(cfg.grid_size) >= 8)


def run_configs(configs, steps: int, *, equilibrate: bool = True, soliton=None,
                backend="auto", batched: bool = True) -> list[dict]:
    """Metrics after `steps` steps of each config (the body of sweep / sweep_2d)."""
    import torch

    from . import Evolver
    from .backend import B200Backend, get_backend
    from .batch import BatchedLattices

    be = backend if isinstance(backend, B200Backend) else get_backend(backend)
    steps = int(steps)
    results: list[dict | None] = [None] * len(configs)
    init = [_initial_state(c, soliton, equilibrate, be) for c in configs]
    # lattices stepped together share the snapshot step
    groups: dict[int, list[int]] = {}
    alone: list[int] = []
    for i, c in enumerate(configs):
        if batched and _batchable(c):
            groups.setdefault(_snapshot_step(c, steps), []).append(i)
        else:
            alone.append(i)
    for snap, idx in groups.items():
        B = BatchedLattices([configs[i] for i in idx], backend=be)
        for b, i in enumerate(idx):
            pr, pi, chi = init[i]
            B.set_psi_real(b, pr)
            if pi is not None:
                B.set_psi_imag(b, pi)
            B.set_chi(b, chi)
        B.evolve(snap)
        prev = [(B._pr[b][B._cur].clone(),
                 None if B._pi[b] is None else B._pi[b][B._cur].clone())
                for b in range(len(idx))]
        B.evolve(steps - snap)
        for b, i in enumerate(idx):
            results[i] = _metrics(be, configs[i], B.device_state(b), *prev[b])
        B.close()
        del B
    for i in alone:
        c = configs[i]
        ev = Evolver(c, backend=be)
        pr, pi, chi = init[i]
        ev.set_psi_real(pr)
        if pi is not None:
            ev.set_psi_imag(pi)
        ev.set_chi(chi)
        snap = _snapshot_step(c, steps)
        ev.evolve(snap)
        st = ev.device_state()
        prev = (st["psi_r"].clone(), None if st.get("psi_i") is None else st["psi_i"].clone())
        ev.evolve(steps - snap)
        results[i] = _metrics(be, c, ev.device_state(), *prev)
    torch.cuda.synchronize(be.device)
    return results  # type: ignore[return-value]


# ------------------------------------------------------------------ sharding
def shard(costs, world: int) -> list[list[int]]:
    """Contiguous groups of run indices, one per rank, balancing the summed
    cost (N^3 per run).  Every index lands in exactly one group; ranks may
    get nothing when there are fewer runs than ranks."""
    costs = [float(c) for c in costs]
    total = sum(costs)
    out: list[list[int]] = [[] for _ in range(world)]
    acc, r = 0.0, 0
    for i, c in enumerate(costs):
        # move on once this rank's share is reached and ranks remain for the rest
        while r < world - 1 and acc >= total * (r + 1) / world:
            r += 1
        out[r].append(i)
        acc += c
    return out


def _distributed():
    try:
        import torch.distributed as dist
    except ImportError:  # pragma: no cover
        return None
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        return dist
    return None


def _run_sharded(configs, steps, runner, **kw) -> list[dict]:
    dist = _distributed()
    if dist is None:
        return runner(configs, steps, **kw)
    world, rank = dist.get_world_size(), dist.get_rank()
    parts = shard([int(c.grid_size) ** 3 for c in configs], world)
    mine = parts[rank]
    rows = runner([configs[i] for i in mine], steps, **kw) if mine else []
    gathered: list = [None] * world
    dist.all_gather_object(gathered, (mine, rows))
    out: list[dict | None] = [None] * len(configs)
    for idx, part_rows in gathered:
        for i, row in zip(idx, part_rows):
            out[i] = row
    return out  # type: ignore[return-value]


def _rows(param_values, configs, steps, metric_names, runner, **kw) -> list[dict[str, Any]]:
    metrics = _run_sharded(configs, steps, runner, **kw)
    rows = []
    for pv, m in zip(param_values, metrics):
        row: dict[str, Any] = dict(pv)
        if metric_names is not None:
            for k in metric_names:
                row[k] = m.get(k)
        else:
            row.update(m)
        rows.append(row)
    return rows


def sweep(config, param: str, values: list, steps: int, metric_names: list | None = None, *,
          equilibrate: bool = True, soliton: dict | None = None, backend="auto",
          batched: bool = True, runner=None) -> list[dict[str, Any]]:
    """Run `steps` for each value of `param`; one row {param: value, **metrics} per value
    (lfm/sweep.py:14-82).  runner replaces the device runner (for tests)."""
    configs, pvs = [], []
    for val in values:
        cfg = deepcopy(config)
        setattr(cfg, param, val)  # as the reference: derived fields (sigma ...) keep the base's
        configs.append(cfg)
        pvs.append({param: val})
    run = runner or run_configs
    kw = dict(equilibrate=equilibrate, soliton=soliton)
    if runner is None:
        kw.update(backend=backend, batched=batched)
    return _rows(pvs, configs, steps, metric_names, run, **kw)


def sweep_2d(config, param1: str, values1: list, param2: str, values2: list, steps: int,
             metric_names: list | None = None, *, equilibrate: bool = True,
             soliton: dict | None = None, backend="auto", batched: bool = True,
             runner=None) -> list[dict[str, Any]]:
    """Every (value1, value2) combination, param1 outermost (lfm/sweep.py:85-157)."""
    configs, pvs = [], []
    for v1, v2 in itertools.product(values1, values2):
        cfg = deepcopy(config)
        setattr(cfg, param1, v1)
        setattr(cfg, param2, v2)
        configs.append(cfg)
        pvs.append({param1: v1, param2: v2})
    run = runner or run_configs
    kw = dict(equilibrate=equilibrate, soliton=soliton)
    if runner is None:
        kw.update(backend=backend, batched=batched)
    return _rows(pvs, configs, steps, metric_names, run, **kw)
