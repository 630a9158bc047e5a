"""Sweeps: packet builder and Poisson equilibration against the reference's
own outputs, the batched sweep against lfm.sweep's rows, and the sharding of
runs across ranks (gloo, two processes, CPU)."""

from __future__ import annotations

import json
import os

import numpy as np
import pytest

from conftest import load_golden
from oracle import oracle as O

# cuFFT's float32 forward transform against pocketfft's: chi ~ 19 agrees to a
# couple of float32 ulps (ulp(19) = 1.9e-6)
CHI_ATOL = 4e-6
# sweep rows after 6-12 steps from that initial chi, relative
ROW_RTOL = 1e-4


def test_oracle_equilibrium_matches_the_reference():
    g = load_golden("equilibrium.npz")
    for N in (16, 20, 24):
        bf = float(g[f"bf_{N}"])
        pr, pi = g[f"pr_{N}"], g[f"pi_{N}"]
        r1, _ = O.gaussian_soliton(N, (N / 2, N / 2 - 2.5, N / 2 + 1.0), 5.0, 2.0, 0.7)
        assert np.array_equal(r1, g[f"soliton1_{N}"])
        assert np.array_equal(O.equilibrate_chi(pr, None, 19.0, 1 / 63, 0.0, bf), g[f"chi_real_{N}"])
        assert np.array_equal(O.equilibrate_chi(pr, pi, 19.0, 1 / 63, 0.0, bf),
                              g[f"chi_complex_{N}"])
        assert np.array_equal(O.equilibrate_chi(pr, pi, 19.0, 2 / 63, 0.5, None), g[f"chi_free_{N}"])
        assert np.array_equal(O.equilibrate_chi(g[f"colr_{N}"], g[f"coli_{N}"], 19.0, 1 / 63, 0.0, bf),
                              g[f"chi_color_{N}"])


def test_product_soliton_builder_matches_the_reference():
    from lfm_b200.sweep import gaussian_soliton

    g = load_golden("equilibrium.npz")
    for N in (16, 20, 24):
        r1, _ = gaussian_soliton(N, (N / 2, N / 2 - 2.5, N / 2 + 1.0), 5.0, 2.0, 0.7)
        assert np.array_equal(r1, g[f"soliton1_{N}"])


@pytest.mark.parametrize("world", [1, 2, 3, 5])
def test_shard_balances_and_covers(world):
    from lfm_b200.sweep import shard

    rng = np.random.default_rng(world)
    costs = rng.choice([32, 48, 64, 80, 96], size=37) ** 3
    parts = shard(costs, world)
    assert len(parts) == world
    flat = [i for p in parts for i in p]
    assert flat == list(range(len(costs)))  # contiguous, each index once
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) <= sum(costs) / world + max(costs)


def _fake_runner(configs, steps, **kw):
    return [{"N": float(c.grid_size), "kappa_x1e3": 1e3 * c.kappa, "steps": float(steps),
             "eq": float(kw["equilibrate"])} for c in configs]


def _gloo_worker(rank, world, port, q):
    import torch.distributed as dist

    from lfm_b200.config import gravity_only
    from lfm_b200.sweep import sweep, sweep_2d

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rows = sweep(gravity_only(16), "grid_size", [16, 32, 24, 48, 20], 7, runner=_fake_runner,
                     equilibrate=False)
        rows2 = sweep_2d(gravity_only(16), "kappa", [0.01, 0.02], "grid_size", [16, 24], 3,
                         metric_names=["N"], runner=_fake_runner)
        q.put((rank, rows, rows2))
    finally:
        dist.destroy_process_group()


def test_sharded_sweep_gathers_every_row_on_every_rank():
    import socket

    import torch.multiprocessing as mp

    from lfm_b200.config import gravity_only
    from lfm_b200.sweep import sweep, sweep_2d

    want = sweep(gravity_only(16), "grid_size", [16, 32, 24, 48, 20], 7, runner=_fake_runner,
                 equilibrate=False)
    want2 = sweep_2d(gravity_only(16), "kappa", [0.01, 0.02], "grid_size", [16, 24], 3,
                     metric_names=["N"], runner=_fake_runner)
    assert [r["grid_size"] for r in want] == [16, 32, 24, 48, 20]
    assert want[1] == {"grid_size": 32, "N": 32.0, "kappa_x1e3": 1e3 * (1.0 / 63.0),
                       "steps": 7.0, "eq": 0.0}
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, rows, rows2 in got:
        assert rows == want, rank
        assert rows2 == want2, rank


# ---------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def be(cuda_device):
    from lfm_b200 import B200Backend, _lib
    from lfm_b200.build import build_library

    build_library()
    _lib.set_step_path(_lib.PATH_AUTO)
    return B200Backend(cuda_device)


@pytest.mark.gpu
def test_device_equilibration_matches_the_reference(be):
    import torch

    from lfm_b200.config import full_physics, gravity_em, gravity_only
    from lfm_b200.sweep import equilibrate_chi

    g = load_golden("equilibrium.npz")
    dev = be.device
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    for N in (16, 20, 24):
        bf = float(g[f"bf_{N}"])
        cases = [
            (gravity_only(N, boundary_fraction=bf), g[f"pr_{N}"], None, g[f"chi_real_{N}"]),
            (gravity_em(N, boundary_fraction=bf, lambda_self=0.0), g[f"pr_{N}"], g[f"pi_{N}"],
             g[f"chi_complex_{N}"]),
            (full_physics(N, boundary_fraction=bf), g[f"colr_{N}"], g[f"coli_{N}"],
             g[f"chi_color_{N}"]),
        ]
        free = gravity_em(N, kappa=2 / 63, e0_sq=0.5)
        free.boundary_type = free.boundary_type.__class__("periodic")
        cases.append((free, g[f"pr_{N}"], g[f"pi_{N}"], g[f"chi_free_{N}"]))
        for cfg, pr, pi, want in cases:
            got = equilibrate_chi(be, cfg, t(pr), None if pi is None else t(pi)).cpu().numpy()
            assert np.abs(got - want).max() <= CHI_ATOL, (N, cfg.field_level)


@pytest.mark.gpu
@pytest.mark.parametrize("batched", [True, False])
def test_sweep_matches_lfm_sweep(be, batched):
    from conftest import golden_json

    from lfm_b200.config import gravity_em, gravity_only
    from lfm_b200.sweep import sweep, sweep_2d

    ref = golden_json(load_golden("sweep.npz")["runs"])
    got = {
        "kappa_real": sweep(gravity_only(16), "kappa", [1.0 / 63.0, 2.0 / 63.0], 12,
                            soliton={"amplitude": 4.0, "sigma": 2.0}, backend=be,
                            batched=batched),
        "grid_complex": sweep(gravity_em(16), "grid_size", [16, 20], 10,
                              soliton={"amplitude": 3.0, "sigma": 2.0, "phase": 0.5},
                              backend=be, batched=batched),
        "plain_noeq": sweep(gravity_only(16), "chi0", [19.0, 18.0], 6, equilibrate=False,
                            backend=be, batched=batched),
        "two_d": sweep_2d(gravity_em(12), "kappa", [1.0 / 63.0, 3.0 / 63.0], "epsilon_w",
                          [0.1, 0.2], 8, metric_names=["chi_min", "energy_total"],
                          soliton={"amplitude": 2.0, "sigma": 1.5}, backend=be,
                          batched=batched),
    }
    for name, rows in ref.items():
        assert len(got[name]) == len(rows), name
        for r_got, r_ref in zip(got[name], rows):
            assert set(r_got) == set(r_ref), (name, set(r_got) ^ set(r_ref))
            for k, v in r_ref.items():
                scale = max(abs(v), 1e-6 if "energy" not in k else abs(v) + 1e-3)
                assert abs(r_got[k] - v) <= ROW_RTOL * scale, (name, k, r_got[k], v)
