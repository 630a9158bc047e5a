"""Slab decomposition of one lattice along i: the plane split, the ghost
exchange between ranks (gloo, CPU) and, on the GPU, slab steps against the
whole-lattice Evolver bit for bit."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest


def bits_equal(a, b) -> bool:
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("N, world", [(16, 1), (16, 2), (16, 3), (13, 4), (128, 8), (9, 9)])
def test_split_planes_covers_the_lattice(N, world):
    from lfm_b200.slab import split_planes

    parts = split_planes(N, world)
    assert len(parts) == world
    assert parts[0][0] == 0 and sum(n for _, n in parts) == N
    for (f0, n0), (f1, _) in zip(parts, parts[1:]):
        assert f1 == f0 + n0
    assert max(n for _, n in parts) - min(n for _, n in parts) <= 1
    with pytest.raises(ValueError):
        split_planes(N, N + 1)


# A stand-in step that only needs the i-neighbours: new[p] = 1*cur[p-1] + 2*cur[p]
# + 4*cur[p+1] + prev[p] on the slab's own planes (exact in float32 for small
# integers), and the same stencil on the whole periodic lattice.
def toy_step(slab, lo, hi):
    c, p = slab.cur, 1 - slab.cur
    for cur_f, prev_f in zip(slab.stencil_fields(c), slab.stencil_fields(p)):
        new = cur_f[lo - 1:hi - 1] + 2 * cur_f[lo:hi] + 4 * cur_f[lo + 1:hi + 1] + prev_f[lo:hi]
        prev_f[lo:hi].copy_(new)


def toy_whole(cur, prev):
    return np.roll(cur, 1, 0) + 2 * cur + 4 * np.roll(cur, -1, 0) + prev


def _cfg(N, cx):
    from lfm_b200.config import gravity_em, gravity_only

    return (gravity_em if cx else gravity_only)(N)


def _gloo_worker(rank, world, port, N, cx, overlap, q):
    import torch.distributed as dist

    from lfm_b200.slab import SlabEvolver

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(3)
        a = rng.integers(-3, 4, size=(N, N, N)).astype(np.float32)
        s = SlabEvolver(_cfg(N, cx), stepper=toy_step, device="cpu")
        s.overlap = overlap
        s.set_psi_real(a)
        s.set_chi(2 * a)
        if cx:
            s.set_psi_imag(-a)
        s.evolve(3)
        q.put((rank, s.get_psi_real(), s.get_chi(), s.get_psi_imag()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world, N, cx, overlap", [(2, 8, False, False), (3, 10, True, True),
                                                   (2, 8, True, True), (3, 8, False, True)])
def test_ghost_exchange_over_gloo_matches_the_whole_lattice(world, N, cx, overlap):
    """With overlap the boundary planes step first and their exchange runs while
    the interior planes step (N=8 over 3 ranks: one slab of 2 planes, too thin to overlap)."""
    import torch.multiprocessing as mp

    rng = np.random.default_rng(3)
    a = rng.integers(-3, 4, size=(N, N, N)).astype(np.float32)
    want = {}
    for name, init in (("psi_r", a), ("chi", 2 * a), ("psi_i", -a)):
        cur, prev = init.copy(), init.copy()
        for _ in range(3):
            cur, prev = toy_whole(cur, prev), cur
        want[name] = cur
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_worker, args=(r, world, port, N, cx, overlap, q))
             for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, pr, chi, pi in got:
        assert np.array_equal(pr, want["psi_r"]), rank
        assert np.array_equal(chi, want["chi"]), rank
        if cx:
            assert np.array_equal(pi, want["psi_i"]), rank


# The reference's REAL step (oracle.numpy_step_real, pinned to the reference's
# fixtures) on a slab's planes with their ghosts: what lfm_slab_step_planes_f32
# computes on the GPU, here on the CPU, so the gloo ranks run the slab plan
# (plane ranges, ghost planes, damping of the previous field on read) with the
# step's own arithmetic.
def oracle_slab_step(slab, lo, hi):
    import torch

    from lfm_b200.mask import boundary_mask
    from oracle import oracle as O

    N, cfg = slab.N, slab.config
    c, p = slab.cur, 1 - slab.cur
    m = boundary_mask(N, cfg.boundary_fraction).reshape(N, N, N)[slab._global_planes()]
    e, x = slab.pr[c].numpy(), slab.chi[c].numpy()
    ep, xp = slab.pr[p].numpy(), slab.chi[p].numpy()
    if slab.damp:  # the previous slot holds the undamped field
        ep = ep * (np.float32(1.0) - m)
    out = O.numpy_step_real(e, ep, x, xp, m, N, cfg.dt**2, cfg.kappa, cfg.lambda_self,
                            cfg.chi0, cfg.e0_sq)
    shape = e.shape
    slab.pr[p][lo:hi] = torch.from_numpy(out[0].reshape(shape)[lo:hi])
    slab.chi[p][lo:hi] = torch.from_numpy(out[2].reshape(shape)[lo:hi])


def _gloo_oracle_worker(rank, world, port, N, overlap, q):
    import torch.distributed as dist

    from lfm_b200.slab import SlabEvolver
    from lfm_b200.workloads import config1_soliton

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = SlabEvolver(_cfg(N, False), stepper=oracle_slab_step, device="cpu")
        s.overlap = overlap
        s.set_psi_real(config1_soliton(N))
        s.evolve(6)
        q.put((rank, s.get_psi_real(), s.get_chi()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world, N, overlap", [(2, 16, True), (3, 16, True), (2, 12, False)])
def test_slab_plan_with_the_real_step_over_gloo_is_bit_exact(world, N, overlap):
    """Every rank steps its slab with the reference's arithmetic (boundary planes, the
    exchange, then the interior with overlap); the gathered lattice equals the oracle's
    whole-lattice steps bit for bit."""
    import torch.multiprocessing as mp

    from lfm_b200.workloads import config1_soliton
    from oracle import oracle as O

    lat = O.OracleLattice(_cfg(N, False))
    lat.set_psi_real(config1_soliton(N))
    lat.step(6)
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_oracle_worker, args=(r, world, port, N, overlap, q))
             for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, pr, chi in got:
        assert bits_equal(pr.ravel(), lat.pr), rank
        assert bits_equal(chi.ravel(), lat.chi), rank


def test_slab_rejects_color():
    from lfm_b200.config import full_physics
    from lfm_b200.slab import SlabEvolver

    with pytest.raises(ValueError):
        SlabEvolver(full_physics(16), stepper=toy_step, device="cpu")


# ---------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def be(cuda_device):
    from lfm_b200 import B200Backend, _lib
    from lfm_b200.build import build_library

    build_library()
    _lib.set_step_path(_lib.PATH_AUTO)
    return B200Backend(cuda_device)


def _state(N, cx, seed):
    rng = np.random.default_rng(seed)
    E = (0.7 * rng.standard_normal((N, N, N))).astype(np.float32)
    chi = (19.0 + 0.05 * rng.standard_normal((N, N, N))).astype(np.float32)
    pi = (0.4 * rng.standard_normal((N, N, N))).astype(np.float32) if cx else None
    return E, pi, chi


def _load(tgt, E, pi, chi):
    tgt.set_psi_real(E)
    if pi is not None:
        tgt.set_psi_imag(pi)
    tgt.set_chi(chi)


@pytest.mark.gpu
@pytest.mark.parametrize("N, world, overlap", [(24, 1, False), (24, 3, False), (20, 2, False),
                                               (128, 4, False), (128, 3, False), (24, 3, True),
                                               (128, 4, True), (20, 2, True)])
@pytest.mark.parametrize("level", ["real", "complex"])
def test_slabs_match_the_whole_lattice(be, N, world, overlap, level):
    from lfm_b200 import Evolver
    from lfm_b200.slab import SlabEvolver, evolve_local, gather_local

    cx = level == "complex"
    cfg = _cfg(N, cx)
    E, pi, chi = _state(N, cx, N + world)
    ev = Evolver(cfg, backend=be)
    _load(ev, E, pi, chi)
    slabs = [SlabEvolver(cfg, backend=be, rank=r, world=world) for r in range(world)]
    for s in slabs:
        _load(s, E, pi, chi)
    steps = 7
    ev.evolve(steps)
    evolve_local(slabs, steps, overlap=overlap)
    assert bits_equal(gather_local(slabs, "psi_r"), ev.get_psi_real())
    assert bits_equal(gather_local(slabs, "chi"), ev.get_chi())
    if cx:
        assert bits_equal(gather_local(slabs, "psi_i"), ev.get_psi_imag())
    from lfm_b200 import _lib

    assert _lib.device_status() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("level, overlap", [("real", False), ("real", True), ("complex", False)])
def test_slabs_of_a_512_lattice_on_the_compile_time_tiles(be, level, overlap):
    """Two slabs of a 512^3 lattice run on the compile-time 512^3 tiles (their slab
    variant: ghost planes, the sponge key of the global plane) and agree bit for bit
    with the whole lattice after 3 steps."""
    from lfm_b200 import Evolver, _lib
    from lfm_b200.slab import SlabEvolver, evolve_local, gather_local

    N, world, steps = 512, 2, 3
    cx = level == "complex"
    cfg = _cfg(N, cx)
    E, pi, chi = _state(N, cx, 77)
    ev = Evolver(cfg, backend=be)
    _load(ev, E, pi, chi)
    ev.evolve(steps)
    want = [ev.get_psi_real(), ev.get_chi()] + ([ev.get_psi_imag()] if cx else [])
    del ev
    slabs = [SlabEvolver(cfg, backend=be, rank=r, world=world) for r in range(world)]
    for sl in slabs:
        _load(sl, E, pi, chi)
    evolve_local(slabs, steps, overlap=overlap)
    got = [gather_local(slabs, "psi_r"), gather_local(slabs, "chi")]
    if cx:
        got.append(gather_local(slabs, "psi_i"))
    for g, w in zip(got, want):
        assert bits_equal(g, w)
    assert _lib.device_status() == 0


@pytest.mark.gpu
def test_single_slab_is_the_whole_lattice(be):
    from lfm_b200 import Evolver
    from lfm_b200.slab import SlabEvolver

    cfg = _cfg(32, True)
    E, pi, chi = _state(32, True, 5)
    ev, s = Evolver(cfg, backend=be), SlabEvolver(cfg, backend=be)
    for t in (ev, s):
        _load(t, E, pi, chi)
    ev.evolve(5)
    s.evolve(5)
    assert s.world == 1 and s.n_local == 32
    assert bits_equal(s.get_psi_real(), ev.get_psi_real())
    assert bits_equal(s.get_chi(), ev.get_chi())
