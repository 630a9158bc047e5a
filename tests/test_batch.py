"""Batched lattices: the work-list plan (host only) and GPU parity of the
persistent batch kernel against the single-lattice Evolver and the oracle.

Each lattice of a batch must come out bit-for-bit as it does when stepped
alone, whatever the batch's mix of sizes, levels and constants.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O


def bits_equal(a, b) -> bool:
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.fixture(scope="module")
def lib():
    from lfm_b200 import _lib
    from lfm_b200.build import build_library

    build_library()
    return _lib.load()


def mixed_configs(sizes, seed=11):
    from lfm_b200.config import gravity_em, gravity_only

    rng = np.random.default_rng(seed)
    out = []
    for k, N in enumerate(sizes):
        make = gravity_em if k % 2 else gravity_only
        out.append(make(N, kappa=float(rng.uniform(0.5, 2.0)) / 63.0,
                        boundary_fraction=float(rng.choice([0.15, 0.3]))))
    return out


def check_coverage(configs, items):
    cov = {}
    for lvl, l, j0, j1, i0, i1 in items:
        N = configs[l].grid_size
        assert lvl == int(configs[l].field_level)
        assert 0 <= j0 < j1 <= N and 0 <= i0 < i1 <= N
        a = cov.setdefault(l, np.zeros((N, N), np.int32))
        a[i0:i1, j0:j1] += 1
    assert sorted(cov) == list(range(len(configs)))
    assert all((a == 1).all() for a in cov.values())


def _batch_shapes():
    """The batch's shape classes (level, N, largest tile), read from kBatchShapes in
    csrc/lfm_batch.h so the test follows the kernel's table."""
    import re
    from pathlib import Path

    src = (Path(__file__).resolve().parents[1] / "lfm-physics_b200" / "csrc" /
           "lfm_batch.h").read_text()
    body = src[src.index("kBatchShapes[kBatchClasses] = {"):]
    body = body[:body.index("};")]
    lv = {"LFM_REAL": 0, "LFM_COMPLEX": 1}
    return [(lv[a], int(b), int(c))
            for a, b, c in re.findall(r"\{(LFM_\w+),\s*(\d+),\s*(\d+)\}", body)]


SHAPES = _batch_shapes()


def shape_class(cfg, threads):
    """The class a lattice's items run in: its (level, N, largest tile) as the planner cuts
    it (as few row tiles as the CTA allows, rows as even as possible), else its level's
    run-time class."""
    level, N = int(cfg.field_level), cfg.grid_size
    tpr = N // (4 if level == 0 else 2)
    tiles = -(-N // (threads // tpr))
    TJ = -(-N // tiles)
    for c, (lv, n, tj) in enumerate(SHAPES):
        if lv == level and (n, tj) == (N, TJ):
            return c
    return next(c for c, (lv, n, _) in enumerate(SHAPES) if lv == level and n == 0)


def test_shape_table_parsed():
    assert len(SHAPES) == 12 and sum(n == 0 for _, n, _ in SHAPES) == 2


# ---------------------------------------------------------------- host only
@pytest.mark.parametrize("tuning", [None, dict(threads=128), dict(stages=5, item_cells=4096),
                                    dict(threads=512, item_cells=1 << 20)])
def test_plan_covers_every_cell_once(lib, tuning):
    from lfm_b200 import batch
    from lfm_b200.workloads import sweep_lattices

    cfgs = [c for c, _, _ in sweep_lattices(64, seed=5)] + mixed_configs([8, 12, 16, 20, 100])
    p = batch.plan(cfgs, tuning)
    check_coverage(cfgs, p["items"])
    threads, smem, grid = p["launch"]
    assert threads % 32 == 0 and 0 < threads <= (tuning or {}).get("threads", 256)
    assert 0 < smem <= 226 * 1024 and 0 < grid
    # REAL items first, then COMPLEX; grouped by shape class, each class's
    # largest items first
    it = p["items"]
    assert (np.diff(it[:, 0]) >= 0).all()
    threads = (tuning or {}).get("threads", 256)
    cls = np.array([shape_class(cfgs[l], threads) for l in it[:, 1]])
    assert (np.diff(cls) >= 0).all()
    for c in np.unique(cls):
        sub = it[cls == c]
        N = np.array([cfgs[l].grid_size for l in sub[:, 1]])
        cost = (sub[:, 3] - sub[:, 2]) * N * (sub[:, 5] - sub[:, 4])
        assert (np.diff(cost) <= 0).all()


def test_plan_of_the_sweep_workload(lib):
    from lfm_b200 import batch
    from lfm_b200.workloads import sweep_lattices

    cfgs = [c for c, _, _ in sweep_lattices()]
    assert len(cfgs) == 256
    assert {c.grid_size for c in cfgs} == {32, 48, 64, 80, 96}
    p = batch.plan(cfgs)
    check_coverage(cfgs, p["items"])
    threads, smem, grid = p["launch"]
    assert grid == 296
    # at 256 threads every lattice of the sweep has a compile-time shape class
    rt = {c for c, (_, n, _) in enumerate(SHAPES) if n == 0}
    assert all(shape_class(c, 256) not in rt for c in cfgs)


@pytest.mark.parametrize("bad, code", [(dict(N=10), 3), (dict(level=2), 3), (dict(N=4), 3)])
def test_plan_rejects_unsupported_lattices(lib, bad, code):
    from lfm_b200 import _lib, batch
    from lfm_b200.config import FieldLevel, full_physics, gravity_only

    if "level" in bad:
        cfg = full_physics(16)
        assert cfg.field_level == FieldLevel.COLOR
    else:
        cfg = gravity_only(16)
        cfg.grid_size = bad["N"]  # bypass the config's own checks
    with pytest.raises(_lib.LfmError) as e:
        batch.plan([gravity_only(16), cfg])
    assert e.value.code == code


@pytest.mark.parametrize("tuning", [dict(threads=48), dict(stages=2), dict(item_cells=10)])
def test_plan_rejects_bad_tuning(lib, tuning):
    from lfm_b200 import _lib, batch
    from lfm_b200.config import gravity_only

    with pytest.raises(_lib.LfmError) as e:
        batch.plan([gravity_only(16)], tuning)
    assert e.value.code == _lib.LFM_ERR_INVALID_ARG


# ---------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def be(cuda_device, lib):
    from lfm_b200 import B200Backend, _lib

    _lib.set_step_path(_lib.PATH_AUTO)
    return B200Backend(cuda_device)


def seed_fields(cfg, rng):
    N = cfg.grid_size
    c = N / 2.0
    from lfm_b200.workloads import add_gaussian

    pr = np.zeros((N, N, N))
    add_gaussian(pr, (c, c - 1.5, c + 0.5), float(rng.uniform(1, 8)), float(rng.uniform(1.5, 3)))
    pr += 1e-3 * rng.standard_normal(pr.shape)
    pi = None
    if int(cfg.field_level) == 1:
        pi = 0.5 * np.roll(pr, 2, axis=1) + 1e-3 * rng.standard_normal(pr.shape)
        pi = pi.astype(np.float32)
    chi = (cfg.chi0 + 1e-3 * rng.uniform(-1, 1, pr.shape)).astype(np.float32)
    return pr.astype(np.float32), pi, chi


def run_pair(be, cfgs, steps, tuning=None, mid=None):
    """Batch and per-lattice Evolvers from the same seeded state."""
    from lfm_b200 import Evolver
    from lfm_b200.batch import BatchedLattices

    rng = np.random.default_rng(3)
    init = [seed_fields(c, rng) for c in cfgs]
    B = BatchedLattices(cfgs, backend=be, tuning=tuning)
    evs = []
    for i, (c, (pr, pi, chi)) in enumerate(zip(cfgs, init)):
        ev = Evolver(c, backend=be)
        for tgt in (B, ev):
            args = (i,) if tgt is B else ()
            tgt.set_psi_real(*args, pr)
            if pi is not None:
                tgt.set_psi_imag(*args, pi)
            tgt.set_chi(*args, chi)
        evs.append(ev)
    first = steps if mid is None else mid[0]
    B.evolve(first)
    for ev in evs:
        ev.evolve(first)
    if mid is not None:
        i, arr_fn = mid[1], mid[2]
        a = arr_fn(cfgs[i].grid_size)
        B.set_psi_real(i, a)
        evs[i].set_psi_real(a)
        B.evolve(steps - first)
        for ev in evs:
            ev.evolve(steps - first)
    return B, evs


def assert_same(B, evs):
    for i, ev in enumerate(evs):
        assert bits_equal(B.get_psi_real(i), ev.get_psi_real()), i
        assert bits_equal(B.get_chi(i), ev.get_chi()), i
        assert bits_equal(B.get_psi_real_prev(i), ev.get_psi_real_prev()), i
        if ev.get_psi_imag() is not None:
            assert bits_equal(B.get_psi_imag(i), ev.get_psi_imag()), i
            assert bits_equal(B.get_psi_imag_prev(i), ev.get_psi_imag_prev()), i


@pytest.mark.gpu
@pytest.mark.parametrize("steps", [1, 2, 7, 37])
def test_batch_matches_single_lattice_evolver(be, steps):
    cfgs = mixed_configs([16, 20, 8, 32, 24, 12, 36, 40, 48, 28])
    B, evs = run_pair(be, cfgs, steps)
    assert_same(B, evs)
    from lfm_b200 import _lib

    assert _lib.device_status() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("tuning", [dict(threads=128), dict(stages=5, item_cells=2048),
                                    dict(threads=512, ctas_per_sm=1)])
def test_batch_tuning_does_not_change_results(be, tuning):
    cfgs = mixed_configs([16, 20, 32, 24, 40, 44])
    B, evs = run_pair(be, cfgs, 9, tuning=tuning)
    assert_same(B, evs)


@pytest.mark.gpu
def test_batch_host_write_between_steps(be):
    cfgs = mixed_configs([16, 20, 24])
    rng = np.random.default_rng(9)
    B, evs = run_pair(be, cfgs, 20, mid=(7, 1, lambda N: rng.standard_normal((N,) * 3)
                                        .astype(np.float32)))
    assert_same(B, evs)


@pytest.mark.gpu
def test_batch_matches_oracle(be):
    from lfm_b200.batch import BatchedLattices

    cfgs = mixed_configs([16, 20])
    rng = np.random.default_rng(5)
    init = [seed_fields(c, rng) for c in cfgs]
    B = BatchedLattices(cfgs, backend=be)
    lats = []
    for i, (c, (pr, pi, chi)) in enumerate(zip(cfgs, init)):
        lat = O.OracleLattice(c)
        for tgt, args in ((B, (i,)), (lat, ())):
            tgt.set_psi_real(*args, pr)
            if pi is not None:
                tgt.set_psi_imag(*args, pi)
            tgt.set_chi(*args, chi)
        lats.append(lat)
    B.evolve(12)
    for i, lat in enumerate(lats):
        lat.step(12)
        assert bits_equal(B.get_psi_real(i).ravel(), lat.pr)
        assert bits_equal(B.get_chi(i).ravel(), lat.chi)
        if lat.pi is not None:
            assert bits_equal(B.get_psi_imag(i).ravel(), lat.pi)


@pytest.mark.gpu
def test_sweep_workload_subset(be):
    from lfm_b200 import Evolver
    from lfm_b200.batch import BatchedLattices
    from lfm_b200.workloads import sweep_lattices

    L = sweep_lattices(12, seed=5)
    cfgs = [c for c, _, _ in L]
    B = BatchedLattices(cfgs, backend=be)
    for i, (c, pr, pi) in enumerate(L):
        B.set_psi_real(i, pr)
        if pi is not None:
            B.set_psi_imag(i, pi)
    B.evolve(24)
    for i, (c, pr, pi) in enumerate(L):
        ev = Evolver(c, backend=be)
        ev.set_psi_real(pr)
        if pi is not None:
            ev.set_psi_imag(pi)
        ev.evolve(24)
        assert bits_equal(B.get_psi_real(i), ev.get_psi_real()), i
        assert bits_equal(B.get_chi(i), ev.get_chi()), i
        m = B.metrics(i)
        assert m["nonfinite_cells"] == 0


@pytest.mark.gpu
def test_autotune_batch_keeps_state_and_bits(be, tmp_path, monkeypatch):
    from lfm_b200 import autotune

    monkeypatch.setenv("LFM_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    cfgs = mixed_configs([16, 20, 32, 24])
    B, evs = run_pair(be, cfgs, 5)
    before = [B.get_psi_real(i) for i in range(len(cfgs))]
    rep = autotune.tune_batch(B, candidates=[dict(threads=128), dict(threads=256, stages=4),
                                             dict(item_cells=2048)], steps=3)
    assert len(rep["trials"]) == 3 and rep["best"] in [t["tuning"] for t in rep["trials"]]
    assert all(bits_equal(B.get_psi_real(i), b) for i, b in enumerate(before))
    assert B.step == 5
    B.evolve(6)
    for ev in evs:
        ev.evolve(6)
    assert_same(B, evs)
    # full search with the cache: a second call is a cache hit
    r1 = autotune.tune_batch(B, steps=2)
    r2 = autotune.tune_batch(B, steps=2)
    assert r1["best"] == r2["best"] and (tmp_path / "tune.json").exists()


@pytest.mark.gpu
def test_autotune_lattice_pins_a_tile(be, tmp_path, monkeypatch):
    from lfm_b200 import Evolver, _lib, autotune
    from lfm_b200.config import gravity_only

    monkeypatch.setenv("LFM_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    cfg = gravity_only(32)
    rng = np.random.default_rng(1)
    pr, _, chi = seed_fields(cfg, rng)
    ev, ref = Evolver(cfg, backend=be), Evolver(cfg, backend=be)
    for e in (ev, ref):
        e.set_psi_real(pr)
        e.set_chi(chi)
        e.evolve(3)
    rep = autotune.tune_lattice(ev, candidates=[dict(vec=4, tj=8, stages=3, ic=0),
                                                dict(vec=2, tj=4, stages=4, ic=16)], steps=3)
    try:
        assert len(rep["trials"]) == 2
        assert ev.step == 3
        ev.evolve(8)
        assert _lib.tune_get(0, 32)["tj"] == rep["best"]["tj"]  # the pinned tile ran
        ref.evolve(8)
        assert bits_equal(ev.get_psi_real(), ref.get_psi_real())
        assert bits_equal(ev.get_chi(), ref.get_chi())
    finally:
        _lib.tune_set(0, 32, 0, 0, 0, 0)
