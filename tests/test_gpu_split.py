"""Split-chi steps (chi = chi0 + hi + lo, float64 chi arithmetic) on the GPU.

* The fused and the direct kernels give the same bits (every operation is an
  explicit _rn intrinsic), in eager steps and in replayed CUDA graphs.
* Against the float64 oracle (the C oracle in float64: the reference's NumPy
  step, lfm/core/backends/numpy_backend.py:80-205, in double), the split path
  stays within the north-star bound of 1e-5 max-relative after 1000 steps of
  the 64^3 REAL workload, where the plain float32 path is at 9e-3.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

# max-relative against float64 after 1000 steps of the 64^3 REAL workload
# (emulated on the CPU before the kernel was written: E 3.9e-6, chi 4.7e-8)
TARGET_E = 1e-5
TARGET_CHI = 1e-6


@pytest.fixture(scope="module")
def be(cuda_device):
    from lfm_b200 import B200Backend
    from lfm_b200.build import build_library

    build_library()
    return B200Backend(cuda_device)


def max_rel(a, ref):
    a = np.asarray(a, np.float64).ravel()
    ref = np.asarray(ref, np.float64).ravel()
    return float(np.abs(a - ref).max() / max(np.abs(ref).max(), 1e-300))


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _state(N, cx, seed=1):
    rng = np.random.default_rng(seed)
    E = O.gaussian_blob(N, (N / 2, N / 2 - 2, N / 2), 4.0, 2.5)
    E = (E + 1e-3 * rng.standard_normal(E.shape)).astype(np.float32)
    pi = (0.5 * np.roll(E, 3, axis=1)).astype(np.float32) if cx else None
    chi = (19.0 + 1e-3 * rng.uniform(-1, 1, E.shape)).astype(np.float32)
    return E, pi, chi


def _run(be, cfg, E, pi, chi, steps, graphs=True):
    from lfm_b200.split import SplitChiEvolver

    ev = SplitChiEvolver(cfg, backend=be)
    ev.use_graphs = graphs
    ev.set_psi_real(E)
    if pi is not None:
        ev.set_psi_imag(pi)
    ev.set_chi(chi)
    ev.evolve(steps)
    return ev


@pytest.mark.parametrize("level, N", [("real", 32), ("real", 48), ("complex", 32),
                                      ("complex", 48), ("real", 256), ("complex", 256)])
def test_fused_and_direct_kernels_agree(be, level, N):
    """Run-time tiles (32, 48) and the compile-time tiles (256) against the direct kernel."""
    from lfm_b200 import _lib
    from lfm_b200.config import gravity_em, gravity_only

    cx = level == "complex"
    cfg = (gravity_em if cx else gravity_only)(N)
    E, pi, chi = _state(N, cx)
    runs = []
    try:
        for path in (_lib.PATH_FUSED, _lib.PATH_DIRECT):
            _lib.set_step_path(path)
            runs.append(_run(be, cfg, E, pi, chi, 9, graphs=False))
    finally:
        _lib.set_step_path(_lib.PATH_AUTO)
    a, b = runs
    assert np.array_equal(bits(a.get_psi_real()), bits(b.get_psi_real()))
    assert np.array_equal(bits(a._hi[a._cur].cpu().numpy()), bits(b._hi[b._cur].cpu().numpy()))
    assert np.array_equal(bits(a._lo[a._cur].cpu().numpy()), bits(b._lo[b._cur].cpu().numpy()))
    if cx:
        assert np.array_equal(bits(a.get_psi_imag()), bits(b.get_psi_imag()))
    assert _lib.device_status() == 0


@pytest.mark.parametrize("level", ["real", "complex"])
def test_graph_replay_equals_eager_steps(be, level):
    from lfm_b200.config import gravity_em, gravity_only

    N = 24
    cx = level == "complex"
    cfg = (gravity_em if cx else gravity_only)(N)
    E, pi, chi = _state(N, cx, seed=3)
    g = _run(be, cfg, E, pi, chi, 21, graphs=True)
    e = _run(be, cfg, E, pi, chi, 21, graphs=False)
    assert np.array_equal(bits(g.get_psi_real()), bits(e.get_psi_real()))
    assert np.array_equal(bits(g.get_chi()), bits(e.get_chi()))
    assert np.array_equal(g.chi64().cpu().numpy(), e.chi64().cpu().numpy())


@pytest.mark.parametrize("level", ["real", "complex"])
def test_split_far_closer_to_float64_than_plain(be, level):
    """30^3 (direct kernel: N % 4 != 0) and 32^3 (fused), 400 steps."""
    from lfm_b200 import Evolver
    from lfm_b200.config import gravity_em, gravity_only

    cx = level == "complex"
    for N in (30, 32):
        cfg = (gravity_em if cx else gravity_only)(N)
        E, pi, chi = _state(N, cx, seed=5)
        lat = O.OracleLattice(cfg, dtype=np.float64)
        lat.set_psi_real(E.astype(np.float64))
        if cx:
            lat.set_psi_imag(pi.astype(np.float64))
        lat.set_chi(chi.astype(np.float64))
        O.set_threads(O.max_threads())
        lat.step(400)
        sp = _run(be, cfg, E, pi, chi, 400)
        pl = Evolver(cfg, backend=be)
        pl.set_psi_real(E)
        if cx:
            pl.set_psi_imag(pi)
        pl.set_chi(chi)
        pl.evolve(400)
        e_sp = max_rel(sp.get_psi_real(), lat.pr)
        c_sp = max_rel(sp.chi64().cpu().numpy(), lat.chi)
        e_pl = max_rel(pl.get_psi_real(), lat.pr)
        c_pl = max_rel(pl.get_chi(), lat.chi)
        print(level, N, "split", e_sp, c_sp, "plain", e_pl, c_pl)
        assert e_sp < 2e-5 and c_sp < 5e-7, (N, e_sp, c_sp)
        # chi is where float32 storage loses bits: 1e3-1e5 times closer at both levels
        # (measured); Psi gains as much at REAL, while the Mexican hat keeps the
        # COMPLEX run's plain float32 Psi within a few 1e-6 already
        assert c_sp < c_pl / 20, (N, c_sp, c_pl)
        assert e_sp < (e_pl / 20 if not cx else e_pl), (N, e_sp, e_pl)
        if cx:
            assert max_rel(sp.get_psi_imag(), lat.pi) < 1e-5


def test_config1_within_the_float64_bound_after_1000_steps(be):
    """The 64^3 REAL workload (gravity_only, packet 6.0 sigma 3 + 1e-4 noise), 1000 steps."""
    from lfm_b200.config import gravity_only
    from lfm_b200.workloads import config1_soliton

    N = 64
    cfg = gravity_only(N)
    E = config1_soliton(N)
    lat = O.OracleLattice(cfg, dtype=np.float64)
    lat.set_psi_real(E.astype(np.float64))
    O.set_threads(O.max_threads())
    lat.step(1000)
    sp = _run(be, cfg, E, None, np.full(E.shape, 19.0, np.float32), 1000)
    e = max_rel(sp.get_psi_real(), lat.pr)
    c = max_rel(sp.chi64().cpu().numpy(), lat.chi)
    print("config 1, split chi, 1000 steps: E", e, "chi", c)
    assert e < TARGET_E and c < TARGET_CHI, (e, c)
