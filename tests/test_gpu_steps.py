"""GPU parity: the CUDA steps against the oracle and the reference fixtures.

The plain float32 kernels repeat NumPy's float32 operations one for one, so
every comparison here is bit-exact (np.array_equal on the raw bits) except
where cuFFT enters (S_a and, through SCV, chi at the COLOR level with
kappa_tube > 0), which is held to stated tolerances against the FP64 oracle.
"""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

from conftest import golden_json, load_golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu

DT = 0.02
DT2 = DT**2
CHI0 = 19.0
KAPPA = 1.0 / 63.0
LAMBDA_H = 4.0 / 31.0
CC = dict(kappa_c=1.0 / 189.0, epsilon_cc=2.0 / 17.0, kappa_string=1.0 / 189.0)
KT = 30.0 / 63.0

# S_a through cuFFT in float32 vs the reference's complex64 forward / float64
# inverse: relative to max|S_a|.
SA_REL_TOL = 2e-6
# chi after steps that include SCV from cuFFT S_a: absolute, chi ~ 19.
CHI_SA_ATOL = 2e-5


def bits_equal(a, b) -> bool:
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def be(cuda_device):
    from lfm_b200 import B200Backend, _lib
    from lfm_b200.build import build_library

    build_library()
    _lib.set_step_path(_lib.PATH_AUTO)
    return B200Backend(cuda_device)


@pytest.fixture(params=["auto", "direct"])
def path(request, be):
    from lfm_b200 import _lib

    _lib.set_step_path(_lib.PATH_AUTO if request.param == "auto" else _lib.PATH_DIRECT)
    yield request.param
    _lib.set_step_path(_lib.PATH_AUTO)


def rand_fields(rng, n, specs):
    return [(off + sc * rng.standard_normal(m * n)).astype(np.float32) for (sc, off, m) in specs]


@pytest.mark.parametrize("N", [12, 13, 16, 32, 64])
def test_protocol_step_real_bit_exact(be, path, N):
    rng = np.random.default_rng(N)
    n = N**3
    ins = rand_fields(rng, n, [(1, 0, 1), (1, 0, 1), (0.5, CHI0, 1), (0.5, CHI0, 1)])
    mask = O.boundary_mask(N, 0.3)
    for lam in (0.0, LAMBDA_H):
        ref = [np.empty(n, np.float32) for _ in range(4)]
        O.OracleBackend().step_real(*ins, mask, *ref, N, DT2, KAPPA, lam, CHI0, 0.01)
        d_in = [be.from_numpy(a) for a in ins]
        d_out = [be.from_numpy(np.zeros(n, np.float32)) for _ in range(4)]
        be.step_real(*d_in, be.from_numpy(mask), *d_out, N, DT2, KAPPA, lam, CHI0, 0.01)
        for k, (r, d) in enumerate(zip(ref, d_out)):
            assert bits_equal(be.to_numpy(d), r), f"output {k} lambda={lam}"


@pytest.mark.parametrize("N", [12, 13, 16, 32, 64])
def test_protocol_step_complex_bit_exact(be, path, N):
    rng = np.random.default_rng(100 + N)
    n = N**3
    ins = rand_fields(rng, n, [(1, 0, 1)] * 4 + [(0.5, CHI0, 1)] * 2)
    mask = O.boundary_mask(N, 0.3)
    ref = [np.empty(n, np.float32) for _ in range(6)]
    O.OracleBackend().step_complex(*ins, mask, *ref, N, DT2, KAPPA, LAMBDA_H, CHI0, 0.0, 0.1)
    d_in = [be.from_numpy(a) for a in ins]
    d_out = [be.from_numpy(np.zeros(n, np.float32)) for _ in range(6)]
    be.step_complex(*d_in, be.from_numpy(mask), *d_out, N, DT2, KAPPA, LAMBDA_H, CHI0, 0.0, 0.1)
    for k, (r, d) in enumerate(zip(ref, d_out)):
        assert bits_equal(be.to_numpy(d), r), f"output {k}"


@pytest.mark.parametrize("N", [12, 13, 16, 32])
@pytest.mark.parametrize("couplings", ["all_but_sa", "none", "cc_only"])
def test_protocol_step_color_bit_exact(be, path, N, couplings):
    rng = np.random.default_rng(200 + N)
    n = N**3
    ins = rand_fields(rng, n, [(1, 0, 3)] * 4 + [(0.5, CHI0, 1)] * 2)
    mask = O.boundary_mask(N, 0.3)
    cc = {"all_but_sa": CC, "none": dict(kappa_c=0.0, epsilon_cc=0.0, kappa_string=0.0),
          "cc_only": dict(kappa_c=0.0, epsilon_cc=CC["epsilon_cc"], kappa_string=0.0)}[couplings]
    shapes = [3 * n] * 4 + [n, n]
    ref = [np.empty(s, np.float32) for s in shapes]
    O.OracleBackend().step_color(*ins, mask, *ref, N, DT2, KAPPA, LAMBDA_H, CHI0, 0.0, 0.1,
                                 cc["kappa_c"], cc["epsilon_cc"], kappa_string=cc["kappa_string"])
    d_in = [be.from_numpy(a) for a in ins]
    d_out = [be.from_numpy(np.zeros(s, np.float32)) for s in shapes]
    be.step_color(*d_in, be.from_numpy(mask), *d_out, N, DT2, KAPPA, LAMBDA_H, CHI0, 0.0, 0.1,
                  cc["kappa_c"], cc["epsilon_cc"], kappa_string=cc["kappa_string"])
    for k, (r, d) in enumerate(zip(ref, d_out)):
        assert bits_equal(be.to_numpy(d), r), f"output {k}"


def test_largest_tested_lattice_fused_and_direct_agree(be):
    """1024^3 REAL, two steps.  The fused kernel (a run-time tile, with the sponge table
    read through L1 at this size) and the direct kernel share the cell arithmetic but
    none of the addressing; their states agree bit for bit.  The oracle is too slow at
    this size; both kernels are held to it bit for bit at the smaller ones."""
    import torch

    from lfm_b200 import Evolver, _lib
    from lfm_b200.config import gravity_only

    N = 1024
    g = torch.Generator(device=be.device).manual_seed(11)
    E = 0.1 * torch.randn(N**3, device=be.device, generator=g)
    chi = 19.0 + 1e-3 * torch.rand(N**3, device=be.device, generator=g)
    states = []
    try:
        for path in (_lib.PATH_FUSED, _lib.PATH_DIRECT):
            _lib.set_step_path(path)
            ev = Evolver(gravity_only(N), backend=be)
            ev.set_psi_real(E)
            ev.set_chi(chi)
            ev.evolve(2)
            if path == _lib.PATH_FUSED:
                assert _lib.tune_get(0, N) is not None
            states.append([t.clone() for t in (ev._pr[ev._cur], ev._pr[1 - ev._cur],
                                               ev._chi[ev._cur], ev._chi[1 - ev._cur])])
            del ev
            torch.cuda.empty_cache()
    finally:
        _lib.set_step_path(_lib.PATH_AUTO)
    for a, b in zip(*states):
        assert torch.equal(a, b)
    assert _lib.device_status() == 0


@pytest.mark.parametrize("N", [64, 128, 256])
def test_color_fused_default_tile_bit_exact(be, N):
    """The COLOR kernel on the planner's own tiles at larger N (two resident CTAs per
    SM where they fit, point fields from global memory, packed cell math): a few
    resident steps with every coupling but S_a against the oracle.  At 256^3 the
    tile is 2 rows x 4 stages, 256 threads."""
    from lfm_b200 import Evolver, _lib

    cfg = _parity_config("color", sa=False, N=N)
    rng = np.random.default_rng(400 + N)
    pr = (0.5 * rng.standard_normal((3, N, N, N))).astype(np.float32)
    pi = (0.5 * rng.standard_normal((3, N, N, N))).astype(np.float32)
    chi = (CHI0 + 0.01 * rng.standard_normal((N, N, N))).astype(np.float32)
    _lib.set_step_path(_lib.PATH_FUSED)
    try:
        ev = Evolver(cfg, backend=be)
        lat = O.OracleLattice(cfg)
        for t in (ev, lat):
            t.set_psi_real(pr)
            t.set_psi_imag(pi)
            t.set_chi(chi)
        ev.evolve(3)
        O.set_threads(O.max_threads())
        lat.step(3)
        used = _lib.tune_get(2, N)
        assert used["vec"] == 2 and used["tj"] >= 2, used
        if N == 256:
            assert (used["tj"], used["stages"], used["threads"]) == (2, 4, 256), used
        assert bits_equal(ev.get_psi_real().ravel(), lat.pr)
        assert bits_equal(ev.get_psi_imag().ravel(), lat.pi)
        assert bits_equal(ev.get_chi().ravel(), lat.chi)
        assert bits_equal(ev.get_psi_real_prev().ravel(), lat.prp)
    finally:
        _lib.set_step_path(_lib.PATH_AUTO)


@pytest.mark.parametrize("N,tj", [(16, 4), (32, 2), (64, 2)])
def test_color_one_cell_per_lane_bit_exact(be, N, tj):
    """The COLOR kernel with one cell per lane (a tuning option), on the streamed
    mask of the protocol step and on the resident layout's table, against the oracle."""
    from lfm_b200 import Evolver, _lib

    rng = np.random.default_rng(250 + N)
    n = N**3
    ins = rand_fields(rng, n, [(1, 0, 3)] * 4 + [(0.5, CHI0, 1)] * 2)
    mask = O.boundary_mask(N, 0.3)
    shapes = [3 * n] * 4 + [n, n]
    ref = [np.empty(s, np.float32) for s in shapes]
    O.OracleBackend().step_color(*ins, mask, *ref, N, DT2, KAPPA, LAMBDA_H, CHI0, 0.0, 0.1,
                                 CC["kappa_c"], CC["epsilon_cc"], kappa_string=CC["kappa_string"])
    _lib.set_step_path(_lib.PATH_FUSED)
    try:
        _lib.tune_set(2, N, tj, 4, 0, 1)
        d_in = [be.from_numpy(a) for a in ins]
        d_out = [be.from_numpy(np.zeros(s, np.float32)) for s in shapes]
        be.step_color(*d_in, be.from_numpy(mask), *d_out, N, DT2, KAPPA, LAMBDA_H, CHI0, 0.0,
                      0.1, CC["kappa_c"], CC["epsilon_cc"], kappa_string=CC["kappa_string"])
        assert _lib.tune_get(2, N)["vec"] == 1
        for k, (r, d) in enumerate(zip(ref, d_out)):
            assert bits_equal(be.to_numpy(d), r), f"output {k}"

        cfg = _parity_config("color", sa=False, N=N)
        E = O.parity_seed_blob(N)
        ev = Evolver(cfg, backend=be)
        lat = O.OracleLattice(cfg)
        _seed(ev, "color", E)
        _seed(lat, "color", E)
        ev.evolve(12)
        lat.step(12)
        assert _lib.tune_get(2, N)["vec"] == 1
        assert bits_equal(ev.get_psi_real().ravel(), lat.pr)
        assert bits_equal(ev.get_psi_imag().ravel(), lat.pi)
        assert bits_equal(ev.get_chi().ravel(), lat.chi)
    finally:
        _lib.tune_set(2, N, 0, 0)
        _lib.set_step_path(_lib.PATH_AUTO)


@pytest.mark.parametrize("N", [12, 16, 32])
def test_protocol_step_color_with_sa(be, N):
    """Psi outputs stay bit-exact; S_a and chi within the stated tolerances."""
    rng = np.random.default_rng(300 + N)
    n = N**3
    ins = rand_fields(rng, n, [(1, 0, 3)] * 4 + [(0.5, CHI0, 1)] * 2)
    mask = O.boundary_mask(N, 0.3)
    shapes = [3 * n] * 4 + [n, n]
    ref = [np.empty(s, np.float32) for s in shapes]
    sa_ref = np.zeros(3 * n, np.float32)
    O.OracleBackend().step_color(*ins, mask, *ref, N, DT2, KAPPA, LAMBDA_H, CHI0, 0.0, 0.1,
                                 CC["kappa_c"], CC["epsilon_cc"], kappa_string=CC["kappa_string"],
                                 kappa_tube=KT, sa_fields_in=sa_ref, sa_fields_out=sa_ref)
    d_in = [be.from_numpy(a) for a in ins]
    d_out = [be.from_numpy(np.zeros(s, np.float32)) for s in shapes]
    d_sa_in = be.from_numpy(np.zeros(3 * n, np.float32))
    d_sa = be.from_numpy(np.zeros(3 * n, np.float32))
    be.step_color(*d_in, be.from_numpy(mask), *d_out, N, DT2, KAPPA, LAMBDA_H, CHI0, 0.0, 0.1,
                  CC["kappa_c"], CC["epsilon_cc"], kappa_string=CC["kappa_string"],
                  kappa_tube=KT, sa_fields_in=d_sa_in, sa_fields_out=d_sa)
    for k in range(4):
        assert bits_equal(be.to_numpy(d_out[k]), ref[k]), f"psi output {k}"
    assert bits_equal(be.to_numpy(d_out[5]), ref[5])
    sa = be.to_numpy(d_sa)
    assert (sa >= 0).all()
    assert np.abs(sa - sa_ref).max() <= SA_REL_TOL * np.abs(sa_ref).max()
    # FP64 S_a: the float32 cuFFT path is within the same bound of it
    e64 = O.color_energy(ins[0].astype(np.float64), ins[2].astype(np.float64), N)
    sa64 = O.helmholtz_sa(e64, N, 0.1, 4.9).ravel()
    assert np.abs(sa - sa64).max() <= SA_REL_TOL * np.abs(sa64).max()
    assert np.abs(be.to_numpy(d_out[4]) - ref[4]).max() <= CHI_SA_ATOL


def test_helmholtz_dc_gain_and_smoothing(be):
    """DC preserved (reference tests/test_config_presets.py:92-114) and S_a smoother than |Psi|^2."""
    import ctypes

    import torch

    from lfm_b200 import _lib
    from lfm_b200.backend import _stream_handle

    N = 32
    rng = np.random.default_rng(9)
    pr = rng.standard_normal(3 * N**3).astype(np.float32)
    pi = rng.standard_normal(3 * N**3).astype(np.float32)
    d_pr, d_pi = be.from_numpy(pr), be.from_numpy(pi)
    sa = torch.empty(3 * N**3, dtype=torch.float32, device=be.device)
    _lib.call("lfm_helmholtz_sa_f32", be.context.handle, d_pr.data_ptr(), d_pi.data_ptr(),
              sa.data_ptr(), N, 0.1, 4.9, _stream_handle(be.device))
    s = be.to_numpy(sa).reshape(3, -1)
    e = (pr * pr + pi * pi).reshape(3, -1)
    assert np.allclose(s.mean(axis=1), e.mean(axis=1), rtol=1e-5)
    assert s.std(axis=1).max() < e.std(axis=1).min()
    del ctypes


def test_overlapping_buffers_rejected(be):
    from lfm_b200._lib import LFM_ERR_INVALID_ARG, LfmError

    N = 16
    n = N**3
    a = [be.from_numpy(np.zeros(n, np.float32)) for _ in range(8)]
    mask = be.from_numpy(O.boundary_mask(N, 0.3))
    with pytest.raises(LfmError) as e:
        be.step_real(a[0], a[1], a[2], a[3], mask, a[0], a[5], a[6], a[7], N, DT2, KAPPA, 0.0,
                     CHI0, 0.0)
    assert e.value.code == LFM_ERR_INVALID_ARG


def test_wrong_dtype_and_size_rejected(be):
    import torch

    N = 16
    n = N**3
    good = [be.from_numpy(np.zeros(n, np.float32)) for _ in range(9)]
    bad = good.copy()
    bad[0] = torch.zeros(n, dtype=torch.float64, device=be.device)
    with pytest.raises(TypeError):
        be.step_real(*bad, N, DT2, KAPPA, 0.0, CHI0, 0.0)
    bad[0] = be.from_numpy(np.zeros(n - 1, np.float32))
    with pytest.raises(ValueError):
        be.step_real(*bad, N, DT2, KAPPA, 0.0, CHI0, 0.0)


# ----------------------------------------------------------------------------
# Evolver runs against the reference fixtures
# ----------------------------------------------------------------------------
def _parity_config(level: str, sa: bool = True, N: int = 16):
    from lfm_b200.config import FieldLevel, SimulationConfig

    if level == "real":
        return SimulationConfig(grid_size=N, boundary_fraction=0.15)
    if level == "complex":
        return SimulationConfig(grid_size=N, boundary_fraction=0.15,
                                field_level=FieldLevel.COMPLEX, lambda_self=LAMBDA_H)
    return SimulationConfig(grid_size=N, boundary_fraction=0.15, field_level=FieldLevel.COLOR,
                            lambda_self=LAMBDA_H, kappa_tube=KT if sa else 0.0, **CC)


def _seed(ev, level, E):
    if level == "color":
        pr = np.zeros((3,) + E.shape, np.float32)
        pr[0] = E
        pi = np.zeros_like(pr)
        pi[1] = 0.5 * E
        ev.set_psi_real(pr)
        ev.set_psi_imag(pi)
    else:
        ev.set_psi_real(E)
        if level == "complex":
            ev.set_psi_imag(0.25 * E)


@pytest.mark.parametrize("N", [20, 24, 48, 128, 256, 512])
@pytest.mark.parametrize("level", ["real", "complex"])
def test_resident_steps_bit_exact_at_every_kernel_shape(be, N, level):
    """Resident steps against the float32 oracle at sizes that reach each kernel
    variant: run-time tiles (24, 48), the direct fallback (20 COMPLEX), and the
    compile-time tiles with packed two-cell arithmetic (128, 256, and 512, the
    throughput workload's size)."""
    from lfm_b200 import Evolver
    from lfm_b200.config import gravity_em, gravity_only

    cfg = (gravity_only if level == "real" else gravity_em)(N, boundary_fraction=0.3)
    rng = np.random.default_rng(N + (7 if level == "complex" else 0))
    E = (0.7 * rng.standard_normal((N, N, N))).astype(np.float32)
    chi = (CHI0 + 0.05 * rng.standard_normal((N, N, N))).astype(np.float32)
    ev = Evolver(cfg, backend=be)
    lat = O.OracleLattice(cfg)
    O.set_threads(O.max_threads())
    for tgt in (ev, lat):
        tgt.set_psi_real(E)
        if level == "complex":
            tgt.set_psi_imag(0.5 * E[::-1].copy())
        tgt.set_chi(chi)
    steps = 3
    ev.use_graphs = False
    ev.evolve(steps)
    lat.step(steps)
    assert bits_equal(ev.get_psi_real().ravel(), lat.pr)
    assert bits_equal(ev.get_chi().ravel(), lat.chi)
    assert bits_equal(ev.get_psi_real_prev().ravel(), lat.prp)
    if level == "complex":
        assert bits_equal(ev.get_psi_imag().ravel(), lat.pi)


@pytest.mark.parametrize("buffers", ["resident", "ab"])
@pytest.mark.parametrize("level", ["real", "complex"])
def test_evolver_fifty_steps_match_reference_bit_exact(be, path, buffers, level):
    from lfm_b200 import Evolver

    g = load_golden("parity_runs.npz")
    ev = Evolver(_parity_config(level), backend=be, buffers=buffers)
    _seed(ev, level, g["seed_E"])
    ev.evolve(50)
    assert ev.step == 50
    assert bits_equal(ev.get_psi_real(), g[f"{level}_psi_r"])
    assert bits_equal(ev.get_psi_real_prev(), g[f"{level}_psi_r_prev"])
    assert bits_equal(ev.get_chi(), g[f"{level}_chi"])
    if level == "complex":
        assert bits_equal(ev.get_psi_imag(), g[f"{level}_psi_i"])


@pytest.mark.parametrize("buffers", ["resident", "ab"])
def test_evolver_color_with_sa_matches_reference(be, buffers):
    from lfm_b200 import Evolver

    g = load_golden("parity_runs.npz")
    ev = Evolver(_parity_config("color"), backend=be, buffers=buffers)
    _seed(ev, "color", g["seed_E"])
    ev.evolve(50)
    for key, got in (("psi_r", ev.get_psi_real()), ("psi_i", ev.get_psi_imag()),
                     ("chi", ev.get_chi())):
        ref = g[f"color_{key}"]
        err = np.abs(got - ref).max() / max(np.abs(ref).max(), 1e-30)
        assert err <= 1e-5, (key, err)
    sa = ev.get_sa_fields()
    ref = g["color_sa"]
    assert np.abs(sa - ref).max() <= 1e-5 * np.abs(ref).max()


@pytest.mark.parametrize("buffers", ["resident", "ab"])
def test_evolver_color_without_sa_bit_exact(be, path, buffers):
    from lfm_b200 import Evolver

    cfg = _parity_config("color", sa=False)
    E = O.parity_seed_blob(16)
    ev = Evolver(cfg, backend=be, buffers=buffers)
    lat = O.OracleLattice(cfg)
    _seed(ev, "color", E)
    _seed(lat, "color", E)
    ev.evolve(30)
    lat.step(30)
    assert bits_equal(ev.get_psi_real().ravel(), lat.pr)
    assert bits_equal(ev.get_psi_imag().ravel(), lat.pi)
    assert bits_equal(ev.get_chi().ravel(), lat.chi)
    assert bits_equal(ev.get_psi_real_prev().ravel(), lat.prp)


def test_config1_real64_thousand_steps_bit_exact(be, path):
    """The 64^3 REAL run of 1000 steps reproduces the reference's final fields exactly."""
    from lfm_b200 import Evolver, gravity_only

    g = load_golden("config1_real64.npz")
    summary = golden_json(g["summary"])
    N = 64
    rng = np.random.default_rng(42)
    E = O.gaussian_blob(N, (32, 32, 32), 6.0, 3.0) + 1e-4 * rng.standard_normal((N,) * 3)
    E = E.astype(np.float32)
    assert sha(E) == summary["E_init_sha256"]
    ev = Evolver(gravity_only(N), backend=be)
    ev.set_psi_real(E)
    ev.evolve(1000)
    assert sha(ev.get_psi_real()) == summary["E_sha256"]
    assert sha(ev.get_psi_real_prev()) == summary["E_prev_sha256"]
    assert sha(ev.get_chi()) == summary["chi_sha256"]


def test_setters_mid_run_keep_reference_semantics(be):
    """set_psi_real_prev / set_chi_current between steps behave as the reference's buffers."""
    from lfm_b200 import Evolver
    from lfm_b200.config import FieldLevel, SimulationConfig

    cfg = SimulationConfig(grid_size=16, field_level=FieldLevel.COMPLEX, lambda_self=LAMBDA_H)
    E = O.parity_seed_blob(16)
    rng = np.random.default_rng(3)
    runs = []
    for buffers in ("resident", "ab"):
        ev = Evolver(cfg, backend=be, buffers=buffers)
        ev.set_psi_real(E)
        ev.set_psi_imag(0.1 * E)
        ev.evolve(7)
        r = np.random.default_rng(3)
        ev.set_psi_real_prev(ev.get_psi_real() + 1e-3 * r.standard_normal(E.shape))
        ev.set_chi_current(ev.get_chi() - 0.01)
        ev.evolve(5)
        runs.append((ev.get_psi_real(), ev.get_psi_imag(), ev.get_chi(), ev.get_psi_real_prev()))
    for a, b in zip(*runs):
        assert bits_equal(a, b)
    del rng


@pytest.mark.parametrize("level", ["real", "complex", "color"])
def test_graph_replay_equals_eager_steps(be, level):
    from lfm_b200 import Evolver

    cfg = _parity_config(level)
    E = O.parity_seed_blob(16)
    runs = []
    for graphs in (True, False):
        ev = Evolver(cfg, backend=be)
        ev.use_graphs = graphs
        _seed(ev, level, E)
        ev.evolve(37)
        ev.evolve(12)
        runs.append((ev.get_psi_real(), ev.get_chi(), ev.get_psi_real_prev(), ev.step))
    for a, b in zip(runs[0][:3], runs[1][:3]):
        assert bits_equal(a, b)
    assert runs[0][3] == runs[1][3] == 49


def test_freeze_chi_holds_chi(be):
    from lfm_b200 import Evolver, gravity_only

    ev = Evolver(gravity_only(16), backend=be)
    ev.set_psi_real(O.parity_seed_blob(16))
    chi0 = ev.get_chi().copy()
    ev.evolve(10, freeze_chi=True)
    assert bits_equal(ev.get_chi(), chi0)
    assert np.abs(ev.get_psi_real()).max() > 0


def test_callback_and_step_counter(be):
    from lfm_b200 import Evolver, gravity_only

    ev = Evolver(gravity_only(16, report_interval=5), backend=be)
    seen = []
    ev.evolve(12, callback=lambda e, s: seen.append(s))
    assert seen == [5, 10] and ev.step == 12


def test_known_answer_energy_density(be):
    """|Psi|^2 = 3^2 + 4^2 = 25 (reference tests/test_evolver.py:121-132)."""
    from lfm_b200 import Evolver
    from lfm_b200.config import FieldLevel, SimulationConfig

    ev = Evolver(SimulationConfig(grid_size=16, field_level=FieldLevel.COMPLEX), backend=be)
    ev.set_psi_real(np.full((16, 16, 16), 3.0, np.float32))
    ev.set_psi_imag(np.full((16, 16, 16), 4.0, np.float32))
    assert np.allclose(ev.get_energy_density(), 25.0)
    with pytest.raises(ValueError):
        Evolver(SimulationConfig(grid_size=16), backend=be).set_psi_imag(np.zeros((16,) * 3))


@pytest.mark.parametrize("level", ["real", "complex", "color"])
def test_empty_universe_stays_empty(be, level):
    """Psi = 0, chi = chi0 is a fixed point (reference tests/test_backends.py)."""
    from lfm_b200 import Evolver

    cfg = _parity_config(level)
    ev = Evolver(cfg, backend=be)
    ev.evolve(20)
    assert np.abs(ev.get_psi_real()).max() < 1e-10
    assert np.abs(ev.get_chi() - CHI0).max() < 1e-5


def test_color_rejects_two_colours(be):
    from lfm_b200 import Evolver
    from lfm_b200.config import FieldLevel, SimulationConfig

    with pytest.raises(ValueError, match="3 colours"):
        Evolver(SimulationConfig(grid_size=16, field_level=FieldLevel.COLOR, n_colors=2),
                backend=be)
