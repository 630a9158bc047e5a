"""The split S_a transform (2-D cuFFT over (j, k) + one fused pass along i).

For power-of-two N the S_a solve (numpy_backend.py:341-356) runs as a 2-D R2C
per plane, the hand-written pass along i (forward FFT, filter, inverse FFT,
csrc/spectral.cu) and a 2-D C2R.  It is checked against the float64 oracle
(NumPy's FFT in float64) and against the 3-D cuFFT path, within the S_a
tolerance the other COLOR tests state (2e-6 of max |S_a|), and the COLOR step
that uses it against the oracle's step.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

SA_REL_TOL = 2e-6


@pytest.fixture(scope="module")
def be(cuda_device):
    from lfm_b200 import B200Backend
    from lfm_b200.build import build_library

    build_library()
    return B200Backend(cuda_device)


def _sa(be, pr, pi, N, mode, gamma=0.1, d=4.9):
    import torch

    from lfm_b200 import _lib
    from lfm_b200.backend import _stream_handle

    _lib.call("lfm_set_sa_transform", mode)
    try:
        d_pr, d_pi = be.from_numpy(pr), be.from_numpy(pi)
        sa = torch.empty(3 * N**3, dtype=torch.float32, device=be.device)
        _lib.call("lfm_helmholtz_sa_f32", be.context.handle, d_pr.data_ptr(), d_pi.data_ptr(),
                  sa.data_ptr(), N, gamma, d, _stream_handle(be.device))
        return np.maximum(be.to_numpy(sa), 0.0).reshape(3, -1)
    finally:
        _lib.call("lfm_set_sa_transform", 1)


def _packets(N, seed):
    rng = np.random.default_rng(seed)
    x = np.arange(N, dtype=np.float64)
    pr = np.zeros((3, N, N, N))
    pi = np.zeros((3, N, N, N))
    for _ in range(3):
        c = rng.uniform(0.3 * N, 0.7 * N, 3)
        s = rng.uniform(2.0, 5.0)
        g = np.exp(-(((x - c[0]) ** 2)[:, None, None] + ((x - c[1]) ** 2)[None, :, None]
                     + ((x - c[2]) ** 2)[None, None, :]) / (2 * s * s))
        th = rng.uniform(0, 2 * np.pi, 3)
        for a in range(3):
            pr[a] += 3.0 * g * np.cos(th[a])
            pi[a] += 3.0 * g * np.sin(th[a])
    pr += 0.05 * rng.standard_normal(pr.shape)
    pi += 0.05 * rng.standard_normal(pi.shape)
    return pr.astype(np.float32).ravel(), pi.astype(np.float32).ravel()


@pytest.mark.parametrize("N", [64, 128, 256])
def test_split_transform_matches_float64_and_the_3d_path(be, N):
    pr, pi = _packets(N, N)
    split = _sa(be, pr, pi, N, 1)
    full = _sa(be, pr, pi, N, 0)
    e64 = O.color_energy(pr.astype(np.float64), pi.astype(np.float64), N)
    ref = O.helmholtz_sa(e64, N, 0.1, 4.9)
    scale = np.abs(ref).max()
    err_split = np.abs(split - ref).max() / scale
    err_full = np.abs(full - ref).max() / scale
    print(N, "split", err_split, "3-D", err_full)
    assert err_split <= SA_REL_TOL and err_full <= SA_REL_TOL, (err_split, err_full)
    assert np.abs(split - full).max() <= SA_REL_TOL * scale


def test_other_filter_parameters_get_their_own_table(be):
    N = 64
    pr, pi = _packets(N, 5)
    e64 = O.color_energy(pr.astype(np.float64), pi.astype(np.float64), N)
    for gamma, d in ((0.1, 4.9), (0.3, 1.5), (0.1, 4.9)):
        got = _sa(be, pr, pi, N, 1, gamma, d)
        ref = O.helmholtz_sa(e64, N, gamma, d)
        assert np.abs(got - ref).max() <= SA_REL_TOL * np.abs(ref).max(), (gamma, d)


def test_color_evolver_64_with_split_transform_against_oracle(be):
    """The resident COLOR Evolver at 64^3 with S_a every step (split transform) stays within
    the COLOR tolerance of the oracle's float32 steps (NumPy S_a) over 20 steps."""
    from lfm_b200 import Evolver
    from lfm_b200.config import full_physics

    N = 64
    cfg = full_physics(N)
    pr, pi = _packets(N, 3)
    ev = Evolver(cfg, backend=be)
    ev.set_psi_real(pr.reshape(3, N, N, N))
    ev.set_psi_imag(pi.reshape(3, N, N, N))
    ev.evolve(20)
    lat = O.OracleLattice(cfg)
    lat.set_psi_real(pr)
    lat.set_psi_imag(pi)
    O.set_threads(O.max_threads())
    lat.step(20)
    for got, want in ((ev.get_psi_real().ravel(), lat.pr), (ev.get_psi_imag().ravel(), lat.pi),
                      (ev.get_chi().ravel(), lat.chi)):
        err = np.abs(got.astype(np.float64) - want).max() / np.abs(want).max()
        assert err < 1e-5, err


@pytest.mark.parametrize("N", [32, 64])
def test_energy_from_the_step_epilogue_equals_a_fresh_energy_pass(be, N):
    """A step writes |Psi_a|^2 of its new fields and the next S_a solve starts from it
    (lfm_leapfrog_color_energy_f32 + lfm_helmholtz_sa_from_energy_f32): the same bits as
    forming |Psi_a|^2 from Psi before every solve (the separate energy pass)."""
    from lfm_b200 import Evolver
    from lfm_b200.config import full_physics

    cfg = full_physics(N)
    pr, pi = _packets(N, 11)
    runs = []
    for reuse in (True, False):
        ev = Evolver(cfg, backend=be)
        ev.set_psi_real(pr.reshape(3, N, N, N))
        ev.set_psi_imag(pi.reshape(3, N, N, N))
        if reuse:
            ev.evolve(13)  # graphs of two steps, energy handed from step to step
        else:
            ev.use_graphs = False
            for _ in range(13):
                ev._energy_ok = False  # form |Psi_a|^2 from Psi before each solve
                ev.evolve(1)
        runs.append((ev.get_psi_real(), ev.get_psi_imag(), ev.get_chi(), ev.get_sa_fields()))
    for a, b in zip(*runs):
        assert np.array_equal(np.ascontiguousarray(a).view(np.uint32),
                              np.ascontiguousarray(b).view(np.uint32))


def test_psi_writes_invalidate_the_handed_energy(be):
    """After set_psi_real / set_psi_imag_current between steps, the next solve forms
    |Psi_a|^2 from the new Psi (the oracle agrees within the COLOR tolerance)."""
    from lfm_b200 import Evolver
    from lfm_b200.config import full_physics

    N = 32
    cfg = full_physics(N)
    pr, pi = _packets(N, 12)
    ev = Evolver(cfg, backend=be)
    ev.set_psi_real(pr.reshape(3, N, N, N))
    ev.set_psi_imag(pi.reshape(3, N, N, N))
    ev.evolve(6)
    new_i = (1.1 * ev.get_psi_imag()).astype(np.float32)
    ev.set_psi_imag_current(new_i)
    ev.evolve(6)
    lat = O.OracleLattice(cfg)
    lat.set_psi_real(pr)
    lat.set_psi_imag(pi)
    lat.step(6)
    lat.pi[:] = new_i.ravel()
    lat.step(6)
    for got, want in ((ev.get_psi_real().ravel(), lat.pr), (ev.get_chi().ravel(), lat.chi)):
        err = np.abs(got.astype(np.float64) - want).max() / np.abs(want).max()
        assert err < 1e-5, err
