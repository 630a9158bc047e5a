"""Checkpoints in the reference's npz format: reading a file the reference
wrote, and (GPU) a resume that is bit-identical to the uninterrupted run."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN


def bits_equal(a, b) -> bool:
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_reads_a_checkpoint_the_reference_wrote():
    from lfm_b200.checkpoint import read_checkpoint
    from lfm_b200.config import FieldLevel, gravity_em

    c = read_checkpoint(GOLDEN / "ref_checkpoint.npz")
    want = gravity_em(12)
    cfg = c["config"]
    assert cfg.field_level == FieldLevel.COMPLEX and cfg.grid_size == 12
    for k in ("chi0", "kappa", "lambda_self", "epsilon_w", "dt", "boundary_fraction"):
        assert getattr(cfg, k) == getattr(want, k), k
    assert c["step"] == 4 and not c["exact"]
    assert c["psi_real"].shape == (12, 12, 12) and c["psi_imag"].shape == (12, 12, 12)
    assert c["history"] == []


def test_config_round_trips_through_json():
    from lfm_b200.checkpoint import config_from_json, config_to_json
    from lfm_b200.config import full_physics

    cfg = full_physics(24, kappa=0.02, boundary_fraction=0.2)
    back = config_from_json(config_to_json(cfg))
    assert vars(back) == vars(cfg)


# ---------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def be(cuda_device):
    from lfm_b200 import B200Backend, _lib
    from lfm_b200.build import build_library

    build_library()
    _lib.set_step_path(_lib.PATH_AUTO)
    return B200Backend(cuda_device)


def _start(be, level):
    from lfm_b200 import Evolver
    from lfm_b200.config import full_physics, gravity_em, gravity_only

    N = 16
    rng = np.random.default_rng(4)
    E = (0.6 * rng.standard_normal((N, N, N))).astype(np.float32)
    cfg = {"real": gravity_only, "complex": gravity_em, "color": full_physics}[level](N)
    ev = Evolver(cfg, backend=be)
    if level == "color":
        pr = np.stack([E, 0.5 * E, -E]).astype(np.float32)
        ev.set_psi_real(pr)
        ev.set_psi_imag(0.3 * pr[::-1].copy())
    else:
        ev.set_psi_real(E)
        if level == "complex":
            ev.set_psi_imag(0.5 * E[::-1].copy())
    ev.set_chi((19.0 + 0.01 * rng.standard_normal((N, N, N))).astype(np.float32))
    return ev


@pytest.mark.gpu
@pytest.mark.parametrize("level", ["real", "complex", "color"])
def test_resume_is_bit_identical(be, tmp_path, level):
    from lfm_b200 import Evolver

    ev = _start(be, level)
    ev.evolve(6)
    path = tmp_path / "ck.npz"
    ev.save_checkpoint(path, history=[{"step": 6.0}])
    back = Evolver.load_checkpoint(path, backend=be)
    assert back.step == 6
    ev.evolve(7)
    back.evolve(7)
    assert bits_equal(back.get_psi_real(), ev.get_psi_real())
    assert bits_equal(back.get_psi_real_prev(), ev.get_psi_real_prev())
    assert bits_equal(back.get_chi(), ev.get_chi())
    assert bits_equal(back.get_chi_prev(), ev.get_chi_prev())
    if level != "real":
        assert bits_equal(back.get_psi_imag(), ev.get_psi_imag())


@pytest.mark.gpu
def test_reference_file_loads_with_prev_equal_to_current(be):
    from lfm_b200.checkpoint import load_checkpoint

    ev, c = load_checkpoint(GOLDEN / "ref_checkpoint.npz", backend=be)
    assert ev.step == 4
    assert bits_equal(ev.get_psi_real(), c["psi_real"])
    assert bits_equal(ev.get_psi_real_prev(), c["psi_real"])
    assert bits_equal(ev.get_chi(), c["chi"])
    assert bits_equal(ev.get_chi_prev(), c["chi"])
    ev.evolve(3)
    assert np.isfinite(ev.get_chi()).all()
