"""Per-step device hooks (lfm_b200.hooks) against the reference's own
Barrier / ContinuousSource / DetectorScreen run (tests/golden/hooks.npz, made
by tests/golden/make_golden.py:hooks_fixture)."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden

N = 16
STEPS = 40


def initial(level: str):
    """The fixture's seeded initial Psi (make_golden.py:hook_initial)."""
    rng = np.random.default_rng(7 if level == "real" else 8)
    pr = (0.2 * rng.standard_normal((N,) * 3)).astype(np.float32)
    pi = (0.2 * rng.standard_normal((N,) * 3)).astype(np.float32) if level == "complex" else None
    return pr, pi


def slits():
    from lfm_b200.hooks import Slit

    return [Slit(center=5, width=3), Slit(center=11, width=3, detector=True,
                                          detector_strength=0.5)]


# ---------------------------------------------------------------- host only
def test_barrier_geometry_matches_reference():
    from lfm_b200.hooks import barrier_geometry

    g = load_golden("hooks.npz")
    _, _, solid, masks = barrier_geometry(N, 2, N // 2, 2, slits(), 0)
    for level in ("real", "complex"):
        assert np.array_equal(solid, g[f"{level}_barrier_mask"])
        assert np.array_equal(np.stack(masks), g[f"{level}_slit_masks"])


def test_default_slits_and_cell_resolution():
    from lfm_b200.hooks import default_slits, resolve_cell, resolve_width

    s = default_slits(64)
    assert [(x.center, x.width) for x in s] == [(24, 2), (40, 2)]
    assert resolve_cell(0.25, 64) == 16 and resolve_cell(3, 64) == 3 and resolve_cell(99, 64) == 63
    assert resolve_width(0.25, 64) == 16.0 and resolve_width(5, 64) == 5.0


def test_source_envelope_matches_reference():
    from lfm_b200.hooks import source_envelope

    g = load_golden("hooks.npz")
    e = source_envelope(N, 0.25)
    for level in ("real", "complex"):
        assert np.array_equal(e.view(np.uint32), g[f"{level}_envelope"].view(np.uint32))


def test_pattern_is_the_sequential_float32_sum_of_frames():
    """The device screen keeps a running float32 sum: the reference's np.sum
    over the frame axis adds the frames in order."""
    g = load_golden("hooks.npz")
    for level in ("real", "complex"):
        acc = np.zeros((N, N), np.float32)
        for f in g[f"{level}_frames"]:
            acc += f
        assert np.array_equal(acc.view(np.uint32), g[f"{level}_pattern"].view(np.uint32))


# ---------------------------------------------------------------- GPU
def run_hooks(level: str, buffers: str, graphs: bool, block: int = 8):
    from lfm_b200 import Evolver
    from lfm_b200.config import FieldLevel, SimulationConfig
    from lfm_b200.hooks import Barrier, ContinuousSource, DetectorScreen

    fl = FieldLevel.REAL if level == "real" else FieldLevel.COMPLEX
    ev = Evolver(SimulationConfig(grid_size=N, field_level=fl, report_interval=1),
                 buffers=buffers)
    ev.use_graphs = graphs
    ev.hook_block = block
    pr, pi = initial(level)
    ev.set_psi_real(pr)
    if pi is not None:
        ev.set_psi_imag(pi)
    barrier = Barrier(ev, axis=2, position=N // 2, thickness=2, slits=slits())
    source = ContinuousSource(ev, axis=2, position=3, omega=19.05, amplitude=2.0,
                              envelope_sigma=0.25, phase=0.7, boost=10.0)
    screen = DetectorScreen(ev, axis=2, position=12)
    ev.evolve(STEPS, hooks=[source, barrier, screen])
    return ev, screen


def same(a, b) -> bool:
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32),
                          np.asarray(b, np.float32).view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("level", ["real", "complex"])
@pytest.mark.parametrize("buffers, graphs, block", [("resident", False, 8),
                                                    ("resident", True, 8),
                                                    ("resident", True, 32),
                                                    ("ab", False, 8)])
def test_hooks_run_bit_identical_to_reference(level, buffers, graphs, block):
    g = load_golden("hooks.npz")
    ev, screen = run_hooks(level, buffers, graphs, block)
    assert ev.step == STEPS
    assert same(ev.get_psi_real(), g[f"{level}_psi_real"])
    if level == "complex":
        assert same(ev.get_psi_imag(), g[f"{level}_psi_imag"])
    assert same(ev.get_chi(), g[f"{level}_chi"])
    assert screen.n_frames == STEPS
    assert same(screen.snapshots, g[f"{level}_frames"])
    assert same(screen.pattern, g[f"{level}_pattern"])


@pytest.mark.gpu
def test_hooks_reject_color_and_screen_helpers():
    from lfm_b200 import Evolver
    from lfm_b200.config import full_physics
    from lfm_b200.hooks import DetectorScreen

    with pytest.raises(ValueError):
        DetectorScreen(Evolver(full_physics(8)))
    ev, screen = run_hooks("real", "resident", True, 8)
    pat = screen.pattern
    assert np.allclose(screen.mean_pattern(), pat / STEPS)
    assert screen.line_profile(0).shape == (N,)
    clicks = screen.click_pattern(500, seed=1)
    assert clicks.sum() == 500 and (clicks[pat == 0] == 0).all()
    screen.reset()
    assert screen.n_frames == 0 and not screen.pattern.any()
