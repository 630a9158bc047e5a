"""The oracle against fixtures produced by the reference itself (tests/golden/).

Bit-exact: the float32 C restatement must reproduce the reference NumPy
backend's float32 output to the last bit, for one step at odd and even N,
for 50-step runs at every field level, and for the 1000-step 64^3 REAL run
(compared by SHA-256 of the final fields).
"""

from __future__ import annotations

import hashlib
import json

import numpy as np
import pytest

from conftest import golden_json, load_golden
from oracle import oracle as O

DT = 0.02
DT2 = DT**2
CHI0 = 19.0
KAPPA = 1.0 / 63.0
LAMBDA_H = 4.0 / 31.0
CC = dict(kappa_c=1.0 / 189.0, epsilon_cc=2.0 / 17.0, kappa_string=1.0 / 189.0)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_masks_match_reference_bit_for_bit():
    g = load_golden("masks.npz")
    for key, ref in g.items():
        if key.startswith("mask_"):
            _, N, bf = key.split("_")
            assert np.array_equal(O.boundary_mask(int(N), float(bf)), ref), key
    for key, h in json.loads(str(g["large_mask_sha256"])).items():
        N, bf = key.split("_")
        assert sha(O.boundary_mask(int(N), float(bf))) == h, key


def test_mask_known_answers():
    # tests/test_backends.py:35-57 of the reference: centre 0, corner 1, float32.
    m = O.boundary_mask(32, 0.3).reshape(32, 32, 32)
    assert m.dtype == np.float32
    assert m[16, 16, 16] == 0.0 and m[0, 0, 0] == 1.0
    assert ((m >= 0) & (m <= 1)).all()


def test_laplacian_matches_reference():
    g = load_golden("laplacian.npz")
    assert np.array_equal(O.laplacian_19pt(g["f32"]), g["lap_f32"])
    assert np.array_equal(O.laplacian_19pt(g["f64"]), g["lap_f64"])


def test_laplacian_known_answers():
    # tests/test_stencils.py of the reference: constant -> 0, x^2 -> 2 inside.
    N = 16
    c = np.full((N, N, N), 7.5)
    assert np.abs(O.laplacian_19pt(c)).max() < 1e-12
    x = np.arange(N, dtype=np.float64)
    X = np.broadcast_to(x[:, None, None] ** 2, (N, N, N)).copy()
    lap = O.laplacian_19pt(X)
    assert np.allclose(lap[2:-2, 2:-2, 2:-2], 2.0, atol=0.1)
    f = np.random.default_rng(1).standard_normal((N, N, N))
    # cubic symmetry: transposing the axes commutes with the stencil
    assert np.allclose(O.laplacian_19pt(f.transpose(1, 2, 0)),
                       O.laplacian_19pt(f).transpose(1, 2, 0), atol=1e-12)


@pytest.mark.parametrize("N", [12, 13])
def test_single_step_real_bit_exact(N):
    g = load_golden("single_step.npz")
    ins = [g[f"real{N}_in_{k}"] for k in ("E", "Ep", "chi", "chip")]
    outs = [np.empty_like(a) for a in ins]
    O.OracleBackend().step_real(*ins, O.boundary_mask(N, 0.3), *outs, N, DT2, KAPPA,
                                LAMBDA_H, CHI0, 0.0)
    for k, a in zip(("E", "Ep", "chi", "chip"), outs):
        assert np.array_equal(a, g[f"real{N}_out_{k}"]), k


@pytest.mark.parametrize("N", [12, 13])
def test_numpy_restatement_of_the_real_step_bit_exact(N):
    """numpy_step_real (the reference's CPU path as NumPy array operations, timed by
    bench.py as the single-core reference baseline) reproduces the reference's step."""
    g = load_golden("single_step.npz")
    ins = [g[f"real{N}_in_{k}"] for k in ("E", "Ep", "chi", "chip")]
    outs = O.numpy_step_real(*ins, O.boundary_mask(N, 0.3), N, DT2, KAPPA, LAMBDA_H, CHI0, 0.0)
    for k, a in zip(("E", "Ep", "chi", "chip"), outs):
        assert a.dtype == np.float32
        assert np.array_equal(a, g[f"real{N}_out_{k}"]), k


@pytest.mark.parametrize("N", [12, 13])
def test_single_step_complex_bit_exact(N):
    g = load_golden("single_step.npz")
    names = ("Pr", "Prp", "Pi", "Pip", "chi", "chip")
    ins = [g[f"complex{N}_in_{k}"] for k in names]
    outs = [np.empty_like(a) for a in ins]
    O.OracleBackend().step_complex(*ins, O.boundary_mask(N, 0.3), *outs, N, DT2, KAPPA,
                                   LAMBDA_H, CHI0, 0.01, 0.1)
    for k, a in zip(names, outs):
        assert np.array_equal(a, g[f"complex{N}_out_{k}"]), k


@pytest.mark.parametrize("N", [12, 13])
@pytest.mark.parametrize("tag,kt", [("nosa", 0.0), ("sa", 30.0 / 63.0)])
def test_single_step_color_bit_exact(N, tag, kt):
    g = load_golden("single_step.npz")
    names = ("Pr", "Prp", "Pi", "Pip", "chi", "chip")
    ins = [g[f"color{N}_in_{k}"] for k in names]
    outs = [np.empty_like(a) for a in ins]
    sa = np.zeros(3 * N**3, np.float32)
    O.OracleBackend().step_color(*ins, O.boundary_mask(N, 0.3), *outs, N, DT2, KAPPA,
                                 LAMBDA_H, CHI0, 0.0, 0.1, CC["kappa_c"], CC["epsilon_cc"],
                                 kappa_string=CC["kappa_string"], kappa_tube=kt,
                                 sa_fields_in=sa, sa_fields_out=sa)
    for k, a in zip(names, outs):
        assert np.array_equal(a, g[f"color{N}{tag}_out_{k}"]), k
    assert np.array_equal(sa, g[f"color{N}{tag}_out_sa"])


def _parity_config(level: str):
    from lfm_b200.config import FieldLevel, SimulationConfig

    if level == "real":
        return SimulationConfig(grid_size=16, boundary_fraction=0.15)
    if level == "complex":
        return SimulationConfig(grid_size=16, boundary_fraction=0.15,
                                field_level=FieldLevel.COMPLEX, lambda_self=LAMBDA_H)
    return SimulationConfig(grid_size=16, boundary_fraction=0.15, field_level=FieldLevel.COLOR,
                            lambda_self=LAMBDA_H, kappa_tube=30.0 / 63.0, **CC)


def seed_parity_lattice(lat, level: str, E: np.ndarray) -> None:
    """Initial state of the 50-step parity runs (tests/golden/make_golden.py)."""
    if level == "color":
        pr = np.zeros((3,) + E.shape, np.float32)
        pr[0] = E
        pi = np.zeros_like(pr)
        pi[1] = 0.5 * E
        lat.set_psi_real(pr)
        lat.set_psi_imag(pi)
    else:
        lat.set_psi_real(E)
        if level == "complex":
            lat.set_psi_imag(0.25 * E)


@pytest.mark.parametrize("level", ["real", "complex", "color"])
def test_fifty_step_runs_bit_exact(level):
    g = load_golden("parity_runs.npz")
    assert np.array_equal(O.parity_seed_blob(16), g["seed_E"])
    lat = O.OracleLattice(_parity_config(level))
    seed_parity_lattice(lat, level, g["seed_E"])
    lat.step(50)
    N = 16
    assert np.array_equal(lat.pr, g[f"{level}_psi_r"].ravel())
    assert np.array_equal(lat.prp, g[f"{level}_psi_r_prev"].ravel())
    assert np.array_equal(lat.chi, g[f"{level}_chi"].ravel())
    if level != "real":
        assert np.array_equal(lat.pi, g[f"{level}_psi_i"].ravel())
    if level == "color":
        assert np.array_equal(lat.sa, g[f"{level}_sa"].reshape(-1))
    assert lat.chi.size == N**3


def config1_initial_E() -> np.ndarray:
    """Config-1 initial E: soliton (6.0, sigma 3) at (32,32,32) + 1e-4 N(0,1) noise, seed 42."""
    N = 64
    rng = np.random.default_rng(42)
    E = O.gaussian_blob(N, (32, 32, 32), 6.0, 3.0) + 1e-4 * rng.standard_normal((N,) * 3)
    return E.astype(np.float32)


def test_config1_real64_thousand_steps_bit_exact():
    from lfm_b200.config import gravity_only

    g = load_golden("config1_real64.npz")
    summary = golden_json(g["summary"])
    E = config1_initial_E()
    assert sha(E) == summary["E_init_sha256"]
    O.set_threads(O.max_threads())
    lat = O.OracleLattice(gravity_only(64))
    lat.set_psi_real(E)
    lat.step(1000)
    assert sha(lat.pr.reshape(64, 64, 64)) == summary["E_sha256"]
    assert sha(lat.prp.reshape(64, 64, 64)) == summary["E_prev_sha256"]
    assert sha(lat.chi.reshape(64, 64, 64)) == summary["chi_sha256"]
