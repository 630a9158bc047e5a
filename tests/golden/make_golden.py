"""Generate the golden fixtures in this folder by running the reference itself.

Run in a checkout that has the reference package importable, e.g.::

    PYTHONPATH=<reference checkout> PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py

Every array here comes from the reference's own code: ``NumpyBackend``
(lfm/core/backends/numpy_backend.py), ``laplacian_19pt``
(lfm/core/stencils.py), ``Evolver`` (lfm/core/evolver.py),
``compute_metrics`` / ``interior_mask`` (lfm/analysis/), ``gaussian_soliton``
(lfm/fields/soliton.py), ``equilibrate_from_fields``
(lfm/fields/equilibrium.py) and ``sweep`` / ``sweep_2d`` (lfm/sweep.py).  The tests compare the oracle
and the CUDA path with these files; the reference is never needed at test
time.
"""

from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np

from lfm.analysis.metrics import compute_metrics
from lfm.analysis.structure import interior_mask
from lfm.config_presets import gravity_only
from lfm.core.backends.numpy_backend import NumpyBackend
from lfm.core.evolver import Evolver
from lfm.core.stencils import laplacian_19pt
from lfm.fields.soliton import gaussian_soliton

OUT = Path(__file__).resolve().parent
DT = 0.02
DT2 = DT**2
CHI0 = 19.0
KAPPA = 1.0 / 63.0
LAMBDA_H = 4.0 / 31.0
COLOR_COUPLINGS = dict(kappa_c=1.0 / 189.0, epsilon_cc=2.0 / 17.0,
                       kappa_string=1.0 / 189.0, kappa_tube=30.0 / 63.0)


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def masks() -> None:
    be = NumpyBackend()
    data = {}
    for N, bf in ((8, 0.3), (13, 0.3), (16, 0.15), (16, 0.3), (32, 0.3), (33, 0.5)):
        data[f"mask_{N}_{bf}"] = be.create_boundary_mask(N, bf)
    hashes = {f"{N}_{bf}": sha(be.create_boundary_mask(N, bf))
              for N, bf in ((64, 0.3), (96, 0.3), (128, 0.3), (256, 0.3))}
    data["large_mask_sha256"] = np.array(json.dumps(hashes))
    for N, bf in ((16, 0.3), (32, 0.3)):
        data[f"interior_{N}_{bf}"] = interior_mask(N, bf)
    np.savez_compressed(OUT / "masks.npz", **data)


def stencil() -> None:
    rng = np.random.default_rng(7)
    f32 = rng.standard_normal((12, 12, 12)).astype(np.float32)
    f64 = rng.standard_normal((13, 13, 13))
    np.savez_compressed(OUT / "laplacian.npz", f32=f32, lap_f32=laplacian_19pt(f32),
                        f64=f64, lap_f64=laplacian_19pt(f64))


def single_steps() -> None:
    """One step of each level on seeded random states, N = 12 and 13."""
    be = NumpyBackend()
    rng = np.random.default_rng(11)
    data = {}
    for N in (12, 13):
        n = N**3
        mask = be.create_boundary_mask(N, 0.3)

        def f(scale=1.0, off=0.0, m=1):
            return (off + scale * rng.standard_normal(m * n)).astype(np.float32)

        ins = [f(), f(), f(0.5, CHI0), f(0.5, CHI0)]
        outs = [np.empty(n, np.float32) for _ in range(4)]
        be.step_real(*ins, mask, *outs, N, DT2, KAPPA, LAMBDA_H, CHI0, 0.0)
        for name, a in zip(("E", "Ep", "chi", "chip"), ins):
            data[f"real{N}_in_{name}"] = a
        for name, a in zip(("E", "Ep", "chi", "chip"), outs):
            data[f"real{N}_out_{name}"] = a

        ins = [f(), f(), f(), f(), f(0.5, CHI0), f(0.5, CHI0)]
        outs = [np.empty(n, np.float32) for _ in range(6)]
        be.step_complex(*ins, mask, *outs, N, DT2, KAPPA, LAMBDA_H, CHI0, 0.01, 0.1)
        names = ("Pr", "Prp", "Pi", "Pip", "chi", "chip")
        for name, a in zip(names, ins):
            data[f"complex{N}_in_{name}"] = a
        for name, a in zip(names, outs):
            data[f"complex{N}_out_{name}"] = a

        ins = [f(m=3), f(m=3), f(m=3), f(m=3), f(0.5, CHI0), f(0.5, CHI0)]
        for tag, kt in (("nosa", 0.0), ("sa", COLOR_COUPLINGS["kappa_tube"])):
            shapes = [3 * n] * 4 + [n, n]
            outs = [np.empty(s, np.float32) for s in shapes]
            sa = np.zeros(3 * n, np.float32)
            cc = dict(COLOR_COUPLINGS, kappa_tube=kt)
            be.step_color(*ins, mask, *outs, N, DT2, KAPPA, LAMBDA_H, CHI0, 0.0, 0.1,
                          cc["kappa_c"], cc["epsilon_cc"], kappa_string=cc["kappa_string"],
                          kappa_tube=kt, sa_fields_in=sa, sa_fields_out=sa, sa_gamma=0.1,
                          sa_d=4.9, dt=DT)
            for name, a in zip(names, outs):
                data[f"color{N}{tag}_out_{name}"] = a
            data[f"color{N}{tag}_out_sa"] = sa
        for name, a in zip(names, ins):
            data[f"color{N}_in_{name}"] = a
    np.savez_compressed(OUT / "single_step.npz", **data)


def parity_runs() -> None:
    """50 steps at N=16 from the blob seed of tests/test_gpu_parity.py:49-60 (bf=0.15)."""
    N, bf, steps = 16, 0.15, 50
    E = np.zeros((N, N, N), np.float32)
    c = N // 2
    for di in range(-2, 3):
        for dj in range(-2, 3):
            for dk in range(-2, 3):
                E[c + di, c + dj, c + dk] = 3.0 * np.exp(-(di * di + dj * dj + dk * dk) / 2.0)
    data = {"seed_E": E}
    from lfm.config import FieldLevel, SimulationConfig

    levels = (
        ("real", FieldLevel.REAL, {}),
        ("complex", FieldLevel.COMPLEX, dict(lambda_self=LAMBDA_H)),
        ("color", FieldLevel.COLOR, dict(lambda_self=LAMBDA_H, **COLOR_COUPLINGS)),
    )
    for tag, level, extra in levels:
        cfg = SimulationConfig(grid_size=N, field_level=level, boundary_fraction=bf, **extra)
        ev = Evolver(cfg, backend="cpu")
        if level == FieldLevel.COLOR:
            pr = np.zeros((3, N, N, N), np.float32)
            pr[0] = E
            pi = np.zeros_like(pr)
            pi[1] = 0.5 * E
            ev.set_psi_real(pr)
            ev.set_psi_imag(pi)
        else:
            ev.set_psi_real(E)
            if level == FieldLevel.COMPLEX:
                ev.set_psi_imag(0.25 * E)
        ev.evolve(steps)
        data[f"{tag}_psi_r"] = ev.get_psi_real()
        data[f"{tag}_psi_r_prev"] = ev.get_psi_real_prev()
        data[f"{tag}_chi"] = ev.get_chi()
        if level != FieldLevel.REAL:
            data[f"{tag}_psi_i"] = ev.get_psi_imag()
        if level == FieldLevel.COLOR:
            data[f"{tag}_sa"] = ev.get_sa_fields()
    np.savez_compressed(OUT / "parity_runs.npz", **data)


def config1() -> None:
    """REAL 64^3, gravity_only, soliton (6.0, sigma 3) at the centre + 1e-4 noise, 1000 steps.

    The state is set through Evolver.set_psi_real, so Simulation.run's
    auto-equilibrate is bypassed and chi starts flat at chi0.
    """
    N, steps = 64, 1000
    cfg = gravity_only(N)
    rng = np.random.default_rng(42)
    E = gaussian_soliton(N, (32, 32, 32), 6.0, 3.0)[0] + 1e-4 * rng.standard_normal((N,) * 3)
    ev = Evolver(cfg, backend="cpu")
    ev.set_psi_real(E)
    e0 = ev.get_psi_real().copy()
    ev.evolve(steps)
    E1 = ev.get_psi_real()
    Ep1 = ev.get_psi_real_prev()
    chi1 = ev.get_chi()
    m = compute_metrics(E1, Ep1, chi1, DT, interior_mask=interior_mask(N, cfg.boundary_fraction))
    summary = {
        "E_init_sha256": sha(e0),
        "E_sha256": sha(E1),
        "E_prev_sha256": sha(Ep1),
        "chi_sha256": sha(chi1),
        "metrics": m,
    }
    np.savez_compressed(OUT / "config1_real64.npz", summary=np.array(json.dumps(summary)),
                        E_mid=E1[32], chi_mid=chi1[32])


def metrics_fixture() -> None:
    """compute_metrics on a small COMPLEX state, for the on-device reductions."""
    N = 16
    rng = np.random.default_rng(5)
    pr = rng.standard_normal((N, N, N)).astype(np.float32)
    prp = (pr + 0.01 * rng.standard_normal((N, N, N))).astype(np.float32)
    pi = rng.standard_normal((N, N, N)).astype(np.float32)
    pip = (pi + 0.01 * rng.standard_normal((N, N, N))).astype(np.float32)
    chi = (18.0 + 2.0 * rng.standard_normal((N, N, N))).astype(np.float32)
    im = interior_mask(N, 0.3)
    m_real = compute_metrics(pr, prp, chi, DT, interior_mask=im)
    m_cplx = compute_metrics(pr, prp, chi, DT, psi_i=pi, psi_i_prev=pip, interior_mask=im)
    np.savez_compressed(OUT / "metrics.npz", pr=pr, prp=prp, pi=pi, pip=pip, chi=chi,
                        real=np.array(json.dumps(m_real)), complex=np.array(json.dumps(m_cplx)))


def equilibrium_fixture() -> None:
    """gaussian_soliton and the Poisson equilibration (lfm/fields/equilibrium.py)."""
    from lfm.fields.equilibrium import equilibrate_from_fields

    data = {}
    for N, bf in ((16, 0.3), (20, 0.15), (24, 0.3)):
        pr1, pi1 = gaussian_soliton(N, (N / 2, N / 2 - 2.5, N / 2 + 1.0), 5.0, 2.0, 0.7)
        pr2, pi2 = gaussian_soliton(N, (N / 2 - 3.0, N / 2 + 3.0, N / 2), 3.0, 1.5, 2.0)
        pr, pi = (pr1 + pr2).astype(np.float32), (pi1 + pi2).astype(np.float32)
        bmask = ~interior_mask(N, bf)
        data[f"pr_{N}"], data[f"pi_{N}"] = pr, pi
        data[f"soliton1_{N}"] = pr1
        data[f"chi_real_{N}"] = equilibrate_from_fields(pr, None, CHI0, KAPPA, 0.0, bmask)
        data[f"chi_complex_{N}"] = equilibrate_from_fields(pr, pi, CHI0, KAPPA, 0.0, bmask)
        data[f"chi_free_{N}"] = equilibrate_from_fields(pr, pi, CHI0, 2 * KAPPA, 0.5, None)
        col_r = np.stack([pr, 0.5 * pr, pi]).astype(np.float32)
        col_i = np.stack([pi, pr, 0.25 * pi]).astype(np.float32)
        data[f"colr_{N}"], data[f"coli_{N}"] = col_r, col_i
        data[f"chi_color_{N}"] = equilibrate_from_fields(col_r, col_i, CHI0, KAPPA, 0.0, bmask)
        data[f"bf_{N}"] = np.float64(bf)
    np.savez_compressed(OUT / "equilibrium.npz", **data)


def sweep_fixture() -> None:
    """lfm.sweep on small lattices (Simulation on the NumPy backend)."""
    from lfm.config_presets import gravity_em
    from lfm.sweep import sweep, sweep_2d

    runs = {
        "kappa_real": sweep(gravity_only(16), "kappa", [1.0 / 63.0, 2.0 / 63.0], 12,
                            soliton={"amplitude": 4.0, "sigma": 2.0}),
        "grid_complex": sweep(gravity_em(16), "grid_size", [16, 20], 10,
                              soliton={"amplitude": 3.0, "sigma": 2.0, "phase": 0.5}),
        "plain_noeq": sweep(gravity_only(16), "chi0", [19.0, 18.0], 6, equilibrate=False),
        "two_d": sweep_2d(gravity_em(12), "kappa", [1.0 / 63.0, 3.0 / 63.0], "epsilon_w",
                          [0.1, 0.2], 8, metric_names=["chi_min", "energy_total"],
                          soliton={"amplitude": 2.0, "sigma": 1.5}),
    }
    np.savez_compressed(OUT / "sweep.npz", runs=np.array(json.dumps(runs)))


def checkpoint_fixture() -> None:
    """A checkpoint written by the reference's Simulation (NumPy backend)."""
    from lfm.config_presets import gravity_em
    from lfm.simulation import Simulation

    sim = Simulation(gravity_em(12), backend="cpu")
    sim.place_soliton((6, 5, 6), amplitude=3.0, sigma=1.5, phase=0.4)
    sim.equilibrate()
    sim.run(steps=4, record_metrics=False)
    sim.save_checkpoint(OUT / "ref_checkpoint.npz")


HOOK_STEPS = 40
HOOK_N = 16


def hook_initial(level: str):
    """The seeded initial Psi of the hooks fixture (also rebuilt by the tests)."""
    rng = np.random.default_rng(7 if level == "real" else 8)
    pr = (0.2 * rng.standard_normal((HOOK_N,) * 3)).astype(np.float32)
    pi = (0.2 * rng.standard_normal((HOOK_N,) * 3)).astype(np.float32) if level == "complex" else None
    return pr, pi


def hooks_fixture() -> None:
    """The reference's experiment hooks (Barrier with a which-path detector slit,
    ContinuousSource, DetectorScreen) driving its Evolver for HOOK_STEPS steps,
    the callbacks in the order of lfm/experiment/source.py's example."""
    from lfm.config import FieldLevel, SimulationConfig
    from lfm.experiment.barrier import Barrier, Slit
    from lfm.experiment.detector import DetectorScreen
    from lfm.experiment.source import ContinuousSource
    from lfm.simulation import Simulation

    data = {}
    for level, fl in (("real", FieldLevel.REAL), ("complex", FieldLevel.COMPLEX)):
        cfg = SimulationConfig(grid_size=HOOK_N, field_level=fl, report_interval=1)
        sim = Simulation(cfg, backend="cpu")
        pr, pi = hook_initial(level)
        sim.set_psi_real(pr)
        if pi is not None:
            sim.set_psi_imag(pi)
        slits = [Slit(center=5, width=3),
                 Slit(center=11, width=3, detector=True, detector_strength=0.5)]
        barrier = Barrier(sim, axis=2, position=HOOK_N // 2, thickness=2, slits=slits)
        source = ContinuousSource(sim, axis=2, position=3, omega=19.05, amplitude=2.0,
                                  envelope_sigma=0.25, phase=0.7, boost=10.0)
        screen = DetectorScreen(sim, axis=2, position=12)

        def cb(ev, step, sim=sim, barrier=barrier, source=source, screen=screen):
            source.step_callback(sim, step)
            barrier.step_callback(sim, step)
            screen.record()

        sim._evolver.evolve(HOOK_STEPS, callback=cb)
        data[f"{level}_psi_real"] = sim.psi_real
        if pi is not None:
            data[f"{level}_psi_imag"] = sim.psi_imag
        data[f"{level}_chi"] = sim.chi
        data[f"{level}_frames"] = screen.snapshots
        data[f"{level}_pattern"] = screen.pattern
        data[f"{level}_barrier_mask"] = barrier.mask
        data[f"{level}_slit_masks"] = np.stack(barrier.slit_masks)
        data[f"{level}_envelope"] = source._envelope
    np.savez_compressed(OUT / "hooks.npz", **data)


if __name__ == "__main__":
    import sys

    every = [masks, stencil, single_steps, parity_runs, metrics_fixture, config1,
             equilibrium_fixture, sweep_fixture, checkpoint_fixture, hooks_fixture]
    chosen = [f for f in every if f.__name__ in sys.argv[1:]] or every
    for f in chosen:
        f()
    print("fixtures written to", OUT)
