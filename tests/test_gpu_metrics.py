"""On-device float64 metrics against the reference's compute_metrics (fixture)."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_json, load_golden

pytestmark = pytest.mark.gpu

# float64 energy sums: the reduction order differs from NumPy's pairwise sum
ENERGY_RTOL = 1e-12
# chi mean/std: the reference averages float32 values with float32 pairwise sums
CHI_MOMENT_RTOL = 2e-6


@pytest.fixture(scope="module")
def be(cuda_device):
    from lfm_b200 import B200Backend
    from lfm_b200.build import build_library

    build_library()
    return B200Backend(cuda_device)


def dev(be, a):
    return be.from_numpy(np.ascontiguousarray(a, np.float32).ravel())


@pytest.mark.parametrize("level", ["real", "complex"])
def test_metrics_match_reference_fixture(be, level):
    from lfm_b200.metrics import device_metrics, interior_mask, n_clusters

    g = load_golden("metrics.npz")
    ref = golden_json(g[level])
    N = 16
    cplx = level == "complex"
    m = device_metrics(be.context.handle, 1 if cplx else 0, N, dev(be, g["pr"]), dev(be, g["prp"]),
                       dev(be, g["pi"]) if cplx else None, dev(be, g["pip"]) if cplx else None,
                       dev(be, g["chi"]), 0.02, 1.0, 0.3)
    for k in ("energy_kinetic", "energy_gradient", "energy_potential", "energy_total",
              "psi_sq_total"):
        assert m[k] == pytest.approx(ref[k], rel=ENERGY_RTOL), k
    assert m["chi_min"] == ref["chi_min"] and m["chi_max"] == ref["chi_max"]
    assert m["chi_mean"] == pytest.approx(ref["chi_mean"], rel=CHI_MOMENT_RTOL)
    assert m["chi_std"] == pytest.approx(ref["chi_std"], rel=CHI_MOMENT_RTOL)
    assert m["well_fraction"] == ref["well_fraction"]
    assert m["void_fraction"] == ref["void_fraction"]
    assert m["nonfinite_cells"] == 0
    im = interior_mask(N, 0.3)
    assert m["interior_cells"] == im.sum()
    e = g["pr"].astype(np.float64) ** 2 + (g["pi"].astype(np.float64) ** 2 if cplx else 0)
    assert n_clusters(e, im) == ref["n_clusters"]


def numpy_energy(pr, prp, pi, pip, chi, dt):
    """energy_components restated with NumPy (lfm/analysis/energy.py:26-113), colour arrays."""
    def gsq(f):
        t = np.zeros(f.shape[1:])
        for a in range(f.shape[0]):
            for ax in range(3):
                t += np.gradient(f[a].astype(np.float64), axis=ax) ** 2
        return t
    dr = (pr.astype(np.float64) - prp) / dt
    di = (pi.astype(np.float64) - pip) / dt
    T = 0.5 * np.sum(dr**2, axis=0) + 0.5 * np.sum(di**2, axis=0)
    G = 0.5 * gsq(pr) + 0.5 * gsq(pi)
    psq = np.sum(pr.astype(np.float64) ** 2, axis=0) + np.sum(pi.astype(np.float64) ** 2, axis=0)
    V = 0.5 * chi.astype(np.float64) ** 2 * psq
    return T.sum(), G.sum(), V.sum(), psq.sum()


def test_color_metrics_match_numpy_energy(be):
    from lfm_b200.metrics import device_metrics

    N = 20
    rng = np.random.default_rng(4)
    pr, prp, pi, pip = (rng.standard_normal((3, N, N, N)).astype(np.float32) for _ in range(4))
    chi = (19 + rng.standard_normal((N, N, N))).astype(np.float32)
    m = device_metrics(be.context.handle, 2, N, dev(be, pr), dev(be, prp), dev(be, pi),
                       dev(be, pip), dev(be, chi), 0.02, 1.0, 0.3)
    T, G, V, P = numpy_energy(pr, prp, pi, pip, chi, 0.02)
    assert m["energy_kinetic"] == pytest.approx(T, rel=ENERGY_RTOL)
    assert m["energy_gradient"] == pytest.approx(G, rel=ENERGY_RTOL)
    assert m["energy_potential"] == pytest.approx(V, rel=ENERGY_RTOL)
    assert m["psi_sq_total"] == pytest.approx(P, rel=ENERGY_RTOL)


def test_evolver_metrics_and_energy_drift_small(be):
    """Energy of a REAL run is conserved to well under a percent over 200 steps."""
    from lfm_b200 import Evolver, gravity_only
    from lfm_b200.workloads import config1_soliton

    ev = Evolver(gravity_only(64), backend=be)
    ev.set_psi_real(config1_soliton(64))
    ev.evolve(1)
    e0 = ev.metrics()["energy_total"]
    ev.evolve(200)
    m = ev.metrics(clusters=True)
    assert m["nonfinite_cells"] == 0 and m["n_clusters"] >= 1
    assert abs(m["energy_total"] - e0) / abs(e0) < 0.05


def test_metrics_reject_bad_arguments(be):
    from lfm_b200._lib import LfmError
    from lfm_b200.metrics import device_metrics

    chi = dev(be, np.full(8**3, 19.0))
    with pytest.raises(LfmError):
        device_metrics(be.context.handle, 1, 8, chi, None, None, None, chi, 0.02)
    with pytest.raises(LfmError):
        device_metrics(be.context.handle, 0, 8, chi, None, None, None, chi, -1.0)
