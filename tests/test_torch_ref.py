"""The float64 torch transcription of the reference step (oracle/torch_ref.py),
which serves as the FP64 oracle on the GPU for lattices too large for the C
oracle, against the C oracle's float64 instantiation (CPU)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import torch_ref as TR


def _state(cfg, seed):
    N = cfg.grid_size
    rng = np.random.default_rng(seed)
    n_psi = 3 if int(cfg.field_level) == 2 else 1
    shape = (n_psi, N, N, N) if n_psi == 3 else (N, N, N)
    pr = 0.6 * rng.standard_normal(shape)
    pi = 0.6 * rng.standard_normal(shape) if int(cfg.field_level) else None
    chi = 19.0 + 0.05 * rng.standard_normal((N, N, N))
    return pr, pi, chi


@pytest.mark.parametrize("preset", ["gravity_only", "gravity_em", "full_physics"])
def test_torch_float64_step_matches_the_c_oracle(preset):
    from lfm_b200 import config as C

    cfg = getattr(C, preset)(12)
    N = cfg.grid_size
    pr, pi, chi = _state(cfg, 4)
    lat = O.OracleLattice(cfg, dtype=np.float64)
    lat.set_psi_real(pr)
    if pi is not None:
        lat.set_psi_imag(pi)
    lat.set_chi(chi)
    steps = 4
    lat.step(steps)

    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float64))  # noqa: E731
    s = {"pr": t(pr), "prp": t(pr), "chi": t(chi), "chip": t(chi)}
    if pi is not None:
        s["pi"], s["pip"] = t(pi), t(pi)
    mask = torch.from_numpy(O.boundary_mask(N, cfg.boundary_fraction).astype(np.float64))
    out = TR.run(cfg, s, steps, mask.view(N, N, N))

    def rel(a, b):
        b = np.asarray(b).ravel()
        return float(np.abs(a.numpy().ravel() - b).max() / np.abs(b).max())

    assert rel(out["pr"], lat.pr) < 1e-12
    assert rel(out["prp"], lat.prp) < 1e-12
    assert rel(out["chi"], lat.chi) < 1e-12
    if pi is not None:
        assert rel(out["pi"], lat.pi) < 1e-12
    if int(cfg.field_level) == 2 and cfg.kappa_tube > 0:
        assert rel(out["sa"], lat.sa) < 1e-12
