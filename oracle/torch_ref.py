"""Plain PyTorch transcription of the reference step.  TEST INFRASTRUCTURE ONLY.

Restates lfm/core/backends/numpy_backend.py:80-205 (REAL and COMPLEX) and the
19-point Laplacian of lfm/core/stencils.py:26-71 with out-of-place torch
operations, in whatever dtype the inputs carry.  In float64 it serves as:
  * the FP64 oracle on the GPU for lattices too large for the C oracle
    (error reports of the float32 and compensated paths);
  * the autograd reference for the hand-written adjoint (every operation is
    differentiable; the clamp is torch.clamp_min).
Only tests and accuracy checks use it; the product never imports it.
"""

from __future__ import annotations

import torch

FACE_W = 1.0 / 3.0
EDGE_W = 1.0 / 6.0


def laplacian_19pt(f: torch.Tensor) -> torch.Tensor:
    """Periodic 19-point Laplacian of an (N, N, N) tensor (np.roll(f, 1, ax) == f[x-1])."""
    r = torch.roll
    faces = (r(f, 1, 0) + r(f, -1, 0) + r(f, 1, 1) + r(f, -1, 1) + r(f, 1, 2) + r(f, -1, 2))
    edges = (r(r(f, 1, 0), 1, 1) + r(r(f, 1, 0), -1, 1) + r(r(f, -1, 0), 1, 1)
             + r(r(f, -1, 0), -1, 1) + r(r(f, 1, 0), 1, 2) + r(r(f, 1, 0), -1, 2)
             + r(r(f, -1, 0), 1, 2) + r(r(f, -1, 0), -1, 2) + r(r(f, 1, 1), 1, 2)
             + r(r(f, 1, 1), -1, 2) + r(r(f, -1, 1), 1, 2) + r(r(f, -1, 1), -1, 2))
    return FACE_W * faces + EDGE_W * edges - 4.0 * f


def _chi_tail(chi, chi_prev, acc, mask, chi0, dt2):
    chi_new = 2.0 * chi - chi_prev + dt2 * acc
    chi_new = torch.clamp_min(chi_new, -chi0)
    absorb = 1.0 - mask
    return mask * chi0 + absorb * chi_new


def step_real(E, E_prev, chi, chi_prev, mask, dt2, kappa, lambda_self, chi0, e0_sq):
    """One REAL step (numpy_backend.py:80-130); returns (E', E_prev', chi', chi_prev')."""
    chi_sq = chi * chi
    E_new = 2.0 * E - E_prev + dt2 * (laplacian_19pt(E) - chi_sq * E)
    acc = laplacian_19pt(chi) - (kappa / chi0) * chi * (E * E - e0_sq)
    if lambda_self > 0:
        acc = acc - 4.0 * lambda_self * chi * (chi_sq - chi0 * chi0)
    absorb = 1.0 - mask
    return E_new * absorb, E * absorb, _chi_tail(chi, chi_prev, acc, mask, chi0, dt2), chi


def momentum_current(Pr, Pi):
    j = 0.0
    for ax in range(3):
        dPr = torch.roll(Pr, -1, ax) - torch.roll(Pr, 1, ax)
        dPi = torch.roll(Pi, -1, ax) - torch.roll(Pi, 1, ax)
        j = j + (Pr * dPi - Pi * dPr)
    return 0.5 * j


def step_complex(Pr, Pr_prev, Pi, Pi_prev, chi, chi_prev, mask, dt2, kappa, lambda_self, chi0,
                 e0_sq, epsilon_w):
    """One COMPLEX step (numpy_backend.py:132-205)."""
    chi_sq = chi * chi
    Pr_new = 2.0 * Pr - Pr_prev + dt2 * (laplacian_19pt(Pr) - chi_sq * Pr)
    Pi_new = 2.0 * Pi - Pi_prev + dt2 * (laplacian_19pt(Pi) - chi_sq * Pi)
    psi_sq = Pr * Pr + Pi * Pi
    src = (kappa / chi0) * chi * (psi_sq + epsilon_w * momentum_current(Pr, Pi) - e0_sq)
    acc = laplacian_19pt(chi) - src
    if lambda_self > 0:
        acc = acc - 4.0 * lambda_self * chi * (chi_sq - chi0 * chi0)
    absorb = 1.0 - mask
    return (Pr_new * absorb, Pr * absorb, Pi_new * absorb, Pi * absorb,
            _chi_tail(chi, chi_prev, acc, mask, chi0, dt2), chi)


def run(cfg, state: dict, steps: int, mask: torch.Tensor) -> dict:
    """Advance a state dict (keys pr, prp, chi, chip [, pi, pip]) by `steps` steps."""
    s = dict(state)
    dt2 = cfg.dt**2
    for _ in range(steps):
        if int(cfg.field_level) == 0:
            s["pr"], s["prp"], s["chi"], s["chip"] = step_real(
                s["pr"], s["prp"], s["chi"], s["chip"], mask, dt2, cfg.kappa, cfg.lambda_self,
                cfg.chi0, cfg.e0_sq)
        else:
            (s["pr"], s["prp"], s["pi"], s["pip"], s["chi"], s["chip"]) = step_complex(
                s["pr"], s["prp"], s["pi"], s["pip"], s["chi"], s["chip"], mask, dt2, cfg.kappa,
                cfg.lambda_self, cfg.chi0, cfg.e0_sq, cfg.epsilon_w)
    return s
