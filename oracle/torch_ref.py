"""Plain PyTorch transcription of the reference step.  TEST INFRASTRUCTURE ONLY.

Restates lfm/core/backends/numpy_backend.py:80-382 (REAL, COMPLEX and COLOR,
with the S_a Helmholtz solve through torch.fft) and the 19-point Laplacian of
lfm/core/stencils.py:26-71 with out-of-place torch operations, in whatever
dtype the inputs carry.  In float64 it serves as:
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


def helmholtz_sa(ea: torch.Tensor, gamma: float, d: float) -> torch.Tensor:
    """max(0, IRFFT[gamma / (gamma + D k^2) RFFT(ea)]) of one colour's |Psi_a|^2
    (numpy_backend.py:338-352), k = 2 pi fftfreq on each axis."""
    N = ea.shape[0]
    dev = ea.device
    kx = torch.fft.fftfreq(N, device=dev, dtype=torch.float64) * (2.0 * torch.pi)
    kz = torch.fft.rfftfreq(N, device=dev, dtype=torch.float64) * (2.0 * torch.pi)
    k_sq = kx[:, None, None] ** 2 + kx[None, :, None] ** 2 + kz[None, None, :] ** 2
    h = gamma / (gamma + d * k_sq)
    sa = torch.fft.irfftn(h * torch.fft.rfftn(ea.double()), s=(N, N, N), dim=(0, 1, 2))
    return torch.clamp_min(sa, 0.0).to(ea.dtype)


def step_color(Pr, Pr_prev, Pi, Pi_prev, chi, chi_prev, mask, dt2, kappa, lambda_self, chi0,
               e0_sq, epsilon_w, kappa_c=0.0, epsilon_cc=0.0, kappa_string=0.0,
               kappa_tube=0.0, sa_gamma=0.1, sa_d=4.9):
    """One COLOR step (numpy_backend.py:207-382) of (3, N, N, N) Psi; returns
    (Pr', Pr_prev', Pi', Pi_prev', chi', chi_prev', S_a)."""
    n_colors = 3
    chi_sq = chi * chi
    if epsilon_cc > 0:
        Pr_avg = sum(Pr[a] for a in range(n_colors)) / n_colors
        Pi_avg = sum(Pi[a] for a in range(n_colors)) / n_colors
    pr_new, pi_new, ea, jd = [], [], [], []
    psi_sq_total = 0.0
    j_total = 0.0
    for a in range(n_colors):
        pr, pi = Pr[a], Pi[a]
        r_new = 2.0 * pr - Pr_prev[a] + dt2 * (laplacian_19pt(pr) - chi_sq * pr)
        i_new = 2.0 * pi - Pi_prev[a] + dt2 * (laplacian_19pt(pi) - chi_sq * pi)
        if epsilon_cc > 0:
            r_new = r_new - dt2 * epsilon_cc * chi_sq * (pr - Pr_avg)
            i_new = i_new - dt2 * epsilon_cc * chi_sq * (pi - Pi_avg)
        pr_new.append(r_new)
        pi_new.append(i_new)
        e = pr * pr + pi * pi
        ea.append(e)
        psi_sq_total = psi_sq_total + e
        js = []
        for ax in range(3):
            dPr = torch.roll(pr, -1, ax) - torch.roll(pr, 1, ax)
            dPi = torch.roll(pi, -1, ax) - torch.roll(pi, 1, ax)
            js.append(pr * dPi - pi * dPr)
        jd.append(js)
        j_total = j_total + 0.5 * (js[0] + js[1] + js[2])
    color_var = 0.0
    if kappa_c > 0:
        sum_sq = ea[0] ** 2 + ea[1] ** 2 + ea[2] ** 2
        total_sq = psi_sq_total * psi_sq_total
        safe = total_sq > 1e-30
        ratio = torch.where(safe, sum_sq / torch.where(safe, total_sq, 1.0), 0.0)
        f_c = (ratio - 1.0 / n_colors) * safe
        color_var = (kappa_c / chi0) * chi * f_c * psi_sq_total
    ccv = 0.0
    if kappa_string > 0:
        for d in range(3):
            sum_j_sq = jd[0][d] ** 2 + jd[1][d] ** 2 + jd[2][d] ** 2
            sum_j = jd[0][d] + jd[1][d] + jd[2][d]
            ccv = ccv + (sum_j_sq - (1.0 / n_colors) * sum_j**2)
    scv = 0.0
    sa = None
    if kappa_tube > 0:
        sa = torch.stack([helmholtz_sa(e, sa_gamma, sa_d) for e in ea])
        sa_sum = sa[0] + sa[1] + sa[2]
        sa_sq_sum = sa[0] * sa[0] + sa[1] * sa[1] + sa[2] * sa[2]
        scv = sa_sq_sum - (1.0 / n_colors) * sa_sum**2
    src = (kappa / chi0) * chi * (psi_sq_total + epsilon_w * j_total - e0_sq)
    acc = laplacian_19pt(chi) - src - color_var - kappa_string * ccv - kappa_tube * scv
    if lambda_self > 0:
        acc = acc - 4.0 * lambda_self * chi * (chi_sq - chi0 * chi0)
    absorb = 1.0 - mask
    return (torch.stack(pr_new) * absorb, Pr * absorb, torch.stack(pi_new) * absorb,
            Pi * absorb, _chi_tail(chi, chi_prev, acc, mask, chi0, dt2), chi, sa)


def run(cfg, state: dict, steps: int, mask: torch.Tensor) -> dict:
    """Advance a state dict (keys pr, prp, chi, chip [, pi, pip]) by `steps` steps."""
    s = dict(state)
    dt2 = cfg.dt**2
    for _ in range(steps):
        if int(cfg.field_level) == 0:
            s["pr"], s["prp"], s["chi"], s["chip"] = step_real(
                s["pr"], s["prp"], s["chi"], s["chip"], mask, dt2, cfg.kappa, cfg.lambda_self,
                cfg.chi0, cfg.e0_sq)
        elif int(cfg.field_level) == 1:
            (s["pr"], s["prp"], s["pi"], s["pip"], s["chi"], s["chip"]) = step_complex(
                s["pr"], s["prp"], s["pi"], s["pip"], s["chi"], s["chip"], mask, dt2, cfg.kappa,
                cfg.lambda_self, cfg.chi0, cfg.e0_sq, cfg.epsilon_w)
        else:  # COLOR: Psi (3, N, N, N); S_a from this step's |Psi_a|^2
            (s["pr"], s["prp"], s["pi"], s["pip"], s["chi"], s["chip"], s["sa"]) = step_color(
                s["pr"], s["prp"], s["pi"], s["pip"], s["chi"], s["chip"], mask, dt2, cfg.kappa,
                cfg.lambda_self, cfg.chi0, cfg.e0_sq, cfg.epsilon_w, cfg.kappa_c, cfg.epsilon_cc,
                cfg.kappa_string, cfg.kappa_tube, cfg.sa_gamma, cfg.sa_d)
    return s
