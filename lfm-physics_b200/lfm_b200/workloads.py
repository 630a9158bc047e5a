"""Seeded synthetic initial states of the benchmark workloads.

The reference measures on synthetic lattices only; these builders produce
states with the shapes, sizes and value distributions of the five workloads
the benchmark and the parity tests use.  Gaussian packets follow
amplitude*exp(-r^2/(2 sigma^2)) as lfm/fields/soliton.py:49-59 builds them,
evaluated on a box of +-6 sigma around each centre (the envelope is below
2e-8 of its peak outside it) so that 512^3 states build in seconds.
"""

from __future__ import annotations

import math

import numpy as np


def add_gaussian(field: np.ndarray, center, amplitude: float, sigma: float,
                 phase_factor: complex | float = 1.0) -> None:
    """Accumulate amplitude*exp(-r^2/(2 sigma^2)) (times phase_factor) into a float64 field."""
    N = field.shape[-1]
    reach = int(math.ceil(6.0 * sigma))
    idx = []
    for c in center:
        lo = int(math.floor(c)) - reach
        idx.append(np.arange(lo, lo + 2 * reach + 2))
    dx = [(ix - c) ** 2 for ix, c in zip(idx, center)]
    r2 = dx[0][:, None, None] + dx[1][None, :, None] + dx[2][None, None, :]
    env = amplitude * np.exp(-r2 / (2.0 * sigma * sigma))
    sel = np.ix_(*(ix % N for ix in idx))
    if 2 * reach + 2 <= N:
        field[sel] += env * phase_factor  # no index repeats inside the box
    else:
        np.add.at(field, sel, env * phase_factor)


def real_solitons(N: int, count: int = 64, seed_chi: int = 1, seed_solitons: int = 2):
    """Throughput state at the REAL level (the 512^3 benchmark workload).

    chi = 19 + U(-1e-3, 1e-3) (seed_chi); `count` packets with amplitude
    U[2, 6] and sigma U[2, 4] cells, centred uniformly inside the sponge-free
    sphere |x - N/2| < 0.35 N - 3 sigma (seed_solitons).  Returns float32
    (E, chi), each (N, N, N); E_prev = E.
    """
    rng_c = np.random.default_rng(seed_chi)
    chi = (19.0 + rng_c.uniform(-1e-3, 1e-3, size=(N, N, N))).astype(np.float32)
    rng = np.random.default_rng(seed_solitons)
    E = np.zeros((N, N, N), dtype=np.float64)
    c0 = N / 2.0
    for _ in range(count):
        amp = rng.uniform(2.0, 6.0)
        sigma = rng.uniform(2.0, 4.0)
        rmax = 0.35 * N - 3.0 * sigma
        while True:
            p = rng.uniform(c0 - rmax, c0 + rmax, size=3)
            if np.sum((p - c0) ** 2) < rmax * rmax:
                break
        add_gaussian(E, tuple(p), amp, sigma)
    return E.astype(np.float32), chi


def config1_soliton(N: int = 64, seed: int = 42):
    """REAL 64^3 parity workload: packet (6.0, sigma 3) at the centre + 1e-4 N(0,1) noise."""
    x = np.arange(N, dtype=np.float32)
    c = N // 2
    r2 = ((x - c) ** 2)[:, None, None] + ((x - c) ** 2)[None, :, None] + ((x - c) ** 2)[None, None, :]
    env = (6.0 * np.exp(-r2 / (2.0 * 3.0**2))).astype(np.float32)
    rng = np.random.default_rng(seed)
    return (env + 1e-4 * rng.standard_normal((N,) * 3)).astype(np.float32)


def color_packets(N: int = 256, seed_phase: int = 3, seed_chi: int = 4):
    """COLOR workload: two colour-charged packets (amplitude 4, sigma 3), 40 cells apart.

    Each packet carries a seeded random colour-phase vector theta_a ~ U[0, 2pi):
    Psi_a = A g(r) e^{i theta_a} / sqrt(3).  chi = 19 +- 1e-3 (seed_chi).
    Returns float32 (psi_r, psi_i) of shape (3, N, N, N) and chi (N, N, N).
    """
    rng = np.random.default_rng(seed_phase)
    pr = np.zeros((3, N, N, N), dtype=np.float64)
    pi = np.zeros((3, N, N, N), dtype=np.float64)
    c = N / 2.0
    centres = ((c, c - 20.0, c), (c, c + 20.0, c))
    for ctr in centres:
        theta = rng.uniform(0.0, 2.0 * np.pi, size=3)
        for a in range(3):
            f = np.exp(1j * theta[a]) / np.sqrt(3.0)
            add_gaussian(pr[a], ctr, 4.0, 3.0, f.real)
            add_gaussian(pi[a], ctr, 4.0, 3.0, f.imag)
    rng_c = np.random.default_rng(seed_chi)
    chi = (19.0 + rng_c.uniform(-1e-3, 1e-3, size=(N, N, N))).astype(np.float32)
    return pr.astype(np.float32), pi.astype(np.float32), chi


def sweep_lattices(count: int = 256, seed: int = 5, sizes=(32, 48, 64, 80, 96)):
    """Batched-sweep workload: `count` independent lattices of uneven sizes.

    One generator (seed) draws, per lattice: N uniformly from `sizes`, the
    level by a fair coin (REAL or COMPLEX), kappa = U[0.5, 2]/63, and one
    packet at the centre with amplitude U[1, 8] and sigma U[2, 4] (COMPLEX
    lattices give it a phase U[0, 2pi)).  chi starts at chi0.  Returns a list
    of (config, psi_r, psi_i or None), float32 (N, N, N) fields.
    """
    from .config import gravity_em, gravity_only

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        N = int(rng.choice(sizes))
        complex_level = bool(rng.integers(0, 2))
        kappa = float(rng.uniform(0.5, 2.0)) / 63.0
        amp = float(rng.uniform(1.0, 8.0))
        sigma = float(rng.uniform(2.0, 4.0))
        theta = float(rng.uniform(0.0, 2.0 * np.pi)) if complex_level else 0.0
        cfg = (gravity_em if complex_level else gravity_only)(N, kappa=kappa)
        c = N / 2.0
        pr = np.zeros((N, N, N), dtype=np.float64)
        add_gaussian(pr, (c, c, c), amp, sigma, math.cos(theta))
        pi = None
        if complex_level:
            pi = np.zeros((N, N, N), dtype=np.float64)
            add_gaussian(pi, (c, c, c), amp, sigma, math.sin(theta))
            pi = pi.astype(np.float32)
        out.append((cfg, pr.astype(np.float32), pi))
    return out


def adjoint_packets(N: int = 96, seed: int = 6):
    """Adjoint workload: the learnable packets and the target run's packets.

    Two packets of sigma 3 cells, 8 cells apart along j around the centre (they
    overlap, so their relative phase shapes |Psi|^2 and the momentum current),
    amplitudes U[4, 6] and phases U[0, 2 pi) (seed).  The target run uses
    different parameters drawn from the same generator: amplitudes x U[1.15,
    1.35], centres moved by U[-2, 2] cells per axis, phases moved by U[-0.8,
    0.8].  The runs start the packets rotating as the reference's
    Simulation.place_soliton does (previous phase + chi0 dt; soliton_state's
    omega_dt), so |Psi|^2 stays put while chi responds.  Under gravity_em at
    dt = 0.02, chi's forced oscillation is near the end of a cycle at step 500:
    chi_T lies within ~1e-5 of chi0, and the two runs' chi differ by ~3e-5
    there, against ~1e-3 mid-run.

    Returns ((amplitude (2,), centre (2, 3), phase (2,)), (the target's three),
    sigma), float64 torch tensors on the CPU.
    """
    import torch

    g = torch.Generator().manual_seed(seed)
    u = lambda *s: torch.rand(*s, generator=g, dtype=torch.float64)  # noqa: E731
    c = N / 2.0
    amp = 4.0 + 2.0 * u(2)
    cen = torch.tensor([[c, c - 4.0, c], [c, c + 4.0, c]], dtype=torch.float64)
    ph = 2.0 * math.pi * u(2)
    amp_t = amp * (1.15 + 0.2 * u(2))
    cen_t = cen + (4.0 * u(2, 3) - 2.0)
    ph_t = ph + (1.6 * u(2) - 0.8)
    return (amp, cen, ph), (amp_t, cen_t, ph_t), 3.0
