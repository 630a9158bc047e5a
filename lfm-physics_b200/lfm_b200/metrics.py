"""Float64 metrics of a lattice state, reduced on the GPU.

``device_metrics`` returns the keys of the reference's compute_metrics
(lfm/analysis/metrics.py:98-111) computed by ``lfm_metrics_f64``: energy
terms in float64 with np.gradient's non-periodic edges
(lfm/analysis/energy.py:26-113), chi statistics, well and void fractions over
interior_mask (lfm/analysis/structure.py:26-171).  Only scalars cross to the
host.  The cluster count needs a connected-component labelling of |Psi|^2 on
the host and is computed only when asked for.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

KEYS = ("energy_kinetic", "energy_gradient", "energy_potential", "energy_total", "chi_min",
        "chi_max", "chi_mean", "chi_std", "well_fraction", "void_fraction", "psi_sq_total",
        "interior_cells", "nonfinite_cells")


def _ptr(t):
    return None if t is None else t.data_ptr()


def device_metrics(ctx, level: int, N: int, psi_r, psi_r_prev, psi_i, psi_i_prev, chi, dt: float,
                   c: float = 1.0, boundary_fraction: float = 0.3, well_threshold: float = 17.0,
                   void_threshold: float = 18.0) -> dict:
    """Metrics of device tensors (flat or shaped float32, contiguous)."""
    import torch

    dev = chi.device
    for t in (psi_r, psi_r_prev, psi_i, psi_i_prev, chi):
        if t is not None and (t.dtype != torch.float32 or not t.is_contiguous() or t.device != dev):
            raise ValueError("metrics take contiguous float32 tensors on one device")
    out = (ctypes.c_double * len(KEYS))()
    stream = torch.cuda.current_stream(dev).cuda_stream
    _lib.call("lfm_metrics_f64", ctx, int(level), _ptr(psi_r), _ptr(psi_r_prev), _ptr(psi_i),
              _ptr(psi_i_prev), _ptr(chi), int(N), float(dt), float(c), float(boundary_fraction),
              float(well_threshold), float(void_threshold), out, stream)
    return dict(zip(KEYS, (float(v) for v in out)))


def n_clusters(psi_sq: np.ndarray, interior: np.ndarray, percentile: float = 90.0) -> int:
    """Connected clusters of |Psi|^2 above a percentile (lfm/analysis/structure.py:84-126)."""
    from scipy import ndimage

    vals = psi_sq[interior]
    if vals.size == 0:
        return 0
    thresh = np.percentile(vals, percentile)
    binary = (psi_sq > thresh) & interior
    return int(ndimage.label(binary)[1])


def interior_mask(N: int, boundary_fraction: float = 0.3) -> np.ndarray:
    """dist <= N/2 * (1 - boundary_fraction), float64 (lfm/analysis/structure.py:148-171)."""
    center = N / 2.0
    radius = center * (1.0 - boundary_fraction)
    x = np.arange(N, dtype=np.float64)
    d2 = ((x - center) ** 2)[:, None, None] + ((x - center) ** 2)[None, :, None] \
        + ((x - center) ** 2)[None, None, :]
    return np.sqrt(d2) <= radius
