"""The cos^2 absorbing sponge and its radial lookup table.

The reference sponge (lfm/core/backends/numpy_backend.py:60-69) is built
from float32 coordinates x - N/2 + 0.5 = (2x - N + 1)/2, so the float32 value
X**2 + Y**2 + Z**2 is exactly q/4 with the integer key
q = (2i-N+1)^2 + (2j-N+1)^2 + (2k-N+1)^2 (every partial sum fits in 24
mantissa bits for N <= 2048).  The mask is therefore a pure function of q.
``radial_values`` applies the reference's float32 operations (sqrt, the
r_freeze shift and scale, clip, sin^2) to q/4, once per distinct key, and the
full mask is a gather from those values -- the same bits as the reference's
per-cell evaluation, without an N^3 host pass.

``MaskTable`` keeps only the band q_lo <= q <= q_hi where the mask is
neither 0 nor 1 (one float32 per key step 2^shift); the resident step
kernels read it instead of streaming a 4 B/cell mask.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib

MAX_N = 2048


def _key_shift(N: int) -> int:
    # (2x-N+1) is odd for even N (q = 3 mod 8) and even for odd N (q = 0 mod 4)
    return 3 if N % 2 == 0 else 2


def radial_keys(N: int) -> np.ndarray:
    """q for every cell, flat int64 in C order."""
    d = (2 * np.arange(N, dtype=np.int64) - N + 1) ** 2
    return (d[:, None, None] + d[None, :, None] + d[None, None, :]).ravel()


def radial_values(N: int, boundary_fraction: float, q: np.ndarray) -> np.ndarray:
    """Mask values for keys q, float32, with the reference's float32 operations."""
    if N > MAX_N:
        raise ValueError(f"N={N} above {MAX_N}: the radial key is no longer exact in float32")
    center = N / 2.0
    r_max = N / 2.0
    r_freeze = (1.0 - boundary_fraction) * r_max
    r2 = (np.asarray(q, dtype=np.float64) / 4.0).astype(np.float32)  # exact: q/4 is dyadic
    R = np.sqrt(r2)
    t = np.clip((R - r_freeze) / (r_max - r_freeze), 0.0, 1.0)
    del center
    return (np.sin(0.5 * np.pi * t) ** 2).astype(np.float32)


def boundary_mask(N: int, boundary_fraction: float) -> np.ndarray:
    """Flat float32 sponge on the host: 0 = transparent interior, 1 = absorbed."""
    q = radial_keys(N)
    uq, inv = np.unique(q, return_inverse=True)
    return radial_values(N, boundary_fraction, uq)[inv].astype(np.float32)


@dataclass
class MaskTable:
    """Host table + descriptor of the sponge band."""

    N: int
    table: np.ndarray
    desc: _lib.MaskLut

    @classmethod
    def for_lattice(cls, N: int, boundary_fraction: float) -> "MaskTable":
        """Table straight from the sponge formula, evaluated on every key step."""
        shift = _key_shift(N)
        q0 = 3 if N % 2 == 0 else 0
        qmax = 3 * (N - 1) ** 2
        cand = np.arange(q0, qmax + 1, 1 << shift, dtype=np.int64)
        vals = radial_values(N, boundary_fraction, cand)
        nz = np.flatnonzero(vals != 0.0)
        n1 = np.flatnonzero(vals != 1.0)
        d = _lib.MaskLut()
        d.N, d.shift = N, shift
        if nz.size == 0:
            d.q_lo, d.q_hi, d.count = np.iinfo(np.int32).max, np.iinfo(np.int32).max - 1, 0
            table = np.zeros(1, np.float32)
        elif n1.size == 0:
            d.q_lo, d.q_hi, d.count = 0, -1, 0
            table = np.zeros(1, np.float32)
        else:
            lo, hi = int(nz[0]), int(n1[-1])
            d.q_lo, d.q_hi = int(cand[lo]), int(cand[hi])
            d.count = hi - lo + 1
            table = vals[lo:hi + 1].copy()
        return cls(N, table, d)

    @classmethod
    def from_mask(cls, N: int, mask: np.ndarray) -> "MaskTable":
        """Table from an arbitrary host mask (checked for radial symmetry by the C builder)."""
        m = np.ascontiguousarray(mask, dtype=np.float32).ravel()
        if m.size != N**3:
            raise ValueError(f"mask has {m.size} values, expected {N**3}")
        cap = (3 * N * N) // 4 + 16
        table = np.zeros(cap, dtype=np.float32)
        desc = _lib.MaskLut()
        _lib.call("lfm_mask_lut_build", int(N), m.ctypes.data, table.ctypes.data, int(cap),
                  ctypes.byref(desc))
        return cls(N, table[: max(desc.count, 1)].copy(), desc)

    def to_device(self, device):
        import torch

        return torch.from_numpy(self.table).to(device)

    def lookup(self, q: np.ndarray) -> np.ndarray:
        """Mask values for keys q (host)."""
        q = np.asarray(q, dtype=np.int64)
        out = np.where(q < self.desc.q_lo, 0.0, 1.0).astype(np.float32)
        band = (q >= self.desc.q_lo) & (q <= self.desc.q_hi)
        out[band] = self.table[(q[band] - self.desc.q_lo) >> self.desc.shift]
        return out

    def device_mask(self, device):
        """The full N^3 mask on `device`, gathered from the table (exact)."""
        import torch

        N = self.N
        x = torch.arange(N, device=device, dtype=torch.int64)
        d = (2 * x - N + 1) ** 2
        q = (d[:, None, None] + d[None, :, None] + d[None, None, :]).reshape(-1)
        out = torch.where(q < self.desc.q_lo, 0.0, 1.0).to(torch.float32)
        band = (q >= self.desc.q_lo) & (q <= self.desc.q_hi)
        if self.desc.count > 0:
            tab = torch.from_numpy(self.table).to(device)
            out[band] = tab[(q[band] - self.desc.q_lo) >> self.desc.shift]
        return out
