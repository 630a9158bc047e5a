"""The cos^2 absorbing sponge and its radial lookup table.

``boundary_mask`` evaluates the sponge on the host with the same float32
NumPy operations as the reference (lfm/core/backends/numpy_backend.py:60-69),
so its bits equal the reference mask on the same machine.  ``MaskTable``
compresses it, through ``lfm_mask_lut_build`` in the C library, into the
per-key table the resident step kernels read (a few tens of KB, L1-resident,
instead of a 4 B/cell stream).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib


def boundary_mask(N: int, boundary_fraction: float) -> np.ndarray:
    """Flat float32 sponge: 0 = transparent interior, 1 = fully absorbed."""
    center = N / 2.0
    r_max = N / 2.0
    r_freeze = (1.0 - boundary_fraction) * r_max
    coords = np.arange(N, dtype=np.float32) - center + 0.5
    X, Y, Z = np.meshgrid(coords, coords, coords, indexing="ij")
    R = np.sqrt(X**2 + Y**2 + Z**2)
    t = np.clip((R - r_freeze) / (r_max - r_freeze), 0.0, 1.0)
    return (np.sin(0.5 * np.pi * t) ** 2).astype(np.float32).ravel()


@dataclass
class MaskTable:
    """Host table + descriptor; ``to_device`` gives the kernels' copy."""

    N: int
    table: np.ndarray
    desc: _lib.MaskLut

    @classmethod
    def from_mask(cls, N: int, mask: np.ndarray) -> "MaskTable":
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
        """Mask values for keys q (host-side check of the table)."""
        q = np.asarray(q, dtype=np.int64)
        out = np.where(q < self.desc.q_lo, 0.0, 1.0).astype(np.float32)
        band = (q >= self.desc.q_lo) & (q <= self.desc.q_hi)
        out[band] = self.table[(q[band] - self.desc.q_lo) >> self.desc.shift]
        return out


def radial_keys(N: int) -> np.ndarray:
    """q = (2i-N+1)^2 + (2j-N+1)^2 + (2k-N+1)^2 for every cell, flat int64."""
    d = (2 * np.arange(N, dtype=np.int64) - N + 1) ** 2
    return (d[:, None, None] + d[None, :, None] + d[None, None, :]).ravel()
