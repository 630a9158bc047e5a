"""Per-step hooks on the device buffers: barrier, continuous source, detector screen.

The reference's double-slit experiment drives the leapfrog through host
callbacks that edit the live buffers between steps:

* ``Barrier.apply`` (lfm/experiment/barrier.py:296-351) rewrites every chi
  buffer (chi0 everywhere, the barrier height in a slab, chi0 again in the
  slit openings), zeroes Psi in the solid barrier cells and damps it at
  which-path detector slits;
* ``ContinuousSource.step_callback`` (lfm/experiment/source.py:196-228) adds
  dt^2 * A * sin(omega t) * boost * envelope to one plane of Psi;
* ``DetectorScreen.record`` (lfm/experiment/detector.py:100-116) stores one
  plane of the energy density |Psi|^2 per call.

They reach the fields through ``Simulation._native_*`` (simulation.py:212-256)
as CuPy arrays, and ``Simulation.run`` copies Psi to the host after every
step (simulation.py:1172-1182).  Here the same edits are torch operations on
the Evolver's device buffers (``Evolver.native_*``), each value computed with
the reference's float32 operations, so a run with hooks is bit-identical to
the reference's.  No hook waits on the host, so ``Evolver.evolve(steps,
hooks=[...])`` captures blocks of steps together with their hooks in one
CUDA graph; the source's per-step drive values are uploaded before each
block, and the detector's frames stay on the device until they are read.

A hook implements ``apply(evolver, step)`` (one call after each step, step
being the evolver's step count after it), and for graph blocks
``prepare_block(evolver, count)`` (allocations, before capture),
``begin_block(evolver, first_step, count)`` (host values for steps
first_step + 1 .. first_step + count, before each replay),
``apply_in_block(evolver, k)`` (the captured work after the block's k-th
step) and ``end_block(evolver, count)``.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .config import CHI0

DEFAULT_BARRIER_HEIGHT = CHI0 + 50.0  # barrier.py:68 (the constant chi0, not the config's)


def _plane(field, axis: int, index: int):
    sl = [slice(None), slice(None), slice(None)]
    sl[axis] = index
    return field[tuple(sl)]


def resolve_cell(value, N: int) -> int:
    """Fractional (a float below 1: that fraction of N, rounded) or absolute
    cell index, clamped to the lattice (source.py:_resolve)."""
    if isinstance(value, float) and value < 1.0:
        return max(0, min(N - 1, round(value * N)))
    return max(0, min(N - 1, int(value)))


def resolve_width(value, N: int) -> float:
    """Fractional (below 1: that fraction of N) or absolute width in cells."""
    if isinstance(value, float) and value < 1.0:
        return value * N
    return float(value)


class DeviceHook:
    """Base of the hooks: eager apply() plus the graph-block protocol."""

    graphable = True

    def apply(self, evolver, step: int) -> None:  # pragma: no cover - abstract
        raise NotImplementedError

    def step_callback(self, evolver, step: int) -> None:
        """The reference's callback signature (sim, step)."""
        self.apply(evolver, step)

    def prepare_block(self, evolver, count: int) -> None:
        pass

    def begin_block(self, evolver, first_step: int, count: int) -> None:
        pass

    def apply_in_block(self, evolver, k: int) -> None:
        self.apply(evolver, -1)

    def end_block(self, evolver, count: int) -> None:
        pass


# ---------------------------------------------------------------- barrier
@dataclass
class Slit:
    """A slit opening (barrier.py:71-90): centre and width along the slit
    axis; an optional which-path detector of the given strength."""

    center: int
    width: int = 4
    detector: bool = False
    detector_strength: float = 1.0


def default_slits(N: int) -> list:
    """Two equal slits symmetric about the centre (barrier.py:149-156)."""
    half_sep = max(4, N // 8)
    slit_w = max(2, N // 32)
    return [Slit(center=N // 2 - half_sep, width=slit_w),
            Slit(center=N // 2 + half_sep, width=slit_w)]


def barrier_geometry(N: int, axis: int, position: int, thickness: int, slits,
                     slit_axis: int):
    """(slab slices, per-slit slices, solid-cell mask, per-slit masks) of a barrier."""
    start = max(0, position - thickness // 2)
    end = min(N, start + thickness)
    slab = [slice(None)] * 3
    slab[axis] = slice(start, end)
    slab = tuple(slab)
    slit_sls = []
    for s in slits:
        s0 = max(0, s.center - s.width // 2)
        s1 = min(N, s0 + s.width)
        sl = [slice(None)] * 3
        sl[axis] = slice(start, end)
        sl[slit_axis] = slice(s0, s1)
        slit_sls.append(tuple(sl))
    solid = np.zeros((N, N, N), dtype=bool)
    solid[slab] = True
    masks = []
    for sl in slit_sls:
        m = np.zeros((N, N, N), dtype=bool)
        m[sl] = True
        masks.append(m)
        solid[sl] = False
    return slab, slit_sls, solid, masks


class Barrier(DeviceHook):
    """A chi barrier slab with slit openings, re-imposed after every step.

    Geometry (barrier.py:157-168, 263-292): the slab covers cells
    [start, start + thickness) along ``axis``, start = max(0, position -
    thickness // 2); slit s opens [s0, s0 + width) along ``slit_axis``, s0 =
    max(0, center - width // 2), across the whole slab and the third axis.

    apply() writes chi0 to every chi buffer, the height to the slab, chi0 to
    the openings (all chi buffers, so chi has no velocity there); with
    ``absorb`` it multiplies Psi by 0 in the solid cells (the reference's
    float32 mask product, signed zeros included; outside the slab the mask
    is 1 and the product the identity, so only the slab is touched); then it
    multiplies Psi at each detector slit by float32(1 - gamma), gamma = 1 -
    (1 - strength)^(1 / transit_steps) (barrier.py:232-249).  Like the
    reference, the constructor applies the barrier once.
    """

    def __init__(self, evolver, axis: int = 2, position: int | None = None,
                 height: float | None = None, thickness: int = 2, slits=None,
                 slit_axis: int | None = None, absorb: bool = True,
                 transit_steps: int = 10) -> None:
        import torch

        _check_level(evolver)
        N = evolver.N
        self._N = N
        self._axis = axis
        self._height = float(height if height is not None else DEFAULT_BARRIER_HEIGHT)
        self._pos = position if position is not None else N // 2
        self._thick = thickness
        self._absorb = absorb
        self._slits = list(slits) if slits is not None else default_slits(N)
        self._slit_axis = slit_axis if slit_axis is not None else (axis + 1) % 3
        self._chi0 = float(evolver.config.chi0)
        (self._slab, self._slit_sls, self._barrier_mask,
         self._slit_masks) = barrier_geometry(N, axis, self._pos, thickness, self._slits,
                                              self._slit_axis)
        # Psi factor inside the slab: 0 at solid cells, 1 in the openings
        self._slab_factor = torch.from_numpy(
            np.ascontiguousarray((~self._barrier_mask[self._slab]).astype(np.float32))).to(
                evolver.device)
        self._det = []
        for s, sl in zip(self._slits, self._slit_sls):
            if s.detector and s.detector_strength > 0.0:
                transit = max(1, transit_steps)
                strength = float(min(1.0, s.detector_strength))
                gamma = 1.0 if strength >= 1.0 else 1.0 - (1.0 - strength) ** (1.0 / transit)
                self._det.append((sl, float(np.float32(1.0 - gamma))))
        self.apply(evolver, evolver.step)

    def apply(self, evolver, step: int = -1) -> None:
        for buf in evolver.native_chi_pair():
            buf.fill_(self._chi0)
            buf[self._slab].fill_(self._height)
            for sl in self._slit_sls:
                buf[sl].fill_(self._chi0)
        psis = [evolver.native_psi_real()]
        pi = evolver.native_psi_imag()
        if pi is not None:
            psis.append(pi)
        for p in psis:
            if self._absorb:
                p[self._slab].mul_(self._slab_factor)
            for sl, f in self._det:
                p[sl].mul_(f)

    @property
    def mask(self) -> np.ndarray:
        """Solid barrier cells (slab minus openings), (N, N, N) bool."""
        return self._barrier_mask

    @property
    def slit_masks(self) -> list:
        return self._slit_masks

    @property
    def slits(self) -> list:
        return list(self._slits)

    def measure_slits(self, evolver) -> dict:
        """Mean energy density at each slit opening (float64 mean on the device)."""
        ed = evolver.native_psi_real().double() ** 2
        pi = evolver.native_psi_imag()
        if pi is not None:
            ed = ed + pi.double() ** 2
        return {f"slit_{i}": float(ed[sl].mean()) for i, sl in enumerate(self._slit_sls)}


# ---------------------------------------------------------------- source
def source_envelope(N: int, envelope_sigma) -> np.ndarray:
    """The transverse float32 Gaussian of a source (source.py:137-147)."""
    sigma = resolve_width(envelope_sigma, N)
    centre = N / 2.0
    c0 = (np.arange(N, dtype=np.float32) - centre).reshape(-1, 1)
    c1 = (np.arange(N, dtype=np.float32) - centre).reshape(1, -1)
    return np.exp(-(c0**2 + c1**2) / (2.0 * sigma**2)).astype(np.float32)


class ContinuousSource(DeviceHook):
    """A monochromatic source on one plane (source.py:79-228).

    After step ``step`` it adds injection * envelope to the plane of Psi_r,
    injection = dt^2 * amplitude * sin(omega * step * dt) * boost (float64
    on the host, then rounded to float32 as NumPy rounds a Python float
    meeting a float32 array), and, when phase != 0 at the COMPLEX level,
    injection * sin(phase) * envelope to Psi_i.  A step whose |injection| <
    1e-30 adds nothing.  The envelope is the reference's float32 transverse
    Gaussian exp(-(c0^2 + c1^2) / (2 sigma^2)), c = arange(N) - N/2.
    """

    def __init__(self, evolver, axis: int = 2, position=0.25, omega: float = 2.0,
                 amplitude: float = 2.0, envelope_sigma=0.25, phase: float = 0.0,
                 boost: float = 10.0) -> None:
        import torch

        _check_level(evolver)
        N = evolver.N
        self._N = N
        self._axis = axis
        self._pos = resolve_cell(position, N)
        self._omega = omega
        self._amplitude = amplitude
        self._phase = phase
        self._boost = boost
        self._dt = float(evolver.config.dt)
        self.envelope = source_envelope(N, envelope_sigma)
        self._env = torch.from_numpy(self.envelope).to(evolver.device)
        self._imag = abs(self._phase) > 1e-12 and evolver.native_psi_imag() is not None
        self._blk = None

    @property
    def position(self) -> int:
        return self._pos

    def injection(self, step: int) -> float:
        """dt^2 * A * sin(omega * t) * boost at t = step * dt (float64)."""
        t = step * self._dt
        return self._dt**2 * self._amplitude * math.sin(self._omega * t) * self._boost

    def apply(self, evolver, step: int) -> None:
        inj = self.injection(step)
        if abs(inj) < 1e-30:
            return
        _plane(evolver.native_psi_real(), self._axis, self._pos).add_(self._env * inj)
        if self._imag:
            pf = inj * math.sin(self._phase)
            _plane(evolver.native_psi_imag(), self._axis, self._pos).add_(self._env * pf)

    # graph blocks: the per-step factors come from device tables
    def prepare_block(self, evolver, count: int) -> None:
        import torch

        if self._blk is None or self._blk[0].numel() != count:
            dev = evolver.device
            self._blk = (torch.zeros(count, dtype=torch.float32, device=dev),
                         torch.zeros(count, dtype=torch.float32, device=dev),
                         torch.zeros(count, dtype=torch.bool, device=dev))

    def begin_block(self, evolver, first_step: int, count: int) -> None:
        import torch

        inj = np.array([self.injection(first_step + 1 + k) for k in range(count)])
        act = np.abs(inj) >= 1e-30
        pf = inj * math.sin(self._phase)
        # pageable host tensors: the copies are staged before copy_ returns,
        # so the host arrays may be reused at once
        self._blk[0].copy_(torch.from_numpy(inj.astype(np.float32)))
        self._blk[1].copy_(torch.from_numpy(pf.astype(np.float32)))
        self._blk[2].copy_(torch.from_numpy(act))

    def apply_in_block(self, evolver, k: int) -> None:
        import torch

        inj, pf, act = self._blk
        p = _plane(evolver.native_psi_real(), self._axis, self._pos)
        p.copy_(torch.where(act[k], p + self._env * inj[k], p))
        if self._imag:
            q = _plane(evolver.native_psi_imag(), self._axis, self._pos)
            q.copy_(torch.where(act[k], q + self._env * pf[k], q))


# ---------------------------------------------------------------- detector
class DetectorScreen(DeviceHook):
    """Frames of one plane of a field, recorded on the device (detector.py:53-260).

    field: ``energy_density`` (|Psi|^2 = Psi_r^2 [+ Psi_i^2] in float32, as
    Evolver.get_energy_density forms it), ``psi_real``, ``psi_imag`` or
    ``chi``.  ``pattern`` is the float32 sum of the frames in recording order
    (NumPy's sum over the frame axis), kept as a running sum on the device.
    """

    def __init__(self, evolver, axis: int = 2, position: int | None = None,
                 field: str = "energy_density") -> None:
        import torch

        _check_level(evolver)
        if field not in ("energy_density", "psi_real", "psi_imag", "chi"):
            raise ValueError(f"Unknown field '{field}'. Choose from 'energy_density', "
                             "'psi_real', 'psi_imag', 'chi'.")
        N = evolver.N
        self._N = N
        self._axis = axis
        self._pos = position if position is not None else int(N * 0.80)
        self._field = field
        self._dev = evolver.device
        self._chunks: list = []  # device tensors of frames, (k, N, N)
        self._sum = torch.zeros((N, N), dtype=torch.float32, device=evolver.device)
        self._n = 0
        self._stage = None

    def _frame(self, evolver):
        import torch

        if self._field == "chi":
            return _plane(evolver.native_chi(), self._axis, self._pos)
        pr = _plane(evolver.native_psi_real(), self._axis, self._pos)
        pi = evolver.native_psi_imag()
        if self._field == "psi_real":
            return pr
        if self._field == "psi_imag":
            return (_plane(pi, self._axis, self._pos) if pi is not None else
                    torch.zeros((self._N, self._N), dtype=torch.float32, device=self._dev))
        e2 = pr * pr
        if pi is not None:
            q = _plane(pi, self._axis, self._pos)
            e2 = e2 + q * q
        return e2

    def record(self, evolver) -> None:
        f = self._frame(evolver).clone()
        self._chunks.append(f.unsqueeze(0))
        self._sum.add_(f)
        self._n += 1

    def apply(self, evolver, step: int) -> None:
        self.record(evolver)

    def prepare_block(self, evolver, count: int) -> None:
        import torch

        if self._stage is None or self._stage.shape[0] != count:
            self._stage = torch.zeros((count, self._N, self._N), dtype=torch.float32,
                                      device=evolver.device)

    def apply_in_block(self, evolver, k: int) -> None:
        self._stage[k].copy_(self._frame(evolver))
        self._sum.add_(self._stage[k])

    def end_block(self, evolver, count: int) -> None:
        self._chunks.append(self._stage[:count].clone())
        self._n += count

    def reset(self) -> None:
        self._chunks.clear()
        self._sum.zero_()
        self._n = 0

    @property
    def n_frames(self) -> int:
        return self._n

    @property
    def pattern(self) -> np.ndarray:
        """Sum of the recorded frames, (N, N) float32 (zeros before any)."""
        return self._sum.cpu().numpy()

    @property
    def snapshots(self) -> np.ndarray:
        """Every recorded frame, (K, N, N) float32."""
        import torch

        if not self._chunks:
            return np.zeros((0, self._N, self._N), dtype=np.float32)
        return torch.cat(self._chunks, dim=0).cpu().numpy()

    def mean_pattern(self) -> np.ndarray:
        if not self._n:
            return np.zeros((self._N, self._N), dtype=np.float32)
        return (self.pattern / self._n).astype(np.float32)

    def line_profile(self, perp_axis: int = 0) -> np.ndarray:
        return self.pattern.sum(axis=perp_axis).astype(np.float32)

    def click_pattern(self, n_particles: int = 1000, seed: int | None = None) -> np.ndarray:
        """Discrete detection events drawn from the pattern (detector.py:181-210)."""
        pat = self.pattern
        total = pat.sum()
        if total == 0:
            return np.zeros(pat.shape, dtype=np.int32)
        prob = pat.ravel() / total
        rng = np.random.default_rng(seed)
        idx = rng.choice(len(prob), size=n_particles, p=prob)
        hist, _ = np.histogram(idx, bins=np.arange(len(prob) + 1))
        return hist.reshape(pat.shape).astype(np.int32)

    @property
    def position(self) -> int:
        return self._pos

    @property
    def axis(self) -> int:
        return self._axis


def _check_level(evolver) -> None:
    if evolver.native_psi_real().dim() != 3:
        raise ValueError("hooks edit (N, N, N) fields: REAL and COMPLEX levels")
