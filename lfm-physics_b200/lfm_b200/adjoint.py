"""Reverse-mode gradients through many leapfrog steps (REAL and COMPLEX).

``leapfrog(config, state, steps)`` advances a state given in the reference
representation -- the six arrays (psi_r, psi_r_prev, psi_i, psi_i_prev, chi,
chi_prev) that one step of lfm/core/backends/numpy_backend.py:80-205 reads
and writes -- and is differentiable with ``torch.autograd``:

* forward: the resident fused steps (lfm_leapfrog_*_f32), keeping a copy of
  the state every ``every`` steps (default ceil(sqrt(steps)));
* backward: segment by segment from the last, the segment's states are
  recomputed from its checkpoint (bit-identical to the forward run) and the
  hand-written adjoint step (lfm_adjoint_step_f32) carries the gradient back
  through each step.

Memory: ceil(steps/every) checkpoints of 4 (REAL) or 6 (COMPLEX) fields plus
`every` recomputed states of 2 or 3 fields, instead of all `steps` states.
"""

from __future__ import annotations

import ctypes
import math

import torch

from . import _lib
from .backend import B200Backend, _stream_handle, get_backend
from .config import FieldLevel
from .mask import MaskTable

FIELDS = ("psi_r", "psi_r_prev", "psi_i", "psi_i_prev", "chi", "chi_prev")


class _Lattice:
    """Resident slots of one lattice plus the calls that step and un-step it."""

    def __init__(self, config, backend: B200Backend) -> None:
        self.config = config
        self.backend = backend
        self.device = backend.device
        self.level = FieldLevel(int(config.field_level))
        if self.level == FieldLevel.COLOR:
            raise ValueError("the adjoint covers the REAL and COMPLEX levels")
        self.N = int(config.grid_size)
        self.n = self.N**3
        self.cx = self.level == FieldLevel.COMPLEX
        t = MaskTable.for_lattice(self.N, config.boundary_fraction)
        self.table = t.to_device(self.device)
        self.desc = t.desc
        self.absorb = 1.0 - t.device_mask(self.device)
        f32 = dict(dtype=torch.float32, device=self.device)
        self.pr = [torch.empty(self.n, **f32) for _ in range(2)]
        self.pi = [torch.empty(self.n, **f32) for _ in range(2)] if self.cx else None
        self.chi = [torch.empty(self.n, **f32) for _ in range(2)]
        self.cur = 0
        self.damp = False
        c = config
        self.common = (float(c.dt) ** 2, float(c.kappa), float(c.lambda_self), float(c.chi0),
                       float(c.e0_sq))

    # the slot tensors of time level i, in the order of a state buffer
    def slots(self, i: int) -> list:
        return [self.pr[i], self.pi[i] if self.cx else None, self.chi[i]]

    def new_state_buffers(self) -> list:
        f32 = dict(dtype=torch.float32, device=self.device)
        return [torch.empty(self.n, **f32), torch.empty(self.n, **f32) if self.cx else None,
                torch.empty(self.n, **f32)]

    def chi32(self, st, k: int):
        """chi of a state buffer as the float32 array the adjoint step linearises at."""
        return st[2]

    # state in the reference representation <-> resident slots
    def load(self, state) -> None:
        self.cur, self.damp = 0, False  # prev slots hold the reference prev (already damped)
        self.pr[0].copy_(state[0].reshape(-1))
        self.pr[1].copy_(state[1].reshape(-1))
        if self.cx:
            self.pi[0].copy_(state[2].reshape(-1))
            self.pi[1].copy_(state[3].reshape(-1))
        self.chi[0].copy_(state[4].reshape(-1))
        self.chi[1].copy_(state[5].reshape(-1))

    def state(self) -> list:
        c, p = self.cur, 1 - self.cur
        damp = (lambda t: t * self.absorb) if self.damp else (lambda t: t.clone())  # noqa: E731
        out = [self.pr[c].clone(), damp(self.pr[p]), None, None, self.chi[c].clone(),
               self.chi[p].clone()]
        if self.cx:
            out[2], out[3] = self.pi[c].clone(), damp(self.pi[p])
        return out

    def step(self) -> None:
        c, p = self.cur, 1 - self.cur
        stream = _stream_handle(self.device)
        tab, desc = self.table.data_ptr(), ctypes.byref(self.desc)
        if self.cx:
            _lib.call("lfm_leapfrog_complex_f32", self.pr[c].data_ptr(), self.pr[p].data_ptr(),
                      self.pi[c].data_ptr(), self.pi[p].data_ptr(), self.chi[c].data_ptr(),
                      self.chi[p].data_ptr(), tab, desc, int(self.damp), self.N, *self.common,
                      float(self.config.epsilon_w), stream)
        else:
            _lib.call("lfm_leapfrog_real_f32", self.pr[c].data_ptr(), self.pr[p].data_ptr(),
                      self.chi[c].data_ptr(), self.chi[p].data_ptr(), tab, desc, int(self.damp),
                      self.N, *self.common, stream)
        self.cur = p
        self.damp = True

    def advance(self, cur, prev, out, damp: bool) -> None:
        """One step out of place: cur / prev / out are (psi_r, psi_i, chi) triples
        (psi_i None at REAL); the new fields go to `out` (lfm_advance_f32)."""
        ptr = lambda t: None if t is None else t.data_ptr()  # noqa: E731
        _lib.call("lfm_advance_f32", int(self.level), cur[0].data_ptr(), prev[0].data_ptr(),
                  out[0].data_ptr(), ptr(cur[1]), ptr(prev[1]), ptr(out[1]), cur[2].data_ptr(),
                  prev[2].data_ptr(), out[2].data_ptr(), self.table.data_ptr(),
                  ctypes.byref(self.desc), int(damp), self.N, *self.common,
                  float(self.config.epsilon_w), _stream_handle(self.device))

    def adjoint_step(self, st, nx, g_out, g_in) -> None:
        """The gradient back through the step from state buffer st to nx."""
        ptr = lambda t: None if t is None else t.data_ptr()  # noqa: E731
        go = (ctypes.c_void_p * 6)(*[ptr(t) for t in g_out])
        gi = (ctypes.c_void_p * 6)(*[ptr(t) for t in g_in])
        _lib.call("lfm_adjoint_step_f32", int(self.level), st[0].data_ptr(), ptr(st[1]),
                  self.chi32(st, 0).data_ptr(), self.chi32(nx, 1).data_ptr(),
                  self.table.data_ptr(),
                  ctypes.byref(self.desc), go, gi, self.N, *self.common,
                  float(self.config.epsilon_w), _stream_handle(self.device))


class _SplitLattice(_Lattice):
    """The same lattice with chi held as chi0 + hi + lo (the split-chi step,
    lfm_leapfrog_*_split_f32): the forward and the recomputed segments carry
    chi to about 48 bits, and chi comes out in float64.  A state buffer is
    (psi_r, psi_i, hi, lo); the adjoint step linearises at chi0 + hi rounded to
    float32 (within one ulp of chi), the same float32 arithmetic as for the
    plain step.  It finds cells held by the
    clamp chi >= -chi0 from that float32 chi, so a clamped cell may be missed
    (the packets of the adjoint workload stay far from the clamp)."""

    def __init__(self, config, backend: B200Backend) -> None:
        super().__init__(config, backend)
        f32 = dict(dtype=torch.float32, device=self.device)
        self.lo = [torch.empty(self.n, **f32) for _ in range(2)]
        self.chi_f32 = [torch.empty(self.n, **f32) for _ in range(2)]
        self.chi0 = float(config.chi0)

    def slots(self, i: int) -> list:
        return [self.pr[i], self.pi[i] if self.cx else None, self.chi[i], self.lo[i]]

    def new_state_buffers(self) -> list:
        return super().new_state_buffers() + [
            torch.empty(self.n, dtype=torch.float32, device=self.device)]

    def chi32(self, st, k: int):
        # chi0 + hi in float32: within one ulp of float32(chi0 + hi + lo), one launch
        return torch.add(st[2], self.chi0, out=self.chi_f32[k])

    def _split(self, chi, hi, lo) -> None:
        d = chi.reshape(-1).to(torch.float64) - self.chi0
        h = d.to(torch.float32)
        hi.copy_(h)
        lo.copy_(d - h.double())

    def _chi64(self, hi, lo):
        return self.chi0 + hi.double() + lo.double()

    def load(self, state) -> None:
        super().load([state[0], state[1], state[2], state[3], state[4].float(),
                      state[5].float()])
        self._split(state[4], self.chi[0], self.lo[0])
        self._split(state[5], self.chi[1], self.lo[1])

    def state(self) -> list:
        out = super().state()
        c, p = self.cur, 1 - self.cur
        out[4] = self._chi64(self.chi[c], self.lo[c])
        out[5] = self._chi64(self.chi[p], self.lo[p])
        return out

    def _split_step(self, cur, prev_io, damp: bool) -> None:
        """One split step: reads cur and prev_io (slot lists), writes the new state over
        prev_io."""
        stream = _stream_handle(self.device)
        tab, desc = self.table.data_ptr(), ctypes.byref(self.desc)
        if self.cx:
            _lib.call("lfm_leapfrog_complex_split_f32", cur[0].data_ptr(),
                      prev_io[0].data_ptr(), cur[1].data_ptr(), prev_io[1].data_ptr(),
                      cur[2].data_ptr(), prev_io[2].data_ptr(), cur[3].data_ptr(),
                      prev_io[3].data_ptr(), tab, desc, int(damp), self.N, *self.common,
                      float(self.config.epsilon_w), stream)
        else:
            _lib.call("lfm_leapfrog_real_split_f32", cur[0].data_ptr(), prev_io[0].data_ptr(),
                      cur[2].data_ptr(), prev_io[2].data_ptr(), cur[3].data_ptr(),
                      prev_io[3].data_ptr(), tab, desc, int(damp), self.N, *self.common,
                      stream)

    def step(self) -> None:
        c, p = self.cur, 1 - self.cur
        self._split_step(self.slots(c), self.slots(p), self.damp)
        self.cur = p
        self.damp = True

    def advance(self, cur, prev, out, damp: bool) -> None:
        """One split step out of place (lfm_advance_split_f32)."""
        ptr = lambda t: None if t is None else t.data_ptr()  # noqa: E731
        args = []
        for f in range(4):
            args += [ptr(cur[f]), ptr(prev[f]), ptr(out[f])]
        _lib.call("lfm_advance_split_f32", int(self.level), *args, self.table.data_ptr(),
                  ctypes.byref(self.desc), int(damp), self.N, *self.common,
                  float(self.config.epsilon_w), _stream_handle(self.device))


class _Plan:
    """Buffers and captured CUDA graphs of one (steps, every) schedule.

    The first forward / backward of a plan runs eagerly and then captures
    itself; later calls replay one graph each (all buffers stay put).
    """

    def __init__(self, lat: _Lattice, steps: int, every: int) -> None:
        self.lat, self.steps, self.every = lat, steps, every
        n = lat.n
        f32 = dict(dtype=torch.float32, device=lat.device)

        # checkpoint k: the (current, previous) slot buffers before step k*every
        self.snaps = [(lat.new_state_buffers(), lat.new_state_buffers())
                      for _ in range(math.ceil(steps / every))]
        self.meta = [False] * len(self.snaps)  # damp flag of each checkpoint
        # recomputed states 1 .. every of a segment (state 0 is the checkpoint)
        self.seg = [lat.new_state_buffers() for _ in range(every)]
        self.g = [[None if (not lat.cx and f in (2, 3)) else torch.zeros(n, **f32)
                   for f in range(6)] for _ in range(2)]
        self.fwd_graph = None
        self.bwd_graph = None
        self.busy = False

    # ---- bodies (run eagerly or under capture) ----
    def forward_body(self) -> None:
        lat = self.lat
        lat.cur, lat.damp = 0, False
        for t in range(self.steps):
            if t % self.every == 0:
                k = t // self.every
                cur, prev = self.snaps[k]
                c, p = lat.cur, 1 - lat.cur
                for dst, src in ((cur, lat.slots(c)), (prev, lat.slots(p))):
                    for d, x in zip(dst, src):
                        if d is not None:
                            d.copy_(x)
                self.meta[k] = lat.damp
            lat.step()

    def backward_body(self) -> int:
        """Adjoint from g[0]; returns the index of the buffer set holding the result.

        Each segment is recomputed out of place from its checkpoint straight
        into the segment buffers (no copies), then walked backwards."""
        lat, every, steps = self.lat, self.every, self.steps
        cur = 0
        for si in range(len(self.snaps) - 1, -1, -1):
            s0 = si * every
            e0 = min(s0 + every, steps)
            c0, p0 = self.snaps[si]
            states = [c0] + self.seg[: e0 - s0]
            for t in range(s0, e0):
                u = t - s0
                lat.advance(states[u], p0 if u == 0 else states[u - 1], states[u + 1],
                            self.meta[si] if u == 0 else True)
            for t in range(e0 - 1, s0 - 1, -1):
                lat.adjoint_step(states[t - s0], states[t - s0 + 1], self.g[cur],
                                 self.g[1 - cur])
                cur = 1 - cur
        return cur

    # ---- drivers ----
    def run_forward(self) -> None:
        if self.fwd_graph is not None:
            self.fwd_graph.replay()
            self.lat.cur, self.lat.damp = self._fwd_end
            return
        self.forward_body()
        self._fwd_end = (self.lat.cur, self.lat.damp)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.forward_body()
        self.fwd_graph = g

    def run_backward(self) -> int:
        if self.bwd_graph is not None:
            self.bwd_graph.replay()
            return self._bwd_out
        self._bwd_out = self.backward_body()
        # capture overwrites nothing: the result is already in g[_bwd_out]
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.backward_body()
        self.bwd_graph = g
        return self._bwd_out


class LeapfrogFunction(torch.autograd.Function):
    """(psi_r, psi_r_prev, psi_i, psi_i_prev, chi, chi_prev) -> the same after `steps` steps.

    At the REAL level psi_i / psi_i_prev are passed as None and come back None.
    """

    @staticmethod
    def forward(ctx, plan: _Plan, *state):
        lat = plan.lat
        plan.busy = True
        lat.load([s.detach() if s is not None else None for s in state])
        plan.run_forward()
        ctx.plan = plan
        out = lat.state()
        return tuple(None if o is None else o.reshape(lat.N, lat.N, lat.N) for o in out)

    @staticmethod
    def backward(ctx, *grads):
        plan = ctx.plan
        lat = plan.lat
        g0 = plan.g[0]
        for f in range(6):
            if g0[f] is None:
                continue
            if grads[f] is None:
                g0[f].zero_()
            else:
                g0[f].copy_(grads[f].reshape(-1))
        res = plan.run_backward()
        out = tuple(None if t is None else t.clone().reshape(lat.N, lat.N, lat.N)
                    for t in plan.g[res])
        plan.busy = False
        ctx.plan = None
        return (None,) + out


_LATTICES: dict = {}


def _lattice_for(config, be: B200Backend, split_chi: bool = False) -> _Lattice:
    c = config
    key = (str(be.device), int(c.grid_size), int(c.field_level), float(c.boundary_fraction),
           float(c.dt), float(c.kappa), float(c.lambda_self), float(c.chi0), float(c.e0_sq),
           float(c.epsilon_w), bool(split_chi))
    lat = _LATTICES.get(key)
    if lat is None:
        lat = _LATTICES[key] = (_SplitLattice if split_chi else _Lattice)(config, be)
        lat.plans = {}
    return lat


def _plan_for(lat: _Lattice, steps: int, every: int) -> _Plan:
    plan = lat.plans.get((steps, every))
    if plan is None:
        plan = lat.plans[(steps, every)] = _Plan(lat, steps, every)
    if plan.busy:  # a forward whose backward has not run yet holds the cached plan
        return _Plan(lat, steps, every)
    return plan


def leapfrog(config, state, steps: int, every: int | None = None, backend="auto",
             split_chi: bool = False):
    """Differentiable `steps` leapfrog steps of a REAL/COMPLEX state.

    state: six tensors (N, N, N) float32 on the device in the reference
    representation (psi_i, psi_i_prev None at the REAL level).  Returns the
    six tensors after the steps.  every: steps between checkpoints
    (default ceil(sqrt(steps))).  Buffers and CUDA graphs are cached per
    lattice and schedule, so repeated calls (an optimisation loop) replay
    one graph for the forward and one for the backward.

    split_chi: step with chi held as chi0 + hi + lo (the split-chi step) in
    the forward and in the recomputed segments; chi and chi_prev may then be
    given in float64 and come back in float64, so a loss on chi keeps about
    48 bits.  The adjoint step is the same float32 one.
    """
    be = backend if isinstance(backend, B200Backend) else get_backend(backend)
    lat = _lattice_for(config, be, split_chi)
    steps = int(steps)
    if steps < 1:
        raise ValueError("steps must be >= 1")
    every = int(every or math.ceil(math.sqrt(steps)))
    every = max(1, min(every, steps))
    if (state[2] is None) == lat.cx:
        raise ValueError("psi_i / psi_i_prev must be given exactly at the COMPLEX level")
    needs_grad = torch.is_grad_enabled() and any(
        s is not None and s.requires_grad for s in state)
    if not needs_grad:
        lat.load(state)
        for _ in range(steps):
            lat.step()
        return tuple(None if o is None else o.reshape(lat.N, lat.N, lat.N) for o in lat.state())
    return LeapfrogFunction.apply(_plan_for(lat, steps, every), *state)


def memory_bytes(config, steps: int, every: int | None = None, split_chi: bool = False) -> dict:
    """Device bytes the checkpoints and the segment buffer of leapfrog() take (split_chi:
    chi's lo slots besides)."""
    n = int(config.grid_size) ** 3
    cx = int(config.field_level) == FieldLevel.COMPLEX
    every = int(every or math.ceil(math.sqrt(steps)))
    snaps = math.ceil(steps / every)
    extra = 1 if split_chi else 0
    per_snap = 2 * ((3 if cx else 2) + extra) * 4 * n
    seg = every * ((3 if cx else 2) + extra) * 4 * n
    return {"checkpoints": snaps, "checkpoint_bytes": snaps * per_snap, "segment_bytes": seg,
            "all_states_bytes": steps * (3 if cx else 2) * 4 * n}


# ------------------------------------------------------------------ initial states
def soliton_state(N: int, amplitude, centre, phase, sigma: float, chi0: float, dchi=None,
                  complex_level: bool = True, device=None, dtype=torch.float32,
                  omega_dt: float | None = None):
    """Differentiable initial state: a sum of Gaussian packets.

    amplitude (S,), centre (S, 3), phase (S,) tensors; packet s is
    amplitude_s exp(-|x - centre_s|^2 / (2 sigma^2)) e^{i phase_s} (as
    lfm/fields/soliton.py:49-59 builds them, without wrap).  chi = chi0 +
    dchi.  Without omega_dt the previous fields equal the current ones, as
    set_psi_real / set_chi leave them; with omega_dt (COMPLEX) each packet's
    previous value carries the phase phase_s + omega_dt, the rotation of a
    packet at rest that the reference's Simulation.place_soliton gives it
    (lfm/simulation.py:585-591, omega = chi0 for zero momentum).  Returns the
    six state tensors.
    """
    dev = device if device is not None else amplitude.device
    x = torch.arange(N, device=dev, dtype=dtype)
    pr = torch.zeros((N, N, N), device=dev, dtype=dtype)
    pi = torch.zeros((N, N, N), device=dev, dtype=dtype)
    prp, pip = pr, pi
    for s in range(amplitude.shape[0]):
        c = centre[s].to(dtype)
        d2 = ((x - c[0]) ** 2)[:, None, None] + ((x - c[1]) ** 2)[None, :, None] \
            + ((x - c[2]) ** 2)[None, None, :]
        env = amplitude[s].to(dtype) * torch.exp(-d2 / (2.0 * sigma * sigma))
        th = phase[s].to(dtype)
        pr = pr + env * torch.cos(th)
        pi = pi + env * torch.sin(th)
        if omega_dt is not None:
            prp = prp + env * torch.cos(th + omega_dt)
            pip = pip + env * torch.sin(th + omega_dt)
    chi = torch.full((N, N, N), float(chi0), device=dev, dtype=dtype)
    if dchi is not None:
        chi = chi + dchi.to(dtype)
    if omega_dt is None:
        prp, pip = pr, pi
    if complex_level:
        return [pr, prp, pi, pip, chi, chi]
    return [pr, prp, None, None, chi, chi]
