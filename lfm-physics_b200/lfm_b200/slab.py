"""One lattice split along i across GPUs (slab decomposition).

The reference steps a whole lattice on one device
(lfm/core/backends/numpy_backend.py:80-205, through lfm/core/evolver.py).
A lattice too large or too slow for one GPU is split into contiguous slabs of
i-planes, one per rank.  Each rank keeps its planes plus one ghost plane on
each side (the 19-point stencil reaches only i +- 1) and steps them with
lfm_slab_step_f32, which gives the whole-lattice step's bits on its planes.
After every step the ghost planes of the new fields are refreshed from the
neighbouring slabs: one plane per stencil field per side (psi_r, psi_i, chi),
sent with ``torch.distributed`` point-to-point operations (NCCL over NVLink
between GPUs; gloo on CPU for the tests).  There is no other communication
while stepping.  With ``overlap`` (the default across ranks) a step runs the
two boundary planes first (lfm_slab_step_planes_f32), starts their exchange,
and steps the interior planes while it is in flight: the interior reads no
ghost plane and writes none, so the exchange and the interior arithmetic
proceed side by side and the step waits only for whichever ends last.

Field accessors take and return the whole lattice (every rank passes the same
host array to the setters, as each would to the reference's Evolver); getters
gather the slabs on every rank.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .config import FieldLevel

TAG_DOWN, TAG_UP = 0, 1  # plane 1 -> previous rank's upper ghost; plane n -> next's lower ghost


def split_planes(N: int, world: int) -> list[tuple[int, int]]:
    """(first global plane, plane count) of every rank: contiguous, the first
    N % world ranks one plane larger."""
    if world < 1 or world > N:
        raise ValueError(f"cannot split {N} planes over {world} ranks")
    base, rem = divmod(N, world)
    out, first = [], 0
    for r in range(world):
        n = base + (1 if r < rem else 0)
        out.append((first, n))
        first += n
    return out


class SlabEvolver:
    """The planes [i_first, i_first + n_local) of one lattice, with ghost planes.

    rank / world default to torch.distributed's when it is initialised, else
    0 / 1 (then the ghosts are the slab's own wrapped planes).  stepper(slab,
    lo, hi) replaces the CUDA step of the local planes [lo, hi) (tests of the
    decomposition on the CPU); exchange replaces the ghost refresh.  Slabs held
    by one process are stepped with evolve_local.
    """

    overlap = True
    """Across ranks: boundary planes, then their exchange beside the interior planes."""

    def __init__(self, config, backend="auto", rank: int | None = None,
                 world: int | None = None, group=None, device=None, stepper=None,
                 exchange=None) -> None:
        import torch

        self.config = config
        self.level = FieldLevel(int(config.field_level))
        if self.level == FieldLevel.COLOR:
            raise ValueError("slabs hold REAL and COMPLEX lattices (COLOR's S_a needs the "
                             "whole lattice's FFT)")
        self.N = N = int(config.grid_size)
        dist = _dist()
        self.group = group
        if rank is None:
            rank = dist.get_rank(group) if dist else 0
        if world is None:
            world = dist.get_world_size(group) if dist else 1
        self.rank, self.world = int(rank), int(world)
        self.i_first, self.n_local = split_planes(N, self.world)[self.rank]
        self.cx = self.level == FieldLevel.COMPLEX
        self._stepper = stepper
        self._exchange_fn = exchange
        self.backend = None
        if stepper is None:
            from .backend import B200Backend, get_backend
            from .mask import MaskTable

            self.backend = backend if isinstance(backend, B200Backend) else get_backend(backend)
            device = self.backend.device
            t = MaskTable.for_lattice(N, config.boundary_fraction)
            self._table = t.to_device(device)
            self._desc = t.desc
        self.device = torch.device(device) if device is not None else torch.device("cpu")
        shape = (self.n_local + 2, N, N)
        f32 = dict(dtype=torch.float32, device=self.device)
        self.pr = [torch.zeros(shape, **f32) for _ in range(2)]
        self.pi = [torch.zeros(shape, **f32) for _ in range(2)] if self.cx else None
        self.chi = [torch.full(shape, float(config.chi0), **f32) for _ in range(2)]
        self.cur = 0
        self.damp = False
        self.step = 0

    # ---------------------------------------------------------------- neighbours
    @property
    def prev_rank(self) -> int:
        return (self.rank - 1) % self.world

    @property
    def next_rank(self) -> int:
        return (self.rank + 1) % self.world

    def _global_planes(self) -> np.ndarray:
        """Global indices of the array's planes, ghosts included."""
        return (np.arange(self.i_first - 1, self.i_first + self.n_local + 1)) % self.N

    def stencil_fields(self, slot: int) -> list:
        """The fields whose neighbours the step reads, in the given slot."""
        out = [self.pr[slot], self.chi[slot]]
        if self.cx:
            out.insert(1, self.pi[slot])
        return out

    # ---------------------------------------------------------------- stepping
    def _step_planes(self, lo: int, hi: int) -> None:
        """Step the local planes [lo, hi) (1 <= lo < hi <= n_local + 1)."""
        if self._stepper is not None:
            self._stepper(self, lo, hi)
            return
        from .backend import _stream_handle

        c, p = self.cur, 1 - self.cur
        cfg = self.config
        ptr = lambda t: None if t is None else t.data_ptr()  # noqa: E731
        _lib.call("lfm_slab_step_planes_f32", int(self.level), self.pr[c].data_ptr(),
                  self.pr[p].data_ptr(), ptr(self.pi[c] if self.cx else None),
                  ptr(self.pi[p] if self.cx else None), self.chi[c].data_ptr(),
                  self.chi[p].data_ptr(), self._table.data_ptr(), ctypes.byref(self._desc),
                  1 if self.damp else 0, self.N, self.n_local, self.i_first, int(lo), int(hi),
                  float(cfg.dt) ** 2, float(cfg.kappa), float(cfg.lambda_self),
                  float(cfg.chi0), float(cfg.e0_sq), float(cfg.epsilon_w),
                  _stream_handle(self.device))

    def _step_local(self) -> None:
        self._step_planes(1, self.n_local + 1)

    def _start_exchange(self, slot: int) -> list:
        """Post the ghost refresh of the fields in `slot`; returns the requests."""
        import torch.distributed as dist

        n = self.n_local
        ops = []
        for f in self.stencil_fields(slot):
            ops.append(dist.P2POp(dist.isend, f[1], self.prev_rank, self.group, TAG_DOWN))
            ops.append(dist.P2POp(dist.isend, f[n], self.next_rank, self.group, TAG_UP))
            ops.append(dist.P2POp(dist.irecv, f[n + 1], self.next_rank, self.group, TAG_DOWN))
            ops.append(dist.P2POp(dist.irecv, f[0], self.prev_rank, self.group, TAG_UP))
        return dist.batch_isend_irecv(ops)

    def exchange(self) -> None:
        """Refresh the ghost planes of the current fields from the neighbours."""
        if self._exchange_fn is not None:
            self._exchange_fn(self)
            return
        n = self.n_local
        if self.world == 1:
            for f in self.stencil_fields(self.cur):
                f[0].copy_(f[n])
                f[n + 1].copy_(f[1])
            return
        for req in self._start_exchange(self.cur):
            req.wait()

    def advance(self, exchange: bool = True) -> None:
        """One step of this slab, then (unless told not to) the ghost refresh; across
        ranks with ``overlap``, the refresh runs beside the interior planes."""
        n = self.n_local
        if (exchange and self.overlap and self.world > 1 and n >= 3
                and self._exchange_fn is None):
            p = 1 - self.cur
            self._step_planes(1, 2)
            self._step_planes(n, n + 1)
            reqs = self._start_exchange(p)  # the new boundary planes, in slot p
            self._step_planes(2, n)
            for req in reqs:
                req.wait()
            self.cur = p
            self.damp = True
            self.step += 1
            return
        self._step_local()
        self.cur = 1 - self.cur
        self.damp = True
        self.step += 1
        if exchange:
            self.exchange()

    def evolve(self, steps: int) -> None:
        for _ in range(int(steps)):
            self.advance()

    # ---------------------------------------------------------------- accessors
    def _planes_of(self, arr):
        import torch

        a = np.asarray(arr, dtype=np.float32).reshape(self.N, self.N, self.N)
        return torch.from_numpy(np.ascontiguousarray(a[self._global_planes()])).to(self.device)

    def _set_both(self, slots, arr) -> None:
        if self.damp:  # the kernel damps stored prev on read: materialise it first
            self._materialise_prev()
        t = self._planes_of(arr)
        slots[self.cur].copy_(t)
        slots[1 - self.cur].copy_(t)

    def _materialise_prev(self) -> None:
        from .mask import boundary_mask

        m = boundary_mask(self.N, self.config.boundary_fraction).reshape(self.N, self.N, self.N)
        import torch

        absorb = torch.from_numpy(np.ascontiguousarray(1.0 - m[self._global_planes()])).to(
            self.device)
        p = 1 - self.cur
        self.pr[p].mul_(absorb)
        if self.cx:
            self.pi[p].mul_(absorb)
        self.damp = False

    def set_psi_real(self, arr) -> None:
        self._set_both(self.pr, arr)

    def set_psi_imag(self, arr) -> None:
        if not self.cx:
            raise ValueError("Cannot set imaginary part for REAL field level")
        self._set_both(self.pi, arr)

    def set_chi(self, arr) -> None:
        self._set_both(self.chi, arr)

    def local(self, field: str):
        """This slab's own planes (no ghosts) of the current field, a device view."""
        src = {"psi_r": self.pr, "psi_i": self.pi, "chi": self.chi}[field]
        return src[self.cur][1:self.n_local + 1]

    def gather(self, field: str) -> np.ndarray:
        """The whole lattice's current field on every rank, (N, N, N) float32."""
        mine = self.local(field).detach().to("cpu").numpy()
        if self.device.type == "cuda":
            _lib.check_device("SlabEvolver.gather", self.device)
        if self.world == 1 or self._exchange_fn is not None:
            return mine
        import torch.distributed as dist

        parts: list = [None] * self.world
        dist.all_gather_object(parts, (self.i_first, mine), group=self.group)
        out = np.empty((self.N, self.N, self.N), np.float32)
        for first, block in parts:
            out[first:first + block.shape[0]] = block
        return out

    def get_psi_real(self) -> np.ndarray:
        return self.gather("psi_r")

    def get_psi_imag(self):
        return self.gather("psi_i") if self.cx else None

    def get_chi(self) -> np.ndarray:
        return self.gather("chi")


def exchange_local(slabs: list, new: bool = False) -> None:
    """Ghost refresh between slabs held by one process (the ring of ranks
    0 .. world-1, all on one device or on devices of this process), of the
    current fields, or with ``new`` of the fields a step is writing."""
    world = len(slabs)
    slot = (lambda t: 1 - t.cur) if new else (lambda t: t.cur)  # noqa: E731
    for r, s in enumerate(slabs):
        nxt, prv = slabs[(r + 1) % world], slabs[(r - 1) % world]
        n = s.n_local
        for f, fn, fp in zip(s.stencil_fields(slot(s)), nxt.stencil_fields(slot(nxt)),
                             prv.stencil_fields(slot(prv))):
            f[n + 1].copy_(fn[1])
            f[0].copy_(fp[prv.n_local])


def evolve_local(slabs: list, steps: int, overlap: bool = False) -> None:
    """Step slabs held by one process together: every slab, then one ghost
    refresh among them, per step.  With ``overlap`` each step runs the order
    of the overlapped advance (boundary planes, refresh, interior planes)."""
    for _ in range(int(steps)):
        if overlap and all(s.n_local >= 3 for s in slabs):
            for s in slabs:
                s._step_planes(1, 2)
                s._step_planes(s.n_local, s.n_local + 1)
            exchange_local(slabs, new=True)
            for s in slabs:
                s._step_planes(2, s.n_local)
                s.cur = 1 - s.cur
                s.damp = True
                s.step += 1
            continue
        for s in slabs:
            s.advance(exchange=False)
        exchange_local(slabs)


def gather_local(slabs: list, field: str) -> np.ndarray:
    """The whole lattice from slabs held by one process."""
    N = slabs[0].N
    out = np.empty((N, N, N), np.float32)
    for s in slabs:
        out[s.i_first:s.i_first + s.n_local] = s.local(field).detach().to("cpu").numpy()
        if s.device.type == "cuda":
            _lib.check_device("gather_local", s.device)
    return out


def _dist():
    try:
        import torch.distributed as dist
    except ImportError:  # pragma: no cover
        return None
    return dist if dist.is_available() and dist.is_initialized() else None
