"""Many independent lattices stepped together on one GPU.

The reference runs a parameter sweep one ``Simulation`` after another
(lfm/sweep.py:52-82: deep-copy the config, build, run, read metrics).  Small
lattices leave most of a B200 idle that way.  ``BatchedLattices`` holds every
lattice of a sweep resident in one device arena and advances all of them with
one persistent kernel launch per step (lfm_batch_step): the CTAs take
(lattice, row tile, plane chunk) items from a work list grouped by lattice
shape (the sweep's shapes at 256 threads run with their geometry fixed at
compile time) and sorted by cost within each group, each marched exactly like
the fused single-lattice kernel, so every lattice's result is bit-for-bit the
one ``Evolver`` gives for it alone.

Lattices may differ in N (multiples of 4), level (REAL or COMPLEX), sponge
and every coupling constant.  ``evolve`` replays a captured CUDA graph of a
block of steps.  Field accessors take the lattice index first and follow the
reference ``Evolver``'s semantics (set_psi_real sets current and previous,
get_psi_real_prev returns the sponge-damped previous field).
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .backend import B200Backend, _stream_handle, get_backend
from .config import FieldLevel
from .mask import MaskTable

_ALIGN = 64  # floats: every slot starts on a 256-byte boundary


class BatchedLattices:
    """REAL / COMPLEX lattices of mixed sizes, one persistent launch per step."""

    graph_block = 16
    """Steps per captured CUDA graph (an even number)."""

    def __init__(self, configs, backend="auto", tuning: dict | str | None = None) -> None:
        """configs: SimulationConfig per lattice.  tuning: None (defaults), a dict
        of lfm_batch_tuning fields, or "auto" (lfm_b200.autotune.tune_batch,
        cached per device and (N, level) mix)."""
        import torch

        self.configs = list(configs)
        if not self.configs:
            raise ValueError("empty batch")
        self.backend = backend if isinstance(backend, B200Backend) else get_backend(backend)
        self.device = self.backend.device
        self.step = 0
        for i, c in enumerate(self.configs):
            lv = FieldLevel(int(c.field_level))
            if lv == FieldLevel.COLOR:
                raise ValueError(f"lattice {i}: batches hold REAL and COMPLEX lattices")
            if c.grid_size % 4:
                raise ValueError(f"lattice {i}: N={c.grid_size} is not a multiple of 4")
        # one arena: per lattice [pr0, pr1, chi0, chi1 (, pi0, pi1)]
        offs, total = [], 0
        for c in self.configs:
            n = int(c.grid_size) ** 3
            nf = 6 if int(c.field_level) == FieldLevel.COMPLEX else 4
            slots = []
            for _ in range(nf):
                slots.append(total)
                total += -(-n // _ALIGN) * _ALIGN
            offs.append(slots)
        self._arena = torch.empty(total, dtype=torch.float32, device=self.device)
        self._pr, self._pi, self._chi = [], [], []
        for c, slots in zip(self.configs, offs):
            n = int(c.grid_size) ** 3
            v = [self._arena[o:o + n] for o in slots]
            v[0].zero_(); v[1].zero_()
            v[2].fill_(float(c.chi0)); v[3].fill_(float(c.chi0))
            self._pr.append(v[0:2])
            self._chi.append(v[2:4])
            if len(v) == 6:
                v[4].zero_(); v[5].zero_()
                self._pi.append(v[4:6])
            else:
                self._pi.append(None)
        # sponge tables, shared between lattices of one (N, boundary_fraction)
        self._tables: dict[tuple, tuple] = {}
        self._descs = (_lib.LatticeDesc * len(self.configs))()
        for i, c in enumerate(self.configs):
            key = (int(c.grid_size), float(c.boundary_fraction))
            if key not in self._tables:
                t = MaskTable.for_lattice(*key)
                self._tables[key] = (t, t.to_device(self.device), None)
            t, tdev, _ = self._tables[key]
            d = self._descs[i]
            d.N = int(c.grid_size)
            d.level = int(c.field_level)
            for s in range(2):
                d.psi_r[s] = self._pr[i][s].data_ptr()
                d.chi[s] = self._chi[i][s].data_ptr()
                d.psi_i[s] = self._pi[i][s].data_ptr() if self._pi[i] is not None else None
            d.mask_table = tdev.data_ptr()
            d.lut = t.desc
            d.dt2 = float(c.dt) ** 2
            d.kappa = float(c.kappa)
            d.lambda_self = float(c.lambda_self)
            d.chi0 = float(c.chi0)
            d.e0_sq = float(c.e0_sq)
            d.epsilon_w = float(c.epsilon_w)
        self._handle = None
        self._cur = 0
        self._damp = False
        self._graphs: dict = {}
        self.tune_report = None
        if tuning == "auto":
            from .autotune import tune_batch

            self.retune(None)
            self.tune_report = tune_batch(self)
        else:
            self.retune(tuning)

    def retune(self, tuning: dict | None) -> None:
        """Re-plan the work list with another tuning (keys of lfm_batch_tuning:
        threads, stages, item_cells, ctas_per_sm; missing or 0 = default).
        The fields are untouched; captured graphs are dropped."""
        t = _lib.BatchTuning()
        for k, v in (tuning or {}).items():
            setattr(t, k, int(v))
        h = ctypes.c_void_p()
        _lib.call("lfm_batch_create", self._descs, len(self.configs), ctypes.byref(t),
                  ctypes.byref(h))
        self._graphs = {}
        if self._handle:
            _lib.load().lfm_batch_destroy(self._handle)
        self._handle = h
        self._tuning = {f: getattr(t, f) for f, _ in t._fields_}

    def __len__(self) -> int:
        return len(self.configs)

    def close(self) -> None:
        self._graphs.clear()
        if getattr(self, "_handle", None):
            _lib.load().lfm_batch_destroy(self._handle)
            self._handle = None

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- plan
    def info(self) -> dict:
        """Launch shape: work items, threads per CTA, persistent CTAs, shared memory."""
        v = [ctypes.c_int(0) for _ in range(4)]
        _lib.call("lfm_batch_info", self._handle, *[ctypes.byref(x) for x in v])
        return dict(zip(("items", "threads", "grid", "smem"), (x.value for x in v)))

    # ---------------------------------------------------------------- stepping
    def _step(self) -> None:
        _lib.call("lfm_batch_step", self._handle, self._cur, 1 if self._damp else 0,
                  _stream_handle(self.device))
        self._cur = 1 - self._cur
        self._damp = True

    def _block_graph(self, steps: int):
        import torch

        key = (self._cur, steps)
        g = self._graphs.get(key)
        if g is None:
            saved = (self._cur, self._damp)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                for _ in range(steps):
                    self._step()
            self._cur, self._damp = saved
            self._graphs[key] = g
        return g

    def warm_graphs(self) -> None:
        """Capture the step-block graphs now (nothing runs); needs one step done."""
        if not self._damp:
            return
        saved = self._cur
        for c in (0, 1):
            self._cur = c
            self._block_graph(self.graph_block)
            self._block_graph(2)
        self._cur = saved

    def evolve(self, steps: int, use_graph: bool = True) -> None:
        """Advance every lattice by `steps` steps."""
        steps = int(steps)
        if not use_graph or steps < 4:
            for _ in range(steps):
                self._step()
            self.step += steps
            return
        if not self._damp:
            self._step()  # the first step after a host write does not damp prev
            steps -= 1
            self.step += 1
        blk = self.graph_block
        while steps >= blk:
            self._block_graph(blk).replay()
            steps -= blk
            self.step += blk
        while steps >= 2:
            self._block_graph(2).replay()
            steps -= 2
            self.step += 2
        if steps:
            self._step()
            self.step += 1

    # ---------------------------------------------------------------- accessors
    def _n(self, i: int) -> int:
        return int(self.configs[i].grid_size)

    def _absorb(self, i: int):
        c = self.configs[i]
        key = (int(c.grid_size), float(c.boundary_fraction))
        t, tdev, absorb = self._tables[key]
        if absorb is None:
            absorb = 1.0 - t.device_mask(self.device)
            self._tables[key] = (t, tdev, absorb)
        return absorb

    def _materialize_prev(self) -> None:
        """Apply the pending sponge factor to every stored previous Psi."""
        if not self._damp:
            return
        p = 1 - self._cur
        for i in range(len(self)):
            a = self._absorb(i)
            self._pr[i][p].mul_(a)
            if self._pi[i] is not None:
                self._pi[i][p].mul_(a)
        self._damp = False

    def _dev(self, i: int, arr):
        import torch

        n = self._n(i) ** 3
        if isinstance(arr, torch.Tensor):
            t = arr.detach().reshape(-1).to(self.device, dtype=torch.float32)
        else:
            t = torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float32).ravel()).to(
                self.device)
        if t.numel() != n:
            raise ValueError(f"lattice {i}: got {t.numel()} values, expected {n}")
        return t

    def _host(self, i: int, t) -> np.ndarray:
        N = self._n(i)
        host = t.detach().to("cpu").numpy().reshape(N, N, N)
        _lib.check_device("BatchedLattices read", self.device)
        return host

    def _imag(self, i: int):
        if self._pi[i] is None:
            raise ValueError("Cannot set imaginary part for REAL field level")
        return self._pi[i]

    def set_psi_real(self, i: int, arr) -> None:
        """Current and previous Psi_real of lattice i."""
        self._materialize_prev()
        t = self._dev(i, arr)
        self._pr[i][self._cur].copy_(t)
        self._pr[i][1 - self._cur].copy_(t)

    def set_psi_imag(self, i: int, arr) -> None:
        self._materialize_prev()
        t = self._dev(i, arr)
        s = self._imag(i)
        s[self._cur].copy_(t)
        s[1 - self._cur].copy_(t)

    def set_psi_real_prev(self, i: int, arr) -> None:
        self._materialize_prev()
        self._pr[i][1 - self._cur].copy_(self._dev(i, arr))

    def set_psi_imag_prev(self, i: int, arr) -> None:
        self._materialize_prev()
        self._imag(i)[1 - self._cur].copy_(self._dev(i, arr))

    def set_chi(self, i: int, arr) -> None:
        """Current and previous chi of lattice i."""
        self._materialize_prev()
        t = self._dev(i, arr)
        self._chi[i][self._cur].copy_(t)
        self._chi[i][1 - self._cur].copy_(t)

    def get_psi_real(self, i: int) -> np.ndarray:
        return self._host(i, self._pr[i][self._cur])

    def get_psi_imag(self, i: int):
        return None if self._pi[i] is None else self._host(i, self._pi[i][self._cur])

    def get_chi(self, i: int) -> np.ndarray:
        return self._host(i, self._chi[i][self._cur])

    def _prev(self, i: int, slots):
        buf = slots[1 - self._cur]
        return buf * self._absorb(i) if self._damp else buf

    def get_psi_real_prev(self, i: int) -> np.ndarray:
        return self._host(i, self._prev(i, self._pr[i]))

    def get_psi_imag_prev(self, i: int):
        return None if self._pi[i] is None else self._host(i, self._prev(i, self._pi[i]))

    def device_state(self, i: int) -> dict:
        N = self._n(i)
        shp = (N, N, N)
        out = {"psi_r": self._pr[i][self._cur].reshape(shp),
               "psi_r_prev": self._prev(i, self._pr[i]).reshape(shp),
               "chi": self._chi[i][self._cur].reshape(shp)}
        if self._pi[i] is not None:
            out["psi_i"] = self._pi[i][self._cur].reshape(shp)
            out["psi_i_prev"] = self._prev(i, self._pi[i]).reshape(shp)
        return out

    def metrics(self, i: int) -> dict:
        """Float64 metrics of lattice i (lfm_metrics_f64), as Evolver.metrics."""
        from .metrics import device_metrics

        st = self.device_state(i)
        c = self.configs[i]
        return device_metrics(self.backend.context.handle, int(c.field_level), self._n(i),
                              st["psi_r"], st["psi_r_prev"].contiguous(), st.get("psi_i"),
                              None if "psi_i_prev" not in st else st["psi_i_prev"].contiguous(),
                              st["chi"], c.dt, getattr(c, "c", 1.0), c.boundary_fraction)

    def metrics_all(self) -> list[dict]:
        return [self.metrics(i) for i in range(len(self))]


def plan(configs, tuning: dict | None = None, sms: int = 148) -> dict:
    """The work list lfm_batch_create would build for these configs (host only, no device).

    Returns {"items": int32 array (n, 6) of (level, lattice, j0, j1, i0, i1),
    "launch": (threads, smem, grid)}.
    """
    descs = (_lib.LatticeDesc * len(configs))()
    for i, c in enumerate(configs):
        descs[i].N = int(c.grid_size)
        descs[i].level = int(c.field_level)
    t = _lib.BatchTuning()
    for k, v in (tuning or {}).items():
        setattr(t, k, int(v))
    lib = _lib.load()
    n = ctypes.c_int(0)
    _lib.check(lib.lfm_batch_plan(descs, len(configs), ctypes.byref(t), int(sms), None, 0,
                                  ctypes.byref(n), None), "lfm_batch_plan")
    items = np.zeros((max(n.value, 1), 6), dtype=np.int32)
    launch = np.zeros(3, dtype=np.int32)
    i32p = ctypes.POINTER(ctypes.c_int32)
    _lib.check(lib.lfm_batch_plan(descs, len(configs), ctypes.byref(t), int(sms),
                                  items.ctypes.data_as(i32p), items.shape[0], ctypes.byref(n),
                                  launch.ctypes.data_as(i32p)), "lfm_batch_plan")
    return {"items": items[:n.value],
            "launch": tuple(int(x) for x in launch)}
