"""Split-chi evolver: float32 Psi, chi as a two-float offset from chi0 (REAL, COMPLEX).

Same equations as :class:`lfm_b200.Evolver` and the reference backends
(lfm/core/backends/numpy_backend.py:80-205).  What limits a float32 run's
accuracy against float64 is chi itself: stored as a float32 near chi0 = 19 it
keeps about 2e-6 of absolute precision, each step's small increment is
rounded into it, and Psi's local frequency follows chi, so the errors add up
along the run.  Here chi is held as chi0 + hi + lo (two float32 slots per
time level, lo the part of the offset below one ulp of hi) and advanced in
float64 by lfm_leapfrog_*_split_f32; the Psi slots are the plain resident
ones.  36 B/cell/step at REAL, 48 B at COMPLEX.

The accessors speak the reference's representation: get_chi returns chi
rounded to float32, chi64() the float64 value on the device.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .backend import B200Backend, _stream_handle, get_backend
from .config import FieldLevel
from .mask import MaskTable


class SplitChiEvolver:
    """Leapfrog evolver with float32 Psi and a two-float chi offset, one lattice, one GPU."""

    use_graphs = True

    def __init__(self, config, backend="auto") -> None:
        import torch

        self.config = config
        self.backend = backend if isinstance(backend, B200Backend) else get_backend(backend)
        self.device = self.backend.device
        self._level = FieldLevel(int(config.field_level))
        if self._level == FieldLevel.COLOR:
            raise ValueError("the split-chi path covers the REAL and COMPLEX levels")
        self.N = int(config.grid_size)
        self.total = self.N**3
        self.step = 0
        self._has_imag = self._level == FieldLevel.COMPLEX
        n = self.total
        f32 = dict(dtype=torch.float32, device=self.device)
        self._table = MaskTable.for_lattice(self.N, config.boundary_fraction)
        self._table_dev = self._table.to_device(self.device)
        self._desc = self._table.desc
        self.boundary_mask = self._table.device_mask(self.device)
        self._absorb = 1.0 - self.boundary_mask
        z = lambda: [torch.zeros(n, **f32), torch.zeros(n, **f32)]  # noqa: E731
        self._pr = z()
        self._pi = z() if self._has_imag else None
        self._hi, self._lo = z(), z()  # chi - chi0 = hi + lo
        self._cur = 0
        self._damp = False  # the previous Psi slot already holds the damped field
        self._graphs = {}

    # ---------------------------------------------------------------- stepping
    def _step(self) -> None:
        c = self.config
        cur, prv = self._cur, 1 - self._cur
        common = (float(c.dt**2), float(c.kappa), float(c.lambda_self), float(c.chi0),
                  float(c.e0_sq))
        stream = _stream_handle(self.device)
        table, desc = self._table_dev.data_ptr(), ctypes.byref(self._desc)
        damp = 1 if self._damp else 0
        chi = (self._hi[cur].data_ptr(), self._hi[prv].data_ptr(), self._lo[cur].data_ptr(),
               self._lo[prv].data_ptr())
        if self._level == FieldLevel.REAL:
            _lib.call("lfm_leapfrog_real_split_f32", self._pr[cur].data_ptr(),
                      self._pr[prv].data_ptr(), *chi, table, desc, damp, self.N, *common, stream)
        else:
            _lib.call("lfm_leapfrog_complex_split_f32", self._pr[cur].data_ptr(),
                      self._pr[prv].data_ptr(), self._pi[cur].data_ptr(),
                      self._pi[prv].data_ptr(), *chi, table, desc, damp, self.N, *common,
                      float(c.epsilon_w), stream)
        self._cur = prv
        self._damp = True

    def _pair_graph(self):
        import torch

        c = self.config
        key = (self._cur, float(c.dt), float(c.kappa), float(c.lambda_self), float(c.chi0),
               float(c.e0_sq), float(c.epsilon_w))
        g = self._graphs.get(key)
        if g is None:
            saved = (self._cur, self._damp)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._step()
                self._step()
            self._cur, self._damp = saved
            self._graphs[key] = g
        return g

    def warm_graphs(self) -> None:
        """Capture the two-step graphs of both parities now (nothing runs).  Needs one
        step done (the first step after a host write does not damp the previous Psi)."""
        if not self._damp:
            return
        saved = self._cur
        for c in (0, 1):
            self._cur = c
            self._pair_graph()
        self._cur = saved

    def evolve(self, steps: int, callback=None) -> None:
        """Run `steps` steps; callback(evolver, step) every report_interval."""
        report = self.config.report_interval
        steps = int(steps)
        if callback is None and self.use_graphs and steps >= 4:
            if not self._damp:  # first step after a host write: no damping of prev
                self._step()
                self.step += 1
                steps -= 1
            pairs = steps // 2
            if pairs:
                g = self._pair_graph()
                for _ in range(pairs):
                    g.replay()
                self.step += 2 * pairs
            if steps % 2:
                self._step()
                self.step += 1
            return
        for _ in range(steps):
            self._step()
            self.step += 1
            if callback is not None and report > 0 and self.step % report == 0:
                callback(self, self.step)

    # ---------------------------------------------------------------- accessors
    def _dev(self, arr, dtype=None):
        import torch

        dtype = dtype or torch.float32
        if isinstance(arr, torch.Tensor):
            return arr.detach().reshape(-1).to(self.device, dtype=dtype)
        return torch.from_numpy(np.ascontiguousarray(arr).ravel()).to(self.device, dtype=dtype)

    def _host(self, t) -> np.ndarray:
        host = t.reshape(self.N, self.N, self.N).detach().to("cpu").numpy()
        _lib.check_device("SplitChiEvolver read", self.device)
        return host

    def _materialize_prev(self) -> None:
        if self._damp:
            p = 1 - self._cur
            self._pr[p].mul_(self._absorb)
            if self._has_imag:
                self._pi[p].mul_(self._absorb)
            self._damp = False

    def _split(self, chi):
        """(hi, lo) of chi - chi0 for float32 or float64 input."""
        import torch

        d = self._dev(chi, torch.float64) - float(self.config.chi0)
        hi = d.to(torch.float32)
        return hi, (d - hi.double()).to(torch.float32)

    def set_psi_real(self, arr) -> None:
        """Set the current and previous Psi_r (no velocity), as the reference's setter."""
        v = self._dev(arr)
        self._materialize_prev()
        self._pr[0].copy_(v)
        self._pr[1].copy_(v)

    def set_psi_imag(self, arr) -> None:
        if not self._has_imag:
            raise ValueError("Cannot set imaginary part for REAL field level")
        v = self._dev(arr)
        self._materialize_prev()
        self._pi[0].copy_(v)
        self._pi[1].copy_(v)

    def set_psi_real_prev(self, arr) -> None:
        self._materialize_prev()
        self._pr[1 - self._cur].copy_(self._dev(arr))

    def set_psi_imag_prev(self, arr) -> None:
        if not self._has_imag:
            raise ValueError("Cannot set imaginary part for REAL field level")
        self._materialize_prev()
        self._pi[1 - self._cur].copy_(self._dev(arr))

    def set_chi(self, arr) -> None:
        """Set the current and previous chi (float32 or float64 values)."""
        hi, lo = self._split(arr)
        for s in (0, 1):
            self._hi[s].copy_(hi)
            self._lo[s].copy_(lo)

    def set_chi_prev(self, arr) -> None:
        hi, lo = self._split(arr)
        self._hi[1 - self._cur].copy_(hi)
        self._lo[1 - self._cur].copy_(lo)

    def chi64(self, prev: bool = False):
        """chi (or the previous chi) in float64 on the device, flat."""
        s = 1 - self._cur if prev else self._cur
        return float(self.config.chi0) + self._hi[s].double() + self._lo[s].double()

    def _prev_psi(self, t):
        return t * self._absorb if self._damp else t

    def get_psi_real(self) -> np.ndarray:
        return self._host(self._pr[self._cur])

    def get_psi_imag(self):
        return self._host(self._pi[self._cur]) if self._has_imag else None

    def get_psi_real_prev(self) -> np.ndarray:
        return self._host(self._prev_psi(self._pr[1 - self._cur]))

    def get_psi_imag_prev(self):
        if not self._has_imag:
            return None
        return self._host(self._prev_psi(self._pi[1 - self._cur]))

    def get_chi(self) -> np.ndarray:
        import torch

        return self._host(self.chi64().to(torch.float32))

    def get_chi_prev(self) -> np.ndarray:
        import torch

        return self._host(self.chi64(prev=True).to(torch.float32))

    def device_state(self) -> dict:
        """Device tensors: psi_r, psi_r_prev (as the reference stores it), chi (float32),
        chi64 (float64) and at COMPLEX psi_i, psi_i_prev."""
        import torch

        c64 = self.chi64()
        out = {"psi_r": self._pr[self._cur],
               "psi_r_prev": self._prev_psi(self._pr[1 - self._cur]),
               "chi": c64.to(torch.float32), "chi64": c64}
        if self._has_imag:
            out["psi_i"] = self._pi[self._cur]
            out["psi_i_prev"] = self._prev_psi(self._pi[1 - self._cur])
        return out

    def metrics(self) -> dict:
        """Float64 metrics (lfm_metrics_f64) of the state with chi rounded to float32."""
        from .metrics import device_metrics

        st = self.device_state()
        cfg = self.config
        return device_metrics(self.backend.context.handle, int(self._level), self.N,
                              st["psi_r"], st["psi_r_prev"].contiguous(), st.get("psi_i"),
                              None if "psi_i_prev" not in st else st["psi_i_prev"].contiguous(),
                              st["chi"], cfg.dt, getattr(cfg, "c", 1.0), cfg.boundary_fraction)
