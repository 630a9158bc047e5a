"""Compensated float32 evolver (Delta form, REAL and COMPLEX levels).

Same equations as :class:`lfm_b200.Evolver` and the reference backends
(lfm/core/backends/numpy_backend.py:80-205), stored as value + increment
(psi, d = psi - psi_prev_as_stored) in float32 and advanced by
lfm_leapfrog_*_comp_f32: the rounding error of each new value is carried in
its increment (two-sum), which keeps the float32 state close to a float64
run over thousands of steps.  32 B/cell/step at REAL.

The public accessors speak the reference's representation: get_psi_real_prev
returns psi - d, set_psi_real sets d = 0 (psi_prev = psi), and so on.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .backend import B200Backend, _stream_handle, get_backend
from .config import FieldLevel
from .mask import MaskTable


class CompensatedEvolver:
    """Leapfrog evolver with compensated float32 state, one lattice on one GPU."""

    use_graphs = True

    def __init__(self, config, backend="auto") -> None:
        import torch

        self.config = config
        self.backend = backend if isinstance(backend, B200Backend) else get_backend(backend)
        self.device = self.backend.device
        self._level = FieldLevel(int(config.field_level))
        if self._level == FieldLevel.COLOR:
            raise ValueError("the compensated path covers the REAL and COMPLEX levels")
        self.N = int(config.grid_size)
        self.total = self.N**3
        self.step = 0
        self._has_imag = self._level == FieldLevel.COMPLEX
        f32 = dict(dtype=torch.float32, device=self.device)
        n = self.total
        self._table = MaskTable.for_lattice(self.N, config.boundary_fraction)
        self._table_dev = self._table.to_device(self.device)
        self._desc = self._table.desc
        self.boundary_mask = self._table.device_mask(self.device)
        self._pr = [torch.zeros(n, **f32), torch.zeros(n, **f32)]
        self._dpr = torch.zeros(n, **f32)
        self._pi = [torch.zeros(n, **f32), torch.zeros(n, **f32)] if self._has_imag else None
        self._dpi = torch.zeros(n, **f32) if self._has_imag else None
        self._chi = [torch.full((n,), float(config.chi0), **f32) for _ in range(2)]
        self._dchi = torch.zeros(n, **f32)
        self._cur = 0
        self._graphs = {}

    # ---------------------------------------------------------------- stepping
    def _step(self) -> None:
        c = self.config
        cur, nxt = self._cur, 1 - self._cur
        common = (float(c.dt**2), float(c.kappa), float(c.lambda_self), float(c.chi0),
                  float(c.e0_sq))
        stream = _stream_handle(self.device)
        table, desc = self._table_dev.data_ptr(), ctypes.byref(self._desc)
        if self._level == FieldLevel.REAL:
            _lib.call("lfm_leapfrog_real_comp_f32", self._pr[cur].data_ptr(),
                      self._pr[nxt].data_ptr(), self._dpr.data_ptr(), self._chi[cur].data_ptr(),
                      self._chi[nxt].data_ptr(), self._dchi.data_ptr(), table, desc, self.N,
                      *common, stream)
        else:
            _lib.call("lfm_leapfrog_complex_comp_f32", self._pr[cur].data_ptr(),
                      self._pr[nxt].data_ptr(), self._dpr.data_ptr(), self._pi[cur].data_ptr(),
                      self._pi[nxt].data_ptr(), self._dpi.data_ptr(), self._chi[cur].data_ptr(),
                      self._chi[nxt].data_ptr(), self._dchi.data_ptr(), table, desc, self.N,
                      *common, float(c.epsilon_w), stream)
        self._cur = nxt

    def _pair_graph(self):
        import torch

        c = self.config
        key = (self._cur, float(c.dt), float(c.kappa), float(c.lambda_self), float(c.chi0),
               float(c.e0_sq), float(c.epsilon_w))
        g = self._graphs.get(key)
        if g is None:
            saved = self._cur
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._step()
                self._step()
            self._cur = saved
            self._graphs[key] = g
        return g

    def warm_graphs(self) -> None:
        """Capture the two-step graphs of both parities now (nothing runs)."""
        saved = self._cur
        for c in (0, 1):
            self._cur = c
            self._pair_graph()
        self._cur = saved

    def evolve(self, steps: int, callback=None, freeze_chi: bool = False) -> None:
        report = self.config.report_interval
        steps = int(steps)
        if callback is None and not freeze_chi and self.use_graphs and steps >= 4:
            if not self._graphs:
                self._step()  # first launches outside capture
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
        frozen = None
        if freeze_chi:
            frozen = (self._chi[self._cur].clone(), self._dchi.clone())
        for _ in range(steps):
            self._step()
            if frozen is not None:
                self._chi[self._cur].copy_(frozen[0])
                self._dchi.copy_(frozen[1])
            self.step += 1
            if callback is not None and report > 0 and self.step % report == 0:
                callback(self, self.step)

    # ---------------------------------------------------------------- accessors
    def _dev(self, arr):
        import torch

        if isinstance(arr, torch.Tensor):
            return arr.detach().reshape(-1).to(self.device, dtype=torch.float32, non_blocking=True)
        return torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float32).ravel()).to(self.device)

    def _shape(self, t):
        return t.reshape(self.N, self.N, self.N)

    def _host(self, t) -> np.ndarray:
        host = self._shape(t).detach().to("cpu").numpy()
        _lib.check_device("CompensatedEvolver read", self.device)
        return host

    def set_psi_real(self, arr) -> None:
        self._pr[self._cur].copy_(self._dev(arr))
        self._dpr.zero_()

    def set_psi_imag(self, arr) -> None:
        if not self._has_imag:
            raise ValueError("Cannot set imaginary part for REAL field level")
        self._pi[self._cur].copy_(self._dev(arr))
        self._dpi.zero_()

    def set_psi_real_prev(self, arr) -> None:
        self._dpr.copy_(self._pr[self._cur] - self._dev(arr))

    def set_psi_imag_prev(self, arr) -> None:
        if not self._has_imag:
            raise ValueError("Cannot set imaginary part for REAL field level")
        self._dpi.copy_(self._pi[self._cur] - self._dev(arr))

    def set_psi_real_current(self, arr) -> None:
        prev = self._pr[self._cur] - self._dpr
        self._pr[self._cur].copy_(self._dev(arr))
        self._dpr.copy_(self._pr[self._cur] - prev)

    def set_chi(self, arr) -> None:
        self._chi[self._cur].copy_(self._dev(arr))
        self._dchi.zero_()

    def set_chi_current(self, arr) -> None:
        prev = self._chi[self._cur] - self._dchi
        self._chi[self._cur].copy_(self._dev(arr))
        self._dchi.copy_(self._chi[self._cur] - prev)

    def set_chi_prev(self, arr) -> None:
        self._dchi.copy_(self._chi[self._cur] - self._dev(arr))

    def get_psi_real(self) -> np.ndarray:
        return self._host(self._pr[self._cur])

    def get_psi_imag(self):
        return self._host(self._pi[self._cur]) if self._has_imag else None

    def get_psi_real_prev(self) -> np.ndarray:
        return self._host(self._pr[self._cur] - self._dpr)

    def get_psi_imag_prev(self):
        return self._host(self._pi[self._cur] - self._dpi) if self._has_imag else None

    def get_chi(self) -> np.ndarray:
        return self._host(self._chi[self._cur])

    def device_state(self) -> dict:
        out = {"psi_r": self._pr[self._cur], "psi_r_prev": self._pr[self._cur] - self._dpr,
               "chi": self._chi[self._cur]}
        if self._has_imag:
            out["psi_i"] = self._pi[self._cur]
            out["psi_i_prev"] = self._pi[self._cur] - self._dpi
        return out

    def metrics(self) -> dict:
        """Float64 metrics (lfm_metrics_f64); the kinetic term uses the stored increment."""
        from .metrics import device_metrics

        st = self.device_state()
        cfg = self.config
        return device_metrics(self.backend.context.handle, int(self._level), self.N,
                              st["psi_r"], st["psi_r_prev"], st.get("psi_i"),
                              st.get("psi_i_prev"), st["chi"], cfg.dt, getattr(cfg, "c", 1.0),
                              cfg.boundary_fraction)
