"""Double-buffered evolver on the B200 library.

Public API of the reference ``Evolver`` (lfm/core/evolver.py:42-536):
``Evolver(config, backend=...)``, ``evolve(steps, callback, freeze_chi)``,
``get_*`` / ``set_*`` field accessors, ``step``, ``_use_buffer_A`` and the
buffer attributes ``psi_r_A`` ... ``chi_prev_B`` / ``sa_A`` that hooks use.

Two buffer layouts, identical results bit for bit:

``buffers="resident"`` (default)
    Two slots per field.  Each step reads (cur, prev) and writes the new
    field over prev (lfm_leapfrog_*_f32), 24 B/cell at REAL.  The stored
    prev then holds the undamped field and the kernel applies the sponge
    factor on read -- the same float32 product the reference stores
    (numpy_backend.py:128), so nothing changes in the results.  The mask
    comes from the radial lookup table.

``buffers="ab"``
    The reference's four-buffer A/B layout (evolver.py:87-135), stepped
    through the protocol calls (lfm_step_*_f32), for callers that need every
    A/B buffer to hold exactly what the reference's would.

COLOR with kappa_tube > 0 runs the S_a Helmholtz solve (cuFFT) from the
current Psi before each step, as numpy_backend.py:341-356 does.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .backend import B200Backend, _stream_handle, get_backend
from .config import FieldLevel
from .mask import MaskTable


class Evolver:
    """Leapfrog evolver for one lattice on one GPU.

    ``freeze_chi`` reproduces the reference bit for bit only with
    ``buffers="ab"``: the reference restores its four chi buffers, two of
    which are stale in an evolved state, so its frozen chi alternates between
    two consecutive steps.  The resident layout holds the active (chi,
    chi_prev) pair instead; the two agree after ``set_chi``.

    Host reads (``get_*``, ``synchronize``) raise ``LfmError`` if a kernel's
    bounded device-side wait gave up since the last read.
    """

    def __init__(self, config, backend="auto", buffers: str = "resident") -> None:
        import torch

        self.config = config
        self.backend = backend if isinstance(backend, B200Backend) else get_backend(backend)
        self.device = self.backend.device
        self.N = int(config.grid_size)
        self.total = self.N**3
        self.step = 0
        self._use_buffer_A = True
        self._level = FieldLevel(int(config.field_level))
        if buffers not in ("resident", "ab"):
            raise ValueError(f"buffers must be 'resident' or 'ab', got {buffers!r}")
        self._mode = buffers
        if self._level == FieldLevel.COLOR and int(config.n_colors) != 3:
            # The reference kernels hard-code three colours (numpy_backend.py:240,
            # kernel_source.py:107) whatever n_colors says; refuse instead.
            raise ValueError(f"COLOR level steps exactly 3 colours, config has n_colors="
                             f"{config.n_colors}")
        self._n_psi = 1 if self._level != FieldLevel.COLOR else 3
        self._has_imag = self._level != FieldLevel.REAL
        self._dt2 = config.dt**2
        self._N = self.N
        self._sa_on = bool(config.kappa_tube > 0.0) and self._level == FieldLevel.COLOR

        N, n = self.N, self.total
        psi_n = self._n_psi * n
        f32 = dict(dtype=torch.float32, device=self.device)
        self._table = MaskTable.for_lattice(N, config.boundary_fraction)
        self.boundary_mask = self._table.device_mask(self.device)
        self._absorb = 1.0 - self.boundary_mask  # float32, as numpy_backend.py:122
        if self._level == FieldLevel.COLOR:
            self._absorb_psi = self._absorb.repeat(3)
        else:
            self._absorb_psi = self._absorb

        self._energy_ok = False
        if self._mode == "resident":
            self._table_dev = self._table.to_device(self.device)
            self._desc = self._table.desc
            self._pr = [torch.zeros(psi_n, **f32), torch.zeros(psi_n, **f32)]
            self._pi = ([torch.zeros(psi_n, **f32), torch.zeros(psi_n, **f32)]
                        if self._has_imag else [None, None])
            self._chi = [torch.full((n,), float(config.chi0), **f32) for _ in range(2)]
            self._cur = 0
            self._damp = False  # prev slots already hold the damped field
            self._sa_raw = torch.zeros(3 * n, **f32) if self._sa_on else None
            # |Psi_a|^2 of the current fields, written by the previous step's kernel
            # (valid while nothing else has written Psi since): the next S_a solve
            # starts from it instead of reading the six Psi arrays again
            self._energy = torch.empty(3 * n, **f32) if self._sa_on else None
        else:
            self._ab = {
                "psi_r_A": torch.zeros(psi_n, **f32), "psi_r_prev_A": torch.zeros(psi_n, **f32),
                "psi_r_B": torch.zeros(psi_n, **f32), "psi_r_prev_B": torch.zeros(psi_n, **f32),
                "chi_A": torch.full((n,), float(config.chi0), **f32),
                "chi_prev_A": torch.full((n,), float(config.chi0), **f32),
                "chi_B": torch.full((n,), float(config.chi0), **f32),
                "chi_prev_B": torch.full((n,), float(config.chi0), **f32),
            }
            if self._has_imag:
                for k in ("psi_i_A", "psi_i_prev_A", "psi_i_B", "psi_i_prev_B"):
                    self._ab[k] = torch.zeros(psi_n, **f32)
            if self._sa_on:
                self._ab["sa_A"] = torch.zeros(3 * n, **f32)
                self._ab["sa_B"] = torch.zeros(3 * n, **f32)

    # ------------------------------------------------------------------
    # buffer attributes of the reference Evolver
    # ------------------------------------------------------------------
    def _materialize_prev(self) -> None:
        """Apply the pending sponge factor to the stored previous Psi (resident mode)."""
        if self._mode == "resident" and self._damp:
            p = 1 - self._cur
            self._pr[p].mul_(self._absorb_psi)
            if self._has_imag:
                self._pi[p].mul_(self._absorb_psi)
            self._damp = False

    def _buf(self, name: str):
        if self._mode == "ab":
            return self._ab.get(name)
        cur, prv = self._cur, 1 - self._cur
        base = name[:-2]
        if base == "psi_r":
            return self._pr[cur]
        if base == "psi_i":
            return self._pi[cur]
        if base == "chi":
            return self._chi[cur]
        if base == "chi_prev":
            return self._chi[prv]
        if base in ("psi_r_prev", "psi_i_prev"):
            self._materialize_prev()
            return (self._pr if base == "psi_r_prev" else self._pi)[prv]
        if base == "sa":
            return self._sa_raw
        raise AttributeError(name)

    def _exposed(self, name: str):
        """A Psi buffer handed to a caller that may write it (the reference's hooks
        address psi_r_A ... by name): the next step forms |Psi_a|^2 afresh."""
        self._energy_ok = False
        return self._buf(name)

    # In resident mode the A and B names both refer to the active slots
    # (the inactive set of the reference holds values no step reads).
    psi_r_A = property(lambda s: s._exposed("psi_r_A"))
    psi_r_B = property(lambda s: s._exposed("psi_r_B"))
    psi_r_prev_A = property(lambda s: s._exposed("psi_r_prev_A"))
    psi_r_prev_B = property(lambda s: s._exposed("psi_r_prev_B"))
    psi_i_A = property(lambda s: s._exposed("psi_i_A"))
    psi_i_B = property(lambda s: s._exposed("psi_i_B"))
    psi_i_prev_A = property(lambda s: s._exposed("psi_i_prev_A"))
    psi_i_prev_B = property(lambda s: s._exposed("psi_i_prev_B"))
    chi_A = property(lambda s: s._buf("chi_A"))
    chi_B = property(lambda s: s._buf("chi_B"))
    chi_prev_A = property(lambda s: s._buf("chi_prev_A"))
    chi_prev_B = property(lambda s: s._buf("chi_prev_B"))
    sa_A = property(lambda s: s._buf("sa_A"))
    sa_B = property(lambda s: s._buf("sa_B"))

    # ------------------------------------------------------------------
    # live device views for per-step hooks (simulation.py:212-256)
    # ------------------------------------------------------------------
    def _view(self, t):
        N = self.N
        return t.view(N, N, N) if self._n_psi == 1 or t.numel() == N**3 else t.view(3, N, N, N)

    def native_psi_real(self):
        """The current Psi_r buffer as an (N, N, N) device view ((3, N, N, N) at COLOR):
        edits are seen by the next step.  The previous-step buffers are not exposed."""
        self._energy_ok = False  # the caller may edit Psi through the view
        if self._mode == "ab":
            return self._view(self._ab["psi_r_A" if self._use_buffer_A else "psi_r_B"])
        return self._view(self._pr[self._cur])

    def native_psi_imag(self):
        """The current Psi_i buffer as a device view, None at the REAL level."""
        if not self._has_imag:
            return None
        self._energy_ok = False
        if self._mode == "ab":
            return self._view(self._ab["psi_i_A" if self._use_buffer_A else "psi_i_B"])
        return self._view(self._pi[self._cur])

    def native_chi(self):
        """The current chi buffer as an (N, N, N) device view."""
        if self._mode == "ab":
            return self._view(self._ab["chi_A" if self._use_buffer_A else "chi_B"])
        return self._view(self._chi[self._cur])

    def native_chi_pair(self):
        """Every chi buffer a step reads, as device views: writing the same values to
        all of them leaves chi without velocity there (the reference's four A/B buffers;
        the resident layout's current and previous slots)."""
        if self._mode == "ab":
            return tuple(self._view(self._ab[k]) for k in ("chi_A", "chi_B", "chi_prev_A",
                                                           "chi_prev_B"))
        return (self._view(self._chi[self._cur]), self._view(self._chi[1 - self._cur]))

    # ------------------------------------------------------------------
    # time loop (evolver.py:137-180)
    # ------------------------------------------------------------------
    use_graphs = True
    """Replay captured CUDA graphs of two steps when evolve() has no per-step host work."""
    hook_block = 32
    """Steps per captured graph when evolve() runs device hooks (even: parity returns)."""

    def evolve(self, steps: int, callback=None, freeze_chi: bool = False, hooks=None) -> None:
        """Run `steps` leapfrog steps; callback(evolver, step) every report_interval.

        hooks: device hooks (lfm_b200.hooks) applied after every step, in order, as the
        reference's per-step callbacks are; with no callback and no freeze_chi, blocks
        of hook_block steps run as captured CUDA graphs together with their hooks.
        """
        report = self.config.report_interval
        hooks = list(hooks or ())
        if hooks:
            if (callback is None and not freeze_chi and self._mode == "resident"
                    and self.use_graphs and all(getattr(h, "graphable", False) for h in hooks)):
                self._evolve_hooked(int(steps), hooks)
                return
        elif (callback is None and not freeze_chi and self._mode == "resident"
                and self.use_graphs and steps >= 4):
            self._evolve_graphed(int(steps))
            return
        frozen = None
        if freeze_chi:
            if self._mode == "ab":
                frozen = [self._ab[k].clone() for k in ("chi_A", "chi_B", "chi_prev_A",
                                                        "chi_prev_B")]
            else:
                frozen = [self._chi[self._cur].clone(), self._chi[1 - self._cur].clone()]
        for _ in range(int(steps)):
            self._step()
            if frozen is not None:
                if self._mode == "ab":
                    for k, v in zip(("chi_A", "chi_B", "chi_prev_A", "chi_prev_B"), frozen):
                        self._ab[k].copy_(v)
                else:
                    self._chi[self._cur].copy_(frozen[0])
                    self._chi[1 - self._cur].copy_(frozen[1])
            self.step += 1
            for h in hooks:
                h.apply(self, self.step)
            if callback is not None and report > 0 and self.step % report == 0:
                callback(self, self.step)

    def _evolve_hooked(self, steps: int, hooks) -> None:
        """Steps with device hooks: whole blocks replay one captured graph each."""
        K = int(self.hook_block) + (int(self.hook_block) % 2)
        self._dt2 = self.config.dt**2
        done = 0

        def eager_step():
            self._step()
            self.step += 1
            for h in hooks:
                h.apply(self, self.step)

        if not self._damp:  # the first step after a host write does not damp prev
            eager_step()
            done = 1
        while steps - done >= K:
            g = self._hook_graph(hooks, K)
            for h in hooks:
                h.begin_block(self, self.step, K)
            g.replay()
            for h in hooks:
                h.end_block(self, K)
            self.step += K
            done += K
        while done < steps:
            eager_step()
            done += 1

    def _hook_graph(self, hooks, K: int):
        import torch

        if not hasattr(self, "_hgraphs"):
            self._hgraphs = {}
        key = (self._param_key(), K, tuple(id(h) for h in hooks))
        g = self._hgraphs.get(key)
        if g is None:
            for h in hooks:
                h.prepare_block(self, K)
            saved = (self._cur, self._damp, self._use_buffer_A, self._energy_ok)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                for k in range(K):
                    self._step_resident()
                    self._use_buffer_A = not self._use_buffer_A
                    for h in hooks:
                        h.apply_in_block(self, k)
            self._cur, self._damp, self._use_buffer_A, self._energy_ok = saved
            self._hgraphs[key] = (g, list(hooks))  # the graph holds the hooks' buffers
        return self._hgraphs[key][0]

    def _param_key(self) -> tuple:
        c = self.config
        return (self._cur, float(c.dt), float(c.kappa), float(c.lambda_self), float(c.chi0),
                float(c.e0_sq), float(c.epsilon_w), float(c.kappa_c), float(c.epsilon_cc),
                float(c.kappa_string), float(c.kappa_tube), float(c.sa_gamma), float(c.sa_d))

    def _pair_graph(self):
        """CUDA graph of two resident steps from the current slot parity."""
        import torch

        if not hasattr(self, "_graphs"):
            self._graphs = {}
        key = self._param_key()
        g = self._graphs.get(key)
        if g is None:
            saved = (self._cur, self._damp, self._use_buffer_A, self._energy_ok)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._step_resident()
                self._step_resident()
            self._cur, self._damp, self._use_buffer_A, self._energy_ok = saved
            self._graphs[key] = g
        return g

    def warm_graphs(self) -> None:
        """Capture the two-step graphs of both slot parities now (nothing runs), so a
        later evolve() does not capture inside a timed region.  Needs one step done."""
        if self._mode != "resident" or not self._damp or (self._sa_on and not self._energy_ok):
            return
        saved = self._cur
        for c in (0, 1):
            self._cur = c
            self._pair_graph()
        self._cur = saved

    def _evolve_graphed(self, steps: int) -> None:
        self._dt2 = self.config.dt**2
        done = 0
        if not self._damp or (self._sa_on and not self._energy_ok):
            # first step after a host write: the kernel must not damp prev, and
            # |Psi_a|^2 comes from Psi, not from the previous step's kernel
            self._step()
            self.step += 1
            done = 1
        pairs = (steps - done) // 2
        if pairs:
            g = self._pair_graph()
            for _ in range(pairs):
                g.replay()
            self.step += 2 * pairs
        if (steps - done) % 2:
            self._step()
            self.step += 1

    def _step(self) -> None:
        if self._mode == "ab":
            self._step_ab()
        else:
            self._step_resident()
        self._use_buffer_A = not self._use_buffer_A

    def _step_resident(self) -> None:
        cfg = self.config
        cur, prv = self._cur, 1 - self._cur
        stream = _stream_handle(self.device)
        table = self._table_dev.data_ptr()
        desc = ctypes.byref(self._desc)
        damp = 1 if self._damp else 0
        common = (float(self._dt2), float(cfg.kappa), float(cfg.lambda_self), float(cfg.chi0),
                  float(cfg.e0_sq))
        if self._level == FieldLevel.REAL:
            _lib.call("lfm_leapfrog_real_f32", self._pr[cur].data_ptr(), self._pr[prv].data_ptr(),
                      self._chi[cur].data_ptr(), self._chi[prv].data_ptr(), table, desc, damp,
                      self.N, *common, stream)
        elif self._level == FieldLevel.COMPLEX:
            _lib.call("lfm_leapfrog_complex_f32", self._pr[cur].data_ptr(),
                      self._pr[prv].data_ptr(), self._pi[cur].data_ptr(), self._pi[prv].data_ptr(),
                      self._chi[cur].data_ptr(), self._chi[prv].data_ptr(), table, desc, damp,
                      self.N, *common, float(cfg.epsilon_w), stream)
        else:
            sa = energy = None
            if self._sa_on:
                ctx = self.backend.context.handle
                if self._energy_ok:
                    _lib.call("lfm_helmholtz_sa_from_energy_f32", ctx, self._energy.data_ptr(),
                              self._sa_raw.data_ptr(), self.N, float(cfg.sa_gamma),
                              float(cfg.sa_d), stream)
                else:
                    _lib.call("lfm_helmholtz_sa_f32", ctx, self._pr[cur].data_ptr(),
                              self._pi[cur].data_ptr(), self._sa_raw.data_ptr(), self.N,
                              float(cfg.sa_gamma), float(cfg.sa_d), stream)
                sa = self._sa_raw.data_ptr()
                energy = self._energy.data_ptr()
            _lib.call("lfm_leapfrog_color_energy_f32", self._pr[cur].data_ptr(),
                      self._pr[prv].data_ptr(), self._pi[cur].data_ptr(),
                      self._pi[prv].data_ptr(), self._chi[cur].data_ptr(),
                      self._chi[prv].data_ptr(), table, desc, damp, self.N, *common,
                      float(cfg.epsilon_w), float(cfg.kappa_c), float(cfg.epsilon_cc),
                      float(cfg.kappa_string), float(cfg.kappa_tube), sa, energy, stream)
            self._energy_ok = self._sa_on
        self._cur = prv
        self._damp = True

    def _step_ab(self) -> None:
        cfg = self.config
        b = self._ab
        src, dst = ("A", "B") if self._use_buffer_A else ("B", "A")
        g = lambda k, s: b.get(f"{k}_{s}")  # noqa: E731
        be = self.backend
        if self._level == FieldLevel.REAL:
            be.step_real(g("psi_r", src), g("psi_r_prev", src), g("chi", src), g("chi_prev", src),
                         self.boundary_mask, g("psi_r", dst), g("psi_r_prev", dst), g("chi", dst),
                         g("chi_prev", dst), self.N, self._dt2, cfg.kappa, cfg.lambda_self,
                         cfg.chi0, cfg.e0_sq)
        elif self._level == FieldLevel.COMPLEX:
            be.step_complex(g("psi_r", src), g("psi_r_prev", src), g("psi_i", src),
                            g("psi_i_prev", src), g("chi", src), g("chi_prev", src),
                            self.boundary_mask, g("psi_r", dst), g("psi_r_prev", dst),
                            g("psi_i", dst), g("psi_i_prev", dst), g("chi", dst),
                            g("chi_prev", dst), self.N, self._dt2, cfg.kappa, cfg.lambda_self,
                            cfg.chi0, cfg.e0_sq, cfg.epsilon_w)
        else:
            be.step_color(g("psi_r", src), g("psi_r_prev", src), g("psi_i", src),
                          g("psi_i_prev", src), g("chi", src), g("chi_prev", src),
                          self.boundary_mask, g("psi_r", dst), g("psi_r_prev", dst),
                          g("psi_i", dst), g("psi_i_prev", dst), g("chi", dst),
                          g("chi_prev", dst), self.N, self._dt2, cfg.kappa, cfg.lambda_self,
                          cfg.chi0, cfg.e0_sq, cfg.epsilon_w, cfg.kappa_c, cfg.epsilon_cc,
                          kappa_string=cfg.kappa_string, kappa_tube=cfg.kappa_tube,
                          sa_fields_in=g("sa", src), sa_fields_out=g("sa", dst),
                          sa_gamma=cfg.sa_gamma, sa_d=cfg.sa_d, dt=cfg.dt)

    # ------------------------------------------------------------------
    # device views of the active state (no host copies)
    # ------------------------------------------------------------------
    def _active(self, field: str):
        s = "A" if self._use_buffer_A else "B"
        return self._buf(f"{field}_{s}")

    def _prev_psi_view(self, imag: bool):
        """Previous Psi with the sponge factor applied, as the reference stores it."""
        if self._mode == "ab":
            return self._active("psi_i_prev" if imag else "psi_r_prev")
        buf = (self._pi if imag else self._pr)[1 - self._cur]
        return buf * self._absorb_psi if self._damp else buf

    def _shape(self, flat):
        if self._level == FieldLevel.COLOR:
            return flat.reshape(3, self.N, self.N, self.N)
        return flat.reshape(self.N, self.N, self.N)

    def device_state(self) -> dict:
        """Device tensors of the current state: psi_r, psi_i, chi, psi_r_prev, psi_i_prev."""
        out = {"psi_r": self._shape(self._active("psi_r")),
               "chi": self._active("chi").reshape(self.N, self.N, self.N),
               "psi_r_prev": self._shape(self._prev_psi_view(False))}
        if self._has_imag:
            out["psi_i"] = self._shape(self._active("psi_i"))
            out["psi_i_prev"] = self._shape(self._prev_psi_view(True))
        return out

    def metrics(self, prev=None, clusters: bool = False) -> dict:
        """Float64 metrics of the current state, reduced on the device.

        prev: None uses the leapfrog previous field for the kinetic term
        (dPsi/dt over one step); pass device tensors to use another snapshot.
        clusters: also count |Psi|^2 clusters on the host (one N^3 copy).
        """
        from .metrics import device_metrics, interior_mask, n_clusters

        st = self.device_state()
        if prev is None:
            pr_prev, pi_prev = st["psi_r_prev"], st.get("psi_i_prev")
        else:
            pr_prev, pi_prev = prev
        cfg = self.config
        m = device_metrics(self.backend.context.handle, int(self._level), self.N,
                           st["psi_r"].contiguous(), pr_prev.contiguous(),
                           st["psi_i"].contiguous() if self._has_imag else None,
                           pi_prev.contiguous() if pi_prev is not None else None,
                           st["chi"].contiguous(), cfg.dt, getattr(cfg, "c", 1.0),
                           cfg.boundary_fraction)
        if clusters:
            e = self.get_energy_density().astype(np.float64)
            m["n_clusters"] = float(n_clusters(e, interior_mask(self.N, cfg.boundary_fraction)))
        return m

    # ------------------------------------------------------------------
    # host accessors (evolver.py:289-536)
    # ------------------------------------------------------------------
    def _to_host(self, t, out=None):
        """Host copy of a device tensor; into `out` (e.g. pinned) without a sync when given."""
        if out is not None:
            out.reshape(-1).copy_(t.reshape(-1), non_blocking=True)
            return out
        host = t.detach().to("cpu").numpy()
        _lib.check_device("Evolver read", self.device)
        return host

    def synchronize(self) -> None:
        """Wait for this lattice's queued work; raise LfmError if a kernel's bounded
        device-side wait gave up (its outputs would be incomplete)."""
        import torch

        torch.cuda.synchronize(self.device)
        _lib.check_device("Evolver.synchronize", self.device)

    def _current_buf(self) -> str:
        return "A" if self._use_buffer_A else "B"

    def get_chi(self, out=None):
        """Current chi, (N, N, N).  With `out` (a host tensor, e.g. pinned) the copy
        is asynchronous on the current stream and `out` is returned."""
        if out is not None:
            return self._to_host(self._active("chi"), out)
        return self._to_host(self._active("chi")).reshape(self.N, self.N, self.N)

    def get_psi_real(self, out=None):
        if out is not None:
            return self._to_host(self._active("psi_r"), out)
        return self._shape(self._to_host(self._active("psi_r")))

    def get_psi_imag(self):
        if not self._has_imag:
            return None
        return self._shape(self._to_host(self._active("psi_i")))

    def get_psi_real_prev(self) -> np.ndarray:
        return self._shape(self._to_host(self._prev_psi_view(False)))

    def get_psi_imag_prev(self):
        if not self._has_imag:
            return None
        return self._shape(self._to_host(self._prev_psi_view(True)))

    def get_chi_prev(self) -> np.ndarray:
        """Previous-step chi as the next step reads it, (N, N, N)."""
        return self._to_host(self._active("chi_prev")).reshape(self.N, self.N, self.N)

    def save_checkpoint(self, path, history=None, psi_snapshot=None) -> None:
        """npz checkpoint in the reference's format plus the leapfrog previous
        fields (lfm_b200.checkpoint): loading it resumes bit for bit."""
        from .checkpoint import save_checkpoint

        save_checkpoint(self, path, history=history, psi_snapshot=psi_snapshot)

    @classmethod
    def load_checkpoint(cls, path, backend="auto", buffers: str = "resident") -> "Evolver":
        """An Evolver restored from a checkpoint written by save_checkpoint or
        by the reference's Simulation.save_checkpoint."""
        from .checkpoint import load_checkpoint

        return load_checkpoint(path, backend=backend, buffers=buffers)[0]

    def get_energy_density(self) -> np.ndarray:
        pr = self.get_psi_real()
        e2 = np.sum(pr**2, axis=0) if pr.ndim == 4 else pr**2
        pi = self.get_psi_imag()
        if pi is not None:
            e2 += np.sum(pi**2, axis=0) if pi.ndim == 4 else pi**2
        return e2

    def _dev(self, arr):
        """Flat float32 view of a host array or tensor (copied to the device by _write)."""
        import torch

        if isinstance(arr, torch.Tensor):
            return arr.detach().reshape(-1).to(dtype=torch.float32)
        return torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float32).ravel())

    def _write(self, names, data) -> None:
        """Copy `data` (host or device) into the named buffers: one host->device
        copy (asynchronous from pinned memory), device->device for the rest."""
        self._energy_ok = False
        first = None
        seen = set()
        for nm in names:
            buf = getattr(self, nm)
            if buf is None or id(buf) in seen:
                continue
            seen.add(id(buf))
            if buf.numel() != data.numel():
                raise ValueError(f"{nm}: got {data.numel()} values, expected {buf.numel()}")
            if first is None:
                buf.copy_(data, non_blocking=True)
                first = buf
            else:
                buf.copy_(first)

    def set_psi_real(self, arr) -> None:
        """Set Psi_real current and previous on both buffer sets."""
        self._write(("psi_r_A", "psi_r_B", "psi_r_prev_A", "psi_r_prev_B"), self._dev(arr))

    def set_psi_imag(self, arr) -> None:
        if not self._has_imag:
            raise ValueError("Cannot set imaginary part for REAL field level")
        self._write(("psi_i_A", "psi_i_B", "psi_i_prev_A", "psi_i_prev_B"), self._dev(arr))

    def set_psi_real_prev(self, arr) -> None:
        self._write(("psi_r_prev_A", "psi_r_prev_B"), self._dev(arr))

    def set_psi_imag_prev(self, arr) -> None:
        if not self._has_imag:
            raise ValueError("Cannot set imaginary part for REAL field level")
        self._write(("psi_i_prev_A", "psi_i_prev_B"), self._dev(arr))

    def set_psi_real_current(self, arr) -> None:
        self._energy_ok = False
        self._active("psi_r").copy_(self._dev(arr), non_blocking=True)

    def set_psi_imag_current(self, arr) -> None:
        if not self._has_imag:
            raise ValueError("Cannot set imaginary part for REAL field level")
        self._energy_ok = False
        self._active("psi_i").copy_(self._dev(arr), non_blocking=True)

    def set_chi(self, arr) -> None:
        self._write(("chi_A", "chi_B", "chi_prev_A", "chi_prev_B"), self._dev(arr))

    def set_chi_current(self, arr) -> None:
        self._write(("chi_A", "chi_B"), self._dev(arr))

    def set_chi_prev(self, arr) -> None:
        self._write(("chi_prev_A", "chi_prev_B"), self._dev(arr))

    def get_sa_fields(self):
        """S_a fields (3, N, N, N) as last computed, clipped at 0; None when off."""
        if not self._sa_on:
            return None
        buf = self._active("sa") if self._mode == "ab" else self._sa_raw
        return self._to_host(buf.clamp_min(0.0)).reshape(3, self.N, self.N, self.N)

    def set_sa_fields(self, arr) -> None:
        if not self._sa_on:
            raise ValueError(
                "SA fields not allocated — set kappa_tube > 0 in SimulationConfig"
                " before creating the Evolver."
            )
        data = self._dev(arr)
        if self._mode == "ab":
            self._ab["sa_A"].copy_(data)
            self._ab["sa_B"].copy_(data)
        else:
            self._sa_raw.copy_(data)
