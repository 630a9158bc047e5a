"""B200 implementation of the reference ``Backend`` protocol.

Drop-in for ``CupyBackend`` (lfm/core/backends/cupy_backend.py:48-363)
behind the protocol of lfm/core/backends/protocol.py:17-144: the same
method names, argument order and meaning, A/B double-buffer semantics and
errors, with torch CUDA float32 tensors as the device arrays and
liblfm_b200.so doing every step.  There is no CPU fallback: constructing
the backend without a CUDA device or without the built library raises.
"""

from __future__ import annotations

import ctypes
import weakref

import numpy as np

from . import _lib
from .mask import boundary_mask as _host_mask


_DEVICE_ARRAY = None


def device_array(t):
    """`t` as a DeviceArray: a torch tensor that also has NumPy/CuPy's ``copy()``.

    The reference Evolver snapshots its chi buffers with ``.copy()`` when it
    evolves with freeze_chi (lfm/core/evolver.py:160-166), which torch tensors
    spell ``clone()``; every array this backend hands out answers both.
    """
    global _DEVICE_ARRAY
    if _DEVICE_ARRAY is None:
        import torch

        class DeviceArray(torch.Tensor):
            def copy(self):
                return self.clone()

        _DEVICE_ARRAY = DeviceArray
    return t.as_subclass(_DEVICE_ARRAY)


def _stream_handle(device) -> int:
    import torch

    return torch.cuda.current_stream(device).cuda_stream


class LibContext:
    """Owns an lfm_context (cuFFT plans and scratch) on one device."""

    def __init__(self, device):
        import torch

        with torch.cuda.device(device):
            h = ctypes.c_void_p()
            _lib.call("lfm_context_create", ctypes.byref(h))
        self.handle = h
        self.device = device
        self._fin = weakref.finalize(self, LibContext._destroy, h)

    @staticmethod
    def _destroy(h) -> None:
        try:
            _lib.load().lfm_context_destroy(h)
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


class B200Backend:
    """GPU compute backend on liblfm_b200.so (sm_100a)."""

    def __init__(self, device=None) -> None:
        import torch

        if not torch.cuda.is_available():
            raise ImportError("the B200 backend needs a CUDA device; there is no CPU fallback")
        _lib.load()
        dev = torch.device(device) if device is not None else torch.device("cuda")
        if dev.type != "cuda":
            raise ValueError(f"the B200 backend runs on CUDA devices, got {dev}")
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self._ctx: LibContext | None = None

    @property
    def name(self) -> str:
        return "b200"

    @property
    def context(self) -> LibContext:
        if self._ctx is None:
            self._ctx = LibContext(self.device)
        return self._ctx

    # -- arrays ---------------------------------------------------------------
    def allocate(self, N: int, n_psi_arrays: int, chi0: float) -> dict:
        import torch

        total = N**3
        z = lambda n: torch.zeros(n, dtype=torch.float32, device=self.device)  # noqa: E731
        f = lambda n: torch.full((n,), float(chi0), dtype=torch.float32, device=self.device)  # noqa: E731
        psi = n_psi_arrays * total
        out = {
            "psi_A": z(psi), "psi_prev_A": z(psi), "chi_A": f(total), "chi_prev_A": f(total),
            "psi_B": z(psi), "psi_prev_B": z(psi), "chi_B": f(total), "chi_prev_B": f(total),
        }
        return {k: device_array(v) for k, v in out.items()}

    def create_boundary_mask(self, N: int, boundary_fraction: float):
        return self.from_numpy(_host_mask(N, boundary_fraction))

    def to_numpy(self, arr) -> np.ndarray:
        out = arr.detach().to("cpu").numpy()
        _lib.check_device("to_numpy", self.device)
        return out

    def from_numpy(self, arr):
        import torch

        return device_array(
            torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float32)).to(self.device))

    def synchronize(self) -> None:
        import torch

        torch.cuda.synchronize(self.device)
        _lib.check_device("synchronize", self.device)

    # -- argument checks --------------------------------------------------------
    def _ptr(self, t, numel: int, what: str) -> int:
        import torch

        if not isinstance(t, torch.Tensor):
            raise TypeError(f"{what}: expected a torch CUDA tensor, got {type(t).__name__}")
        if t.device != self.device:
            raise ValueError(f"{what}: tensor on {t.device}, backend on {self.device}")
        if t.dtype != torch.float32:
            raise TypeError(f"{what}: expected float32, got {t.dtype}")
        if not t.is_contiguous():
            raise ValueError(f"{what}: tensor must be contiguous")
        if t.numel() != numel:
            raise ValueError(f"{what}: {t.numel()} elements, expected {numel}")
        return t.data_ptr()

    # -- protocol steps -----------------------------------------------------------
    def step_real(self, psi_in, psi_prev_in, chi_in, chi_prev_in, boundary_mask,
                  psi_out, psi_prev_out, chi_out, chi_prev_out,
                  N, dt2, kappa, lambda_self, chi0, e0_sq) -> None:
        """One leapfrog step for real E (numpy_backend.py:80-130)."""
        n = N**3
        names = ("psi_in", "psi_prev_in", "chi_in", "chi_prev_in", "boundary_mask",
                 "psi_out", "psi_prev_out", "chi_out", "chi_prev_out")
        arrs = (psi_in, psi_prev_in, chi_in, chi_prev_in, boundary_mask,
                psi_out, psi_prev_out, chi_out, chi_prev_out)
        ptrs = [self._ptr(a, n, nm) for a, nm in zip(arrs, names)]
        _lib.call("lfm_step_real_f32", *ptrs, int(N), float(dt2), float(kappa),
                  float(lambda_self), float(chi0), float(e0_sq), _stream_handle(self.device))

    def step_complex(self, psi_r_in, psi_r_prev_in, psi_i_in, psi_i_prev_in, chi_in,
                     chi_prev_in, boundary_mask, psi_r_out, psi_r_prev_out, psi_i_out,
                     psi_i_prev_out, chi_out, chi_prev_out,
                     N, dt2, kappa, lambda_self, chi0, e0_sq, epsilon_w) -> None:
        """One leapfrog step for complex Psi (numpy_backend.py:132-205)."""
        n = N**3
        arrs = (psi_r_in, psi_r_prev_in, psi_i_in, psi_i_prev_in, chi_in, chi_prev_in,
                boundary_mask, psi_r_out, psi_r_prev_out, psi_i_out, psi_i_prev_out, chi_out,
                chi_prev_out)
        ptrs = [self._ptr(a, n, f"arg{i}") for i, a in enumerate(arrs)]
        _lib.call("lfm_step_complex_f32", *ptrs, int(N), float(dt2), float(kappa),
                  float(lambda_self), float(chi0), float(e0_sq), float(epsilon_w),
                  _stream_handle(self.device))

    def step_color(self, psi_r_in, psi_r_prev_in, psi_i_in, psi_i_prev_in, chi_in,
                   chi_prev_in, boundary_mask, psi_r_out, psi_r_prev_out, psi_i_out,
                   psi_i_prev_out, chi_out, chi_prev_out,
                   N, dt2, kappa, lambda_self, chi0, e0_sq, epsilon_w,
                   kappa_c=0.0, epsilon_cc=0.0, kappa_string=0.0, kappa_tube=0.0,
                   sa_fields_in=None, sa_fields_out=None, sa_gamma=0.1, sa_d=4.9,
                   dt=0.02) -> None:
        """One leapfrog step for three colours (numpy_backend.py:207-382)."""
        n = N**3
        psi = (psi_r_in, psi_r_prev_in, psi_i_in, psi_i_prev_in)
        outs = (psi_r_out, psi_r_prev_out, psi_i_out, psi_i_prev_out)
        p_in = [self._ptr(a, 3 * n, f"psi_in{i}") for i, a in enumerate(psi)]
        p_c = [self._ptr(a, n, nm) for a, nm in ((chi_in, "chi_in"), (chi_prev_in, "chi_prev_in"),
                                                   (boundary_mask, "boundary_mask"))]
        p_out = [self._ptr(a, 3 * n, f"psi_out{i}") for i, a in enumerate(outs)]
        p_co = [self._ptr(a, n, nm) for a, nm in ((chi_out, "chi_out"),
                                                    (chi_prev_out, "chi_prev_out"))]
        sa_in = None if sa_fields_in is None else self._ptr(sa_fields_in, 3 * n, "sa_fields_in")
        sa_out = None if sa_fields_out is None else self._ptr(sa_fields_out, 3 * n,
                                                               "sa_fields_out")
        ctx = self.context.handle if (kappa_tube > 0 and sa_out is not None) else None
        _lib.call("lfm_step_color_f32", ctx, *p_in, *p_c, *p_out, *p_co, int(N), float(dt2),
                  float(kappa), float(lambda_self), float(chi0), float(e0_sq),
                  float(epsilon_w), float(kappa_c), float(epsilon_cc), float(kappa_string),
                  float(kappa_tube), sa_in, sa_out, float(sa_gamma), float(sa_d), float(dt),
                  _stream_handle(self.device))


def get_backend(preference: str = "auto"):
    """Backend factory with the reference's preference names (backends/__init__.py:28-73).

    'auto', 'gpu' and 'b200' give the B200 backend; 'cpu' and 'remote' are
    outside this package and raise ValueError.
    """
    pref = preference.lower()
    if pref in ("auto", "gpu", "b200", "cuda"):
        return B200Backend()
    raise ValueError(
        f"Unknown backend preference '{preference}'. lfm_b200 provides 'auto', 'gpu' or 'b200'."
    )
