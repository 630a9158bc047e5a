"""ctypes binding of liblfm_b200.so (the C ABI in include/lfm_b200.h).

The library is the only compute path: importing this module on a machine
without the built library raises, and every entry point's status code is
turned into a ``RuntimeError`` carrying the library's own message.
"""

from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_float, c_int, c_int32, c_int64, c_void_p

from .build import LIB_PATH

LFM_OK = 0
LFM_ERR_INVALID_ARG = 1
LFM_ERR_UNSUPPORTED = 3
LFM_ERR_MASK = 6
LFM_ERR_DEVICE_TIMEOUT = 7
LFM_ERR_NONFINITE = 8
LFM_ERR_CAPACITY = 9

PATH_AUTO, PATH_DIRECT, PATH_FUSED = 0, 1, 2


class MaskLut(ctypes.Structure):
    """lfm_mask_lut: the sponge lookup-table descriptor."""

    _fields_ = [("N", c_int32), ("shift", c_int32), ("q_lo", c_int32), ("q_hi", c_int32),
                ("count", c_int32)]


class LatticeDesc(ctypes.Structure):
    """lfm_lattice_desc: one lattice of a batch (slot pointers, mask, constants)."""

    _fields_ = [("N", c_int32), ("level", c_int32), ("psi_r", c_void_p * 2),
                ("psi_i", c_void_p * 2), ("chi", c_void_p * 2), ("mask_table", c_void_p),
                ("lut", MaskLut), ("dt2", c_double), ("kappa", c_double),
                ("lambda_self", c_double), ("chi0", c_double), ("e0_sq", c_double),
                ("epsilon_w", c_double)]


class BatchTuning(ctypes.Structure):
    """lfm_batch_tuning: CTA size cap, stages, cells per work item, CTAs per SM (0 = default)."""

    _fields_ = [("threads", c_int32), ("stages", c_int32), ("item_cells", c_int32),
                ("ctas_per_sm", c_int32)]


class LfmError(RuntimeError):
    """A liblfm_b200 entry point returned a non-zero status."""

    def __init__(self, code: int, where: str, detail: str):
        self.code = code
        super().__init__(f"{where}: {detail} (status {code})")


_P = c_void_p
_D = c_double

# name -> argtypes; every function returns int (the status)
_SIGNATURES = {
    "lfm_abi_version": [],
    "lfm_set_step_path": [c_int],
    "lfm_set_sa_transform": [c_int],
    "lfm_mask_lut_build": [c_int, _P, _P, c_int, POINTER(MaskLut)],
    "lfm_step_real_f32": [_P] * 9 + [c_int] + [_D] * 5 + [_P],
    "lfm_step_complex_f32": [_P] * 13 + [c_int] + [_D] * 6 + [_P],
    "lfm_step_color_f32": [_P] * 14 + [c_int] + [_D] * 10 + [_P, _P] + [_D] * 3 + [_P],
    "lfm_context_create": [POINTER(c_void_p)],
    "lfm_context_destroy": [_P],
    "lfm_leapfrog_real_f32": [_P] * 5 + [POINTER(MaskLut), c_int, c_int] + [_D] * 5 + [_P],
    "lfm_leapfrog_complex_f32": [_P] * 7 + [POINTER(MaskLut), c_int, c_int] + [_D] * 6 + [_P],
    "lfm_leapfrog_color_f32": [_P] * 7 + [POINTER(MaskLut), c_int, c_int] + [_D] * 10
    + [_P, _P],
    "lfm_leapfrog_color_energy_f32": [_P] * 7 + [POINTER(MaskLut), c_int, c_int] + [_D] * 10
    + [_P, _P, _P],
    "lfm_helmholtz_sa_from_energy_f32": [_P] * 3 + [c_int, _D, _D, _P],
    "lfm_leapfrog_real_comp_f32": [_P] * 7 + [POINTER(MaskLut), c_int] + [_D] * 5 + [_P],
    "lfm_leapfrog_complex_comp_f32": [_P] * 10 + [POINTER(MaskLut), c_int] + [_D] * 6 + [_P],
    "lfm_leapfrog_real_split_f32": [_P] * 7 + [POINTER(MaskLut), c_int, c_int] + [_D] * 5
    + [_P],
    "lfm_leapfrog_complex_split_f32": [_P] * 9 + [POINTER(MaskLut), c_int, c_int] + [_D] * 6
    + [_P],
    "lfm_advance_split_f32": [c_int] + [_P] * 13 + [POINTER(MaskLut), c_int, c_int] + [_D] * 6
    + [_P],
    "lfm_helmholtz_sa_f32": [_P] * 4 + [c_int, _D, _D, _P],
    "lfm_sa_clip_f32": [_P, _P, c_int64, _P],
    "lfm_device_status": [POINTER(c_int), c_int],
    "lfm_metrics_f64": [_P, c_int] + [_P] * 5 + [c_int] + [_D] * 5 + [_P, _P],
    "lfm_metrics_f64_noalloc": [c_int] + [_P] * 5 + [c_int] + [_D] * 5 + [_P, _P],
    "lfm_slab_step_f32": [c_int] + [_P] * 7 + [POINTER(MaskLut), c_int, c_int, c_int, c_int]
    + [_D] * 6 + [_P],
    "lfm_slab_step_planes_f32": [c_int] + [_P] * 7 + [POINTER(MaskLut)] + [c_int] * 6
    + [_D] * 6 + [_P],
    "lfm_poisson_chi_f32": [_P, c_int, _P, _P, c_int] + [_D] * 4 + [c_int, _P, _P],
    "lfm_advance_f32": [c_int] + [_P] * 10 + [POINTER(MaskLut), c_int, c_int] + [_D] * 6
    + [_P],
    "lfm_adjoint_step_f32": [c_int] + [_P] * 5 + [POINTER(MaskLut), POINTER(c_void_p),
                                                    POINTER(c_void_p), c_int] + [_D] * 6 + [_P],
    "lfm_batch_create": [POINTER(LatticeDesc), c_int, POINTER(BatchTuning), POINTER(c_void_p)],
    "lfm_batch_step": [_P, c_int, c_int, _P],
    "lfm_batch_info": [_P] + [POINTER(c_int)] * 4,
    "lfm_batch_destroy": [_P],
    "lfm_batch_plan": [POINTER(LatticeDesc), c_int, POINTER(BatchTuning), c_int, POINTER(c_int32),
                       c_int, POINTER(c_int), POINTER(c_int32)],
    "lfm_tune_set": [c_int] * 6,
    "lfm_tune_get": [c_int, c_int] + [POINTER(c_int)] * 6,
    "lfm_selftest_device_timeout": [ctypes.c_ulonglong, _P],
}

_lib = None


def load() -> ctypes.CDLL:
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m lfm_b200.build` "
                "(there is no CPU fallback)"
            )
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, args in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = c_int
        lib.lfm_strerror.argtypes = [c_int]
        lib.lfm_strerror.restype = ctypes.c_char_p
        lib.lfm_last_error_detail.argtypes = []
        lib.lfm_last_error_detail.restype = ctypes.c_char_p
        _lib = lib
    return _lib


def exported_symbols() -> list[str]:
    return sorted(list(_SIGNATURES) + ["lfm_strerror", "lfm_last_error_detail"])


def check(code: int, where: str) -> None:
    if code != LFM_OK:
        lib = load()
        detail = lib.lfm_last_error_detail().decode(errors="replace")
        name = lib.lfm_strerror(code).decode()
        raise LfmError(code, where, f"{name}: {detail}")


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args), name)


def set_step_path(path: int) -> None:
    """Choose the step kernel: 0 automatic, 1 direct, 2 fused 2.5D only."""
    call("lfm_set_step_path", int(path))


def tune_set(level: int, N: int, tj: int, stages: int, ic: int = 0, vec: int = 0) -> None:
    """Force the fused kernel's tile configuration for (level, N); tj <= 0 clears it."""
    call("lfm_tune_set", int(level), int(N), int(vec), int(tj), int(stages), int(ic))


def tune_get(level: int, N: int) -> dict | None:
    """The tile configuration the last fused step of (level, N) used, or None."""
    vals = [c_int(0) for _ in range(6)]
    rc = load().lfm_tune_get(int(level), int(N), *[ctypes.byref(v) for v in vals])
    if rc != LFM_OK:
        return None
    return dict(zip(("vec", "tj", "stages", "ic", "threads", "smem"), (v.value for v in vals)))


def device_status(clear: bool = True) -> int:
    """The device status word (0 = no device-side wait gave up); synchronises the device."""
    v = c_int(0)
    call("lfm_device_status", ctypes.byref(v), 1 if clear else 0)
    return v.value


def check_device(where: str, device=None) -> None:
    """Raise LfmError if a kernel's bounded wait gave up since the last check.

    A step kernel whose wait runs out records LFM_ERR_DEVICE_TIMEOUT in the
    device status word and returns with its outputs partly written; the host
    learns of it here (the word is read after a device synchronisation and
    cleared), so the corrupted state is never returned silently.
    """
    if device is not None:
        import torch

        with torch.cuda.device(device):
            code = device_status(clear=True)
    else:
        code = device_status(clear=True)
    if code:
        raise LfmError(code, where, "a device-side wait gave up; the fields written by that "
                       "launch are incomplete")


__all__ = ["MaskLut", "LfmError", "load", "check", "call", "set_step_path", "device_status",
           "check_device",
           "exported_symbols", "c_float"]
