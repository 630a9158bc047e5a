"""CPU oracle for the leapfrog hot path.  TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this module, and only as the checker or the timed CPU
baseline.  The product package never imports it.

Contents
--------
* ``boundary_mask`` -- the cos^2 sponge, restating
  lfm/core/backends/numpy_backend.py:49-69 with the same float32 NumPy ops.
* ``helmholtz_sa`` -- the S_a smoothing, restating numpy_backend.py:341-356
  (NumPy's rfftn on float32 input returns complex64; the float64 filter
  promotes the product to complex128, so the inverse runs in float64).
* ``OracleBackend`` -- ``step_real`` / ``step_complex`` / ``step_color`` with
  the reference ``Backend`` signatures (lfm/core/backends/protocol.py:65-136),
  computed by the C restatement in ``lfm_oracle.cpp`` (float32: bit-exact to
  NumPy's float32 path; float64: the FP64 oracle).
* ``numpy_step_real`` -- the REAL step as the reference's NumPy whole-array
  operations (one core), the timed stand-in for the reference's CPU path.
* ``gaussian_soliton`` / ``equilibrate_chi`` / ``interior_mask`` -- the
  packet builder and the Poisson equilibration of lfm/fields/soliton.py and
  lfm/fields/equilibrium.py (NumPy restatements).
* seeded initial-condition builders for the benchmark and parity workloads.

Parity pins: ``tests/golden/`` holds fixtures produced by the reference
itself (``tests/golden/make_golden.py``); ``tests/test_oracle_golden.py``
checks this module against them bit for bit.
"""

from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "liblfm_oracle.so"
_lib = None


def build(force: bool = False) -> Path:
    """Compile lfm_oracle.cpp into liblfm_oracle.so beside it (g++, std::thread)."""
    src = _HERE / "lfm_oracle.cpp"
    if force or not _LIB_PATH.exists() or _LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.check_call(["make", "-s", "-C", str(_HERE)])
    return _LIB_PATH


def _load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(str(_LIB_PATH))
        f32 = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
        f64 = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        d = ctypes.c_double
        for suffix, p in (("f32", f32), ("f64", f64)):
            fn = getattr(lib, f"oracle_step_real_{suffix}")
            fn.argtypes = [p] * 9 + [ctypes.c_int] + [d] * 5
            fn.restype = None
            fn = getattr(lib, f"oracle_step_complex_{suffix}")
            fn.argtypes = [p] * 13 + [ctypes.c_int] + [d] * 6
            fn.restype = None
            fn = getattr(lib, f"oracle_step_color_{suffix}")
            fn.argtypes = [p] * 13 + [ctypes.c_int] + [d] * 10 + [ctypes.c_void_p]
            fn.restype = None
            fn = getattr(lib, f"oracle_laplacian_{suffix}")
            fn.argtypes = [p, p, ctypes.c_int]
            fn.restype = None
        lib.oracle_set_threads.argtypes = [ctypes.c_int]
        lib.oracle_set_plane_range.argtypes = [ctypes.c_int, ctypes.c_int]
        lib.oracle_max_threads.restype = ctypes.c_int
        _lib = lib
    return _lib


def set_threads(n: int) -> None:
    _load().oracle_set_threads(int(n))


def set_plane_range(i0: int = 0, i1: int = -1) -> None:
    """Step only planes [i0, i1) of the slowest axis (i1 < 0: to the end)."""
    _load().oracle_set_plane_range(int(i0), int(i1))


def max_threads() -> int:
    return int(_load().oracle_max_threads())


# --------------------------------------------------------------------------
# sponge mask and Helmholtz solve (NumPy restatements)
# --------------------------------------------------------------------------
def boundary_mask(N: int, boundary_fraction: float) -> np.ndarray:
    """Flat float32 cos^2 sponge, 0 inside, 1 outside (numpy_backend.py:60-69)."""
    center = N / 2.0
    r_max = N / 2.0
    r_freeze = (1.0 - boundary_fraction) * r_max
    c = np.arange(N, dtype=np.float32) - center + 0.5
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    R = np.sqrt(X**2 + Y**2 + Z**2)
    t = np.clip((R - r_freeze) / (r_max - r_freeze), 0.0, 1.0)
    return (np.sin(0.5 * np.pi * t) ** 2).astype(np.float32).ravel()


def helmholtz_filter(N: int, sa_gamma: float, sa_d: float) -> np.ndarray:
    """gamma / (gamma + D |k|^2) on the rfftn half spectrum, float64 (numpy_backend.py:342-346)."""
    kx = np.fft.fftfreq(N) * (2.0 * np.pi)
    kz = np.fft.rfftfreq(N) * (2.0 * np.pi)
    k_sq = kx[:, None, None] ** 2 + kx[None, :, None] ** 2 + kz[None, None, :] ** 2
    return np.float64(sa_gamma) / (np.float64(sa_gamma) + np.float64(sa_d) * k_sq)


def helmholtz_sa(color_energy: np.ndarray, N: int, sa_gamma: float, sa_d: float) -> np.ndarray:
    """Clipped S_a (3, N^3) from |Psi_a|^2 (3, N^3), in the input's precision.

    float32 input follows the reference exactly (complex64 forward, float64
    inverse, clip, cast to float32); float64 input is the FP64 oracle.
    """
    h = helmholtz_filter(N, sa_gamma, sa_d)
    out_dtype = color_energy.dtype
    out = np.empty((3, N**3), dtype=out_dtype)
    for a in range(3):
        hat = np.fft.rfftn(color_energy[a].reshape(N, N, N))
        s3 = np.fft.irfftn(h * hat, s=(N, N, N), axes=(0, 1, 2))
        out[a] = np.clip(s3, 0.0, None).astype(out_dtype).ravel()
    return out


def gaussian_soliton(N: int, position, amplitude: float, sigma: float, phase: float = 0.0):
    """Gaussian packet as lfm/fields/soliton.py:49-59 evaluates it: float32
    grid, float32 r^2 and envelope, times cos / sin of the phase."""
    x = np.arange(N, dtype=np.float32)
    px, py, pz = position
    r2 = ((x - px) ** 2)[:, None, None] + ((x - py) ** 2)[None, :, None] \
        + ((x - pz) ** 2)[None, None, :]
    env = amplitude * np.exp(-r2 / (2.0 * sigma**2))
    return (env * np.cos(phase)).astype(np.float32), (env * np.sin(phase)).astype(np.float32)


def interior_mask(N: int, boundary_fraction: float) -> np.ndarray:
    """lfm/analysis/structure.py:148-171: dist <= N/2 (1 - bf), float64 distances."""
    c = N / 2.0
    x = np.arange(N, dtype=np.float64)
    d2 = ((x - c) ** 2)[:, None, None] + ((x - c) ** 2)[None, :, None] \
        + ((x - c) ** 2)[None, None, :]
    return np.sqrt(d2) <= c * (1.0 - boundary_fraction)


def equilibrate_chi(psi_r: np.ndarray, psi_i, chi0: float, kappa: float, e0_sq: float = 0.0,
                    boundary_fraction: float | None = None) -> np.ndarray:
    """Poisson-equilibrated chi, restating lfm/fields/equilibrium.py:26-121.

    |Psi|^2 in float32 (colour sums over axis 0), rhs = kappa (|Psi|^2 - e0^2)
    in float32, a float32 forward FFT (NumPy >= 2 keeps single precision),
    the -1/k^2 divide in float64 (DC set to 0), a float64 inverse, then
    chi = chi0 + dchi in float32 and chi0 on the frozen shell
    (~interior_mask) when boundary_fraction is given.
    """
    if psi_r.ndim == 3:
        psi_sq = psi_r**2
        if psi_i is not None:
            psi_sq = psi_sq + psi_i**2
    else:
        psi_sq = np.sum(psi_r**2, axis=0)
        if psi_i is not None:
            psi_sq = psi_sq + np.sum(psi_i**2, axis=0)
    N = psi_sq.shape[0]
    rhs = kappa * (psi_sq - e0_sq)
    src = np.fft.rfftn(rhs)
    k = np.fft.fftfreq(N) * 2.0 * np.pi
    kz = np.fft.rfftfreq(N) * 2.0 * np.pi
    k2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + kz[None, None, :] ** 2
    k2[0, 0, 0] = 1.0
    phi = -src / k2
    phi[0, 0, 0] = 0.0
    dchi = np.fft.irfftn(phi, s=(N, N, N), axes=(0, 1, 2)).astype(np.float32)
    chi = (chi0 + dchi).astype(np.float32)
    if boundary_fraction is not None:
        chi[~interior_mask(N, boundary_fraction)] = chi0
    return chi


def color_energy(psi_r: np.ndarray, psi_i: np.ndarray, N: int) -> np.ndarray:
    """|Psi_a|^2 per colour, (3, N^3), in the input precision (numpy_backend.py:289)."""
    pr = psi_r.reshape(3, N**3)
    pi = psi_i.reshape(3, N**3)
    return pr * pr + pi * pi


def laplacian_19pt(field: np.ndarray) -> np.ndarray:
    """Periodic 19-point Laplacian of an (N, N, N) float32/float64 field (stencils.py:26-71)."""
    f = np.ascontiguousarray(field)
    N = f.shape[0]
    if f.shape != (N, N, N):
        raise ValueError("laplacian_19pt takes a cubic (N, N, N) field")
    out = np.empty_like(f)
    getattr(_load(), f"oracle_laplacian_{_dtype_suffix(f)}")(f.ravel(), out.ravel(), N)
    return out


# --------------------------------------------------------------------------
# the reference's CPU path as NumPy whole-array operations (for timing)
# --------------------------------------------------------------------------
# Neighbour offsets of the 19-point stencil in the order the reference sums
# them (lfm/core/stencils.py:43-71): np.roll(f, s, axis) is the f[x - s]
# neighbour; faces first, then the xy, xz and yz edges.
_FACE_ROLLS = ((1, 0), (-1, 0), (1, 1), (-1, 1), (1, 2), (-1, 2))
_EDGE_ROLLS = tuple(((s, a), (t, b)) for a, b in ((0, 1), (0, 2), (1, 2))
                    for s in (1, -1) for t in (1, -1))


def numpy_laplacian(f: np.ndarray) -> np.ndarray:
    """The 19-point Laplacian as the reference's NumPy code evaluates it: one rolled
    temporary per neighbour, summed left to right, then the three weightings."""
    faces = None
    for s, a in _FACE_ROLLS:
        t = np.roll(f, s, axis=a)
        faces = t if faces is None else faces + t
    edges = None
    for (s, a), (t_, b) in _EDGE_ROLLS:
        t = np.roll(np.roll(f, s, axis=a), t_, axis=b)
        edges = t if edges is None else edges + t
    return (1.0 / 3.0) * faces + (1.0 / 6.0) * edges + (-4.0) * f


def numpy_step_real(E, E_prev, chi, chi_prev, mask, N, dt2, kappa, lambda_self, chi0,
                    e0_sq):
    """One REAL step with NumPy whole-array operations, single-threaded, in the
    reference's order (numpy_backend.py:80-130).  Returns (E', E_prev', chi', chi_prev'),
    flat.  bench.py times it as the reference's own CPU path; tests pin it to the C oracle.
    Fields given as (P, N, N) arrays step as P planes wrapped in i (a slab with its
    ghost planes: its inner planes come out as the whole lattice's)."""
    shape = np.shape(E) if np.ndim(E) == 3 else (N, N, N)
    E, E_prev, chi, chi_prev, mask = (np.asarray(a).reshape(shape)
                                      for a in (E, E_prev, chi, chi_prev, mask))
    lap_e = numpy_laplacian(E)
    lap_x = numpy_laplacian(chi)
    chi_sq = chi * chi
    e_new = 2.0 * E - E_prev + dt2 * (lap_e - chi_sq * E)
    acc = lap_x - (kappa / chi0) * chi * (E * E - e0_sq)
    if lambda_self > 0:
        acc -= 4.0 * lambda_self * chi * (chi_sq - chi0 * chi0)
    chi_new = 2.0 * chi - chi_prev + dt2 * acc
    np.clip(chi_new, -chi0, None, out=chi_new)
    absorb = 1.0 - mask
    e_new *= absorb
    chi_new = mask * chi0 + absorb * chi_new
    return e_new.ravel(), (E * absorb).ravel(), chi_new.ravel(), chi.ravel().copy()


# --------------------------------------------------------------------------
# reference-signature step functions
# --------------------------------------------------------------------------
def _dtype_suffix(arr: np.ndarray) -> str:
    if arr.dtype == np.float32:
        return "f32"
    if arr.dtype == np.float64:
        return "f64"
    raise TypeError(f"oracle takes float32 or float64 arrays, got {arr.dtype}")


class OracleBackend:
    """CPU oracle with the reference Backend's step signatures."""

    name = "oracle"

    def create_boundary_mask(self, N: int, boundary_fraction: float) -> np.ndarray:
        return boundary_mask(N, boundary_fraction)

    def step_real(self, psi_in, psi_prev_in, chi_in, chi_prev_in, boundary_mask,
                  psi_out, psi_prev_out, chi_out, chi_prev_out,
                  N, dt2, kappa, lambda_self, chi0, e0_sq) -> None:
        suf = _dtype_suffix(psi_in)
        mask = np.ascontiguousarray(boundary_mask, dtype=psi_in.dtype)
        getattr(_load(), f"oracle_step_real_{suf}")(
            psi_in, psi_prev_in, chi_in, chi_prev_in, mask,
            psi_out, psi_prev_out, chi_out, chi_prev_out,
            int(N), float(dt2), float(kappa), float(lambda_self), float(chi0), float(e0_sq))

    def step_complex(self, psi_r_in, psi_r_prev_in, psi_i_in, psi_i_prev_in, chi_in,
                     chi_prev_in, boundary_mask, psi_r_out, psi_r_prev_out, psi_i_out,
                     psi_i_prev_out, chi_out, chi_prev_out,
                     N, dt2, kappa, lambda_self, chi0, e0_sq, epsilon_w) -> None:
        suf = _dtype_suffix(psi_r_in)
        mask = np.ascontiguousarray(boundary_mask, dtype=psi_r_in.dtype)
        getattr(_load(), f"oracle_step_complex_{suf}")(
            psi_r_in, psi_r_prev_in, psi_i_in, psi_i_prev_in, chi_in, chi_prev_in, mask,
            psi_r_out, psi_r_prev_out, psi_i_out, psi_i_prev_out, chi_out, chi_prev_out,
            int(N), float(dt2), float(kappa), float(lambda_self), float(chi0),
            float(e0_sq), float(epsilon_w))

    def step_color(self, psi_r_in, psi_r_prev_in, psi_i_in, psi_i_prev_in, chi_in,
                   chi_prev_in, boundary_mask, psi_r_out, psi_r_prev_out, psi_i_out,
                   psi_i_prev_out, chi_out, chi_prev_out,
                   N, dt2, kappa, lambda_self, chi0, e0_sq, epsilon_w,
                   kappa_c=0.0, epsilon_cc=0.0, kappa_string=0.0, kappa_tube=0.0,
                   sa_fields_in=None, sa_fields_out=None, sa_gamma=0.1, sa_d=4.9,
                   dt=0.02) -> None:
        suf = _dtype_suffix(psi_r_in)
        dtype = psi_r_in.dtype
        mask = np.ascontiguousarray(boundary_mask, dtype=dtype)
        sa = None
        if kappa_tube > 0 and sa_fields_out is not None:
            sa = helmholtz_sa(color_energy(psi_r_in, psi_i_in, N), N, sa_gamma, sa_d)
            np.copyto(sa_fields_out, sa.ravel())
        sa_ptr = None if sa is None else sa.ctypes.data
        getattr(_load(), f"oracle_step_color_{suf}")(
            psi_r_in, psi_r_prev_in, psi_i_in, psi_i_prev_in, chi_in, chi_prev_in, mask,
            psi_r_out, psi_r_prev_out, psi_i_out, psi_i_prev_out, chi_out, chi_prev_out,
            int(N), float(dt2), float(kappa), float(lambda_self), float(chi0),
            float(e0_sq), float(epsilon_w), float(kappa_c), float(epsilon_cc),
            float(kappa_string), float(kappa_tube), sa_ptr)


def _level_of(cfg) -> int:
    return int(getattr(cfg, "field_level"))


class OracleLattice:
    """Double-buffered oracle state driven like the reference Evolver (evolver.py:182-281).

    Holds flat arrays in ``dtype`` (float32 for the bit-exact path, float64
    for the FP64 oracle) and steps them with :class:`OracleBackend`.
    """

    def __init__(self, cfg, dtype=np.float32):
        self.cfg = cfg
        self.N = int(cfg.grid_size)
        self.dtype = np.dtype(dtype)
        self.level = _level_of(cfg)
        n = self.N**3
        npsi = 3 * n if self.level == 2 else n
        z = lambda m: np.zeros(m, dtype=self.dtype)  # noqa: E731
        self.pr, self.prp = z(npsi), z(npsi)
        self.pi, self.pip = (z(npsi), z(npsi)) if self.level > 0 else (None, None)
        self.chi = np.full(n, cfg.chi0, dtype=self.dtype)
        self.chip = self.chi.copy()
        self.sa = z(3 * n) if (self.level == 2 and cfg.kappa_tube > 0) else None
        self.mask = boundary_mask(self.N, cfg.boundary_fraction).astype(self.dtype)
        self._be = OracleBackend()
        self._out = [None if a is None else np.empty_like(a)
                     for a in (self.pr, self.prp, self.pi, self.pip, self.chi, self.chip)]
        self.step_count = 0

    def set_psi_real(self, a):
        self.pr[:] = np.asarray(a, dtype=self.dtype).ravel()
        self.prp[:] = self.pr

    def set_psi_imag(self, a):
        self.pi[:] = np.asarray(a, dtype=self.dtype).ravel()
        self.pip[:] = self.pi

    def set_chi(self, a):
        self.chi[:] = np.asarray(a, dtype=self.dtype).ravel()
        self.chip[:] = self.chi

    def step(self, steps: int = 1) -> None:
        c = self.cfg
        dt2 = c.dt**2
        for _ in range(steps):
            o = self._out
            if self.level == 0:
                self._be.step_real(self.pr, self.prp, self.chi, self.chip, self.mask,
                                   o[0], o[1], o[4], o[5], self.N, dt2, c.kappa,
                                   c.lambda_self, c.chi0, c.e0_sq)
            elif self.level == 1:
                self._be.step_complex(self.pr, self.prp, self.pi, self.pip, self.chi,
                                      self.chip, self.mask, o[0], o[1], o[2], o[3], o[4],
                                      o[5], self.N, dt2, c.kappa, c.lambda_self, c.chi0,
                                      c.e0_sq, c.epsilon_w)
            else:
                self._be.step_color(self.pr, self.prp, self.pi, self.pip, self.chi,
                                    self.chip, self.mask, o[0], o[1], o[2], o[3], o[4],
                                    o[5], self.N, dt2, c.kappa, c.lambda_self, c.chi0,
                                    c.e0_sq, c.epsilon_w, c.kappa_c, c.epsilon_cc,
                                    kappa_string=c.kappa_string, kappa_tube=c.kappa_tube,
                                    sa_fields_in=self.sa, sa_fields_out=self.sa,
                                    sa_gamma=c.sa_gamma, sa_d=c.sa_d, dt=c.dt)
            cur = [self.pr, self.prp, self.pi, self.pip, self.chi, self.chip]
            self.pr, self.prp, self.pi, self.pip, self.chi, self.chip = o
            self._out = cur
            self.step_count += 1


# --------------------------------------------------------------------------
# seeded initial conditions (shapes and value ranges of the benchmark configs)
# --------------------------------------------------------------------------
def gaussian_blob(N: int, center, amplitude: float, sigma: float) -> np.ndarray:
    """amplitude*exp(-r^2/(2 sigma^2)) on the N^3 grid in float32 (lfm/fields/soliton.py:49-59)."""
    x = np.arange(N, dtype=np.float32)
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    px, py, pz = center
    r2 = (X - px) ** 2 + (Y - py) ** 2 + (Z - pz) ** 2
    return (amplitude * np.exp(-r2 / (2.0 * sigma**2))).astype(np.float32)


def parity_seed_blob(N: int) -> np.ndarray:
    """5x5x5 blob 3*exp(-r^2/2) at the centre: the seed of tests/test_gpu_parity.py:49-60."""
    E = np.zeros((N, N, N), dtype=np.float32)
    c = N // 2
    for di in range(-2, 3):
        for dj in range(-2, 3):
            for dk in range(-2, 3):
                E[c + di, c + dj, c + dk] = 3.0 * np.exp(-(di * di + dj * dj + dk * dk) / 2.0)
    return E
