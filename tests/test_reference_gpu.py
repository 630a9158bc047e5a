"""The reference's own CUDA step kernels on the same GPU: a tolerance check and a timing.

The reference's GPU backend (lfm/core/backends/cupy_backend.py) compiles three
RawKernel sources (lfm/core/backends/kernel_source.py) and launches one thread
per cell.  oracle/build_ref_gpu.py builds those sources, unchanged, into
oracle/_ref/libref_gpu.so with launchers of the same shape.  The kernels
contract multiplies into FMAs and sum their stencils in their own order, so
they are not bit-exact to the NumPy path; the reference holds them to
atol 2e-4 / rtol 1e-4 after 50 steps against NumPy (tests/test_gpu_parity.py
of the reference), and so does this file, against the oracle.

Run as a script to time them beside the fused kernels at the benchmark sizes:

    python tests/test_reference_gpu.py            # REAL 512^3, COMPLEX 256^3, COLOR 256^3
"""

from __future__ import annotations

import ctypes
import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
for _p in (ROOT, ROOT / "lfm-physics_b200"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

LIB = ROOT / "oracle" / "_ref" / "libref_gpu.so"
_F = ctypes.c_float
_P = ctypes.c_void_p


def load_ref():
    if not LIB.exists():
        pytest.skip("oracle/_ref/libref_gpu.so not built (needs the reference checkout)")
    lib = ctypes.CDLL(str(LIB))
    lib.ref_evolve_real.argtypes = [_P] * 9 + [ctypes.c_int] + [_F] * 5 + [_P]
    lib.ref_evolve_complex.argtypes = [_P] * 13 + [ctypes.c_int] + [_F] * 6 + [_P]
    lib.ref_evolve_color.argtypes = ([_P] * 13 + [ctypes.c_int] + [_F] * 8 + [_P] + [_F] * 2
                                     + [_P])
    for f in (lib.ref_evolve_real, lib.ref_evolve_complex, lib.ref_evolve_color):
        f.restype = ctypes.c_int
    return lib


class RefLattice:
    """A/B buffers stepped by the reference's kernel (as cupy_backend.py steps them)."""

    def __init__(self, lib, cfg, device):
        import torch

        from lfm_b200.mask import boundary_mask

        self.lib, self.cfg = lib, cfg
        N = cfg.grid_size
        self.level = int(cfg.field_level)
        comps = 3 if self.level == 2 else 1
        n = N**3
        z = lambda m: torch.zeros(m, dtype=torch.float32, device=device)  # noqa: E731
        self.names = ["pr", "prp", "chi", "chip"] + (["pi", "pip"] if self.level else [])
        size = {"pr": comps * n, "prp": comps * n, "pi": comps * n, "pip": comps * n,
                "chi": n, "chip": n}
        self.A = {k: z(size[k]) for k in self.names}
        self.B = {k: z(size[k]) for k in self.names}
        self.mask = torch.from_numpy(boundary_mask(N, cfg.boundary_fraction)).to(device)
        self.sa = z(3 * n if self.level == 2 else 4)  # read only with the tube coupling
        self.stream = torch.cuda.current_stream(device).cuda_stream

    def set(self, key, arr):
        import torch

        t = torch.as_tensor(np.ascontiguousarray(arr, dtype=np.float32).ravel())
        self.A[key].copy_(t)
        self.A[key + "p" if key != "chi" else "chip"].copy_(t)

    def step(self):
        c, a, b = self.cfg, self.A, self.B
        p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
        common = [c.grid_size, c.dt**2, c.kappa, c.lambda_self, c.chi0, c.e0_sq]
        if self.level == 0:
            rc = self.lib.ref_evolve_real(p(a["pr"]), p(a["prp"]), p(a["chi"]), p(a["chip"]),
                                          p(self.mask), p(b["pr"]), p(b["prp"]), p(b["chi"]),
                                          p(b["chip"]), *common, ctypes.c_void_p(self.stream))
        else:
            ins = [p(a["pr"]), p(a["prp"]), p(a["pi"]), p(a["pip"]), p(a["chi"]), p(a["chip"]),
                   p(self.mask)]
            outs = [p(b["pr"]), p(b["prp"]), p(b["pi"]), p(b["pip"]), p(b["chi"]), p(b["chip"])]
            if self.level == 1:
                rc = self.lib.ref_evolve_complex(*ins, *outs, *common, c.epsilon_w,
                                                 ctypes.c_void_p(self.stream))
            else:
                rc = self.lib.ref_evolve_color(*ins, *outs, *common, c.epsilon_w, c.kappa_c,
                                               c.epsilon_cc, p(self.sa), c.kappa_string,
                                               c.kappa_tube, ctypes.c_void_p(self.stream))
        assert rc == 0, rc
        self.A, self.B = self.B, self.A

    def get(self, key):
        return self.A[key].cpu().numpy()


def _config(level: str, N: int):
    from lfm_b200.config import FieldLevel, SimulationConfig

    if level == "real":
        return SimulationConfig(grid_size=N, boundary_fraction=0.15)
    if level == "complex":
        return SimulationConfig(grid_size=N, boundary_fraction=0.15,
                                field_level=FieldLevel.COMPLEX, lambda_self=4.0 / 31.0)
    return SimulationConfig(grid_size=N, boundary_fraction=0.15, field_level=FieldLevel.COLOR,
                            lambda_self=4.0 / 31.0, kappa_c=1.0 / 189.0,
                            epsilon_cc=2.0 / 17.0, kappa_string=1.0 / 189.0, kappa_tube=0.0)


@pytest.mark.gpu
@pytest.mark.parametrize("level", ["real", "complex", "color"])
def test_reference_kernels_against_the_oracle(cuda_device, level):
    """50 steps from the reference's GPU-parity seed (N = 16): the reference's own
    kernels stay within the reference's own GPU/NumPy tolerance of the oracle."""
    from oracle import oracle as O

    lib = load_ref()
    N = 16
    cfg = _config(level, N)
    E = O.parity_seed_blob(N)
    ref = RefLattice(lib, cfg, cuda_device)
    lat = O.OracleLattice(cfg)
    if level == "color":
        pr = np.zeros((3, N, N, N), np.float32)
        pr[0] = E
        pi = np.zeros_like(pr)
        pi[1] = 0.5 * E
        ref.set("pr", pr)
        ref.set("pi", pi)
        lat.set_psi_real(pr)
        lat.set_psi_imag(pi)
    else:
        ref.set("pr", E)
        lat.set_psi_real(E)
        if level == "complex":
            ref.set("pi", 0.25 * E)
            lat.set_psi_imag(0.25 * E)
    ref.set("chi", np.full((N, N, N), cfg.chi0, np.float32))
    for _ in range(50):
        ref.step()
    lat.step(50)
    np.testing.assert_allclose(ref.get("pr"), lat.pr, atol=2e-4, rtol=1e-4)
    np.testing.assert_allclose(ref.get("chi"), lat.chi, atol=2e-4, rtol=1e-4)
    if level != "real":
        np.testing.assert_allclose(ref.get("pi"), lat.pi, atol=2e-4, rtol=1e-4)
    # not bit-exact: FMA contraction and the kernels' own summation order
    print(level, "max |ref kernel - oracle|:", float(np.abs(ref.get("pr") - lat.pr).max()),
          float(np.abs(ref.get("chi") - lat.chi).max()))


def timing_report(device: str = "cuda:0", steps: int = 100) -> dict:
    """Reference kernels and fused kernels, device-timed on the same workloads."""
    import torch

    from lfm_b200 import B200Backend, Evolver
    from lfm_b200.config import full_physics, gravity_em, gravity_only
    from lfm_b200.workloads import color_packets, real_solitons

    lib = load_ref()
    be = B200Backend(device)
    s = torch.cuda.current_stream(device)

    def timed(fn, k):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        for _ in range(k):
            fn()
        b.record(s)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / k

    out = {}
    for name, cfg, ref_bytes, our_bytes in (
            ("REAL 512^3", gravity_only(512), 36, 24),
            ("COMPLEX 256^3", gravity_em(256), 52, 36),
            ("COLOR 256^3 stencil (no tube coupling)", full_physics(256, kappa_tube=0.0), 116, 84)):
        N = cfg.grid_size
        lvl = int(cfg.field_level)
        if lvl == 2:
            pr, pi, chi = color_packets(N)
        else:
            pr, chi = real_solitons(N)
            pi = 0.5 * pr if lvl == 1 else None
        ref = RefLattice(lib, cfg, device)
        ref.set("pr", pr)
        if pi is not None:
            ref.set("pi", pi)
        ref.set("chi", chi)
        for _ in range(4):
            ref.step()
        ms_ref = timed(ref.step, steps)
        del ref
        torch.cuda.empty_cache()
        ev = Evolver(cfg, backend=be)
        ev.set_psi_real(pr)
        if pi is not None:
            ev.set_psi_imag(pi)
        ev.set_chi(chi)
        ev.evolve(4)
        ev.warm_graphs()
        ms_ours = timed(lambda: ev.evolve(steps), 1) / steps
        del ev
        torch.cuda.empty_cache()
        cells = N**3
        out[name] = {
            "reference_kernel": {"ms_per_step": ms_ref, "gcells": cells / ms_ref / 1e6,
                                 "bytes_per_cell": ref_bytes,
                                 "gbs": ref_bytes * cells / ms_ref / 1e6},
            "fused_kernel": {"ms_per_step": ms_ours, "gcells": cells / ms_ours / 1e6,
                             "bytes_per_cell": our_bytes,
                             "gbs": our_bytes * cells / ms_ours / 1e6},
            "speedup": ms_ref / ms_ours,
        }
        print(name, json.dumps(out[name]), flush=True)
    return out


if __name__ == "__main__":
    print(json.dumps(timing_report(), indent=1))
