"""The five workload configurations at their stated sizes, against float64.

Each test runs one workload at the size and step count it is specified with
and compares the CUDA path with a float64 run of the reference step
(oracle/torch_ref.py: lfm/core/backends/numpy_backend.py:80-382 transcribed to
torch, run in float64 on the same GPU), or, for the batched sweep, with the
single-lattice path bit for bit:

1. REAL 64^3, 1000 steps (gravity_only, one packet of amplitude 6): E and chi
   of the plain and compensated float32 paths, chi_min and well_fraction over
   the interior; plus the float64 run's own sensitivity: the same run from an
   initial state perturbed by one float32 ulp (per cell at random, E scaled
   coherently, chi shifted uniformly) and the run with float64 arithmetic whose
   state is rounded to float32 after every step (all fields, Psi only, chi only).
2. REAL 512^3, 2000 steps (64 packets): E and chi errors and energy drift of
   both float32 paths.
3. COLOR 256^3, 500 steps (full_physics, S_a every step): every field.
4. The 256-lattice sweep, 200 steps in one CUDA graph: every lattice bit for
   bit as a single-lattice Evolver gives it.
5. The adjoint, COMPLEX 96^3, 500 steps (gravity_em): gradients of
   |chi_T - chi_target|^2 against float64 autograd through the transcription
   (checkpointed segments) and against float64 central differences (h = 1e-3).

Errors are max-relative per field, max|x - x64| / max|x64|.  Every number is
also written to the JSON file that LFM_ACCURACY_JSON names, when it is set:

    LFM_ACCURACY_JSON=profiles/accuracy.json python -m pytest tests/test_gpu_configs.py -m gpu
"""

from __future__ import annotations

import json
import math
import os
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import torch_ref as TR
from test_gpu_accuracy import accuracy_report, color_report, max_rel

pytestmark = pytest.mark.gpu

# Stated tolerances (max-relative against float64), about 1.5x what the
# configurations measured; see the recorded numbers in the JSON output.
TOL = {
    # config 1, 1000 steps: plain float32 E 8.8e-3, chi 5.2e-4; compensated 4.0e-3, 9.7e-5
    "c1_plain_E": 1.5e-2, "c1_plain_chi": 8e-4,
    "c1_comp_E": 6e-3, "c1_comp_chi": 1.5e-4,
    # split chi: the north-star bound itself (CPU emulation before the kernel: 3.9e-6, 4.7e-8)
    "split_E": 1e-5, "split_chi": 1e-6,
    # config 2, 2000 steps: plain E 1.1e-1, chi 1.6e-3; compensated 4.8e-3, 1.5e-4
    "c2_plain_E": 0.17, "c2_plain_chi": 2.5e-3,
    "c2_comp_E": 7.5e-3, "c2_comp_chi": 2.5e-4,
    "c2_drift_pp": 0.1,  # |float32 drift - float64 drift|, percentage points
    # config 3, 500 steps: every field <= 5.0e-5
    "c3_field": 1e-4,
    # config 5: the adjoint's own accuracy (CUDA adjoint and float64 VJP, one cotangent),
    # measured 2.5e-5 over 40 steps; over the 500 steps the float32 trajectory's drift
    # dominates (measured up to 2.5e-2 for psi_i)
    "c5_seeded": 1e-4, "c5_state_500": 5e-2,
    # config 5: float64 autograd against float64 central differences (h = 1e-3);
    # the per-cell chi offset's difference quotient carries the O(h^2) truncation
    # (measured 1.6e-3 with the standing packets)
    "c5_autograd_vs_fd": 1e-4, "c5_autograd_vs_fd_dchi": 5e-3,
    # config 5 with the split-chi forward: the workload's own loss against float64
    # central differences (h = 1e-3), amplitude, centre and phase
    "c5_split_vs_fd": 1e-4,
}


def record(section: str, data: dict) -> None:
    """Merge one section into the JSON file named by LFM_ACCURACY_JSON (if set)."""
    path = os.environ.get("LFM_ACCURACY_JSON")
    print(section, json.dumps(data, indent=1, default=float))
    if not path:
        return
    p = Path(path)
    doc = json.loads(p.read_text()) if p.exists() else {}
    doc[section] = data
    p.parent.mkdir(parents=True, exist_ok=True)
    p.write_text(json.dumps(doc, indent=1, sort_keys=True, default=float) + "\n")


@pytest.fixture(scope="module")
def be(cuda_device):
    from lfm_b200 import B200Backend
    from lfm_b200.build import build_library

    build_library()
    return B200Backend(cuda_device)


def _mask64(N, cfg, dev):
    from lfm_b200.mask import boundary_mask

    return torch.from_numpy(boundary_mask(N, cfg.boundary_fraction)).to(dev).double().view(
        N, N, N)


def _chi_stats(chi, interior):
    """chi_min and well_fraction (chi < 17) over the interior, in float64."""
    c = chi.double()[interior]
    return float(c.min()), float((c < 17.0).double().mean())


# ---------------------------------------------------------------- config 1
def test_config1_real64_1000_steps(be):
    from lfm_b200 import Evolver
    from lfm_b200.compensated import CompensatedEvolver
    from lfm_b200.config import gravity_only
    from lfm_b200.metrics import interior_mask
    from lfm_b200.split import SplitChiEvolver
    from lfm_b200.workloads import config1_soliton

    N, steps = 64, 1000
    cfg = gravity_only(N)
    dev = be.device
    E = config1_soliton(N)
    mask = _mask64(N, cfg, dev)
    interior = torch.from_numpy(interior_mask(N, cfg.boundary_fraction)).to(dev)

    def run64(e0, chi0=None, round_fields=()):
        e = torch.from_numpy(e0).to(dev).double() if isinstance(e0, np.ndarray) else e0
        x = torch.full_like(e, cfg.chi0) if chi0 is None else chi0
        s = {"pr": e, "prp": e.clone(), "chi": x, "chip": x.clone()}
        if not round_fields:
            return TR.run(cfg, s, steps, mask)
        for _ in range(steps):
            s = TR.run(cfg, s, 1, mask)
            for k in round_fields:
                s[k] = s[k].float().double()
        return s

    ref = run64(E)
    out = {"N": N, "steps": steps, "workload": "REAL gravity_only, packet 6.0 sigma 3 + 1e-4 noise"}
    cmin, wf = _chi_stats(ref["chi"], interior)
    out["fp64"] = {"chi_min": cmin, "well_fraction": wf}
    for name, cls in (("plain_f32", Evolver), ("compensated_f32", CompensatedEvolver),
                      ("split_f32", SplitChiEvolver)):
        ev = cls(cfg, backend=be)
        ev.set_psi_real(E)
        ev.evolve(steps)
        st = ev.device_state()
        pr, chi = st["psi_r"].view(N, N, N), st["chi"].view(N, N, N)
        m = ev.metrics()
        cmin32, wf32 = _chi_stats(chi, interior)
        out[name] = {"max_rel_error_E": max_rel(pr, ref["pr"]),
                     "max_rel_error_chi": max_rel(st.get("chi64", chi).view(N, N, N),
                                                  ref["chi"]),
                     "chi_min": m["chi_min"], "chi_min_interior_check": cmin32,
                     "well_fraction": m["well_fraction"], "well_fraction_check": wf32}
    # sensitivity of the float64 run itself
    rng = np.random.default_rng(7)
    up = np.where(rng.integers(0, 2, E.shape) == 1, np.inf, -np.inf).astype(np.float32)
    sens = {}
    variants = {
        "E_random_1ulp": dict(e0=np.nextafter(E, up)),
        "E_scaled_1ulp": dict(e0=torch.from_numpy(E).to(dev).double() * (1.0 + 2.0**-24)),
        "chi_plus_1ulp": dict(e0=E, chi0=torch.full((N, N, N), cfg.chi0 + 2.0**-19,
                                                    dtype=torch.float64, device=dev)),
        "f32_storage_every_step": dict(e0=E, round_fields=("pr", "prp", "chi", "chip")),
        "f32_storage_psi_only": dict(e0=E, round_fields=("pr", "prp")),
        "f32_storage_chi_only": dict(e0=E, round_fields=("chi", "chip")),
    }
    for k, kw in variants.items():
        s = run64(**kw)
        sens[k] = {"max_rel_E": max_rel(s["pr"], ref["pr"]),
                   "max_rel_chi": max_rel(s["chi"], ref["chi"])}
    out["fp64_sensitivity"] = sens
    record("config1_real64_1000", out)

    p, c, sp = out["plain_f32"], out["compensated_f32"], out["split_f32"]
    assert p["max_rel_error_E"] < TOL["c1_plain_E"] and p["max_rel_error_chi"] < TOL["c1_plain_chi"]
    assert c["max_rel_error_E"] < TOL["c1_comp_E"] and c["max_rel_error_chi"] < TOL["c1_comp_chi"]
    assert c["max_rel_error_chi"] < p["max_rel_error_chi"]
    # within 1e-5 of float64 after 1000 float32-stored steps
    assert sp["max_rel_error_E"] < TOL["split_E"] and sp["max_rel_error_chi"] < TOL["split_chi"]
    for r in (p, c, sp):
        assert r["chi_min"] == r["chi_min_interior_check"]
        assert r["well_fraction"] == pytest.approx(r["well_fraction_check"], abs=1e-12)
        assert abs(r["chi_min"] - cmin) < 1e-3 * abs(cmin)
        assert abs(r["well_fraction"] - wf) < 2e-3
    # a random one-ulp perturbation of the initial state stays far below the float32 paths'
    # error: their error is made along the run, not inherited from the initial rounding
    assert sens["E_random_1ulp"]["max_rel_E"] < 1e-5


# ---------------------------------------------------------------- config 2
def test_config2_real512_2000_steps(be):
    r = accuracy_report(512, 2000, be.device)
    record("config2_real512_2000", r)
    p, c = r["plain_f32"], r["compensated_f32"]
    assert p["max_rel_error_E"] < TOL["c2_plain_E"] and p["max_rel_error_chi"] < TOL["c2_plain_chi"]
    assert c["max_rel_error_E"] < TOL["c2_comp_E"] and c["max_rel_error_chi"] < TOL["c2_comp_chi"]
    for q in (p, c):
        assert q["energy_T"] == pytest.approx(q["energy_T_energy64"], rel=1e-9)
        assert abs(q["drift_minus_fp64_drift"]) < TOL["c2_drift_pp"]
    assert abs(c["drift_minus_fp64_drift"]) <= abs(p["drift_minus_fp64_drift"])


# ---------------------------------------------------------------- config 3
def test_config3_color256_500_steps(be):
    r = color_report(256, 500, be.device)
    record("config3_color256_500", r)
    errs = {k: v for k, v in r.items() if k.startswith("max_rel")}
    assert all(np.isfinite(v) for v in errs.values()), errs
    assert max(errs.values()) < TOL["c3_field"], errs


# ---------------------------------------------------------------- config 4
def test_config4_all_256_lattices_bit_exact(be):
    from lfm_b200 import Evolver
    from lfm_b200.batch import BatchedLattices
    from lfm_b200.workloads import sweep_lattices

    steps = 200
    L = sweep_lattices(256, seed=5)
    B = BatchedLattices([c for c, _, _ in L], backend=be)
    B.graph_block = steps
    for i, (_, pr, pi) in enumerate(L):
        B.set_psi_real(i, pr)
        if pi is not None:
            B.set_psi_imag(i, pi)
    B.evolve(steps)
    mismatched = []
    for i, (c, pr, pi) in enumerate(L):
        ev = Evolver(c, backend=be)
        ev.set_psi_real(pr)
        if pi is not None:
            ev.set_psi_imag(pi)
        ev.evolve(steps)
        same = (np.array_equal(B.get_psi_real(i).view(np.uint32), ev.get_psi_real().view(np.uint32))
                and np.array_equal(B.get_chi(i).view(np.uint32), ev.get_chi().view(np.uint32))
                and np.array_equal(B.get_psi_real_prev(i).view(np.uint32),
                                   ev.get_psi_real_prev().view(np.uint32)))
        if pi is not None:
            same = same and np.array_equal(B.get_psi_imag(i).view(np.uint32),
                                           ev.get_psi_imag().view(np.uint32))
        if not same:
            mismatched.append(i)
        del ev
    record("config4_sweep256_200", {"lattices": len(L), "steps": steps,
                                    "cells": int(sum(c.grid_size**3 for c, _, _ in L)),
                                    "bit_exact_lattices": len(L) - len(mismatched)})
    assert not mismatched, mismatched


# ---------------------------------------------------------------- config 5
def _state64(N, params, sigma, cfg, dchi, dev):
    from lfm_b200.adjoint import soliton_state

    amp, cen, ph = params
    return soliton_state(N, amp, cen, ph, sigma, cfg.chi0, dchi, True, device=dev,
                         dtype=torch.float64, omega_dt=cfg.chi0 * cfg.dt)


def _run64(cfg, st, steps, mask, seg: int = 0):
    """chi after `steps` float64 steps; with seg > 0, autograd keeps only the
    state at every seg-th step and recomputes the steps between (checkpoints)."""
    from torch.utils.checkpoint import checkpoint

    keys = ("pr", "prp", "pi", "pip", "chi", "chip")
    s = dict(zip(keys, st))

    def advance(n, *t):
        out = TR.run(cfg, dict(zip(keys, t)), n, mask)
        return tuple(out[k] for k in keys)

    done = 0
    while done < steps:
        n = min(seg, steps - done) if seg > 0 else steps - done
        t = tuple(s[k] for k in keys)
        if seg > 0 and torch.is_grad_enabled():
            t = checkpoint(advance, n, *t, use_reentrant=False)
        else:
            t = advance(n, *t)
        s = dict(zip(keys, t))
        done += n
    return s["chi"]


def test_config5_adjoint_complex96_500_steps(be):
    """Gradients of the adjoint workload's loss |chi_T - chi_target|^2.

    Three comparisons: (1) the CUDA adjoint against the float64 VJP, both
    seeded with the same smooth cotangent 2 (chi64_T - chi_target) -- the
    adjoint's own accuracy at full size; (2) float64 autograd against float64
    central differences (h = 1e-3) -- the pin of the float64 gradient; (3) the
    gradient of the float32 run's own loss against the float64 one, beside the
    part of that gap the float32 forward's chi error explains (the float64 VJP
    seeded with the float32 run's cotangent): at step 500 chi has swung back
    to within ~1e-5 of chi0 (its forced oscillation under the Mexican hat is
    near the end of a cycle), below the float32 chi error of ~1e-4, so the
    float32 run's loss gradient is set by that error, not by the adjoint."""
    from lfm_b200.adjoint import leapfrog, soliton_state
    from lfm_b200.config import gravity_em
    from lfm_b200.workloads import adjoint_packets

    N, steps = 96, 500
    cfg = gravity_em(N)
    dev = be.device
    mask = _mask64(N, cfg, dev)
    (amp, cen, ph), tgt, sigma = adjoint_packets(N)
    params = [t.to(dev) for t in (amp, cen, ph)]
    with torch.no_grad():
        target = _run64(cfg, _state64(N, [t.to(dev) for t in tgt], sigma, cfg, None, dev),
                        steps, mask)

    def cuda_run():
        p32 = [p.float().clone().requires_grad_(True) for p in params]
        d32 = torch.zeros((N, N, N), device=dev, requires_grad=True)
        st = soliton_state(N, *p32, sigma, cfg.chi0, d32, True, omega_dt=cfg.chi0 * cfg.dt)
        out = leapfrog(cfg, st, steps, backend=be)
        return p32 + [d32], out[4].view(N, N, N)

    # float64 autograd through the transcription, checkpointed every 25 steps
    def f64_grads(cotangent=None):
        p = [t.clone().requires_grad_(True) for t in params]
        d = torch.zeros((N, N, N), device=dev, dtype=torch.float64, requires_grad=True)
        chi = _run64(cfg, _state64(N, p, sigma, cfg, d, dev), steps, mask, seg=25)
        loss = ((chi - target) ** 2).sum() if cotangent is None else (cotangent * chi).sum()
        return loss, torch.autograd.grad(loss, p + [d]), chi.detach()

    loss64, g64, chi64 = f64_grads()
    cot64 = 2.0 * (chi64 - target)

    # (1) the adjoint's own output, seeded with the float64 cotangent: the gradient with
    # respect to the whole initial state (six fields), against the float64 VJP from the
    # same (float32-rounded) initial state; over 40 steps with a random cotangent (the
    # float32 and float64 trajectories still agree to ~1e-6) and over the 500 steps
    with torch.no_grad():
        st0 = [t.float() for t in _state64(N, params, sigma, cfg, None, dev)]

    def state_grads(n, cot):
        st32 = [t.clone().requires_grad_(True) for t in st0]
        out = leapfrog(cfg, st32, n, backend=be)
        g32_ = torch.autograd.grad(out[4].view(N, N, N), st32, grad_outputs=cot.float())
        st64 = [t.double().requires_grad_(True) for t in st0]
        chi_s = _run64(cfg, st64, n, mask, seg=25)
        g64_ = torch.autograd.grad((cot * chi_s).sum(), st64)
        return g32_, g64_

    fields = ("psi_r", "psi_r_prev", "psi_i", "psi_i_prev", "chi", "chi_prev")
    gen = torch.Generator().manual_seed(3)
    g_short = state_grads(40, torch.randn(N, N, N, generator=gen, dtype=torch.float64).to(dev))
    gst32, gst64 = state_grads(steps, cot64)
    # ... and contracted to the packet parameters
    inp, chi32 = cuda_run()
    g_seed32 = torch.autograd.grad(chi32, inp, grad_outputs=cot64.float())
    _, g_seed64, _ = f64_grads(cot64)
    # (3) the float32 run's own loss
    inp, chi32 = cuda_run()
    loss32 = ((chi32.double() - target) ** 2).sum()
    g32 = torch.autograd.grad(loss32, inp)
    cot32 = 2.0 * (chi32.detach().double() - target)
    _, g_floor, _ = f64_grads(cot32)

    # (4) the split-chi forward (chi as chi0 + hi + lo, to about 48 bits, returned in
    # float64): the gradient of the workload's own loss
    def cuda_run_split():
        p32 = [p.float().clone().requires_grad_(True) for p in params]
        d64 = torch.zeros((N, N, N), device=dev, dtype=torch.float64, requires_grad=True)
        st = soliton_state(N, *p32, sigma, cfg.chi0, None, True, omega_dt=cfg.chi0 * cfg.dt)
        st[4] = st[5] = cfg.chi0 + d64
        out = leapfrog(cfg, st, steps, backend=be, split_chi=True)
        return p32 + [d64], out[4].view(N, N, N)

    inp, chi_sp = cuda_run_split()
    loss_sp = ((chi_sp - target) ** 2).sum()
    g_sp = torch.autograd.grad(loss_sp, inp)

    # (2) float64 central differences, h = 1e-3
    h = 1e-3
    probes = [(0, (0,)), (0, (1,)), (1, (0, 0)), (1, (0, 1)), (1, (1, 2)), (2, (0,)), (2, (1,))]
    c0 = int(round(float(cen[0, 0])))
    cells = [(c0, int(round(float(cen[0, 1]))), c0), (c0, int(round(float(cen[1, 1]))) + 2, c0),
             (c0 + 3, N // 2, c0 - 1)]
    probes += [(3, cell) for cell in cells]
    fd = {}
    with torch.no_grad():
        for pi_, idx in probes:
            vals = []
            for sgn in (1.0, -1.0):
                p = [t.clone() for t in params]
                d = torch.zeros((N, N, N), device=dev, dtype=torch.float64)
                (p + [d])[pi_][idx] += sgn * h
                chi = _run64(cfg, _state64(N, p, sigma, cfg, d, dev), steps, mask)
                vals.append(float(((chi - target) ** 2).sum()))
            fd[(pi_, idx)] = (vals[0] - vals[1]) / (2.0 * h)

    names = ("amplitude", "centre", "phase", "dchi")

    def rel(a, b):
        return float((a.double() - b.double()).abs().max() / b.double().abs().max())

    def rel_fd(g):
        """max over probes of |g - fd| / max|g64 of that parameter group|"""
        worst = {}
        for (pi_, idx), v in fd.items():
            scale = float(g64[pi_].abs().max())
            e = abs(float(g[pi_][idx]) - v) / scale
            worst[names[pi_]] = max(worst.get(names[pi_], 0.0), e)
        return worst

    res = {
        "N": N, "steps": steps, "workload": "COMPLEX 96^3 gravity_em, two rotating packets "
        "(prev phase + chi0 dt, as Simulation.place_soliton) + per-cell chi offset, loss "
        "|chi_T - chi_target|^2 (lfm_b200.workloads.adjoint_packets)",
        "loss_f32": float(loss32.detach()), "loss_f64": float(loss64.detach()),
        "chi_f32_max_abs_error": float((chi32.detach().double() - chi64).abs().max()),
        "chi_minus_target_max_abs": float((chi64 - target).abs().max()),
        "chi_minus_chi0_max_abs": float((chi64 - cfg.chi0).abs().max()),
        "grad_max_f64": {n: float(g.abs().max()) for n, g in zip(names, g64)},
        "adjoint_state_gradient_vs_f64_vjp_40_steps": {
            f: rel(a, b) for f, a, b in zip(fields, *g_short)},
        "adjoint_state_gradient_vs_f64_vjp": {
            f: rel(a, b) for f, a, b in zip(fields, gst32, gst64)},
        "adjoint_vs_f64_vjp_same_cotangent": {n: rel(a, b)
                                              for n, a, b in zip(names, g_seed32, g_seed64)},
        "state_gradient_max_f64": float(max(g.abs().max() for g in gst64)),
        "f64_autograd_vs_fd": rel_fd(g64),
        "f32_loss_gradient_vs_f64": {n: rel(a, b) for n, a, b in zip(names, g32, g64)},
        "float32_forward_floor": {n: rel(a, b) for n, a, b in zip(names, g_floor, g64)},
        "f32_loss_gradient_vs_fd": rel_fd(g32),
        "chi_split_max_abs_error": float((chi_sp.detach() - chi64).abs().max()),
        "split_loss_gradient_vs_f64": {n: rel(a, b) for n, a, b in zip(names, g_sp, g64)},
        "split_loss_gradient_vs_fd": rel_fd(g_sp),
        "fd_h": h, "fd_probes": len(fd),
    }
    record("config5_adjoint_complex96_500", res)
    # (1) the adjoint itself: its output, the gradient of every initial field.  Where the
    # float32 trajectory it linearises about still agrees with the float64 one (40 steps)
    # it matches the float64 VJP to the stated bound; over the 500 steps the float32
    # forward's drift (chi ~1e-4 absolute) moves the linearisation point, and the state
    # gradient follows it (measured 5e-5 for chi up to 2.5e-2 for psi_i near the packets).
    # The packet parameters' gradients contract the state gradient over the lattice; at
    # step 500 those sums cancel to a few 1e-8 against per-cell values near 1e-4.
    assert max(res["adjoint_state_gradient_vs_f64_vjp_40_steps"].values()) < TOL["c5_seeded"]
    assert max(res["adjoint_state_gradient_vs_f64_vjp"].values()) < TOL["c5_state_500"]
    assert res["adjoint_vs_f64_vjp_same_cotangent"]["dchi"] < TOL["c5_seeded"]
    # (2) the float64 gradient against differences (the per-cell chi offset's central
    # difference carries an O(h^2) truncation error at h = 1e-3)
    fd_err = res["f64_autograd_vs_fd"]
    assert max(fd_err[n] for n in ("amplitude", "centre", "phase")) < TOL["c5_autograd_vs_fd"]
    assert fd_err["dchi"] < TOL["c5_autograd_vs_fd_dchi"]
    # (3) the float32 forward's chi error accounts for the rest
    for n in names:
        assert res["f32_loss_gradient_vs_f64"][n] <= 1.5 * res["float32_forward_floor"][n] + 1e-3
    assert math.isfinite(res["loss_f32"]) and res["loss_f64"] > 0.0
    # (4) with the split-chi forward the workload's own loss is resolved
    sp = res["split_loss_gradient_vs_fd"]
    assert max(sp[n] for n in ("amplitude", "centre", "phase")) < TOL["c5_split_vs_fd"]


if __name__ == "__main__":
    import sys

    sys.exit(pytest.main([__file__, "-m", "gpu", "-q", "-s"]))
