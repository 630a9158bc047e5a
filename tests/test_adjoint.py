"""Adjoint of the leapfrog step against float64 autograd and central differences.

The oracle is the plain PyTorch transcription of the reference step
(oracle/torch_ref.py) run in float64: its autograd gradients are pinned
against central finite differences on the CPU first, then the CUDA adjoint
(float32 forward and adjoint) is compared with them.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import torch_ref as TR

# float32 forward + float32 adjoint against float64 gradients, relative to the
# largest gradient component (max-norm)
GRAD_RTOL = 1e-4


def rel(a, b) -> float:
    a = torch.as_tensor(a, dtype=torch.float64).reshape(-1)
    b = torch.as_tensor(b, dtype=torch.float64).reshape(-1).to(a.device)
    return float((a - b).abs().max() / b.abs().max().clamp_min(1e-300))


def make_params(n_sol, N, seed, device, dtype):
    g = torch.Generator().manual_seed(seed)
    amp = (1.0 + 3.0 * torch.rand(n_sol, generator=g, dtype=torch.float64))
    cen = N / 2.0 + (torch.rand(n_sol, 3, generator=g, dtype=torch.float64) - 0.5) * (N / 4.0)
    ph = 2.0 * np.pi * torch.rand(n_sol, generator=g, dtype=torch.float64)
    dchi = 1e-3 * torch.randn(N, N, N, generator=g, dtype=torch.float64)
    return [t.to(device=device, dtype=dtype) for t in (amp, cen, ph, dchi)]


def ref_loss(cfg, params, target, steps, sigma, complex_level):
    """Loss through the float64 transcription (differentiable in every parameter)."""
    from lfm_b200.adjoint import soliton_state
    from lfm_b200.mask import boundary_mask

    amp, cen, ph, dchi = params
    N = cfg.grid_size
    st = soliton_state(N, amp, cen, ph, sigma, cfg.chi0, dchi, complex_level,
                       device=amp.device, dtype=torch.float64)
    mask = torch.from_numpy(boundary_mask(N, cfg.boundary_fraction).reshape(N, N, N)).to(
        amp.device, torch.float64)
    s = {"pr": st[0], "prp": st[1], "chi": st[4], "chip": st[5]}
    if complex_level:
        s.update(pi=st[2], pip=st[3])
    out = TR.run(cfg, s, steps, mask)
    return loss_of(out["chi"], out["pr"], target)


def loss_of(chi, pr, target):
    """(chi - target)^2 summed, or, with target = (w, v), sum(w chi + v psi_r):
    a loss whose cotangents float32 state resolves to full precision."""
    if isinstance(target, tuple):
        w, v = target
        return (w * chi.double()).sum() + (v * pr.double()).sum()
    return ((chi.double() - target) ** 2).sum()


def linear_target(N, device, seed=12):
    g = torch.Generator().manual_seed(seed)
    w = torch.randn(N, N, N, generator=g, dtype=torch.float64).to(device)
    v = torch.randn(N, N, N, generator=g, dtype=torch.float64).to(device)
    return (w, v)


# ---------------------------------------------------------------- host only
def test_checkpoint_memory_of_both_forms():
    from lfm_b200.adjoint import memory_bytes
    from lfm_b200.config import gravity_em

    cfg = gravity_em(96)
    n = 96**3
    plain, split = memory_bytes(cfg, 500), memory_bytes(cfg, 500, split_chi=True)
    # every = ceil(sqrt(500)) = 23 steps, 22 checkpoints
    assert plain["checkpoints"] == split["checkpoints"] == 22
    assert plain["checkpoint_bytes"] == 22 * 6 * 4 * n
    assert split["checkpoint_bytes"] == 22 * 8 * 4 * n
    assert plain["segment_bytes"] == 23 * 3 * 4 * n
    assert split["segment_bytes"] == 23 * 4 * 4 * n


# ---------------------------------------------------------------- oracle pin (CPU)
@pytest.mark.parametrize("level", ["real", "complex"])
def test_float64_autograd_matches_central_differences(level):
    from lfm_b200.config import gravity_em, gravity_only

    N, steps, sigma = 8, 6, 1.5
    cfg = (gravity_em if level == "complex" else gravity_only)(N, kappa=2.0 / 63.0)
    cx = level == "complex"
    params = make_params(1, N, 3, "cpu", torch.float64)
    target = torch.full((N, N, N), cfg.chi0, dtype=torch.float64) + 1e-3
    for p in params:
        p.requires_grad_(True)
    loss = ref_loss(cfg, params, target, steps, sigma, cx)
    grads = torch.autograd.grad(loss, params)
    h = 1e-4
    with torch.no_grad():
        for pi_, idx in ((0, (0,)), (1, (0, 1)), (2, (0,)), (3, (3, 4, 2))):
            if pi_ == 2 and not cx:
                continue
            p = params[pi_]
            old = p[idx].item()
            p[idx] = old + h
            lp = ref_loss(cfg, params, target, steps, sigma, cx).item()
            p[idx] = old - h
            lm = ref_loss(cfg, params, target, steps, sigma, cx).item()
            p[idx] = old
            fd = (lp - lm) / (2 * h)
            ad = grads[pi_][idx].item()
            assert abs(fd - ad) <= 1e-6 * max(abs(ad), 1e-3), (pi_, idx, fd, ad)


# ---------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def be(cuda_device):
    from lfm_b200 import B200Backend, _lib
    from lfm_b200.build import build_library

    build_library()
    _lib.set_step_path(_lib.PATH_AUTO)
    return B200Backend(cuda_device)


def random_state(N, cx, device, seed):
    g = torch.Generator().manual_seed(seed)
    r = lambda s: torch.randn(N, N, N, generator=g, dtype=torch.float64) * s  # noqa: E731
    pr, prp = r(1.0), r(1.0)
    pi, pip = (r(1.0), r(1.0)) if cx else (None, None)
    chi, chip = 19.0 + r(0.1), 19.0 + r(0.1)
    return [None if t is None else t.to(device) for t in (pr, prp, pi, pip, chi, chip)]


@pytest.mark.gpu
@pytest.mark.parametrize("level", ["real", "complex"])
def test_one_adjoint_step_is_the_float64_vjp(be, level):
    from lfm_b200.adjoint import _Lattice
    from lfm_b200.config import gravity_em, gravity_only
    from lfm_b200.mask import boundary_mask

    N = 16
    cx = level == "complex"
    cfg = (gravity_em if cx else gravity_only)(N, kappa=1.5 / 63.0)
    dev = be.device
    st = random_state(N, cx, dev, 1)
    cot = [None if t is None else t2 for t, t2 in zip(st, random_state(N, cx, dev, 2))]
    mask = torch.from_numpy(boundary_mask(N, cfg.boundary_fraction).reshape(N, N, N)).to(
        dev, torch.float64)
    inp = [None if t is None else t.clone().requires_grad_(True) for t in st]
    if cx:
        out = TR.step_complex(*inp, mask, cfg.dt**2, cfg.kappa, cfg.lambda_self, cfg.chi0,
                              cfg.e0_sq, cfg.epsilon_w)
    else:
        o = TR.step_real(inp[0], inp[1], inp[4], inp[5], mask, cfg.dt**2, cfg.kappa,
                         cfg.lambda_self, cfg.chi0, cfg.e0_sq)
        out = (o[0], o[1], None, None, o[2], o[3])
    pairs = [(o, c) for o, c in zip(out, cot) if o is not None]
    vjp = torch.autograd.grad([o for o, _ in pairs], [t for t in inp if t is not None],
                              [c for _, c in pairs])
    want = []
    it = iter(vjp)
    for t in inp:
        want.append(None if t is None else next(it))

    lat = _Lattice(cfg, be)
    f32 = lambda t: None if t is None else t.to(torch.float32).reshape(-1).contiguous()  # noqa: E731
    chi_next = f32(out[4].detach())
    g_out = [f32(c) for c in cot]
    g_in = [None if c is None else torch.empty_like(c) for c in g_out]
    lat.adjoint_step([f32(st[0]), f32(st[2]), f32(st[4])], [None, None, chi_next], g_out, g_in)
    torch.cuda.synchronize()
    for f, (got, w) in enumerate(zip(g_in, want)):
        if w is None:
            continue
        assert rel(got, w) < 2e-6, (f, rel(got, w))


def config5_like(N, cx):
    from lfm_b200.config import gravity_em, gravity_only

    return (gravity_em if cx else gravity_only)(N)


def ours_loss_and_grads(be, cfg, params, target, steps, sigma, cx, every=None):
    from lfm_b200.adjoint import leapfrog, soliton_state

    p32 = [p.detach().to(torch.float32).clone().requires_grad_(True) for p in params]
    st = soliton_state(cfg.grid_size, *p32[:3], sigma, cfg.chi0, p32[3], cx)
    out = leapfrog(cfg, st, steps, every=every, backend=be)
    loss = loss_of(out[4], out[0], target)
    grads = torch.autograd.grad(loss, p32)
    return loss.item(), grads


@pytest.mark.gpu
@pytest.mark.parametrize("level", ["real", "complex"])
def test_gradients_match_float64_autograd_and_differences(be, level):
    N, steps, sigma = 20, 40, 2.0
    cx = level == "complex"
    cfg = config5_like(N, cx)
    dev = be.device
    params = make_params(2, N, 6, dev, torch.float64)
    # a linear loss in (chi, psi_r): a squared distance to a target near chi
    # (chi ~ 19, deviations ~1e-3) would hand the adjoint a cotangent that the
    # float32 forward state only resolves to ~1e-3 relative
    target = linear_target(N, dev)
    ref_params = [p.clone().requires_grad_(True) for p in params]
    ref = ref_loss(cfg, ref_params, target, steps, sigma, cx)
    ref_grads = torch.autograd.grad(ref, ref_params)
    loss, grads = ours_loss_and_grads(be, cfg, params, target, steps, sigma, cx)
    # the loss sums +-19 w chi terms: compare against the size of the terms,
    # since the float32 forward itself carries ~1e-6 relative error per cell
    w, v = target
    terms = float((w.abs() * 19.0).sum() + (v.abs() * 8.0).sum())
    errs = {"loss": abs(loss - ref.item()) / terms}
    names = ("amplitude", "centre", "phase", "dchi")
    for name, g, r in zip(names, grads, ref_grads):
        if name == "phase" and not cx:
            continue
        errs[name] = rel(g, r)
    # central differences (h = 1e-3) of the float64 loss on the scalar parameters
    h = 1e-3
    with torch.no_grad():
        for pi_, idx in ((0, (0,)), (0, (1,)), (1, (0, 2)), (1, (1, 0)), (2, (1,))):
            if pi_ == 2 and not cx:
                continue
            pp = [p.clone() for p in params]
            pp[pi_][idx] += h
            lp = ref_loss(cfg, pp, target, steps, sigma, cx).item()
            pp[pi_][idx] -= 2 * h
            lm = ref_loss(cfg, pp, target, steps, sigma, cx).item()
            fd = (lp - lm) / (2 * h)
            scale = float(grads[pi_].abs().max())
            errs[f"fd{pi_}{idx}"] = abs(grads[pi_][idx].item() - fd) / scale
    print(level, "errors:", errs)
    assert errs.pop("loss") < 1e-6, errs
    assert max(errs.values()) < GRAD_RTOL, errs


@pytest.mark.gpu
def test_target_distance_loss_of_the_adjoint_workload(be):
    """The adjoint workload's own loss, |chi_T - chi_target|^2 with the target from a
    forward run at perturbed packet parameters (COMPLEX, gravity_em, two packets).

    Its cotangent 2 (chi_T - chi_target) is a difference of two values near 19, so the
    float32 forward's own chi error (~1e-6 absolute) moves it by a part in 10^2 - 10^3:
    that is a property of float32 storage, not of the adjoint.  The adjoint is
    therefore checked against the float64 VJP seeded with the same cotangent (within
    GRAD_RTOL); the gradient of the all-float64 loss is printed beside it."""
    from lfm_b200.adjoint import leapfrog, soliton_state

    N, steps, sigma = 20, 40, 2.0
    cfg = config5_like(N, True)
    dev = be.device
    params = make_params(2, N, 6, dev, torch.float64)
    amp, cen, ph, _ = params
    with torch.no_grad():
        st_t = soliton_state(N, (1.2 * amp).float(), (cen + 1.5).float(), (ph + 0.7).float(),
                             sigma, cfg.chi0, torch.zeros(N, N, N, device=dev), True)
        target = leapfrog(cfg, st_t, steps, backend=be)[4].double().clone()

    p32 = [p.detach().to(torch.float32).clone().requires_grad_(True) for p in params]
    st = soliton_state(N, *p32[:3], sigma, cfg.chi0, p32[3], True)
    out = leapfrog(cfg, st, steps, backend=be)
    loss = ((out[4].double() - target) ** 2).sum()
    grads = torch.autograd.grad(loss, p32)
    cot = (2.0 * (out[4].detach().double() - target)).reshape(N, N, N)
    assert float(cot.abs().max()) > 0.0

    ref_params = [p.clone().requires_grad_(True) for p in params]
    seeded = ref_loss(cfg, ref_params, (cot, torch.zeros_like(cot)), steps, sigma, True)
    want = torch.autograd.grad(seeded, ref_params)
    ref_params = [p.clone().requires_grad_(True) for p in params]
    full = ref_loss(cfg, ref_params, target.reshape(N, N, N), steps, sigma, True)
    want_full = torch.autograd.grad(full, ref_params)

    names = ("amplitude", "centre", "phase", "dchi")
    errs = {n: rel(g, w) for n, g, w in zip(names, grads, want)}
    errs_full = {n: rel(g, w) for n, g, w in zip(names, grads, want_full)}
    print("seeded float64 VJP:", errs, "| all-float64 loss:", errs_full,
          "| loss", loss.item(), "vs", full.item())
    assert max(errs.values()) < GRAD_RTOL, errs


@pytest.mark.gpu
def test_split_chi_forward_resolves_the_target_distance_loss(be):
    """The same loss with leapfrog(split_chi=True): chi runs as chi0 + hi + lo (about 48
    bits) and comes back in float64, so the gradient of the float32-state run's own loss
    matches the gradient of the all-float64 loss (which the float32 forward cannot)."""
    from lfm_b200.adjoint import leapfrog, soliton_state

    N, steps, sigma = 20, 40, 2.0
    cfg = config5_like(N, True)
    dev = be.device
    params = make_params(2, N, 6, dev, torch.float64)
    amp, cen, ph, _ = params
    from lfm_b200.mask import boundary_mask

    # the target: the float64 transcription from perturbed packet parameters
    with torch.no_grad():
        st_t = soliton_state(N, 1.2 * amp, cen + 1.5, ph + 0.7, sigma, cfg.chi0,
                             torch.zeros(N, N, N, device=dev, dtype=torch.float64), True,
                             device=dev, dtype=torch.float64)
        mask = torch.from_numpy(boundary_mask(N, cfg.boundary_fraction).reshape(N, N, N)).to(
            dev, torch.float64)
        s = {"pr": st_t[0], "prp": st_t[1], "pi": st_t[2], "pip": st_t[3], "chi": st_t[4],
             "chip": st_t[5]}
        target = TR.run(cfg, s, steps, mask)["chi"].reshape(N, N, N)

    p32 = [p.detach().to(torch.float32).clone().requires_grad_(True) for p in params[:3]]
    d64 = params[3].detach().clone().requires_grad_(True)
    st = soliton_state(N, *p32, sigma, cfg.chi0, None, True)
    st[4] = st[5] = cfg.chi0 + d64
    out = leapfrog(cfg, st, steps, backend=be, split_chi=True)
    assert out[4].dtype == torch.float64
    loss = ((out[4] - target) ** 2).sum()
    grads = torch.autograd.grad(loss, p32 + [d64])

    # the all-float64 loss from the same (float32-rounded) packet parameters
    fp = [p.detach().double().clone().requires_grad_(True) for p in p32] + [
        params[3].clone().requires_grad_(True)]
    full = ref_loss(cfg, fp, target, steps, sigma, True)
    want = torch.autograd.grad(full, fp)
    names = ("amplitude", "centre", "phase", "dchi")
    errs = {n: rel(g, w) for n, g, w in zip(names, grads, want)}
    print("split chi, all-float64 loss:", errs, "| loss", loss.item(), "vs", full.item())
    assert max(errs.values()) < GRAD_RTOL, errs


@pytest.mark.gpu
@pytest.mark.parametrize("level", ["real", "complex"])
def test_split_chi_checkpoint_interval_does_not_change_gradients(be, level):
    from lfm_b200.adjoint import leapfrog, soliton_state

    N, steps, sigma = 16, 24, 2.0
    cx = level == "complex"
    cfg = config5_like(N, cx)
    params = make_params(2, N, 7, be.device, torch.float64)
    runs = []
    for every in (1, 5, 24):
        p32 = [p.detach().float().clone().requires_grad_(True) for p in params[:3]]
        d64 = params[3].detach().clone().requires_grad_(True)
        st = soliton_state(N, *p32, sigma, cfg.chi0, None, cx)
        st[4] = st[5] = cfg.chi0 + d64
        out = leapfrog(cfg, st, steps, every=every, backend=be, split_chi=True)
        loss = ((out[4] - cfg.chi0) ** 2).sum()
        runs.append((loss.item(), torch.autograd.grad(loss, p32 + [d64])))
    for loss, grads in runs[1:]:
        assert loss == runs[0][0]
        for g, g0 in zip(grads, runs[0][1]):
            assert torch.equal(g, g0)


@pytest.mark.gpu
def test_checkpoint_interval_does_not_change_gradients(be):
    N, steps, sigma = 16, 24, 2.0
    cfg = config5_like(N, True)
    params = make_params(2, N, 7, be.device, torch.float64)
    target = torch.full((N, N, N), cfg.chi0, dtype=torch.float64, device=be.device)
    runs = [ours_loss_and_grads(be, cfg, params, target, steps, sigma, True, every=e)
            for e in (1, 5, 24)]
    for loss, grads in runs[1:]:
        assert loss == runs[0][0]
        for g, g0 in zip(grads, runs[0][1]):
            assert torch.equal(g, g0)


@pytest.mark.gpu
@pytest.mark.parametrize("level", ["real", "complex"])
def test_split_chi_forward_matches_split_evolver(be, level):
    """leapfrog(split_chi=True) steps as SplitChiEvolver does: the same bits of Psi and of
    chi's float64 value."""
    from lfm_b200.adjoint import leapfrog, soliton_state
    from lfm_b200.split import SplitChiEvolver

    N, steps = 16, 13
    cx = level == "complex"
    cfg = config5_like(N, cx)
    params = make_params(2, N, 8, be.device, torch.float64)
    st = soliton_state(N, *[p.float() for p in params[:3]], 2.0, cfg.chi0, None, cx)
    st[4] = st[5] = cfg.chi0 + params[3]
    out = leapfrog(cfg, st, steps, backend=be, split_chi=True)
    ev = SplitChiEvolver(cfg, backend=be)
    ev.set_psi_real(st[0])
    if cx:
        ev.set_psi_imag(st[2])
    ev.set_chi(st[4])
    ev.evolve(steps)
    assert torch.equal(out[0].cpu(), torch.from_numpy(ev.get_psi_real()))
    if cx:
        assert torch.equal(out[2].cpu(), torch.from_numpy(ev.get_psi_imag()))
    assert torch.equal(out[4].reshape(-1).cpu(), ev.chi64().cpu())


@pytest.mark.gpu
def test_leapfrog_forward_matches_evolver(be):
    from lfm_b200 import Evolver
    from lfm_b200.adjoint import leapfrog, soliton_state

    N, steps = 16, 13
    cfg = config5_like(N, True)
    params = make_params(2, N, 8, be.device, torch.float32)
    st = soliton_state(N, *params[:3], 2.0, cfg.chi0, params[3], True)
    out = leapfrog(cfg, st, steps, backend=be)
    ev = Evolver(cfg, backend=be)
    ev.set_psi_real(st[0])
    ev.set_psi_imag(st[2])
    ev.set_chi(st[4])
    ev.evolve(steps)
    assert torch.equal(out[0].cpu(), torch.from_numpy(ev.get_psi_real()))
    assert torch.equal(out[4].cpu(), torch.from_numpy(ev.get_chi()))
    assert torch.equal(out[1].cpu(), torch.from_numpy(ev.get_psi_real_prev()))
