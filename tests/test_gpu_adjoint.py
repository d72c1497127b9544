"""GPU tests of the discrete adjoint (gmt_adjoint_step), the band-limited KE loss gradient and the
checkpointed gradient driver.

Checks, in FP64: the adjoint of one step against forward-mode tangents of the oracle's CPU step
along 8 random directions (<w, J v> = <J^T w, v>, the ForwardDiff check); gradients of the KE shell
power with respect to the forcing amplitude and to an initial velocity/B perturbation against
central finite differences (eps = 1e-6) with dt frozen; independence of the checkpoint interval;
the autograd wrapper; and the FP32 gradient against the FP64 one.
"""
import math

import numpy as np
import pytest
import torch

from tests.gpu_util import perturbed_glm_state, to_dev

pytestmark = pytest.mark.gpu

GAMMA = 5.0 / 3.0
FD_TOL = 1e-4          # gradient vs central finite differences (relative)
DOT_TOL = 1e-11        # adjoint vs forward-mode tangents, relative to sum |w_i (J v)_i|


def _solver(n, dtype="f64", **kw):
    from glmmhdturb_b200 import Solver
    args = dict(dtype=dtype, gamma=GAMMA, turb_amp=2.0, turb_T=0.5, turb_ndt=100, turb_seed=0, courant=0.3)
    args.update(kw)
    return Solver(n, **args)


def _rel(a, b):
    return abs(a - b) / max(abs(a), abs(b), 1e-300)


def test_band_loss_matches_spectrum_and_fd():
    from glmmhdturb_b200 import adjoint as AD
    n = 16
    s = _solver(n)
    u = s.alloc()
    s.ic_turbulent(u, mach=1.0, seed=5)
    E = s.ke_spectrum(u, kmax=7)
    L, g = s.ke_band_loss(u, 2, 5)
    assert _rel(L, E[2:6].sum()) <= 1e-12
    assert torch.all(g[4:] == 0)
    gen = torch.Generator(device="cuda").manual_seed(3)
    d = torch.randn(u.shape, generator=gen, device="cuda", dtype=torch.float64)
    d[0] = 0.05 * d[0].abs() * u[0]
    d[4:] = 0
    eps = 1e-6
    lp, _ = s.ke_band_loss(u + eps * d, 2, 5)
    lm, _ = s.ke_band_loss(u - eps * d, 2, 5)
    fd = (lp - lm) / (2 * eps)
    assert _rel(AD.dot(g, d), fd) <= 1e-7, (AD.dot(g, d), fd)


@pytest.mark.parametrize("recon,riemann", [("mc", "hlld"), ("mc", "hll"), ("minmod", "hlld"), ("mc", "llf")])
def test_one_step_adjoint_vs_oracle_forward_mode(oracle, recon, riemann):
    """<w, J v> from forward-mode tangents of the oracle's FP64 step (the ForwardDiff check) along
    8 random directions, and along the forcing amplitude, equals <J^T w, v> from the GPU adjoint
    (forcing kick and psi damping included)."""
    n = 16
    u0 = perturbed_glm_state(oracle, (n, n, n), seed=11, gamma=GAMMA)
    u0[5:7] += 0.03 * np.random.default_rng(5).standard_normal(u0[5:7].shape)
    cfg = oracle.Config(n=(n, n, n), gamma=GAMMA, recon=recon, riemann=riemann, iflo=True)
    s = _solver(n, recon=recon, riemann=riemann)
    s.forcing_reset()
    s.forcing_advance()
    modes = s.get_modes()
    cmax, smax = oracle.cfl(cfg, u0)
    dt = 0.3 * cfg.dx / cmax
    ch = smax
    fac = math.exp(-(ch / 0.18) * dt)
    t = 0.2
    rng = np.random.default_rng(7)
    w = rng.standard_normal(u0.shape)
    gin = torch.empty_like(to_dev(u0))
    s.set_modes(modes)
    s.adjoint_step(to_dev(u0), to_dev(w), gin, dt, t=t, ch=ch, glm_fac=fac, do_turb=True)
    jtw = gin.cpu().numpy()
    amp_part = s.adjoint_amp_grad(reset=True)
    v = rng.standard_normal((8,) + u0.shape) * np.abs(u0).max(axis=(1, 2, 3), keepdims=True)
    _, jv = oracle.jvp_unsplit(cfg, u0, v, dt, ch, fac, ramp=min(t / 0.5, 1.0), modes=modes)
    for k in range(8):
        lhs = float((w * jv[k]).sum())
        rhs = float((jtw * v[k]).sum())
        assert abs(lhs - rhs) <= DOT_TOL * float(np.abs(w * jv[k]).sum()), (k, lhs, rhs)
    # the amplitude partial of one step (relative tangent 1 -> divide by the amplitude)
    _, ja = oracle.jvp_unsplit(cfg, u0, None, dt, ch, fac, ramp=min(t / 0.5, 1.0), modes=modes, amp_rel=1.0)
    fwd_amp = float((w * ja).sum()) / 2.0
    assert abs(amp_part - fwd_amp) <= DOT_TOL * float(np.abs(w * ja).sum()) / 2.0, (amp_part, fwd_amp)


def _scaled(sched, f):
    import copy
    s2 = copy.copy(sched)
    s2.modes = [m * f for m in sched.modes]
    return s2


def _forced_base(n, seed=0, sigma=1e-3, dtype="f64"):
    """The 64^3 parity run's kind of state: uniform (rho 1, p 0.6, B (0.775,0,0)) plus a seeded Gaussian
    perturbation (sigma) of v and B; returns (solver, u0, direction of the perturbation)."""
    from glmmhdturb_b200 import adjoint as AD
    s = _solver(n, dtype=dtype)
    u = s.alloc()
    s.ic_uniform(u, 1.0, 0.6, (0.775, 0.0, 0.0))
    tdt = torch.float64 if dtype == "f64" else torch.float32
    gen = torch.Generator(device="cuda").manual_seed(seed)
    gv = sigma * torch.randn((3, n, n, n), generator=gen, device="cuda", dtype=torch.float64).to(tdt)
    gb = sigma * torch.randn((3, n, n, n), generator=gen, device="cuda", dtype=torch.float64).to(tdt)
    # u0 = the perturbed state: primitives perturbed, then converted
    rho = u[0].clone()
    u0 = u.clone()
    u0[1:4] = rho * gv
    u0[5:8] = u[5:8] + gb
    u0[4] = 0.6 / (GAMMA - 1) + 0.5 * (u0[1:4] ** 2).sum(0) / rho + 0.5 * (u0[5:8] ** 2).sum(0)
    d = AD.velocity_b_direction(u0, gv, gb)
    return s, u0, d


def test_gradient_amp_and_initial_fields_vs_fd():
    """16^3 FP64, 12 forced steps, loss = KE shell power 2 <= |k| <= 4, checkpoints every 4."""
    from glmmhdturb_b200 import adjoint as AD
    n, nsteps = 16, 12
    s, u0, d = _forced_base(n, seed=1)
    r = AD.ke_band_gradient(s, u0, nsteps, kmin=2, kmax=4, checkpoint_every=4)
    sched = r["schedule"]
    L0 = r["loss"]
    assert L0 > 0 and math.isfinite(r["grad_amp"])

    def loss_of(u_init, sch):
        uN = AD.replay(s, u_init, sch)
        return s.ke_band_loss(uN, 2, 4)[0]

    assert _rel(loss_of(u0, sched), L0) == 0.0   # replay is bit-identical to the forward
    ea = 1e-6
    fd_amp = (loss_of(u0, _scaled(sched, 1 + ea)) - loss_of(u0, _scaled(sched, 1 - ea))) / (2 * ea * 2.0)
    assert _rel(r["grad_amp"], fd_amp) <= FD_TOL, (r["grad_amp"], fd_amp)
    eu = 1e-6
    fd_u = (loss_of(u0 + eu * d, sched) - loss_of(u0 - eu * d, sched)) / (2 * eu)
    ad_u = AD.dot(r["grad_u0"], d)
    assert _rel(ad_u, fd_u) <= FD_TOL, (ad_u, fd_u)

    # a random direction in all nine fields, from a generic state (rho, p and psi of the uniform
    # state are constant along every axis, a kink of the limiter; 4 forced steps make them vary)
    ug, _, _ = AD.forward(s, u0, 4)
    r2 = AD.ke_band_gradient(s, ug, 8, kmin=2, kmax=4, checkpoint_every=3)
    gen = torch.Generator(device="cuda").manual_seed(9)
    v = 1e-3 * torch.randn(u0.shape, generator=gen, device="cuda", dtype=torch.float64)
    v[8] *= 0.1
    sch2 = r2["schedule"]
    fd_v = (loss_of(ug + eu * v, sch2) - loss_of(ug - eu * v, sch2)) / (2 * eu)
    assert _rel(AD.dot(r2["grad_u0"], v), fd_v) <= FD_TOL, (AD.dot(r2["grad_u0"], v), fd_v)


def test_checkpoint_interval_does_not_change_the_gradient():
    from glmmhdturb_b200 import adjoint as AD
    n, nsteps = 16, 9
    s, u0, _ = _forced_base(n, seed=2)
    ref = None
    for K in (1, 3, 4, 9):
        r = AD.ke_band_gradient(s, u0, nsteps, kmin=2, kmax=4, checkpoint_every=K)
        if ref is None:
            ref = r
            continue
        assert torch.equal(r["grad_u0"], ref["grad_u0"]) and r["loss"] == ref["loss"]
        assert _rel(r["grad_amp"], ref["grad_amp"]) <= 1e-13
    assert AD.checkpoint_interval(200, 75 << 20, 40 << 30) >= 1
    assert AD.checkpoint_interval(100, 1) == 10


def test_step_function_autograd_matches_adjoint():
    from glmmhdturb_b200 import adjoint as AD
    n = 16
    s, u0, _ = _forced_base(n, seed=3)
    s.forcing_reset()
    s.forcing_advance()
    dt, t = 2e-3, 0.1
    ch, fac = s.cfl(u0)[1], 0.99
    x = u0.clone().requires_grad_(True)
    y1 = AD.StepFunction.apply(x, s, dt, t, ch, fac, True)
    y2 = AD.StepFunction.apply(y1, s, dt, t + dt, ch, fac, True)
    gen = torch.Generator(device="cuda").manual_seed(4)
    w = torch.randn(u0.shape, generator=gen, device="cuda", dtype=torch.float64)
    (y2 * w).sum().backward()
    # the same chain by hand
    u1 = torch.empty_like(u0)
    s.step(u0, u1, dt, t=t, ch=ch, glm_fac=fac, do_turb=True)
    g1 = torch.empty_like(u0)
    g0 = torch.empty_like(u0)
    s.adjoint_step(u1, w, g1, dt, t=t + dt, ch=ch, glm_fac=fac, do_turb=True)
    s.adjoint_step(u0, g1, g0, dt, t=t, ch=ch, glm_fac=fac, do_turb=True)
    assert torch.equal(x.grad, g0)


def test_fp32_gradient_tracks_fp64():
    from glmmhdturb_b200 import adjoint as AD
    n, nsteps = 16, 8
    out = {}
    for dt_ in ("f64", "f32"):
        s, u0, d = _forced_base(n, seed=4, dtype=dt_)
        r = AD.ke_band_gradient(s, u0, nsteps, kmin=2, kmax=4, checkpoint_every=4)
        out[dt_] = (r["grad_amp"], r["grad_u0"].double().cpu(), d.double().cpu())
    ga64, g64, d64 = out["f64"]
    ga32, g32, _ = out["f32"]
    rel = float((g32 - g64).norm() / g64.norm())
    print("FP32 vs FP64 gradient: amplitude %.2e, initial state (relative L2) %.2e" % (_rel(ga32, ga64), rel))
    assert _rel(ga32, ga64) <= 1e-2, (ga32, ga64)
    assert rel <= 1e-2, rel   # measured 2.6e-3 (8 steps, 16^3, loss ~1e-8)


def test_adjoint_rejects_ppm_and_aliasing():
    from glmmhdturb_b200 import GmtError
    s = _solver(16, recon="ppm", riemann="hll")
    u = s.alloc()
    s.ic_uniform(u)
    g = torch.zeros_like(u)
    with pytest.raises(GmtError):
        s.adjoint_step(u, g, torch.empty_like(u), 1e-3, ch=1.0, glm_fac=1.0)
    s2 = _solver(16)
    u2 = s2.alloc()
    s2.ic_uniform(u2)
    g2 = torch.zeros_like(u2)
    with pytest.raises(GmtError):
        s2.adjoint_step(u2, g2, g2, 1e-3, ch=1.0, glm_fac=1.0)


def test_adjoint_64cube_50_steps_fp64():
    """The differentiable-run configuration: 64^3, 50 forced steps with dt frozen, loss = KE shell
    power 4 <= |k| <= 8 at the last step, checkpoints every 10; gradients with respect to the OU
    amplitude and the seeded (sigma = 1e-3) initial velocity/B perturbation vs central differences."""
    from glmmhdturb_b200 import adjoint as AD
    n, nsteps = 64, 50
    s, u0, d = _forced_base(n, seed=0)
    r = AD.ke_band_gradient(s, u0, nsteps, kmin=4, kmax=8, checkpoint_every=10)
    sched = r["schedule"]

    def loss_of(u_init, sch):
        return s.ke_band_loss(AD.replay(s, u_init, sch), 4, 8)[0]

    ea = 1e-6
    fd_amp = (loss_of(u0, _scaled(sched, 1 + ea)) - loss_of(u0, _scaled(sched, 1 - ea))) / (2 * ea * 2.0)
    eu = 1e-6
    fd_u = (loss_of(u0 + eu * d, sched) - loss_of(u0 - eu * d, sched)) / (2 * eu)
    ad_u = AD.dot(r["grad_u0"], d)
    print("64^3 x 50 adjoint: loss %.6e  dL/damp adjoint %.10e fd %.10e  dL/dalpha adjoint %.10e fd %.10e"
          % (r["loss"], r["grad_amp"], fd_amp, ad_u, fd_u))
    assert _rel(r["grad_amp"], fd_amp) <= FD_TOL
    assert _rel(ad_u, fd_u) <= FD_TOL


def test_adjoint_64cube_forward_mode_directions_fp64(oracle):
    """The 64^3 x 50-step gradient against the oracle's forward-mode directional derivatives over all 50
    steps along 7 random state directions (all nine fields) and the forcing amplitude."""
    from glmmhdturb_b200 import adjoint as AD
    n, nsteps = 64, 50
    s, u0, _ = _forced_base(n, seed=0)
    r = AD.ke_band_gradient(s, u0, nsteps, kmin=4, kmax=8, checkpoint_every=10)
    sched = r["schedule"]
    _, gN = s.ke_band_loss(r["u_final"], 4, 8)
    gN = gN.cpu().numpy()
    g0 = r["grad_u0"].cpu().numpy()
    cfg = oracle.Config(n=(n, n, n), gamma=GAMMA, recon="mc", riemann="hlld", iflo=True)
    rng = np.random.default_rng(21)
    u = u0.cpu().numpy()
    scale = np.abs(u).max(axis=(1, 2, 3), keepdims=True) + 1e-3
    dirs = np.zeros((8,) + u.shape)
    dirs[:7] = 1e-3 * rng.standard_normal((7,) + u.shape) * scale
    rel = np.zeros(8)
    rel[7] = 1.0
    du = dirs.copy()
    for rec in sched.steps:
        u, du = oracle.jvp_unsplit(cfg, u, du, rec.dt, rec.ch, rec.glm_fac, ramp=min(rec.t / 0.5, 1.0),
                                   modes=sched.modes[rec.modes], amp_rel=rel)
    np.testing.assert_array_equal(u, r["u_final"].cpu().numpy())   # FP64 GPU forward == oracle
    for k in range(7):
        fwd = float((gN * du[k]).sum())
        adj = float((g0 * dirs[k]).sum())
        assert _rel(fwd, adj) <= 1e-8, (k, fwd, adj)
    fwd_amp = float((gN * du[7]).sum()) / 2.0
    assert _rel(fwd_amp, r["grad_amp"]) <= 1e-8, (fwd_amp, r["grad_amp"])


def test_adjoint_128cube_200_steps_in_40gb():
    """The large adjoint: 128^3 FP32, 200 forced steps, checkpoint interval from a 40 GB budget
    with recomputation; finite gradients, device memory within the budget."""
    import time
    from glmmhdturb_b200 import adjoint as AD
    n, nsteps, budget = 128, 200, 40 << 30
    s, u0, d = _forced_base(n, seed=2, dtype="f32")
    state_bytes = u0.numel() * u0.element_size()
    K = AD.checkpoint_interval(nsteps, state_bytes, budget)
    free0, total = torch.cuda.mem_get_info()
    torch.cuda.reset_peak_memory_stats()
    t0 = time.perf_counter()
    r = AD.ke_band_gradient(s, u0, nsteps, kmin=4, kmax=8, checkpoint_every=K)
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    peak = torch.cuda.max_memory_allocated() + AD.adjoint_scratch_bytes(s)
    print(f"adjoint 128^3 x {nsteps}: K={K}, {elapsed:.2f} s forward+backward, "
          f"peak {peak / 2**30:.2f} GB (torch tensors + adjoint scratch), dL/damp {r['grad_amp']:.4e}")
    assert math.isfinite(r["grad_amp"]) and bool(torch.isfinite(r["grad_u0"]).all())
    assert peak <= budget


@pytest.mark.parametrize("recon,riemann", [("mc", "hlld"), ("mc", "hll"), ("minmod", "hlld"), ("minmod", "hll")])
def test_fp32_record_tile_matches_per_cell_passes(recon, riemann):
    """The FP32 adjoint's record tile (passes 1-3 as the forward step's tile march: the 32x16
    compile-time tile, interior tiles staged by TMA at 128x128x16) against the same three passes run
    per cell, with the forcing kick on: ubar and dL/d(amplitude) agree to FP32 round-off."""
    n = (128, 128, 16)
    s = _solver(n, dtype="f32", recon=recon, riemann=riemann)
    s.forcing_advance()
    s.forcing_advance()
    u = s.alloc()
    s.ic_turbulent(u, 1.0, 0.6, (0.775, 0.0, 0.0), mach=1.0, db=0.2, seed=7)
    assert s.kernel_info()["tile"][:2] == (32, 16)
    gen = torch.Generator(device="cuda").manual_seed(11)
    ubn = torch.randn(u.shape, generator=gen, device="cuda", dtype=torch.float32)
    cm, sm = s.cfl(u)
    dt = 0.3 * s.dx / cm
    out = {}
    for percell in (False, True):
        s.adjoint_set_passes(percell)
        ub = torch.empty_like(u)
        s.adjoint_step(u, ubn, ub, dt, t=0.2, ch=sm, do_turb=True)
        out[percell] = (ub.double().cpu().numpy(), s.adjoint_amp_grad(reset=True))
    s.adjoint_set_passes(False)
    (a, ga), (b, gb) = out[False], out[True]
    assert np.isfinite(a).all() and np.isfinite(b).all()
    l2 = [float(np.linalg.norm(a[v] - b[v]) / max(np.linalg.norm(b[v]), 1e-300)) for v in range(9)]
    mx = [float(np.abs(a[v] - b[v]).max() / max(np.abs(b[v]).max(), 1e-300)) for v in range(9)]
    print(f"{recon}/{riemann}: record vs per-cell L2 {max(l2):.2e}, max {max(mx):.2e}, amp {ga:.6e} vs {gb:.6e}")
    # L2 to FP32 round-off; pointwise, a limiter or fan-region switch that flips on a one-ulp
    # difference of a face state leaves a larger local difference
    assert max(l2) <= 1e-5 and max(mx) <= 1e-3, (l2, mx)
    assert _rel(ga, gb) <= 1e-4, (ga, gb)
