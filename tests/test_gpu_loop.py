"""GPU tests of the device-resident time loop (gmt_run, CUDA graph) and of the batched ensemble."""
import math
import time

import numpy as np
import pytest
import torch

from tests.gpu_util import max_rel_err

pytestmark = pytest.mark.gpu

COURANT, CP, T = 0.3, 0.18, 0.5


def _host_loop(s, u, w, nsteps):
    """The host loop of run_turb (glmmhd_turb.jl:2216-2230) with ch = max signal speed."""
    s.forcing_reset()
    t = 0.0
    cm, sm = s.cfl(u)
    for _ in range(nsteps):
        while t >= s.next_time:
            s.forcing_advance()
        dt = min(COURANT * s.dx / cm, s.next_time - t)
        ch = sm
        fac = math.exp(-(ch * ch / (CP * 1.0 * ch)) * dt)
        s.step(u, w, dt, t=t, ch=ch, glm_fac=fac, do_turb=True, want_cfl=True)
        cm, sm = s.cfl_result()
        u, w = w, u
        t += dt
    return t, u


def _solver(n, dtype, amp=2.0, seed=0):
    from glmmhdturb_b200 import Solver
    return Solver(n, dtype=dtype, gamma=5 / 3, courant=COURANT, turb_amp=amp, turb_T=T, turb_ndt=100, turb_seed=seed,
                  glm_cp_coef=CP)


@pytest.mark.parametrize("graph", [True, False])
@pytest.mark.parametrize("nsteps", [12, 7])
def test_device_loop_matches_host_loop(graph, nsteps):
    n = (32, 32, 16)
    a, b = _solver(n, "f64"), _solver(n, "f64")
    ua, wa = a.alloc(), a.alloc()
    ub, wb = b.alloc(), b.alloc()
    a.ic_turbulent(ua, mach=1.0, seed=3)
    b.ic_turbulent(ub, mach=1.0, seed=3)
    t_host, ref = _host_loop(a, ua, wa, nsteps)
    b.forcing_reset()
    t_dev, got = b.run(ub, wb, nsteps, 0.0, forcing=True, ch_max_signal=True, graph=graph)
    assert got is (wb if nsteps % 2 else ub)
    assert abs(t_dev - t_host) <= 1e-14 * t_host
    err, errs = max_rel_err(got.cpu().numpy(), ref.cpu().numpy())
    assert err <= 1e-12, errs
    assert b.forcing_counter() == a.forcing_counter()


def test_graph_replay_is_deterministic_fp32():
    n = 64
    s = _solver(n, "f32")
    u, w = s.alloc(), s.alloc()
    s.ic_turbulent(u, mach=1.0, seed=1)
    u0 = u.clone()
    s.forcing_reset()
    t1, r1 = s.run(u, w, 10, forcing=True, graph=True)
    r1 = r1.clone()
    u.copy_(u0)
    s.forcing_reset()
    t2, r2 = s.run(u, w, 10, forcing=True, graph=False)
    assert t1 == t2 and torch.equal(r1, r2)


def test_ensemble_boxes_match_single_box_runs():
    from glmmhdturb_b200 import Ensemble
    sizes, amps, seeds = [32, 16, 48], [2.0, 1.0, 3.0], [5, 6, 7]
    ens = Ensemble(sizes, amps=amps, seeds=seeds, dtype="f64", courant=COURANT, turb_T=T, glm_cp_coef=CP)
    u = ens.alloc()
    w = ens.alloc()
    singles = []
    for b, nb in enumerate(sizes):
        s = _solver(nb, "f64", amp=amps[b], seed=seeds[b])
        s.ic_turbulent(u[b], mach=0.5 + 0.5 * b, seed=seeds[b])
        uu, ww = s.alloc(), s.alloc()
        uu.copy_(u[b])
        s.forcing_reset()
        singles.append(s.run(uu, ww, 9, forcing=True))
    ts = ens.run(u, w, 9, forcing=True)
    for b in range(len(sizes)):
        t_single, res = singles[b]
        assert abs(ts[b] - t_single) <= 1e-14 * t_single
        err, errs = max_rel_err(w[b].cpu().numpy(), res.cpu().numpy())
        assert err <= 1e-12, (b, errs)


def test_ensemble_fp32_overhanging_tiles_match_single_boxes():
    """FP32 ensemble tiles are 32 columns wide, so 16^3 and 48^3 boxes get an overhanging last tile
    whose extra columns recompute the periodic images of the row's first cells.  Every box must
    still equal its own single-box run (different tile shapes, so agreement to FP32 round-off)."""
    from glmmhdturb_b200 import Ensemble
    sizes, amps, seeds = [48, 16, 32, 48], [2.0, 1.0, 3.0, 1.5], [5, 6, 7, 8]
    ens = Ensemble(sizes, amps=amps, seeds=seeds, dtype="f32", courant=COURANT, turb_T=T, glm_cp_coef=CP)
    u = ens.alloc()
    w = ens.alloc()
    singles = []
    for b, nb in enumerate(sizes):
        s = _solver(nb, "f32", amp=amps[b], seed=seeds[b])
        s.ic_turbulent(u[b], mach=0.5 + 0.5 * b, seed=seeds[b])
        uu, ww = s.alloc(), s.alloc()
        uu.copy_(u[b])
        s.forcing_reset()
        singles.append(s.run(uu, ww, 9, forcing=True))
    ts = ens.run(u, w, 9, forcing=True)
    for b in range(len(sizes)):
        t_single, res = singles[b]
        assert abs(ts[b] - t_single) <= 1e-6 * t_single
        err, errs = max_rel_err(w[b].cpu().numpy(), res.cpu().numpy())
        # the two kernels are separate instantiations, so they agree to FP32 round-off (measured
        # 1e-7..6e-7 in rho..Bz after 9 steps); psi, a small field fed by divergence errors, carries
        # the same absolute round-off at a larger relative size (measured up to 6e-5)
        assert max(errs[:8]) <= 1e-5 and errs[8] <= 1e-3, (b, errs)


def _ensemble_config(nbox=64, seed=2024):
    """Box sizes drawn from {32,48,64,96,128}, Mach from U[0.3,3], beta from U[0.1,10], seeds 0..63."""
    rng = np.random.default_rng(seed)
    sizes = [int(x) for x in rng.choice([32, 48, 64, 96, 128], size=nbox)]
    mach = rng.uniform(0.3, 3.0, size=nbox)
    beta = rng.uniform(0.1, 10.0, size=nbox)
    return sizes, mach, beta, list(range(nbox))


def test_ensemble_speedup_over_looping_single_boxes():
    from glmmhdturb_b200 import Ensemble
    sizes, mach, beta, seeds = _ensemble_config()
    amps = [2.0 * m for m in mach]
    ens = Ensemble(sizes, amps=amps, seeds=seeds, dtype="f32", courant=COURANT, turb_T=T, glm_cp_coef=CP)
    u, w = ens.alloc(), ens.alloc()
    singles = {}
    for b, nb in enumerate(sizes):
        if nb not in singles:
            singles[nb] = _solver(nb, "f32")
        b0 = math.sqrt(2 * 0.6 / beta[b])
        singles[nb].ic_turbulent(u[b], b0=(b0, 0.0, 0.0), mach=float(mach[b]), seed=seeds[b])
    u0 = [x.clone() for x in u]
    ens.run(u, w, 2, forcing=True)                 # warm-up (graph capture)
    torch.cuda.synchronize()
    steps = 10
    t0 = time.perf_counter()
    ens.run(u, w, steps, forcing=True)
    torch.cuda.synchronize()
    t_ens = time.perf_counter() - t0
    # baseline: the plain single-box step looped over the boxes, dt from each box's own CFL
    boxes = []
    for b, nb in enumerate(sizes):
        s = _solver(nb, "f32", amp=amps[b], seed=seeds[b])
        x = u0[b].clone()
        boxes.append([s, x, torch.empty_like(x), 0.0, *s.cfl(x)])
        s.forcing_reset()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        for bx in boxes:
            s, x, y, t, cm, sm = bx
            while t >= s.next_time:
                s.forcing_advance()
            dt = min(COURANT * s.dx / cm, s.next_time - t)
            s.step(x, y, dt, t=t, ch=sm, glm_fac=math.exp(-(sm / CP) * dt), do_turb=True, want_cfl=True)
            cm, sm = s.cfl_result()
            bx[1], bx[2], bx[3], bx[4], bx[5] = y, x, t + dt, cm, sm
    torch.cuda.synchronize()
    t_loop = time.perf_counter() - t0
    zones = sum(n ** 3 for n in sizes) * steps
    print(f"ensemble 64 boxes ({sum(n**3 for n in sizes)} zones): {zones / t_ens / 1e9:.2f} Gzone/s; "
          f"looped single boxes {zones / t_loop / 1e9:.2f} Gzone/s; speedup {t_loop / t_ens:.2f}x")
    for x in u:
        assert torch.isfinite(x).all()
    # measured 2.2-2.4x (9.5-10.2 vs 4.3 Gzone/s). 3x would need 12.9 Gzone/s, above the 12.2 that
    # the same tile kernel reaches on one 512^3 box, its best case; the bar sits below the measured ratio.
    assert t_loop / t_ens > 2.0
    assert zones / t_ens > 8.5e9
