"""Gradients through many unsplit GLM steps: the discrete adjoint of gmt_step with dt frozen, and
checkpointing with recomputation.

Forward: the reference driver's host loop (the OU update whenever t reaches the next update time,
glmmhd_turb.jl:2075-2161; dt = courant*dx/max sum_d(|v_d|+c_f), glmmhd_turb.jl:1963-1978, clamped to
the next forcing update; ch and glm_fac as in glmmhd_turb.jl:582-583 with ch = the global max fast
signal speed).  Each step's dt, t, ch, glm_fac and the forcing modes it used are recorded in a
Schedule, and the state is kept every K steps.  Backward: every segment is recomputed from its
checkpoint with the recorded schedule (so it reproduces the forward bit for bit), then
gmt_adjoint_step runs over it in reverse.  Device memory: ceil(N/K) checkpoints + K segment states +
two adjoint registers + the adjoint scratch of the context (207 state planes).

The reference has no adjoint; StepFunction is the Python counterpart of a ChainRulesCore rrule on the
step function (its backward is gmt_adjoint_step).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import torch

from .solver import Solver


@dataclass
class StepRecord:
    dt: float
    t: float
    ch: float
    glm_fac: float
    modes: int            # index into Schedule.modes (-1: no forcing)


@dataclass
class Schedule:
    steps: list = field(default_factory=list)
    modes: list = field(default_factory=list)   # (61, 3, 2) FP64 arrays, one per OU update
    forcing: bool = True

    def __len__(self):
        return len(self.steps)


def checkpoint_interval(nsteps: int, state_bytes: int, budget_bytes: int | None = None) -> int:
    """K minimising the checkpoint + segment memory ceil(N/K) + K states (about sqrt(N)), or the
    largest K whose total, with the adjoint registers and scratch, fits `budget_bytes`."""
    k_opt = max(1, int(round(math.sqrt(nsteps))))
    if budget_bytes is None:
        return k_opt
    fixed = (2 + 207 / 9) * state_bytes
    best = None
    for k in range(1, nsteps + 1):
        need = (math.ceil(nsteps / k) + k) * state_bytes + fixed
        if need <= budget_bytes and (best is None or need < best[1]):
            best = (k, need)
    if best is None:
        raise ValueError("the budget holds fewer than two states beside the adjoint scratch")
    return best[0]


def forward(solver: Solver, u0: torch.Tensor, nsteps: int, *, forcing: bool = True, checkpoint_every: int = 10,
            courant: float | None = None, t0: float = 0.0):
    """Run `nsteps` host-loop steps from u0 (u0 is not modified); returns (u_final, schedule,
    checkpoints) with checkpoints[i] = the state before step i for i = 0, K, 2K, ..."""
    courant = solver.params.courant if courant is None else courant
    sched = Schedule(forcing=forcing)
    ckpt = {}
    u = u0.clone()
    w = torch.empty_like(u)
    t = t0
    if forcing:
        solver.forcing_reset()
    for i in range(nsteps):
        if forcing:
            while t >= solver.next_time:
                solver.forcing_advance()
                sched.modes.append(solver.get_modes())
        if i % checkpoint_every == 0:
            ckpt[i] = u.clone()
        cmax, smax = solver.cfl(u)
        dt = courant * solver.dx / cmax
        if forcing:
            dt = min(dt, solver.next_time - t)
        ch = smax
        fac = solver.glm_fac(ch, dt)
        sched.steps.append(StepRecord(dt, t, ch, fac, len(sched.modes) - 1 if forcing else -1))
        solver.step(u, w, dt, t=t, ch=ch, glm_fac=fac, do_turb=forcing)
        u, w = w, u
        t += dt
    return u, sched, ckpt


def _apply_modes(solver: Solver, sched: Schedule, rec: StepRecord, current: list):
    if rec.modes >= 0 and current[0] != rec.modes:
        solver.set_modes(sched.modes[rec.modes])
        current[0] = rec.modes


def replay(solver: Solver, u0: torch.Tensor, sched: Schedule, start: int = 0, stop: int | None = None,
           keep: bool = False):
    """Re-run steps start..stop-1 of a recorded schedule from u0 (the state before step `start`).
    Returns the final state, and with keep=True the list of the states before each step."""
    stop = len(sched) if stop is None else stop
    u = u0.clone()
    w = torch.empty_like(u)
    states = []
    cur = [None]
    for i in range(start, stop):
        rec = sched.steps[i]
        _apply_modes(solver, sched, rec, cur)
        if keep:
            states.append(u.clone())
        solver.step(u, w, rec.dt, t=rec.t, ch=rec.ch, glm_fac=rec.glm_fac, do_turb=rec.modes >= 0)
        u, w = w, u
    return (u, states) if keep else u


def backward(solver: Solver, sched: Schedule, ckpt: dict, ubar_final: torch.Tensor):
    """dL/du0 and dL/d(turb_amp) from dL/du_N through the recorded steps (dt, ch, glm_fac frozen)."""
    solver.adjoint_amp_grad(reset=True)
    ubar = ubar_final.clone()
    tmp = torch.empty_like(ubar)
    starts = sorted(ckpt)
    n = len(sched)
    for si in range(len(starts) - 1, -1, -1):
        a = starts[si]
        b = starts[si + 1] if si + 1 < len(starts) else n
        _, states = replay(solver, ckpt[a], sched, a, b, keep=True)
        cur = [None]
        for i in range(b - 1, a - 1, -1):
            rec = sched.steps[i]
            _apply_modes(solver, sched, rec, cur)
            solver.adjoint_step(states[i - a], ubar, tmp, rec.dt, t=rec.t, ch=rec.ch, glm_fac=rec.glm_fac,
                                do_turb=rec.modes >= 0)
            ubar, tmp = tmp, ubar
        del states
    return ubar, solver.adjoint_amp_grad(reset=True)


def ke_band_gradient(solver: Solver, u0: torch.Tensor, nsteps: int, *, kmin: int = 4, kmax: int = 8,
                     checkpoint_every: int = 10, forcing: bool = True):
    """Loss L = KE shell power for kmin <= |k| <= kmax after nsteps; returns a dict with the loss,
    dL/du0 (a state-shaped tensor), dL/d(turb_amp), the final state and the schedule."""
    uN, sched, ckpt = forward(solver, u0, nsteps, forcing=forcing, checkpoint_every=checkpoint_every)
    loss, gN = solver.ke_band_loss(uN, kmin, kmax)
    g0, damp = backward(solver, sched, ckpt, gN)
    return {"loss": loss, "grad_u0": g0, "grad_amp": damp, "u_final": uN, "schedule": sched}


def velocity_b_direction(u0: torch.Tensor, g_v: torch.Tensor, g_b: torch.Tensor) -> torch.Tensor:
    """du0/dalpha for the primitive perturbation v += alpha g_v, B += alpha g_B at fixed rho and p:
    dm = rho g_v, dB = g_B, dE = m.g_v + B.g_B (g_v, g_b: (3, nz, ny, nx))."""
    d = torch.zeros_like(u0)
    rho = u0[0]
    d[1:4] = rho * g_v
    d[5:8] = g_b
    d[4] = (u0[1:4] * g_v).sum(0) + (u0[5:8] * g_b).sum(0)
    return d


class StepFunction(torch.autograd.Function):
    """u' = step(u) with a backward through gmt_adjoint_step (dt, ch, glm_fac frozen).  The forcing
    amplitude's gradient goes to the solver's accumulator (Solver.adjoint_amp_grad)."""

    @staticmethod
    def forward(ctx, u, solver, dt, t, ch, glm_fac, do_turb):
        out = torch.empty_like(u)
        solver.step(u, out, dt, t=t, ch=ch, glm_fac=glm_fac, do_turb=do_turb)
        ctx.save_for_backward(u)
        ctx.args = (solver, dt, t, ch, glm_fac, do_turb)
        return out

    @staticmethod
    def backward(ctx, gout):
        (u,) = ctx.saved_tensors
        solver, dt, t, ch, glm_fac, do_turb = ctx.args
        gin = torch.empty_like(u)
        solver.adjoint_step(u, gout.contiguous(), gin, dt, t=t, ch=ch, glm_fac=glm_fac, do_turb=do_turb)
        return gin, None, None, None, None, None, None


def adjoint_scratch_bytes(solver: Solver) -> int:
    """Device bytes the context's adjoint scratch holds (207 state planes)."""
    return 207 * solver.n * (8 if solver.dtype_name == "f64" else 4)


def dot(a: torch.Tensor, b: torch.Tensor) -> float:
    return float((a.double() * b.double()).sum())


__all__ = ["Schedule", "StepRecord", "StepFunction", "forward", "replay", "backward", "ke_band_gradient",
           "checkpoint_interval", "velocity_b_direction", "adjoint_scratch_bytes", "dot", "step_cost"]


def step_cost(n: int, dtype: str = "f32", reps: int = 10) -> dict:
    """Device time of one forward step and of one adjoint step on the same seeded turbulent state
    (PLM-MC + HLLD + GLM + forcing, CUDA events, after 3 warm-up calls): the adjoint cost ratio."""
    s = Solver(n, dtype=dtype, gamma=5.0 / 3.0, turb_amp=2.0, turb_T=0.5, turb_seed=1, courant=0.3)
    u = s.alloc()
    s.ic_turbulent(u, mach=1.0, seed=1)
    s.forcing_reset()
    s.forcing_advance()
    w = torch.empty_like(u)
    g = torch.randn_like(u)
    gb = torch.empty_like(u)
    cm, sm = s.cfl(u)
    dt = s.params.courant * s.dx / cm
    fac = s.glm_fac(sm, dt)
    calls = {"forward": lambda: s.step(u, w, dt, t=0.1, ch=sm, glm_fac=fac, do_turb=True),
             "adjoint": lambda: s.adjoint_step(u, g, gb, dt, t=0.1, ch=sm, glm_fac=fac, do_turb=True)}
    out = {}
    for name, f in calls.items():
        for _ in range(3):
            f()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            f()
        e1.record()
        torch.cuda.synchronize()
        out[name + "_ms"] = e0.elapsed_time(e1) / reps
    out["ratio"] = out["adjoint_ms"] / out["forward_ms"]
    return out


if __name__ == "__main__":   # python -m glmmhdturb_b200.adjoint [n] [f32|f64]
    import sys
    n = int(sys.argv[1]) if len(sys.argv) > 1 else 128
    dt_name = sys.argv[2] if len(sys.argv) > 2 else "f32"
    r = step_cost(n, dt_name)
    print(f"{n}^3 {dt_name}: forward {r['forward_ms']:.3f} ms, adjoint {r['adjoint_ms']:.3f} ms, ratio {r['ratio']:.2f}")
