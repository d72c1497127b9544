"""Host-side mirror of the GLMMHDTurb step API (glmmhd_turb.jl), backed by libglmmhd_b200.so.

Same names, argument meaning and error behaviour as the reference's Julia functions, with
torch CUDA tensors of shape (9, N, N, N) (the memory image of the reference's (N,N,N,9) array):

    Params, dxof, pfloor, NV                         glmmhd_turb.jl:28-59
    step_plm(uold, unew, afield, p, dt, t; ...)      glmmhd_turb.jl:878-908
    step_tiled(uold, unew, afield, p, dt, t; ...)    glmmhd_turb.jl:746-767
    step_fused(uold, unew, afield, p, dt, t, be; ..) glmmhd_turb.jl:578-589
    step_multi(uold, unew, rec, flx, ct, afield, p, dt, t, be; ...)  glmmhd_turb.jl:1981-1992
    compute_dt(uold, ct, p, be)                      glmmhd_turb.jl:1973-1978
    diagnostics(u, ct, p, be)                        glmmhd_turb.jl:2006-2018
    Forcing(p, be; amp), ou_advance(f, p, be)        glmmhd_turb.jl:2116-2161 (mode-sum OU)
    ic_ot, ic_uniform, run_ot, run_turb              glmmhd_turb.jl:2021-2068, 2164-2240

`afield` is a `Forcing` (the 61-mode OU state) or None; `rec`, `flx`, `ct` and `be` are
accepted for signature compatibility and unused (the library keeps its own scratch).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, replace

import torch

from .solver import Solver

NV = 9
TB = 4


@dataclass(frozen=True)
class Params:
    N: int = 256
    boxlen: float = 1.0
    gamma: float = 1.01
    courant: float = 0.7
    smallr: float = 1.0e-6
    smallc: float = 1.0e-4
    glm_ch_scale: float = 0.25
    glm_cp_coef: float = 0.18
    switch_llf_dmin: float = 0.0
    switch_llf_pmin: float = 0.0
    rho0: float = 1.0
    cs0: float = 1.0
    b0: float = 1.0
    turb_rms: float = 130.0
    turb_T: float = 0.3
    turb_Ndt: int = 100
    comp_frac: float = 0.5
    turb_min_rho: float = 1.0e-5
    turb_seed: int = 1


def dxof(p: Params) -> float:
    return p.boxlen / p.N


def pfloor(p: Params) -> float:
    return p.smallr * p.smallc ** 2 / p.gamma


def _dtype_of(u: torch.Tensor) -> str:
    if u.dtype == torch.float32:
        return "f32"
    if u.dtype == torch.float64:
        return "f64"
    raise TypeError(f"state dtype must be float32 or float64, got {u.dtype}")


_SOLVERS: dict = {}


def solver_for(p: Params, dtype: str, recon: str, riemann: str, iflo: bool, tile=(0, 0, 0)) -> Solver:
    """Cached engine for (Params, precision, scheme)."""
    key = (p, dtype, recon, riemann, iflo, tuple(tile), torch.cuda.current_device())
    s = _SOLVERS.get(key)
    if s is None:
        s = Solver(p.N, dtype=dtype, recon=recon, riemann=riemann, iflo=iflo, boxlen=p.boxlen, gamma=p.gamma,
                   courant=p.courant, smallr=p.smallr, smallc=p.smallc, glm_ch_scale=p.glm_ch_scale,
                   glm_cp_coef=p.glm_cp_coef, llf_dmin=p.switch_llf_dmin, llf_pmin=p.switch_llf_pmin,
                   turb_min_rho=p.turb_min_rho, turb_amp=p.turb_rms, turb_T=p.turb_T, turb_ndt=p.turb_Ndt,
                   turb_seed=p.turb_seed, tile=tile)
        _SOLVERS[key] = s
    return s


def glm_parameters(p: Params, dt: float):
    """ch = courant*dx/dt/3*glm_ch_scale; glm_fac = exp(-(ch^2/(cp*L*ch))*dt) (glmmhd_turb.jl:582-583)."""
    ch = p.courant * dxof(p) / dt / 3.0 * p.glm_ch_scale
    fac = math.exp(-(ch * ch / (p.glm_cp_coef * p.boxlen * ch)) * dt) if p.glm_cp_coef > 0 else 1.0
    return ch, fac


class Forcing:
    """OU turbulent forcing: 61 solenoidal +/- mode pairs (1 <= |k| <= 3) on the device.

    Replaces the reference's 64^3 FFT field (glmmhd_turb.jl:2116-2161); `next_time` and the
    update cadence turb_T/turb_Ndt follow the reference host loop."""

    def __init__(self, p: Params, be=None, *, amp: float | None = None, dtype: str = "f32"):
        self.p = replace(p, turb_rms=p.turb_rms if amp is None else float(amp))
        self.amp = self.p.turb_rms
        self.solver = solver_for(self.p, dtype, "mc", "hlld", True)
        self.solver.forcing_reset()
        self.next_time = 0.0
        self.version = 0

    def modes(self):
        return self.solver.get_modes()


def ou_advance(f: Forcing, p: Params = None, be=None):
    """Advance the OU modes by one turb_T/turb_Ndt interval (glmmhd_turb.jl:2146-2161)."""
    f.solver.forcing_advance()
    f.next_time += f.p.turb_T / f.p.turb_Ndt
    f.version += 1


def _forcing_into(s: Solver, afield, do_turb: bool):
    if not do_turb:
        return
    if not isinstance(afield, Forcing):
        raise TypeError("do_turb=True needs a Forcing as afield")
    if afield.solver is s:
        return
    if getattr(s, "_forcing_version", None) != (id(afield), afield.version):
        s.set_modes(afield.modes())
        s._forcing_version = (id(afield), afield.version)


def _step(uold, unew, afield, p, dt, t, recon, riemann, iflo, do_turb, tile=(0, 0, 0)):
    s = solver_for(p, _dtype_of(uold), recon, riemann, iflo, tile)
    _forcing_into(s, afield, do_turb)
    ch, fac = glm_parameters(p, dt)
    s.step(uold, unew, dt, t, ch=ch, glm_fac=fac, do_turb=do_turb)


def step_plm(uold, unew, afield, p: Params, dt: float, t: float, *, do_turb=False, nthreads=192, tb=0, half=True,
             riemann="hll", recon="plm"):
    """Production PLM/PPM step (glmmhd_turb.jl:878-908).  `half` selected 16-bit shared tiles in the
    reference; this build always stages FP32/FP64 tiles.  Any (recon, riemann) pair is supported."""
    if tb == 0:
        tb = 6 if p.N % 6 == 0 else 4
    if p.N % tb != 0:
        raise ValueError(f"N={p.N} not divisible by tb={tb} (need N%6==0 for the fast TB=6 path, or N%4==0)")
    if recon not in ("plm", "ppm"):
        raise ValueError(f"step_plm!: unsupported recon={recon}")
    if riemann not in ("hll", "llf", "hlld"):
        raise ValueError(f"step_plm!: unsupported riemann={riemann}")
    rs = {"hll": "hll", "llf": "llf_bound", "hlld": "hlld"}[riemann]
    _step(uold, unew, afield, p, dt, t, "ppm" if recon == "ppm" else "mc", rs, True, do_turb)


def step_tiled(uold, unew, afield, p: Params, dt: float, t: float, *, use_hlld=True, do_turb=False, nthreads=192,
               maxregs=0, lean=False):
    """Tiled HLLD step (glmmhd_turb.jl:746-767); lean = minmod slopes + LLF with the bound speed."""
    if p.N % TB != 0:
        raise ValueError(f"N must be a multiple of {TB}")
    if lean:
        _step(uold, unew, afield, p, dt, t, "minmod", "llf_bound", True, do_turb)
    else:
        _step(uold, unew, afield, p, dt, t, "mc", "hlld" if use_hlld else "llf", True, do_turb)


def step_fused(uold, unew, afield, p: Params, dt: float, t: float, be=None, *, use_hlld=True, do_turb=False):
    """Recompute step (glmmhd_turb.jl:578-589): no interface-state revert."""
    _step(uold, unew, afield, p, dt, t, "mc", "hlld" if use_hlld else "llf", False, do_turb)


def step_multi(uold, unew, rec, flx, ct, afield, p: Params, dt: float, t: float, be=None, *, use_hlld=True,
               do_turb=False):
    """Multi-kernel validation step (glmmhd_turb.jl:1981-1992): no interface-state revert."""
    _step(uold, unew, afield, p, dt, t, "mc", "hlld" if use_hlld else "llf", False, do_turb)


def compute_dt(uold, ct, p: Params, be=None) -> float:
    """courant*dx/max(sum_d(|v_d|+c_f)) (glmmhd_turb.jl:1973-1978)."""
    return solver_for(p, _dtype_of(uold), "mc", "hlld", True).compute_dt(uold)


def diagnostics(u, ct, p: Params, be=None) -> dict:
    """mass, vrms, Mach, centred div B max, rhomin, finite (glmmhd_turb.jl:2006-2018)."""
    d = solver_for(p, _dtype_of(u), "mc", "hlld", True).diagnostics(u)
    return {"mass": d["mass"], "vrms": d["vrms"], "mach": d["vrms"] / p.cs0, "divbmax": d["divbmax"],
            "rhomin": d["rhomin"], "finite": bool(d["finite"]), "etot": d["etot"], "divb_l2": d["divb_l2"]}


def ic_ot(u, p: Params):
    """Orszag-Tang (glmmhd_turb.jl:2021-2036)."""
    solver_for(p, _dtype_of(u), "mc", "hlld", True).ic_orszag_tang(u)


def ic_uniform(u, p: Params, rho0=None, p0=None, b0=None):
    """Uniform state rho0, p0 = rho0*cs0^2/gamma, Bx = b0 (glmmhd_turb.jl:2164-2172)."""
    rho0 = p.rho0 if rho0 is None else rho0
    p0 = p.rho0 * p.cs0 ** 2 / p.gamma if p0 is None else p0
    b0 = (p.b0, 0.0, 0.0) if b0 is None else b0
    solver_for(p, _dtype_of(u), "mc", "hlld", True).ic_uniform(u, rho0, p0, b0)


def run_ot(*, N=128, t_end=0.5, use_hlld=True, dtype="f32", courant=0.7):
    """Orszag-Tang to t_end on the step_multi! semantics (glmmhd_turb.jl:2041-2068)."""
    p = Params(N=N, gamma=5.0 / 3.0, cs0=1.0, courant=courant)
    s = solver_for(p, dtype, "mc", "hlld", True)
    u1 = s.alloc()
    u2 = s.alloc()
    ic_ot(u1, p)
    t, step = 0.0, 0
    while t < t_end:
        dt = min(compute_dt(u1, None, p), t_end - t)
        step_multi(u1, u2, None, None, None, None, p, dt, t, use_hlld=use_hlld)
        u1, u2 = u2, u1
        t += dt
        step += 1
    d = diagnostics(u1, None, p)
    d.update(steps=step, t=t)
    return d


def run_turb(*, N=128, t_end=0.6, amp=130.0, use_hlld=True, nstepmax=20000, dtype="f32", solver="tiled"):
    """Driven turbulence (glmmhd_turb.jl:2191-2240) with the mode-sum OU forcing."""
    p0_ = 1.0 / 1.01
    p = Params(N=N, turb_rms=amp, switch_llf_dmin=0.01, switch_llf_pmin=0.01 * p0_)
    s = solver_for(p, dtype, "mc", "hlld", True)
    u1 = s.alloc()
    u2 = s.alloc()
    ic_uniform(u1, p)
    f = Forcing(p, amp=amp, dtype=dtype)
    ou_advance(f, p)
    t, step = 0.0, 0
    while t < t_end and step < nstepmax:
        while t >= f.next_time:
            ou_advance(f, p)
        dt = compute_dt(u1, None, p)
        dt = min(dt, f.next_time - t, t_end - t)
        if solver == "plm":
            step_plm(u1, u2, f, p, dt, t, do_turb=True, riemann="hll")
        else:
            step_tiled(u1, u2, f, p, dt, t, use_hlld=use_hlld, do_turb=True)
        u1, u2 = u2, u1
        t += dt
        step += 1
    d = diagnostics(u1, None, p)
    d.update(steps=step, t=t)
    return d
