"""ctypes binding of the CPU oracle (oracle/gmt_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, as the checker or the timed CPU baseline.  The
product package (glmmhdturb_b200) never imports this module.

Arrays are numpy, SoA planes of shape (nvar, nz, ny, nx) (x fastest), i.e. the
memory image of the reference's (N,N,N,9) column-major state
(glmmhd_turb.jl:57,63-64).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libgmt_oracle.so")

RECON = {"mc": 0, "plm": 0, "minmod": 1, "ppm": 2}
RIEMANN = {"hlld": 0, "hll": 1, "llf": 2, "llf_bound": 3}
EMF = {"average": 0, "contact": 1}
NMODES = 61


class OrcParams(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("recon", C.c_int32), ("riemann", C.c_int32), ("iflo", C.c_int32),
                ("emf", C.c_int32), ("ct_halfslope", C.c_int32),
                ("boxlen", C.c_double), ("gamma", C.c_double), ("smallr", C.c_double),
                ("smallc", C.c_double), ("smallp", C.c_double), ("llf_dmin", C.c_double),
                ("llf_pmin", C.c_double), ("turb_min_rho", C.c_double), ("nsp", C.c_int32), ("pad", C.c_int32)]


class OrcStepArgs(C.Structure):
    _fields_ = [("dt", C.c_double), ("ch", C.c_double), ("glm_fac", C.c_double),
                ("ramp", C.c_double), ("do_turb", C.c_int32), ("pad", C.c_int32),
                ("modes", C.POINTER(C.c_double))]


class OrcDiag(C.Structure):
    _fields_ = [("mass", C.c_double), ("ke2", C.c_double), ("vrms", C.c_double),
                ("divbmax", C.c_double), ("rhomin", C.c_double), ("etot", C.c_double),
                ("divb_l2", C.c_double), ("psi_l2", C.c_double), ("finite", C.c_int32),
                ("pad", C.c_int32)]


_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (g++, OpenMP, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
        fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
        P, A = C.POINTER(OrcParams), C.POINTER(OrcStepArgs)
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_num_modes.restype = C.c_int
        L.orc_mode_k.argtypes = [np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")]
        L.orc_trig_table.argtypes = [C.c_int, dp]
        u32 = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
        L.orc_philox4x32_10.argtypes = [u32, u32, u32]
        L.orc_forcing_sigma0.argtypes = [C.c_double] * 3
        L.orc_forcing_sigma0.restype = C.c_double
        L.orc_ou_update.argtypes = [dp, C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double]
        L.orc_accel_f64.argtypes = [P, dp, C.c_double, dp]
        for nm, ptr in (("f64", dp), ("f32", fp)):
            for fn in ("orc_step_unsplit_", "orc_step_march1d_", "orc_ct_step_"):
                f = getattr(L, fn + nm)
                f.argtypes = [P, A, ptr, ptr]
                f.restype = C.c_int
            getattr(L, "orc_cfl_" + nm).argtypes = [P, ptr, dp]
            getattr(L, "orc_diag_" + nm).argtypes = [P, ptr, C.POINTER(OrcDiag)]
        L.orc_jvp_unsplit_f64.argtypes = [P, A, dp, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, dp]
        L.orc_jvp_unsplit_f64.restype = C.c_int
        L.orc_ct_cfl_f64.argtypes = [P, dp, dp]
        L.orc_ct_divb_max_f64.argtypes = [P, dp]
        L.orc_ct_divb_max_f64.restype = C.c_double
        L.orc_ic_ot_f64.argtypes = [P, dp]
        L.orc_ic_uniform_f64.argtypes = [P] + [C.c_double] * 5 + [dp]
        L.orc_ct_ic_ot_f64.argtypes = [P, dp]
        L.orc_count_reset.argtypes = [C.c_int]
        L.orc_count_get.argtypes = [np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS"), C.c_int]
        _lib = L
    return _lib


def set_threads(n: int) -> int:
    return lib().orc_set_threads(int(n))


# names of the branch counters, in the order of ORC_CNT_* (gmt_oracle.h)
COUNTERS = ("hancock_revert", "iflo_revert", "void_floor", "llf_switch", "hlld_degen", "hlld_L", "hlld_Ls",
            "hlld_Rs", "hlld_R", "ppm_fallback", "face_floor", "pred1d_floor")


class branch_counts:
    """Context manager: count how often each guarded branch of the reference fires inside it.

        with branch_counts() as bc:
            step_unsplit(...)
        bc.counts["void_floor"] > 0
    """

    def __enter__(self):
        lib().orc_count_reset(1)
        self.counts = {}
        return self

    def __exit__(self, *exc):
        out = np.zeros(len(COUNTERS), dtype=np.int64)
        lib().orc_count_get(out, len(COUNTERS))
        lib().orc_count_reset(0)
        self.counts = dict(zip(COUNTERS, (int(v) for v in out)))
        return False


@dataclass
class Config:
    """Scheme + physical constants.  Defaults follow Params (glmmhd_turb.jl:28-52)."""
    n: tuple = (64, 64, 64)          # (nx, ny, nz)
    recon: str = "mc"
    riemann: str = "hlld"
    iflo: bool = True
    emf: str = "average"
    ct_halfslope: bool = False
    boxlen: float = 1.0
    gamma: float = 1.01
    smallr: float = 1e-6
    smallc: float = 1e-4
    smallp: float = 1e-6
    llf_dmin: float = 0.0
    llf_pmin: float = 0.0
    turb_min_rho: float = 1e-5
    nsp: int = 0                 # march only: passive species planes after the 9 MHD planes

    def c(self) -> OrcParams:
        nx, ny, nz = self.n
        return OrcParams(nx, ny, nz, RECON[self.recon], RIEMANN[self.riemann], int(self.iflo),
                         EMF[self.emf], int(self.ct_halfslope), self.boxlen, self.gamma,
                         self.smallr, self.smallc, self.smallp, self.llf_dmin, self.llf_pmin,
                         self.turb_min_rho, int(self.nsp), 0)

    @property
    def dx(self) -> float:
        return self.boxlen / self.n[0]


def _args(dt, ch, glm_fac, ramp=0.0, modes=None):
    a = OrcStepArgs(dt, ch, glm_fac, ramp, 0, 0, None)
    if modes is not None:
        m = np.ascontiguousarray(modes, dtype=np.float64)
        a.do_turb = 1
        a.modes = m.ctypes.data_as(C.POINTER(C.c_double))
        a._keep = m
    return a


def _fn(name, u):
    return getattr(lib(), name + ("f64" if u.dtype == np.float64 else "f32"))


def empty_state(cfg: Config, nvar=9, dtype=np.float64):
    nx, ny, nz = cfg.n
    return np.zeros((nvar, nz, ny, nx), dtype=dtype)


def step_unsplit(cfg: Config, u, dt, ch, glm_fac, ramp=0.0, modes=None):
    out = np.empty_like(u)
    a = _args(dt, ch, glm_fac, ramp, modes)
    _fn("orc_step_unsplit_", u)(C.byref(cfg.c()), C.byref(a), np.ascontiguousarray(u), out)
    return out


JVP_MAXDIR = 8


def jvp_unsplit(cfg: Config, u, du, dt, ch, glm_fac, ramp=0.0, modes=None, amp_rel=None):
    """(step output, directional derivatives) of the FP64 unsplit step by forward-mode tangents
    through the same code (the ForwardDiff counterpart).  `du`: one state direction or a stack
    (k, 9, nz, ny, nx) of k <= 8, or None; `amp_rel`: relative forcing-amplitude change per
    direction (scalar or length k), or None.  Returns dout shaped like `du` (or one state)."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    single = du is None or np.ndim(du) == u.ndim
    if du is None:
        k = 1 if amp_rel is None or np.ndim(amp_rel) == 0 else len(amp_rel)
        dstack = None
    else:
        dstack = np.ascontiguousarray(np.asarray(du, dtype=np.float64).reshape((-1,) + u.shape))
        k = dstack.shape[0]
    if not 1 <= k <= JVP_MAXDIR:
        raise ValueError("1 to 8 directions per call")
    rel = None if amp_rel is None else np.ascontiguousarray(np.broadcast_to(np.asarray(amp_rel, dtype=np.float64), (k,)))
    out = np.empty_like(u)
    dout = np.empty((k,) + u.shape)
    a = _args(dt, ch, glm_fac, ramp, modes)
    rc = lib().orc_jvp_unsplit_f64(C.byref(cfg.c()), C.byref(a), u, k,
                                   None if dstack is None else dstack.ctypes.data_as(C.c_void_p),
                                   None if rel is None else rel.ctypes.data_as(C.c_void_p),
                                   out.ctypes.data_as(C.c_void_p), dout)
    if rc:
        raise ValueError("orc_jvp_unsplit_f64 failed")
    return out, (dout[0] if single else dout)


def step_march1d(cfg: Config, u, dt, ch, glm_fac):
    out = np.empty_like(u)
    a = _args(dt, ch, glm_fac)
    _fn("orc_step_march1d_", u)(C.byref(cfg.c()), C.byref(a), np.ascontiguousarray(u), out)
    return out


def ct_step(cfg: Config, q, dt, ramp=0.0, modes=None):
    out = np.empty_like(q)
    a = _args(dt, 0.0, 1.0, ramp, modes)
    _fn("orc_ct_step_", q)(C.byref(cfg.c()), C.byref(a), np.ascontiguousarray(q), out)
    return out


def cfl(cfg: Config, u):
    out = np.zeros(2)
    _fn("orc_cfl_", u)(C.byref(cfg.c()), np.ascontiguousarray(u), out)
    return float(out[0]), float(out[1])


def ct_cfl(cfg: Config, q):
    out = np.zeros(2)
    lib().orc_ct_cfl_f64(C.byref(cfg.c()), np.ascontiguousarray(q, dtype=np.float64), out)
    return float(out[0]), float(out[1])


def diagnostics(cfg: Config, u) -> dict:
    d = OrcDiag()
    _fn("orc_diag_", u)(C.byref(cfg.c()), np.ascontiguousarray(u), C.byref(d))
    return {k: getattr(d, k) for k, _ in OrcDiag._fields_ if k != "pad"}


def ct_divb_max(cfg: Config, q) -> float:
    return lib().orc_ct_divb_max_f64(C.byref(cfg.c()), np.ascontiguousarray(q, dtype=np.float64))


def ic_ot(cfg: Config):
    u = empty_state(cfg)
    lib().orc_ic_ot_f64(C.byref(cfg.c()), u)
    return u


def ct_ic_ot(cfg: Config):
    q = empty_state(cfg, nvar=8)
    lib().orc_ct_ic_ot_f64(C.byref(cfg.c()), q)
    return q


def ic_uniform(cfg: Config, rho0=1.0, p0=0.6, b0=(0.775, 0.0, 0.0)):
    u = empty_state(cfg)
    lib().orc_ic_uniform_f64(C.byref(cfg.c()), rho0, p0, b0[0], b0[1], b0[2], u)
    return u


# ----------------------------------------------------------------------------------------
# forcing helpers
# ----------------------------------------------------------------------------------------
def mode_k() -> np.ndarray:
    k = np.zeros(3 * NMODES, dtype=np.int32)
    lib().orc_mode_k(k)
    return k.reshape(NMODES, 3)


def trig_table(n: int) -> np.ndarray:
    t = np.zeros(8 * n)
    lib().orc_trig_table(n, t)
    return t.reshape(4, 2, n)


def philox(ctr, key) -> np.ndarray:
    out = np.zeros(4, dtype=np.uint32)
    lib().orc_philox4x32_10(np.asarray(ctr, dtype=np.uint32), np.asarray(key, dtype=np.uint32), out)
    return out


@dataclass
class OUForcing:
    """Deterministic OU mode forcing (the oracle's copy of the library's definition)."""
    amp: float
    T: float = 0.5
    ndt: int = 100
    seed: int = 0
    counter: int = 0
    modes: np.ndarray = field(default_factory=lambda: np.zeros((NMODES, 3, 2)))
    next_time: float = 0.0

    @property
    def dtf(self):
        return self.T / self.ndt

    @property
    def alpha(self):
        return 1.0 - self.dtf / self.T

    @property
    def beta(self):
        return math.sqrt(2.0 * self.dtf / self.T)

    def advance(self):
        L = lib()
        s0 = L.orc_forcing_sigma0(self.amp, self.alpha, self.beta)
        m = np.ascontiguousarray(self.modes.reshape(-1))
        L.orc_ou_update(m, self.seed, self.counter, self.alpha, self.beta, s0)
        self.modes = m.reshape(NMODES, 3, 2)
        self.counter += 1
        self.next_time += self.dtf

    def ramp(self, t):
        return min(t / self.T, 1.0)


def accel(cfg: Config, modes, ramp=1.0):
    a = np.zeros((3,) + tuple(reversed(cfg.n)))
    lib().orc_accel_f64(C.byref(cfg.c()), np.ascontiguousarray(modes, dtype=np.float64), ramp, a)
    return a


# ----------------------------------------------------------------------------------------
# drivers mirroring the reference's host loops
# ----------------------------------------------------------------------------------------
def glm_ch_reference(cfg: Config, courant: float, dt: float, glm_ch_scale=0.25):
    """ch = courant*dx/dt/3*glm_ch_scale (glmmhd_turb.jl:582)."""
    return courant * cfg.dx / dt / 3.0 * glm_ch_scale


def glm_fac(ch, dt, cp_coef=0.18, boxlen=1.0):
    """exp(-(ch^2/(cp_coef*L*ch))*dt) (glmmhd_turb.jl:583)."""
    return math.exp(-(ch * ch / (cp_coef * boxlen * ch)) * dt) if cp_coef > 0 else 1.0


def run_ot(cfg: Config, t_end=0.2, courant=0.7):
    """validate_tiled_ot / run_ot host loop (glmmhd_turb.jl:2041-2068, 2278-2294), FP64."""
    u = ic_ot(cfg)
    t, step = 0.0, 0
    while t < t_end:
        cmax, _ = cfl(cfg, u)
        dt = courant * cfg.dx / cmax
        dt = min(dt, t_end - t)
        ch = glm_ch_reference(cfg, courant, dt)
        u = step_unsplit(cfg, u, dt, ch, glm_fac(ch, dt))
        t += dt
        step += 1
    d = diagnostics(cfg, u)
    d["steps"] = step
    d["t"] = t
    return u, d
