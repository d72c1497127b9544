"""Solver: one gmt_ctx (include/glmmhd_b200.h) driven with device tensors.

torch is used only to own device memory and streams; every kernel is in libglmmhd_b200.so.
State tensors are contiguous (nvar, nz, ny, nx) arrays -- the memory image of the reference's
(N,N,N,9) column-major state (glmmhd_turb.jl:57,63-64).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _lib
from ._lib import GmtDiag, GmtParams, GmtStepArgs, check, lib

_DT = {"f32": (_lib.F32, torch.float32), "f64": (_lib.F64, torch.float64)}


def _stream_handle(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


class Solver:
    """A configured time-step engine for one grid, precision and scheme.

    Parameters mirror `Params` (glmmhd_turb.jl:28-52) plus the scheme selectors of step_plm!
    (recon, riemann) and step_tiled! (lean / use_hlld), the CT options and the forcing.
    """

    def __init__(self, n, *, dtype="f32", scheme="unsplit", recon="mc", riemann="hlld", iflo=True,
                 emf="average", ct_halfslope=False, boxlen=1.0, gamma=1.01, courant=0.7, smallr=1e-6,
                 smallc=1e-4, smallp=1e-6, glm_ch_scale=0.25, glm_cp_coef=0.18, llf_dmin=0.0, llf_pmin=0.0,
                 turb_min_rho=1e-5, turb_amp=0.0, turb_T=0.3, turb_ndt=100, turb_seed=1, tile=(0, 0, 0)):
        if isinstance(n, int):
            n = (n, n, n)
        self.nx, self.ny, self.nz = (int(v) for v in n)
        if dtype not in _DT:
            raise ValueError("dtype must be 'f32' or 'f64'")
        self.dtype_name = dtype
        self.code, self.torch_dtype = _DT[dtype]
        self.scheme = scheme
        self.nvar = 8 if scheme == "ct" else 9
        p = GmtParams()
        check(lib().gmt_params_init(C.byref(p), self.nx))
        p.nx, p.ny, p.nz = self.nx, self.ny, self.nz
        p.dtype = self.code
        p.scheme = _lib.SCHEME[scheme]
        p.recon = _lib.RECON[recon]
        p.riemann = _lib.RIEMANN[riemann]
        p.iflo = int(bool(iflo))
        p.emf = _lib.EMF[emf]
        p.ct_halfslope = int(bool(ct_halfslope))
        p.tile_x, p.tile_y, p.tile_z = (int(v) for v in tile)
        p.boxlen, p.gamma, p.courant = boxlen, gamma, courant
        p.smallr, p.smallc, p.smallp = smallr, smallc, smallp
        p.glm_ch_scale, p.glm_cp_coef = glm_ch_scale, glm_cp_coef
        p.llf_dmin, p.llf_pmin, p.turb_min_rho = llf_dmin, llf_pmin, turb_min_rho
        p.turb_amp, p.turb_T, p.turb_ndt, p.turb_seed = turb_amp, turb_T, int(turb_ndt), int(turb_seed)
        self.params = p
        self.device = torch.device("cuda", torch.cuda.current_device())
        self._ctx = C.c_void_p()
        check(lib().gmt_create(C.byref(p), C.byref(self._ctx)))
        self.next_time = 0.0   # forcing bookkeeping of the host loop (glmmhd_turb.jl:2146-2161)

    # ------------------------------------------------------------------ basics
    @property
    def n(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def dx(self) -> float:
        return self.params.boxlen / self.nx

    def close(self):
        if self._ctx:
            lib().gmt_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def alloc(self, nvar=None) -> torch.Tensor:
        return torch.empty((nvar or self.nvar, self.nz, self.ny, self.nx), dtype=self.torch_dtype,
                           device=self.device)

    def _ptr(self, u: torch.Tensor, nvar=None) -> int:
        nvar = nvar or self.nvar
        if not isinstance(u, torch.Tensor) or not u.is_cuda:
            raise TypeError("state must be a CUDA tensor")
        if u.dtype != self.torch_dtype:
            raise TypeError(f"state dtype {u.dtype} does not match the solver ({self.torch_dtype})")
        if u.numel() != nvar * self.n or not u.is_contiguous():
            raise ValueError(f"state must be contiguous with {nvar} planes of {self.nx}x{self.ny}x{self.nz}")
        return u.data_ptr()

    def kernel_info(self) -> dict:
        regs = C.c_int32()
        smem = C.c_int64()
        tile = (C.c_int32 * 3)()
        check(lib().gmt_kernel_info(self._ctx, C.byref(regs), C.byref(smem), tile))
        return {"regs": regs.value, "smem": smem.value, "tile": tuple(tile)}

    # ------------------------------------------------------------------ GLM parameters
    def glm_reference(self, dt: float):
        """ch = courant*dx/dt/3*glm_ch_scale, glm_fac = exp(-ch*dt/(cp*L)) (glmmhd_turb.jl:582-583)."""
        p = self.params
        ch = p.courant * self.dx / dt / 3.0 * p.glm_ch_scale
        return ch, self.glm_fac(ch, dt)

    def glm_fac(self, ch: float, dt: float) -> float:
        p = self.params
        return math.exp(-(ch * ch / (p.glm_cp_coef * p.boxlen * ch)) * dt) if p.glm_cp_coef > 0 else 1.0

    # ------------------------------------------------------------------ stepping
    def step(self, uold, unew, dt, t=0.0, ch=None, glm_fac=None, do_turb=False, want_cfl=False, stream=None):
        """One step uold -> unew.  ch/glm_fac default to the reference policy."""
        if ch is None:
            ch, fac = self.glm_reference(dt)
            glm_fac = fac if glm_fac is None else glm_fac
        elif glm_fac is None:
            glm_fac = self.glm_fac(ch, dt)
        a = GmtStepArgs(float(dt), float(t), float(ch), float(glm_fac), int(bool(do_turb)), int(bool(want_cfl)))
        fn = lib().gmt_ct_step if self.scheme == "ct" else lib().gmt_step
        check(fn(self._ctx, self._ptr(uold), self._ptr(unew), C.byref(a), _stream_handle(stream)))

    def cfl_async(self, u, stream=None):
        fn = lib().gmt_ct_cfl_async if self.scheme == "ct" else lib().gmt_cfl_async
        check(fn(self._ctx, self._ptr(u), _stream_handle(stream)))

    def cfl_result(self, stream=None):
        out = (C.c_double * 2)()
        check(lib().gmt_cfl_result(self._ctx, out, _stream_handle(stream)))
        return out[0], out[1]

    def cfl(self, u, stream=None):
        """(max sum_d(|v_d|+cf_d), max max_d(|v_d|+cf_d)) over the grid."""
        self.cfl_async(u, stream)
        return self.cfl_result(stream)

    def compute_dt(self, u, stream=None) -> float:
        """courant*dx/max(ctot) (glmmhd_turb.jl:1973-1978)."""
        cmax, _ = self.cfl(u, stream)
        return self.params.courant * self.dx / cmax

    def diagnostics(self, u, stream=None) -> dict:
        if self.scheme == "ct":
            return {"divbmax": self.ct_divb_max(u, stream)}
        d = GmtDiag()
        check(lib().gmt_diagnostics(self._ctx, self._ptr(u), C.byref(d), _stream_handle(stream)))
        return {k: getattr(d, k) for k, _ in GmtDiag._fields_}

    def ct_divb_max(self, q, stream=None) -> float:
        out = C.c_double()
        check(lib().gmt_ct_divb_max(self._ctx, self._ptr(q), C.byref(out), _stream_handle(stream)))
        return out.value

    # ------------------------------------------------------------------ forcing
    def forcing_reset(self, stream=None):
        check(lib().gmt_forcing_reset(self._ctx, _stream_handle(stream)))
        self.next_time = 0.0

    def forcing_advance(self, stream=None):
        """One OU update of the 61 modes; advances next_time by turb_T/turb_ndt."""
        check(lib().gmt_forcing_advance(self._ctx, _stream_handle(stream)))
        self.next_time += self.params.turb_T / self.params.turb_ndt

    def set_modes(self, modes: np.ndarray, stream=None):
        m = np.ascontiguousarray(modes, dtype=np.float64).reshape(-1)
        if m.size != _lib.NMODES * 6:
            raise ValueError("modes must have 61*3*2 entries")
        check(lib().gmt_forcing_set_modes(self._ctx, m.ctypes.data_as(C.POINTER(C.c_double)),
                                          _stream_handle(stream)))

    def get_modes(self, stream=None) -> np.ndarray:
        m = np.zeros(_lib.NMODES * 6)
        check(lib().gmt_forcing_get_modes(self._ctx, m.ctypes.data_as(C.POINTER(C.c_double)),
                                          _stream_handle(stream)))
        return m.reshape(_lib.NMODES, 3, 2)

    def forcing_counter(self) -> int:
        c = C.c_uint32()
        check(lib().gmt_forcing_counter(self._ctx, C.byref(c)))
        return c.value

    # ------------------------------------------------------------------ initial conditions
    def ic_orszag_tang(self, u, stream=None):
        fn = lib().gmt_ct_ic_orszag_tang if self.scheme == "ct" else lib().gmt_ic_orszag_tang
        check(fn(self._ctx, self._ptr(u), _stream_handle(stream)))

    def ic_uniform(self, u, rho0=1.0, p0=0.6, b0=(0.775, 0.0, 0.0), stream=None):
        check(lib().gmt_ic_uniform(self._ctx, self._ptr(u), rho0, p0, b0[0], b0[1], b0[2],
                                   _stream_handle(stream)))

    def ic_turbulent(self, u, rho0=1.0, p0=0.6, b0=(0.775, 0.0, 0.0), mach=1.0, db=0.1, seed=1, stream=None):
        """Seeded synthetic turbulent state (gmt_ic_turbulent): rms Mach ~ `mach`, |dB| ~ `db`."""
        check(lib().gmt_ic_turbulent(self._ctx, self._ptr(u), rho0, p0, b0[0], b0[1], b0[2], mach, db, int(seed),
                                     _stream_handle(stream)))
