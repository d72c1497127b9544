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
                 turb_min_rho=1e-5, turb_amp=0.0, turb_T=0.3, turb_ndt=100, turb_seed=1, tile=(0, 0, 0), nsp=0):
        if isinstance(n, int):
            n = (n, n, n)
        self.nx, self.ny, self.nz = (int(v) for v in n)
        if dtype not in _DT:
            raise ValueError("dtype must be 'f32' or 'f64'")
        self.dtype_name = dtype
        self.code, self.torch_dtype = _DT[dtype]
        self.scheme = scheme
        self.nsp = int(nsp)   # march scheme: passive species planes (rho*X) after the 9 MHD planes
        self.nvar = 8 if scheme == "ct" else 9 + self.nsp
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
        p.nsp = self.nsp
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

    def ke_spectrum(self, u, kmax=8, stream=None) -> np.ndarray:
        """Shell-binned kinetic-energy spectrum E(k), k = 0..kmax, of w = sqrt(rho) v (FP64)."""
        out = np.zeros(kmax + 1)
        check(lib().gmt_ke_spectrum(self._ctx, self._ptr(u), int(kmax), out.ctypes.data_as(C.POINTER(C.c_double)),
                                    _stream_handle(stream)))
        return out

    def density_pdf(self, u, nbins=64, smin=-4.0, smax=4.0, stream=None):
        """(pdf, stats) of s = ln(rho/<rho>): pdf per bin of [smin, smax) (density, FP64) and
        stats = {'rho_mean', 's_mean', 'sigma_s'}."""
        pdf = np.zeros(int(nbins))
        st = np.zeros(3)
        check(lib().gmt_density_pdf(self._ctx, self._ptr(u), int(nbins), float(smin), float(smax),
                                    pdf.ctypes.data_as(C.POINTER(C.c_double)), st.ctypes.data_as(C.POINTER(C.c_double)),
                                    _stream_handle(stream)))
        return pdf, {"rho_mean": st[0], "s_mean": st[1], "sigma_s": st[2]}

    def ke_band_loss(self, u, kmin=4, kmax=8, ubar=None, stream=None):
        """(L, dL/du) for L = sum_{kmin<=k<=kmax} E(k) of ke_spectrum; dL/du goes to `ubar` (allocated
        when None)."""
        if ubar is None:
            ubar = self.alloc()
        out = C.c_double()
        check(lib().gmt_ke_band_loss(self._ctx, self._ptr(u), int(kmin), int(kmax), C.byref(out), self._ptr(ubar),
                                     _stream_handle(stream)))
        return out.value, ubar

    # ------------------------------------------------------------------ discrete adjoint
    def adjoint_step(self, u, ubar_next, ubar, dt, t=0.0, ch=None, glm_fac=None, do_turb=False, stream=None):
        """ubar = (du'/du)^T ubar_next for the step u -> u' taken with the same dt, t, ch, glm_fac,
        do_turb and forcing modes; adds the step's dL/d(turb_amp) to the context's accumulator."""
        if ch is None:
            ch, fac = self.glm_reference(dt)
            glm_fac = fac if glm_fac is None else glm_fac
        elif glm_fac is None:
            glm_fac = self.glm_fac(ch, dt)
        a = GmtStepArgs(float(dt), float(t), float(ch), float(glm_fac), int(bool(do_turb)), 0)
        check(lib().gmt_adjoint_step(self._ctx, self._ptr(u), self._ptr(ubar_next), self._ptr(ubar), C.byref(a),
                                     _stream_handle(stream)))

    def adjoint_set_passes(self, percell: bool):
        """percell=True: the FP32 adjoint runs its first three passes per cell instead of as the
        record-mode tile march (the check of the tile form; gmt_adjoint_set_passes)."""
        check(lib().gmt_adjoint_set_passes(self._ctx, int(bool(percell))))

    def test_wait_limit(self, budget_cycles=0, withhold=False):
        """Failure-path tests only: bounded-wait budget in SM cycles, and withhold=True to skip the
        staging of each next plane so every wait runs out (gmt_test_wait_limit); (0, False)
        restores production behaviour."""
        check(lib().gmt_test_wait_limit(self._ctx, int(budget_cycles), int(bool(withhold))))

    def adjoint_amp_grad(self, reset=True, stream=None) -> float:
        out = C.c_double()
        check(lib().gmt_adjoint_amp_grad(self._ctx, C.byref(out), int(bool(reset)), _stream_handle(stream)))
        return out.value

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

    def forcing_state(self, stream=None) -> dict:
        """The whole forcing state: modes, the Philox counter of the next OU update, next update time."""
        m = np.zeros(_lib.NMODES * 6)
        c = C.c_uint32()
        nt = C.c_double()
        check(lib().gmt_forcing_get_state(self._ctx, m.ctypes.data_as(C.POINTER(C.c_double)), C.byref(c),
                                          C.byref(nt), _stream_handle(stream)))
        return {"modes": m.reshape(_lib.NMODES, 3, 2), "counter": c.value, "next_time": nt.value}

    def set_forcing_state(self, state: dict, stream=None):
        """Restore a forcing_state() (from this or another context: the forcing is grid-independent)."""
        m = np.ascontiguousarray(state["modes"], dtype=np.float64).reshape(-1)
        if m.size != _lib.NMODES * 6:
            raise ValueError("modes must have 61*3*2 entries")
        check(lib().gmt_forcing_set_state(self._ctx, m.ctypes.data_as(C.POINTER(C.c_double)), int(state["counter"]),
                                          float(state["next_time"]), _stream_handle(stream)))
        self.next_time = float(state["next_time"])

    # ------------------------------------------------------------------ device-resident loop
    def run(self, u, w, nsteps, t0=0.0, t_end=1e300, *, ch_max_signal=True, forcing=False, graph=True, stream=None):
        """nsteps steps with dt, ch, glm_fac and the forcing cadence decided on the device (gmt_run);
        returns (t reached, result tensor)."""
        flags = ((_lib.RUN_CH_MAXSIGNAL if ch_max_signal else 0) | (_lib.RUN_FORCING if forcing else 0) |
                 (_lib.RUN_GRAPH if graph else 0))
        t = C.c_double()
        which = C.c_int32()
        check(lib().gmt_run(self._ctx, self._ptr(u), self._ptr(w), int(nsteps), float(t0), float(t_end), flags,
                            _stream_handle(stream), C.byref(t), C.byref(which)))
        if forcing:
            self.next_time = self.forcing_state(stream)["next_time"]
        return t.value, (w if which.value else u)

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


class Ensemble:
    """Many periodic GLM boxes of different sizes advanced together: one persistent kernel per step
    over a queue of tile work items of all boxes (32x16 columns in FP32, 16x16 in FP64, z-chunks of
    at most 64 planes), every box with its own dt, forcing amplitude and seed (gmt_ensemble_*)."""

    def __init__(self, sizes, *, amps=None, seeds=None, dtype="f32", recon="mc", riemann="hlld", gamma=5.0 / 3.0,
                 courant=0.3, turb_T=0.5, turb_ndt=100, **kw):
        self.sizes = [int(n) for n in sizes]
        self.dtype_name = dtype
        self.code, self.torch_dtype = _DT[dtype]
        p = GmtParams()
        check(lib().gmt_params_init(C.byref(p), 16))
        p.dtype = self.code
        p.recon = _lib.RECON[recon]
        p.riemann = _lib.RIEMANN[riemann]
        p.gamma, p.courant, p.turb_T, p.turb_ndt = gamma, courant, turb_T, int(turb_ndt)
        for k, v in kw.items():
            setattr(p, k, v)
        nb = len(self.sizes)
        n_arr = (C.c_int32 * nb)(*self.sizes)
        a_arr = (C.c_double * nb)(*(amps if amps is not None else [0.0] * nb))
        s_arr = (C.c_uint32 * nb)(*(seeds if seeds is not None else list(range(nb))))
        self._e = C.c_void_p()
        check(lib().gmt_ensemble_create(C.byref(p), nb, n_arr, a_arr, s_arr, C.byref(self._e)))
        self.device = torch.device("cuda", torch.cuda.current_device())

    def alloc(self):
        return [torch.empty((9, n, n, n), dtype=self.torch_dtype, device=self.device) for n in self.sizes]

    def run(self, u, w, nsteps, t_end=1e300, *, ch_max_signal=True, forcing=True, graph=True, stream=None):
        """nsteps ensemble steps; returns the list of times reached (result in u if nsteps is even)."""
        nb = len(self.sizes)
        for x, n in zip(list(u) + list(w), self.sizes + self.sizes):
            if x.dtype != self.torch_dtype or x.numel() != 9 * n ** 3 or not x.is_contiguous():
                raise ValueError("ensemble states must be contiguous 9 x n^3 tensors of the ensemble dtype")
        ua = (C.c_void_p * nb)(*[x.data_ptr() for x in u])
        wa = (C.c_void_p * nb)(*[x.data_ptr() for x in w])
        t = (C.c_double * nb)()
        flags = ((_lib.RUN_CH_MAXSIGNAL if ch_max_signal else 0) | (_lib.RUN_FORCING if forcing else 0) |
                 (_lib.RUN_GRAPH if graph else 0))
        check(lib().gmt_ensemble_run(self._e, C.cast(ua, C.c_void_p), C.cast(wa, C.c_void_p), int(nsteps),
                                     float(t_end), flags, _stream_handle(stream), t))
        return list(t)

    def close(self):
        if self._e:
            lib().gmt_ensemble_destroy(self._e)
            self._e = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
