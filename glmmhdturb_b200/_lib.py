"""ctypes binding of libglmmhd_b200.so (include/glmmhd_b200.h).

The library is built in-tree by ``glmmhdturb_b200/csrc/Makefile``.  There is no fallback: if the
shared object is missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libglmmhd_b200.so")
CSRC = os.path.join(HERE, "csrc")

GMT_ABI_VERSION = 1
GMT_OK, GMT_ERR_ARG, GMT_ERR_CUDA, GMT_ERR_UNSUPPORTED, GMT_ERR_STATE, GMT_ERR_NOMEM, GMT_ERR_TIMEOUT = range(7)
F32, F64 = 0, 1
SCHEME = {"unsplit": 0, "march1d": 1, "ct": 2}
RECON = {"mc": 0, "plm": 0, "minmod": 1, "ppm": 2}
RIEMANN = {"hlld": 0, "hll": 1, "llf": 2, "llf_bound": 3}
EMF = {"average": 0, "contact": 1}
NMODES = 61
NOALLOC_MAX_PLANES = 2048
RUN_CH_MAXSIGNAL, RUN_FORCING, RUN_GRAPH = 1, 2, 4

# every symbol declared in include/glmmhd_b200.h
EXPORTS = (
    "gmt_version", "gmt_last_error", "gmt_params_init", "gmt_create", "gmt_destroy", "gmt_kernel_info",
    "gmt_step", "gmt_step_planes", "gmt_cfl_async", "gmt_cfl_result", "gmt_compute_dt", "gmt_diagnostics", "gmt_diagnostics_noalloc",
    "gmt_forcing_reset", "gmt_forcing_advance", "gmt_forcing_set_modes", "gmt_forcing_get_modes",
    "gmt_forcing_counter", "gmt_forcing_get_state", "gmt_forcing_set_state", "gmt_ic_orszag_tang", "gmt_ic_uniform", "gmt_ic_turbulent", "gmt_ct_step", "gmt_ct_cfl_async",
    "gmt_ct_divb_max", "gmt_ct_ic_orszag_tang", "gmt_ke_spectrum", "gmt_run", "gmt_ensemble_create", "gmt_ensemble_destroy",
    "gmt_ensemble_run", "gmt_density_pdf", "gmt_ke_band_loss", "gmt_adjoint_step", "gmt_adjoint_amp_grad",
    "gmt_adjoint_set_passes", "gmt_test_wait_limit", "march_nv", "march_nx", "march_nsp", "march_set_dtdx",
    "march_set_glm", "march_set_gamma", "march_run_dev", "march_set_nx", "ct_run", "ct_regs", "ct_shmem",
)


class GmtParams(C.Structure):
    _fields_ = [("abi_version", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("dtype", C.c_int32), ("scheme", C.c_int32), ("recon", C.c_int32), ("riemann", C.c_int32),
                ("iflo", C.c_int32), ("emf", C.c_int32), ("ct_halfslope", C.c_int32),
                ("tile_x", C.c_int32), ("tile_y", C.c_int32), ("tile_z", C.c_int32), ("nsp", C.c_int32),
                ("boxlen", C.c_double), ("gamma", C.c_double), ("courant", C.c_double),
                ("smallr", C.c_double), ("smallc", C.c_double), ("smallp", C.c_double),
                ("glm_ch_scale", C.c_double), ("glm_cp_coef", C.c_double), ("llf_dmin", C.c_double),
                ("llf_pmin", C.c_double), ("turb_min_rho", C.c_double), ("turb_amp", C.c_double),
                ("turb_T", C.c_double), ("turb_ndt", C.c_int32), ("turb_seed", C.c_uint32)]


class GmtStepArgs(C.Structure):
    _fields_ = [("dt", C.c_double), ("t", C.c_double), ("ch", C.c_double), ("glm_fac", C.c_double),
                ("do_turb", C.c_int32), ("want_cfl", C.c_int32)]


class GmtDiag(C.Structure):
    _fields_ = [("mass", C.c_double), ("ke2", C.c_double), ("vrms", C.c_double), ("divbmax", C.c_double),
                ("rhomin", C.c_double), ("etot", C.c_double), ("divb_l2", C.c_double), ("psi_l2", C.c_double),
                ("finite", C.c_int32), ("nonfinite_cells", C.c_int32)]


class GmtError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"glmmhd_b200 error {code}: {msg}")
        self.code = code


_lib = None


def build(jobs: int = 8) -> str:
    """Compile the library for sm_100a with nvcc (csrc/Makefile)."""
    subprocess.run(["make", "-s", f"-j{jobs}", "-C", CSRC], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {CSRC}` "
                               "(or __graft_entry__.build()); there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        vp, i32, dbl = C.c_void_p, C.c_int32, C.c_double
        P, A = C.POINTER(GmtParams), C.POINTER(GmtStepArgs)
        sig = {
            "gmt_version": ([], C.c_char_p), "gmt_last_error": ([], C.c_char_p),
            "gmt_params_init": ([P, C.c_int], C.c_int), "gmt_create": ([P, C.POINTER(vp)], C.c_int),
            "gmt_destroy": ([vp], C.c_int),
            "gmt_kernel_info": ([vp, C.POINTER(i32), C.POINTER(C.c_int64), C.POINTER(i32)], C.c_int),
            "gmt_step": ([vp, vp, vp, A, vp], C.c_int), "gmt_step_planes": ([vp, vp, vp, A, vp], C.c_int),
            "gmt_cfl_async": ([vp, vp, vp], C.c_int), "gmt_cfl_result": ([vp, C.POINTER(dbl), vp], C.c_int),
            "gmt_compute_dt": ([vp, vp, C.POINTER(dbl), vp], C.c_int),
            "gmt_diagnostics": ([vp, vp, C.POINTER(GmtDiag), vp], C.c_int),
            "gmt_diagnostics_noalloc": ([vp, i32, i32, i32, i32, dbl, dbl, C.POINTER(GmtDiag), vp], C.c_int),
            "gmt_forcing_reset": ([vp, vp], C.c_int), "gmt_forcing_advance": ([vp, vp], C.c_int),
            "gmt_forcing_set_modes": ([vp, C.POINTER(dbl), vp], C.c_int),
            "gmt_forcing_get_modes": ([vp, C.POINTER(dbl), vp], C.c_int),
            "gmt_forcing_counter": ([vp, C.POINTER(C.c_uint32)], C.c_int),
            "gmt_forcing_get_state": ([vp, C.POINTER(dbl), C.POINTER(C.c_uint32), C.POINTER(dbl), vp], C.c_int),
            "gmt_forcing_set_state": ([vp, C.POINTER(dbl), C.c_uint32, dbl, vp], C.c_int),
            "gmt_ic_orszag_tang": ([vp, vp, vp], C.c_int),
            "gmt_ic_uniform": ([vp, vp, dbl, dbl, dbl, dbl, dbl, vp], C.c_int),
            "gmt_ic_turbulent": ([vp, vp, dbl, dbl, dbl, dbl, dbl, dbl, dbl, C.c_uint32, vp], C.c_int),
            "gmt_ct_step": ([vp, vp, vp, A, vp], C.c_int), "gmt_ct_cfl_async": ([vp, vp, vp], C.c_int),
            "gmt_ct_divb_max": ([vp, vp, C.POINTER(dbl), vp], C.c_int),
            "gmt_ct_ic_orszag_tang": ([vp, vp, vp], C.c_int),
            "gmt_ke_spectrum": ([vp, vp, i32, C.POINTER(dbl), vp], C.c_int),
            "gmt_ke_band_loss": ([vp, vp, i32, i32, C.POINTER(dbl), vp, vp], C.c_int),
            "gmt_density_pdf": ([vp, vp, i32, dbl, dbl, C.POINTER(dbl), C.POINTER(dbl), vp], C.c_int),
            "gmt_adjoint_step": ([vp, vp, vp, vp, A, vp], C.c_int),
            "gmt_adjoint_amp_grad": ([vp, C.POINTER(dbl), i32, vp], C.c_int),
            "gmt_adjoint_set_passes": ([vp, i32], C.c_int),
            "gmt_test_wait_limit": ([vp, C.c_int64, i32], C.c_int),
            "gmt_run": ([vp, vp, vp, i32, dbl, dbl, i32, vp, C.POINTER(dbl), C.POINTER(i32)], C.c_int),
            "gmt_ensemble_create": ([P, i32, C.POINTER(i32), C.POINTER(dbl), C.POINTER(C.c_uint32), C.POINTER(vp)],
                                    C.c_int),
            "gmt_ensemble_destroy": ([vp], C.c_int),
            "gmt_ensemble_run": ([vp, vp, vp, i32, dbl, i32, vp, C.POINTER(dbl)], C.c_int),
            "march_nv": ([], C.c_int), "march_nx": ([], C.c_int), "march_nsp": ([], C.c_int),
            "march_set_dtdx": ([C.c_float], None), "march_set_glm": ([C.c_float, C.c_float], None),
            "march_set_gamma": ([C.c_float], None), "march_set_nx": ([C.c_int], None),
            "march_run_dev": ([vp, vp, C.c_int], C.c_double),
            "ct_run": ([vp, vp, vp, C.c_int], C.c_double), "ct_regs": ([], C.c_int), "ct_shmem": ([], C.c_int),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def check(rc: int):
    if rc != GMT_OK:
        raise GmtError(rc, lib().gmt_last_error().decode())


def version() -> str:
    return lib().gmt_version().decode()
