"""Host-side mirror of MarchBridge (march_bridge/MarchBridge.jl) over libglmmhd_b200.so.

    open_lib(path) -> Lib(NV, N)      MarchBridge.jl:34-42 (dlopen + march_nv/march_nx)
    close_lib(m)                      :44
    set_dtdx(m, v)                    :47
    set_glm(m, ch, glmfac)            :51-54
    set_gamma(m, g)                   :58-62
    run(m, q, o, nsteps) -> ms        :73-81 (float** of device addresses, result left in q)

q and o are lists of NV float32 CUDA tensors of N^3 cells; like the Julia bridge, `run` passes
a host array of device addresses through the C ABI.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import _lib


@dataclass
class Lib:
    h: C.CDLL
    NV: int
    N: int
    has_glm: bool


def open_lib(path: str | None = None) -> Lib:
    L = C.CDLL(path) if path else _lib.lib()
    if path:
        L.march_nv.restype = C.c_int
        L.march_nx.restype = C.c_int
        L.march_run_dev.restype = C.c_double
        L.march_run_dev.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.march_set_dtdx.argtypes = [C.c_float]
        L.march_set_glm.argtypes = [C.c_float, C.c_float]
        L.march_set_gamma.argtypes = [C.c_float]
    has_glm = hasattr(L, "march_set_glm")
    return Lib(L, int(L.march_nv()), int(L.march_nx()), has_glm)


def close_lib(m: Lib):
    pass


def set_dtdx(m: Lib, v: float):
    """Set the kernel's fixed dt/dx."""
    m.h.march_set_dtdx(C.c_float(v))


def set_glm(m: Lib, ch: float, glmfac: float):
    """Set the Dedner cleaning speed ch and the per-step psi factor glmfac."""
    if not m.has_glm:
        raise RuntimeError(f"this lib (NV={m.NV}) has no march_set_glm -- not a GLM-MHD build")
    m.h.march_set_glm(C.c_float(ch), C.c_float(glmfac))


def set_gamma(m: Lib, g: float):
    m.h.march_set_gamma(C.c_float(g))


def _addrs(planes):
    return (C.c_void_p * len(planes))(*[p.data_ptr() for p in planes])


def run(m: Lib, q, o, nsteps: int) -> float:
    """Run nsteps periodic marches; the result is left in q.  Returns kernel ms (CUDA events)."""
    if not (len(q) == m.NV == len(o)):
        raise AssertionError(f"expected {m.NV} SoA planes")
    for x in list(q) + list(o):
        if tuple(x.shape) != (m.N, m.N, m.N) or not x.is_cuda or not x.is_contiguous():
            raise AssertionError(f"planes must be contiguous {m.N}^3 CUDA tensors")
    qa, oa = _addrs(q), _addrs(o)
    return float(m.h.march_run_dev(C.cast(qa, C.c_void_p), C.cast(oa, C.c_void_p), int(nsteps)))
