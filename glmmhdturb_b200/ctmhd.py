"""Host-side mirror of CTMHD (ct_mhd.jl), backed by libglmmhd_b200.so.

    step(U, bxf, byf, bzf, bccx, bccy, bccz, Fx, Fy, Fz, ex, ey, ez, dt, dx, N)   ct_mhd.jl:174-184
    divB_max(bxf, byf, bzf, dx)                                                  ct_mhd.jl:190-194
    scratch(N)                                                                   ct_mhd.jl:186-188

U is a (5, N, N, N) CUDA tensor [rho, mx, my, mz, E] and bxf/byf/bzf are (N, N, N) lower-face
fields, updated in place like the reference.  The Bcc/F/e scratch arguments are accepted for
signature compatibility; the library keeps its own.  ct_mhd.jl's constants (gamma = 5/3,
SMALLR = SMALLP = 1e-6, HLL, Balsara-Spicer EMF, its slope halving) are the defaults.
"""
from __future__ import annotations

import torch

from .solver import Solver

GAMMA = 5.0 / 3.0
SMALLR = 1e-6
SMALLP = 1e-6

_SOLVERS: dict = {}


def solver(N: int, dtype="f32", *, riemann="hll", recon="mc", emf="average", halfslope=True, boxlen=None,
           dx=None) -> Solver:
    L = boxlen if boxlen is not None else (dx * N if dx is not None else 1.0)
    key = (N, dtype, riemann, recon, emf, halfslope, L, torch.cuda.current_device())
    s = _SOLVERS.get(key)
    if s is None:
        s = Solver(N, dtype=dtype, scheme="ct", recon=recon, riemann=riemann, emf=emf, ct_halfslope=halfslope,
                   gamma=GAMMA, smallr=SMALLR, smallp=SMALLP, boxlen=L)
        _SOLVERS[key] = s
    return s


def scratch(N, dtype=torch.float32, device="cuda"):
    z = lambda *s: torch.zeros(*s, dtype=dtype, device=device)  # noqa: E731
    return (z(N, N, N), z(N, N, N), z(N, N, N), z(8, N, N, N), z(8, N, N, N), z(8, N, N, N),
            z(N, N, N), z(N, N, N), z(N, N, N))


def step(U, bxf, byf, bzf, bccx=None, bccy=None, bccz=None, Fx=None, Fy=None, Fz=None, ex=None, ey=None, ez=None,
         dt=None, dx=None, N=None, **kw):
    """One CT step with fixed dt, in place on (U, bxf, byf, bzf)."""
    if dt is None or dx is None or N is None:
        raise TypeError("step needs dt, dx and N")
    dtype = "f64" if U.dtype == torch.float64 else "f32"
    s = solver(int(N), dtype, dx=float(dx), **kw)
    q = torch.cat([U.reshape(5, -1), bxf.reshape(1, -1), byf.reshape(1, -1), bzf.reshape(1, -1)], 0).contiguous()
    o = torch.empty_like(q)
    s.step(q, o, float(dt))
    U.copy_(o[:5].reshape(U.shape))
    bxf.copy_(o[5].reshape(bxf.shape))
    byf.copy_(o[6].reshape(byf.shape))
    bzf.copy_(o[7].reshape(bzf.shape))


def divB_max(bxf, byf, bzf, dx) -> float:
    """max |(upper - lower face)/dx| summed over dims (ct_mhd.jl:190-194)."""
    d = (torch.roll(bxf, -1, dims=-1) - bxf + torch.roll(byf, -1, dims=-2) - byf + torch.roll(bzf, -1, dims=-3)
         - bzf) / dx
    return float(d.abs().max().double())
