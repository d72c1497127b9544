"""Checkpoints of a GLM state and the spin-up generator of pre-evolved turbulent states.

The reference writes no files (its state lives only in device memory).  A checkpoint here is one
file: an 8-byte magic, an 8-byte header length, a JSON header (shape, dtype, time, step, forcing
counter and next update time, the parameters), the 61x3x2 forcing mode amplitudes (FP64), then
the raw SoA state -- 9 planes of nx*ny*nz reals, x fastest, the memory image of the reference's
(N,N,N,9) array -- so the body can also be memory-mapped by other tools.
"""
from __future__ import annotations

import json
import math
import struct

import numpy as np
import torch

from .solver import Solver

MAGIC = b"GMTCKPT1"
_DT = {"float32": (torch.float32, np.float32), "float64": (torch.float64, np.float64)}


def save(path: str, u: torch.Tensor, *, t: float = 0.0, step: int = 0, solver: Solver | None = None,
         extra: dict | None = None) -> None:
    """Write state `u` (nvar, nz, ny, nx) and, when `solver` is given, its forcing state."""
    u_host = u.detach().contiguous().cpu().numpy()
    fs = solver.forcing_state() if solver is not None else {"modes": np.zeros((61, 3, 2)), "counter": 0,
                                                              "next_time": 0.0}
    modes = fs["modes"]
    header = {"version": 1, "shape": list(u_host.shape), "dtype": str(u_host.dtype), "t": float(t),
              "step": int(step), "forcing_counter": int(fs["counter"]), "next_time": float(fs["next_time"]),
              "extra": extra or {}}
    if solver is not None:
        p = solver.params
        header["params"] = {k: getattr(p, k) for k, _ in p._fields_}
    hb = json.dumps(header).encode()
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<Q", len(hb)))
        f.write(hb)
        f.write(np.ascontiguousarray(modes, dtype=np.float64).tobytes())
        f.write(u_host.tobytes())


def load(path: str, device="cuda"):
    """Return (state tensor on `device`, header dict with 'modes')."""
    with open(path, "rb") as f:
        if f.read(8) != MAGIC:
            raise ValueError(f"{path} is not a checkpoint")
        (n,) = struct.unpack("<Q", f.read(8))
        header = json.loads(f.read(n))
        header["modes"] = np.frombuffer(f.read(61 * 6 * 8), dtype=np.float64).reshape(61, 3, 2).copy()
        tdt, ndt = _DT[header["dtype"]]
        count = int(np.prod(header["shape"]))
        data = np.frombuffer(f.read(count * np.dtype(ndt).itemsize), dtype=ndt)
    if data.size != count:
        raise ValueError(f"{path} is truncated")
    u = torch.from_numpy(data.reshape(header["shape"]).copy()).to(device)
    return u, header


def restore_forcing(solver: Solver, header: dict) -> None:
    """Put a checkpoint's forcing modes, counter and next update time back into `solver`."""
    solver.set_forcing_state({"modes": header["modes"], "counter": header["forcing_counter"],
                              "next_time": header["next_time"]})


def prolong(u: torch.Tensor) -> torch.Tensor:
    """Conserved state on the grid twice as fine: each cell's values in its 2x2x2 children (exact
    conservation of mass, momentum, energy and field)."""
    return u.repeat_interleave(2, dim=1).repeat_interleave(2, dim=2).repeat_interleave(2, dim=3).contiguous()


def spinup_levels(n: int, *, seed: int = 1, amp: float = 2.0, mach_target: float = 1.0, n0: int = 64,
                  mach_coarse: float = 0.95, dt_level: float = 0.03, t_max: float = 5.0, dtype: str = "f32",
                  chunk: int = 50, gamma: float = 5.0 / 3.0, courant: float = 0.3, b0: float = 0.775,
                  p0: float = 0.6, tile=(0, 0, 0)):
    """The forced spin-up of `spinup`, run on a ladder of grids so that a large box costs seconds:
    from the uniform state on n0^3 until the rms Mach number reaches mach_coarse * mach_target;
    then each finer grid (2 n0, 4 n0, ..., n) takes the prolonged state and the forcing state
    (modes, OU counter, next update time: the forcing is a mode sum, the same on every grid) and runs
    for at least dt_level of simulated time; the final grid runs until the rms Mach number reaches
    mach_target.  Returns (state, t, info, solver) with info = [(grid, t_end, steps, mach)]."""
    if n < n0 or n % n0 != 0 or (n // n0) & (n // n0 - 1):
        raise ValueError("n must be n0 times a power of two")
    cs = math.sqrt(gamma * p0)
    info = []
    t, fstate, u, s = 0.0, None, None, None
    m = n0
    while True:
        final = m == n
        s = Solver(m, dtype=dtype, gamma=gamma, courant=courant, turb_amp=amp, turb_T=0.5, turb_ndt=100,
                   turb_seed=seed, tile=tile if final else (0, 0, 0))
        w = s.alloc()
        if u is None:
            u = s.alloc()
            s.ic_uniform(u, 1.0, p0, (b0, 0.0, 0.0))
            s.forcing_reset()
        else:
            u = prolong(u)
            s.set_forcing_state(fstate)
        t_start, steps = t, 0
        target = mach_target if final else (mach_coarse * mach_target if m == n0 else 0.0)
        while t < t_max:
            t, res = s.run(u, w, chunk, t0=t, t_end=t_max, forcing=True, ch_max_signal=True)
            steps += chunk
            if res is w:
                u, w = w, u
            mach = s.diagnostics(u)["vrms"] / cs
            if mach >= target and (m == n0 or t - t_start >= dt_level):
                break
        info.append((m, t, steps, mach))
        fstate = s.forcing_state()
        if final:
            return u, t, info, s
        del w
        m *= 2


def spinup(n: int, *, seed: int = 1, amp: float = 2.0, mach_target: float = 1.0, t_max: float = 5.0,
           dtype: str = "f32", chunk: int = 50, gamma: float = 5.0 / 3.0, courant: float = 0.3,
           b0: float = 0.775, p0: float = 0.6):
    """Drive the uniform state (rho 1, p p0, B (b0,0,0)) with the OU forcing of `seed` until the
    rms Mach number reaches `mach_target` (or t_max); returns (state, t, steps, solver)."""
    s = Solver(n, dtype=dtype, gamma=gamma, courant=courant, turb_amp=amp, turb_T=0.5, turb_ndt=100, turb_seed=seed)
    u, w = s.alloc(), s.alloc()
    s.ic_uniform(u, 1.0, p0, (b0, 0.0, 0.0))
    s.forcing_reset()
    t, steps = 0.0, 0
    cs = math.sqrt(gamma * p0)
    while t < t_max:
        t, res = s.run(u, w, chunk, t0=t, t_end=t_max, forcing=True, ch_max_signal=True)
        steps += chunk
        if res is w:
            u, w = w, u
        mach = s.diagnostics(u)["vrms"] / cs
        if mach >= mach_target:
            break
    return u, t, steps, s
