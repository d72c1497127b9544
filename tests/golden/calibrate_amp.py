"""Calibrate the forcing amplitude of the 64^3 parity configuration with the CPU oracle.

The configuration: 3-D periodic GLM-MHD on a 64^3 unit box, gamma = 5/3, rho = 1, v = 0, p = 0.6
(c_s = 1), B0 = (0.775, 0, 0), psi = 0; PLM-MC + MUSCL-Hancock + HLLD; ch = the global max signal
speed, glm_fac = exp(-ch dt / 0.18); the library's OU forcing (61 solenoidal modes, 1 <= |k| <= 3,
correlation time tau = 0.5, seed 0) with "amplitude tuned so rms Mach reaches ~1"; CFL 0.3.

Procedure: run the FP64 oracle from that state with forcing amplitude A up to t_cal = 2 tau = 1.0 (two
correlation times, the span the reference's turbulence driver runs: t_end = 0.6 at turb_T = 0.3,
glmmhd_turb.jl:2191-2230) and measure the mass-weighted rms Mach number sqrt(<rho v^2>/<rho>)/c_s.
Bisect A (on log A, secant steps inside the bracket) until |Mach - 1| <= 0.01.  The result is written
to amp_calibration.json beside this file; the parity tests and bench.py use its amplitude.

    python tests/golden/calibrate_amp.py [threads]
"""
import json
import math
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
N = (64, 64, 64)
TAU, T_CAL, SEED, COURANT, CP = 0.5, 1.0, 0, 0.3, 0.18


def mach_at(amp, t_cal=T_CAL):
    """rms Mach at t_cal of the forced run with amplitude amp (and the steps taken)."""
    cfg = O.Config(n=N, gamma=5 / 3, recon="mc", riemann="hlld", iflo=True)
    u = O.ic_uniform(cfg, 1.0, 0.6, (0.775, 0.0, 0.0))
    f = O.OUForcing(amp=amp, T=TAU, ndt=100, seed=SEED)
    f.advance()
    t, steps = 0.0, 0
    while t < t_cal:
        while t >= f.next_time:
            f.advance()
        cmax, smax = O.cfl(cfg, u)
        dt = min(COURANT * cfg.dx / cmax, f.next_time - t, t_cal - t)
        fac = math.exp(-(smax / CP) * dt)
        u = O.step_unsplit(cfg, u, dt, smax, fac, ramp=min(t / TAU, 1.0), modes=f.modes)
        t += dt
        steps += 1
    d = O.diagnostics(cfg, u)
    assert d["finite"]
    return d["vrms"] / 1.0, steps


def calibrate(lo=0.5, hi=8.0, tol=0.01, maxit=12):
    hist = []
    mlo, s = mach_at(lo)
    hist.append((lo, mlo, s))
    mhi, s = mach_at(hi)
    hist.append((hi, mhi, s))
    print(hist, flush=True)
    assert mlo < 1.0 < mhi, hist
    a, m = hi, mhi
    for _ in range(maxit):
        # secant on log A against Mach, kept inside the bracket
        x = math.log(lo) + (1.0 - mlo) * (math.log(hi) - math.log(lo)) / (mhi - mlo)
        x = min(max(x, math.log(lo) + 0.1 * (math.log(hi) - math.log(lo))),
                math.log(hi) - 0.1 * (math.log(hi) - math.log(lo)))
        a = math.exp(x)
        m, s = mach_at(a)
        hist.append((a, m, s))
        print(hist[-1], flush=True)
        if abs(m - 1.0) <= tol:
            break
        if m < 1.0:
            lo, mlo = a, m
        else:
            hi, mhi = a, m
    return a, m, hist


if __name__ == "__main__":
    if len(sys.argv) > 1:
        O.set_threads(int(sys.argv[1]))
    t0 = time.time()
    amp, mach, hist = calibrate()
    out = {"amp": round(amp, 4), "mach_at_t_cal": mach, "t_cal": T_CAL, "tau": TAU, "seed": SEED, "n": N,
           "courant": COURANT, "tol": 0.01,
           "history": [{"amp": a, "mach": m, "steps": s} for a, m, s in hist], "cpu_seconds": time.time() - t0}
    json.dump(out, open(os.path.join(HERE, "amp_calibration.json"), "w"), indent=1)
    print(json.dumps(out, indent=1))
