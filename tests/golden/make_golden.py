"""Generate the golden step fixtures in tests/golden/ from the CPU oracle.

The reference ships no golden vectors (its checks are printed Orszag-Tang scalars, pinned
separately in tests/test_oracle.py).  These fixtures freeze one FP64 oracle step of a seeded
8x8x8 state for every scheme variant, so that the oracle (CPU tests) and the GPU kernels
(-m gpu tests) are checked against the same committed numbers.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
N = (8, 8, 8)
GAMMA = 5.0 / 3.0
DT, CH, FAC, RAMP = 2.0e-3, 1.7, 0.97, 0.3

# (name, scheme, recon, riemann, iflo, emf, halfslope, forcing)
CASES = [
    ("unsplit_mc_hlld_iflo", "unsplit", "mc", "hlld", True, None, False, True),
    ("unsplit_mc_hlld", "unsplit", "mc", "hlld", False, None, False, False),
    ("unsplit_mc_hll", "unsplit", "mc", "hll", True, None, False, True),
    ("unsplit_mc_llf", "unsplit", "mc", "llf", True, None, False, False),
    ("unsplit_minmod_llfb", "unsplit", "minmod", "llf_bound", True, None, False, False),
    ("unsplit_ppm_hll", "unsplit", "ppm", "hll", True, None, False, True),
    ("unsplit_ppm_hlld", "unsplit", "ppm", "hlld", True, None, False, False),
    ("march_plm", "march1d", "mc", "hll", False, None, False, False),
    ("march_ppm", "march1d", "ppm", "hll", False, None, False, False),
    ("ct_plm_hll_avg", "ct", "mc", "hll", False, "average", False, False),
    ("ct_plm_hlld_contact", "ct", "mc", "hlld", False, "contact", False, True),
    ("ct_ppm_hll_contact", "ct", "ppm", "hll", False, "contact", False, False),
    ("ct_julia_halfslope", "ct", "mc", "hll", False, "average", True, False),
]


def glm_state(seed=0):
    """Orszag-Tang-like smooth state with seeded 3-D perturbations and a psi field."""
    cfg = O.Config(n=N, gamma=GAMMA)
    u = O.ic_ot(cfg)
    rng = np.random.default_rng(seed)
    u[0] *= 1.0 + 0.1 * rng.random(u[0].shape)
    u[1:4] += 0.05 * rng.standard_normal(u[1:4].shape)
    u[4] *= 1.0 + 0.05 * rng.random(u[4].shape)
    u[7] += 0.03 * rng.standard_normal(u[7].shape)
    u[8] = 0.01 * rng.standard_normal(u[8].shape)
    return u


def ct_state(seed=0):
    cfg = O.Config(n=N, gamma=GAMMA)
    q = O.ct_ic_ot(cfg)
    rng = np.random.default_rng(seed)
    q[0] *= 1.0 + 0.1 * rng.random(q[0].shape)
    q[1:4] += 0.05 * rng.standard_normal(q[1:4].shape)
    return q


def forcing_modes():
    f = O.OUForcing(amp=3.0, T=0.5, ndt=100, seed=0)
    for _ in range(3):
        f.advance()
    return f.modes


def cfg_of(case):
    name, scheme, recon, riem, iflo, emf, half, turb = case
    return O.Config(n=N, gamma=GAMMA, recon=recon, riemann=riem, iflo=iflo, emf=emf or "average",
                    ct_halfslope=half, smallp=1e-6)


def compute():
    out = {"glm_in": glm_state(), "ct_in": ct_state(), "modes": forcing_modes(),
           "scalars": np.array([DT, CH, FAC, RAMP, GAMMA])}
    for case in CASES:
        name, scheme, recon, riem, iflo, emf, half, turb = case
        cfg = cfg_of(case)
        modes = out["modes"] if turb else None
        if scheme == "unsplit":
            out[name] = O.step_unsplit(cfg, out["glm_in"], DT, CH, FAC, RAMP, modes)
        elif scheme == "march1d":
            out[name] = O.step_march1d(cfg, out["glm_in"], DT, CH, FAC)
        else:
            out[name] = O.ct_step(cfg, out["ct_in"], DT, RAMP, modes)
    return out


if __name__ == "__main__":
    np.savez_compressed(os.path.join(HERE, "steps_8cube.npz"), **compute())
    print("wrote", os.path.join(HERE, "steps_8cube.npz"))
