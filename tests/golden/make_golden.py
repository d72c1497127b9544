"""Generate the golden step fixtures in tests/golden/ from the CPU oracle.

The reference ships no golden vectors (its checks are printed Orszag-Tang scalars, pinned
separately in tests/test_oracle.py).  These fixtures freeze FP64 oracle steps, so that the oracle
(CPU tests) and the GPU kernels (-m gpu tests) are checked against the same committed numbers:

  steps_8cube.npz     one step of a smooth seeded 8x8x8 state for every scheme variant;
  edge_16x16x8.npz    one step of a 16x16x8 state built so that every guarded branch of the
                      reference fires (edge_state / ct_edge_state below), with the oracle's branch
                      counts of each case.

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


def calibrated_amp():
    """The forcing amplitude of the 64^3 parity configuration (amp_calibration.json, written by
    calibrate_amp.py: rms Mach 1 at t = 2 tau with the FP64 oracle)."""
    import json
    return float(json.load(open(os.path.join(HERE, "amp_calibration.json")))["amp"])


def forcing_modes():
    f = O.OUForcing(amp=3.0, T=0.5, ndt=100, seed=0)
    for _ in range(3):
        f.advance()
    return f.modes


def cfg_of(case):
    name, scheme, recon, riem, iflo, emf, half, turb = case
    return O.Config(n=N, gamma=GAMMA, recon=recon, riemann=riem, iflo=iflo, emf=emf or "average",
                    ct_halfslope=half, smallp=1e-6)


# ---------------------------------------------------------------------------------------------
# Edge-case fixtures: states on which the reference's guarded branches fire.
#   void ball      near-vacuum (rho a few smallr, p log-uniform from below pfl up to 1e-10, weak
#                  field) with a radial outflow of speed 3: the unsplit predictor revert
#                  (glmmhd_turb.jl:393-395), the interface-state revert iflo (:618), the void
#                  floor of the update (:450-453), the LLF switch on llf_dmin (:287-289) and the
#                  march / CT face and predictor floors (spike_mhd.cu:149-161, 199-223);
#   shear band     p ~ 1e-6 with Mach ~ 2000 random velocities: pressure reverts and the LLF
#                  switch on llf_pmin;
#   aligned slab   uniform field-aligned flow with B = (1.5, 0, 0) (Alfven speed above the sound
#                  speed): the degenerate HLLD star state |denK| < 1e-12 on x faces (:225-238).
# Feature positions are fractions of the box, so the same state scales to any grid (the GPU tests
# build it at sizes whose tiles stage by TMA).
# ---------------------------------------------------------------------------------------------
EDGE_N = (16, 16, 8)
EDGE_SMALLR_CT = 1e-3      # CT: a higher density floor keeps the void's Alfven speed (B0 = 1) moderate
LLF_DMIN, LLF_PMIN = 0.05, 0.01


def edge_state(n, seed=0, gamma=GAMMA, smallr=1e-6):
    nx, ny, nz = n
    z, y, x = np.meshgrid((np.arange(nz) + 0.5) / nz, (np.arange(ny) + 0.5) / ny, (np.arange(nx) + 0.5) / nx,
                          indexing="ij")
    rng = np.random.default_rng(seed)
    rho = 1.0 + 0.1 * rng.random(x.shape)
    p = 0.6 * (1.0 + 0.05 * rng.random(x.shape))
    v = 0.05 * rng.standard_normal((3,) + x.shape)
    B = np.zeros((3,) + x.shape)
    B[0] = 0.775
    B += 0.03 * rng.standard_normal(B.shape)
    psi = 0.01 * rng.standard_normal(x.shape)
    for cx, cy, cz in ((0.5, 0.5, 0.5), (0.0, 0.0, 0.5)):          # two void balls
        ddx, ddy, ddz = ((x - cx + 0.5) % 1.0 - 0.5, (y - cy + 0.5) % 1.0 - 0.5, (z - cz + 0.5) % 1.0 - 0.5)
        r = np.sqrt(ddx ** 2 + ddy ** 2 + ddz ** 2)
        m = r < 0.22
        k = int(m.sum())
        rho[m] = smallr * 10.0 ** rng.uniform(-0.2, 1.0, k)
        p[m] = 10.0 ** rng.uniform(-16.0, -10.0, k)
        B[:, m] = 1e-4 * rng.standard_normal((3, k))
        psi[m] = 0.0
        for a, d in enumerate((ddx, ddy, ddz)):
            v[a][m] = 3.0 * d[m] / np.maximum(r[m], 1e-3)
    band = np.abs(y - 0.25) < 0.08                                    # low-pressure shear band
    p[band] = 1e-6 * (1.0 + rng.random(int(band.sum())))
    v[0][band] = 2.0 * rng.standard_normal(int(band.sum()))
    v[1][band] = 2.0 * rng.standard_normal(int(band.sum()))
    slab = (np.abs(y - 0.75) < 0.1) & (np.abs(z - 0.25) < 0.2)       # field-aligned slab
    rho[slab] = 1.0
    p[slab] = 0.3
    v[:, slab] = 0.0
    v[0][slab] = 0.2
    B[0][slab] = 1.5
    B[1][slab] = 0.0
    B[2][slab] = 0.0
    psi[slab] = 0.0
    u = np.zeros((9, nz, ny, nx))
    u[0] = rho
    u[1:4] = rho * v
    u[5:8] = B
    u[8] = psi
    u[4] = p / (gamma - 1) + 0.5 * rho * (v ** 2).sum(0) + 0.5 * (B ** 2).sum(0)
    return u


def ct_edge_state(n, seed=0, gamma=GAMMA, smallr=EDGE_SMALLR_CT):
    """edge_state's hydro fields with a face field B = (1, 0, 0) + curl(Az(x, y) z), Az vanishing on
    the aligned slab's rows: discretely divergence-free, field-aligned on the slab."""
    nx, ny, nz = n
    u = edge_state(n, seed, gamma, smallr)
    rho = u[0]
    v = u[1:4] / rho
    p = (gamma - 1) * (u[4] - 0.5 * rho * (v ** 2).sum(0) - 0.5 * (u[5:8] ** 2).sum(0))
    X, Y = np.meshgrid(np.arange(nx) / nx, np.arange(ny) / ny, indexing="xy")   # edge (i-1/2, j-1/2)
    w = np.where(np.abs(Y + 0.5 / ny - 0.75) < 0.15, 0.0, 1.0)
    Az = 0.02 * np.sin(2 * np.pi * X) * np.sin(4 * np.pi * Y) * w
    q = np.zeros((8, nz, ny, nx))
    q[5] = (1.0 + (np.roll(Az, -1, axis=0) - Az) * nx)[None]      # Bx(i-1/2, j) = dAz/dy
    q[6] = (-(np.roll(Az, -1, axis=1) - Az) * nx)[None]           # By(i, j-1/2) = -dAz/dx
    bc = np.stack([0.5 * (q[5] + np.roll(q[5], -1, axis=2)), 0.5 * (q[6] + np.roll(q[6], -1, axis=1)),
                   0.5 * (q[7] + np.roll(q[7], -1, axis=0))])
    q[0] = rho
    q[1:4] = rho * v
    q[4] = p / (gamma - 1) + 0.5 * rho * (v ** 2).sum(0) + 0.5 * (bc ** 2).sum(0)
    return q


# (name, scheme, recon, riemann, iflo, emf, forcing, llf switch, branches that must fire)
_GLM_BRANCHES = ("hancock_revert", "void_floor", "hlld_degen", "hlld_L", "hlld_Ls", "hlld_Rs", "hlld_R")
EDGE_CASES = [
    ("edge_mc_hlld_sw", "unsplit", "mc", "hlld", True, None, True, True, _GLM_BRANCHES + ("iflo_revert", "llf_switch")),
    ("edge_mc_hlld", "unsplit", "mc", "hlld", True, None, False, False, _GLM_BRANCHES + ("iflo_revert",)),
    ("edge_mc_hlld_noiflo", "unsplit", "mc", "hlld", False, None, False, False, _GLM_BRANCHES),
    ("edge_mc_hll", "unsplit", "mc", "hll", True, None, True, False, ("hancock_revert", "iflo_revert", "void_floor")),
    ("edge_minmod_hlld_sw", "unsplit", "minmod", "hlld", True, None, False, True, _GLM_BRANCHES + ("llf_switch",)),
    ("edge_minmod_hll", "unsplit", "minmod", "hll", True, None, False, False, ("hancock_revert", "void_floor")),
    ("edge_ppm_hlld_sw", "unsplit", "ppm", "hlld", True, None, True, True,
     _GLM_BRANCHES + ("iflo_revert", "llf_switch", "ppm_fallback")),
    ("edge_ppm_hll", "unsplit", "ppm", "hll", True, None, False, False,
     ("hancock_revert", "iflo_revert", "void_floor", "ppm_fallback")),
    ("edge_march_plm", "march1d", "mc", "hll", False, None, False, False, ("face_floor", "pred1d_floor")),
    ("edge_march_ppm", "march1d", "ppm", "hll", False, None, False, False, ("face_floor", "pred1d_floor")),
    ("edge_ct_plm_hlld_contact", "ct", "mc", "hlld", False, "contact", True, False,
     ("void_floor", "face_floor", "pred1d_floor", "hlld_degen", "hlld_L", "hlld_Ls", "hlld_Rs", "hlld_R")),
    ("edge_ct_ppm_hll_avg", "ct", "ppm", "hll", False, "average", False, False, ("void_floor", "face_floor", "pred1d_floor")),
]


def edge_cfg(case, n=EDGE_N):
    name, scheme, recon, riem, iflo, emf, turb, sw, _ = case
    kw = dict(n=n, gamma=GAMMA, recon=recon, riemann=riem, iflo=iflo, emf=emf or "average", smallp=1e-6)
    if sw:
        kw.update(llf_dmin=LLF_DMIN, llf_pmin=LLF_PMIN)
    if scheme == "ct":
        kw.update(smallr=EDGE_SMALLR_CT)
    return O.Config(**kw)


def edge_dt(n=EDGE_N):
    """dt, ch, glm_fac of the edge fixtures: CFL 0.3 of the GLM and CT edge states, ch = the max
    signal speed, glm_fac = exp(-ch dt / 0.18)."""
    cm, sm = O.cfl(O.Config(n=n, gamma=GAMMA), edge_state(n))
    dt = 0.3 * (1.0 / n[0]) / cm
    ctm, _ = O.ct_cfl(O.Config(n=n, gamma=GAMMA, smallr=EDGE_SMALLR_CT), ct_edge_state(n))
    return dt, sm, float(np.exp(-sm * dt / 0.18)), 0.3 * (1.0 / n[0]) / ctm


def edge_step(case, u, dt, ch, fac, ct_dt, modes, n=EDGE_N):
    """One oracle step of an edge case; returns (output, branch counts)."""
    name, scheme, recon, riem, iflo, emf, turb, sw, _ = case
    cfg = edge_cfg(case, n)
    m = modes if turb else None
    with O.branch_counts() as bc:
        if scheme == "unsplit":
            out = O.step_unsplit(cfg, u, dt, ch, fac, RAMP, m)
        elif scheme == "march1d":
            out = O.step_march1d(cfg, u, dt, ch, fac)
        else:
            out = O.ct_step(cfg, u, ct_dt, RAMP, m)
    return out, bc.counts


def compute_edge():
    glm, ct = edge_state(EDGE_N), ct_edge_state(EDGE_N)
    dt, ch, fac, ct_dt = edge_dt(EDGE_N)
    modes = forcing_modes()
    out = {"glm_in": glm, "ct_in": ct, "modes": modes, "scalars": np.array([dt, ch, fac, RAMP, GAMMA, ct_dt])}
    for case in EDGE_CASES:
        res, counts = edge_step(case, ct if case[1] == "ct" else glm, dt, ch, fac, ct_dt, modes)
        out[case[0]] = res
        out[case[0] + "__counts"] = np.array([counts[k] for k in O.COUNTERS], dtype=np.int64)
    return out


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
    np.savez_compressed(os.path.join(HERE, "edge_16x16x8.npz"), **compute_edge())
    print("wrote", os.path.join(HERE, "edge_16x16x8.npz"))
