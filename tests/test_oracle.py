"""CPU tests of the oracle: pins against the reference's published numbers, known-answer
vectors of the RNG, forcing definition, and the committed golden fixtures."""
import numpy as np
import pytest

from tests.golden import make_golden as G


def test_orszag_tang_64_hlld_pin(oracle):
    # validate_tiled_ot (glmmhd_turb.jl:2278): N=64, gamma=5/3, courant 0.7, t_end 0.2, HLLD.
    # Published: vrms 0.7887, div.B 2.9 (REPORT.md:24-26; BENCHMARKS.md:179), fp32 on an A6000.
    cfg = oracle.Config(n=(64, 64, 1), gamma=5 / 3, recon="mc", riemann="hlld", iflo=True)
    _, d = oracle.run_ot(cfg, t_end=0.2, courant=0.7)
    assert d["finite"]
    assert abs(d["vrms"] - 0.7887) < 5e-4
    assert abs(d["divbmax"] - 2.9) < 0.1
    assert abs(d["rhomin"] - 0.0835) < 1e-3


def test_orszag_tang_120_ppm_hll_pin(oracle):
    # BENCHMARKS.md:178: N=120 MHD PPM(+HLL): vrms 0.7910, div.B 1.16, rhomin 0.0835
    cfg = oracle.Config(n=(120, 120, 1), gamma=5 / 3, recon="ppm", riemann="hll", iflo=True)
    _, d = oracle.run_ot(cfg, t_end=0.2, courant=0.7)
    assert abs(d["vrms"] - 0.7910) < 5e-4
    assert abs(d["divbmax"] - 1.16) < 0.05
    assert abs(d["rhomin"] - 0.0835) < 1e-3


def test_multikernel_equals_tiled_on_ot(oracle):
    # BENCHMARKS.md:179: tiled (iflo) and multi-kernel paths are identical on OT (no revert fires)
    a = oracle.Config(n=(32, 32, 1), gamma=5 / 3, iflo=True)
    b = oracle.Config(n=(32, 32, 1), gamma=5 / 3, iflo=False)
    ua, _ = oracle.run_ot(a, t_end=0.05)
    ub, _ = oracle.run_ot(b, t_end=0.05)
    assert np.array_equal(ua, ub)


def test_philox_known_answers(oracle):
    # Philox4x32-10 known-answer vectors (Salmon et al., SC'11 / Random123 kat_vectors)
    assert [hex(x) for x in oracle.philox([0, 0, 0, 0], [0, 0])] == \
        ["0x6627e8d5", "0xe169c58d", "0xbc57ac4c", "0x9b00dbd8"]
    assert [hex(x) for x in oracle.philox([0xffffffff] * 4, [0xffffffff] * 2)] == \
        ["0x408f276d", "0x41c83b0e", "0xa20bc7c6", "0x6d5451fd"]
    assert [hex(x) for x in oracle.philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344],
                                          [0xa4093822, 0x299f31d0])] == \
        ["0xd16cfe09", "0x94fdcceb", "0x5001e420", "0x24126ea1"]


def test_mode_table(oracle):
    k = oracle.mode_k()
    k2 = (k ** 2).sum(1)
    assert k.shape == (61, 3) and k2.min() == 1 and k2.max() == 9
    # half space, no +-k duplicates, sorted by kx
    keys = {tuple(r) for r in k}
    assert len(keys) == 61 and not any(tuple(-np.array(r)) in keys for r in k)
    assert (np.diff(k[:, 0]) >= 0).all()
    # all 122 integer vectors with 1 <= |k|^2 <= 9 are covered by +-k
    allk = {(a, b, c) for a in range(-3, 4) for b in range(-3, 4) for c in range(-3, 4) if 1 <= a*a+b*b+c*c <= 9}
    assert len(allk) == 122 and keys | {tuple(-np.array(r)) for r in k} == allk


def test_forcing_is_solenoidal_and_normalised(oracle):
    f = oracle.OUForcing(amp=2.0, T=0.5, ndt=100, seed=3)
    k = oracle.mode_k().astype(float)
    acc = []
    for i in range(2000):
        f.advance()
        if i > 200 and i % 10 == 0:
            m = f.modes
            # k . ahat = 0 (real and imaginary parts)
            assert np.abs(np.einsum("qc,qcr->qr", k, m)).max() < 1e-12
            acc.append(2.0 * (m ** 2).sum())     # <|a|^2> = sum_H 2|ahat|^2
    rms = np.sqrt(np.mean(acc))
    assert 0.8 * 2.0 < rms < 1.2 * 2.0


def test_accel_matches_direct_mode_sum(oracle):
    cfg = oracle.Config(n=(8, 6, 4))
    f = oracle.OUForcing(amp=1.0, seed=1)
    f.advance()
    a = oracle.accel(cfg, f.modes, ramp=0.5)
    k = oracle.mode_k()
    nx, ny, nz = cfg.n
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    z = (np.arange(nz) + 0.5) / nz
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    ref = np.zeros((3, nz, ny, nx))
    for q in range(61):
        th = 2 * np.pi * (k[q, 0] * X + k[q, 1] * Y + k[q, 2] * Z)
        for c in range(3):
            ref[c] += 2 * (f.modes[q, c, 0] * np.cos(th) - f.modes[q, c, 1] * np.sin(th))
    np.testing.assert_allclose(a, 0.5 * ref, atol=1e-13)


def test_fp32_oracle_tracks_fp64(oracle, golden):
    cfg = G.cfg_of(G.CASES[0])
    u = golden["glm_in"]
    r64 = oracle.step_unsplit(cfg, u, G.DT, G.CH, G.FAC, G.RAMP, golden["modes"])
    r32 = oracle.step_unsplit(cfg, u.astype(np.float32), G.DT, G.CH, G.FAC, G.RAMP, golden["modes"])
    for v in range(9):
        scale = max(np.abs(r64[v]).max(), 1e-30)
        assert np.abs(r32[v] - r64[v]).max() / scale < 2e-5


@pytest.mark.parametrize("case", G.CASES, ids=[c[0] for c in G.CASES])
def test_oracle_reproduces_golden(oracle, golden, case):
    fresh = G.compute() if not hasattr(test_oracle_reproduces_golden, "_c") else test_oracle_reproduces_golden._c
    test_oracle_reproduces_golden._c = fresh
    assert np.array_equal(fresh[case[0]], golden[case[0]])


def test_ct_oracle_preserves_divb(oracle):
    cfg = oracle.Config(n=(16, 16, 8), gamma=5 / 3, riemann="hlld", emf="contact")
    q = oracle.ct_ic_ot(cfg)
    rng = np.random.default_rng(1)
    q[1:4] += 0.05 * rng.standard_normal(q[1:4].shape)
    d0 = oracle.ct_divb_max(cfg, q)
    for _ in range(10):
        cmax, _ = oracle.ct_cfl(cfg, q)
        q = oracle.ct_step(cfg, q, 0.3 * cfg.dx / cmax)
    assert d0 < 1e-12 and oracle.ct_divb_max(cfg, q) < 1e-11


def test_conservation_unsplit(oracle, golden):
    cfg = G.cfg_of(G.CASES[1])
    u = golden["glm_in"]
    r = oracle.step_unsplit(cfg, u, G.DT, G.CH, 1.0)
    for v in range(8):   # rho, momentum, E, B conserved by the flux form (psi has no source at fac=1)
        assert abs(r[v].sum() - u[v].sum()) <= 1e-12 * max(np.abs(u[v]).sum(), 1.0)


def _generic_state(O, n, seed):
    """Orszag-Tang plus noise on every field, so no primitive is constant along an axis (a
    limiter kink) at the evaluation point."""
    cfg = O.Config(n=(n, n, n), gamma=5 / 3)
    u = O.ic_ot(cfg)
    rng = np.random.default_rng(seed)
    u[0] *= 1.0 + 0.1 * rng.random(u[0].shape)
    u[1:4] += 0.05 * rng.standard_normal(u[1:4].shape)
    u[4] *= 1.0 + 0.05 * rng.random(u[4].shape)
    u[5:8] += 0.03 * rng.standard_normal(u[5:8].shape)
    u[8] = 0.01 * rng.standard_normal(u[8].shape)
    return u


def test_oracle_jvp_matches_step_and_finite_differences(oracle):
    """The forward-mode tangent step reproduces the FP64 step bit for bit and its directional
    derivative agrees with central differences along a state direction and the amplitude."""
    import math
    O = oracle
    n = 8
    u = _generic_state(O, n, 3)
    cfg = O.Config(n=(n, n, n), gamma=5 / 3, recon="mc", riemann="hlld", iflo=True)
    f = O.OUForcing(amp=2.0, T=0.5, ndt=100, seed=0)
    f.advance()
    cmax, smax = O.cfl(cfg, u)
    dt = 0.3 * cfg.dx / cmax
    fac = math.exp(-(smax / 0.18) * dt)
    kw = dict(ramp=0.4, modes=f.modes)
    rng = np.random.default_rng(4)
    v = rng.standard_normal(u.shape) * np.abs(u).max(axis=(1, 2, 3), keepdims=True)
    v[0] *= 0.1
    v[4] *= 0.1
    out, jv = O.jvp_unsplit(cfg, u, v, dt, smax, fac, **kw)
    np.testing.assert_array_equal(out, O.step_unsplit(cfg, u, dt, smax, fac, **kw))
    eps = 1e-8
    fd = (O.step_unsplit(cfg, u + eps * v, dt, smax, fac, **kw) - O.step_unsplit(cfg, u - eps * v, dt, smax, fac, **kw)) / (2 * eps)
    assert np.abs(fd - jv).max() <= 1e-5 * np.abs(jv).max()
    # amplitude direction: the modes scale with the amplitude
    _, ja = O.jvp_unsplit(cfg, u, None, dt, smax, fac, amp_rel=1.0, **kw)
    ea = 1e-6
    fa = (O.step_unsplit(cfg, u, dt, smax, fac, ramp=0.4, modes=f.modes * (1 + ea)) -
          O.step_unsplit(cfg, u, dt, smax, fac, ramp=0.4, modes=f.modes * (1 - ea))) / (2 * ea)
    assert np.abs(fa - ja).max() <= 1e-5 * np.abs(ja).max()   # FD roundoff ~1e-16/ea
    assert np.abs(ja[[0, 5, 6, 7, 8]]).max() == 0.0   # the kick moves momentum and energy only


def _march_species_state(O, n, nsp, seed):
    cfg = O.Config(n=(n, n, n), gamma=5 / 3, recon="mc", riemann="hll", nsp=nsp)
    u = _generic_state(O, n, seed)
    rng = np.random.default_rng(seed + 100)
    sp = np.empty((nsp,) + u.shape[1:])
    for s in range(nsp):
        sp[s] = u[0] * (0.2 + 0.6 * rng.random(u.shape[1:]))
    return cfg, np.ascontiguousarray(np.concatenate([u, sp])), u


@pytest.mark.parametrize("recon", ["mc", "ppm"])
def test_march_species_cma_properties(oracle, recon):
    """Passive species on the march scheme (spike_mhd.cu NSP, CMA): the MHD planes are untouched by
    the species, sum(rho X) is conserved, and a uniform fraction stays uniform."""
    O = oracle
    n = 8
    cfg, u, u9 = _march_species_state(O, n, 2, 5)
    cfg.recon = recon
    cfg9 = O.Config(n=(n, n, n), gamma=5 / 3, recon=recon, riemann="hll")
    cmax, smax = O.cfl(cfg9, u9)
    dt = 0.3 * cfg.dx / cmax
    out = O.step_march1d(cfg, u, dt, smax, 0.98)
    np.testing.assert_array_equal(out[:9], O.step_march1d(cfg9, u9, dt, smax, 0.98))
    for s in (9, 10):
        assert abs(out[s].sum() - u[s].sum()) <= 1e-12 * np.abs(u[s]).sum()
    # a uniform fraction X = 0.3 stays 0.3
    u[9] = 0.3 * u[0]
    out = O.step_march1d(cfg, u, dt, smax, 0.98)
    X = out[9] / np.maximum(out[0], cfg.smallr)
    assert np.abs(X - 0.3).max() <= 1e-13


# ---------------------------------------------------------------------------------------------
# Edge-case fixtures: every guarded branch of the reference fires in the committed fixture
# ---------------------------------------------------------------------------------------------
@pytest.fixture(scope="module")
def edge():
    import os
    return dict(np.load(os.path.join(os.path.dirname(G.__file__), "edge_16x16x8.npz")))


def test_edge_fixture_states_are_regenerated_exactly(edge):
    assert np.array_equal(G.edge_state(G.EDGE_N), edge["glm_in"])
    assert np.array_equal(G.ct_edge_state(G.EDGE_N), edge["ct_in"])
    assert np.array_equal(np.array(G.edge_dt(G.EDGE_N)), edge["scalars"][[0, 1, 2, 5]])


@pytest.mark.parametrize("case", G.EDGE_CASES, ids=[c[0] for c in G.EDGE_CASES])
def test_edge_golden_and_branch_counts(oracle, edge, case):
    """The oracle reproduces each committed edge-case step bit for bit, with the same branch
    counts, and every branch the case is built for fires at least once."""
    dt, ch, fac, _, _, ct_dt = edge["scalars"]
    src = edge["ct_in"] if case[1] == "ct" else edge["glm_in"]
    out, counts = G.edge_step(case, src, dt, ch, fac, ct_dt, edge["modes"])
    assert np.array_equal(out, edge[case[0]])
    assert [counts[k] for k in oracle.COUNTERS] == list(edge[case[0] + "__counts"])
    for br in case[8]:
        assert counts[br] > 0, (case[0], br, counts)
    assert np.isfinite(out).all()
    cdiv = oracle.ct_divb_max(G.edge_cfg(case), out) if case[1] == "ct" else 0.0
    assert cdiv < 1e-12


def test_edge_iflo_changes_the_step(edge):
    # with the interface-state revert on, the step differs from the one without it
    a, b = edge["edge_mc_hlld"], edge["edge_mc_hlld_noiflo"]
    assert np.abs(a - b).max() > 1e-6


def test_branch_counts_zero_on_a_smooth_state(oracle, golden):
    # the smooth 8^3 fixture state triggers none of the revert / floor branches
    cfg = oracle.Config(n=G.N, gamma=G.GAMMA, recon="mc", riemann="hlld", iflo=True)
    with oracle.branch_counts() as bc:
        oracle.step_unsplit(cfg, golden["glm_in"], G.DT, G.CH, G.FAC)
    for k in ("hancock_revert", "iflo_revert", "void_floor", "llf_switch", "hlld_degen"):
        assert bc.counts[k] == 0, (k, bc.counts)
    assert sum(bc.counts[k] for k in ("hlld_L", "hlld_Ls", "hlld_Rs", "hlld_R")) >= 3 * 512


def test_calibrated_amplitude_is_used_everywhere():
    """The configs' forcing amplitude comes from the committed calibration (rms Mach 1 at t = 2 tau,
    FP64 oracle at 64^3, tests/golden/calibrate_amp.py) and the bench uses the same number."""
    import json
    import os
    cal = json.load(open(os.path.join(os.path.dirname(G.__file__), "amp_calibration.json")))
    assert abs(cal["mach_at_t_cal"] - 1.0) <= cal["tol"]
    assert G.calibrated_amp() == cal["amp"]
    import bench
    assert bench.AMP == cal["amp"]
