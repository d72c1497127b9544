"""GPU parity of the CT step, the 1-D Hancock march scheme and the legacy bridge ABI."""
import ctypes as C

import numpy as np
import pytest
import torch

from tests.golden import make_golden as G
from tests.gpu_util import max_rel_err, to_dev

pytestmark = pytest.mark.gpu

MARCH = [c for c in G.CASES if c[1] == "march1d"]
CT = [c for c in G.CASES if c[1] == "ct"]


def _solver(case, dtype, n=G.N, **kw):
    from glmmhdturb_b200 import Solver
    name, scheme, recon, riem, iflo, emf, half, turb = case
    return Solver(n, dtype=dtype, scheme=scheme, recon=recon, riemann=riem, iflo=iflo, emf=emf or "average",
                  ct_halfslope=half, gamma=G.GAMMA, smallp=1e-6, turb_T=1.0, **kw)


@pytest.mark.parametrize("case", MARCH + CT, ids=[c[0] for c in MARCH + CT])
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_golden(golden, case, dtype):
    s = _solver(case, dtype)
    tdt = torch.float64 if dtype == "f64" else torch.float32
    src = golden["ct_in"] if case[1] == "ct" else golden["glm_in"]
    u = to_dev(src, tdt)
    out = torch.empty_like(u)
    if case[7]:
        s.set_modes(golden["modes"])
    s.step(u, out, G.DT, t=G.RAMP, ch=G.CH, glm_fac=G.FAC, do_turb=case[7])
    err, errs = max_rel_err(out.cpu().numpy(), golden[case[0]])
    print(f"{case[0]} {dtype}: max rel err {err:.3e}")
    assert err <= (1e-12 if dtype == "f64" else 3e-5), errs


@pytest.mark.parametrize("n", [(24, 16, 12), (96, 40, 10)])   # the second has TMA-staged tiles
@pytest.mark.parametrize("emf,riem", [("average", "hll"), ("contact", "hlld")])
def test_ct_noncubic_vs_oracle_and_divb(oracle, emf, riem, n):
    from glmmhdturb_b200 import Solver
    cfg = oracle.Config(n=n, gamma=5 / 3, riemann=riem, emf=emf)
    q0 = oracle.ct_ic_ot(cfg)
    rng = np.random.default_rng(3)
    q0[1:4] += 0.05 * rng.standard_normal(q0[1:4].shape)
    s = Solver(n, dtype="f64", scheme="ct", riemann=riem, emf=emf, gamma=5 / 3)
    q = to_dev(q0)
    w = torch.empty_like(q)
    ref = q0
    for _ in range(5):
        cmax, _ = oracle.ct_cfl(cfg, ref)
        dt = 0.3 * cfg.dx / cmax
        ref = oracle.ct_step(cfg, ref, dt)
        s.step(q, w, dt)
        q, w = w, q
    err, errs = max_rel_err(q.cpu().numpy(), ref)
    assert err <= 1e-12, errs
    assert s.ct_divb_max(q) < 1e-11


def test_ct_fp32_divb_roundoff():
    from glmmhdturb_b200 import Solver
    s = Solver(32, dtype="f32", scheme="ct", riemann="hlld", emf="contact", gamma=5 / 3)
    q = s.alloc()
    s.ic_orszag_tang(q)
    w = torch.empty_like(q)
    d0 = s.ct_divb_max(q)
    for _ in range(20):
        dt = 0.3 * s.dx / s.cfl(q)[0]
        s.step(q, w, dt)
        q, w = w, q
    assert s.ct_divb_max(q) < 1e-4 and d0 < 1e-4   # FP32 round-off floor (BENCHMARKS.md:60-62)


def _legacy_planes(src, nvar):
    q = [torch.from_numpy(np.ascontiguousarray(src[v])).float().cuda() for v in range(nvar)]
    o = [torch.zeros_like(x) for x in q]
    return q, o


@pytest.mark.parametrize("nsteps", [1, 2, 3])
def test_march_run_dev_legacy_abi(golden, nsteps):
    """march_run_dev over a host array of device plane pointers (MarchBridge.jl:64-81)."""
    from glmmhdturb_b200 import Solver, march_bridge as MB
    m = MB.open_lib()
    m.h.march_set_nx(G.N[0])
    m = MB.open_lib()
    assert m.NV == 9 and m.N == G.N[0] and m.has_glm
    MB.set_gamma(m, G.GAMMA)
    MB.set_dtdx(m, G.DT / (1.0 / G.N[0]))
    MB.set_glm(m, G.CH, G.FAC)
    q, o = _legacy_planes(golden["glm_in"], 9)
    ms = MB.run(m, q, o, nsteps)
    assert ms >= 0.0
    got = torch.stack(q).cpu().numpy()
    s = Solver(G.N, dtype="f32", scheme="march1d", riemann="hll", gamma=G.GAMMA, smallp=1e-6)
    u = to_dev(golden["glm_in"], torch.float32)
    w = torch.empty_like(u)
    dt = float(np.float32(G.DT / (1.0 / G.N[0]))) * (1.0 / G.N[0])
    for _ in range(nsteps):
        s.step(u, w, dt, ch=float(np.float32(G.CH)), glm_fac=float(np.float32(G.FAC)))
        u, w = w, u
    assert np.array_equal(got, u.cpu().numpy())
    if nsteps == 1:
        err, _ = max_rel_err(got, golden["march_plm"])
        assert err < 3e-5


def test_ct_run_legacy_abi(golden):
    from glmmhdturb_b200 import _lib
    L = _lib.lib()
    L.march_set_nx(G.N[0])
    L.march_set_gamma(C.c_float(G.GAMMA))
    L.march_set_dtdx(C.c_float(G.DT * G.N[0]))
    q, o = _legacy_planes(golden["ct_in"], 8)
    cc = [torch.zeros_like(q[0]) for _ in range(3)]
    arr = lambda xs: C.cast((C.c_void_p * len(xs))(*[x.data_ptr() for x in xs]), C.c_void_p)  # noqa: E731
    ms = L.ct_run(arr(q), arr(o), arr(cc), 1)
    assert ms >= 0.0
    got = torch.stack(q).cpu().numpy()
    err, errs = max_rel_err(got, golden["ct_plm_hll_avg"])
    assert err < 3e-5, errs
    assert L.ct_regs() > 0


@pytest.mark.parametrize("n", [16, 96])
@pytest.mark.parametrize("recon", ["mc", "ppm"])
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_march_passive_species_vs_oracle(oracle, recon, dtype, n):
    """Two passive species on the march scheme (CMA, spike_mhd.cu NSP): FP64 bit-exact against the
    oracle, FP32 within 1e-5 of it; the MHD planes match the species-free (tiled) step; at 16^3
    and at 96^3 (three 32-column tiles of the step, periodic wrap of the 5-point species stencils)."""
    import math
    import numpy as np
    from glmmhdturb_b200 import Solver
    from tests.gpu_util import to_dev
    from tests.test_oracle import _march_species_state
    nsp = 2
    cfg, u, u9 = _march_species_state(oracle, n, nsp, 7)
    cfg.recon = recon
    cfg9 = oracle.Config(n=(n, n, n), gamma=5 / 3, recon=recon, riemann="hll")
    cmax, smax = oracle.cfl(cfg9, u9)
    dt = 0.3 * cfg.dx / cmax
    fac = math.exp(-(smax / 0.18) * dt)
    ref = oracle.step_march1d(cfg, u, dt, smax, fac)
    s = Solver(n, dtype=dtype, scheme="march1d", recon=recon, riemann="hll", gamma=5 / 3, smallp=cfg.smallp, nsp=nsp)
    tdt = torch.float64 if dtype == "f64" else torch.float32
    ud = to_dev(u, tdt)
    out = torch.empty_like(ud)
    s.step(ud, out, dt, ch=smax, glm_fac=fac)
    got = out.cpu().numpy().astype(np.float64)
    if dtype == "f64":
        np.testing.assert_array_equal(got, ref)
    else:
        err, errs = max_rel_err(got, ref)
        assert err <= 1e-5, errs
    # without species the step runs the tiled march kernel: the same MHD planes (bit for bit in FP64;
    # FP32 builds the tiled kernel with fast math)
    s9 = Solver(n, dtype=dtype, scheme="march1d", recon=recon, riemann="hll", gamma=5 / 3, smallp=cfg.smallp)
    o9 = torch.empty_like(ud[:9])
    s9.step(ud[:9].contiguous(), o9, dt, ch=smax, glm_fac=fac)
    if dtype == "f64":
        assert torch.equal(o9, out[:9])
    else:
        err, errs = max_rel_err(o9.cpu().numpy(), ref[:9])
        assert err <= 1e-5, errs


@pytest.mark.parametrize("recon", ["mc", "ppm"])
@pytest.mark.parametrize("n,tile", [((32, 24, 20), (0, 0, 0)), ((32, 32, 16), (16, 8, 5)), ((24, 16, 12), (8, 16, 0)),
                                    ((96, 40, 10), (32, 8, 0))])   # the last has TMA-staged tiles
def test_tiled_march_vs_oracle(oracle, recon, n, tile):
    """The tiled march kernel (one solve per face, z-march) against the oracle on non-cubic grids,
    odd z-chunks and several tiles; FP64 bit-exact, and the fused CFL equals the oracle's."""
    import math
    from glmmhdturb_b200 import Solver
    from tests.gpu_util import perturbed_glm_state
    u0 = perturbed_glm_state(oracle, n, seed=9, gamma=5 / 3)
    cfg = oracle.Config(n=n, gamma=5 / 3, recon=recon, riemann="hll")
    cmax, smax = oracle.cfl(cfg, u0)
    dt = 0.3 * cfg.dx / cmax
    fac = math.exp(-(smax / 0.18) * dt)
    ref = oracle.step_march1d(cfg, u0, dt, smax, fac)
    s = Solver(n, dtype="f64", scheme="march1d", recon=recon, riemann="hll", gamma=5 / 3, smallp=cfg.smallp, tile=tile)
    ud = to_dev(u0)
    out = torch.empty_like(ud)
    s.step(ud, out, dt, ch=smax, glm_fac=fac, want_cfl=True)
    np.testing.assert_array_equal(out.cpu().numpy(), ref)
    assert s.cfl_result() == oracle.cfl(cfg, ref)


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_ct_turbulent_state_is_divergence_free(dtype):
    """The CT turbulent initial state takes face fields from an edge vector potential: face div B
    at round-off, turbulent velocity of the requested Mach number, and CT steps keep div B there."""
    import math
    from glmmhdturb_b200 import Solver
    n = 32
    s = Solver(n, dtype=dtype, scheme="ct", recon="mc", riemann="hlld", emf="contact", gamma=5 / 3, smallp=1e-6)
    q = s.alloc()
    s.ic_turbulent(q, 1.0, 0.6, (0.775, 0.0, 0.0), mach=1.0, db=0.3, seed=3)
    tol = 1e-12 if dtype == "f64" else 2e-5
    assert s.ct_divb_max(q) <= tol
    rho = q[0].double()
    v2 = ((q[1:4].double() / rho) ** 2).sum(0)
    mach = math.sqrt(float(v2.mean())) / math.sqrt(5 / 3 * 0.6)
    assert 0.5 < mach < 2.0
    dbf = (q[5:8].double() - torch.tensor([0.775, 0.0, 0.0], dtype=torch.float64, device=q.device)[:, None, None, None])
    assert 0.05 < float(dbf.pow(2).sum(0).mean().sqrt()) < 1.0
    w = torch.empty_like(q)
    cm, _ = s.cfl(q)
    for _ in range(5):
        s.step(q, w, 0.3 * s.dx / cm, ch=1.0, glm_fac=1.0)
        q, w = w, q
    assert s.ct_divb_max(q) <= 10 * tol and bool(torch.isfinite(q).all())


def _misaligned_like(u0):
    """A float32 copy of u0 whose base address is 4 bytes past a 16-byte boundary: the library
    cannot describe it by a tensor map, so every tile stages by cp.async."""
    big = torch.empty(u0.size + 1, dtype=torch.float32, device="cuda")
    q = big[1:].view(u0.shape)
    q.copy_(torch.from_numpy(np.ascontiguousarray(u0)).float())
    return q


@pytest.mark.parametrize("scheme,recon,riem", [("unsplit", "mc", "hlld"), ("unsplit", "ppm", "hll"),
                                               ("march1d", "mc", "hll"), ("ct", "mc", "hlld"), ("ct", "ppm", "hll")])
def test_fp32_production_tile_vs_oracle(oracle, scheme, recon, riem):
    """The FP32 step kernels specialised at compile time for the 32x16 production tile (the shape
    the autotuner picks at 512^3) against the FP64 oracle on a 128x128x16 grid, three steps; the
    same step with every tile staged by cp.async (a misaligned state) bit for bit; and the same
    FP32 step on a runtime 16x16 tile.  At this size the 32x16 tiles clear of the box edges stage
    by TMA and the others by cp.async."""
    import math
    from glmmhdturb_b200 import Solver
    from tests.gpu_util import perturbed_glm_state
    n = (128, 128, 16)
    if scheme == "ct":
        cfg = oracle.Config(n=n, gamma=5 / 3, recon=recon, riemann=riem, emf="contact")
        u0 = oracle.ct_ic_ot(cfg)
        rng = np.random.default_rng(5)
        u0[1:4] += 0.05 * rng.standard_normal(u0[1:4].shape)
    else:
        cfg = oracle.Config(n=n, gamma=5 / 3, recon=recon, riemann=riem)
        u0 = perturbed_glm_state(oracle, n, seed=11, gamma=5 / 3)
    kw = dict(dtype="f32", scheme=scheme, recon=recon, riemann=riem, gamma=5 / 3)
    if scheme == "ct":
        kw["emf"] = "contact"
    if scheme == "march1d":
        kw["smallp"] = cfg.smallp
    outs = {}
    for tile, misaligned in (((32, 16, 0), False), ((32, 16, 0), True), ((16, 16, 0), False)):
        s = Solver(n, tile=tile, **kw)
        assert s.kernel_info()["tile"][:2] == tile[:2]
        if misaligned:
            q, w = _misaligned_like(u0), _misaligned_like(u0)
        else:
            q = to_dev(u0, torch.float32)
            w = torch.empty_like(q)
        ref = u0
        for _ in range(3):
            if scheme == "ct":
                cmax, _ = oracle.ct_cfl(cfg, ref)
                dt = 0.3 * cfg.dx / cmax
                ref = oracle.ct_step(cfg, ref, dt)
                s.step(q, w, dt)
            else:
                cmax, smax = oracle.cfl(cfg, ref)
                dt = 0.3 * cfg.dx / cmax
                fac = math.exp(-(smax / 0.18) * dt)
                if scheme == "march1d":
                    ref = oracle.step_march1d(cfg, ref, dt, smax, fac)
                else:
                    ref = oracle.step_unsplit(cfg, ref, dt, smax, fac)
                s.step(q, w, dt, ch=smax, glm_fac=fac)
            q, w = w, q
        got = q.cpu().numpy()
        err, errs = max_rel_err(got, ref)
        rel2 = [float(np.linalg.norm(got[v] - ref[v]) / max(np.linalg.norm(ref[v]), 1e-300)) for v in range(8)]
        # the 8 MHD fields to FP32 round-off in the L2 norm; pointwise, a discrete switch (PPM's
        # pressure-jump fallback, a limiter branch) that flips between FP32 and FP64 at a few cells
        # leaves a larger local difference
        assert max(rel2) <= 1e-5 and max(errs[:8]) <= 1e-3, (tile, misaligned, errs, rel2)
        if scheme != "ct":
            assert errs[8] <= 1e-2, (tile, misaligned, errs)
        outs[(tile, misaligned)] = got
    # TMA staging and cp.async staging deliver the same bytes
    np.testing.assert_array_equal(outs[((32, 16, 0), False)], outs[((32, 16, 0), True)])
    err, errs = max_rel_err(outs[((32, 16, 0), False)], outs[((16, 16, 0), False)].astype(np.float64))
    assert max(errs[:8]) <= 1e-5, errs


def _offset_copy(t):
    """The values of t in a buffer one element further on, so that every plane starts 4 bytes off a
    16-byte boundary: the library then stages by cp.async and takes its one-cell-per-thread passes."""
    big = torch.empty(t.numel() + 4, dtype=t.dtype, device=t.device)
    v = big[1:1 + t.numel()].view(t.shape)
    v.copy_(t)
    assert v.data_ptr() % 16 != 0
    return v


def test_fp32_quad_passes_match_one_cell_passes():
    """In FP32 the CT edge and face passes and the species pass run four cells per thread when every
    plane is 16-byte aligned (and nx is a multiple of 4); misaligned planes take the one-cell
    passes.  CT: bit-identical.  Species: equal up to the last bit of the fraction divisions."""
    from glmmhdturb_b200 import Solver
    n = (64, 32, 16)
    s = Solver(n, dtype="f32", scheme="ct", recon="mc", riemann="hlld", emf="contact", gamma=5 / 3, turb_amp=2.0,
               turb_T=0.5)
    q = s.alloc()
    s.ic_turbulent(q, mach=1.0, seed=3)
    s.forcing_advance()
    a = torch.empty_like(q)
    s.step(q, a, 1e-4, t=0.2, do_turb=True)
    qm = _offset_copy(q)
    am = _offset_copy(torch.zeros_like(q))
    s.step(qm, am, 1e-4, t=0.2, do_turb=True)
    torch.cuda.synchronize()
    assert torch.equal(a, am)

    nsp = 2
    m = Solver(n, dtype="f32", scheme="march1d", recon="mc", riemann="hll", gamma=5 / 3, nsp=nsp)
    u = m.alloc()
    g = Solver(n, dtype="f32", gamma=5 / 3)
    u9 = g.alloc()
    g.ic_turbulent(u9, 1.0, 0.6, (0.775, 0.0, 0.0), mach=1.0, db=0.1, seed=4)
    u.zero_()
    u[:9] = u9
    x = torch.arange(n[0], device="cuda", dtype=torch.float32)
    u[9] = u9[0] * (0.3 + 0.2 * torch.sin(0.4 * x))
    u[10] = u9[0] * (0.7 - 0.2 * torch.sin(0.4 * x))
    cm, sm = m.cfl(u)
    dt = 0.3 * m.dx / cm
    w = torch.empty_like(u)
    m.step(u, w, dt, ch=sm, glm_fac=0.99)
    um = _offset_copy(u)
    wm = _offset_copy(torch.zeros_like(u))
    m.step(um, wm, dt, ch=sm, glm_fac=0.99)
    torch.cuda.synchronize()
    assert torch.equal(w[:9], wm[:9])
    d = (w[9:] - wm[9:]).abs().max().item()
    assert d <= 1e-6 * w[9:].abs().max().item(), d


def test_fp32_ct_cfl_quad_pass_matches_one_cell_pass():
    """The FP32 CT CFL reduction (cell-centred field from the face field) reads four cells per
    thread on aligned planes and one cell per thread otherwise; the maxima are equal."""
    from glmmhdturb_b200 import Solver
    n = (64, 32, 16)
    s = Solver(n, dtype="f32", scheme="ct", recon="mc", riemann="hlld", emf="contact", gamma=5 / 3)
    q = s.alloc()
    s.ic_turbulent(q, mach=1.5, seed=5)
    a = s.cfl(q)
    b = s.cfl(_offset_copy(q))
    assert a == b and a[0] > 0.0
