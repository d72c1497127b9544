"""GPU tests of the C ABI's error behaviour and of the reference-named host mirror."""
import ctypes as C

import numpy as np
import pytest
import torch

from tests.golden import make_golden as G
from tests.gpu_util import max_rel_err, perturbed_glm_state, to_dev

pytestmark = pytest.mark.gpu


def test_error_codes_no_hang():
    from glmmhdturb_b200 import GmtError, Solver, _lib
    s = Solver(16, dtype="f32")
    u = s.alloc()
    s.ic_uniform(u)
    with pytest.raises(GmtError) as e:
        s.step(u, u, 1e-3, ch=1.0, glm_fac=1.0)          # in-place is refused
    assert e.value.code == _lib.GMT_ERR_ARG
    w = torch.empty_like(u)
    with pytest.raises(GmtError):
        s.step(u, w, -1.0, ch=1.0, glm_fac=1.0)          # dt <= 0
    with pytest.raises(GmtError):
        s.step(u, w, float("nan"), ch=1.0, glm_fac=1.0)
    with pytest.raises(GmtError):
        Solver((24, 16, 16), tile=(32, 8, 0))            # tile does not divide the grid
    with pytest.raises(TypeError):
        s.step(u.double(), w.double(), 1e-3)
    with pytest.raises(ValueError):
        s.step(u[:5], w[:5], 1e-3)
    with pytest.raises(GmtError):
        Solver(16, scheme="march1d", riemann="hlld")     # the march scheme is HLL only
    # the context still works after the refused calls
    s.step(u, w, 1e-3, ch=1.0, glm_fac=1.0)
    torch.cuda.synchronize()
    assert torch.isfinite(w).all()
    # null pointers through the raw ABI return an error code
    L = _lib.lib()
    a = _lib.GmtStepArgs(1e-3, 0.0, 1.0, 1.0, 0, 0)
    assert L.gmt_step(s._ctx, None, w.data_ptr(), C.byref(a), None) == _lib.GMT_ERR_ARG
    assert L.gmt_step(None, u.data_ptr(), w.data_ptr(), C.byref(a), None) == _lib.GMT_ERR_ARG


def test_turb_mirror_matches_solver(oracle):
    from glmmhdturb_b200 import turb
    p = turb.Params(N=16, gamma=5 / 3, courant=0.5)
    u0 = perturbed_glm_state(oracle, (16, 16, 16), seed=9)
    u = to_dev(u0)
    dt = turb.compute_dt(u, None, p)
    cfg = oracle.Config(n=(16, 16, 16), gamma=5 / 3)
    assert dt == 0.5 * cfg.dx / oracle.cfl(cfg, u0)[0]
    ch, fac = turb.glm_parameters(p, dt)
    w = torch.empty_like(u)
    turb.step_tiled(u, w, None, p, dt, 0.0)
    ref = oracle.step_unsplit(cfg, u0, dt, ch, fac)
    assert max_rel_err(w.cpu().numpy(), ref)[0] <= 1e-12
    turb.step_multi(u, w, None, None, None, None, p, dt, 0.0)
    ref = oracle.step_unsplit(oracle.Config(n=(16, 16, 16), gamma=5 / 3, iflo=False), u0, dt, ch, fac)
    assert max_rel_err(w.cpu().numpy(), ref)[0] <= 1e-12
    turb.step_plm(u, w, None, p, dt, 0.0, riemann="hll", recon="ppm")
    ref = oracle.step_unsplit(oracle.Config(n=(16, 16, 16), gamma=5 / 3, recon="ppm", riemann="hll"), u0, dt, ch, fac)
    assert max_rel_err(w.cpu().numpy(), ref)[0] <= 1e-12
    with pytest.raises(ValueError):
        turb.step_plm(u, w, None, turb.Params(N=16), dt, 0.0, tb=6)   # N % tb != 0, as the reference asserts
    d = turb.diagnostics(u, None, p)
    assert d["finite"] and abs(d["vrms"] - oracle.diagnostics(cfg, u0)["vrms"]) < 1e-13


def test_turb_forcing_mirror(oracle):
    from glmmhdturb_b200 import turb
    p = turb.Params(N=16, gamma=5 / 3, turb_rms=2.0, turb_T=0.5, turb_Ndt=100, turb_seed=0)
    f = turb.Forcing(p, dtype="f64")
    turb.ou_advance(f, p)
    turb.ou_advance(f, p)
    of = oracle.OUForcing(amp=2.0, T=0.5, ndt=100, seed=0)
    of.advance(); of.advance()
    np.testing.assert_allclose(f.modes(), of.modes, rtol=1e-12, atol=1e-14)
    assert abs(f.next_time - of.next_time) < 1e-15
    u0 = oracle.ic_uniform(oracle.Config(n=(16, 16, 16), gamma=5 / 3), 1.0, 0.6, (0.775, 0, 0))
    u = to_dev(u0)
    w = torch.empty_like(u)
    turb.step_tiled(u, w, f, p, 1e-3, 0.2, do_turb=True)
    ch, fac = turb.glm_parameters(p, 1e-3)
    ref = oracle.step_unsplit(oracle.Config(n=(16, 16, 16), gamma=5 / 3), u0, 1e-3, ch, fac, ramp=0.4,
                              modes=f.modes())
    assert max_rel_err(w.cpu().numpy(), ref)[0] <= 1e-12


def test_ctmhd_mirror(oracle):
    from glmmhdturb_b200 import ctmhd
    N = 16
    cfg = oracle.Config(n=(N, N, N), gamma=5 / 3, riemann="hll", emf="average", ct_halfslope=True)
    q0 = oracle.ct_ic_ot(cfg)
    U = to_dev(q0[:5]).float()
    bxf, byf, bzf = (to_dev(q0[5 + i]).float() for i in range(3))
    sc = ctmhd.scratch(N)
    ctmhd.step(U, bxf, byf, bzf, *sc, dt=1e-3, dx=1.0 / N, N=N)
    ref = oracle.ct_step(cfg, q0, 1e-3)
    got = np.concatenate([U.cpu().numpy(), bxf.cpu().numpy()[None], byf.cpu().numpy()[None],
                          bzf.cpu().numpy()[None]])
    assert max_rel_err(got, ref)[0] < 3e-5
    assert ctmhd.divB_max(bxf, byf, bzf, 1.0 / N) < 1e-4


def test_kernel_info_reports_resources():
    from glmmhdturb_b200 import Solver
    info = Solver(64, dtype="f32").kernel_info()
    assert 0 < info["regs"] <= 255 and info["smem"] > 0 and info["tile"][0] * info["tile"][1] <= 512


@pytest.mark.parametrize("scheme,riemann", [("unsplit", "hlld"), ("march1d", "hll"), ("ct", "hlld")])
def test_autotuner_picks_a_valid_tile(tmp_path, monkeypatch, scheme, riemann):
    """The autotuner times tile x z-chunk candidates of each scheme, returns the fastest and caches it."""
    from glmmhdturb_b200 import autotune
    monkeypatch.setattr(autotune, "CACHE", str(tmp_path / "tune.json"))
    tile, ms, res = autotune.tune(32, dtype="f32", scheme=scheme, riemann=riemann, tiles=[(16, 8), (32, 8)],
                                  chunks=[16, 0], reps=1, steps=1)
    assert len(res) >= 2 and ms == min(r[0] for r in res) and ms > 0
    assert tile[0] in (16, 32) and tile[1] == 8
    c = autotune.cached(32, "f32", scheme, "mc", riemann)
    assert c and tuple(c["tile"]) == tuple(tile)
