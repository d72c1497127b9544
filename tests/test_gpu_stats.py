"""GPU tests of the kinetic-energy spectrum, checkpoints and the spin-up generator."""
import numpy as np
import pytest
import torch

from tests.gpu_util import perturbed_glm_state, to_dev

pytestmark = pytest.mark.gpu


def _numpy_spectrum(u, kmax):
    rho = u[0]
    nz, ny, nx = rho.shape
    w = u[1:4] / np.sqrt(rho)
    what = np.fft.fftn(w, axes=(1, 2, 3)) / (nx * ny * nz)
    kz = np.fft.fftfreq(nz) * nz
    ky = np.fft.fftfreq(ny) * ny
    kx = np.fft.fftfreq(nx) * nx
    K = np.sqrt(kz[:, None, None] ** 2 + ky[None, :, None] ** 2 + kx[None, None, :] ** 2)
    shell = np.floor(K + 0.5).astype(int)
    p = 0.5 * (np.abs(what) ** 2).sum(0)
    return np.array([p[shell == s].sum() for s in range(kmax + 1)])


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_ke_spectrum_matches_numpy_fft(oracle, dtype):
    from glmmhdturb_b200 import Solver
    n = (32, 24, 20)
    u0 = perturbed_glm_state(oracle, n, seed=4)
    s = Solver(n, dtype=dtype, gamma=5 / 3)
    tdt = torch.float64 if dtype == "f64" else torch.float32
    E = s.ke_spectrum(to_dev(u0, tdt), kmax=8)
    ref = _numpy_spectrum(u0.astype(np.float32 if dtype == "f32" else np.float64).astype(np.float64), 8)
    np.testing.assert_allclose(E, ref, rtol=1e-9 if dtype == "f64" else 1e-5, atol=1e-14)
    # Parseval: all shells together carry the mean kinetic energy of the resolved low-k band
    assert E.sum() <= 0.5 * ((u0[1:4] ** 2).sum(0) / u0[0]).mean() * (1 + 1e-9)


def test_checkpoint_round_trip(tmp_path):
    from glmmhdturb_b200 import Solver, checkpoint
    s = Solver(16, dtype="f32", gamma=5 / 3, turb_amp=2.0, turb_T=0.5, turb_seed=3)
    u = s.alloc()
    s.ic_turbulent(u, mach=1.0, seed=3)
    s.forcing_reset()
    s.forcing_advance()
    s.forcing_advance()
    path = str(tmp_path / "state.gmt")
    checkpoint.save(path, u, t=0.25, step=7, solver=s)
    v, h = checkpoint.load(path)
    assert torch.equal(u, v) and h["t"] == 0.25 and h["step"] == 7 and h["forcing_counter"] == 2
    np.testing.assert_array_equal(h["modes"], s.get_modes())
    s2 = Solver(16, dtype="f32", gamma=5 / 3, turb_amp=2.0, turb_T=0.5, turb_seed=3)
    checkpoint.restore_forcing(s2, h)
    np.testing.assert_array_equal(s2.get_modes(), s.get_modes())


def test_spinup_reaches_target_mach():
    from glmmhdturb_b200 import checkpoint
    u, t, steps, s = checkpoint.spinup(32, seed=1, amp=8.0, mach_target=0.3, t_max=2.0, chunk=40)
    d = s.diagnostics(u)
    assert d["finite"] and d["vrms"] / np.sqrt(5 / 3 * 0.6) >= 0.3 and t < 2.0
    E = s.ke_spectrum(u, kmax=8)
    assert E[1:4].sum() > E[5:9].sum() > 0   # energy injected at |k| <= 3 dominates


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_density_pdf_matches_numpy(oracle, dtype):
    from glmmhdturb_b200 import Solver
    n = (32, 24, 20)
    u0 = perturbed_glm_state(oracle, n, seed=6)
    s = Solver(n, dtype=dtype, gamma=5 / 3)
    tdt = torch.float64 if dtype == "f64" else torch.float32
    ud = to_dev(u0, tdt)
    pdf, st = s.density_pdf(ud, nbins=40, smin=-2.0, smax=2.0)
    rho = ud[0].double().cpu().numpy()
    sv = np.log(rho / rho.mean())
    counts, _ = np.histogram(sv, bins=40, range=(-2.0, 2.0))
    np.testing.assert_allclose(pdf * rho.size * 0.1, counts, rtol=0, atol=1e-9)
    assert abs(st["rho_mean"] - rho.mean()) <= 1e-13 * rho.mean()
    assert abs(st["sigma_s"] - sv.std()) <= 1e-10 * sv.std()
    again, st2 = s.density_pdf(ud, nbins=40, smin=-2.0, smax=2.0)
    assert np.array_equal(again, pdf) and st2 == st    # deterministic


def test_checkpoint_restart_continues_the_run_bit_for_bit(tmp_path):
    """A forced device-loop run split by a checkpoint (state and the whole forcing state: modes, OU
    counter, next update time) into a fresh context equals the unsplit run bit for bit."""
    from glmmhdturb_b200 import Solver, checkpoint
    kw = dict(dtype="f32", gamma=5 / 3, courant=0.3, turb_amp=3.0, turb_T=0.5, turb_ndt=100, turb_seed=5)
    a = Solver(32, **kw)
    u, w = a.alloc(), a.alloc()
    a.ic_turbulent(u, mach=1.0, seed=2)
    u0 = u.clone()
    a.forcing_reset()
    t, res = a.run(u, w, 40, forcing=True, graph=False)
    want = res.clone()
    b = Solver(32, **kw)
    u.copy_(u0)
    b.forcing_reset()
    t1, res = b.run(u, w, 20, forcing=True, graph=False)
    path = str(tmp_path / "half.gmt")
    checkpoint.save(path, res, t=t1, step=20, solver=b)
    v, h = checkpoint.load(path)
    c = Solver(32, **kw)
    checkpoint.restore_forcing(c, h)
    assert c.forcing_state()["counter"] == b.forcing_state()["counter"] > 0
    w2 = torch.empty_like(v)
    t2, res2 = c.run(v, w2, 20, t0=h["t"], forcing=True, graph=False)
    assert t2 == t and torch.equal(res2, want)


def test_spinup_levels_reaches_the_target_on_every_grid():
    from glmmhdturb_b200 import checkpoint
    u, t, info, s = checkpoint.spinup_levels(64, n0=16, seed=1, amp=3.7737, mach_target=0.6, mach_coarse=0.9,
                                             dt_level=0.02, t_max=3.0, chunk=20)
    assert [m for m, *_ in info] == [16, 32, 64]
    assert all(b[1] > a[1] for a, b in zip(info, info[1:]))          # time advances through the ladder
    assert info[0][3] >= 0.54 and info[-1][3] >= 0.6 and t < 3.0
    d = s.diagnostics(u)
    assert d["finite"] and abs(d["vrms"] / np.sqrt(5 / 3 * 0.6) - info[-1][3]) < 1e-12
    assert s.forcing_state()["counter"] > 0
    assert u.shape == (9, 64, 64, 64)
