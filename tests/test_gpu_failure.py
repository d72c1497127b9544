"""Failure path of the bounded in-kernel waits, made to run out on purpose without a GPU fault.

The tile kernels (GLM, march, CT and the adjoint's record tile) wait for each staged plane on an
mbarrier with a wait bounded by a budget of SM clock cycles.  The test hook gmt_test_wait_limit
shortens that budget and withholds the staging of each next plane: no copy is issued and no thread
arrives on the mbarrier (a flag that nothing sets), so every wait runs out with nothing in flight.
The kernel records the failure and finishes; the host reports GMT_ERR_TIMEOUT.  With the hook
cleared, the same context then steps normally and reproduces a fresh context's step bit for bit.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

BUDGET = 20000       # SM clock cycles per wait (about 10 us at 1.965 GHz)
N = (32, 32, 12)     # several tiles, several planes per z-chunk


def _solver(scheme, dtype, **kw):
    from glmmhdturb_b200 import Solver
    return Solver(N, dtype=dtype, scheme=scheme, recon="mc", riemann="hll" if scheme == "march1d" else "hlld",
                  gamma=5 / 3, smallp=1e-6, **kw)


def _state(s):
    u = s.alloc()
    s.ic_turbulent(u, 1.0, 0.6, (0.775, 0.0, 0.0), mach=1.0, db=0.2, seed=4)   # CT: divergence-free faces
    return u


def _step(s, u, w):
    if s.scheme == "ct":
        s.step(u, w, 2e-3)
        s.cfl_async(w)
    else:
        s.step(u, w, 2e-3, ch=2.0, glm_fac=0.99, want_cfl=True)


@pytest.mark.parametrize("scheme,dtype", [("unsplit", "f32"), ("unsplit", "f64"), ("march1d", "f32"), ("ct", "f32"),
                                          ("ct", "f64")])
def test_wait_timeout_is_reported_and_the_context_recovers(scheme, dtype):
    from glmmhdturb_b200 import GmtError, _lib
    ref = _solver(scheme, dtype)
    u = _state(ref)
    want = torch.empty_like(u)
    _step(ref, u, want)
    ref.cfl_result()
    s = _solver(scheme, dtype)
    w = torch.empty_like(u)
    s.test_wait_limit(BUDGET, withhold=True)
    _step(s, u, w)
    with pytest.raises(GmtError) as e:
        s.cfl_result()
    assert e.value.code == _lib.GMT_ERR_TIMEOUT
    s.test_wait_limit(0, withhold=False)
    _step(s, u, w)
    s.cfl_result()                      # the flag was cleared by the report
    assert torch.equal(w, want)


def test_device_loop_reports_the_timeout():
    from glmmhdturb_b200 import GmtError, _lib
    s = _solver("unsplit", "f32")
    u = _state(s)
    w = torch.empty_like(u)
    s.test_wait_limit(BUDGET, withhold=True)
    with pytest.raises(GmtError) as e:
        s.run(u, w, 2, t_end=1.0, graph=False)
    assert e.value.code == _lib.GMT_ERR_TIMEOUT
    s.test_wait_limit(0, withhold=False)
    u = _state(s)
    t, which = s.run(u, w, 2, t_end=1.0, graph=False)
    assert t > 0.0


def test_adjoint_record_tile_reports_the_timeout():
    from glmmhdturb_b200 import GmtError, _lib
    s = _solver("unsplit", "f32", turb_amp=2.0, turb_T=0.5)
    s.forcing_advance()
    u = _state(s)
    gen = torch.Generator(device="cuda").manual_seed(1)
    ubn = torch.randn(u.shape, generator=gen, device="cuda", dtype=u.dtype)
    ub_ref = torch.empty_like(u)
    s.adjoint_step(u, ubn, ub_ref, 2e-3, t=0.2, ch=2.0, glm_fac=0.99, do_turb=True)
    g_ref = s.adjoint_amp_grad(reset=True)
    ub = torch.empty_like(u)
    s.test_wait_limit(BUDGET, withhold=True)
    s.adjoint_step(u, ubn, ub, 2e-3, t=0.2, ch=2.0, glm_fac=0.99, do_turb=True)
    with pytest.raises(GmtError) as e:
        s.adjoint_amp_grad(reset=True)
    assert e.value.code == _lib.GMT_ERR_TIMEOUT
    s.test_wait_limit(0, withhold=False)
    s.adjoint_step(u, ubn, ub, 2e-3, t=0.2, ch=2.0, glm_fac=0.99, do_turb=True)
    g = s.adjoint_amp_grad(reset=True)
    # ubar is deterministic; the amplitude partials are summed by atomics in any order
    assert torch.equal(ub, ub_ref) and abs(g - g_ref) <= 1e-9 * abs(g_ref)


def test_hook_rejects_a_negative_budget():
    from glmmhdturb_b200 import GmtError
    s = _solver("unsplit", "f32")
    with pytest.raises(GmtError):
        s.test_wait_limit(-1, withhold=False)
