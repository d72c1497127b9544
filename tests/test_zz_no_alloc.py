"""gmt_diagnostics_noalloc: diagnostics of a GLM state for callers that may not allocate.

Some callers of this library must not allocate device memory. One example is a driver loop that
logs diagnostics between steps and cannot afford the device-wide synchronisation of
cudaMalloc/cudaFree. Another is a host framework whose own pool owns the GPU memory budget.
A third is a hook that holds only a state pointer and no context. For them the library has this
one entry point. Its scratch is a static array inside the library, one row per z-plane. So it
allocates nothing, and it refuses grids with more than GMT_NOALLOC_MAX_PLANES z-planes.

The test calls it through the C ABI twice in a row, on two different states, and checks each
result against gmt_diagnostics (the context-based entry point). The two results agree to the
rounding of their different summation orders. The file is named so that pytest collects it
last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from tests.gpu_util import perturbed_glm_state, to_dev

pytestmark = pytest.mark.gpu

KEYS = ("mass", "ke2", "vrms", "divbmax", "rhomin", "etot", "divb_l2", "psi_l2")


def _noalloc(L, u, n, dtype_code, boxlen, smallr):
    from glmmhdturb_b200._lib import GmtDiag
    d = GmtDiag()
    rc = L.gmt_diagnostics_noalloc(u.data_ptr(), n[0], n[1], n[2], dtype_code, boxlen, smallr, C.byref(d),
                                   torch.cuda.current_stream().cuda_stream)
    return rc, d


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_noalloc_diagnostics_match_context_diagnostics(oracle, dtype):
    from glmmhdturb_b200 import Solver, _lib
    L = _lib.lib()
    code = _lib.F64 if dtype == "f64" else _lib.F32
    tdt = torch.float64 if dtype == "f64" else torch.float32
    n = (24, 16, 20)
    s = Solver(n, dtype=dtype, gamma=5 / 3)
    states = [to_dev(perturbed_glm_state(oracle, n, seed=s_), tdt) for s_ in (11, 12)]
    states[1][4, 3, 2, 1] = float("nan")   # the second call must not see the first call's sums
    rel = 1e-12 if dtype == "f64" else 1e-6
    for call, u in enumerate(states):
        free_before = torch.cuda.mem_get_info()[0]
        rc, d = _noalloc(L, u, n, code, 1.0, 1e-6)
        assert rc == _lib.GMT_OK, L.gmt_last_error().decode()
        if call == 1:
            assert torch.cuda.mem_get_info()[0] == free_before   # nothing allocated by the call
        ref = s.diagnostics(u)
        for k in KEYS:
            assert np.isclose(getattr(d, k), ref[k], rtol=rel, atol=1e-300, equal_nan=True), (call, k, getattr(d, k), ref[k])
        assert d.finite == ref["finite"] and d.nonfinite_cells == ref["nonfinite_cells"]
    assert d.finite == 0 and d.nonfinite_cells == 1


def test_noalloc_rejects_too_many_planes():
    from glmmhdturb_b200 import _lib
    L = _lib.lib()
    u = torch.zeros(9, dtype=torch.float32, device="cuda")
    nz = _lib.NOALLOC_MAX_PLANES + 1
    rc, _ = _noalloc(L, u, (1, 1, nz), _lib.F32, 1.0, 1e-6)
    assert rc == _lib.GMT_ERR_ARG
    assert "z-planes" in L.gmt_last_error().decode()
