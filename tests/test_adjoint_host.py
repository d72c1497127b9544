"""Host-side logic of the checkpointed adjoint driver (no GPU needed)."""
import math

import pytest

from glmmhdturb_b200 import adjoint as AD


def test_checkpoint_interval_minimises_memory():
    # no budget: about sqrt(N)
    assert AD.checkpoint_interval(100, 1) == 10
    assert AD.checkpoint_interval(200, 1) == 14
    # with a budget: the K with the least ceil(N/K) + K states that fits, scratch included
    state = 75_497_472                       # 128^3 x 9 FP32
    k = AD.checkpoint_interval(200, state, 40 << 30)
    need = (math.ceil(200 / k) + k) * state + (2 + 207 / 9) * state
    assert need <= 40 << 30 and 10 <= k <= 20
    # a budget that cannot hold the scratch
    try:
        AD.checkpoint_interval(200, state, state)
    except ValueError:
        pass
    else:
        raise AssertionError("expected ValueError")


def test_schedule_records():
    s = AD.Schedule()
    s.steps.append(AD.StepRecord(dt=1e-3, t=0.0, ch=1.0, glm_fac=0.99, modes=-1))
    assert len(s) == 1 and s.forcing


def test_reverse_sweeps_match_dual_numbers(tmp_path):
    """The hand-written reverse sweeps of the adjoint (HLLD over every fan region and the degenerate
    star state, HLL, cons2prim, prim2cons, the x flux, the update epilogue with its floors) agree
    with forward-mode dual-number VJPs of the same FP64 forward functions.  Host code only, built
    with nvcc from tests/host/adjoint_sweeps.cu."""
    import os
    import shutil
    import subprocess
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    here = os.path.dirname(os.path.abspath(__file__))
    exe = str(tmp_path / "adjoint_sweeps")
    subprocess.run([nvcc, "-std=c++17", "-O2", "--expt-relaxed-constexpr", "-Wno-deprecated-gpu-targets", "-o", exe,
                    os.path.join(here, "host", "adjoint_sweeps.cu")], check=True, capture_output=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    lines = {ln.split()[0]: ln.split()[1:] for ln in out.strip().splitlines()}
    for name in ("hlld", "hll", "cons2prim", "prim2cons", "phys_flux_x", "epilogue"):
        assert float(lines[name][1]) <= 1e-12, (name, lines[name])
    assert all(int(c) > 0 for c in lines["hlld_regions"]), lines["hlld_regions"]
