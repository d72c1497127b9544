"""Host-side logic of the checkpointed adjoint driver (no GPU needed)."""
import math

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
