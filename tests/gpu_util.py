"""Shared helpers of the GPU tests (imported only by tests marked gpu)."""
import numpy as np
import torch


def to_dev(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def max_rel_err(got, ref):
    """max over fields of max|got-ref| / max|ref| (field-scale relative error)."""
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    errs = []
    for v in range(ref.shape[0]):
        scale = max(float(np.abs(ref[v]).max()), 1e-300)
        errs.append(float(np.abs(got[v] - ref[v]).max()) / scale)
    return max(errs), errs


def perturbed_glm_state(O, n, seed=0, gamma=5.0 / 3.0):
    cfg = O.Config(n=n, gamma=gamma)
    u = O.ic_ot(cfg)
    rng = np.random.default_rng(seed)
    u[0] *= 1.0 + 0.1 * rng.random(u[0].shape)
    u[1:4] += 0.05 * rng.standard_normal(u[1:4].shape)
    u[4] *= 1.0 + 0.05 * rng.random(u[4].shape)
    u[7] += 0.03 * rng.standard_normal(u[7].shape)
    u[8] = 0.01 * rng.standard_normal(u[8].shape)
    return u
