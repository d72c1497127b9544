"""Autotuner of the step kernel's launch shape: tile (x, y), threads per block and z-chunk length,
for the unsplit GLM step, the march scheme and the constrained-transport step.

Each candidate is a separate context (the tile is fixed at gmt_create); candidates are timed with
CUDA events on the caller's state, best-of-`reps`, and the winner is cached in a JSON file keyed
by (grid, precision, scheme, recon, riemann, GPU name).
"""
from __future__ import annotations

import json
import os

import torch

from .solver import Solver

CACHE = os.environ.get("GMT_TUNE_CACHE", os.path.join(os.path.dirname(os.path.abspath(__file__)), "_tune_cache.json"))

TILES = {
    "f32": [(32, 8), (16, 8), (16, 16), (32, 4), (64, 4), (32, 16), (64, 8), (16, 32), (128, 4)],
    "f64": [(32, 8), (16, 8), (16, 16), (32, 4), (8, 8)],
}
CHUNKS = [16, 32, 64, 128, 256, 0]


def _key(n, dtype, scheme, recon, riemann):
    name = torch.cuda.get_device_name()
    return f"{name}|{n[0]}x{n[1]}x{n[2]}|{dtype}|{scheme}|{recon}|{riemann}"


def load_cache() -> dict:
    try:
        return json.load(open(CACHE))
    except Exception:
        return {}


def cached(n, dtype="f32", scheme="unsplit", recon="mc", riemann="hlld"):
    if isinstance(n, int):
        n = (n, n, n)
    return load_cache().get(_key(n, dtype, scheme, recon, riemann))


def tune(n, *, dtype="f32", scheme="unsplit", recon="mc", riemann="hlld", gamma=5.0 / 3.0, reps=3, steps=2,
         tiles=None, chunks=None, save=True, log=None, **solver_kw):
    """Time every (tile, chunk) candidate on a seeded turbulent state; return the best tile tuple."""
    if isinstance(n, int):
        n = (n, n, n)
    tiles = tiles or TILES[dtype]
    chunks = chunks or CHUNKS
    solver_kw = dict(solver_kw, scheme=scheme)
    probe = Solver(n, dtype=dtype, recon=recon, riemann=riemann, gamma=gamma, **solver_kw)
    u = probe.alloc()
    w = probe.alloc()
    probe.ic_turbulent(u, 1.0, 0.6, (0.775, 0.0, 0.0), mach=1.0, db=0.1, seed=1)
    cm, sm = probe.cfl(u)
    dt = 0.3 * probe.dx / cm
    probe.close()
    results = []
    for (tx, ty) in tiles:
        if n[0] % tx or n[1] % ty:
            continue
        for lz in chunks:
            lz_eff = lz if lz and lz <= n[2] else 0
            try:
                s = Solver(n, dtype=dtype, recon=recon, riemann=riemann, gamma=gamma, tile=(tx, ty, lz_eff), **solver_kw)
            except Exception:
                continue
            best = float("inf")
            for r in range(reps + 1):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(steps):
                    s.step(u, w, dt, ch=sm, glm_fac=0.99)
                e1.record()
                torch.cuda.synchronize()
                if r > 0:
                    best = min(best, e0.elapsed_time(e1) / steps)
            tile = s.kernel_info()["tile"]
            results.append((best, tile))
            if log:
                log(f"tile {tile}: {best:.3f} ms/step")
            s.close()
    results.sort()
    best_ms, best_tile = results[0]
    if save:
        c = load_cache()
        c[_key(n, dtype, scheme, recon, riemann)] = {"tile": list(best_tile), "ms": best_ms,
                                                       "candidates": [[list(t), ms] for ms, t in results]}
        try:
            json.dump(c, open(CACHE, "w"), indent=1)
        except OSError:
            pass
    return tuple(best_tile), best_ms, results
