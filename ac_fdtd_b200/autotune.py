"""Pick the sweeps' launch geometry by timing the candidates on the device.

The geometry -- threads per block and how many consecutive x planes a block marches through --
changes only the speed, never the result (every cell is computed by one thread with the same
arithmetic). Timing runs on a throwaway solver with the same shape, precision and physics so
the caller's state is untouched. Results are cached per process, keyed by the shape class,
dtype and which terms are active, and optionally in a JSON file named by ``ACF_TUNE_CACHE``.
"""

from __future__ import annotations

import json
import os
from pathlib import Path

import numpy as np

__all__ = ["CANDIDATES", "BATCH_CANDIDATES", "STAGED_CANDIDATES", "tune", "apply_tuned",
           "tune_batch", "apply_tuned_batch"]

#: (threads per block, planes per block) tried by default.
CANDIDATES = ((64, 4), (64, 8), (128, 2), (128, 4), (128, 8), (256, 4), (256, 8))

#: (scheme, threads per tile, planes per tile, CTAs per SM; 0 = one CTA per tile) for batches.
BATCH_CANDIDATES = (("fused", 128, 16, 0), ("fused", 128, 8, 0), ("fused", 64, 8, 0),
                    ("fused", 128, 32, 0), ("two_sweeps", 128, 8, 0), ("two_sweeps", 256, 4, 0),
                    ("two_sweeps", 128, 4, 0), ("two_sweeps", 256, 4, 4))

_cache: dict[str, tuple[int, int]] = {}


#: (rows per CTA, ring buffers (0: automatic), planes per CTA, z elements per thread) tried
#: for the staged scheme.
STAGED_CANDIDATES = ((2, 3, 32, 4), (2, 4, 32, 4), (2, 3, 16, 4), (2, 3, 64, 4), (1, 3, 32, 4),
                     (1, 3, 32, 2))

#: Schemes raced by default; all give bit-identical results.
SCHEMES = ("staged", "fused", "two_sweeps")


def _apply(solver, candidate) -> None:
    """Put ``solver`` on ``candidate`` = (scheme, *geometry); RuntimeError if it cannot run."""
    scheme, *geometry = candidate
    if scheme == "staged":
        rows, stages, planes, vector = geometry
        solver.set_staging(rows, stages, planes, vector)
    else:
        solver.set_launch(*geometry)
    solver.set_scheme(scheme)


def _candidates(schemes, candidates, staged_candidates):
    for scheme in schemes:
        for geometry in (staged_candidates if scheme == "staged" else candidates):
            yield (scheme, *geometry)


def _key(solver, schemes=SCHEMES) -> str:
    nx, ny, nz = solver._shape
    block = solver.coefficients
    key = [nx, ny, nz, solver.dtype.name, block.n_relax, block.layer_cell is not None,
           block.wall_shell is not None]
    if tuple(schemes) != SCHEMES:       # a race over other schemes is cached apart
        key.append(sorted(schemes))
    return json.dumps(key)


def _load_file() -> dict:
    path = os.environ.get("ACF_TUNE_CACHE")
    if path and Path(path).exists():
        try:
            return json.loads(Path(path).read_text())
        except (OSError, ValueError):
            return {}
    return {}


def _store_file(key: str, value) -> None:
    path = os.environ.get("ACF_TUNE_CACHE")
    if not path:
        return
    data = _load_file()
    data[key] = list(value)
    Path(path).write_text(json.dumps(data, indent=1))


def _race(twin, candidates, apply, steps: int, repeats: int, passes: int) -> dict:
    """Best ms/step of each candidate that ``apply`` accepts. The candidates are raced in
    ``passes`` passes, every other pass in reverse order, so that none is timed only while the
    GPU is still settling (measured: the first configs of a sequence run ~2 % slow)."""
    order = list(candidates)
    timings: dict = {}
    for n in range(passes):
        for candidate in (order if n % 2 == 0 else order[::-1]):
            try:
                apply(twin, candidate)
            except RuntimeError:
                continue
            twin.run(2)
            for _ in range(repeats):
                twin.profile(True)
                twin.run(steps)
                velocity_ms, pressure_ms, count = twin.profile_read()
                twin.profile(False)
                ms = (velocity_ms + pressure_ms) / max(count, 1)
                timings[candidate] = min(timings.get(candidate, float("inf")), ms)
    return timings


def tune(solver, candidates=CANDIDATES, steps: int = 12, repeats: int = 2, schemes=SCHEMES,
         staged_candidates=STAGED_CANDIDATES, passes: int = 2):
    """Time each (scheme, threads, planes) -- (scheme, rows, stages, planes, vector) for the
    staged scheme -- on a scratch twin of ``solver``; return (best, {candidate: ms/step})."""
    from .solver import CudaAcousticFDTD

    twin = CudaAcousticFDTD(solver.grid, solver.medium, solver.courant, solver.dtype,
                            solver.walls, solver.absorbing_layer, solver.air_absorption,
                            steps_per_graph=0)
    twin.p[:] = np.random.default_rng(0).standard_normal(twin.p.shape) * 1e-3
    try:
        timings = _race(twin, _candidates(schemes, candidates, staged_candidates), _apply, steps,
                        repeats, passes)
    finally:
        twin.close()
    winner = min(timings, key=timings.get)
    return winner, timings


def apply_tuned(solver, candidates=CANDIDATES, schemes=SCHEMES,
                staged_candidates=STAGED_CANDIDATES):
    """Set the fastest scheme and geometry for this configuration (tuned once per shape
    class); returns (scheme, threads, planes) or ("staged", rows, stages, planes, vector)."""
    key = _key(solver, schemes)
    if key not in _cache:
        stored = _load_file().get(key)
        if stored:
            _cache[key] = tuple(stored)
        else:
            winner, _ = tune(solver, candidates, schemes=schemes,
                             staged_candidates=staged_candidates)
            _cache[key] = winner
            _store_file(key, winner)
    _apply(solver, _cache[key])
    return _cache[key]


def _apply_batch(batch, candidate) -> None:
    batch.set_scheme(candidate[0])
    batch.set_launch(*candidate[1:])


def tune_batch(batch, candidates=BATCH_CANDIDATES, steps: int = 12, repeats: int = 2,
               passes: int = 2):
    """Time each batch geometry on a scratch twin batch; return (best, {candidate: ms/step})."""
    from .batch import RoomBatch

    twin = RoomBatch(batch.specs, dtype=batch.dtype, steps_per_graph=0)
    try:
        for r in range(len(twin)):
            twin.set_field(r, 0, np.random.default_rng(r).standard_normal(twin.shapes[r]) * 1e-3)
        timings = _race(twin, candidates, _apply_batch, steps, repeats, passes)
    finally:
        twin.close()
    return min(timings, key=timings.get), timings


def apply_tuned_batch(batch, candidates=BATCH_CANDIDATES):
    key = json.dumps(["batch", [list(s) for s in batch.shapes], batch.dtype.name])
    if key not in _cache:
        winner, _ = tune_batch(batch, candidates)
        _cache[key] = winner
    _apply_batch(batch, _cache[key])
    return _cache[key]
