"""Schedule cache over the native autotuner (hodlr_autotune).

The tuner times candidate launch schedules on a loaded system; the result
depends only on the system's shape, so it is cached in a JSON file keyed by
(N, nrhs, rank, threshold, precision) and reused for later systems of the
same shape:

    from fastsolver_b200 import autotune
    sched = autotune.tuned(matrix, fs.PREC_MIXED, cache="hodlr_schedules.json")
"""
from __future__ import annotations

import json
import os

from ._lib import PREC_MIXED


def shape_key(matrix, precision: int) -> str:
    return (f"N={matrix.rhs_rows},m={matrix.rhs_cols},r={matrix.rank},"
            f"t={matrix.threshold},p={int(precision)}")


def load(path: str) -> dict:
    if path and os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def tuned(matrix, precision: int = PREC_MIXED, cache: str | None = None, tol: float = 1e-12,
          reps: int = 2) -> dict:
    """Installs the cached schedule for the matrix's shape, or tunes it on the
    matrix's current data (and stores it) when the cache has none."""
    table = load(cache) if cache else {}
    key = shape_key(matrix, precision)
    if key in table:
        matrix.schedule = table[key]["schedule"]
        return table[key]["schedule"]
    best, ms, trials = matrix.autotune(precision, tol=tol, reps=reps)
    if cache:
        table[key] = {"schedule": best, "ms": ms, "trials": len(trials)}
        tmp = cache + ".tmp"
        with open(tmp, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
        os.replace(tmp, cache)
    return best
