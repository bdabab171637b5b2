"""Autotuner of the batched pass's tile shapes and schedule (no counterpart in the reference).

A factor's triangular pass is one launch per tree level and direction of 64-row output tiles on
the float64 tensor cores. Two choices shape it, and the best of each depends on the tree -- its
level sizes and separator widths -- and on the batch width:

- the split schedule: on a level with few tiles, long inner dimensions are split over several
  tiles (more CTAs, shorter dependent chains, atomic accumulation): which levels, and into how
  long pieces (``ob_chol_tile``);
- the tile width, the right-hand sides a CTA takes: 64 columns, or 32 (twice the CTAs, half the
  columns each, 64 instead of 96 registers a thread) on the levels with fewer tiles than some
  number of waves of the resident grid (``ob_chol_tile_columns``).

``tune_pass`` times one pass of a factor at ``k`` columns (CUDA events, ``ob_chol_time_solve``)
for each candidate split schedule, then, under the fastest, for each candidate width rule, keeps
the fastest of all and reports every candidate's time. ``tune_shared`` tunes one factor and gives
its schedule to the factors sharing its analysis: the heat and Poisson factors of a mesh have one
supernodal tree and one block layout, so their passes are the same launches over different values
(the tuner's timings of the two differ by noise) and one search serves both.
"""

from __future__ import annotations

import ctypes
from typing import Any

from ordito_b200 import _lib

# (split chunk, waves): the inner range of a split tile (0: never split) and the level size, in
# waves of the resident grid, below which a level is split. The factor's default is (64, 2).
CANDIDATES: tuple[tuple[int, int], ...] = (
    (64, 2), (0, 0), (32, 2), (128, 2), (64, 1), (64, 4), (128, 4), (32, 1),
)
# Width rules: the levels with fewer tiles than this many waves take 32-column tiles (0: none,
# 64: every level, the factor's default, under which the split schedules are timed).
WIDTHS: tuple[int, ...] = (64, 0, 1, 2, 4)
DEFAULT_WIDTH = 64


def _time(factor: Any, k: int, reps: int) -> float:
    ms = ctypes.c_float(0.0)
    _lib.call("ob_chol_time_solve", factor.handle, int(k), 1, ctypes.byref(ms), None)  # warm
    _lib.call("ob_chol_time_solve", factor.handle, int(k), int(reps), ctypes.byref(ms), None)
    return float(ms.value)


def apply_schedule(factor: Any, report: dict) -> None:
    """Give ``factor`` the schedule ``tune_pass`` chose for a factor of the same analysis."""
    _lib.call("ob_chol_tile", factor.handle, int(report["best"][0]), int(report["best"][1]), None)
    _lib.call("ob_chol_tile_columns", factor.handle, int(report["narrow_waves"]), None)


def tune_shared(factors: dict[str, Any], k: int, *, reps: int = 10) -> dict:
    """Tune the first of ``factors`` (role -> factor, all of one analysis) and apply its schedule
    to the others; every role's entry is the first's report, the others marked ``shared``."""
    roles = list(factors)
    report = tune_pass(factors[roles[0]], k, reps=reps)
    out = {roles[0]: report}
    for role in roles[1:]:
        apply_schedule(factors[role], report)
        out[role] = dict(report, shared=roles[0])
    return out


def tune_pass(factor: Any, k: int, *, reps: int = 10,
              candidates: tuple[tuple[int, int], ...] = CANDIDATES) -> dict:
    """Time ``factor``'s forward + backward pass at ``k`` columns under each candidate schedule
    and keep the fastest. No pass of the factor may be in flight (retiling waits for the device
    and makes every recording over the factor's buffers record again on its next launch).
    Returns ``{"best": (chunk, waves), "ms": {(chunk, waves): ms, ...}}``."""
    times: dict[tuple[int, int], float] = {}
    widths: dict[int, float] = {}
    _lib.call("ob_chol_tile_columns", factor.handle, DEFAULT_WIDTH, None)
    if getattr(factor, "deterministic", False):
        # A deterministic factor never splits (its passes take no atomics): one schedule.
        times[(0, 0)] = _time(factor, k, reps)
        best = (0, 0)
    else:
        for chunk, waves in candidates:
            _lib.call("ob_chol_tile", factor.handle, int(chunk), int(waves), None)
            times[(chunk, waves)] = _time(factor, k, reps)
        best = min(times, key=times.get)
        _lib.call("ob_chol_tile", factor.handle, best[0], best[1], None)
    # Batches of up to 16 columns take the register kernel or the 16-column tiles whatever the
    # width rule: nothing to search.
    for narrow in WIDTHS if k > 16 else (DEFAULT_WIDTH,):
        _lib.call("ob_chol_tile_columns", factor.handle, int(narrow), None)
        widths[narrow] = times[best] if narrow == DEFAULT_WIDTH else _time(factor, k, reps)
    width = min(widths, key=widths.get)
    _lib.call("ob_chol_tile_columns", factor.handle, int(width), None)
    return {"best": best, "ms": times, "narrow_waves": width, "width_ms": widths}
