"""Empirical tuning of the engine's launch shapes on the inputs it holds.

The score sweep's shape is mostly fixed by cost models (lane orientation,
strip class, list-scheduling plan); what is left to measurement is the share
of multi-strip items cut into chained one-strip entries (PW_TUNE_CHAIN_MIN):
more chaining shortens the longest items and keeps boundary rows in L2, less
chaining saves the pipeline fill of each chain.  `autotune` times the score
sweep (device time of its launches, pw_run_info.score_kernel_ms) for each
candidate on the engine's current queries and targets and keeps the fastest.
The reference has no counterpart: its shapes are template constants
(pyPaSWAS/Core/cuda/default_main.cu:7-30).
"""
from . import _native

CHAIN_MIN_CANDIDATES = (250, 500, 1000, 2000)


def autotune(engine, candidates=CHAIN_MIN_CANDIDATES, repeats=2):
    """Sets PW_TUNE_CHAIN_MIN on `engine` to the fastest candidate; returns
    {"chain_min": best, "score_kernel_ms": {candidate: best time}}."""
    times = {}
    for value in candidates:
        engine.set_tuning(_native.PW_TUNE_CHAIN_MIN, int(value))
        engine.align(score_only=True)  # builds and caches the plan for this value
        best = None
        for _ in range(max(1, repeats)):
            ms = engine.align(score_only=True).score_kernel_ms
            best = ms if best is None else min(best, ms)
        times[int(value)] = best
    choice = min(times, key=lambda v: (times[v], v))
    engine.set_tuning(_native.PW_TUNE_CHAIN_MIN, choice)
    return {"chain_min": choice, "score_kernel_ms": times}
