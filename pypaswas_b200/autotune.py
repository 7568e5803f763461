"""Empirical tuning of the score sweep's shape on the inputs the engine holds.

Most of the shape comes from cost models (lane orientation, strip class,
list-scheduling plan); what is left to measurement is tuned here, one knob
after the other, each time keeping the fastest setting: the wall time of a
score-only pw_align that rebuilds its plan (pw_run_info.total_ms, best of
`repeats`), so that a setting whose kernels gain less than its plan costs
loses -- every call with new inputs plans anew:

  1. lane width (PW_TUNE_LANES): the 16x2 sweep -- two 16-bit cells per
     32-bit lane, pairs that reach the 16-bit limit recomputed on 32-bit
     lanes -- against the 32-bit sweep;
  2. register form of the 16x2 sweep (PW_TUNE_DUAL): two strips against one
     lane sequence, one strip against two lane sequences, or the cost model's
     pick;
  3. chaining (PW_TUNE_CHAIN_MIN): the share of multi-strip items cut into
     chained one-strip entries -- more chaining shortens the longest items,
     less saves each chain's pipeline fill.

The reference has no counterpart: its shapes are template constants
(pyPaSWAS/Core/cuda/default_main.cu:7-30).
"""
from . import _native

CHAIN_MIN_CANDIDATES = (250, 500, 1000, 2000)
DUAL_CANDIDATES = (0, 1, 2)  # cost model, always dual lanes, always strip pairs
LANE_CANDIDATES = (0, 32)    # 16x2 where possible, 32-bit


def _time(engine, repeats):
    engine.align(score_only=True, replan=True)  # warm
    best = None
    for _ in range(max(1, repeats)):
        info = engine.align(score_only=True, replan=True)
        best = info.total_ms if best is None else min(best, info.total_ms)
    return best, info


def _pick(engine, key, candidates, repeats):
    times, infos = {}, {}
    for value in candidates:
        engine.set_tuning(key, int(value))
        times[int(value)], infos[int(value)] = _time(engine, repeats)
    choice = min(times, key=lambda v: (times[v], v))
    engine.set_tuning(key, choice)
    return choice, times, infos


def autotune(engine, repeats=2, chain_candidates=CHAIN_MIN_CANDIDATES):
    """Sets the engine's lane width, 16x2 form and chaining threshold to the
    fastest measured values; returns the choices and the times behind them."""
    out = {}
    lanes, t_lanes, infos = _pick(engine, _native.PW_TUNE_LANES, LANE_CANDIDATES, repeats)
    out["lanes"] = 16 if lanes == 0 else 32
    out["lanes_ms"] = {("16x2" if k == 0 else "32"): v for k, v in t_lanes.items()}
    if lanes == 0 and infos[0].score_path == 0:
        dual, t_dual, _ = _pick(engine, _native.PW_TUNE_DUAL, DUAL_CANDIDATES, repeats)
        out["dual"] = {0: "cost model", 1: "dual lanes", 2: "strip pairs"}[dual]
        out["dual_ms"] = t_dual
        chain, t_chain, _ = _pick(engine, _native.PW_TUNE_CHAIN_MIN, chain_candidates, repeats)
        out["chain_min"] = chain
        out["score_phase_ms"] = t_chain
    return out
