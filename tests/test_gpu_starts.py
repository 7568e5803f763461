"""Starting points of the engine (pw_get_starting_points: the 36-byte
StartingPoint records of default_main.cu:66-76 / StartingPoint.py:7-17) against
the oracle and the reference's own raw batch results.

The reference emits a starting point for every cell that passes the traceback
kernel's candidate test (default_main.cu:609-627 linear, :840-862 affine) in
atomicAdd order; the engine and the oracle emit them in the order of a
sequential run of the reference's launches.  Compared here: every record field
(query, target, block and in-block coordinates, score, pair maximum, the
maxPossibleScore bound) and the emission order."""
import numpy as np
import pytest

import cases
import golden_util as G
from engine_helpers import configure
from pypaswas_b200 import _native

pytestmark = pytest.mark.gpu

KINDS = ["dna", "protein", "dna_ambiguous", "dna_float"]


def _engine_starts(lib, queries, targets, score, settings, q_keys=None, t_keys=None, **align_kw):
    e = _native.Engine(0, lib=lib)
    try:
        configure(e, score, settings)
        e.set_queries([q.encode() for q in queries], np.arange(len(queries)) if q_keys is None else q_keys)
        e.set_targets([t.encode() for t in targets],
                      np.arange(len(targets)) + len(queries) if t_keys is None else t_keys)
        e.align(**align_kw)
        return e.starting_points()
    finally:
        e.close()


def _as_tuples(starts):
    return [tuple(int(s[f]) for f in ("sequence", "target", "block_x", "block_y", "value_x", "value_y")) +
            tuple(float(s[f]) for f in ("score", "max_score", "pos_score")) for s in starts]


def _emission_key(t):
    """Global emission order of the reference's launches run one after another
    (block anti-diagonal descending, block x descending, target, query, cell
    anti-diagonal descending, row): the order the reference's own kernels give
    in every golden fixture batch (tests/test_oracle_golden.py)."""
    q, tg, bx, by, vx, vy = t[:6]
    return (-(bx + by), -bx, tg, q, -(vx + vy), vy)


def _by_pair(tuples):
    out = {}
    for t in tuples:
        out.setdefault((t[0], t[1]), []).append(t)
    return out


def _check_against_oracle(got, oracle_starts):
    g, o = _as_tuples(got), _as_tuples(oracle_starts)
    # every record, per pair in the same order (the oracle emits pair by pair)
    assert _by_pair(g) == _by_pair(o)
    # and across pairs in the launches' global order
    assert [_emission_key(t) for t in g] == sorted(_emission_key(t) for t in g)


@pytest.mark.parametrize("seed", range(16))
def test_starting_points_equal_oracle_in_emission_order(engine_lib, oracle_mod, seed):
    queries, targets, score, st = cases.make_case(3000 + seed, KINDS[seed % len(KINDS)])
    p = cases.oracle_params(oracle_mod, score)
    pos = cases.pos_scores(score, st, queries, targets)
    o = oracle_mod.run(p, queries, targets, pos, float(st.minimum_score))
    got = _engine_starts(engine_lib, queries, targets, score, st)
    assert len(got) > 0 or len(o["starts"]) == 0
    _check_against_oracle(got, o["starts"])


def test_starting_points_with_memory_waves_equal_oracle(engine_lib, oracle_mod):
    # many traced pairs under a small cell-code budget: starts gathered over
    # several memory waves keep the single-run emission order
    rng = np.random.default_rng(41)
    motif = "".join(cases.DNA[i] for i in rng.integers(0, 4, 60))
    q = []
    for _ in range(120):
        s = "".join(cases.DNA[i] for i in rng.integers(0, 4, int(rng.integers(30, 140))))
        p = int(rng.integers(0, len(s) + 1))
        q.append(s[:p] + cases.mutate(rng, motif, cases.DNA, 0.1, 1) + s[p:])
    t = [motif, motif[::-1], "".join(cases.DNA[i] for i in rng.integers(0, 4, 90))]
    from pypaswas_b200 import scores
    st = cases.Settings(minimum_score="12", lower_limit_score="0.8", filter_factor="0.1")
    score = scores.make_score(st)
    o = oracle_mod.run(cases.oracle_params(oracle_mod, score), q, t, cases.pos_scores(score, st, q, t),
                       float(st.minimum_score))
    e = _native.Engine(0, lib=engine_lib)
    try:
        configure(e, score, st)
        e.set_queries([s.encode() for s in q], np.arange(len(q)))
        e.set_targets([s.encode() for s in t], np.arange(len(t)) + len(q))
        e.set_wave_limit(64 << 10)
        info = e.align()
        assert info.waves >= 2
        got = e.starting_points()
    finally:
        e.close()
    _check_against_oracle(got, o["starts"])


@pytest.mark.parametrize("name", [n for n in G.names() if "exception" not in G.load(n)])
def test_starting_points_equal_reference_batches(engine_lib, name):
    """Per pair, the reference's own raw starting points (its kernels, its
    batches): same cells, scores, maxima and bounds, in the same order."""
    fx = G.load(name)
    st = G.FixtureSettings(fx)
    from pypaswas_b200 import scores
    score = scores.make_score(st)
    queries = [s for _, s in fx["queries"]]
    targets = [s for _, s in fx["targets"]]
    # distinct keys: the reference's kernels emit starts of same-id pairs too
    got = _engine_starts(engine_lib, queries, targets, score, st)
    mine = {}
    for s in got:
        mine.setdefault((int(s["sequence"]), int(s["target"])), []).append(
            (int(s["block_x"]) * 8 + int(s["value_x"]), int(s["block_y"]) * 8 + int(s["value_y"]),
             float(s["score"]), float(s["max_score"]), float(s["pos_score"])))
    ref = {}
    for b, (s0, t0) in zip(fx["batches"], fx["batch_offsets"]):
        for u, f in zip(b["starts_u32"], b["starts_f32"]):
            ref.setdefault((s0 + u[0], t0 + u[1]), []).append(
                (u[2] * 8 + u[4], u[3] * 8 + u[5], float(np.float32(f[0])), float(np.float32(f[1])),
                 float(np.float32(f[2]))))
    assert mine == ref
