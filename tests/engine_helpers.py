"""Drives the engine through the C ABI the way the package driver does."""
import numpy as np

from pypaswas_b200 import _native


def configure(engine, score, settings):
    gap, ext, affine, ll, mn = score.kernel_constants()
    engine.set_scoring(score.matrix_array(), score.char_offset_code(), gap, ext, affine, ll, mn,
                       float(settings.minimum_score), float(score.highest_score), float(settings.filter_factor))


def run_engine(lib, queries, targets, score, settings, q_keys=None, t_keys=None, tuning=None, **align_kw):
    e = _native.Engine(0, lib=lib)
    try:
        configure(e, score, settings)
        e.set_queries([q.encode() for q in queries], np.arange(len(queries)) if q_keys is None else q_keys)
        e.set_targets([t.encode() for t in targets],
                      np.arange(len(targets)) + len(queries) if t_keys is None else t_keys)
        for key, value in (tuning or {}).items():
            e.set_tuning(key, value)
        info = e.align(**align_kw)
        pm = e.pair_max()
        hits = decode_hits(*e.hits()) if not align_kw.get("score_only") else []
        return pm, hits, info, e.launch_count()
    finally:
        e.close()


def decode_hits(hits, sb):
    out = []
    for h in hits:
        n, o = int(h["n_cols"]), int(h["str_offset"])
        out.append({"query": int(h["query"]), "target": int(h["target"]),
                    "s_start": int(h["s_start"]), "s_end": int(h["s_end"]),
                    "t_start": int(h["t_start"]), "t_end": int(h["t_end"]),
                    "score": float(h["score"]), "matches": int(h["matches"]), "mismatches": int(h["mismatches"]),
                    "sequence_match": sb[o:o + n].decode("latin-1"),
                    "alignment": sb[o + n:o + 2 * n].decode("latin-1"),
                    "target_match": sb[o + 2 * n:o + 3 * n].decode("latin-1")})
    return out
