"""Loading of the golden fixtures (tests/golden/*.json, made by
tests/golden/make_golden.py from the reference's own code)."""
import glob
import json
import os

import numpy as np

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    return sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(GOLDEN_DIR, "*.json")))


def load(name):
    with open(os.path.join(GOLDEN_DIR, name + ".json")) as f:
        return json.load(f)


class FixtureSettings(object):
    """The fixture's settings over the reference defaults (defaults.cfg)."""

    def __init__(self, fx):
        from pypaswas_b200.workloads import Settings
        base = Settings()
        for k, v in fx["settings"].items():
            setattr(base, k, v)
        self.__dict__.update(base.__dict__)


def global_pair_max(fx):
    """Pair maxima [query, target] assembled from the fixture's batches."""
    nq, nt = len(fx["queries"]), len(fx["targets"])
    pm = np.full((nq, nt), np.nan, dtype=np.float64)
    for b, (s0, t0) in zip(fx["batches"], fx["batch_offsets"]):
        m = np.array(b["pair_max"], dtype=np.float32)
        for i in range(m.shape[0]):
            for j in range(m.shape[1]):
                if s0 + i < nq and t0 + j < nt:
                    pm[s0 + i, t0 + j] = m[i, j]
    return pm


def starts_by_pair(fx):
    """{(query, target): [(x, y, score), ...] in emission order}."""
    out = {}
    for b, (s0, t0) in zip(fx["batches"], fx["batch_offsets"]):
        for u, f in zip(b["starts_u32"], b["starts_f32"]):
            q, t = s0 + u[0], t0 + u[1]
            out.setdefault((q, t), []).append((u[2] * 8 + u[4], u[3] * 8 + u[5], float(np.float32(f[0]))))
    return out


def hits_by_pair(hits):
    out = {}
    for h in hits:
        out.setdefault((h["seq_id"], h["target_id"]), []).append(h)
    return out
