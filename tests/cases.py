"""Seeded synthetic alignment cases shared by the parity tests.

Each case is a small all-vs-all workload (queries x targets) with planted
homologous segments, so that hits, gaps, ties and collisions between walks all
occur.  Sizes stay small enough for the CPU oracle to finish in seconds."""
import numpy as np

from pypaswas_b200 import scores

DNA = "ACGT"
DNA_AMBIGUOUS = "ACGTNKMRYSW"
PROTEIN = "ARNDCQEGHILKMFPSTWYVBZX"


class Settings(object):
    def __init__(self, **kw):
        self.gap_score = "-5"
        self.gap_extension = "0"
        self.match_score = "1"
        self.mismatch_score = "-3"
        self.other_score = "-1"
        self.any_score = "1"
        self.lower_limit_score = "1.0"
        self.minimum_score = "8"
        self.matrix_name = "DNA-RNA"
        self.filter_factor = "0.2"
        for k, v in kw.items():
            setattr(self, k, v)


def mutate(rng, seq, alphabet, sub_rate, indel_events):
    a = list(seq)
    for j in range(len(a)):
        if rng.random() < sub_rate:
            a[j] = alphabet[int(rng.integers(0, len(alphabet)))]
    for _ in range(indel_events):
        if len(a) > 1 and rng.random() < 0.5:
            del a[int(rng.integers(0, len(a)))]
        else:
            a.insert(int(rng.integers(0, len(a) + 1)), alphabet[int(rng.integers(0, len(alphabet)))])
    return "".join(a)


def make_case(seed, kind="dna", max_queries=45, max_qlen=150, max_tlen=200):
    """Returns (queries, targets, score, settings)."""
    rng = np.random.default_rng(seed)
    alphabet = {"dna": DNA, "dna_float": DNA, "dna_ambiguous": DNA_AMBIGUOUS, "protein": PROTEIN}[kind]

    def rs(k):
        return "".join(alphabet[i] for i in rng.integers(0, len(alphabet), k))

    tlen = int(rng.choice([rng.integers(1, 20), rng.integers(20, 70), rng.integers(60, max_tlen)]))
    motif = rs(tlen)
    queries = []
    for _ in range(int(rng.integers(1, max_queries))):
        s = rs(int(rng.integers(1, max_qlen)))
        if rng.random() < 0.6:
            cut = int(rng.integers(0, max(1, len(motif) // 3)))
            frag = mutate(rng, motif[cut:], alphabet, 0.15, int(rng.integers(0, 3)))
            p = int(rng.integers(0, len(s) + 1))
            s = s[:p] + frag + s[p:]
        queries.append(s)
    targets = [motif] + [rs(int(rng.integers(1, max_tlen))) for _ in range(int(rng.integers(0, 3)))]
    if rng.random() < 0.3:
        targets.append(motif[::-1])
    affine = bool(rng.random() < 0.5)
    kw = dict(lower_limit_score=str(float(rng.choice([1.0, 0.9, 0.5, 0.2]))),
              filter_factor=str(float(rng.choice([0.2, 0.1, 0.0]))),
              minimum_score=str(float(rng.choice([2.0, 5.0, 8.0, 15.5]))))
    if kind == "protein":
        kw.update(matrix_name="BLOSUM62", gap_score=str(float(rng.choice([-11.0, -8.0, -5.0]))),
                  gap_extension="-1" if affine else "0")
    elif kind == "dna_float":
        kw.update(match_score="1.5", mismatch_score="-2.25", any_score="0.5", gap_score="-3.5",
                  gap_extension="-0.75" if affine else "0")
    else:
        kw.update(gap_extension="-1" if affine else "0")
    st = Settings(**kw)
    return queries, targets, scores.make_score(st), st


def oracle_params(oracle, score):
    gap, ext, affine, ll, mn = score.kernel_constants()
    return oracle.OracleParams(score.matrix_array(), score.char_offset_code(), gap, ext, affine, ll, mn)


def pos_scores(score, settings, queries, targets):
    """maxPossibleScore per pair, [target, query] (SmithWatermanCuda.py:269-275)."""
    hi, ff = float(score.highest_score), float(settings.filter_factor)
    return np.array([[np.float32(hi * min(len(q), len(t)) * ff) for q in queries] for t in targets], np.float32)
