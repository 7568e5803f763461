"""Seeded synthetic workloads with the shapes of the benchmark configurations.

The reference names no public benchmark suite; these generators stand in with
the stated sizes, length distributions and residue frequencies.  Every
generator is deterministic for a given seed (NumPy PCG64).
"""
import numpy as np

DNA = np.frombuffer(b"ACGT", dtype=np.uint8)
AMINO = np.frombuffer(b"ARNDCQEGHILKMFPSTWYV", dtype=np.uint8)
# background amino-acid frequencies (Robinson & Robinson 1991), order of AMINO
AMINO_FREQ = np.array([0.07805, 0.05129, 0.04487, 0.05364, 0.01925, 0.04264, 0.06295, 0.07377, 0.02199, 0.05142,
                       0.09019, 0.05744, 0.02243, 0.03856, 0.05203, 0.07120, 0.05841, 0.01330, 0.03216, 0.06441])
AMINO_FREQ = AMINO_FREQ / AMINO_FREQ.sum()
_COMPLEMENT = bytes.maketrans(b"ACGTUNKMRYSWBDHVacgtunkmryswbdhv", b"TGCAANMKYRSWVHDBtgcaanmkyrswvhdb")


def reverse_complement(seq):
    """IUPAC reverse complement of a byte string (case kept)."""
    return seq.translate(_COMPLEMENT)[::-1]


def _random_seq(rng, n, alphabet, p=None):
    return alphabet[rng.choice(len(alphabet), size=n, p=p)].tobytes()


def _mutate(rng, seq, alphabet, sub_rate, p=None, indel_rate=0.0):
    a = np.frombuffer(seq, dtype=np.uint8).copy()
    m = rng.random(len(a)) < sub_rate
    a[m] = alphabet[rng.choice(len(alphabet), size=int(m.sum()), p=p)]
    if indel_rate <= 0:
        return a.tobytes()
    out = bytearray()
    r = rng.random(len(a))
    ins = rng.random(len(a)) < 0.5
    for i, c in enumerate(a):
        if r[i] < indel_rate:
            if ins[i]:
                out.append(c)
                out.append(int(alphabet[rng.integers(0, len(alphabet))]))
            # else: deletion
        else:
            out.append(c)
    return bytes(out)


class Workload(object):
    """queries / targets as lists of (id, upper-case byte string)."""

    def __init__(self, name, queries, targets, settings, pairs=None):
        self.name = name
        self.queries = queries
        self.targets = targets
        self.settings = settings
        self.pairs = pairs

    @property
    def cells(self):
        if self.pairs is not None:
            return sum(len(self.queries[q][1]) * len(self.targets[t][1]) for q, t in self.pairs)
        return sum(len(s) for _, s in self.queries) * sum(len(s) for _, s in self.targets)


def dna_reads_vs_adapters(seed=1, n_reads=1000, read_len=150, n_adapters=50, adapter_len=(30, 60),
                          planted=0.30, sub_rate=0.05):
    """Reads of uniform ACGT; a fraction carry one adapter copy with substitutions.
    Targets are the adapters plus their reverse complements (the reference adds
    them for DNA, Readers.complement_records), sorted by length descending."""
    rng = np.random.default_rng(seed)
    adapters = [_random_seq(rng, int(rng.integers(adapter_len[0], adapter_len[1] + 1)), DNA)
                for _ in range(n_adapters)]
    reads = []
    for i in range(n_reads):
        r = _random_seq(rng, read_len, DNA)
        if rng.random() < planted:
            a = _mutate(rng, adapters[int(rng.integers(0, n_adapters))], DNA, sub_rate)
            p = int(rng.integers(0, read_len))
            r = (r[:p] + a + r[p:])[:read_len]
        reads.append(("read%d" % i, r))
    targets = [("adapter%d" % i, a) for i, a in enumerate(adapters)]
    targets += [(tid + "_RC", reverse_complement(s)) for tid, s in targets]
    reads.sort(key=lambda r: len(r[1]), reverse=True)
    targets.sort(key=lambda r: len(r[1]), reverse=True)
    return reads, targets


def protein_batched(seed=2, n_queries=200, n_targets=2000, q_median=350.0, q_sigma=0.5, q_clip=(100, 1000),
                    t_range=(50, 2000), domain_len=150, domain_identity=0.40, shared_pairs=0.10):
    """Queries log-normal in length, targets uniform; residues from background
    frequencies.  One ancestral domain is planted exactly in a fraction f of
    the queries and as a copy at the stated identity in a fraction f of the
    targets, f = sqrt(shared_pairs), so that that fraction of pairs share it."""
    rng = np.random.default_rng(seed)
    qlens = np.clip(np.round(rng.lognormal(np.log(q_median), q_sigma, n_queries)), q_clip[0], q_clip[1]).astype(int)
    tlens = rng.integers(t_range[0], t_range[1] + 1, n_targets)
    domain = _random_seq(rng, domain_len, AMINO, AMINO_FREQ)
    f = float(np.sqrt(shared_pairs))

    def plant(seq, dom):
        if len(seq) < len(dom):
            return seq
        p = int(rng.integers(0, len(seq) - len(dom) + 1))
        return seq[:p] + dom + seq[p + len(dom):]

    queries = []
    for i, n in enumerate(qlens):
        s = _random_seq(rng, int(n), AMINO, AMINO_FREQ)
        if rng.random() < f:
            s = plant(s, domain)
        queries.append(("query%d" % i, s))
    targets = []
    for i, n in enumerate(tlens):
        s = _random_seq(rng, int(n), AMINO, AMINO_FREQ)
        if rng.random() < f:
            s = plant(s, _mutate(rng, domain, AMINO, 1.0 - domain_identity, AMINO_FREQ))
        targets.append(("target%d" % i, s))
    queries.sort(key=lambda r: len(r[1]), reverse=True)
    targets.sort(key=lambda r: len(r[1]), reverse=True)
    return queries, targets


class Settings(object):
    """pyPaSWAS option names (pyPaSWAS/__init__.py:71-251) with string values,
    defaults from pyPaSWAS/Core/cfg/defaults.cfg."""

    DEFAULTS = dict(out_format="TXT", program="aligner", gap_score="-5", gap_extension="0", match_score="5",
                    mismatch_score="-3", other_score="-1", any_score="0", matrix_name="DNA-RNA",
                    lower_limit_score="1.0", minimum_score="30", filter_factor="0.2", query_coverage="0.2",
                    query_identity="0.2", relative_score="2.0", base_score="2.0", device_number="0",
                    maximum_memory_usage="0.8", limit_length="100000", max_genome_length="100000", recompile="T",
                    short_sequences="F", framework="CUDA", device_type="GPU", custom_matrix=None)

    def __init__(self, **kw):
        for k, v in self.DEFAULTS.items():
            setattr(self, k, v)
        for k, v in kw.items():
            setattr(self, k, v)


# Threshold knobs the benchmark configurations leave open, recorded here.
C1_SETTINGS = dict(matrix_name="DNA-RNA", match_score="1", mismatch_score="-3", gap_score="-5", gap_extension="0",
                   any_score="1", minimum_score="15", lower_limit_score="1.0", filter_factor="0.2",
                   relative_score="0", base_score="0", query_identity="0", query_coverage="0")
C2_SETTINGS = dict(matrix_name="BLOSUM62", gap_score="-11", gap_extension="-1", minimum_score="30",
                   lower_limit_score="1.0", filter_factor="0.2", relative_score="0", base_score="0",
                   query_identity="0", query_coverage="0")


def config1(seed=1):
    q, t = dna_reads_vs_adapters(seed)
    return Workload("C1 DNA reads x adapters (+RC), linear gap", q, t, Settings(**C1_SETTINGS))


def config2(seed=2, **kw):
    q, t = protein_batched(seed, **kw)
    return Workload("C2 protein 200 x 2000, BLOSUM62 affine -11/-1", q, t, Settings(**C2_SETTINGS))
