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
    def n_queries(self):
        return len(self.queries) if self.queries is not None else int(self.reads.shape[0])

    def head(self, n_queries):
        """The same workload on its first n queries (all targets; explicit
        pairs kept where both ends remain)."""
        qs = self.queries[:n_queries] if self.queries is not None else [
            (self.read_ids[i], self.reads[i].tobytes()) for i in range(min(n_queries, len(self.read_ids)))]
        pairs = None if self.pairs is None else [(q, t) for q, t in self.pairs if q < n_queries]
        return Workload("%s, first %d queries" % (self.name, len(qs)), qs, self.targets, self.settings, pairs)

    @property
    def cells(self):
        if self.queries is None:  # packed reads
            return int(self.reads.shape[0]) * int(self.reads.shape[1]) * sum(len(s) for _, s in self.targets)
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


C3_SETTINGS = dict(matrix_name="DNA-RNA", match_score="1", mismatch_score="-3", gap_score="-5", gap_extension="0",
                   any_score="1", minimum_score="100", lower_limit_score="1.0", filter_factor="0.01",
                   relative_score="0", base_score="0", query_identity="0", query_coverage="0")
C4_SETTINGS = dict(C1_SETTINGS, program="trimmer", out_format="trimmedFasta", minimum_score="8")
C5_SETTINGS = dict(C2_SETTINGS)


def config1(seed=1):
    q, t = dna_reads_vs_adapters(seed)
    return Workload("C1 DNA reads x adapters (+RC), linear gap", q, t, Settings(**C1_SETTINGS))


def config2(seed=2, **kw):
    q, t = protein_batched(seed, **kw)
    return Workload("C2 protein 200 x 2000, BLOSUM62 affine -11/-1", q, t, Settings(**C2_SETTINGS))


def long_dna_pairs(seed=3, n_pairs=64, length=(10000, 50000), shared=(2000, 20000), identity=0.85,
                   indel_rate=0.02):
    """Pairs of uniform-ACGT sequences sharing one homologous region: the region
    is planted in the query as drawn and in the target with (1 - identity)
    substitutions and the stated indel rate.  Returns (queries, targets, pairs)
    where target i + n_pairs is the reverse complement of target i and each
    query i is paired with targets i and i + n_pairs."""
    rng = np.random.default_rng(seed)
    queries, fwd = [], []
    for i in range(n_pairs):
        lq = int(rng.integers(length[0], length[1] + 1))
        lt = int(rng.integers(length[0], length[1] + 1))
        ls = int(rng.integers(shared[0], min(shared[1], lq, lt) + 1))
        region = _random_seq(rng, ls, DNA)
        q = _random_seq(rng, lq, DNA)
        t = _random_seq(rng, lt, DNA)
        pq = int(rng.integers(0, lq - ls + 1))
        q = q[:pq] + region + q[pq + ls:]
        hom = _mutate(rng, region, DNA, 1.0 - identity, indel_rate=indel_rate)
        pt = int(rng.integers(0, max(1, lt - len(hom)) + 1))
        t = (t[:pt] + hom + t[pt + len(hom):])[:max(lt, len(hom))]
        queries.append(("long%d" % i, q))
        fwd.append(("ref%d" % i, t))
    targets = fwd + [(tid + "_RC", reverse_complement(s)) for tid, s in fwd]
    pairs = [(i, i) for i in range(n_pairs)] + [(i, i + n_pairs) for i in range(n_pairs)]
    return queries, targets, pairs


def trimmer_reads(seed=4, n_reads=10_000_000, read_len=150, n_adapters=24, adapter_len=(20, 40), planted=0.40,
                  frag_len=(8, 40), max_subs=3):
    """Reads of uniform ACGT; in a fraction of them the 3' end is replaced by a
    prefix fragment of one adapter (length 8-40, clipped to the adapter) with
    0-3 substitutions.  Targets: the adapters plus their reverse complements.
    Vectorised: 10 M reads take a few seconds."""
    rng = np.random.default_rng(seed)
    adapters = [_random_seq(rng, int(rng.integers(adapter_len[0], adapter_len[1] + 1)), DNA)
                for _ in range(n_adapters)]
    reads = DNA[rng.integers(0, 4, size=(n_reads, read_len), dtype=np.uint8)]
    carry = np.nonzero(rng.random(n_reads) < planted)[0]
    which = rng.integers(0, n_adapters, size=len(carry))
    flen = rng.integers(frag_len[0], frag_len[1] + 1, size=len(carry))
    nsub = rng.integers(0, max_subs + 1, size=len(carry))
    amat = np.zeros((n_adapters, adapter_len[1]), dtype=np.uint8)
    alen = np.array([len(a) for a in adapters])
    for i, a in enumerate(adapters):
        amat[i, :len(a)] = np.frombuffer(a, dtype=np.uint8)
    n = np.minimum(flen, alen[which])
    for m in np.unique(n):
        sel = np.nonzero(n == m)[0]
        reads[carry[sel], read_len - m:] = amat[which[sel], :m]
    for s in range(1, max_subs + 1):
        sel = np.nonzero(nsub >= s)[0]
        pos = read_len - n[sel] + (rng.random(len(sel)) * n[sel]).astype(int)
        reads[carry[sel], pos] = DNA[rng.integers(0, 4, size=len(sel))]
    ids = ["read%d" % i for i in range(n_reads)]
    targets = [("adapter%d" % i, a) for i, a in enumerate(adapters)]
    targets += [(tid + "_RC", reverse_complement(s)) for tid, s in targets]
    targets.sort(key=lambda r: len(r[1]), reverse=True)
    return ids, reads, targets


def protein_database(seed=5, n_seqs=100_000, median=300.0, sigma=0.5, clip=(50, 1500)):
    """Resident database: log-normal lengths, background residue frequencies."""
    rng = np.random.default_rng(seed)
    lens = np.clip(np.round(rng.lognormal(np.log(median), sigma, n_seqs)), clip[0], clip[1]).astype(int)
    flat = AMINO[rng.choice(len(AMINO), size=int(lens.sum()), p=AMINO_FREQ)].tobytes()
    out, o = [], 0
    for i, n in enumerate(lens):
        out.append(("db%d" % i, flat[o:o + int(n)]))
        o += int(n)
    return out


def query_stream(seed=6, n=1000, median=300.0, sigma=0.5, max_len=5000, min_len=20, rate_hz=100.0,
                 traceback_fraction=0.30):
    """Poisson arrivals: (arrival_s, id, sequence, full_traceback) tuples."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_hz, size=n)
    t = np.cumsum(gaps) - gaps[0]
    lens = np.clip(np.round(rng.lognormal(np.log(median), sigma, n)), min_len, max_len).astype(int)
    tb = rng.random(n) < traceback_fraction
    return [(float(t[i]), "req%d" % i, _random_seq(rng, int(lens[i]), AMINO, AMINO_FREQ), bool(tb[i]))
            for i in range(n)]


def config3(seed=3, n_pairs=64, **kw):
    q, t, pairs = long_dna_pairs(seed, n_pairs=n_pairs, **kw)
    return Workload("C3 long DNA, %d pairs of 10-50 kb (+RC), linear gap" % n_pairs, q, t, Settings(**C3_SETTINGS),
                    pairs)


def config4(seed=4, n_reads=10_000_000):
    """Reads as one contiguous byte block: (ids, reads uint8[n, 150]) plus targets."""
    ids, reads, targets = trimmer_reads(seed, n_reads=n_reads)
    w = Workload("C4 trimmer, %d reads of 150 nt x 24 adapters (+RC)" % n_reads, None, targets,
                 Settings(**C4_SETTINGS))
    w.read_ids = ids
    w.reads = reads
    return w
