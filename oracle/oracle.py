"""Python wrapper around the C oracle (oracle/paswas_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, never by the engine.  The oracle is a literal CPU
restatement of the reference path; see the header of paswas_oracle.c.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpaswas_oracle.so")
SRC_PATH = os.path.join(HERE, "paswas_oracle.c")


def build(force=False):
    """Compiles the oracle with gcc (strict IEEE fp32: no contraction)."""
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= os.path.getmtime(SRC_PATH):
        return LIB_PATH
    tmp = LIB_PATH + ".tmp"
    subprocess.run(["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fno-fast-math", "-shared", "-fPIC",
                    "-o", tmp, SRC_PATH, "-lm"], check=True)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


class _Params(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("char_offset", ctypes.c_int), ("matrix", ctypes.c_void_p),
                ("gap", ctypes.c_float), ("ext", ctypes.c_float), ("affine", ctypes.c_int),
                ("lower_limit", ctypes.c_float), ("minimum_score", ctypes.c_float)]


START_DTYPE = np.dtype([("sequence", "<u4"), ("target", "<u4"), ("block_x", "<u4"), ("block_y", "<u4"),
                        ("value_x", "<u4"), ("value_y", "<u4"), ("score", "<f4"), ("max_score", "<f4"),
                        ("pos_score", "<f4")])
HIT_DTYPE = np.dtype([("query", "<i4"), ("target", "<i4"), ("s_start", "<i4"), ("s_end", "<i4"),
                      ("t_start", "<i4"), ("t_end", "<i4"), ("score", "<f4"), ("matches", "<i4"),
                      ("mismatches", "<i4"), ("n_cols", "<i4"), ("str_offset", "<i8")])

_lib = None


def _load():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        _lib.orc_run.restype = ctypes.c_int
        _lib.orc_pair_max.restype = None
    return _lib


def _pack(seqs):
    lens = np.array([len(s) for s in seqs], dtype=np.int64)
    off = np.zeros(len(seqs) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    buf = np.frombuffer(b"".join(s.encode("latin-1") if isinstance(s, str) else bytes(s) for s in seqs) or b"\0",
                        dtype=np.uint8).copy()
    return buf, off


class OracleParams(object):
    """Kernel constants as the reference compiles them (PaSWAS.py:55-72)."""

    def __init__(self, matrix, char_offset, gap, ext, affine, lower_limit, minimum_score):
        self.matrix = np.ascontiguousarray(matrix, dtype=np.float32)
        self.dim = int(self.matrix.shape[0])
        self.char_offset = int(char_offset)
        self.gap = np.float32(gap)
        self.ext = np.float32(ext)
        self.affine = bool(affine)
        self.lower_limit = np.float32(lower_limit)
        self.minimum_score = np.float32(minimum_score)

    def _c(self):
        return _Params(self.dim, self.char_offset, self.matrix.ctypes.data, float(self.gap), float(self.ext),
                       int(self.affine), float(self.lower_limit), float(self.minimum_score))


def pair_max(params, queries, targets):
    """Pair maxima [nq, nt] (calculateScore[AffineGap] block-maxima chain)."""
    lib = _load()
    qb, qo = _pack(queries)
    tb, to = _pack(targets)
    out = np.zeros((len(queries), len(targets)), dtype=np.float32)
    cp = params._c()
    lib.orc_pair_max(ctypes.byref(cp), len(queries), qb.ctypes.data_as(ctypes.c_void_p),
                     qo.ctypes.data_as(ctypes.c_void_p), len(targets), tb.ctypes.data_as(ctypes.c_void_p),
                     to.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p))
    return out


def run(params, queries, targets, pos_score, host_min_score, q_idkey=None, t_idkey=None, start_cap=-1):
    """Full path: pair maxima, starting points (emission order) and walked hits.

    queries/targets: upper-cased strings.  pos_score: [nt, nq] float32 like the
    reference's maxPossibleScore array.  Returns a dict."""
    lib = _load()
    nq, nt = len(queries), len(targets)
    qb, qo = _pack(queries)
    tb, to = _pack(targets)
    q_idkey = np.arange(nq, dtype=np.int32) if q_idkey is None else np.asarray(q_idkey, dtype=np.int32)
    t_idkey = (np.arange(nt, dtype=np.int32) + nq) if t_idkey is None else np.asarray(t_idkey, dtype=np.int32)
    pos = np.ascontiguousarray(pos_score, dtype=np.float32).reshape(nt, nq)
    pmax = np.zeros((nq, nt), dtype=np.float32)
    max_starts = max(1024, 4 * nq * nt)
    max_hits = max_starts
    str_cap = 1 << 22
    while True:
        starts = np.zeros(max_starts, dtype=START_DTYPE)
        hits = np.zeros(max_hits, dtype=HIT_DTYPE)
        strbuf = np.zeros(str_cap, dtype=np.uint8)
        n_starts, n_hits, used = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        cp = params._c()
        v = ctypes.c_void_p
        rc = lib.orc_run(ctypes.byref(cp), nq, qb.ctypes.data_as(v), qo.ctypes.data_as(v), nt,
                         tb.ctypes.data_as(v), to.ctypes.data_as(v), q_idkey.ctypes.data_as(v),
                         t_idkey.ctypes.data_as(v), pos.ctypes.data_as(v), ctypes.c_double(host_min_score),
                         ctypes.c_int64(start_cap), pmax.ctypes.data_as(v), starts.ctypes.data_as(v),
                         ctypes.c_int64(max_starts), ctypes.byref(n_starts), hits.ctypes.data_as(v),
                         ctypes.c_int64(max_hits), ctypes.byref(n_hits), strbuf.ctypes.data_as(v),
                         ctypes.c_int64(str_cap), ctypes.byref(used))
        if rc == 0:
            break
        max_starts = max(max_starts, int(n_starts.value) + 1)
        max_hits = max(max_hits, int(n_hits.value) + 1)
        str_cap = max(str_cap, int(used.value) + 1)
    hits = hits[: n_hits.value]
    sb = strbuf.tobytes()
    out_hits = []
    for h in hits:
        n, o = int(h["n_cols"]), int(h["str_offset"])
        out_hits.append({
            "query": int(h["query"]), "target": int(h["target"]),
            "s_start": int(h["s_start"]), "s_end": int(h["s_end"]),
            "t_start": int(h["t_start"]), "t_end": int(h["t_end"]),
            "score": float(h["score"]), "matches": int(h["matches"]), "mismatches": int(h["mismatches"]),
            "sequence_match": sb[o:o + n].decode("latin-1"),
            "alignment": sb[o + n:o + 2 * n].decode("latin-1"),
            "target_match": sb[o + 2 * n:o + 3 * n].decode("latin-1"),
        })
    return {"pair_max": pmax, "starts": starts[: n_starts.value], "hits": out_hits}
