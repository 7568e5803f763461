"""ctypes binding of libpaswas_b200.so (include/paswas_b200.h).

The library is built in-tree by ``pypaswas_b200.build`` (nvcc, sm_100a).  There
is no CPU fallback: when the library or a CUDA device is missing, loading or
creating an engine raises.
"""
import ctypes
import os

import numpy as np

from .exceptions import CudaException, HardwareException, InvalidOptionException

PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(PACKAGE_DIR, "libpaswas_b200.so")

PW_OK = 0
PW_ERR_ARG = -1
PW_ERR_DEVICE = -2
PW_ERR_KERNEL = -3
PW_ERR_NOMEM = -4
PW_ERR_CAPACITY = -5
PW_ERR_STATE = -6
PW_ERR_TIMEOUT = -7
PW_SERVE_TOP = 0
PW_SERVE_TRACEBACK = 1

PW_FLAG_SCORE_ONLY = 1
PW_FLAG_PLAIN = 2
PW_FLAG_INT32 = 4
PW_FLAG_NO_CHAIN = 8
PW_FLAG_REPLAN = 16
PW_TUNE_CHAIN_MIN = 0
PW_TUNE_GRID_SHARE = 1
PW_TUNE_SEGMENT = 2
PW_TUNE_DUAL = 3
PW_TUNE_CAND_SLOT = 4
PW_TUNE_WAIT_NS = 5
PW_TUNE_STALL_TEST = 6
PW_TUNE_LANES = 7
PW_TUNE_TRACE_STORE = 8
PW_TUNE_TILE_TRACE = 9
PW_SERVE_TUNE_POLICY = 100
PW_SERVE_TUNE_AGE_MS = 101
PW_SERVE_TUNE_MAX_BATCH = 102
PW_SERVE_TUNE_MAX_RESIDUES = 103
PW_FORMAT_FASTA = 0
PW_FORMAT_FASTQ = 1
PW_RECORDS_AS_READ = 0
PW_RECORDS_APPEND_RC = 1
PW_RECORDS_RC_ONLY = 2
PW_RECORDS_APPEND_REVERSED = 3
PW_REUSE_QUERIES = 1
PW_REUSE_TARGETS = 2
PW_REUSE_PLAN = 4

# symbols the header declares, checked by the CPU test-suite
EXPORTED_SYMBOLS = (
    "pw_create", "pw_destroy", "pw_last_error", "pw_device_free_memory", "pw_set_scoring",
    "pw_set_queries", "pw_set_targets", "pw_align", "pw_get_pair_max", "pw_get_hits", "pw_get_hits_view",
    "pw_get_starting_points", "pw_last_launch_count", "pw_measure_int_peak", "pw_score_max_noalloc",
    "pw_set_wave_limit", "pw_set_tuning", "pw_set_pairs", "pw_server_create", "pw_server_destroy", "pw_server_last_error", "pw_server_set_scoring",
    "pw_server_load_db", "pw_server_submit", "pw_server_wait", "pw_server_top_hits", "pw_server_hits",
    "pw_server_release", "pw_server_stats", "pw_server_tune", "pw_trimmed_fasta", "pw_txt_records",
    "pw_sam_records",
    "pw_records_parse", "pw_records_read", "pw_records_sizes", "pw_records_copy", "pw_records_free",
    "pw_id_ranks", "pw_set_query_trace",
)


class PwHit(ctypes.Structure):
    _fields_ = [("query", ctypes.c_int32), ("target", ctypes.c_int32), ("s_start", ctypes.c_int32),
                ("s_end", ctypes.c_int32), ("t_start", ctypes.c_int32), ("t_end", ctypes.c_int32),
                ("score", ctypes.c_float), ("matches", ctypes.c_int32), ("mismatches", ctypes.c_int32),
                ("n_cols", ctypes.c_int32), ("str_offset", ctypes.c_int64)]


HIT_DTYPE = np.dtype([("query", "<i4"), ("target", "<i4"), ("s_start", "<i4"), ("s_end", "<i4"),
                      ("t_start", "<i4"), ("t_end", "<i4"), ("score", "<f4"), ("matches", "<i4"),
                      ("mismatches", "<i4"), ("n_cols", "<i4"), ("str_offset", "<i8")])
assert HIT_DTYPE.itemsize == ctypes.sizeof(PwHit)

START_DTYPE = np.dtype([("sequence", "<u4"), ("target", "<u4"), ("block_x", "<u4"), ("block_y", "<u4"),
                        ("value_x", "<u4"), ("value_y", "<u4"), ("score", "<f4"), ("max_score", "<f4"),
                        ("pos_score", "<f4")])


class PwRunInfo(ctypes.Structure):
    _fields_ = [("pairs", ctypes.c_int64), ("cells", ctypes.c_int64), ("traced_pairs", ctypes.c_int64),
                ("minimum_pairs", ctypes.c_int64),
                ("starting_points", ctypes.c_int64), ("hits", ctypes.c_int64), ("string_bytes", ctypes.c_int64),
                ("kernel_launches", ctypes.c_int32), ("truncated", ctypes.c_int32), ("score_ms", ctypes.c_double),
                ("trace_ms", ctypes.c_double), ("walk_ms", ctypes.c_double),
                ("score_kernel_ms", ctypes.c_double), ("trace_kernel_ms", ctypes.c_double),
                ("score_launches", ctypes.c_int32), ("trace_launches", ctypes.c_int32),
                ("orientation", ctypes.c_int32), ("trace_orientation", ctypes.c_int32),
                ("overflow_pairs", ctypes.c_int64), ("traced_cells", ctypes.c_int64),
                ("warp_pairs", ctypes.c_int64), ("cand_overflow_pairs", ctypes.c_int64),
                ("setup_ms", ctypes.c_double), ("finish_ms", ctypes.c_double), ("total_ms", ctypes.c_double),
                ("score_path", ctypes.c_int32), ("dual_lanes", ctypes.c_int32),
                ("waves", ctypes.c_int32), ("reuse", ctypes.c_int32),
                ("h2d_bytes", ctypes.c_int64), ("d2h_bytes", ctypes.c_int64),
                ("trace_store", ctypes.c_int32), ("tile_pairs", ctypes.c_int32),
                ("paired_cells", ctypes.c_int64)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class PwRequestInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("mode", ctypes.c_int32), ("batch_queries", ctypes.c_int32),
                ("worker", ctypes.c_int32), ("cells", ctypes.c_int64), ("n_hits", ctypes.c_int64),
                ("string_bytes", ctypes.c_int64), ("reserved_bytes", ctypes.c_int64), ("queue_ms", ctypes.c_double),
                ("run_ms", ctypes.c_double), ("latency_ms", ctypes.c_double),
                ("batch_score_kernel_ms", ctypes.c_double), ("batch_setup_ms", ctypes.c_double),
                ("batch_call_ms", ctypes.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class PwServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("batches", ctypes.c_int64),
                ("cells", ctypes.c_int64), ("pending", ctypes.c_int64), ("budget_bytes", ctypes.c_int64),
                ("reserved_bytes", ctypes.c_int64), ("peak_reserved_bytes", ctypes.c_int64),
                ("busy_ms", ctypes.c_double), ("traced_fraction", ctypes.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


def bind(lib):
    """Declares the argument and result types of every exported function."""
    P, I32, I64, U32, F, D = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint32, ctypes.c_float, \
        ctypes.c_double
    sig = {
        "pw_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
        "pw_destroy": (None, [P]),
        "pw_last_error": (ctypes.c_char_p, [P]),
        "pw_device_free_memory": (ctypes.c_int, [P, ctypes.POINTER(I64), ctypes.POINTER(I64)]),
        "pw_set_scoring": (ctypes.c_int, [P, P, ctypes.c_int, ctypes.c_int, F, F, ctypes.c_int, F, F, D, D, D]),
        "pw_set_queries": (ctypes.c_int, [P, P, P, I32, P]),
        "pw_set_targets": (ctypes.c_int, [P, P, P, I32, P]),
        "pw_align": (ctypes.c_int, [P, U32, I64, ctypes.POINTER(PwRunInfo)]),
        "pw_get_pair_max": (ctypes.c_int, [P, P, I64]),
        "pw_get_hits": (ctypes.c_int, [P, P, I64, P, I64]),
        "pw_get_hits_view": (ctypes.c_int, [P, P, P, P, P]),
        "pw_get_starting_points": (ctypes.c_int, [P, P, I64, ctypes.POINTER(I64)]),
        "pw_last_launch_count": (ctypes.c_int, [P, ctypes.POINTER(I64)]),
        "pw_measure_int_peak": (ctypes.c_int, [P, ctypes.POINTER(D), ctypes.POINTER(D), ctypes.POINTER(D)]),
        "pw_score_max_noalloc": (ctypes.c_int, [ctypes.c_int, P, ctypes.c_int, ctypes.c_int, F, F, ctypes.c_int,
                                                P, P, I32, P, P, I32, P, ctypes.c_char_p, I32]),
        "pw_set_wave_limit": (ctypes.c_int, [P, I64]),
        "pw_set_tuning": (ctypes.c_int, [P, ctypes.c_int, I64]),
        "pw_set_pairs": (ctypes.c_int, [P, P, P, I64]),
        "pw_server_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, I64,
                                            ctypes.POINTER(ctypes.c_void_p)]),
        "pw_server_destroy": (None, [P]),
        "pw_server_last_error": (ctypes.c_char_p, [P]),
        "pw_server_set_scoring": (ctypes.c_int, [P, P, ctypes.c_int, ctypes.c_int, F, F, ctypes.c_int, F, F, D, D,
                                                 D]),
        "pw_server_load_db": (ctypes.c_int, [P, P, P, I32, P]),
        "pw_server_submit": (ctypes.c_int, [P, P, I64, I32, I32, ctypes.POINTER(I64)]),
        "pw_server_wait": (ctypes.c_int, [P, I64, I32, ctypes.POINTER(PwRequestInfo)]),
        "pw_server_top_hits": (ctypes.c_int, [P, I64, P, P, I32]),
        "pw_server_hits": (ctypes.c_int, [P, I64, P, I64, P, I64]),
        "pw_server_release": (ctypes.c_int, [P, I64]),
        "pw_server_stats": (ctypes.c_int, [P, ctypes.POINTER(PwServerStats)]),
        "pw_server_tune": (ctypes.c_int, [P, ctypes.c_int, I64]),
        "pw_trimmed_fasta": (ctypes.c_int, [P, I64, I32, I32, P, P, P, P, P, P, P, P, P, P, P, P, P, P, I64,
                                            ctypes.POINTER(I64)]),
        "pw_txt_records": (ctypes.c_int, [P, I64, I32, I32, P, I64, P, P, P, P, P, P, P, P, P, P, P, P, I64,
                                          ctypes.POINTER(I64)]),
        "pw_sam_records": (ctypes.c_int, [P, I64, I32, I32, P, I64, P, P, P, P, P, P, P, P, P, P, P, P, P, P,
                                          I64, ctypes.POINTER(I64)]),
        "pw_records_parse": (ctypes.c_int, [P, I64, ctypes.c_int, I64, I64, I64, ctypes.c_int, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p, I32]),
        "pw_records_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, I64, I64, I64, ctypes.c_int,
                                           ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p, I32]),
        "pw_records_sizes": (ctypes.c_int, [P, ctypes.POINTER(I64), ctypes.POINTER(I64), ctypes.POINTER(I64),
                                            ctypes.POINTER(I64)]),
        "pw_records_copy": (ctypes.c_int, [P, P, P, P, P]),
        "pw_records_free": (None, [P]),
        "pw_id_ranks": (ctypes.c_int, [P, P, I64, P]),
        "pw_set_query_trace": (ctypes.c_int, [P, P, I32]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = None


def load_library():
    """Loads the in-tree engine library; raises HardwareException when absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY_PATH):
            raise HardwareException("libpaswas_b200.so is not built (run pypaswas_b200.build.build())")
        _lib = bind(ctypes.CDLL(LIBRARY_PATH))
    return _lib


def _check(lib, handle, rc, what):
    if rc == PW_OK:
        return
    msg = lib.pw_last_error(handle) if handle else None
    msg = "%s failed (%d): %s" % (what, rc, msg.decode() if msg else "")
    if rc == PW_ERR_ARG:
        raise InvalidOptionException(msg)
    if rc == PW_ERR_DEVICE:
        raise HardwareException(msg)
    raise CudaException(msg)


# a new bytes object of n bytes, its contents not yet written
_new_bytes = ctypes.pythonapi.PyBytes_FromStringAndSize
_new_bytes.restype = ctypes.py_object
_new_bytes.argtypes = (ctypes.c_void_p, ctypes.c_ssize_t)


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None and a.size else ctypes.c_void_p(0)


def pack_sequences(seqs):
    """Concatenates byte strings; returns (residues uint8, offsets int64)."""
    lens = np.fromiter((len(s) for s in seqs), dtype=np.int64, count=len(seqs))
    off = np.zeros(len(seqs) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    buf = np.frombuffer(b"".join(seqs), dtype=np.uint8) if len(seqs) else np.zeros(0, np.uint8)
    return np.ascontiguousarray(buf), off


class Engine(object):
    """One device engine (one CUDA stream).  Thin, stateful wrapper of the C ABI."""

    def __init__(self, device=0, lib=None):
        self.lib = lib if lib is not None else load_library()
        h = ctypes.c_void_p()
        rc = self.lib.pw_create(int(device), ctypes.byref(h))
        if rc != PW_OK:
            raise HardwareException("Failed to initialize device %d (status %d)" % (device, rc))
        self.handle = h
        self.n_queries = 0
        self.n_targets = 0
        self.last_info = None

    def close(self):
        if getattr(self, "handle", None):
            self.lib.pw_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def free_memory(self):
        f, t = ctypes.c_int64(), ctypes.c_int64()
        _check(self.lib, self.handle, self.lib.pw_device_free_memory(self.handle, ctypes.byref(f), ctypes.byref(t)),
               "pw_device_free_memory")
        return f.value, t.value

    def set_scoring(self, matrix, char_offset, gap, ext, affine, lower_limit, minimum_score, host_minimum,
                    highest, filter_factor):
        m = np.ascontiguousarray(matrix, dtype=np.float32)
        self._matrix = m
        rc = self.lib.pw_set_scoring(self.handle, _ptr(m), int(m.shape[0]), int(char_offset), float(gap), float(ext),
                                     int(bool(affine)), float(lower_limit), float(minimum_score), float(host_minimum),
                                     float(highest), float(filter_factor))
        _check(self.lib, self.handle, rc, "pw_set_scoring")

    def set_queries(self, seqs, id_keys):
        buf, off = pack_sequences(seqs)
        keys = np.ascontiguousarray(id_keys, dtype=np.int32)
        _check(self.lib, self.handle,
               self.lib.pw_set_queries(self.handle, _ptr(buf), _ptr(off), len(seqs), _ptr(keys)), "pw_set_queries")
        self.n_queries = len(seqs)

    def set_queries_packed(self, residues, offsets, id_keys):
        """Queries as one concatenated uint8 array plus int64 offsets (n + 1):
        no per-sequence Python objects (millions of reads)."""
        buf = np.ascontiguousarray(residues, dtype=np.uint8).reshape(-1)
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        keys = np.ascontiguousarray(id_keys, dtype=np.int32)
        n = len(off) - 1
        _check(self.lib, self.handle, self.lib.pw_set_queries(self.handle, _ptr(buf), _ptr(off), n, _ptr(keys)),
               "pw_set_queries")
        self.n_queries = n

    def set_targets_packed(self, residues, offsets, id_keys):
        """Targets as one concatenated uint8 array plus int64 offsets (n + 1)."""
        buf = np.ascontiguousarray(residues, dtype=np.uint8).reshape(-1)
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        keys = np.ascontiguousarray(id_keys, dtype=np.int32)
        n = len(off) - 1
        _check(self.lib, self.handle, self.lib.pw_set_targets(self.handle, _ptr(buf), _ptr(off), n, _ptr(keys)),
               "pw_set_targets")
        self.n_targets = n

    def set_targets(self, seqs, id_keys):
        buf, off = pack_sequences(seqs)
        keys = np.ascontiguousarray(id_keys, dtype=np.int32)
        _check(self.lib, self.handle,
               self.lib.pw_set_targets(self.handle, _ptr(buf), _ptr(off), len(seqs), _ptr(keys)), "pw_set_targets")
        self.n_targets = len(seqs)

    def align(self, score_only=False, plain=False, start_cap=-1, int32=False, chain=True, replan=False):
        info = PwRunInfo()
        flags = (PW_FLAG_SCORE_ONLY if score_only else 0) | (PW_FLAG_PLAIN if plain else 0) | \
            (PW_FLAG_INT32 if int32 else 0) | (0 if chain else PW_FLAG_NO_CHAIN) | (PW_FLAG_REPLAN if replan else 0)
        rc = self.lib.pw_align(self.handle, flags, int(start_cap), ctypes.byref(info))
        _check(self.lib, self.handle, rc, "pw_align")
        self.last_info = info
        return info

    def pair_max(self):
        out = np.zeros((self.n_queries, self.n_targets), dtype=np.float32)
        _check(self.lib, self.handle, self.lib.pw_get_pair_max(self.handle, _ptr(out), out.size), "pw_get_pair_max")
        return out

    def hits(self, strings=True):
        """Returns (structured array of hits in HitList order, string bytes);
        strings=False skips the alignment strings (b"")."""
        n = int(self.last_info.hits) if self.last_info is not None else 0
        nb = int(self.last_info.string_bytes) if self.last_info is not None and strings else 0
        hits = np.empty(n, dtype=HIT_DTYPE)
        if not strings:
            _check(self.lib, self.handle, self.lib.pw_get_hits(self.handle, _ptr(hits) if n else None, n, None, 0),
                   "pw_get_hits")
            return hits, b""
        if nb < 2:
            strbuf = np.empty(max(nb, 1), dtype=np.uint8)
            _check(self.lib, self.handle, self.lib.pw_get_hits(self.handle, _ptr(hits) if n else None, n,
                                                                _ptr(strbuf), nb), "pw_get_hits")
            return hits, strbuf[:nb].tobytes()
        # the strings go straight into a new, unshared bytes object (one copy)
        text = _new_bytes(None, nb)
        _check(self.lib, self.handle, self.lib.pw_get_hits(self.handle, _ptr(hits) if n else None, n,
                                                            ctypes.cast(ctypes.c_char_p(text), ctypes.c_void_p),
                                                            nb), "pw_get_hits")
        return hits, text

    def hits_view(self):
        """(hit records, strings) of the last align without a copy: a numpy
        view and a memoryview of the engine's own host copies, valid until the
        next align or set_* call on this engine."""
        hp, n, sp, nb = ctypes.c_void_p(), ctypes.c_int64(), ctypes.c_void_p(), ctypes.c_int64()
        _check(self.lib, self.handle, self.lib.pw_get_hits_view(self.handle, ctypes.byref(hp), ctypes.byref(n),
                                                                 ctypes.byref(sp), ctypes.byref(nb)),
               "pw_get_hits_view")
        if n.value == 0:
            hits = np.zeros(0, dtype=HIT_DTYPE)
        else:
            raw = (ctypes.c_char * (n.value * HIT_DTYPE.itemsize)).from_address(hp.value)
            hits = np.frombuffer(raw, dtype=HIT_DTYPE)
        strings = memoryview((ctypes.c_char * nb.value).from_address(sp.value)).cast("B") if nb.value else \
            memoryview(b"")
        return hits, strings

    def starting_points(self):
        n = ctypes.c_int64()
        _check(self.lib, self.handle, self.lib.pw_get_starting_points(self.handle, None, 0, ctypes.byref(n)),
               "pw_get_starting_points")
        out = np.zeros(n.value, dtype=START_DTYPE)
        _check(self.lib, self.handle,
               self.lib.pw_get_starting_points(self.handle, _ptr(out), n.value, ctypes.byref(n)),
               "pw_get_starting_points")
        return out

    def measure_int_peak(self):
        """(ops/s on 32-bit lanes, ops/s on 16x2 lanes, probe ms) of the DPX add-max probes."""
        r32, r16, ms = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(self.lib, self.handle,
               self.lib.pw_measure_int_peak(self.handle, ctypes.byref(r32), ctypes.byref(r16), ctypes.byref(ms)),
               "pw_measure_int_peak")
        return r32.value, r16.value, ms.value

    def set_pairs(self, query_idx, target_idx):
        """Explicit (query, target) pairs for the next align() calls; empty lists restore all-vs-all."""
        qi = np.ascontiguousarray(query_idx, dtype=np.int32)
        ti = np.ascontiguousarray(target_idx, dtype=np.int32)
        if qi.shape != ti.shape:
            raise InvalidOptionException("query and target index lists differ in length")
        self._pairs = (qi, ti)
        _check(self.lib, self.handle, self.lib.pw_set_pairs(self.handle, _ptr(qi), _ptr(ti), len(qi)), "pw_set_pairs")

    def set_tuning(self, key, value):
        _check(self.lib, self.handle, self.lib.pw_set_tuning(self.handle, int(key), int(value)), "pw_set_tuning")

    def set_query_trace(self, mask):
        """Per query: traced (nonzero) or maxima only (0); None clears the mask."""
        if mask is None:
            _check(self.lib, self.handle, self.lib.pw_set_query_trace(self.handle, None, 0), "pw_set_query_trace")
            return
        m = np.ascontiguousarray(np.asarray(mask) != 0, dtype=np.uint8)
        _check(self.lib, self.handle, self.lib.pw_set_query_trace(self.handle, _ptr(m), len(m)), "pw_set_query_trace")

    def set_wave_limit(self, nbytes):
        _check(self.lib, self.handle, self.lib.pw_set_wave_limit(self.handle, int(nbytes)), "pw_set_wave_limit")

    def launch_count(self):
        n = ctypes.c_int64()
        _check(self.lib, self.handle, self.lib.pw_last_launch_count(self.handle, ctypes.byref(n)),
               "pw_last_launch_count")
        return n.value


def score_max_noalloc(device, matrix, char_offset, gap, ext, affine, queries, targets, lib=None):
    """Pair maxima [n_queries, n_targets] through pw_score_max_noalloc: the
    library allocates no device memory for this call (see the header)."""
    lib = lib if lib is not None else load_library()
    m = np.ascontiguousarray(matrix, dtype=np.float32)
    qb, qo = pack_sequences(queries)
    tb, to = pack_sequences(targets)
    out = np.zeros((len(queries), len(targets)), dtype=np.float32)
    err = ctypes.create_string_buffer(512)
    rc = lib.pw_score_max_noalloc(int(device), _ptr(m), int(m.shape[0]), int(char_offset), float(gap), float(ext),
                                  int(bool(affine)), _ptr(qb), _ptr(qo), len(queries), _ptr(tb), _ptr(to),
                                  len(targets), _ptr(out), err, len(err))
    if rc != PW_OK:
        msg = "pw_score_max_noalloc failed (%d): %s" % (rc, err.value.decode())
        if rc == PW_ERR_ARG:
            raise InvalidOptionException(msg)
        if rc == PW_ERR_DEVICE:
            raise HardwareException(msg)
        raise CudaException(msg)
    return out
