"""Runs the reference pyPaSWAS host code (unmodified, imported read-only from the
reference tree) on top of the reference's own CUDA kernels compiled for the CPU
by ``build_ref.py``.

TEST INFRASTRUCTURE ONLY (oracle).  Used in this container to generate golden
fixtures (tests/golden/make_golden.py); it never runs on the GPU box.

What is the reference's own code here:
  * pyPaSWAS/Core/SmithWaterman.py  -- batching, launch loops (:592-655), the
    host traceback walk ``_print_alignments`` (:665-841), the hit filter;
  * pyPaSWAS/Core/SmithWatermanCuda.py -- buffer shapes, ``_set_max_possible_score``
    (:269-275), direction-array view (:287-298); only the device calls are
    replaced by the emulated launches below;
  * pyPaSWAS/Core/Programs.py Aligner/Trimmer.process, Hit, HitList, StartingPoint;
  * the kernels pyPaSWAS/Core/cuda/default_main.cu via build_ref.py.
What is ours: stand-ins for the packages that are absent here (Bio.Seq /
Bio.SeqRecord, pycuda), two NumPy-2 compatibility patches (``numpy.fromstring``
binary mode and ``numpy.asscalar`` were removed), and the memory emulation.

Pinned choices (the reference is nondeterministic or undefined here):
  * starting points are emitted in the emulator's linear thread order, so equal
    scores are walked in a fixed order (the GPU's atomicAdd order is unordered);
  * the zero-copy direction buffer is zeroed before every batch
    ("fresh allocation" semantics; the reference reuses a pinned buffer between
    same-shape batches without clearing it);
  * the device-side starting-point buffer has room for 1000 points per pair
    (the size the kernel assumes, default_main.cu:22), so overflow of the
    host's 100-per-pair view is truncation, never memory corruption.
"""
import ctypes
import logging
import math
import os
import sys
import types
import warnings

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import build_ref  # noqa: E402

REFERENCE_ROOT = build_ref.REFERENCE_ROOT

_IUPAC_COMPLEMENT = {
    "A": "T", "C": "G", "G": "C", "T": "A", "U": "A", "M": "K", "R": "Y", "W": "W", "S": "S",
    "Y": "R", "K": "M", "V": "B", "H": "D", "D": "H", "B": "V", "X": "X", "N": "N",
}


class _Seq(object):
    """Minimal stand-in for Bio.Seq.Seq (string semantics only)."""

    def __init__(self, data, alphabet=None):
        self._data = str(data)
        self.alphabet = alphabet

    def __str__(self):
        return self._data

    def __repr__(self):
        return "Seq(%r)" % self._data

    def __len__(self):
        return len(self._data)

    def __getitem__(self, i):
        if isinstance(i, slice):
            return _Seq(self._data[i], self.alphabet)
        return self._data[i]

    def __add__(self, other):
        return _Seq(self._data + str(other), self.alphabet)

    def __eq__(self, other):
        return self._data == str(other)

    def __hash__(self):
        return hash(self._data)

    def upper(self):
        return _Seq(self._data.upper(), self.alphabet)

    def lower(self):
        return _Seq(self._data.lower(), self.alphabet)

    def reverse_complement(self):
        out = []
        for ch in reversed(self._data):
            c = _IUPAC_COMPLEMENT.get(ch.upper(), ch.upper())
            out.append(c if ch.isupper() else c.lower())
        return _Seq("".join(out), self.alphabet)


class _SeqRecord(object):
    """Minimal stand-in for Bio.SeqRecord.SeqRecord."""

    def __init__(self, seq, id="<unknown id>", name="<unknown name>", description="<unknown description>"):
        self.seq = seq
        self.id = id
        self.name = name
        self.description = description

    def __len__(self):
        return len(self.seq)

    def __getitem__(self, i):
        return self.seq[i]


def _install_stand_ins():
    if "Bio" not in sys.modules:
        bio = types.ModuleType("Bio")
        bio_seq = types.ModuleType("Bio.Seq")
        bio_seq.Seq = _Seq
        bio_rec = types.ModuleType("Bio.SeqRecord")
        bio_rec.SeqRecord = _SeqRecord
        bio_io = types.ModuleType("Bio.SeqIO")
        bio.Seq, bio.SeqRecord, bio.SeqIO = bio_seq, bio_rec, bio_io
        sys.modules.update({"Bio": bio, "Bio.Seq": bio_seq, "Bio.SeqRecord": bio_rec, "Bio.SeqIO": bio_io})
    if "pycuda" not in sys.modules:
        pycuda = types.ModuleType("pycuda")
        drv = types.ModuleType("pycuda.driver")
        drv.Context = None
        comp = types.ModuleType("pycuda.compiler")
        comp.SourceModule = None
        pycuda.driver, pycuda.compiler = drv, comp
        sys.modules.update({"pycuda": pycuda, "pycuda.driver": drv, "pycuda.compiler": comp})
    # NumPy 2 removed binary-mode fromstring and asscalar, both used by
    # StartingPoint.parse_byte_string (StartingPoint.py:43-75).
    if not getattr(numpy, "_paswas_ref_patched", False):
        numpy.fromstring = lambda s, dtype=float, **kw: numpy.frombuffer(
            numpy.ascontiguousarray(s).tobytes(), dtype=dtype)
        numpy.asscalar = lambda a: a.item()
        # NumPy 2 refuses the abstract ``numpy.character`` as a dtype; the
        # reference uses it to build whole-string byte arrays
        # (SmithWaterman.py:162,412,514), which is what ``bytes_`` gives.
        numpy.character = numpy.bytes_
        numpy._paswas_ref_patched = True
    if REFERENCE_ROOT not in sys.path:
        sys.path.insert(0, REFERENCE_ROOT)


_install_stand_ins()
with warnings.catch_warnings():
    warnings.simplefilter("ignore")
    from pyPaSWAS.Core import Scores as ref_scores  # noqa: E402
    from pyPaSWAS.Core.SmithWatermanCuda import SmithWatermanCuda  # noqa: E402
    from pyPaSWAS.Core.SWSeqRecord import SWSeqRecord  # noqa: E402
    from pyPaSWAS.Core.HitList import HitList  # noqa: E402
    from pyPaSWAS.Core import Programs  # noqa: E402
    from pyPaSWAS.Core import Formatters  # noqa: E402
    from pyPaSWAS.Core.Exceptions import CudaException  # noqa: E402


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


class SmithWatermanEmu(SmithWatermanCuda):
    """The reference CUDA backend with its device calls routed to the emulated
    reference kernels.  ``device_memory`` stands in for free device memory and
    so controls the reference's own batching (SmithWaterman.py:202-221)."""

    def __init__(self, logger, score, settings, device_memory=8 << 30):
        self.device_memory = int(device_memory)
        self.lib = None
        self.raw_batches = []
        self.batch_offsets = []
        SmithWatermanCuda.__init__(self, logger, score, settings)

    def __del__(self):
        pass

    def _initialize_device(self, device_number):
        pass

    def _device_global_mem_size(self):
        return self.device_memory

    def _clear_memory(self):
        for name in ("d_sequences", "d_targets", "d_matrix", "d_matrix_i", "d_matrix_j", "d_global_maxima",
                     "d_global_direction", "h_starting_points_zero_copy", "h_global_direction_zero_copy",
                     "d_max_possible_score_zero_copy"):
            setattr(self, name, None)

    def _init_memory(self):
        nx, ny, ns, nt = (self.length_of_x_sequences, self.length_of_y_sequences,
                          self.number_of_sequences, self.number_targets)
        cells = nx * ny * ns * nt
        self.d_sequences = numpy.zeros(nx * ns, dtype=numpy.uint8)
        self.d_targets = numpy.zeros(ny * nt, dtype=numpy.uint8)
        self.d_matrix = numpy.zeros(cells, dtype=numpy.float32)
        if self.gap_extension:
            self.d_matrix_i = numpy.zeros(cells, dtype=numpy.float32)
            self.d_matrix_j = numpy.zeros(cells, dtype=numpy.float32)
        self.d_global_maxima = numpy.zeros(self.x_div_shared_x * self.y_div_shared_y * ns * nt, dtype=numpy.float32)
        self.d_global_direction = numpy.zeros(cells, dtype=numpy.uint8)
        # room for the kernel's own bound of 1000 points per pair (default_main.cu:22)
        self.h_starting_points_zero_copy = numpy.zeros((self.size_of_startingpoint * 1000 * ns * nt, 1),
                                                       dtype=numpy.int8)
        self.h_global_direction_zero_copy = numpy.zeros((cells, 1), dtype=numpy.int8)
        self.d_max_possible_score_zero_copy = numpy.zeros(ns * self.number_of_targets, dtype=numpy.float32)
        self.d_index_increment = numpy.zeros(1, dtype=numpy.uint32)

    def _init_zero_copy(self):
        self.d_index_increment[0] = 0
        self.h_global_direction_zero_copy[:] = 0  # pinned: fresh-allocation semantics

    def _compile_code(self):
        so = build_ref.build(self.score, self.number_of_sequences, self.number_targets,
                             self.length_of_x_sequences, self.length_of_y_sequences, "cuda")
        self.lib = ctypes.CDLL(so)

    def copy_sequences(self, h_sequences, h_targets):
        s = numpy.frombuffer(numpy.ascontiguousarray(h_sequences).tobytes(), dtype=numpy.uint8)
        t = numpy.frombuffer(numpy.ascontiguousarray(h_targets).tobytes(), dtype=numpy.uint8)
        self.d_sequences[: len(s)] = s
        self.d_targets[: len(t)] = t

    def _copy_min_score(self):
        n = min(len(self.min_score_np), len(self.d_max_possible_score_zero_copy))
        self.d_max_possible_score_zero_copy[:n] = self.min_score_np[:n]

    def _execute_calculate_score_kernel(self, number_of_blocks, idx, idy):
        gx, gy = self.number_of_sequences, self.number_targets * number_of_blocks
        u = ctypes.c_uint
        if self.gap_extension:
            self.lib.emu_calculateScoreAffineGap(u(gx), u(gy), _ptr(self.d_matrix), _ptr(self.d_matrix_i),
                                                 _ptr(self.d_matrix_j), u(idx), u(idy), u(number_of_blocks),
                                                 _ptr(self.d_sequences), _ptr(self.d_targets),
                                                 _ptr(self.d_global_maxima), _ptr(self.d_global_direction))
        else:
            self.lib.emu_calculateScore(u(gx), u(gy), _ptr(self.d_matrix), u(idx), u(idy), u(number_of_blocks),
                                        _ptr(self.d_sequences), _ptr(self.d_targets),
                                        _ptr(self.d_global_maxima), _ptr(self.d_global_direction))

    def _execute_traceback_kernel(self, number_of_blocks, idx, idy):
        gx, gy = self.number_of_sequences, self.number_targets * number_of_blocks
        u = ctypes.c_uint
        if self.gap_extension:
            self.lib.emu_tracebackAffineGap(u(gx), u(gy), _ptr(self.d_matrix), _ptr(self.d_matrix_i),
                                            _ptr(self.d_matrix_j), u(idx), u(idy), u(number_of_blocks),
                                            _ptr(self.d_global_maxima), _ptr(self.d_global_direction),
                                            _ptr(self.h_global_direction_zero_copy), _ptr(self.d_index_increment),
                                            _ptr(self.h_starting_points_zero_copy),
                                            _ptr(self.d_max_possible_score_zero_copy))
        else:
            self.lib.emu_traceback(u(gx), u(gy), _ptr(self.d_matrix), u(idx), u(idy), u(number_of_blocks),
                                   _ptr(self.d_global_maxima), _ptr(self.d_global_direction),
                                   _ptr(self.h_global_direction_zero_copy), _ptr(self.d_index_increment),
                                   _ptr(self.h_starting_points_zero_copy), _ptr(self.d_max_possible_score_zero_copy))

    def _print_alignments(self, sequences, targets, start_seq, start_target, hit_list=None):
        self.batch_offsets.append([int(start_seq), int(start_target)])
        return SmithWatermanCuda._print_alignments(self, sequences, targets, start_seq, start_target, hit_list)

    def _get_number_of_starting_points(self):
        n = int(self.d_index_increment[0])
        # record the raw device results of this batch for lower-level checks
        sp = numpy.frombuffer(self.h_starting_points_zero_copy[: n * 36].tobytes(), dtype=numpy.uint8)
        recs = sp.reshape(n, 36) if n else sp.reshape(0, 36)
        u32 = recs[:, :24].copy().view(numpy.uint32).reshape(n, 6) if n else numpy.zeros((0, 6), numpy.uint32)
        f32 = recs[:, 24:].copy().view(numpy.float32).reshape(n, 3) if n else numpy.zeros((0, 3), numpy.float32)
        xb, yb = self.x_div_shared_x, self.y_div_shared_y
        maxima = self.d_global_maxima.reshape(self.number_of_sequences, self.number_targets, xb, yb)[:, :, -1, -1]
        self.raw_batches.append({
            "X": self.length_of_x_sequences, "Y": self.length_of_y_sequences,
            "n_seq": self.number_of_sequences, "n_tgt": self.number_targets,
            "pair_max": maxima.copy(), "starts_u32": u32, "starts_f32": f32,
        })
        return n


class Settings(object):
    """Attribute bag with the option names of pyPaSWAS/__init__.py:71-251, filled
    from the reference's defaults.cfg, values kept as strings like optparse."""

    def __init__(self, **overrides):
        import configparser
        cfg = configparser.ConfigParser()
        cfg.read(os.path.join(REFERENCE_ROOT, "pyPaSWAS", "Core", "cfg", "defaults.cfg"))
        keys = {
            ("General", "out_format"): "out_format", ("General", "program"): "program",
            ("Aligner", "gap_score"): "gap_score", ("Aligner", "gap_extension"): "gap_extension",
            ("Aligner", "match_score"): "match_score", ("Aligner", "mismatch_score"): "mismatch_score",
            ("Aligner", "other_score"): "other_score", ("Aligner", "any_score"): "any_score",
            ("Aligner", "matrix_name"): "matrix_name", ("Aligner", "lower_limit_score"): "lower_limit_score",
            ("Aligner", "minimum_score"): "minimum_score",
            ("Filter", "filter_factor"): "filter_factor", ("Filter", "query_coverage"): "query_coverage",
            ("Filter", "query_identity"): "query_identity", ("Filter", "relative_score"): "relative_score",
            ("Filter", "base_score"): "base_score",
            ("Device", "device_number"): "device_number", ("Device", "maximum_memory_usage"): "maximum_memory_usage",
            ("Device", "limit_length"): "limit_length", ("Device", "max_genome_length"): "max_genome_length",
            ("Device", "recompile"): "recompile", ("Device", "short_sequences"): "short_sequences",
        }
        for (sec, key), attr in keys.items():
            setattr(self, attr, cfg.get(sec, key))
        self.framework = "CUDA"
        self.device_type = "GPU"
        self.custom_matrix = None
        for k, v in overrides.items():
            setattr(self, k, v)


def make_score(settings, logger):
    name = settings.matrix_name.upper()
    cls = {"DNA-RNA": ref_scores.DnaRnaScore, "BASIC": ref_scores.BasicScore,
           "BLOSUM62": ref_scores.Blosum62Score, "BLOSUM80": ref_scores.Blosum80Score,
           "IRYS": ref_scores.IrysScore}[name]
    return cls(logger, settings)


def make_records(pairs):
    """pairs: list of (id, sequence string) -> reference SWSeqRecord list."""
    return [SWSeqRecord(_Seq(s), identifier=i) for i, s in pairs]


def run_reference(queries, targets, settings, program="aligner", device_memory=8 << 30, logger=None):
    """Runs the reference Aligner/Trimmer ``process`` over already prepared
    (sorted / complemented) record lists.  Returns (hitlist, backend)."""
    logger = logger or logging.getLogger("paswas_ref")
    score = make_score(settings, logger)
    cls = Programs.Trimmer if program == "trimmer" else Programs.Aligner
    prog = cls.__new__(cls)
    prog.logger, prog.score, prog.settings = logger, score, settings
    prog.hitlist = HitList(logger)
    prog.smith_waterman = SmithWatermanEmu(logger, score, settings, device_memory)
    prog.process(queries, targets, None)
    return prog.hitlist, prog.smith_waterman
