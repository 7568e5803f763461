"""The pyPaSWAS command line on the B200 engine.

    python -m pypaswas_b200 [options] FILE_1 FILE_2

Restates pyPaSWAS's driver (pyPaSWAS/pypaswasall.py:20-266, options of
pyPaSWAS/__init__.py:71-251, defaults of Core/cfg/defaults.cfg): the same option
names, defaults and meaning, the same chunked loop over the query file
(--start_query / --end_query / --query_step) and the target file
(--start_target / --end_target / --sequence_step), the same scoring models,
programs (aligner, trimmer), output formats (TXT, SAM, FASTA, trimmedFasta) and
output-file rules.  The records are read by the native reader
(pypaswas_b200.readers) and aligned by one engine that stays alive across all
chunks (the reference re-initialises its device state per chunk).

Two output paths give the same file:
  * objects: every chunk goes through Aligner/Trimmer.process into one HitList
    of Hit objects, which the formatter prints (the reference's path);
  * native: when the output is TXT, SAM or trimmedFasta, ids are unique within each
    file and per-hit log records are off (level above INFO), the engine's hit
    records of all chunks go straight to the native formatter
    (pw_txt_records / pw_sam_records / pw_trimmed_fasta) -- no Hit objects.
"""
import configparser
import logging
import optparse
import os

import numpy as np

from . import _native, formatters, readers
from .exceptions import InvalidOptionException, ReaderException
from .hits import HitList
from .programs import Aligner, Trimmer
from .scores import make_score

# defaults.cfg (pyPaSWAS/Core/cfg/defaults.cfg), section by section
DEFAULTS = {
    "General": dict(out_file="output", out_format="TXT", loglevel="DEBUG", program="aligner", filetype1="fasta",
                    filetype2="fasta", override_output="T"),
    "Input": dict(start_query="0", end_query="0", start_target="0", end_target="0", sequence_step="100000000",
                  query_step="1000000"),
    "Aligner": dict(gap_score="-5", gap_extension="0", match_score="5", mismatch_score="-3", other_score="-1",
                    any_score="0", matrix_name="DNA-RNA", highest_score="5", lower_limit_score="1.0",
                    minimum_score="30"),
    "Filter": dict(filter_factor="0.2", query_coverage="0.2", query_identity="0.2", relative_score="2.0",
                   base_score="2.0"),
    "Device": dict(device_number="0", maximum_memory_usage="0.8", number_of_compute_units="0", sub_device="0",
                   limit_length="100000", max_genome_length="100000", recompile="T", short_sequences="F"),
    "Framework": dict(language="B200"),
}

# option: (short, long, dest, section, key) -- pyPaSWAS/__init__.py:93-242
_OPTIONS = [
    ("-L", "--logfile", "logfile", None, None), ("", "--loglevel", "loglevel", "General", "loglevel"),
    ("-o", "--out", "out_file", "General", "out_file"), ("", "--outputformat", "out_format", "General", "out_format"),
    ("-p", "--program", "program", "General", "program"), ("-1", "--filetype1", "filetype1", "General", "filetype1"),
    ("-2", "--filetype2", "filetype2", "General", "filetype2"),
    ("-O", "--override_output", "override_output", "General", "override_output"),
    ("-c", "--configfile", "config_file", None, None),
    ("", "--start_query", "start_query", "Input", "start_query"), ("", "--end_query", "end_query", "Input", "end_query"),
    ("", "--start_target", "start_target", "Input", "start_target"),
    ("", "--end_target", "end_target", "Input", "end_target"),
    ("", "--sequence_step", "sequence_step", "Input", "sequence_step"),
    ("", "--query_step", "query_step", "Input", "query_step"),
    ("", "--customMatrix", "custom_matrix", None, None),
    ("-G", "--gap_score", "gap_score", "Aligner", "gap_score"),
    ("-g", "--gap_extension", "gap_extension", "Aligner", "gap_extension"),
    ("-M", "--matrixname", "matrix_name", "Aligner", "matrix_name"),
    ("-q", "--mismatch_score", "mismatch_score", "Aligner", "mismatch_score"),
    ("-r", "--match_score", "match_score", "Aligner", "match_score"),
    ("", "--any", "any_score", "Aligner", "any_score"), ("", "--other", "other_score", "Aligner", "other_score"),
    ("", "--minimum", "minimum_score", "Aligner", "minimum_score"),
    ("", "--llimit", "lower_limit_score", "Aligner", "lower_limit_score"),
    ("", "--filter_factor", "filter_factor", "Filter", "filter_factor"),
    ("", "--query_coverage", "query_coverage", "Filter", "query_coverage"),
    ("", "--query_identity", "query_identity", "Filter", "query_identity"),
    ("", "--relative_score", "relative_score", "Filter", "relative_score"),
    ("", "--base_score", "base_score", "Filter", "base_score"),
    ("", "--device", "device_number", "Device", "device_number"),
    ("", "--limit_length", "limit_length", "Device", "limit_length"),
    ("", "--maximum_memory_usage", "maximum_memory_usage", "Device", "maximum_memory_usage"),
    ("", "--recompile", "recompile", "Device", "recompile"),
    ("", "--short_sequences", "short_sequences", "Device", "short_sequences"),
    ("", "--framework", "framework", "Framework", "language"),
]


def _config(path):
    cfg = configparser.ConfigParser()
    cfg.read_dict(DEFAULTS)
    if path:
        try:
            cfg.read(path)
        except configparser.ParsingError:
            raise configparser.ParsingError("Unable to parse the defaults file ({})".format(path))
    return cfg


def parse_cli(argv=None, config_file=None):
    """(settings, arguments) like parse_cli (pyPaSWAS/__init__.py:71-251):
    defaults (optionally from another defaults file), then the command line,
    then a --configfile."""
    cfg = _config(config_file)
    parser = optparse.OptionParser(usage="%prog [options] FILE_1 FILE_2")
    for short, long_, dest, sec, key in _OPTIONS:
        names = [n for n in (short, long_) if n]
        default = cfg.get(sec, key) if sec else (False if dest == "config_file" else None)
        parser.add_option(*names, dest=dest, default=default)
    settings, arguments = parser.parse_args(argv)
    if settings.config_file:
        # _override_settings (pyPaSWAS/__init__.py:254-276): every non-empty
        # key of the file whose name is a setting replaces that setting, the
        # command line's values included
        override = configparser.ConfigParser()
        try:
            override.read(settings.config_file)
        except configparser.ParsingError:
            raise configparser.ParsingError("Unable to parse the given configuration file ({})".format(
                settings.config_file))
        for section in override.sections():
            for key, value in override.items(section):
                if value and hasattr(settings, key):
                    setattr(settings, key, value)
    if len(arguments) < 2:
        raise InvalidOptionException("Missing input files")
    return settings, arguments


def set_logger(settings):
    """Log level and destination (pyPaSWAS/__init__.py:17-68): the console, or
    the file given with --logfile."""
    level = getattr(logging, str(settings.loglevel).upper(), None)
    if not isinstance(level, int):
        raise InvalidOptionException("Invalid log level: %s" % settings.loglevel)
    logger = logging.getLogger("pypaswas_b200.cli")
    logger.handlers = []
    logger.propagate = False
    logger.setLevel(level)
    if settings.logfile:
        try:
            handler = logging.FileHandler(settings.logfile)
        except IOError:
            raise InvalidOptionException("Invalid log file or writing forbidden: %s" % settings.logfile)
        handler.setFormatter(logging.Formatter("%(asctime)s - %(levelname)s - %(message)s"))
    else:
        handler = logging.StreamHandler()
        handler.setFormatter(logging.Formatter("%(levelname)s - %(message)s"))
    handler.setLevel(level)
    logger.addHandler(handler)
    return logger


class Pypaswas(object):
    """pyPaSWAS's main program (pypaswasall.py:20-266) on the B200 engine."""

    def __init__(self, config=None):
        self.config_file = config
        self.settings = None
        self.arguments = None
        self.logger = logging.getLogger("pypaswas_b200.cli")
        self.outputfile = None
        self.score = None
        self.program = None
        self.output_format = None
        self.native_output = None  # whether the last run wrote through the native formatter

    def _set_outfile(self):
        """pypaswasall.py:74-96."""
        path = self.settings.out_file
        if path in (None, "", "."):
            path = "output"
        path = os.path.abspath(os.path.expanduser(path))
        if self.settings.override_output != "T" and os.path.exists(path):
            raise IOError("File {0} already exists.".format(path))
        d = os.path.split(path)[0]
        if os.path.isdir(d):
            if not os.access(d, os.W_OK):
                raise IOError("Cannot write to {0}.".format(d))
        else:
            try:
                os.makedirs(d)
            except OSError:
                raise IOError("Cannot create direcory {0}.".format(d))
        self.outputfile = path

    def _set_output_format(self):
        """pypaswasall.py:150-164."""
        fmt = str(self.settings.out_format).upper()
        names = {"SAM": "SAM", "TXT": "TXT", "TRIMMEDFASTA": "trimmedFasta", "FASTA": "FASTA"}
        if fmt not in names:
            raise InvalidOptionException("Invalid output format {0}.".format(self.settings.out_format))
        self.output_format = names[fmt]

    def _set_program(self):
        """pypaswasall.py:166-173."""
        if self.settings.program == "aligner":
            self.program = Aligner(self.logger, self.score, self.settings)
        elif self.settings.program == "trimmer":
            self.program = Trimmer(self.logger, self.score, self.settings)
        else:
            raise InvalidOptionException("Invalid program selected {0}".format(self.settings.program))

    def _native_ok(self, query_path, target_path):
        if self.output_format not in ("TXT", "SAM", "trimmedFasta"):
            return False
        if self.logger.isEnabledFor(logging.INFO):
            return False  # the object path logs every HitList append
        return all(_ids_unique(p, ft) for p, ft in ((query_path, self.settings.filetype1),
                                                    (target_path, self.settings.filetype2)))

    def run(self, argv=None):
        """Reads, aligns chunk by chunk and writes the output file
        (pypaswasall.py:175-251)."""
        self.settings, self.arguments = parse_cli(argv, self.config_file)
        self.logger = set_logger(self.settings)
        self.logger.info("Initializing application...")
        self._set_outfile()
        self.score = make_score(self.settings, self.logger)
        self._set_output_format()
        self._set_program()
        try:
            native = self._native_ok(self.arguments[0], self.arguments[1])
            self.native_output = native
            chunks = self._chunks()
            return self._run_native(chunks) if native else self._run_objects(chunks)
        finally:
            self.program.smith_waterman.close()

    def _chunks(self):
        """The chunk loop of pypaswasall.py:190-244: yields (query records,
        target records) per processed chunk, in the reference's order.  Like
        the reference, the target loop also ends after a chunk holding no more
        records than its end index (pypaswasall.py:234-237)."""
        st = self.settings
        q_step, s_step = int(st.query_step), int(st.sequence_step)
        q_start = int(st.start_query)
        q_end = q_start + q_step
        if q_end > int(st.end_query) and int(st.start_query) != int(st.end_query):
            q_end = int(st.end_query)
        queries_left = True
        while queries_left:
            try:
                queries = readers.read_query_records(st, self.arguments[0], q_start, q_end, self.logger)
            except ReaderException:
                queries_left = False
                queries = None
            targets_left = True
            s_start = int(st.start_target)
            s_end = s_start + s_step
            if s_end > int(st.end_target) and int(st.start_target) != int(st.end_target):
                s_end = int(st.end_target)
            while queries_left and targets_left:
                try:
                    targets = readers.read_target_records(st, self.score, self.arguments[1], s_start, s_end,
                                                          self.logger)
                except ReaderException:
                    targets_left = False
                    targets = None
                if not targets_left or len(queries) == 0 or len(targets) == 0:
                    targets_left = False
                else:
                    self.logger.info("Processing {0}- vs {1}-sequences".format(len(queries), len(targets)))
                    yield queries, targets
                if targets_left and len(targets) <= s_end:
                    targets_left = False
                s_start += s_step
                s_end += s_step
                if 0 < int(st.end_target) < s_end:
                    targets_left = False
            if 0 < int(st.end_query) < q_end:
                queries_left = False
            q_start += q_step
            q_end += q_step

    def _run_objects(self, chunks):
        results = HitList(self.logger)
        for queries, targets in chunks:
            results.extend(self.program.process(queries.records(), targets.records(), self))
        n = len(results.hits)
        self.logger.info("Processing OK ({} hits found).".format(n))
        if n == 0:
            self.logger.warning("No suitable hits produced, exiting...")
            return results
        formatters.formatter_for(self.output_format)(self.logger, results, self.outputfile).print_results()
        self.logger.info("Finished")
        return results

    def _run_native(self, chunks):
        """Hit records of every chunk, indices made global, one native
        formatter call over all of them."""
        sw = self.program.smith_waterman
        parts = []
        q_base = t_base = 0
        for queries, targets in chunks:
            hits, strbuf = sw.align_packed(queries, targets)
            hits = hits.copy()
            hits["query"] += q_base
            hits["target"] += t_base
            parts.append((hits, strbuf, queries, targets))
            q_base += len(queries)
            t_base += len(targets)
        text = _native_text(parts, self.output_format, self.settings)
        if not text:
            self.logger.warning("No suitable hits produced, exiting...")
            return None
        with open(self.outputfile, "w") as f:
            f.write(text)
        self.logger.info("Finished")
        return None


def _ids_unique(path, filetype):
    """Whether the file's record ids are all distinct (then chunks cannot
    share a HitList key, and one native formatter call equals the HitList
    merge of the chunks)."""
    try:
        rs = readers.read_records(path, filetype, 0, None, 0, _native.PW_RECORDS_AS_READ, False)
    except ReaderException:
        return True
    ids = rs.ids
    return len(set(ids)) == len(ids)


def formatters_hitlist():
    from .hits import HitList
    return HitList(None)


def _native_text(parts, output_format, settings):
    """The output file's text from the hit records of every chunk: one native
    formatter call over all of them, with record indices and string offsets
    made global."""
    if not parts:
        return "".join(line + "\n" for line in formatters.SamFormatter(None, formatters_hitlist(), None).lines()) \
            if output_format == "SAM" else ""
    hits = np.concatenate([p[0] for p in parts])
    queries = readers.concat([p[2] for p in parts])
    targets = readers.concat([p[3] for p in parts])
    if output_format in ("TXT", "SAM"):
        k = shift = 0
        for h, sb, _, _ in parts:
            hits["str_offset"][k:k + len(h)] += shift
            k += len(h)
            shift += len(sb)
        fmt = formatters.txt_records if output_format == "TXT" else formatters.sam_records
        return fmt(hits, b"".join(p[1] for p in parts), queries, targets, settings)
    return formatters.trimmed_fasta(hits, queries, targets, settings)


def main(argv=None):
    """pypaswas.py: run, and print the exception's message on failure."""
    ppw = Pypaswas()
    try:
        ppw.run(argv)
    except Exception as exc:  # noqa: BLE001 -- the reference's entry point reports every failure
        if ppw.settings is not None and ppw.logger.getEffectiveLevel() == logging.DEBUG:
            ppw.logger.exception(str(exc))
        else:
            print("Program ended. The message was: ", ",".join(str(a) for a in exc.args))
            print("Please use the option --help for information on command line arguments.")
        return 1
    return 0
