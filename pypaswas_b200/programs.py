"""The aligner and trimmer programs (pyPaSWAS/Core/Programs.py:9-120) on the
B200 backend.  ``process`` keeps the reference's loop over target blocks and
merges the per-block HitLists with HitList.extend."""
import logging

from .hits import HitList
from .scores import make_score
from .smith_waterman import SmithWatermanB200


def _is_packed(records):
    return hasattr(records, "id_blob") and hasattr(records, "residues")


def _one_block(program, records_seqs, targets, max_length=None, strings=True):
    """The driver's single target block (the engine takes every target):
    the engine's hit records, their strings and the block.  Records given as
    packed sets (pypaswas_b200.readers.RecordSet) go to the engine as they are."""
    if _is_packed(records_seqs) and _is_packed(targets):
        hits, strbuf = program.smith_waterman.align_packed(records_seqs, targets, strings)
        return hits, strbuf, targets
    all_targets_length = sum(len(s.seq) for s in targets)
    all_sequences_length = sum(len(s.seq) for s in records_seqs)
    program.smith_waterman.set_total_work_size(all_targets_length * all_sequences_length)
    last = program.smith_waterman.set_targets(targets, 0, max_length, records_seqs)
    if last != len(targets):
        raise AssertionError("the engine takes every target in one block")
    return program.smith_waterman.align_records(records_seqs, targets, 0)


class Aligner(object):
    """Aligns query records against target records (Programs.py:9-86)."""

    def __init__(self, logger, score, settings, device=None):
        self.logger = logger or logging.getLogger("pypaswas_b200")
        self.settings = settings
        self.score = score if score is not None else make_score(settings, self.logger)
        self.hitlist = HitList(self.logger)
        self.smith_waterman = SmithWatermanB200(self.logger, self.score, settings, device=device)

    def process(self, records_seqs, targets, pypaswas=None):
        self.hitlist = HitList(self.logger)
        target_index = 0
        all_targets_length = sum(len(s.seq) for s in targets)
        all_sequences_length = sum(len(s.seq) for s in records_seqs)
        self.smith_waterman.set_total_work_size(all_targets_length * all_sequences_length)
        while target_index < len(targets):
            last = self.smith_waterman.set_targets(targets, target_index, records_seqs=records_seqs,
                                                   use_all_records_seqs=False)
            results = self.smith_waterman.align_sequences(records_seqs, targets, target_index)
            self.hitlist.extend(results)
            target_index = last
        return self.hitlist

    def process_pairs(self, records_seqs, targets, pairs):
        """Explicit (query index, target index) pairs; returns the HitList that
        process() gives for each pair on its own, merged
        (SmithWatermanB200.align_pairs)."""
        self.hitlist = HitList(self.logger)
        self.hitlist.extend(self.smith_waterman.align_pairs(records_seqs, targets, pairs))
        return self.hitlist

    def txt(self, records_seqs, targets):
        """The TXT output of process() + DefaultFormatter, byte for byte, with
        the HitList and the records built in native code
        (formatters.txt_records).  Records: lists of record objects, or packed
        record sets (pypaswas_b200.readers)."""
        from .formatters import txt_records
        if len(targets) == 0:
            return ""
        hits, strbuf, block = _one_block(self, records_seqs, targets)
        return txt_records(hits, strbuf, records_seqs, block, self.settings)

    def sam(self, records_seqs, targets):
        """The SAM output of process() + SamFormatter, byte for byte, with the
        HitList and the records built in native code (formatters.sam_records)."""
        from .formatters import sam_records
        if len(targets) == 0:
            import numpy as np
            from . import _native
            return sam_records(np.zeros(0, dtype=_native.HIT_DTYPE), b"", records_seqs, targets, self.settings)
        hits, strbuf, block = _one_block(self, records_seqs, targets)
        return sam_records(hits, strbuf, records_seqs, block, self.settings)


class Trimmer(Aligner):
    """Same loop; output goes through the trimmedFasta formatter (Programs.py:95-120)."""

    def process(self, records_seqs, targets, pypaswas=None):
        self.hitlist = HitList(self.logger)
        target_index = 0
        max_length = len(targets[0]) if len(targets) > 0 and getattr(self.settings, "recompile", "T") == "F" \
            else None
        all_targets_length = sum(len(s.seq) for s in targets)
        all_sequences_length = sum(len(s.seq) for s in records_seqs)
        self.smith_waterman.set_total_work_size(all_targets_length * all_sequences_length)
        while target_index < len(targets):
            last = self.smith_waterman.set_targets(targets, target_index, max_length, records_seqs)
            results = self.smith_waterman.align_sequences(records_seqs, targets, target_index)
            self.hitlist.extend(results)
            target_index = last
        return self.hitlist

    def trimmed_fasta(self, records_seqs, targets):
        """The trimmedFasta output of process() + TrimmerFormatter, byte for
        byte, with the HitList and the records built in native code
        (formatters.trimmed_fasta).  The engine takes every target in one
        block, so the per-block HitList merge does not arise.  Records: lists
        of record objects, or packed record sets (pypaswas_b200.readers)."""
        from .formatters import trimmed_fasta
        if len(targets) == 0:
            return ""
        max_length = len(targets[0]) if getattr(self.settings, "recompile", "T") == "F" and \
            not _is_packed(targets) else None
        hits, _, block = _one_block(self, records_seqs, targets, max_length, strings=False)
        return trimmed_fasta(hits, records_seqs, block, self.settings)
