"""Sequence records with the attributes the driver and Hit read.

Mirrors pyPaSWAS/Core/SWSeqRecord.py (a Biopython SeqRecord subclass that
upper-cases its sequence and carries original_length / start_position /
distance) without depending on Biopython.
"""
from .workloads import reverse_complement as _rc_bytes


class Sequence(str):
    """Upper-case residue string with the few Bio.Seq methods the path uses."""

    def upper(self):
        return Sequence(str.upper(self))

    def reverse_complement(self):
        return Sequence(_rc_bytes(self.encode("latin-1")).decode("latin-1"))

    def __getitem__(self, i):
        r = str.__getitem__(self, i)
        return Sequence(r) if isinstance(i, slice) else r


class SeqRecord(object):
    """A query or target record (SWSeqRecord.py:13-34)."""

    start_position = 0
    distance = 0

    def __init__(self, seq, identifier, start_position=0, original_length=None, distance=0, ref_id=None):
        if isinstance(seq, (bytes, bytearray)):
            seq = seq.decode("latin-1")
        self.seq = Sequence(str(seq)).upper()
        self.id = identifier
        self.start_position = start_position
        self.original_length = len(self.seq) if original_length is None else original_length
        self.distance = distance
        self.refID = ref_id

    def __len__(self):
        return len(self.seq)

    def __getitem__(self, i):
        return self.seq[i]

    def __repr__(self):
        return "SeqRecord(id=%r, len=%d)" % (self.id, len(self.seq))


def complement_records(records, rc_string="_RC"):
    """Appends reverse complements with ``_RC`` ids (Readers.py:68-73)."""
    return list(records) + [SeqRecord(r.seq.reverse_complement(), str(r.id) + rc_string) for r in records]


def sort_records(records, reverse=True):
    """Sorts by length, longest first by default (Readers.py:30-34)."""
    return sorted(records, key=lambda r: len(r.seq), reverse=reverse)
