"""Output formatters of the aligner and trimmer programs
(pyPaSWAS/Core/Formatters.py:3-150).

Both formatters visit HitList.real_hits sorted by (query id, target id, score)
(Formatters.py:34-37; a stable sort, so equal keys keep HitList order) and
produce the reference's text byte for byte:

* DefaultFormatter ("TXT"): one comma-separated summary line per hit followed by
  the three alignment strings (Formatters.py:19-31).
* TrimmerFormatter ("trimmedFasta"): one FASTA record per hit, the query with
  the span [target_start, target_end] cut out (Hit.get_trimmed_line,
  pyPaSWAS/Core/Hit.py:274-286, which slices the query by the hit's TARGET
  coordinates; that is the reference's behaviour and is kept).
"""
from .exceptions import CudaException


def ordered_hits(hitlist):
    return sorted(hitlist.real_hits.values(), key=lambda h: (h.get_seq_id(), h.get_target_id(), h.score))


def txt_record(hit):
    """The DefaultFormatter record of one hit (Formatters.py:19-31)."""
    n_cols = len(hit.alignment)
    gaps = n_cols - hit.matches - hit.mismatches
    q_len = hit.sequence_info.original_length
    t_len = hit.target_info.original_length
    head = ", ".join(str(v) for v in (
        hit.get_seq_id(), hit.get_target_id(), hit.seq_location[0], hit.seq_location[1], hit.target_location[0],
        hit.target_location[1], hit.score, hit.matches, hit.mismatches, gaps, n_cols, hit.score / n_cols, q_len,
        t_len, hit.score / q_len, hit.score / t_len, hit.distance))
    return "\n".join((head, hit.sequence_match, hit.alignment, hit.target_match))


def _strip_rc(identifier):
    return identifier[:-3] if identifier[-2:] == "RC" else identifier


def trimmed_record(hit):
    """The trimmedFasta record of one hit (Hit.get_trimmed_line, Hit.py:274-286)."""
    if not hit.sequence_match or not hit.target_match or not hit.alignment:
        raise CudaException("sequence_match, target_match and alignment should be set and have lengths > 0.")
    seq = str(hit.sequence_info.seq)
    t0, t1 = hit.target_location
    return "".join((">", _strip_rc(hit.get_target_id()), " ", hit.sequence_info.id, "\n", seq[:t0], seq[t1 + 1:]))


class DefaultFormatter(object):
    """TXT output (Formatters.py:3-47)."""

    record = staticmethod(txt_record)

    def __init__(self, logger, hitlist, outputfile):
        self.logger = logger
        self.hitlist = hitlist
        self.outputfile = outputfile

    def lines(self):
        return [self.record(h) for h in ordered_hits(self.hitlist)]

    def print_results(self):
        with open(self.outputfile, "w") as out:
            for line in self.lines():
                out.write(line + "\n")


class TrimmerFormatter(DefaultFormatter):
    """trimmedFasta output (Formatters.py:110-150)."""

    record = staticmethod(trimmed_record)
