"""Alignment results: Hit and HitList with the reference's semantics
(pyPaSWAS/Core/Hit.py, pyPaSWAS/Core/HitList.py).

A Hit validates its locations exactly like the reference (start < end, both
inside the sequence), so a one-column alignment raises CudaException as it does
there.  HitList keeps the reference's de-duplication by start/end keys.

The output-side methods (get_sam_line, get_sam_sq, get_trimmed_line,
get_fasta, get_full_fasta, _check_rc) restate Hit.py:159-406 so the
reference's own formatters (Formatters.py) print these hits unchanged.
"""
from .exceptions import CudaException


def _strip_rc(identifier):
    """An id without its reverse-complement suffix: ids ending in "RC" lose
    their last three characters (the "_RC" that Readers.complement_records
    appends), as every output method of Hit.py does."""
    return identifier[:-3] if identifier[-2:] == "RC" else identifier


def _reverse_complement(seq):
    """IUPAC reverse complement of a residue string (case kept), the
    complement the reverse-complement targets are built with."""
    from .workloads import reverse_complement
    return reverse_complement(str(seq).encode("latin-1")).decode("latin-1")


class Hit(object):
    """One alignment between a query (sequence) and a target (Hit.py:11-119)."""

    def __init__(self, logger, sequence_info, target_info, sequence_location, target_location):
        self.logger = logger
        self.sequence_info = sequence_info
        self.target_info = target_info
        self.seq_location = ()
        self.target_location = ()
        self._set_seq_location(sequence_location)
        self._set_target_location(target_location)
        self.sequence_match = ""
        self.alignment = ""
        self.target_match = ""
        self.score = 0
        self.matches = 0
        self.mismatches = 0
        self.query_identity = 0
        self.query_coverage = 0
        self.relative_score = 0
        self.base_score = 0
        self.distance = None
        self.rc = False

    @staticmethod
    def _is_a_valid_location(location, sequence_length):
        return (isinstance(location, tuple) and len(location) == 2 and isinstance(location[0], int)
                and isinstance(location[1], int) and 0 <= location[0] < sequence_length
                and 0 <= location[1] < sequence_length and location[0] < location[1])

    def _set_seq_location(self, location):
        if self._is_a_valid_location(location, self.sequence_info.original_length):
            self.seq_location = location
        else:
            raise CudaException("Invalid sequence location: {0}, length={1}, {2}".format(
                location, len(self.sequence_info.seq), self.sequence_info.original_length))

    def _set_target_location(self, location):
        if self._is_a_valid_location(location, self.target_info.original_length):
            self.target_location = location
        else:
            raise CudaException("Invalid target location: {0}".format(location))

    def set_scores(self, score, matches, mismatches):
        """Score and derived ratios (Hit.py:91-119)."""
        if (isinstance(score, float) or isinstance(score, int)) and score >= 0.0:
            self.score = score
        else:
            raise CudaException("Score should be a float or an integer, not {0}".format(score))
        if isinstance(matches, int) and matches >= 0:
            self.matches = matches
        else:
            raise CudaException("Matches  should be integers. Passed value is {0}".format(matches))
        if isinstance(mismatches, int) and mismatches >= 0:
            self.mismatches = mismatches
        else:
            raise CudaException("Mismatches should be integers. Passed value is {0}.".format(mismatches))
        # relative to the shorter of the two sequences
        if self.sequence_info.original_length > self.target_info.original_length:
            shortest = self.target_info.original_length
        else:
            shortest = self.sequence_info.original_length
        self.relative_score = float(self.score) / float(shortest)
        span = self.seq_location[1] - self.seq_location[0] + 1
        self.query_identity = float(matches) / float(span)
        self.query_coverage = float(span) / float(self.sequence_info.original_length)
        self.base_score = float(self.score) / float(len(self.alignment))

    def set_sequence_match(self, sequence_match):
        self.sequence_match = sequence_match

    def set_target_match(self, target_match):
        self.target_match = target_match

    def set_alignment(self, alignment):
        self.alignment = alignment

    def get_seq_id(self):
        return self.sequence_info.id

    def get_target_id(self):
        return self.target_info.id

    def _check_rc(self):
        """True when both ids carry the reverse-complement suffix (Hit.py:159-164)."""
        return self.get_seq_id()[-2:] == "RC" and self.get_target_id()[-2:] == "RC"

    def get_euclidian_distance(self):
        """The target record's distance, 0.0 when unset (Hit.py:174-179)."""
        d = getattr(self.target_info, "distance", None)
        return 0.0 if d is None else d

    def _require_strings(self):
        if len(self.sequence_match) == 0 or len(self.target_match) == 0 or len(self.alignment) == 0:
            raise CudaException("sequence_match, target_match and alignment should be set and have lengths > 0.")

    # ---------------------------------------------------------------- SAM
    def get_sam_line(self):
        """One SAM alignment line (Hit.py:222-272): QNAME and RNAME without the
        RC suffix, FLAG 16 on an RC id, POS 1-based on the target, MAPQ 255,
        the extended CIGAR, SEQ the query (reverse-complemented on RC), then
        the AS/RS/BS/QC/QI fields.  On an RC hit the alignment and query match
        strings are reversed in place, as the reference does, before the CIGAR
        is read from them."""
        query_id, target_id = self.get_seq_id(), self.get_target_id()
        self.rc = query_id[-2:] == "RC" or target_id[-2:] == "RC"
        pos = self.target_location[0] + 1
        sam_seq = str(self.sequence_info.seq)
        if self.rc:
            self.alignment = self.alignment[::-1]
            self.sequence_match = self.sequence_match[::-1]
            sam_seq = _reverse_complement(sam_seq)
            pos = self.target_info.original_length - self.target_location[1]
        self._require_strings()
        fields = (_strip_rc(query_id), self._get_sam_flag(), _strip_rc(target_id), str(pos), Hit._get_sam_mapq(),
                  self._get_sam_cigar(), "*", "0", "0", sam_seq, "*", self._get_sam_alignment_score(),
                  self._get_sam_relative_score(), self._get_sam_relative_base_score(),
                  self._get_sam_query_coverage(), self._get_sam_query_identity())
        return "\t".join(fields)

    def get_sam_sq(self):
        """The @SQ header line of the hit's target (Hit.py:298-304)."""
        return "\t".join(("@SQ", "SN:{0}".format(_strip_rc(self.get_target_id())),
                          "LN:{0}".format(self.target_info.original_length)))

    def _get_sam_alignment_score(self):
        return "AS:i:" + str(int(self.score))

    def _get_sam_flag(self):
        rc = self.get_seq_id()[-2:] == "RC" or self.get_target_id()[-2:] == "RC"
        return "16" if rc else "0"

    @staticmethod
    def _get_sam_mapq():
        return "255"

    def _get_sam_cigar(self):
        """Extended CIGAR (Hit.py:338-372): soft clips for the query outside
        the alignment (mirrored on RC hits), then one run per maximal stretch
        of equal alignment characters, named by the last column of the run."""
        parts = []
        if self.rc:
            parts.append(str(len(self.sequence_info.seq) - self.seq_location[1] - 1) + "S")
        elif self.seq_location[0] > 0:
            parts.append(str(self.seq_location[0]) + "S")
        aln = self.alignment
        run_start = 0
        for i in range(1, len(aln)):
            if aln[i] != aln[run_start]:
                parts.append(str(i - run_start) + self._get_cigar_char(i - 1))
                run_start = i
        parts.append(str(len(aln) - run_start) + self._get_cigar_char(len(aln) - 1))
        tail = self.seq_location[0] if self.rc else self.sequence_info.original_length - self.seq_location[1] - 1
        if tail > 0:
            parts.append(str(tail) + "S")
        return "".join(parts)

    def _get_sam_relative_score(self):
        return "RS:f:" + str(self.relative_score)

    def _get_sam_query_coverage(self):
        return "QC:f:" + str(self.query_coverage)

    def _get_sam_query_identity(self):
        return "QI:f:" + str(self.query_identity)

    def _get_sam_relative_base_score(self):
        return "BS:f:" + str(self.base_score)

    def _get_cigar_char(self, position):
        """'=' for a match column, 'X' for a mismatch, 'D' for a gap in the
        query, 'I' for a gap in the target (Hit.py:392-406)."""
        c = self.alignment[position]
        if c == "|":
            return "="
        if c == ".":
            return "X"
        return "D" if self.sequence_match[position] == "-" else "I"

    # ------------------------------------------------------------- FASTA
    def get_trimmed_line(self):
        """trimmedFasta record (Hit.py:274-286): the query with the span
        [target_start, target_end] cut out -- the reference slices the QUERY
        by the TARGET coordinates, and that is kept."""
        self._require_strings()
        seq = self.sequence_info.seq
        t0, t1 = self.target_location
        return "".join((">", _strip_rc(self.get_target_id()), " ", self.sequence_info.id, "\n",
                        str(seq[:t0] + seq[t1 + 1:])))

    def get_fasta(self):
        """Same record as get_trimmed_line (Hit.py:289-301)."""
        return self.get_trimmed_line()

    def get_full_fasta(self):
        """The whole query as a FASTA record (Hit.py:303-305)."""
        return ">{}\n{}".format(self.get_seq_id(), str(self.sequence_info.seq))

    def keys(self):
        """De-duplication keys: start and end positions per id pair (Hit.py:151-158)."""
        start = (self.get_seq_id(), self.get_target_id(), self.seq_location[0], self.target_location[0])
        end = (self.get_seq_id(), self.get_target_id(), self.seq_location[1], self.target_location[1])
        return [start, end, start]


class HitList(object):
    """Hits keyed by start and end location; a new hit replaces an older one
    with the same key only if it scores higher (HitList.py:28-52)."""

    def __init__(self, logger=None):
        self.logger = logger
        self.hits = {}
        self.real_hits = {}

    def extend(self, hit_list):
        self.hits.update(hit_list.hits)
        self.real_hits.update(hit_list.real_hits)

    def add(self, hit):
        keys = hit.keys()
        self.hits[keys[0]] = hit
        self.real_hits[keys[0]] = hit

    def append(self, hit):
        keys = hit.keys()
        if keys is None:
            return
        hits = self.hits
        k0, k1 = keys[0], keys[1]
        old0, old1 = hits.get(k0), hits.get(k1)
        better_start = old0 is not None and old0.score < hit.score
        better_end = old1 is not None and old1.score < hit.score
        new = old0 is None and old1 is None
        if better_start or better_end or new:
            if better_end and old1.keys()[2] in self.real_hits:
                # same end location: drop the previous hit's start entry
                del self.real_hits[old1.keys()[2]]
            hits[k0] = hit
            hits[k1] = hit
            self.real_hits[keys[2]] = hit
            if self.logger is not None:
                self.logger.info("Added hit (query ID: %s, target ID: %s) to hitlist", hit.get_seq_id(),
                                 hit.get_target_id())
        elif self.logger is not None:
            self.logger.debug("Rejected hit (query ID: %s, target ID: %s) from addition to hitlist",
                              hit.get_seq_id(), hit.get_target_id())
