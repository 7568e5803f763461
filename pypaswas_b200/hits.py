"""Alignment results: Hit and HitList with the reference's semantics
(pyPaSWAS/Core/Hit.py, pyPaSWAS/Core/HitList.py).

A Hit validates its locations exactly like the reference (start < end, both
inside the sequence), so a one-column alignment raises CudaException as it does
there.  HitList keeps the reference's de-duplication by start/end keys.
"""
from .exceptions import CudaException


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
