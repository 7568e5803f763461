"""Scoring models of the pyPaSWAS path (pyPaSWAS/Core/Scores.py), as data the
engine consumes: a substitution matrix indexed ``residue - char_offset``, gap
penalties, the kernel thresholds and ``highest_score``.

Values keep the reference's conventions so that results are identical:
  * ``gap_extension`` of 0 (or unset) selects the linear-gap kernel
    (Scores.py:54-58, SmithWaterman.py:149);
  * ``highest_score`` is the match score for DNA-RNA / BASIC / IRYS and
    ``max(max(matrix))`` with Python's list ordering for BLOSUM and CUSTOM
    matrices (Scores.py:133,191,243,285), i.e. the maximum of the
    lexicographically largest row;
  * the 26x26 BLOSUM tables are the reference's tables (rows and columns A..Z),
    which extend the 24-symbol NCBI tables with J, O and U rows.
"""
import numpy as np

from .exceptions import InvalidOptionException

_BLOSUM62 = """
A   4  -2   0  -2  -1  -2   0  -2  -1  -1  -1  -1  -1  -2  -4  -1  -1  -1   1   0  -4   0  -3  -1  -2  -1
B  -2   4  -3   4   1  -3  -1   0  -3  -3   0  -4  -3   4  -4  -2   0  -1   0  -1  -4  -3  -4  -1  -3   0
C   0  -3   9  -3  -4  -2  -3  -3  -1  -1  -3  -1  -1  -3  -4  -3  -3  -3  -1  -1  -4  -1  -2  -1  -2  -3
D  -2   4  -3   6   2  -3  -1  -1  -3  -3  -1  -4  -3   1  -4  -1   0  -2   0  -1  -4  -3  -4  -1  -3   1
E  -1   1  -4   2   5  -3  -2   0  -3  -3   1  -3  -2   0  -4  -1   2   0   0  -1  -4  -2  -3  -1  -2   4
F  -2  -3  -2  -3  -3   6  -3  -1   0   0  -3   0   0  -3  -4  -4  -3  -3  -2  -2  -4  -1   1  -1   3  -3
G   0  -1  -3  -1  -2  -3   6  -2  -4  -4  -2  -4  -3   0  -4  -2  -2  -2   0  -2  -4  -3  -2  -1  -3  -2
H  -2   0  -3  -1   0  -1  -2   8  -3  -3  -1  -3  -2   1  -4  -2   0   0  -1  -2  -4  -3  -2  -1   2   0
I  -1  -3  -1  -3  -3   0  -4  -3   4   3  -3   2   1  -3  -4  -3  -3  -3  -2  -1  -4   3  -3  -1  -1  -3
J  -1  -3  -1  -3  -3   0  -4  -3   3   3  -3   3   2  -3  -4  -3  -2  -2  -2  -1  -4   2  -2  -1  -1  -3
K  -1   0  -3  -1   1  -3  -2  -1  -3  -3   5  -2  -1   0  -4  -1   1   2   0  -1  -4  -2  -3  -1  -2   1
L  -1  -4  -1  -4  -3   0  -4  -3   2   3  -2   4   2  -3  -4  -3  -2  -2  -2  -1  -4   1  -2  -1  -1  -3
M  -1  -3  -1  -3  -2   0  -3  -2   1   2  -1   2   5  -2  -4  -2   0  -1  -1  -1  -4   1  -1  -1  -1  -1
N  -2   4  -3   1   0  -3   0   1  -3  -3   0  -3  -2   6  -4  -2   0   0   1   0  -4  -3  -4  -1  -2   0
O  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4
P  -1  -2  -3  -1  -1  -4  -2  -2  -3  -3  -1  -3  -2  -2  -4   7  -1  -2  -1  -1  -4  -2  -4  -1  -3  -1
Q  -1   0  -3   0   2  -3  -2   0  -3  -2   1  -2   0   0  -4  -1   5   1   0  -1  -4  -2  -2  -1  -1   4
R  -1  -1  -3  -2   0  -3  -2   0  -3  -2   2  -2  -1   0  -4  -2   1   5  -1  -1  -4  -3  -3  -1  -2   0
S   1   0  -1   0   0  -2   0  -1  -2  -2   0  -2  -1   1  -4  -1   0  -1   4   1  -4  -2  -3  -1  -2   0
T   0  -1  -1  -1  -1  -2  -2  -2  -1  -1  -1  -1  -1   0  -4  -1  -1  -1   1   5  -4   0  -2  -1  -2  -1
U  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4  -4
V   0  -3  -1  -3  -2  -1  -3  -3   3   2  -2   1   1  -3  -4  -2  -2  -3  -2   0  -4   4  -3  -1  -1  -2
W  -3  -4  -2  -4  -3   1  -2  -2  -3  -2  -3  -2  -1  -4  -4  -4  -2  -3  -3  -2  -4  -3  11  -1   2  -2
X  -1  -1  -1  -1  -1  -1  -1  -1  -1  -1  -1  -1  -1  -1  -4  -1  -1  -1  -1  -1  -4  -1  -1  -1  -1  -1
Y  -2  -3  -2  -3  -2   3  -3   2  -1  -1  -2  -1  -1  -2  -4  -3  -1  -2  -2  -2  -4  -1   2  -1   7  -2
Z  -1   0  -3   1   4  -3  -2   0  -3  -3   1  -3  -1   0  -4  -1   4   0   0  -1  -4  -2  -2  -1  -2   4
"""
_BLOSUM80 = """
A   7  -3  -1  -3  -2  -4   0  -3  -3  -8  -1  -3  -2  -3  -8  -1  -2  -3   2   0  -8  -1  -5  -1  -4  -2
B  -3   6  -6   6   1  -6  -2  -1  -6  -8  -1  -7  -5   5  -8  -4  -1  -2   0  -1  -8  -6  -8  -3  -5   0
C  -1  -6  13  -7  -7  -4  -6  -7  -2  -8  -6  -3  -3  -5  -8  -6  -5  -6  -2  -2  -8  -2  -5  -4  -5  -7
D  -3   6  -7  10   2  -6  -3  -2  -7  -8  -2  -7  -6   2  -8  -3  -1  -3  -1  -2  -8  -6  -8  -3  -6   1
E  -2   1  -7   2   8  -6  -4   0  -6  -8   1  -6  -4  -1  -8  -2   3  -1  -1  -2  -8  -4  -6  -2  -5   6
F  -4  -6  -4  -6  -6  10  -6  -2  -1  -8  -5   0   0  -6  -8  -6  -5  -5  -4  -4  -8  -2   0  -3   4  -6
G   0  -2  -6  -3  -4  -6   9  -4  -7  -8  -3  -7  -5  -1  -8  -5  -4  -4  -1  -3  -8  -6  -6  -3  -6  -4
H  -3  -1  -7  -2   0  -2  -4  12  -6  -8  -1  -5  -4   1  -8  -4   1   0  -2  -3  -8  -5  -4  -2   3   0
I  -3  -6  -2  -7  -6  -1  -7  -6   7  -8  -5   2   2  -6  -8  -5  -5  -5  -4  -2  -8   4  -5  -2  -3  -6
J  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8
K  -1  -1  -6  -2   1  -5  -3  -1  -5  -8   8  -4  -3   0  -8  -2   2   3  -1  -1  -8  -4  -6  -2  -4   1
L  -3  -7  -3  -7  -6   0  -7  -5   2  -8  -4   6   3  -6  -8  -5  -4  -4  -4  -3  -8   1  -4  -2  -2  -5
M  -2  -5  -3  -6  -4   0  -5  -4   2  -8  -3   3   9  -4  -8  -4  -1  -3  -3  -1  -8   1  -3  -2  -3  -3
N  -3   5  -5   2  -1  -6  -1   1  -6  -8   0  -6  -4   9  -8  -4   0  -1   1   0  -8  -5  -7  -2  -4  -1
O  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8
P  -1  -4  -6  -3  -2  -6  -5  -4  -5  -8  -2  -5  -4  -4  -8  12  -3  -3  -2  -3  -8  -4  -7  -3  -6  -2
Q  -2  -1  -5  -1   3  -5  -4   1  -5  -8   2  -4  -1   0  -8  -3   9   1  -1  -1  -8  -4  -4  -2  -3   5
R  -3  -2  -6  -3  -1  -5  -4   0  -5  -8   3  -4  -3  -1  -8  -3   1   9  -2  -2  -8  -4  -5  -2  -4   0
S   2   0  -2  -1  -1  -4  -1  -2  -4  -8  -1  -4  -3   1  -8  -2  -1  -2   7   2  -8  -3  -6  -1  -3  -1
T   0  -1  -2  -2  -2  -4  -3  -3  -2  -8  -1  -3  -1   0  -8  -3  -1  -2   2   8  -8   0  -5  -1  -3  -2
U  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8  -8
V  -1  -6  -2  -6  -4  -2  -6  -5   4  -8  -4   1   1  -5  -8  -4  -4  -4  -3   0  -8   7  -5  -2  -3  -4
W  -5  -8  -5  -8  -6   0  -6  -4  -5  -8  -6  -4  -3  -7  -8  -7  -4  -5  -6  -5  -8  -5  16  -5   3  -5
X  -1  -3  -4  -3  -2  -3  -3  -2  -2  -8  -2  -2  -2  -2  -8  -3  -2  -2  -1  -1  -8  -2  -5  -2  -3  -1
Y  -4  -5  -5  -6  -5   4  -6   3  -3  -8  -4  -2  -3  -4  -8  -6  -3  -4  -3  -3  -8  -3   3  -3  11  -4
Z  -2   0  -7   1   6  -6  -4   0  -6  -8   1  -5  -3  -1  -8  -2   5   0  -1  -2  -8  -4  -5  -1  -4   6
"""


def _table(text):
    m = []
    for line in text.strip().splitlines():
        parts = line.split()
        m.append([int(v) for v in parts[1:]])
    return m


def _max_of_max(matrix):
    # max(max(matrix)) on lists of lists: the largest row compares first
    return max(max(matrix))


class Score(object):
    """Common part of every scoring model (Scores.py:5-98)."""

    score_type = "Unknown"

    def __init__(self, settings, logger=None):
        self.logger = logger
        self.matrix = None
        self.dimensions = 255
        self.char_offset = "\1"
        self.highest_score = 0
        self.set_gap_score(settings.gap_score)
        self.set_gap_extension(settings.gap_extension)
        self.set_lower_limit_score(settings.lower_limit_score)
        self.lower_limit_max_score = float(settings.lower_limit_score)
        self.minimum_score = float(settings.minimum_score)

    def set_gap_score(self, gap_score):
        self.gap_score = float(gap_score) if gap_score else None

    def set_gap_extension(self, gap_extension):
        self.gap_extension = float(gap_extension) if gap_extension and float(gap_extension) != 0 else None

    def set_lower_limit_score(self, lower_limit_score):
        llscore = float(lower_limit_score)
        if llscore < 1.0 and self.logger is not None:
            self.logger.warning("Lower limit score is set < 1.0 ({}), this can result in too many hits to "
                                "properly handle.".format(llscore))
        self.lower_limit_score = llscore

    # ------------------------------------------------------------ engine view
    def matrix_array(self):
        return matrix_array(self)

    def char_offset_code(self):
        return char_offset_code(self)

    def kernel_constants(self):
        return kernel_constants(self)


# ---------------------------------------------------------------------------
# The engine's view of a scoring model, read from the public attributes that
# every Score of the reference has (Scores.py:9-98): matrix, dimensions,
# char_offset, gap_score, gap_extension, lower_limit_score, minimum_score and
# highest_score.  They accept this module's Score classes and the reference's
# own pyPaSWAS.Core.Scores objects alike, so the driver can be handed either.

def _compiled_float(value):
    """A Python value formatted with str() and read back as a C float literal,
    which is how the reference bakes constants into its kernels
    (PaSWAS.py:64-72 substitutes str(value) into default_score.cu)."""
    return np.float32(float(str(value)))


def matrix_array(score):
    """float32 [dim, dim] substitution matrix, rows and columns 0..dim-1 as
    Score.__str__ emits them (Scores.py:87-98).  The generated source holds
    each entry as a double literal in a float array, so the value is the
    decimal read as a double and rounded to float -- what float() followed by
    the float32 conversion does, for numbers and for the IRYS model's string
    entries alike."""
    dim = int(score.dimensions)
    m = score.matrix
    return np.array([[float(v) for v in row[:dim]] for row in m[:dim]], dtype=np.float32)


def char_offset_code(score):
    """Residue code of matrix row 0 (``CHAR_OFFSET``, default_variable.cu)."""
    return ord(score.char_offset)


def kernel_constants(score):
    """(gap, ext, affine, lower_limit, minimum_score) as the kernel sees them:
    an unset gap extension selects the linear kernel and compiles as 0.0
    (PaSWAS.py:58-61, SmithWaterman.py:149)."""
    gap = _compiled_float(score.gap_score if score.gap_score is not None else 0.0)
    ext = _compiled_float(score.gap_extension if score.gap_extension is not None else 0.0)
    return (gap, ext, score.gap_extension is not None, _compiled_float(score.lower_limit_score),
            _compiled_float(score.minimum_score))


def highest_score(score):
    """``highest_score`` as a float (the per-pair bound of
    SmithWatermanCuda._set_max_possible_score multiplies it as a float)."""
    return float(score.highest_score)


class BasicScore(Score):
    """Match / mismatch over all 255 byte values (Scores.py:101-138)."""

    score_type = "BASIC"

    def __init__(self, settings, logger=None):
        Score.__init__(self, settings, logger)
        self.match_score = settings.match_score
        self.mismatch_score = settings.mismatch_score
        self.matrix = [[self.mismatch_score] * self.dimensions for _ in range(self.dimensions)]
        for i in range(self.dimensions):
            self.matrix[i][i] = self.match_score
        self.highest_score = self.match_score


class Blosum62Score(Score):
    """BLOSUM62 over A..Z (Scores.py:193-243)."""

    score_type = "BLOSUM62"

    def __init__(self, settings, logger=None):
        Score.__init__(self, settings, logger)
        self.dimensions = 26
        self.char_offset = "A"
        self.matrix = _table(_BLOSUM62)
        self.highest_score = _max_of_max(self.matrix)


class Blosum80Score(Score):
    """BLOSUM80 over A..Z (Scores.py:141-191)."""

    score_type = "BLOSUM80"

    def __init__(self, settings, logger=None):
        Score.__init__(self, settings, logger)
        self.dimensions = 26
        self.char_offset = "A"
        self.matrix = _table(_BLOSUM80)
        self.highest_score = _max_of_max(self.matrix)


class CustomScore(Score):
    """User matrix: 26 lists of 26 numbers (Scores.py:247-285)."""

    score_type = "CUSTOM"

    def __init__(self, settings, logger=None):
        Score.__init__(self, settings, logger)
        matrix = getattr(settings, "custom_matrix", None)
        if matrix is None:
            raise InvalidOptionException("Required argument {0} is missing".format("matrix"))
        self.char_offset = "A"
        self.dimensions = 26
        if len(matrix) != self.dimensions or (len(matrix) > 0 and len(matrix[0]) != self.dimensions):
            raise InvalidOptionException("A matrix should consist of a list containing 26 lists of "
                                         "26 integers each.")
        self.matrix = matrix
        self.highest_score = _max_of_max(self.matrix)


class DnaRnaScore(Score):
    """Nucleotides with IUPAC two-base ambiguity codes (Scores.py:288-360):
    identical letters and ambiguity codes covering the other letter score as a
    match; N against anything scores ``any_score``; other pairs involving a
    nucleotide score ``mismatch_score``; everything else ``other_score``."""

    score_type = "DNA_RNA"

    def __init__(self, settings, logger=None):
        Score.__init__(self, settings, logger)
        self.match_score = settings.match_score
        self.mismatch_score = settings.mismatch_score
        self.other_score = settings.other_score
        self.any_score = settings.any_score
        self.char_offset = "A"
        self.dimensions = 26
        idx = lambda c: ord(c) - ord("A")
        nucleotides = [idx(c) for c in "ATCGU"]
        ambiguity = {idx("K"): "GT", idx("M"): "AC", idx("R"): "AG", idx("Y"): "CT", idx("S"): "CG", idx("W"): "AT"}
        ambiguity = {k: [idx(c) for c in v] for k, v in ambiguity.items()}
        any_code = idx("N")
        m = [[self.other_score] * 26 for _ in range(26)]
        for r in range(26):
            for c in range(26):
                covers = r == c or (r in ambiguity and c in ambiguity[r]) or (c in ambiguity and r in ambiguity[c])
                if covers:
                    m[r][c] = self.match_score
                elif r == any_code or c == any_code:
                    m[r][c] = self.any_score
                elif r in nucleotides or c in nucleotides:
                    m[r][c] = self.mismatch_score
        self.matrix = m
        self.highest_score = self.match_score


class IrysScore(Score):
    """Optical-map style distance scoring over 'A'..'~' (Scores.py:363-402)."""

    score_type = "IRYS"

    def __init__(self, settings, logger=None):
        Score.__init__(self, settings, logger)
        self.match_score = settings.match_score
        self.mismatch_score = settings.mismatch_score
        self.other_score = settings.other_score
        self.any_score = settings.any_score
        self.char_offset = "A"
        self.dimensions = ord("~") - ord(self.char_offset) + 1
        m = [[self.other_score] * self.dimensions for _ in range(self.dimensions)]
        for r in range(self.dimensions):
            for c in range(self.dimensions):
                m[r][c] = self.match_score if r == c else str(float(self.mismatch_score) * abs(r - c))
        self.matrix = m
        self.highest_score = self.match_score


SCORES = {"DNA-RNA": DnaRnaScore, "BASIC": BasicScore, "BLOSUM62": Blosum62Score, "BLOSUM80": Blosum80Score,
          "CUSTOM": CustomScore, "IRYS": IrysScore}


def make_score(settings, logger=None):
    """Scoring model named by ``settings.matrix_name`` (pypaswasall.py:126-147)."""
    name = settings.matrix_name.upper()
    if name not in SCORES:
        raise InvalidOptionException(name + " is not a valid substitution matrix")
    return SCORES[name](settings, logger)
