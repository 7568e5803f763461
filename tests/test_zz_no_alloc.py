"""pw_score_max_noalloc: pair maxima for callers that cannot allocate device memory.

Some callers cannot let a library call cudaMalloc: code that runs where another
component owns the device memory (a framework's caching allocator, a serving
process with a fixed budget), or a latency-critical path that must not pay for
cudaMalloc's implicit device synchronisation.  For them the library has one
entry point whose device working memory is a fixed array built into the
library.  These tests call it through the C ABI and check it against the
regular entry point (pw_align with PW_FLAG_SCORE_ONLY): the pair maxima must be
bit-identical, on two different calls in a row so that anything the first call
leaves in the shared array cannot leak into the second.

The file is named so that pytest collects it last, and it needs nothing from
the other test files: it passes on its own in a fresh process and after the
rest of the suite.
"""
import numpy as np
import pytest

import cases
from engine_helpers import run_engine
from pypaswas_b200 import _native
from pypaswas_b200.exceptions import CudaException

pytestmark = pytest.mark.gpu


def _no_alloc_pair_max(lib, queries, targets, score):
    gap, ext, affine, _, _ = score.kernel_constants()
    return _native.score_max_noalloc(0, score.matrix_array(), score.char_offset_code(), gap, ext, affine,
                                     [q.encode() for q in queries], [t.encode() for t in targets], lib=lib)


def _workload(seed, kind, n_q, n_t, q_len, t_len):
    """Queries x targets with planted shared segments; lengths chosen so that
    targets fall in every strip class, long ones included."""
    rng = np.random.default_rng(seed)
    alphabet = cases.DNA if kind == "dna" else cases.PROTEIN
    draw = lambda n: "".join(alphabet[i] for i in rng.integers(0, len(alphabet), n))
    targets = [draw(int(rng.integers(*t_len))) for _ in range(n_t)]
    queries = []
    for _ in range(n_q):
        s = draw(int(rng.integers(*q_len)))
        t = targets[int(rng.integers(0, n_t))]
        cut = int(rng.integers(0, max(1, len(t) // 2)))
        p = int(rng.integers(0, len(s) + 1))
        queries.append(s[:p] + cases.mutate(rng, t[cut:], alphabet, 0.1, 2) + s[p:])
    st = cases.Settings(matrix_name="DNA-RNA" if kind == "dna" else "BLOSUM62",
                        gap_score="-5" if kind == "dna" else "-11",
                        gap_extension="0" if kind == "dna" else "-1")
    from pypaswas_b200 import scores
    return queries, targets, scores.make_score(st), st


def test_no_alloc_matches_regular_entry_point_twice(engine_lib):
    # first call: DNA, linear gap, targets up to 300 long (several strips)
    q1, t1, s1, st1 = _workload(101, "dna", 90, 40, (5, 200), (1, 300))
    # second call: protein, affine gap, smaller, so that stale contents of the
    # shared array from the first call would show if they leaked
    q2, t2, s2, st2 = _workload(202, "protein", 37, 23, (3, 120), (1, 90))
    got1 = _no_alloc_pair_max(engine_lib, q1, t1, s1)
    got2 = _no_alloc_pair_max(engine_lib, q2, t2, s2)
    want1 = run_engine(engine_lib, q1, t1, s1, st1, score_only=True)[0]
    want2 = run_engine(engine_lib, q2, t2, s2, st2, score_only=True)[0]
    np.testing.assert_array_equal(got1, want1)
    np.testing.assert_array_equal(got2, want2)
    # and the first input again, after the second left its contents behind
    np.testing.assert_array_equal(_no_alloc_pair_max(engine_lib, q1, t1, s1), want1)


def test_no_alloc_call_takes_no_device_memory(engine_lib):
    # the property the entry point exists for: after a first call (which loads
    # the library's kernels and its fixed array), further calls leave the
    # device's free memory exactly where it was
    import torch
    q, t, s, _ = _workload(303, "dna", 70, 30, (5, 160), (1, 200))
    first = _no_alloc_pair_max(engine_lib, q, t, s)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(0)[0]
    again = [_no_alloc_pair_max(engine_lib, q, t, s) for _ in range(3)]
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free_before
    for a in again:
        np.testing.assert_array_equal(a, first)
    assert torch.cuda.current_device() == 0


def test_no_alloc_rejects_inputs_beyond_its_limit(engine_lib):
    # 4096 x 4096 pair maxima alone need 64 MiB of results: over the limit
    q = ["ACGT"] * 4096
    t = ["ACGTACGT"] * 4096
    from pypaswas_b200 import scores
    score = scores.make_score(cases.Settings())
    with pytest.raises(CudaException, match="no-allocation limit"):
        _no_alloc_pair_max(engine_lib, q, t, score)
