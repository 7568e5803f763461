"""The reference's own OpenCL CPU kernels as bench.py's reference arm
(oracle/ref/ocl_cpu_arm.py): with linear gaps their pair maxima equal the
oracle's (the OpenCL CPU and CUDA kernels agree on real cells), which checks
the launch loops and buffers the arm drives them with.  Needs the reference
tree (template code); skipped elsewhere."""
import os
import sys

import numpy as np
import pytest

import cases

REF = os.environ.get("PASWAS_REFERENCE_ROOT", "/root/reference")
pytestmark = pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "pyPaSWAS")), reason="reference tree absent")


def _arm():
    here = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "ref")
    if here not in sys.path:
        sys.path.insert(0, here)
    import build_ref
    import ocl_cpu_arm
    import ref_driver as R
    return build_ref, ocl_cpu_arm, R


@pytest.mark.parametrize("seed", range(3))
def test_linear_pair_maxima_equal_the_oracle(oracle_mod, seed):
    import ctypes
    import logging
    build_ref, arm, R = _arm()
    queries, targets, score, st = cases.make_case(700 + seed, "dna", max_queries=12, max_qlen=60, max_tlen=70)
    queries = sorted(queries, key=len, reverse=True)
    targets = sorted(targets, key=len, reverse=True)
    settings = dict(gap_score="-5", gap_extension="0", match_score="1", mismatch_score="-3", any_score="1",
                    minimum_score=st.minimum_score, lower_limit_score=st.lower_limit_score,
                    filter_factor=st.filter_factor)
    ref_score = R.make_score(R.Settings(**settings), logging.getLogger("t"))
    X, Y = arm._pad8(max(map(len, queries))), arm._pad8(max(map(len, targets)))
    so = build_ref.build(ref_score, len(queries), len(targets), X, Y, "ocl_cpu")
    lib = ctypes.CDLL(so)
    pm, _ = arm.run_batch(lib, queries, targets, X, Y, False, float(ref_score.highest_score),
                          float(st.filter_factor), 4)
    want = oracle_mod.pair_max(cases.oracle_params(oracle_mod, score), queries, targets)
    np.testing.assert_array_equal(pm, want)
