"""The queue planner of the chained 16-bit score sweep (pypaswas_b200/csrc/
pw_plan.h), compiled on the host and checked for the properties the kernel's
waits rely on: every item is queued exactly once (whole) or as all its strips
in order, and every strip comes after its predecessor."""
import os
import subprocess
import tempfile

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = r"""
#include "pw_plan.h"
#include <cstdio>
int main() {
    int n, warps; long long permille; int lead;
    if (scanf("%d %d %lld %d", &n, &warps, &permille, &lead) != 4) return 2;
    std::vector<int> ns(n); std::vector<int64_t> xm(n);
    for (int k = 0; k < n; ++k) { long long a; if (scanf("%d %lld", &ns[k], &a) != 2) return 2; xm[k] = a; }
    pw::ChainPlan p;
    pw::plan_chain_queue(ns, xm, warps, permille, lead, p);
    for (auto& e : p.queue) printf("%d %d %d %d\n", e.item, e.chain, e.strip, e.pred);
    return 0;
}
"""


def _plan(nstr, xm4, warps, permille=500, lead=64):
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "plan.cpp"), os.path.join(d, "plan")
        with open(src, "w") as f:
            f.write(DRIVER)
        subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(REPO, "pypaswas_b200", "csrc"), "-o", exe,
                        src], check=True)
        inp = "%d %d %d %d\n" % (len(nstr), warps, permille, lead) + "".join(
            "%d %d\n" % (a, b) for a, b in zip(nstr, xm4))
        out = subprocess.run([exe], input=inp, capture_output=True, text=True, check=True).stdout
    return [tuple(map(int, ln.split())) for ln in out.splitlines()]


def _check(nstr, xm4, q):
    seen = {}
    chain_item = {}
    for pos, (item, chain, strip, pred) in enumerate(q):
        if chain < 0:
            assert strip == -1 and pred == -1
            assert item not in seen
            seen[item] = "whole"
            continue
        assert chain_item.setdefault(chain, item) == item
        got = seen.setdefault(item, [])
        assert got != "whole" and strip == len(got)  # strips in order
        if strip == 0:
            assert pred == -1
        else:
            assert 0 <= pred < pos and q[pred][1] == chain and q[pred][2] == strip - 1
        got.append(pos)
    assert set(seen) == set(range(len(nstr)))
    for item, v in seen.items():
        assert v == "whole" or len(v) == nstr[item]


def test_planner_queues_every_strip_after_its_predecessor():
    rng = np.random.default_rng(1)
    for n, warps, permille in ((300, 64, 500), (50, 1776, 500), (200, 32, 1), (10, 8, 100000)):
        ns = rng.integers(2, 40, n)
        xm = rng.integers(1, 500, n) * 4
        order = np.argsort(-(ns * xm), kind="stable")
        ns, xm = ns[order], xm[order]
        q = _plan(ns.tolist(), xm.tolist(), warps, permille)
        _check(ns.tolist(), xm.tolist(), q)
        chained = sum(1 for e in q if e[1] >= 0)
        if permille == 1:
            assert chained == int(ns.sum())      # everything chained
        if permille == 100000:
            assert chained == 0                  # nothing chained
