"""The CUDA path against the reference's own outputs (G-PathGen and its
suffix tree, run once on a B200 and packed into tests/golden/ref_goldens.npz).

In the reference division mode the CUDA path evaluates the child cost with
the reference's source expression under the reference's --use_fast_math, so
the costs must match bit for bit.
"""
import os

import numpy as np
import pytest

import cases
import cpg_b200

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "ref_goldens.npz")


def _names(key):
    z = np.load(GOLD)
    return [n for n in cases.CASES if f"{n}/{key}" in z]


@pytest.mark.parametrize("name", _names("sfxt_dist"))
def test_sfxt_matches_reference(name):
    z = np.load(GOLD)
    n, src, dst, w = cases.load_case(name)
    with cpg_b200.CpGen() as g:
        g.load_edges(n, src, dst, w)
        d, s, _ = g.get_sfxt()
    np.testing.assert_array_equal(d, z[f"{name}/sfxt_dist"])
    np.testing.assert_array_equal(s, z[f"{name}/sfxt_succ"])


@pytest.mark.parametrize("name", _names("costs"))
def test_costs_match_reference_bit_exact(name):
    z = np.load(GOLD)
    ref = z[f"{name}/costs"]
    k = int(z[f"{name}/k"])
    n, src, dst, w = cases.load_case(name)
    with cpg_b200.CpGen(division=cpg_b200.DIV_REFERENCE) as g:
        g.load_edges(n, src, dst, w)
        g.report_paths(k)
        got = g.get_slacks(k)
    assert len(got) == len(ref)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), (
        f"first mismatch at {np.flatnonzero(got != ref)[:5]}")
