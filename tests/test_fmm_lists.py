"""FMM interaction lists: the tables libpfblob builds (host-only C ABI call,
no GPU) equal the independent CPU restatement bit for bit, and every (target
leaf, source leaf) pair is covered exactly once."""
import ctypes

import pytest

from oracle import lists


def lib_tables(L, kb, w0, cutoff, theta=0.5):
    import pfblob._lib as lb
    need = ctypes.c_int64(0)
    s = lb.lib.pf_fmm_lists(L, kb, w0, cutoff, theta, None, 0, ctypes.byref(need))
    assert s == 6 and need.value > 0
    buf = (ctypes.c_int32 * need.value)()
    lb.check(lb.lib.pf_fmm_lists(L, kb, w0, cutoff, theta, buf, need.value, ctypes.byref(need)))
    return list(buf)


CASES = [
    (4, 1, 1.0, 0.0), (5, 1, 1.0, 0.01), (6, 1, 1.0, 0.05), (8, 1, 1.0, 0.0158),
    (9, 1, 3.0, 0.0061), (7, 0, 1.0, 0.02), (6, 2, 2.0, 0.03), (10, 1, 2.0, 0.0127),
]


@pytest.mark.parametrize("L,kb,w0,cutoff", CASES)
def test_tables_bit_exact_vs_restatement(L, kb, w0, cutoff):
    assert lib_tables(L, kb, w0, cutoff) == lists.flatten(lists.build(L, kb, w0, cutoff))


@pytest.mark.parametrize("L,kb,w0,cutoff", [(4, 1, 1.0, 0.0), (4, 1, 1.0, 0.07), (5, 1, 1.0, 0.03),
                                            (4, 0, 1.0, 0.05), (4, 2, 1.0, 0.05)])
def test_every_leaf_pair_covered_once(L, kb, w0, cutoff):
    assert lists.coverage_counts(lists.build(L, kb, w0, cutoff)) == {1}


def test_far_pairs_respect_theta_and_cutoff():
    L, kb, w0, c = 8, 1, 1.0, 0.0158
    t = lists.build(L, kb, w0, c)
    for l in range(1, L + 1):
        w = w0 / 2 ** l
        for f in t["far"][l]:
            for (i, j) in f:
                assert lists.well_separated(i, j, w, c, 0.5)


def test_invalid_arguments_rejected():
    import pfblob._lib as lb
    need = ctypes.c_int64(0)
    assert lb.lib.pf_fmm_lists(0, 1, 1.0, 0.0, 0.5, None, 0, ctypes.byref(need)) == 1
    assert lb.lib.pf_fmm_lists(5, 1, 1.0, 0.0, 1.5, None, 0, ctypes.byref(need)) == 1
