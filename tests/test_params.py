"""Blob-to-FMM parameter conversion on the host (no GPU): the reference's
xopt / cutoff derivation (src/python/blobs/base/induced/_induced.py:236-239)
and this library's tolerance-lowered default near-field radius."""
import math

import pytest

from pfblob.induced import FMM_ALPHA, default_cutoff, fmm_parameters


@pytest.mark.parametrize("sigma", [1e-5, 0.002, 0.0125, 0.3])
def test_xopt_is_the_reference_conversion(sigma):
    ks, xopt, _ = fmm_parameters(sigma, k=2.0)
    assert ks == 2.0 * sigma * sigma
    assert xopt == math.sqrt(1.2564312086261696770 * ks)
    # the FMM's Oseen shape alpha / xopt^2 is the blob kernel's 1 / (k sigma^2)
    assert abs(FMM_ALPHA / (xopt * xopt) * ks - 1.0) < 1e-15


def test_default_cutoff_never_exceeds_the_reference_radius():
    for sigma in (1e-4, 0.002, 0.05):
        ks = 2.0 * sigma * sigma
        five_xopt = 5.0 * math.sqrt(FMM_ALPHA * ks)
        assert default_cutoff(ks, 0.0) == five_xopt  # no tolerance: the reference's 5 xopt
        for tol in (1e-3, 1e-6, 1e-9, 1e-12):
            cut = default_cutoff(ks, tol)
            assert cut <= five_xopt
            if cut < five_xopt:
                # lowered: the core's correction exp(-r^2 / k sigma^2) at the radius is tol / 100
                assert abs(math.exp(-cut * cut / ks) / (tol / 100) - 1.0) < 1e-9


def test_tolerance_binds_until_the_reference_radius_is_tighter():
    ks = 8e-6
    five_xopt = 5.0 * math.sqrt(FMM_ALPHA * ks)
    # 5 xopt leaves a correction of exp(-25 alpha) ~ 2e-14: tolerances above
    # 2e-12 lower the radius, tighter ones keep 5 xopt
    assert default_cutoff(ks, 1e-6) < five_xopt
    assert default_cutoff(ks, 1e-13) == five_xopt
    assert abs(math.exp(-25.0 * FMM_ALPHA) - 2.3e-14) < 1e-15


def test_explicit_cutoff_is_honoured():
    ks, xopt, cut = fmm_parameters(0.002, cutoff=0.123)
    assert cut == 0.123
