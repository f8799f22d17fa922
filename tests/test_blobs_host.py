"""Host logic of the Blobs class (no GPU): the diffusion time step and its
multiple of the convection step (src/python/blobs/__blobsClass.py:2248-2318),
with the reference's Python-2 rounding of halves."""
import pytest


def _blobs(method, nu, h, deltaTc, c2="optimized"):
    from pfblob.blobs import Blobs
    b = Blobs.__new__(Blobs)
    b._nu, b._h, b._deltaTc = float(nu), float(h), float(deltaTc)
    b._diffusionParams = {"method": method, "c2": c2}
    return b


def test_wee_optimized_step_is_rounded_to_a_multiple_of_deltaTc():
    # ideal deltaTd = h^2 / (3 nu) = 1/3 * 1e-4 / 1e-3 = 0.0333..; / 0.01 = 3.33 -> 3 steps
    b = _blobs("regrid_wee", nu=1e-3, h=0.01, deltaTc=0.01)
    dtd, step = b._compute_deltaTd()
    assert step == 3 and dtd == 3 * 0.01


def test_wee_half_way_ratio_rounds_up_like_the_reference():
    # ideal deltaTd = c2 h^2 / nu = 0.625; deltaTc = 0.25: ratio exactly 2.5.
    # The reference's Python-2 round gives 3 (Python 3's round would give 2).
    b = _blobs("regrid_wee", nu=1.0, h=1.0, deltaTc=0.25, c2=0.625)
    dtd, step = b._compute_deltaTd()
    assert step == 3 and dtd == 0.75
    b = _blobs("regrid_wee", nu=1.0, h=1.0, deltaTc=0.25, c2=0.875)  # ratio 3.5 -> 4
    assert b._compute_deltaTd() == (1.0, 4)


def test_wee_step_too_large_raises():
    b = _blobs("regrid_wee", nu=1.0, h=0.01, deltaTc=1.0)
    with pytest.raises(ValueError, match="Regrid Wee"):
        b._compute_deltaTd()


def test_inviscid_has_no_diffusion():
    for m in ("regrid_wee", "regrid_tutty"):
        assert _blobs(m, nu=0.0, h=0.01, deltaTc=0.1)._compute_deltaTd() == (0.0, 0)


def test_tutty_diffuses_every_step_within_its_stability_limit():
    b = _blobs("regrid_tutty", nu=1e-3, h=0.01, deltaTc=0.01)  # hNu/h = 0.316
    assert b._compute_deltaTd() == (0.01, 1)
    b = _blobs("regrid_tutty", nu=1e-3, h=0.01, deltaTc=0.06)  # hNu/h = 0.775 > 1/sqrt(2)
    with pytest.raises(ValueError, match="Regrid Tutty"):
        b._compute_deltaTd()


def test_round_half_away():
    from pfblob.blobs import _round_half_away
    assert [_round_half_away(v) for v in (1.0, 1.49999, 1.5, 2.5, 2.5000001, 7.0)] == \
        [1, 1, 2, 3, 3, 7]


def test_blobs_from_a_vorticity_function_sit_at_cell_centres():
    """wField = (w, xBounds, yBounds): floor(width / h) blobs per direction at
    xBounds[0] + h/2 + i h, x varying fastest, circulation w h^2
    (__blobsClass.py:1406-1419)."""
    import numpy as np
    from pfblob.blobs import Blobs
    b = Blobs.__new__(Blobs)
    x, y, g = b._blobs_from_function((lambda x, y: x + 10.0 * y, [-1.0, 1.0], [0.0, 1.2]), 0.5)
    assert np.array_equal(x, [-0.75, -0.25, 0.25, 0.75] * 2)
    assert np.array_equal(y, [0.25] * 4 + [0.75] * 4)
    assert np.array_equal(g, (x + 10.0 * y) * 0.25)


def _blobs_with_state(n):
    import torch
    from pfblob.blobs import Blobs
    b = Blobs.__new__(Blobs)
    b.device = torch.device("cpu")  # the host logic only; the state is a plain tensor here
    b._x = torch.arange(n, dtype=torch.float64)
    b._y = 10.0 * b._x
    b._g = 100.0 * b._x
    return b


def test_remove_blobs_like_the_reference():
    """int64 indices delete (negative ones from the end, as numpy.delete);
    a bool mask of numBlobs entries KEEPS the selected blobs, because the
    reference indexes with it (__blobsClass.py:935-955)."""
    import numpy as np
    b = _blobs_with_state(6)
    b.removeBlobs(np.array([0, 3, -1], dtype=np.int64))
    assert b._x.tolist() == [1.0, 2.0, 4.0] and b._g.tolist() == [100.0, 200.0, 400.0]
    b.removeBlobs(np.array([True, False, True]))
    assert b._x.tolist() == [1.0, 4.0] and b._y.tolist() == [10.0, 40.0]


def test_remove_blobs_rejects_what_the_reference_rejects():
    import numpy as np
    b = _blobs_with_state(4)
    for bad in ([1, 2], np.array([4], dtype=np.int64), np.array([True, False]),
                np.array([1.0, 2.0])):
        with pytest.raises(TypeError):
            b.removeBlobs(bad)
    assert b.numBlobs == 4
