"""Panel influence matrix (vs the reference Cython assemble_influenceMatrix)
and the on-device LU factor / solve of the panel system (vs numpy's solve)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_influence_matrix_vs_reference_golden(golden):
    import pfblob
    d = golden("panel_influence")
    A = pfblob.influenceMatrix(d["xcp"], d["ycp"], d["xs"], d["ys"], d["xe"], d["ye"], d["cosa"],
                               d["sina"])
    assert A.shape == d["A"].shape
    assert np.abs(A - d["A"]).max() <= 1e-12 * np.abs(d["A"]).max()


@pytest.mark.parametrize("n", [1, 31, 96, 700])
def test_lu_solve_matches_numpy(golden, n):
    import pfblob
    rng = np.random.default_rng(n)
    if n == 96:
        A = golden("panel_influence")["A"]
    else:
        A = rng.standard_normal((n, n)) + n * np.eye(n) * 0.1
    b = rng.standard_normal(n)
    lu, piv = pfblob.lu_factor(A)
    x = pfblob.lu_solve((lu, piv), b)
    ref = np.linalg.solve(A, b)
    assert np.abs(x - ref).max() <= 1e-10 * np.abs(ref).max()
    assert np.abs(A @ x - b).max() <= 1e-12 * np.abs(A).max() * np.abs(x).max() * n
    # device tensors in, device tensors out, same numbers
    At = torch.from_numpy(A).cuda()
    lt, pt = pfblob.lu_factor(At)
    xt = pfblob.lu_solve((lt, pt), torch.from_numpy(b).cuda())
    assert np.array_equal(xt.cpu().numpy(), x)
    assert torch.equal(At, torch.from_numpy(A).cuda())  # input not overwritten


def test_partial_pivoting_and_singular_warning():
    import pfblob
    A = np.array([[0.0, 2.0, 1.0], [1.0, 1.0, 0.0], [3.0, 0.0, 1.0]])
    b = np.array([1.0, 2.0, 3.0])
    lu, piv = pfblob.lu_factor(A)
    assert piv[0] == 2  # largest |a_i0| is row 2
    assert np.allclose(pfblob.lu_solve((lu, piv), b), np.linalg.solve(A, b), rtol=1e-14)
    S = np.array([[1.0, 2.0], [2.0, 4.0]])
    with pytest.warns(RuntimeWarning):
        pfblob.lu_factor(S)
