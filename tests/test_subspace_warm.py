"""CPU: the warm start of the batched Davidson's subspace eigensolver
(k_db_sritz, pyscf-forge_b200/csrc/davbatch.cu).  The first m0 basis
vectors were diagonalised at the previous iteration (eigenvectors Q_prev,
eigenvalues d_prev); in the basis diag(Q_prev, I) the new subspace matrix is
diag(d_prev) bordered by Q_prev^T h[:m0, m0:] and h[m0:, m0:].  Restated with
numpy: that matrix has the eigenvalues of h, and diag(Q_prev, I) times its
eigenvectors are eigenvectors of h.  After a restart the basis is the Ritz
vectors, h = diag(e), and Q_prev is the identity."""
import numpy as np
import pytest


def _warm(h, m0, qprev, dprev):
    m = h.shape[0]
    a = np.array(h, dtype=float)
    a[:m0, :m0] = np.diag(dprev)
    border = qprev.T @ h[:m0, m0:]
    a[:m0, m0:] = border
    a[m0:, :m0] = border.T
    qt = np.eye(m)
    qt[:m0, :m0] = qprev
    return a, qt


@pytest.mark.parametrize("m0,knew,seed", [(5, 1, 0), (12, 3, 1), (30, 4, 2), (1, 8, 3)])
def test_warm_started_subspace_matrix(m0, knew, seed):
    rng = np.random.default_rng(seed)
    m = m0 + knew
    b = rng.standard_normal((m, m))
    h = 0.5 * (b + b.T) + np.diag(np.linspace(-3.0, 1.0, m))
    dprev, qprev = np.linalg.eigh(h[:m0, :m0])
    a, qt = _warm(h, m0, qprev, dprev)
    np.testing.assert_allclose(a, a.T, atol=0.0)
    w_ref, _ = np.linalg.eigh(h)
    w, r = np.linalg.eigh(a)
    np.testing.assert_allclose(w, w_ref, atol=1e-12)
    q = qt @ r
    np.testing.assert_allclose(h @ q, q * w, atol=1e-11)


def test_restart_basis_is_diagonal():
    """After a restart h = diag(e) over the kept Ritz vectors: the warm
    matrix equals h and the starting basis is the identity."""
    e = np.array([-2.0, -1.5, -0.25])
    h = np.diag(e)
    a, qt = _warm(h, 3, np.eye(3), e)
    np.testing.assert_array_equal(a, h)
    np.testing.assert_array_equal(qt, np.eye(3))
