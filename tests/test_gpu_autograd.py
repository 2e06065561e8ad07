"""GPU: the differentiable energy (pyscf_forge_b200.autograd) — backward
equals the RDMs of the reference's make_rdm12 (GAS library in oracle/_ref)
and central finite differences of the solver energy."""
import itertools

import numpy as np
import pytest
import torch

import gasref
from conftest import seeded_integrals

pytestmark = pytest.mark.gpu


def _images(p, q, r, s):
    """Distinct index tuples related to (pq|rs) by the 8-fold symmetry."""
    out = set()
    for a, b, c, d in ((p, q, r, s), (q, p, r, s), (p, q, s, r), (q, p, s, r)):
        out.add((a, b, c, d))
        out.add((c, d, a, b))
    return sorted(out)


def _solver(smult, nroots):
    import pyscf_forge_b200 as P
    sol = P.csf_solver(None, smult=smult)
    sol.nroots = nroots
    sol.conv_tol = 1e-13
    sol.conv_tol_residual = 1e-8
    # the seeded random integrals couple strongly off the diagonal, so the
    # diagonal preconditioner needs a large subspace and many cycles to reach
    # the residual that a finite-difference check needs
    sol.max_space = 30
    sol.max_cycle = 400
    return sol


def _check(norb, nelec, smult, nroots, rank, nfd, seed, step=1e-5, atol=2e-7, ref_rdm=True):
    from pyscf_forge_b200.autograd import csf_fci_energy
    h1, eri = seeded_integrals(norb, rank, seed=seed)
    w = torch.full((nroots,), 1.0 / nroots, dtype=torch.float64)
    h1t = torch.tensor(h1, requires_grad=True)
    erit = torch.tensor(eri, requires_grad=True)
    sol = _solver(smult, nroots)
    e = csf_fci_energy(h1t, erit, norb, nelec, smult=smult, nroots=nroots, solver=sol)
    assert np.all(np.atleast_1d(sol.converged))
    esa = (w * e).sum()
    esa.backward()
    gh1 = h1t.grad.numpy()
    geri = erit.grad.numpy()
    cis = sol.ci if isinstance(sol.ci, list) else [sol.ci]
    if ref_rdm and gasref.available():
        # backward == weighted reference RDMs (make_rdm12 of the GAS library)
        d1 = np.zeros((norb, norb))
        d2 = np.zeros((norb,) * 4)
        for k, c in enumerate(cis):
            r1, r2 = gasref.make_rdm12(c.cpu().numpy(), c.cpu().numpy(), norb, nelec)
            d1 += w[k].item() * r1
            d2 += w[k].item() * r2
        np.testing.assert_allclose(gh1, d1.T, atol=1e-8)        # RDM tolerance 1e-8
        np.testing.assert_allclose(geri, 0.5 * d2, atol=1e-8)
    # central finite differences on random symmetric perturbations
    ci0 = [c.clone() for c in cis]
    rng = np.random.default_rng(seed + 100)

    def energy(h1p, erip):
        s = _solver(smult, nroots)
        ee, _ = s.kernel(h1p, erip, norb, nelec, ci0=ci0)
        return float(np.dot(w.numpy(), np.atleast_1d(ee)))

    for t in range(nfd):
        if t % 2 == 0:
            p, q = sorted(rng.integers(0, norb, size=2))
            d = np.zeros((norb, norb))
            d[p, q] = d[q, p] = 1.0
            fd = (energy(h1 + step * d, eri) - energy(h1 - step * d, eri)) / (2 * step)
            an = gh1[p, q] + (gh1[q, p] if p != q else 0.0)
        else:
            p, q, r, s_ = rng.integers(0, norb, size=4)
            d = np.zeros((norb,) * 4)
            imgs = _images(p, q, r, s_)
            for ix in imgs:
                d[ix] = 1.0
            fd = (energy(h1, eri + step * d) - energy(h1, eri - step * d)) / (2 * step)
            an = sum(geri[ix] for ix in imgs)
        assert abs(fd - an) < atol, (t, fd, an)


def test_autograd_small_two_roots():
    _check(6, (3, 3), 3, 2, 8, nfd=20, seed=11)


def test_autograd_doublet():
    _check(7, (4, 3), 2, 1, 10, nfd=10, seed=12)


def test_autograd_cas14_triplet_state_average():
    """norb=14 (7,7) triplet, 2 roots averaged with equal weights: backward
    against central differences (step 1e-5) on 50 random h1/eri entries and
    against the reference make_rdm12."""
    _check(14, (7, 7), 3, 2, 28, nfd=50, seed=0, atol=5e-7)
