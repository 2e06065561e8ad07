"""GPU: the deterministic sigma (CSFFCI_SIGMA_DETERMINISTIC).  Each
scattered contribution goes into three int64 digit planes by integer
atomics, so a rerun gives the same bits whatever order the atomics land
in.  Checked: two runs are bit-identical (torch.equal) in the general,
spin-symmetric (eta = +1) and antisymmetric (eta = -1) modes and with
accumulation, from 4 orbitals up to the benchmarked CAS(16,16) (8,8); the
result agrees with the FP64-atomic kernel to 1e-12 and with the
reference's own CPU sigma (fci_contract_gas_plan_execute,
pyscf/lib/mcscf/fci_contract_gas.c:2423-2452) to the 1e-9 sigma bar; a
whole solve with deterministic_sigma repeats bit for bit."""
from math import comb

import numpy as np
import pytest
import torch

import gasref
import restate as R
from conftest import seeded_integrals

pytestmark = pytest.mark.gpu

SIGMA_ATOL = 1e-9      # sigma bar against the reference
KERNEL_ATOL = 1e-12    # against the FP64-atomic kernel (different summation)


def _case(norb, nelec, eta, seed):
    h1, eri = seeded_integrals(norb, 2 * norb, seed=seed)
    h2e_np = R.absorb_h1e(h1, eri, norb, nelec, 0.5)
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((comb(norb, nelec[0]), comb(norb, nelec[1])))
    if eta is not None:
        c = c + eta * c.T
    c /= np.linalg.norm(c)
    return h2e_np, c


@pytest.mark.parametrize("norb,nelec,eta", [(10, (5, 5), None), (10, (5, 5), 1), (10, (5, 5), -1),
                                            (12, (6, 5), None), (12, (6, 6), 1), (14, (7, 7), -1),
                                            (8, (4, 3), None), (6, (3, 3), 1), (4, (2, 1), None),
                                            (7, (4, 3), None)])
def test_deterministic_sigma_repeats_and_matches(norb, nelec, eta):
    from pyscf_forge_b200.fci import direct_spin1 as D
    h2e_np, c = _case(norb, nelec, eta, seed=norb * 13 + nelec[1])
    h2e = torch.as_tensor(h2e_np, device="cuda")
    cd = torch.as_tensor(c.ravel(), device="cuda")
    a = D.dev_contract_2e(h2e, cd, norb, nelec, eta=eta, deterministic=True)
    b = D.dev_contract_2e(h2e, cd, norb, nelec, eta=eta, deterministic=True)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    fp = D.dev_contract_2e(h2e, cd, norb, nelec, eta=eta)
    assert float((a - fp).abs().max()) < KERNEL_ATOL
    # accumulate: out += sigma, also bit-identical
    acc1 = cd.clone()
    acc2 = cd.clone()
    D.dev_contract_2e(h2e, cd, norb, nelec, eta=eta, out=acc1, accumulate=True, deterministic=True)
    D.dev_contract_2e(h2e, cd, norb, nelec, eta=eta, out=acc2, accumulate=True, deterministic=True)
    assert torch.equal(acc1, acc2)
    assert float((acc1 - (cd + a)).abs().max()) < KERNEL_ATOL
    if gasref.available() and c.size <= 3_000_000:
        ref = gasref.contract_2e(h2e_np, c, norb, nelec).ravel()
        assert float(np.abs(a.cpu().numpy() - ref).max()) < SIGMA_ATOL


@pytest.mark.skipif(not gasref.available(), reason="oracle/_ref not built")
def test_deterministic_sigma_cas16():
    """The benchmarked space, CAS(16,16) (8,8), singlet vector in the
    spin-symmetric mode: two runs bit-identical, against the reference sigma
    (about 25 s on 16 host threads) and the FP64-atomic kernel."""
    from pyscf_forge_b200.fci import direct_spin1 as D
    norb, nelec = 16, (8, 8)
    h1, eri = seeded_integrals(norb, 32, seed=0)
    h2e_np = R.absorb_h1e(h1, eri, norb, nelec, 0.5)
    rng = np.random.default_rng(7)
    n = comb(16, 8)
    c = rng.standard_normal((n, n))
    c = c + c.T
    c /= np.linalg.norm(c)
    h2e = torch.as_tensor(h2e_np, device="cuda")
    cd = torch.as_tensor(c.ravel(), device="cuda")
    a = D.dev_contract_2e(h2e, cd, norb, nelec, eta=1, deterministic=True)
    b = D.dev_contract_2e(h2e, cd, norb, nelec, eta=1, deterministic=True)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    del b
    fp = D.dev_contract_2e(h2e, cd, norb, nelec, eta=1)
    assert float((a - fp).abs().max()) < KERNEL_ATOL
    del fp
    ref = torch.as_tensor(gasref.contract_2e(h2e_np, c, norb, nelec).ravel(), device="cuda")
    assert float((a - ref).abs().max()) < SIGMA_ATOL


@pytest.mark.parametrize("device_resident", [False, True])
def test_deterministic_solve_repeats(device_resident):
    """FCISolver with deterministic_sigma, in the host-driven Davidson loop
    and in the device-resident plan (every reduction in a fixed order in
    both): two solves of CAS(10,10) with three
    singlet roots give the same energies and CI vectors bit for bit, and
    energies within 1e-9 Eh of the default solver and of the exact singlet
    roots (scipy eigsh over the reference's sigma, S^2 from the oracle:
    -17.31158032, -17.19811638, -16.82364217).  max_space 30: these seeded
    integrals are weakly diagonally dominant, and with the default 12 the
    third root converges in 100 iterations neither in the host loop nor in
    the reference's own solver (csf.py with davidson1 on the stand-in ends
    at -16.823056 Eh)."""
    import pyscf_forge_b200 as P
    h1, eri = seeded_integrals(10, 20, seed=21)
    res = []
    for det in (True, True, False):
        sol = P.csf_solver(None, smult=1)
        sol.nroots = 3
        sol.conv_tol = 1e-11
        sol.max_space = 30
        sol.max_cycle = 400
        sol.deterministic_sigma = det
        sol.device_resident = device_resident
        e, ci = sol.kernel(h1, eri, 10, (5, 5))
        assert np.all(sol.converged)
        res.append((np.asarray(e), [np.asarray(x) for x in ci]))
    (e1, c1), (e2, c2), (e3, _) = res
    assert np.array_equal(e1, e2)
    assert all(np.array_equal(x, y) for x, y in zip(c1, c2))
    np.testing.assert_allclose(e1, e3, atol=1e-9)
    np.testing.assert_allclose(e1, [-17.31158032, -17.19811638, -16.82364217], atol=1e-7)


def test_deterministic_sigma_many():
    """The job-table form (csffci_sigma_batch with every job flagged
    CSFFCI_SIGMA_JOB_DETERMINISTIC): mixed orbital counts 4..16, general,
    symmetric and antisymmetric jobs in one call; two calls bit-identical,
    each job against the one-problem deterministic sigma (bit-identical:
    the same digit sums) and the reference sigma."""
    from pyscf_forge_b200 import batched as B
    from pyscf_forge_b200.fci import direct_spin1 as D
    cases = [(4, (2, 1), None), (6, (3, 3), 1), (8, (4, 4), -1), (8, (4, 3), None), (10, (5, 5), 1),
             (12, (6, 5), None), (12, (2, 2), -1), (16, (3, 2), None)]
    items, host = [], []
    for i, (norb, nelec, eta) in enumerate(cases):
        h2e_np, c = _case(norb, nelec, eta, seed=40 + i)
        items.append((torch.as_tensor(h2e_np, device="cuda"), torch.as_tensor(c.ravel(), device="cuda"),
                      norb, nelec, eta))
        host.append((h2e_np, c))
    a = B.sigma_many(items, deterministic=True)
    b = B.sigma_many(items, deterministic=True)
    for (h2e, cd, norb, nelec, eta), x, y, (h2e_np, c) in zip(items, a, b, host):
        assert torch.equal(x, y), (norb, nelec, eta)
        one = D.dev_contract_2e(h2e, cd, norb, nelec, eta=eta, deterministic=True)
        assert torch.equal(x, one), (norb, nelec, eta)
        if gasref.available():
            ref = gasref.contract_2e(h2e_np, c, norb, nelec).ravel()
            assert float(np.abs(x.cpu().numpy() - ref).max()) < SIGMA_ATOL


def test_deterministic_batched_solver_repeats():
    """BatchedCSFSolver(deterministic=True): an uneven batch (norb 6..10,
    1-4 roots, several spins) solved twice gives the same energies and CI
    vectors bit for bit, and energies within 1e-10 Eh of the default
    batched solver."""
    from pyscf_forge_b200 import batched as B
    probs = B.make_uneven_batch(10, seed0=5000, norb_lo=6, norb_hi=10)
    kw = dict(conv_tol=1e-12, conv_tol_residual=1e-7, max_cycle=400, max_space=30)
    r1 = B.BatchedCSFSolver(deterministic=True, **kw).kernel(probs, with_rdm=False)
    r2 = B.BatchedCSFSolver(deterministic=True, **kw).kernel(probs, with_rdm=False)
    r3 = B.BatchedCSFSolver(**kw).kernel(probs, with_rdm=False)
    for p, x, y, z in zip(probs, r1, r2, r3):
        assert x[3] and y[3] and z[3]
        assert np.array_equal(np.asarray(x[0]), np.asarray(y[0])), (p.norb, p.nelec, p.smult)
        assert all(np.array_equal(np.asarray(u), np.asarray(v)) for u, v in zip(x[1], y[1]))
        np.testing.assert_allclose(x[0], z[0], atol=1e-10)
