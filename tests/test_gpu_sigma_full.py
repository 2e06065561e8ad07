"""Sigma parity at the benchmarked sizes: the warp-specialised kernels
(variant 4 from 14 orbitals; variants 5 and 6 -- registers re-split
between the warp roles, 6 with the alpha rows moved by the bulk-copy engine
-- at 16) and the phase-serial
kernel (variant 1) against the
reference's own CPU sigma (fci_contract_gas_plan_execute,
pyscf/lib/mcscf/fci_contract_gas.c:2423-2452, one GAS subspace = full CAS)
on the same seeded vectors.

  * CAS(16,16) (8,8): a symmetric vector (the singlet case of the
    benchmark) in the general and the spin-symmetric (eta = +1) mode, and an
    antisymmetric vector in the eta = -1 mode;
  * CAS(16,16) (8,7): general mode (Na != Nb);
  * CAS(14,14) (7,7): singlet and triplet vectors built from random CSFs
    (eta = +1 and -1, the vectors the CSF Davidson feeds to sigma).

Tolerance: 1e-9 max abs (the sigma bar of the north-star target), and
1e-12 between the GPU kernels.  One reference sigma at CAS(16,16)
takes about 25 s on 16 host threads."""
from math import comb

import numpy as np
import pytest
import torch

import gasref
import restate as R
from conftest import seeded_integrals

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gasref.available(), reason="oracle/_ref not built")]

SIGMA_ATOL = 1e-9      # sigma bar against the reference
KERNEL_ATOL = 1e-12    # between the GPU kernels (same arithmetic, different order)


def _dev_sigma(h2e, c, norb, nelec, eta, variant, monkeypatch):
    from pyscf_forge_b200.fci import direct_spin1 as D
    monkeypatch.setenv("CSFFCI_SIGMA_VARIANT", str(variant))
    try:
        out = D.dev_contract_2e(h2e, c, norb, nelec, eta=eta)
        torch.cuda.synchronize()
        return out
    finally:
        monkeypatch.delenv("CSFFCI_SIGMA_VARIANT")


def _check(h2e_np, c_np, norb, nelec, etas, monkeypatch, variants=(4, 1)):
    """Every variant against the reference sigma, and against the first
    variant."""
    ref = gasref.contract_2e(h2e_np, c_np, norb, nelec).ravel()
    h2e = torch.as_tensor(h2e_np, device="cuda")
    cd = torch.as_tensor(c_np.ravel(), device="cuda")
    refd = torch.as_tensor(ref, device="cuda")
    del ref
    scale = float(refd.abs().max())
    errs = {}
    for eta in etas:
        outs = {}
        for v in variants:
            outs[v] = _dev_sigma(h2e, cd, norb, nelec, eta, v, monkeypatch)
            errs[(eta, v)] = float((outs[v] - refd).abs().max())
            assert errs[(eta, v)] < SIGMA_ATOL, (eta, v, errs[(eta, v)], scale)
        for v in variants[1:]:
            d = float((outs[variants[0]] - outs[v]).abs().max())
            assert d < KERNEL_ATOL, (eta, v, d)
        del outs
    return errs


def _integrals(norb, nelec, rank, seed):
    h1, eri = seeded_integrals(norb, rank, seed=seed)
    return R.absorb_h1e(h1, eri, norb, nelec, 0.5)


@pytest.fixture(scope="module")
def cas16_h2e():
    return _integrals(16, (8, 8), 32, 0)


def test_cas16_symmetric_general_and_spin_symmetric(cas16_h2e, monkeypatch):
    """The benchmarked configuration: CAS(16,16) (8,8), c = c^T."""
    n = comb(16, 8)
    rng = np.random.default_rng(1)
    c = rng.normal(size=(n, n))
    c += c.T
    c /= np.linalg.norm(c)
    _check(cas16_h2e, c, 16, (8, 8), (None, 1), monkeypatch, variants=(6, 5, 4, 1))


def test_cas16_antisymmetric(cas16_h2e, monkeypatch):
    """CAS(16,16) (8,8), c = -c^T, spin-symmetric mode with eta = -1."""
    n = comb(16, 8)
    rng = np.random.default_rng(2)
    c = rng.normal(size=(n, n))
    c -= c.T
    c /= np.linalg.norm(c)
    _check(cas16_h2e, c, 16, (8, 8), (-1,), monkeypatch, variants=(6, 5, 4, 1))


def test_cas16_8_7_general(monkeypatch):
    """CAS(16,16) with (8,7) electrons: Na != Nb, general mode only."""
    h2e = _integrals(16, (8, 7), 32, 3)
    rng = np.random.default_rng(4)
    c = rng.normal(size=comb(16, 8) * comb(16, 7))
    c /= np.linalg.norm(c)
    _check(h2e, c, 16, (8, 7), (None,), monkeypatch, variants=(6, 5, 4, 1))


@pytest.mark.parametrize("smult", [1, 3])
def test_cas14_from_csfs(smult, monkeypatch):
    """CAS(14,14) (7,7) vectors built from random CSFs of spin multiplicity
    smult: the singlet takes eta = +1, the triplet eta = -1."""
    from pyscf_forge_b200.csf_fci.csfstring import CSFTransformer
    norb, nelec = 14, (7, 7)
    t = CSFTransformer(norb, 7, 7, smult)
    g = torch.Generator(device="cpu").manual_seed(5 + smult)
    x = torch.randn(t.ncsf, generator=g, dtype=torch.float64).cuda()
    c = t.dev_csf2det(x)[0]
    c /= torch.linalg.norm(c)
    eta = t.spin_parity
    assert eta == (1 if smult == 1 else -1)
    h2e = _integrals(norb, nelec, 28, 6)
    _check(h2e, c.cpu().numpy(), norb, nelec, (None, eta), monkeypatch)
