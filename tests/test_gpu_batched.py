"""GPU: the batched many-problem path (pyscf_forge_b200.batched) — batched
sigma and det<->CSF transforms against the one-problem kernels and the
oracle, and the lockstep solver against the one-problem solver and the
reference make_rdm12 (GAS library in oracle/_ref)."""
from math import comb

import numpy as np
import pytest
import torch

import gasref
import restate
from conftest import seeded_integrals

pytestmark = pytest.mark.gpu


def _h2e(h1, eri, norb, nelec):
    from pyscf_forge_b200.fci import direct_spin1 as D
    from pyscf_forge_b200._runtime import eri_pair_matrix
    return D.dev_absorb_h1e(h1, eri_pair_matrix(eri, norb), norb, nelec, 0.5)


def test_sigma_many_matches_single_and_oracle():
    """Jobs of mixed norb (two launches), electron counts and symmetric /
    general modes in one call; each against csffci_sigma and the oracle."""
    from pyscf_forge_b200 import batched as B
    from pyscf_forge_b200.fci import direct_spin1 as D
    rng = np.random.default_rng(5)
    cases = [(6, (3, 3), True), (6, (3, 2), False), (6, (2, 2), False), (6, (3, 3), False),
             (8, (4, 4), True), (8, (4, 3), False), (8, (1, 0), False), (8, (4, 4), False)]
    items, host = [], []
    for norb, nelec, sym in cases:
        h1, eri = seeded_integrals(norb, 2 * norb, seed=norb * 10 + nelec[0] + nelec[1])
        h2e = _h2e(h1, eri, norb, nelec)
        na, nb = comb(norb, nelec[0]), comb(norb, nelec[1])
        c = rng.standard_normal((na, nb))
        eta = None
        if sym:
            c = c + c.T
            eta = 1
        items.append((h2e, torch.as_tensor(c.ravel(), device="cuda"), norb, nelec, eta))
        host.append((h1, eri, norb, nelec, c))
    outs = B.sigma_many(items)
    for (h2e, cd, norb, nelec, eta), out, (h1, eri, _, _, c) in zip(items, outs, host):
        one = D.dev_contract_2e(h2e, cd, norb, nelec, eta=eta)
        np.testing.assert_allclose(out.cpu().numpy(), one.cpu().numpy(), atol=1e-11)
        h2e_np = restate.absorb_h1e(h1, eri, norb, nelec, 0.5)
        ref = restate.contract_2e(h2e_np, c, norb, nelec).ravel()
        np.testing.assert_allclose(out.cpu().numpy(), ref, atol=1e-9)    # sigma tolerance 1e-9


@pytest.mark.parametrize("variant", ["4", "7"])
def test_sigma_many_warp_specialised_job_table(monkeypatch, variant):
    """The warp-specialised kernel over a job table: variant 4 (8-row MMA
    warps, 4..16 orbitals; the default at 10..12 and 14..16) and variant 7
    (16-row MMA warps in 8-warp CTAs, 8..12 orbitals), both autotuner
    candidates.  Jobs past a variant's orbital range run the default kernel:
    jobs of mixed electron counts and symmetric / general / antisymmetric
    modes, several orbital counts, against the one-problem kernel and the
    oracle."""
    from pyscf_forge_b200 import batched as B
    from pyscf_forge_b200.fci import direct_spin1 as D
    rng = np.random.default_rng(11)
    cases = [(8, (4, 4), 1), (8, (4, 3), None), (8, (1, 0), None), (9, (5, 4), None), (9, (4, 4), -1),
             (10, (5, 5), 1), (10, (4, 3), None), (11, (6, 5), None), (11, (5, 5), 1), (12, (6, 6), 1),
             (12, (7, 6), None), (12, (5, 5), None), (12, (6, 6), -1), (12, (2, 1), None),
             (13, (6, 5), None), (14, (5, 5), 1), (16, (3, 3), 1), (16, (3, 2), None)]
    items, host = [], []
    for norb, nelec, eta in cases:
        h1, eri = seeded_integrals(norb, 2 * norb, seed=norb * 7 + nelec[0] - nelec[1])
        h2e = _h2e(h1, eri, norb, nelec)
        c = rng.standard_normal((comb(norb, nelec[0]), comb(norb, nelec[1])))
        if eta is not None:
            c = c + eta * c.T
        items.append((h2e, torch.as_tensor(c.ravel(), device="cuda"), norb, nelec, eta))
        host.append((h1, eri, c))
    monkeypatch.setenv("CSFFCI_SIGMA_VARIANT", variant)
    outs = B.sigma_many(items)
    monkeypatch.delenv("CSFFCI_SIGMA_VARIANT")
    for (h2e, cd, norb, nelec, eta), out, (h1, eri, c) in zip(items, outs, host):
        one = D.dev_contract_2e(h2e, cd, norb, nelec, eta=eta)
        np.testing.assert_allclose(out.cpu().numpy(), one.cpu().numpy(), atol=1e-11)
        if norb <= 10:
            h2e_np = restate.absorb_h1e(h1, eri, norb, nelec, 0.5)
            ref = restate.contract_2e(h2e_np, c, norb, nelec).ravel()
            np.testing.assert_allclose(out.cpu().numpy(), ref, atol=1e-9)    # sigma tolerance 1e-9
        elif gasref.available() and c.size <= 4_000_000:
            ref = gasref.contract_2e(restate.absorb_h1e(h1, eri, norb, nelec, 0.5), c, norb, nelec).ravel()
            np.testing.assert_allclose(out.cpu().numpy(), ref, atol=1e-9)


def test_transform_many_round_trip():
    """Batched csf->det and det->csf against the per-transformer kernels for
    several spaces at once; det->csf(csf->det(x)) == x.  Blocks of at most
    16 CSFs and 256 determinants take the row-per-thread path, the others
    (norb 10 and 11 below) the 32 x 32 tiles."""
    from pyscf_forge_b200 import batched as B
    from pyscf_forge_b200.csf_fci.csfstring import CSFTransformer
    rng = np.random.default_rng(9)
    spaces = [(6, 3, 3, 1), (6, 3, 3, 3), (7, 4, 3, 2), (8, 4, 4, 5), (5, 1, 0, 2), (8, 3, 3, 1),
              (10, 5, 5, 1), (11, 6, 5, 2), (12, 6, 6, 3)]
    ts = [CSFTransformer(*s) for s in spaces]
    xs = [torch.as_tensor(rng.standard_normal((1 + i % 3, t.ncsf)), device="cuda") for i, t in enumerate(ts)]
    dets = B.transform_many(list(zip(ts, xs)), reverse=True)
    for t, x, d in zip(ts, xs, dets):
        np.testing.assert_allclose(d.cpu().numpy(), t.dev_csf2det(x).cpu().numpy(), atol=1e-13)
    back = B.transform_many(list(zip(ts, dets)), reverse=False)
    for t, x, d, y in zip(ts, xs, dets, back):
        np.testing.assert_allclose(y.cpu().numpy(), t.dev_det2csf(d).cpu().numpy(), atol=1e-13)
        np.testing.assert_allclose(y.cpu().numpy(), x.cpu().numpy(), atol=1e-12)


def test_batched_solver_matches_plain():
    """An uneven batch (norb 6..9, 1-4 roots, several spins, exact and
    Davidson problems): energies within 1e-9 of the one-problem solver,
    every root converged, RDMs against the one-problem solver and the
    reference make_rdm12."""
    from pyscf_forge_b200 import batched as B
    probs = B.make_uneven_batch(12, seed0=2000, norb_lo=6, norb_hi=9)
    kw = dict(conv_tol=1e-12, conv_tol_residual=1e-7, max_cycle=400)
    res = B.BatchedCSFSolver(**kw).kernel(probs)
    plain = B.solve_plain(probs, **kw)
    for p, (eb, cib, rdb, conv), (ep, cip, rdp) in zip(probs, res, plain):
        assert conv, (p.norb, p.nelec, p.smult, p.nroots)
        np.testing.assert_allclose(eb, ep, atol=1e-9)
        for k in range(len(eb)):
            # non-degenerate roots only: RDMs are phase-invariant
            gaps = np.abs(np.delete(eb, k) - eb[k])
            if gaps.size and gaps.min() < 1e-4:
                continue
            np.testing.assert_allclose(rdb[k][0], rdp[k][0], atol=1e-6)
            np.testing.assert_allclose(rdb[k][1], rdp[k][1], atol=1e-6)
            if gasref.available():
                c = cib[k]
                r1, r2 = gasref.make_rdm12(c, c, p.norb, p.nelec)
                np.testing.assert_allclose(rdb[k][0], r1, atol=1e-8)   # RDM tolerance 1e-8
                np.testing.assert_allclose(rdb[k][1], r2, atol=1e-8)
        assert cib[0].shape == (comb(p.norb, p.nelec[0]), comb(p.norb, p.nelec[1]))


def test_device_engine_matches_host_engine_and_graph_replay():
    """The device-resident plan (every Davidson step on the GPU, one
    iteration replayed as a CUDA graph) against the same plan launched
    eagerly and against the host-driven lockstep engine: same energies,
    every problem converged; the autotuner reports a valid tile variant
    for each orbital count."""
    from pyscf_forge_b200 import batched as B
    probs = B.make_uneven_batch(10, seed0=3000, norb_lo=7, norb_hi=10)
    kw = dict(conv_tol=1e-12, conv_tol_residual=1e-7, max_cycle=400)
    sg = B.BatchedCSFSolver(engine="device", use_graph=True, **kw)
    rg = sg.kernel(probs, with_rdm=False)
    re_ = B.BatchedCSFSolver(engine="device", use_graph=False, autotune=False, **kw).kernel(probs, with_rdm=False)
    rh = B.BatchedCSFSolver(engine="host", **kw).kernel(probs, with_rdm=False)
    for a, b, c in zip(rg, re_, rh):
        assert a[3] and b[3] and c[3]
        np.testing.assert_allclose(a[0], b[0], atol=1e-10)
        np.testing.assert_allclose(a[0], c[0], atol=1e-10)
    assert sg.tile_variants and all(0 <= v <= 4 or v == 7 for v in sg.tile_variants.values())
    assert set(sg.tile_variants) <= {p.norb for p in probs}


@pytest.mark.parametrize("variant", ["4", "7"])
def test_device_engine_warp_specialised_gated(monkeypatch, variant):
    """The device-resident plan with every orbital count from 8 up on a
    warp-specialised job-table kernel (autotuner off, the variant named):
    its jobs are gated as problems converge, so units of converged problems
    are skipped inside the launch.  Same energies as the tile-shape kernel
    (variant 2)."""
    from pyscf_forge_b200 import batched as B
    probs = B.make_uneven_batch(12, seed0=3100, norb_lo=8, norb_hi=11)
    kw = dict(conv_tol=1e-12, conv_tol_residual=1e-7, max_cycle=400)
    monkeypatch.setenv("CSFFCI_SIGMA_VARIANT", "2")
    ref = B.BatchedCSFSolver(engine="device", autotune=False, **kw).kernel(probs, with_rdm=False)
    monkeypatch.setenv("CSFFCI_SIGMA_VARIANT", variant)
    sw = B.BatchedCSFSolver(engine="device", autotune=False, **kw)
    got = sw.kernel(probs, with_rdm=False)
    monkeypatch.delenv("CSFFCI_SIGMA_VARIANT")
    for p, a, b in zip(probs, got, ref):
        assert a[3] and b[3]
        np.testing.assert_allclose(a[0], b[0], atol=1e-10)
    assert all(v == int(variant) for n, v in sw.tile_variants.items() if 8 <= n <= 12)


def test_c3_batch_energies_vs_reference():
    """The benchmark's 128-problem uneven batch (C3) through the device
    batched solver, against the energies of the reference's own csf.py
    kernel on the stand-in (tests/golden/c3_batch128.npz, made by
    tests/golden/make_c3_golden.py with the same solver settings): the
    batch generator makes the fixture's problems, every problem converges,
    and every root is within 1e-9 Eh of the reference."""
    import os
    from conftest import GOLDEN
    path = os.path.join(GOLDEN, "c3_batch128.npz")
    if not os.path.exists(path):
        pytest.skip("C3 fixture not generated")
    from pyscf_forge_b200 import batched as B
    g = np.load(path)
    conv_tol, max_cycle, max_space = g["settings"]
    probs = B.make_uneven_batch(128)
    got = np.array([(i, p.norb, p.nelec[0], p.nelec[1], p.smult, p.nroots) for i, p in enumerate(probs)])
    assert np.array_equal(got, g["problems"])
    assert g["converged"].all()
    sol = B.BatchedCSFSolver(conv_tol=float(conv_tol), max_cycle=int(max_cycle), max_space=int(max_space))
    res = sol.kernel(probs, with_rdm=False)
    for i, r in enumerate(res):
        e = np.asarray(r[0])
        assert bool(np.all(r[3])), ("problem %d not converged" % i)
        np.testing.assert_allclose(e, g["energies"][i, :len(e)], atol=1e-9, err_msg="problem %d" % i)
