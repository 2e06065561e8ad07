"""Generate tests/golden/c3_batch128.npz: reference energies of the 128
seeded uneven problems of the batched-solve configuration (C3), and the
reference's own CPU time per problem.

Each problem is solved by the reference's unmodified pyscf/csf_fci/csf.py
kernel (read from the reference checkout) on the PySCF stand-in under
oracle/shim: transforms by the reference's csfstring.py, sigma by the
reference's own C (libfci_gas, one GAS subspace), Davidson by the
restatement of lib.davidson1 in oracle/davidson_np.py; the 1-/2-RDMs of
every root then come from the reference's C (fci_rdm_gas).  Solver settings
are those of the benchmark: conv_tol 1e-10, max_cycle 400, max_space 30.
The reference defaults (max_space 12) leave one of these problems (index
82, norb 10, (6,5) doublet, root 1) unconverged after 400 iterations, in the
reference's iteration and in ours alike: its integrals are far from
diagonally dominant (lowest CSF diagonal -17.5 Eh against E0 = -20.54 Eh)
and root 1 lies 5 mEh below root 2, so a 16-vector restarted subspace
converges at a Krylov-like rate; with max_space 30 it converges to the
eigenvalue scipy's eigsh gives (-20.26509696).

The problem list is restated here from its definition (seed 1000+i; norb
U{6..12}; N = 2*ceil(norb/2) + U{-2..2} clipped to [2, 2 norb - 2]; MS = 0
or 1/2; S redrawn from U{0,1,2} (+1/2) until the reference's
count_all_csfs accepts it; nroots U{1..4} capped at ncsf; integrals of rank
2 norb) and stored with the energies, so the GPU test checks that the
library's batch generator makes the same problems.  Only this container can
run it (it needs the reference checkout); one worker process per core, one
thread each.

    python tests/golden/make_c3_golden.py [--workers 8]
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
SETTINGS = dict(conv_tol=1e-10, max_cycle=400, max_space=30)


def _paths():
    for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "oracle", "shim")):
        if p not in sys.path:
            sys.path.insert(0, p)


def seeded_integrals(norb, rank, seed):
    rng = np.random.default_rng(seed)
    h1 = rng.normal(0.0, 0.3, (norb, norb))
    h1 = 0.5 * (h1 + h1.T)
    np.fill_diagonal(h1, np.linspace(-2.0, 0.5, norb))
    L = rng.normal(0.0, 0.2, (rank, norb * norb)).reshape(rank, norb, norb)
    L = 0.5 * (L + L.transpose(0, 2, 1))
    return h1, 0.5 * np.einsum("xpq,xrs->pqrs", L, L)


def problems(nprob=128, seed0=1000, norb_lo=6, norb_hi=12):
    _paths()
    from pyscf.csf_fci.csfstring import ImpossibleCIvecError, count_all_csfs
    out = []
    for i in range(nprob):
        rng = np.random.default_rng(seed0 + i)
        norb = int(rng.integers(norb_lo, norb_hi + 1))
        ntot = 2 * ((norb + 1) // 2) + int(rng.integers(-2, 3))
        ntot = max(2, min(ntot, 2 * norb - 2))
        ms2 = ntot % 2
        na, nb = (ntot + ms2) // 2, (ntot - ms2) // 2
        while True:
            s2 = ms2 + 2 * int(rng.integers(0, 3))
            try:
                ncsf = int(count_all_csfs(norb, na, nb, s2 + 1))
            except ImpossibleCIvecError:
                continue
            if ncsf > 0:
                break
        nroots = min(int(rng.integers(1, 5)), ncsf)
        out.append((i, norb, na, nb, s2 + 1, nroots, seed0 + i))
    return out


def solve(p):
    os.environ["OMP_NUM_THREADS"] = "1"
    _paths()
    import davidson_np
    import gasref
    from pyscf.csf_fci import csf_solver
    from pyscf.fci import direct_spin1 as shim_ds1
    i, norb, na, nb, smult, nroots, seed = p
    h1, eri = seeded_integrals(norb, 2 * norb, seed)
    sol = csf_solver(None, smult=smult)
    sol.nroots = nroots
    for k, v in SETTINGS.items():
        setattr(sol, k, v)
    stats = {}
    shim_eig = shim_ds1.FCISolver.eig

    def eig(self, op, x0=None, precond=None, **kw):
        if isinstance(op, np.ndarray):
            return shim_eig(self, op, x0, precond, **kw)
        nr = kw.get("nroots", 1)
        conv, e, ci = davidson_np.davidson1(op, x0, precond, tol=kw.get("tol", 1e-10),
                                            max_cycle=kw.get("max_cycle", 50),
                                            max_space=kw.get("max_space", 12),
                                            lindep=kw.get("lindep", 1e-14), nroots=nr, stats=stats)
        self.converged = conv
        return (e[0], ci[0]) if nr == 1 else (e, ci)

    shim_ds1.FCISolver.eig = eig
    t0 = time.time()
    e, ci = sol.kernel(h1, eri, norb, (na, nb))
    t_solve = time.time() - t0
    cis = ci if isinstance(ci, list) else [ci]
    tr = []
    for c in cis:
        dm1, dm2 = gasref.make_rdm12(c, c, norb, (na, nb))
        tr.append(float(np.trace(dm1)))
    t_all = time.time() - t0
    conv = np.atleast_1d(getattr(sol, "converged", True))
    return i, np.atleast_1d(np.asarray(e, dtype=np.float64)), bool(np.all(conv)), stats.get("niter", 0), \
        t_solve, t_all


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workers", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    probs = problems()
    from multiprocessing import get_context
    energies = np.full((len(probs), 4), np.nan)
    conv = np.zeros(len(probs), dtype=bool)
    niter = np.zeros(len(probs), dtype=np.int32)
    secs = np.zeros((len(probs), 2))
    t0 = time.time()
    with get_context("spawn").Pool(args.workers) as pool:
        for i, e, c, it, ts, ta in pool.imap_unordered(solve, sorted(probs, key=lambda p: -p[1])):
            energies[i, :len(e)] = e
            conv[i] = c
            niter[i] = it
            secs[i] = (ts, ta)
            print("%3d  norb %2d  converged %s  iterations %3d  %.1fs  E=%s" % (i, probs[i][1], c, it, ta, e),
                  flush=True)
    wall = time.time() - t0
    arr = np.array([p[:6] for p in probs], dtype=np.int32)
    path = os.path.join(HERE, "c3_batch128.npz")
    np.savez_compressed(path, problems=arr, energies=energies, converged=conv, iterations=niter,
                        seconds=secs, wall_seconds=np.array(wall), workers=np.array(args.workers),
                        settings=np.array([SETTINGS["conv_tol"], SETTINGS["max_cycle"], SETTINGS["max_space"]]))
    print("C3: %d problems, %d converged, %.0f s wall on %d workers -> %s" % (
        len(probs), int(conv.sum()), wall, args.workers, path))


if __name__ == "__main__":
    main()
