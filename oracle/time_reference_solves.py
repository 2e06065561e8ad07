"""ORACLE / TEST INFRASTRUCTURE: time the reference's own CPU solves.

Runs the reference's unmodified pyscf/csf_fci/csf.py kernel (read from the
reference checkout, so only the build container can run it) on the PySCF
stand-in under oracle/shim -- transforms by the reference's csfstring.py,
sigma and RDMs by the reference's C (oracle/_ref/libfci_gas.so, OpenMP on
all cores), Davidson by the restatement of lib.davidson1 -- followed by
make_rdm12 of every root, for the single-problem configurations:

  C0  norb 8  (4,4) singlet, 1 root, rank-16 integrals
  C1  norb 12 (6,6) singlet, 3 roots, rank 24
  C2  norb 14 (7,7) triplet, 2 roots, rank 28

Solver settings: conv_tol 1e-10, max_cycle 400, max_space 30 (the seeded
integrals are weakly diagonally dominant; see tests/golden/make_c3_golden.py).
Prints one JSON line per configuration: seconds, solves+RDMs per second,
energies, threads.  Its output of the three configurations (8 threads in
the build container) is committed as tests/golden/ref_solves_c0_c2.jsonl,
which bench.py reads for the reference energies and CPU times it reports
beside the GPU solves:

    python oracle/time_reference_solves.py C0 C1 C2 > tests/golden/ref_solves_c0_c2.jsonl
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [HERE, os.path.join(HERE, "shim")]

CONFIGS = {"C0": (8, (4, 4), 1, 1, 16), "C1": (12, (6, 6), 1, 3, 24), "C2": (14, (7, 7), 3, 2, 28)}
SETTINGS = dict(conv_tol=1e-10, max_cycle=400, max_space=30)


def seeded_integrals(norb, rank, seed=0):
    rng = np.random.default_rng(seed)
    h1 = rng.normal(0.0, 0.3, (norb, norb))
    h1 = 0.5 * (h1 + h1.T)
    np.fill_diagonal(h1, np.linspace(-2.0, 0.5, norb))
    L = rng.normal(0.0, 0.2, (rank, norb * norb)).reshape(rank, norb, norb)
    L = 0.5 * (L + L.transpose(0, 2, 1))
    return h1, 0.5 * np.einsum("xpq,xrs->pqrs", L, L)


def run(tag):
    import davidson_np
    import gasref
    from pyscf.csf_fci import csf_solver
    from pyscf.fci import direct_spin1 as shim_ds1
    norb, nelec, smult, nroots, rank = CONFIGS[tag]
    h1, eri = seeded_integrals(norb, rank)
    shim_eig = shim_ds1.FCISolver.eig
    stats = {}

    def eig(self, op, x0=None, precond=None, **kw):
        if isinstance(op, np.ndarray):
            return shim_eig(self, op, x0, precond, **kw)
        nr = kw.get("nroots", 1)
        conv, e, ci = davidson_np.davidson1(op, x0, precond, tol=kw.get("tol", 1e-10),
                                            max_cycle=kw.get("max_cycle", 50), max_space=kw.get("max_space", 12),
                                            lindep=kw.get("lindep", 1e-14), nroots=nr, stats=stats)
        self.converged = conv
        return (e[0], ci[0]) if nr == 1 else (e, ci)

    shim_ds1.FCISolver.eig = eig
    sol = csf_solver(None, smult=smult)
    sol.nroots = nroots
    for k, v in SETTINGS.items():
        setattr(sol, k, v)
    t0 = time.perf_counter()
    e, ci = sol.kernel(h1, eri, norb, nelec)
    t1 = time.perf_counter()
    cis = ci if isinstance(ci, list) else [ci]
    for c in cis:
        gasref.make_rdm12(c, c, norb, nelec)
    t2 = time.perf_counter()
    return {"config": tag, "norb": norb, "nelec": list(nelec), "smult": smult, "nroots": nroots,
            "energies": [float(x) for x in np.atleast_1d(e)],
            "converged": [bool(x) for x in np.atleast_1d(getattr(sol, "converged", True))],
            "iterations": stats.get("niter"), "solve_s": t1 - t0, "rdm_s": t2 - t1,
            "solves_rdms_per_s": 1.0 / (t2 - t0), "threads": int(os.environ.get("OMP_NUM_THREADS", "0")),
            "cores": len(os.sched_getaffinity(0))}


if __name__ == "__main__":
    os.environ.setdefault("OMP_NUM_THREADS", str(len(os.sched_getaffinity(0))))
    for tag in (sys.argv[1:] or ["C0", "C1", "C2"]):
        print(json.dumps(run(tag)), flush=True)
