"""ORACLE / TEST INFRASTRUCTURE: block Davidson-Liu eigensolver (numpy).

Restates the semantics the reference obtains from PySCF's lib.davidson1 via
``fci.eig`` (pyscf/csf_fci/csf.py:487-490): lowest ``nroots`` eigenpairs of a
symmetric operator given as a matrix-vector callable, subspace bounded by
``max_space + nroots`` with restart from the current Ritz vectors, energy
convergence ``tol`` and residual convergence ``sqrt(tol)``, linear-dependence
threshold ``lindep``, and roots followed by overlap (``follow_state``).
The preconditioners restate Davidson's diagonal correction and Olsen's
correction with an exact p-space block (J. Olsen, P. Jorgensen, J. Simons,
Chem. Phys. Lett. 169, 463 (1990)); the reference builds them through
fci.make_precond (csf.py:433).  Iteration counts are not a parity target --
converged energies and vectors are.
"""
import numpy as np


def make_diag_precond(hdiag, level_shift=1e-3):
    hdiag = np.asarray(hdiag)

    def precond(x, e, *args):
        d = hdiag - (e - level_shift)
        d[np.abs(d) < 1e-8] = 1e-8
        return x / d
    return precond


def make_pspace_precond(hdiag, pspaceig, pspaceci, addr, level_shift=1e-3):
    hdiag = np.asarray(hdiag)
    addr = np.asarray(addr)

    def precond(r, e0, x0, *args):
        h0e0inv = (pspaceci / (pspaceig - (e0 - level_shift))) @ pspaceci.T
        hinv = 1.0 / (hdiag - (e0 - level_shift))
        hinv[np.abs(hinv) > 1e8] = 1e8
        h0x0 = x0 * hinv
        h0x0[addr] = h0e0inv @ x0[addr]
        h0r = r * hinv
        h0r[addr] = h0e0inv @ r[addr]
        e1 = np.dot(x0, h0r) / np.dot(x0, h0x0)
        return (r - e1 * x0) * hinv
    return precond


def davidson(aop, x0, precond, tol=1e-10, max_cycle=100, max_space=12, lindep=1e-14,
             nroots=1, follow_state=True, verbose=False):
    if callable(x0):
        x0 = x0()
    if isinstance(x0, np.ndarray) and x0.ndim == 1:
        x0 = [x0]
    xt = [np.asarray(x, dtype=np.float64).ravel().copy() for x in x0]
    toloose = np.sqrt(tol)
    space = max_space + nroots
    V, AV = [], []
    e_prev = None
    x_prev = None
    conv = [False] * nroots
    e = x = None
    for icyc in range(max_cycle):
        new = []
        for v in xt:
            for _ in range(2):
                for b in V + new:
                    v = v - np.dot(b, v) * b
            nv = np.linalg.norm(v)
            if nv * nv > lindep:
                new.append(v / nv)
        if not new:
            break
        V += new
        AV += [np.asarray(aop(v), dtype=np.float64).ravel() for v in new]
        Vm = np.array(V)
        AVm = np.array(AV)
        h = Vm @ AVm.T
        h = 0.5 * (h + h.T)
        w, c = np.linalg.eigh(h)
        k = min(nroots, len(w))
        if follow_state and x_prev is not None and any(conv):
            ov = np.abs((np.array(x_prev) @ Vm.T) @ c)
            idx = []
            for i in range(len(x_prev)):
                order = np.argsort(-ov[i])
                j = next(j for j in order if j not in idx)
                idx.append(j)
            idx = sorted(idx, key=lambda j: w[j])[:k]
        else:
            idx = list(range(k))
        e = w[idx]
        cc = c[:, idx]
        x = cc.T @ Vm
        ax = cc.T @ AVm
        r = ax - e[:, None] * x
        rn = np.linalg.norm(r, axis=1)
        de = e - e_prev if e_prev is not None and len(e_prev) == len(e) else np.full(len(e), np.inf)
        conv = [bool(abs(de[i]) < tol and rn[i] < toloose) for i in range(len(e))]
        if verbose:
            print(icyc, e, rn, de)
        if all(conv):
            break
        e_prev = e
        x_prev = list(x)
        xt = []
        for i in range(len(e)):
            if conv[i]:
                continue
            t = precond(r[i], e[i], x[i])
            nt = np.linalg.norm(t)
            if nt > 0:
                xt.append(t / nt)
        if len(V) + len(xt) > space:
            V = list(x)
            AV = list(ax)
            # re-orthonormalise the restart basis
            Q, R = np.linalg.qr(np.array(V).T)
            V = list(Q.T)
            AV = list((np.array(AV).T @ np.linalg.inv(R)).T)
    return conv, e, list(x)
