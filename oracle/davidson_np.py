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


def davidson1(aop, x0, precond, tol=1e-10, max_cycle=50, max_space=12, lindep=1e-14, nroots=1,
              follow_state=True, tol_residual=None, verbose=False, stats=None):
    """Restatement of the iteration of PySCF's lib.davidson1 (the solver
    fci.eig hands the reference's CSF problem to, pyscf/csf_fci/csf.py:487-490)
    as its published code behaves, for the symmetric case with the subspace in
    core:

      * the subspace limit is max_space + 4 (nroots - 1);
      * every iteration takes the LOWEST nroots Ritz pairs; the previous
        energies are re-ordered to the current roots by the largest overlap
        of the old Ritz vectors with the new ones before the energy change
        is formed (states may swap order between iterations);
      * a root is converged when |dE| < tol and |r| < tol_residual
        (sqrt(tol) by default); only unconverged roots get a correction,
        preconditioned at the LOWEST Ritz value e[0] for every root;
      * corrections are orthogonalised against the subspace (two passes) and
        among themselves, normalised, and dropped below lindep;
      * when the subspace would overflow, the next iteration restarts from
        the current Ritz vectors alone (their images are recomputed), and
        the corrections of that iteration are discarded;
      * with follow_state, a residual that jumps by more than a factor 3
        above 1 restores the previous Ritz vectors and restarts.
    Returns (converged, energies, vectors); stats (a dict, optional)
    receives the iteration count as stats["niter"]."""
    if callable(x0):
        x0 = x0()
    if isinstance(x0, np.ndarray) and x0.ndim == 1:
        x0 = [x0]
    x0 = [np.asarray(x, dtype=np.float64).ravel().copy() for x in x0]
    toloose = np.sqrt(tol) if tol_residual is None else tol_residual
    max_space = max_space + (nroots - 1) * 4
    fresh_start = True
    e = v = None
    conv = np.zeros(nroots, dtype=bool)
    xs, ax = [], []
    xt = None
    max_dx_last = 1e9

    def orthonormal(vecs, basis):
        out = []
        for x in vecs:
            x = x.copy()
            for _ in range(2):
                for b in basis + out:
                    x -= np.dot(b, x) * b
            nx = np.linalg.norm(x)
            if nx * nx > lindep:
                out.append(x / nx)
        return out

    niter = 0
    for icyc in range(max_cycle):
        niter = icyc + 1
        if fresh_start:
            xs, ax = [], []
            xt = orthonormal(x0, [])
            max_dx_last = 1e9
            if not xt:
                break
        axt = [np.asarray(aop(x), dtype=np.float64).ravel() for x in xt]
        xs += xt
        ax += axt
        space = len(xs)
        elast, vlast, conv_last = e, v, conv
        X = np.array(xs)
        h = X @ np.array(ax).T
        h = 0.5 * (h + h.T)
        w, vv = np.linalg.eigh(h)
        k = min(nroots, space)
        e = w[:k]
        v = vv[:, :k]
        conv = np.zeros(k, dtype=bool)
        if elast is not None and not fresh_start:
            head = vlast.shape[0]
            ov = np.abs(v[:head].T @ vlast)
            idx = np.argmax(ov, axis=1)
            elast = np.array([elast[i] for i in idx])
            conv_last = np.array([conv_last[i] for i in idx])
        if elast is None or len(elast) != len(e):
            de = e.copy()
        else:
            de = e - elast
        x0 = list(v.T @ X)
        ax0 = v.T @ np.array(ax)
        dx = np.zeros(k)
        res = [None] * k
        for i in range(k):
            res[i] = ax0[i] - e[i] * x0[i]
            dx[i] = np.linalg.norm(res[i])
            conv[i] = abs(de[i]) < tol and dx[i] < toloose
        if verbose:
            print(icyc, space, e, dx, de)
        if conv.all():
            break
        if follow_state and dx.max() > 1 and dx.max() / max_dx_last > 3 and space > nroots + 2:
            x0 = list(vlast.T @ X[:vlast.shape[0]])
            fresh_start = True
            continue
        corr = []
        for i in range(k):
            if not conv[i] and dx[i] ** 2 > lindep:
                t = precond(res[i], e[0], x0[i])
                corr.append(t / np.linalg.norm(t))
        xt = orthonormal(corr, xs)
        if not xt:
            conv = dx < toloose
            break
        max_dx_last = dx.max()
        fresh_start = space + nroots > max_space
    if stats is not None:
        stats["niter"] = niter
    return [bool(c) for c in conv], e, x0
