"""Block Davidson-Liu eigensolver with the Krylov space resident on the GPU.

Role of pyscf lib.davidson1 as called through fci.eig at
pyscf/csf_fci/csf.py:487-490: lowest ``nroots`` eigenpairs, subspace of at
most ``max_space + nroots`` vectors with restart from the Ritz vectors,
energy convergence ``tol`` and residual convergence ``sqrt(tol)`` (or
``tol_residual``), linear-dependence cut ``lindep``, roots followed by
overlap (``follow_state``).  Vectors, Gram blocks, orthogonalisation and the
preconditioner run as CUDA kernels (libcsffci_b200); only the
(max_space+nroots)^2 subspace matrix is diagonalised on the host.
"""
import numpy as np
import torch

from .. import _capi
from .._runtime import ptr, stream, workspace


def gram(x, y):
    """x (m, n), y (k, n) device -> numpy (m, k) = x y^T."""
    m, k, n = x.shape[0], y.shape[0], x.shape[1]
    out = torch.empty((m, k), dtype=torch.float64, device=x.device)
    if m and k:
        nbytes = _capi.query("csffci_gram_workspace", m, k, n)
        ws = workspace("gram", nbytes)
        _capi.call("csffci_gram", m, ptr(x), x.stride(0), k, ptr(y), y.stride(0), n, ptr(out),
                   ptr(ws), nbytes, stream())
    return out


def combine(y, x, coef, beta=0.0):
    """y[r] = beta*y[r] + sum_i coef[r, i] x[i]  (all device; coef numpy/torch)."""
    ny, nx = coef.shape
    if nx == 0:
        if beta == 0.0:
            y[:ny].zero_()
        return y
    c = torch.as_tensor(np.ascontiguousarray(coef, dtype=np.float64), device=y.device) \
        if not isinstance(coef, torch.Tensor) else coef.to(y.device, torch.float64).contiguous()
    _capi.call("csffci_combine", ny, ptr(y), y.stride(0), float(beta), nx, ptr(x), x.stride(0),
               ptr(c), x.shape[1], stream())
    return y


class DiagPrecond:
    """t = (r - e1 x) / (hdiag - (e - shift)) with e1 from Olsen's formula;
    the optional p-space block (addr, pspaceig, pspaceci) enters e1 exactly
    (the role of make_pspace_precond, reached through csf.py:433)."""

    def __init__(self, hdiag, level_shift=1e-3, pspaceig=None, pspaceci=None, addr=None):
        self.hdiag = hdiag.contiguous()
        self.shift = float(level_shift)
        self.pw = None if pspaceig is None else np.asarray(pspaceig)
        self.pv = None if pspaceci is None else np.asarray(pspaceci)
        self.addr = None if addr is None else torch.as_tensor(np.asarray(addr, dtype=np.int64),
                                                              device=hdiag.device)
        self.hd_addr = None if addr is None else self.hdiag[self.addr].cpu().numpy()

    def __call__(self, r, e, x):
        n = r.numel()
        t = torch.empty_like(r)
        nbytes = _capi.query("csffci_precond_workspace")
        ws = workspace("precond", nbytes)
        if self.pw is None:
            _capi.call("csffci_precond", n, ptr(r), ptr(x), ptr(self.hdiag), float(e), self.shift, 1,
                       0.0, ptr(t), ptr(ws), stream())
            return t
        dots = torch.empty(2, dtype=torch.float64, device=r.device)
        _capi.call("csffci_precond_dots", n, ptr(r), ptr(x), ptr(self.hdiag), float(e), self.shift,
                   ptr(dots), ptr(ws), stream())
        a, b = dots.cpu().numpy()
        es = e - self.shift
        xa = x[self.addr].cpu().numpy()
        ra = r[self.addr].cpu().numpy()
        hinv = 1.0 / (self.hd_addr - es)
        hinv[np.abs(hinv) > 1e8] = 1e8
        # replace the diagonal inverse on the p-space by the exact block
        a -= np.dot(xa * hinv, ra)
        b -= np.dot(xa * hinv, xa)
        h0e0inv = (self.pv / (self.pw - es)) @ self.pv.T
        a += xa @ (h0e0inv @ ra)
        b += xa @ (h0e0inv @ xa)
        e1 = a / b if b != 0 else 0.0
        _capi.call("csffci_precond", n, ptr(r), ptr(x), ptr(self.hdiag), float(e), self.shift, 2,
                   float(e1), ptr(t), ptr(ws), stream())
        return t


def _orthonormalise_per_vector(V, m, new, lindep):
    """Append the vectors of new to V[m:] one at a time, each orthogonalised
    (two passes) against V[:m] and the ones already appended, dropping those
    whose remaining squared norm is below lindep; returns their rows."""
    added = []
    for i in range(new.shape[0]):
        t = new[i:i + 1].clone()
        for _ in range(2):
            if m + len(added):
                cf = gram(V[:m + len(added)], t).cpu().numpy().T
                combine(t, V[:m + len(added)], -cf, beta=1.0)
        nrm2 = float(gram(t, t).cpu().numpy()[0, 0])
        if nrm2 > lindep:
            V[m + len(added)].copy_(t[0] / np.sqrt(nrm2))
            added.append(m + len(added))
    return added


def _orthonormalise_into(V, m, new, lindep):
    """The same result as _orthonormalise_per_vector for a block of new
    vectors, with the subspace read once per pass: two passes of block
    Gram-Schmidt against V[:m] (one Gram block and one combine each), then
    Gram-Schmidt among the block on its small Gram matrix (host), checked:
    if the appended block is not orthonormal to 1e-8 the per-vector form
    runs instead."""
    k = new.shape[0]
    if k == 1:
        return _orthonormalise_per_vector(V, m, new, lindep)
    T = new.clone()
    for _ in range(2):
        if m:
            cf = gram(V[:m], T).cpu().numpy()          # (m, k)
            combine(T, V[:m], -cf.T, beta=1.0)
    G = gram(T, T).cpu().numpy()
    G = 0.5 * (G + G.T)
    acc = []
    for i in range(k):
        c = np.zeros(k)
        c[i] = 1.0
        for _ in range(2):
            for a in acc:
                c = c - float(a @ G @ c) * a
        nrm2 = float(c @ G @ c)
        if nrm2 > lindep:
            acc.append(c / np.sqrt(nrm2))
    if not acc:
        return []
    C = np.array(acc)
    Q = V[m:m + len(acc)]
    combine(Q, T, C)
    Gq = gram(Q, Q).cpu().numpy()
    if np.abs(Gq - np.eye(len(acc))).max() > 1e-8:
        return _orthonormalise_per_vector(V, m, new, lindep)
    return list(range(m, m + len(acc)))


def davidson(aop, x0, precond, tol=1e-10, max_cycle=100, max_space=12, lindep=1e-14, nroots=1,
             follow_state=True, tol_residual=None, verbose=0, log=None, stats=None):
    """aop(X) maps a device (k, n) block to (k, n).  x0: device (m, n) or a
    list of device vectors.  Returns (converged list, energies numpy,
    device (nroots, n) eigenvectors); stats (a dict, optional) receives the
    number of iterations as stats["niter"]."""
    if callable(x0):
        x0 = x0()
    if isinstance(x0, (list, tuple)):
        x0 = torch.stack([v.reshape(-1) for v in x0])
    x0 = x0.reshape(-1, x0.shape[-1])
    n = x0.shape[1]
    dev = x0.device
    toloose = np.sqrt(tol) if tol_residual is None else tol_residual
    space = max_space + nroots
    V = torch.empty((space + nroots, n), dtype=torch.float64, device=dev)
    AV = torch.empty_like(V)
    X = torch.empty((nroots, n), dtype=torch.float64, device=dev)
    AX = torch.empty_like(X)
    R = torch.empty_like(X)
    h = np.zeros((space + nroots, space + nroots))
    m = 0
    e_prev = None
    x_prev = None  # host coefficients of the previous Ritz vectors in V
    conv = [False] * nroots
    e = None
    new = x0.clone()
    nrm = np.sqrt(np.maximum(np.diag(gram(new, new).cpu().numpy()), 1e-300))
    new = new / torch.as_tensor(nrm, device=dev)[:, None]
    for icyc in range(max_cycle):
        if stats is not None:
            stats["niter"] = icyc + 1
        added = _orthonormalise_into(V, m, new, lindep)
        if not added:
            break
        k0 = m
        m += len(added)
        AV[k0:m] = aop(V[k0:m])
        blk = gram(V[:m], AV[k0:m]).cpu().numpy()
        h[:m, k0:m] = blk
        h[k0:m, :m] = blk.T
        w, c = np.linalg.eigh(h[:m, :m])
        k = min(nroots, m)
        # follow roots by overlap only once some root has converged; before
        # that the lowest Ritz values are taken (a poor early guess would
        # otherwise lock a root onto a high-lying state)
        if follow_state and x_prev is not None and any(conv):
            ov = np.abs(x_prev[:, :m] @ c)
            idx = []
            for i in range(ov.shape[0]):
                order = np.argsort(-ov[i])
                j = next(j for j in order if j not in idx)
                idx.append(j)
            idx = sorted(idx, key=lambda j: w[j])[:k]
        else:
            idx = list(range(k))
        e = w[idx]
        cc = np.ascontiguousarray(c[:, idx].T)
        combine(X, V[:m], cc)
        combine(AX, AV[:m], cc)
        R[:k].copy_(AX[:k])
        combine(R, X, -np.diag(e), beta=1.0)
        rn = np.sqrt(np.maximum(np.diag(gram(R[:k], R[:k]).cpu().numpy()), 0.0))
        de = e - e_prev if (e_prev is not None and len(e_prev) == len(e)) else np.full(k, np.inf)
        conv = [bool(abs(de[i]) < tol and rn[i] < toloose) for i in range(k)]
        if log is not None:
            log("davidson %d  m=%d  e=%s  |r|=%s  de=%s" % (icyc, m, e, rn, de))
        if all(conv):
            break
        e_prev = e
        x_prev = np.zeros((k, space + nroots))
        x_prev[:, :m] = cc
        ts = []
        for i in range(k):
            if conv[i]:
                continue
            t = precond(R[i], e[i], X[i]).reshape(1, -1)
            nt = float(np.sqrt(max(gram(t, t).cpu().numpy()[0, 0], 0.0)))
            if nt > 0.0:
                ts.append(t / nt)
        new = torch.cat(ts) if ts else X[:0]
        if m + new.shape[0] > space:
            # restart from the Ritz vectors (orthonormal, h diagonal)
            V[:k].copy_(X[:k])
            AV[:k].copy_(AX[:k])
            m = k
            h[:] = 0.0
            blk = gram(V[:m], AV[:m]).cpu().numpy()
            h[:m, :m] = 0.5 * (blk + blk.T)
            x_prev = np.zeros((k, space + nroots))
            x_prev[:, :k] = np.eye(k)
    return conv, e, X[:len(e)].clone()
