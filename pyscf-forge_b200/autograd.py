"""Differentiable CSF-FCI energies.

``csf_fci_energy(h1, eri, norb, nelec, smult, nroots)`` returns the lowest
``nroots`` eigenvalues of H(h1, eri) in the spin-``smult`` CSF space as a
torch tensor that carries gradients to ``h1`` and ``eri``.  The backward is
the adjoint of sigma: by Hellmann-Feynman, for an eigenpair (E_k, c_k),

    dE_k/dh1[p,q]      = <c_k|E_pq|c_k>                = dm1_k[q,p]
    dE_k/deri[p,q,r,s] = 1/2 <c_k|E_pq E_rs - d_qr E_ps|c_k> = 1/2 dm2_k[p,q,r,s]

so the backward runs the RDM kernel (csffci_rdm12, the transition-density
contraction that is the transpose of the sigma gather/scatter) on the
solved vectors, processing the determinant space in slabs instead of
storing D(pq, J).  A state average is ``(w * E).sum()``; its gradient is the
w-weighted sum of the per-root RDMs.  ``eri`` is the full (n,n,n,n)
tensor; its gradient is returned in the same layout.  No counterpart in the
reference (whose CASSCF obtains the same RDMs through make_rdm12).
"""
import numpy as np
import torch

from .csf_fci.csf import FCISolver
from .fci import direct_spin1


class _CSFEnergy(torch.autograd.Function):

    @staticmethod
    def forward(ctx, h1, eri, norb, nelec, smult, nroots, solver, ci0):
        sol = solver if solver is not None else FCISolver(None, smult=smult)
        sol.smult = smult
        sol.nroots = nroots
        h1d = h1.detach().to("cuda", torch.float64)
        erid = eri.detach().to("cuda", torch.float64)
        e, ci = sol.kernel(h1d, erid, norb, nelec, ci0=ci0)
        cis = ci if isinstance(ci, list) else [ci]
        e = np.atleast_1d(np.asarray(e, dtype=np.float64))
        ctx.norb = norb
        ctx.nelec = direct_spin1._unpack_nelec(nelec)
        ctx.cis = [c.reshape(-1) for c in cis]
        ctx.h1_shape, ctx.eri_shape = h1.shape, eri.shape
        ctx.h1_device, ctx.eri_device = h1.device, eri.device
        ctx.solver = sol
        return torch.as_tensor(e, dtype=torch.float64, device=h1.device)

    @staticmethod
    def backward(ctx, g):
        n = ctx.norb
        g = g.detach().to("cpu", torch.float64).numpy().reshape(-1)
        gh1 = torch.zeros((n, n), dtype=torch.float64, device="cuda")
        geri = torch.zeros((n, n, n, n), dtype=torch.float64, device="cuda")
        for k, c in enumerate(ctx.cis):
            if g[k] == 0.0:
                continue
            dm1, dm2 = direct_spin1.dev_rdm12(c, None, n, ctx.nelec)
            gh1 += g[k] * dm1.T
            geri += (0.5 * g[k]) * dm2
        return (gh1.reshape(ctx.h1_shape).to(ctx.h1_device), geri.reshape(ctx.eri_shape).to(ctx.eri_device),
                None, None, None, None, None, None)


def csf_fci_energy(h1, eri, norb, nelec, smult=1, nroots=1, solver=None, ci0=None):
    """Differentiable energies (tensor of length nroots); see the module
    docstring.  ``solver`` may be a configured FCISolver (conv_tol, ...)."""
    if not isinstance(h1, torch.Tensor):
        h1 = torch.as_tensor(np.asarray(h1, dtype=np.float64))
    if not isinstance(eri, torch.Tensor):
        eri = torch.as_tensor(np.asarray(eri, dtype=np.float64))
    if eri.numel() != norb ** 4:
        raise ValueError("eri must be the full (norb,norb,norb,norb) tensor for differentiation")
    return _CSFEnergy.apply(h1, eri, norb, nelec, smult, nroots, solver, ci0)


def state_average_rdm12(ci_list, weights, norb, nelec):
    """Weighted 1- and 2-RDMs of several det-basis vectors (device)."""
    nelec = direct_spin1._unpack_nelec(nelec)
    dm1 = dm2 = None
    for w, c in zip(weights, ci_list):
        c = c if isinstance(c, torch.Tensor) else torch.as_tensor(np.asarray(c), device="cuda")
        d1, d2 = direct_spin1.dev_rdm12(c.reshape(-1).to("cuda", torch.float64), None, norb, nelec)
        dm1 = w * d1 if dm1 is None else dm1 + w * d1
        dm2 = w * d2 if dm2 is None else dm2 + w * d2
    return dm1, dm2
