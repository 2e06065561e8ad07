"""B200-native CSF-basis FCI engine with the API of pyscf.csf_fci.

    from pyscf_forge_b200 import csf_solver
    sol = csf_solver(None, smult=1)
    e, ci = sol.kernel(h1e, eri, norb, (na, nb))
    dm1, dm2 = sol.make_rdm12(ci, norb, (na, nb))

All compute runs in libcsffci_b200.so (hand-written sm_100a CUDA); there is
no CPU fallback.
"""
from . import _capi  # noqa: F401
from .csf_fci import csf_solver, FCISolver, CSFTransformer  # noqa: F401

__all__ = ["csf_solver", "FCISolver", "CSFTransformer"]
