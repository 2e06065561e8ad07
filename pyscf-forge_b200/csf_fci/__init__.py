"""CSF-basis FCI (pyscf/csf_fci/__init__.py:1-12)."""
from . import csf, csfstring, csdstring  # noqa: F401
from .csf import FCISolver
from .csfstring import CSFTransformer


def csf_solver(mol=None, smult=None, symm=None):
    """pyscf/csf_fci/__init__.py:6-12 (point-group symmetric solvers are not
    implemented)."""
    if symm:
        raise NotImplementedError("csf_symm.FCISolver is not implemented")
    return FCISolver(mol, smult=smult)
