"""CSF-basis FCI (pyscf/csf_fci/__init__.py:1-12)."""
from . import csf, csfstring, csdstring, csf_symm, spin_op  # noqa: F401
from .csf import FCISolver
from .csfstring import CSFTransformer


def csf_solver(mol=None, smult=None, symm=None):
    """pyscf/csf_fci/__init__.py:6-12: the point-group-symmetric solver when
    symm (default: mol.symmetry) is true, else the plain one."""
    if mol and symm is None:
        symm = getattr(mol, 'symmetry', False)
    if symm:
        return csf_symm.FCISolver(mol, smult=smult)
    return FCISolver(mol, smult=smult)
