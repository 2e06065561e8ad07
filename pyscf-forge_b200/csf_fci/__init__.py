"""CSF-basis FCI (pyscf/csf_fci/__init__.py:1-12)."""
from . import csf, csfstring, csdstring, csf_symm, gas, spin_op  # noqa: F401
from .csf import FCISolver
from .csfstring import CSFTransformer


def csf_solver(mol=None, smult=None, symm=None, gas_orbs=None, gas_restr=None,
               gas_restr_type=gas.GAS_RESTR_SPIN_SUPERGROUP):
    """pyscf/csf_fci/__init__.py:6-12: the point-group-symmetric solver when
    symm (default: mol.symmetry) is true, else the plain one.  gas_orbs,
    gas_restr and gas_restr_type (the arguments of the reference's GAS
    solver, pyscf/mcscf/fci_gas.py:778-801) restrict either to a GAS
    space."""
    if mol and symm is None:
        symm = getattr(mol, 'symmetry', False)
    sol = csf_symm.FCISolver(mol, smult=smult) if symm else FCISolver(mol, smult=smult)
    if gas_orbs is not None:
        sol.gas_orbs = tuple(gas_orbs)
        sol.gas_restr = gas_restr
        sol.gas_restr_type = gas_restr_type
    return sol
