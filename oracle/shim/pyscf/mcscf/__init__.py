"""ORACLE / TEST INFRASTRUCTURE: stand-in package for pyscf.mcscf.  The
reference's own GAS modules (pyscf/mcscf/{addons_gas,fci_gas,_gaslib}.py)
are found through a second path entry pointing at the reference checkout;
``addons`` below stands in for the PySCF-core module they import."""
import os as _os
__path__.append(_os.path.join(_os.environ.get("CSF_REF_ROOT", "/root/reference"), "pyscf", "mcscf"))
