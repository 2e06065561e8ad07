"""ORACLE / TEST INFRASTRUCTURE: the names pyscf/mcscf/addons_gas.py imports
from PySCF-core ``pyscf.mcscf.addons`` (base classes of its state-average
wrappers and ``sort_mo``).  Only the restriction helpers of addons_gas and
the GAS solver of fci_gas are exercised through the stand-in; the wrappers
are never instantiated here."""


class StateAverageFCISolver:
    pass


class StateAverageMCSCFSolver:
    pass


def sort_mo(*args, **kwargs):
    raise NotImplementedError("sort_mo is not part of the stand-in")
