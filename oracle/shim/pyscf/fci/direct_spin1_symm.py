"""import-only stub (point-group symmetry is outside the stand-in)."""
from pyscf.fci import direct_spin1


def _gen_strs_irrep(strs, orbsym):
    raise NotImplementedError("point-group symmetry is not part of the stand-in")


class FCISolver(direct_spin1.FCISolver):
    pass


def _id_wfnsym(*a, **k):
    raise NotImplementedError
