"""Point-group pieces of pyscf.fci.direct_spin1_symm that the reference's
csf_symm/csfstring call (test infrastructure for the oracle; restated from
their documented behaviour, D2h and subgroups only, irrep ids whose direct
product is XOR)."""
import numpy as np

from pyscf.fci import direct_spin1


def _gen_strs_irrep(strs, orbsym):
    """Irrep of each occupation string: XOR of the irreps of its occupied
    orbitals."""
    orbsym = np.asarray(orbsym, dtype=np.int64) % 10
    strs = np.asarray(strs, dtype=np.int64)
    out = np.zeros(strs.shape, dtype=np.int64)
    for p, s in enumerate(orbsym.tolist()):
        out ^= ((strs >> p) & 1) * int(s)
    return out


def _id_wfnsym(cisolver, norb, nelec, orbsym, wfnsym):
    """With no wfnsym: the irrep of the aufbau occupation (XOR of orbitals
    nelecb..neleca-1); ids modulo 10."""
    if wfnsym is None:
        neleca, nelecb = direct_spin1._unpack_nelec(nelec)
        wfnsym = 0
        for i in np.asarray(orbsym)[nelecb:neleca]:
            wfnsym ^= int(i) % 10
    elif isinstance(wfnsym, str):
        raise NotImplementedError("irrep labels need pyscf.symm")
    return int(wfnsym) % 10


class FCISolver(direct_spin1.FCISolver):
    orbsym = None
    wfnsym = None

    def guess_wfnsym(self, norb, nelec, fcivec=None, orbsym=None, wfnsym=None, **kwargs):
        if orbsym is None:
            orbsym = self.orbsym
        if fcivec is None:
            return _id_wfnsym(self, norb, nelec, orbsym, wfnsym)
        raise NotImplementedError("wfnsym from a CI vector is not part of the stand-in")
