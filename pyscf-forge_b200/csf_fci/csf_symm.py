"""Point-group-symmetric CSF-basis FCI solver on the GPU with the API of
pyscf.csf_fci.csf_symm.FCISolver (pyscf/csf_fci/csf_symm.py:25-107).

The Davidson iteration runs in the packed space of the CSFs whose electron
configuration has the irrep ``wfnsym``: the det <-> CSF transforms form only
those configurations (csffci_block_t.conf_sel), so the vectors, the
preconditioner and the p-space all live in that subspace, while sigma runs
on the determinant vector as before.  Irreps follow the PySCF convention for
D2h and its subgroups (integer ids whose direct product is XOR).
"""
import numpy as np
import torch

from .._runtime import to_dev
from ..fci.direct_spin1 import _unpack_nelec
from . import csf as _csf
from .csfstring import CSFTransformer, gen_strs_irrep

# PySCF irrep ids of D2h and its subgroups (ids are the XOR-product labels)
IRREP_IDS = {
    'D2h': {'Ag': 0, 'B1g': 1, 'B2g': 2, 'B3g': 3, 'Au': 4, 'B1u': 5, 'B2u': 6, 'B3u': 7},
    'C2v': {'A1': 0, 'A2': 1, 'B1': 2, 'B2': 3},
    'C2h': {'Ag': 0, 'Bg': 1, 'Au': 2, 'Bu': 3},
    'D2': {'A': 0, 'B1': 1, 'B2': 2, 'B3': 3},
    'Cs': {"A'": 0, 'A"': 1},
    'C2': {'A': 0, 'B': 1},
    'Ci': {'Ag': 0, 'Au': 1},
    'C1': {'A': 0},
}


def irrep_name2id(groupname, name):
    """Irrep label -> PySCF irrep id for D2h and its subgroups (the role of
    pyscf.symm.irrep_name2id as called by direct_spin1_symm._id_wfnsym)."""
    table = IRREP_IDS.get(groupname)
    if table is None or name not in table:
        raise KeyError('irrep %r of point group %r' % (name, groupname))
    return table[name]


def _id_wfnsym(solver, norb, nelec, orbsym, wfnsym):
    """direct_spin1_symm._id_wfnsym semantics: with no wfnsym the irrep of
    the aufbau occupation (the XOR of the singly occupied orbitals' irreps,
    orbitals nelecb..neleca-1); a label is converted to its id; ids are
    taken modulo 10 (the D2h parent irrep)."""
    if wfnsym is None:
        neleca, nelecb = _unpack_nelec(nelec)
        wfnsym = 0
        for i in np.asarray(orbsym)[nelecb:neleca]:
            wfnsym ^= int(i) % 10
    elif isinstance(wfnsym, str):
        groupname = getattr(getattr(solver, 'mol', None), 'groupname', None)
        wfnsym = irrep_name2id(groupname, wfnsym)
    return int(wfnsym) % 10


def guess_wfnsym_from_ci(fcivec, norb, nelec, orbsym):
    """Irrep of a determinant-basis CI vector: that of its largest
    coefficient (the role of fci.addons.guess_wfnsym)."""
    from math import comb
    from .. import _capi
    from .._runtime import ptr, stream
    neleca, nelecb = _unpack_nelec(nelec)
    c = to_dev(fcivec[0] if isinstance(fcivec, (list, tuple)) else fcivec).reshape(-1)
    imax = int(torch.argmax(c.abs()).item())
    nb = comb(norb, nelecb)
    ia, ib = divmod(imax, nb)
    strs = []
    for ne, i in ((neleca, ia), (nelecb, ib)):
        s = torch.empty(comb(norb, ne), dtype=torch.int64, device=c.device)
        _capi.call("csffci_gen_strings", norb, ne, ptr(s), stream())
        strs.append(s[i:i + 1])
    sa = gen_strs_irrep(strs[0], orbsym)
    sb = gen_strs_irrep(strs[1], orbsym)
    return int((sa ^ sb).item())


class FCISolver(_csf.FCISolver):
    """csf_symm.py:25-107: CSF-basis Davidson restricted to one irrep;
    ``ci`` and ``ci0`` in the determinant basis."""

    def __init__(self, mol=None, smult=None, orbsym=None, wfnsym=None):
        super().__init__(mol, smult=smult)
        self.orbsym = orbsym if orbsym is not None else getattr(mol, 'orbsym', None)
        self.wfnsym = wfnsym

    def guess_wfnsym(self, norb, nelec, fcivec=None, orbsym=None, wfnsym=None, **kwargs):
        if orbsym is None:
            orbsym = self.orbsym
        if fcivec is None or wfnsym is not None:
            return _id_wfnsym(self, norb, nelec, orbsym, wfnsym)
        return guess_wfnsym_from_ci(fcivec, norb, nelec, orbsym)

    def kernel(self, h1e, eri, norb, nelec, ci0=None, **kwargs):
        """csf_symm.py:36-88."""
        kwargs.pop('max_memory', None)
        if 'nroots' not in kwargs:
            kwargs['nroots'] = self.nroots
        orbsym_back, wfnsym_back = self.orbsym, self.wfnsym
        orbsym = kwargs.pop('orbsym', self.orbsym)
        if orbsym is None:
            raise ValueError('orbsym is required by the point-group-symmetric solver')
        wfnsym_in = kwargs.pop('wfnsym', self.wfnsym)
        self.norb = norb
        self.nelec = nelec
        if 'smult' in kwargs:
            self.smult = kwargs.pop('smult')
        self.orbsym = orbsym
        wfnsym = self.guess_wfnsym(norb, nelec, ci0, orbsym=orbsym, wfnsym=wfnsym_in)
        self.wfnsym = wfnsym
        self.check_transformer_cache()
        if self.transformer.wfnsym > 9:
            raise NotImplementedError('High-momentum point groups in Dooh/Coov')
        idx_sym = self.transformer.idx_sym
        e, c = _csf.kernel(self, h1e, eri, norb, nelec, smult=self.smult, idx_sym=idx_sym, ci0=ci0,
                           transformer=self.transformer, **kwargs)
        if not isinstance(h1e, torch.Tensor):
            c = [ci.cpu().numpy() for ci in c] if isinstance(c, list) else c.cpu().numpy()
        self.eci, self.ci = e, c
        self.orbsym, self.wfnsym = orbsym_back, wfnsym_back
        return e, c

    def get_init_guess(self, norb, nelec, nroots, hdiag_csf, **kwargs):
        """csf_symm.py:90-100."""
        self.orbsym = kwargs.get('orbsym', self.orbsym)
        self.wfnsym = kwargs.get('wfnsym', self.wfnsym)
        assert self.orbsym is not None and self.wfnsym is not None
        self.norb = norb
        self.nelec = nelec
        self.check_transformer_cache()
        x = _csf.get_init_guess(norb, nelec, nroots, hdiag_csf, self.transformer)
        return self.transformer.dev_csf2det(x)

    def check_transformer_cache(self):
        """csf_symm.py:102-115."""
        assert isinstance(self.smult, (int, np.integer))
        neleca, nelecb = _unpack_nelec(self.nelec)
        wfnsym = self.wfnsym
        if isinstance(wfnsym, str):
            wfnsym = irrep_name2id(getattr(self.mol, 'groupname', None), wfnsym)
        if self.transformer is None:
            self.transformer = CSFTransformer(self.norb, neleca, nelecb, self.smult, orbsym=self.orbsym,
                                              wfnsym=wfnsym, max_memory=self.max_memory)
        else:
            self.transformer.gas = None
            self.transformer._update_spin_cache(self.norb, neleca, nelecb, self.smult)
            self.transformer._update_symm_cache(self.orbsym)
            self.transformer.wfnsym = wfnsym
        self._apply_gas()
