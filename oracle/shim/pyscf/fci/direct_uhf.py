import numpy as np
from pyscf.lib import restate


def make_hdiag(h1e, eri, norb, nelec):
    h1 = np.asarray([np.asarray(h1e[0]), np.asarray(h1e[1])])
    return restate.make_hdiag(h1, eri[0], norb, nelec)


def contract_1e(f1e, fcivec, norb, nelec, link_index=None):
    return restate.contract_1e_ab(np.asarray(f1e[0]), np.asarray(f1e[1]), fcivec, norb, nelec)
