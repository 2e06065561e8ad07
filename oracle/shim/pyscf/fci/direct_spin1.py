"""Stand-in for the direct_spin1 entry points the reference csf_fci uses.

contract_2e -> the reference's GAS C sigma (oracle/gasref.py); absorb_h1e,
link tables, init guess, preconditioner and Davidson -> oracle/restate.py
and oracle/davidson_np.py.
"""
import numpy as np
import scipy.linalg
from pyscf.lib import restate, gasref
from pyscf import lib


def _unpack_nelec(nelec, spin=None):
    if isinstance(nelec, (int, np.integer)):
        if spin is None:
            spin = nelec % 2
        na = (nelec + spin) // 2
        return na, nelec - na
    return int(nelec[0]), int(nelec[1])


def _unpack(norb, nelec, link_index, spin=None):
    if link_index is None:
        na, nb = _unpack_nelec(nelec, spin)
        return restate.link_table(norb, na), restate.link_table(norb, nb)
    return link_index


def _get_init_guess(na, nb, nroots, hdiag, nelec):
    hdiag = np.asarray(hdiag).ravel()
    addrs = np.argsort(hdiag, kind="stable")[:nroots]
    ci0 = []
    for a in addrs:
        x = np.zeros(na * nb)
        x[a] = 1.0
        ci0.append(x)  # flat vectors, as PySCF returns them
    return ci0


def kernel_ms1(*a, **k):
    raise NotImplementedError


def absorb_h1e(h1e, eri, norb, nelec, fac=1):
    return restate.absorb_h1e(h1e, eri, norb, nelec, fac)


def contract_2e(eri, fcivec, norb, nelec, link_index=None):
    nelec = _unpack_nelec(nelec)
    return gasref.contract_2e(np.asarray(eri), np.asarray(fcivec), norb, nelec)


def make_pspace_precond(hdiag, pspaceig, pspaceci, addr, level_shift=0):
    import davidson_np
    return davidson_np.make_pspace_precond(hdiag, pspaceig, pspaceci, addr, level_shift)


class FCISolver(lib.StreamObject):
    _keys = {"max_memory", "nroots", "davidson_only", "conv_tol", "conv_tol_residual", "lindep",
             "max_cycle", "max_space", "level_shift", "pspace_size", "spin", "verbose", "mol"}
    max_memory = 64000
    nroots = 1
    davidson_only = False
    conv_tol = 1e-10
    conv_tol_residual = None
    lindep = 1e-14
    max_cycle = 100
    max_space = 12
    level_shift = 1e-3
    pspace_size = 400
    spin = None
    verbose = 0

    def __init__(self, mol=None):
        self.mol = mol

    def check_sanity(self):
        return self

    def absorb_h1e(self, h1e, eri, norb, nelec, fac=1):
        return absorb_h1e(h1e, eri, norb, nelec, fac)

    def contract_2e(self, eri, fcivec, norb, nelec, link_index=None, **kw):
        return contract_2e(eri, fcivec, norb, nelec, link_index)

    def make_precond(self, hdiag, pspaceig=None, pspaceci=None, addr=None):
        import davidson_np
        if pspaceig is None:
            return davidson_np.make_diag_precond(hdiag, self.level_shift)
        return davidson_np.make_pspace_precond(hdiag, pspaceig, pspaceci, addr, self.level_shift)

    def eig(self, op, x0=None, precond=None, **kw):
        if isinstance(op, np.ndarray):
            self.converged = True
            return scipy.linalg.eigh(op)
        import davidson_np
        nroots = kw.get("nroots", 1)
        conv, e, ci = davidson_np.davidson(op, x0, precond, tol=kw.get("tol", 1e-10),
                                           max_cycle=kw.get("max_cycle", 100),
                                           max_space=kw.get("max_space", 12),
                                           lindep=kw.get("lindep", 1e-14), nroots=nroots)
        self.converged = conv
        if nroots == 1:
            return e[0], ci[0]
        return e, ci

    def make_rdm12(self, civec, norb, nelec, link_index=None, reorder=True):
        return gasref.make_rdm12(civec, civec, norb, _unpack_nelec(nelec))


def _not_in_stand_in(name):
    def fn(*a, **k):
        raise NotImplementedError("direct_spin1.%s is not part of the stand-in" % name)
    fn.__name__ = name
    fn.__doc__ = "direct_spin1.%s (not part of the stand-in)" % name
    return fn


# names the reference's GAS solver (pyscf/mcscf/fci_gas.py) refers to; its
# GAS kernels replace them, so the stand-in only has to provide the names
for _n in ("make_rdm1", "make_rdm1s", "make_rdm12", "make_rdm12s",
           "trans_rdm1", "trans_rdm1s", "trans_rdm12", "trans_rdm12s"):
    globals()[_n] = _not_in_stand_in(_n)
