"""ORACLE / TEST INFRASTRUCTURE -- never imported by the product path.

ctypes access to the reference's own CPU code built by ``oracle/Makefile``
into ``oracle/_ref/``:

* ``libfci_gas.so`` (pyscf/lib/mcscf/fci_*_gas.c): with a single GAS
  subspace this is a full-CAS determinant FCI whose sigma, diagonal and RDMs
  the reference's own tests pin to PySCF ``direct_spin1``
  (pyscf/mcscf/test/test_gasci.py:272-293, 765-786).
* ``libcsf.so`` (pyscf/lib/csf/csfstring.c): Clebsch-Gordan spin
  eigenvectors, genealogical addressing and the within-configuration H blocks
  used by ``make_hdiag_csf``.

Only tests, ``__graft_entry__.smoke`` and the CPU-baseline arm of ``bench.py``
use this module, always as the checker or the timed CPU reference.

The ctypes structure below restates the layout of ``gas_space_t`` declared
in pyscf/lib/mcscf/fci_gas.h:123-152 (the layout has to be identical for the
calls to work; the fields are only passed through, never interpreted here
except ``ndet``).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


class _Row(ctypes.Structure):
    _fields_ = [("off", ctypes.c_uint32), ("n", ctypes.c_uint32)]


class _Space(ctypes.Structure):
    # fci_gas.h:123-152 (168 bytes, checked by a _Static_assert there)
    _fields_ = [
        ("ngas", ctypes.c_int), ("norb_tot", ctypes.c_int),
        ("norb", ctypes.c_void_p), ("start", ctypes.c_void_p),
        ("na", ctypes.c_int), ("nb", ctypes.c_int),
        ("ndet", ctypes.c_uint32), ("nsector", ctypes.c_uint16),
        ("sector_padding", ctypes.c_uint16),
        ("sector_nstr", ctypes.c_void_p), ("sector_occ", ctypes.c_void_p),
        ("sector_stride", ctypes.c_void_p),
        ("nblock", ctypes.c_uint32), ("block", ctypes.c_void_p),
        ("D", ctypes.c_void_p * 4),
        ("ntable", ctypes.c_uint32), ("link_format", ctypes.c_uint8),
        ("link_format_padding", ctypes.c_uint8 * 3),
        ("table", ctypes.c_void_p),
        ("T", ctypes.c_void_p * 2), ("R", ctypes.c_void_p * 3),
    ]


assert ctypes.sizeof(_Space) == 168


class _LinkTable(ctypes.Structure):
    # fci_gas.h:113-119
    _fields_ = [("link", ctypes.c_void_p), ("active_op", ctypes.c_void_p),
                ("nsrc", ctypes.c_uint32), ("nlink", ctypes.c_uint32),
                ("nop", ctypes.c_uint16)]


assert ctypes.sizeof(_LinkTable) == 32

_dp = ctypes.POINTER(ctypes.c_double)
_LIB_GAS = None
_LIB_CSF = None


def available():
    return (os.path.exists(os.path.join(REF_DIR, "libfci_gas.so"))
            and os.path.exists(os.path.join(REF_DIR, "libcsf.so")))


def lib_gas():
    global _LIB_GAS
    if _LIB_GAS is None:
        lib = ctypes.CDLL(os.path.join(REF_DIR, "libfci_gas.so"))
        sp = ctypes.POINTER(_Space)
        ip = ctypes.POINTER(ctypes.c_int)
        lib.gas_space_from_blocks.argtypes = [sp, ctypes.c_int, ip, ctypes.c_int,
                                              ctypes.c_int, ctypes.c_int, ip]
        lib.gas_space_from_blocks.restype = ctypes.c_int
        lib.gas_space_compress_links.argtypes = [sp]
        lib.gas_space_compress_links.restype = ctypes.c_int
        lib.gas_space_free.argtypes = [sp]
        lib.gas_space_free.restype = None
        lib.fci_make_hdiag_gas.argtypes = [sp, _dp, _dp, _dp]
        lib.fci_make_hdiag_gas.restype = ctypes.c_int
        lib.fci_contract_gas_plan_create.argtypes = [ctypes.POINTER(ctypes.c_void_p),
                                                     sp, _dp, _dp]
        lib.fci_contract_gas_plan_create.restype = ctypes.c_int
        lib.fci_contract_gas_plan_execute.argtypes = [ctypes.c_void_p, _dp, _dp]
        lib.fci_contract_gas_plan_execute.restype = ctypes.c_int
        lib.fci_contract_gas_plan_free.argtypes = [ctypes.c_void_p]
        lib.fci_rdm_gas_plan_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), sp]
        lib.fci_rdm_gas_plan_create.restype = ctypes.c_int
        lib.fci_rdm_gas_plan_make_rdm12s.argtypes = [ctypes.c_void_p] + [_dp] * 7
        lib.fci_rdm_gas_plan_make_rdm12s.restype = ctypes.c_int
        lib.fci_rdm_gas_plan_free.argtypes = [ctypes.c_void_p]
        _LIB_GAS = lib
    return _LIB_GAS


def lib_csf():
    global _LIB_CSF
    if _LIB_CSF is None:
        _LIB_CSF = ctypes.CDLL(os.path.join(REF_DIR, "libcsf.so"))
    return _LIB_CSF


def _ptr(a):
    return a.ctypes.data_as(_dp)


def _check(status, name):
    if status != 0:
        raise RuntimeError("%s failed with status %d" % (name, status))


class CASSpace:
    """One-subspace GAS space == full CAS(norb; na, nb) in colex det order.

    Mirrors pyscf/mcscf/fci_gas.py:421-456 (GasSpace with a single block).
    """

    def __init__(self, norb, nelec, compress=False):
        self.lib = lib_gas()
        self.norb = int(norb)
        self.na, self.nb = int(nelec[0]), int(nelec[1])
        self._s = _Space()
        norb_arr = (ctypes.c_int * 1)(self.norb)
        occ = (ctypes.c_int * 2)(self.na, self.nb)
        _check(self.lib.gas_space_from_blocks(ctypes.byref(self._s), 1, norb_arr,
                                              self.na, self.nb, 1, occ),
               "gas_space_from_blocks")
        if compress:
            _check(self.lib.gas_space_compress_links(ctypes.byref(self._s)),
                   "gas_space_compress_links")

    @property
    def ndet(self):
        return int(self._s.ndet)

    def raw_link_table(self, spin):
        """Return the raw link table of one spin as int64 [nstr, nlink, 4]
        columns (cre, des, addr, sign) -- the layout of fci_gas.h:94-105."""
        nt = int(self._s.ntable)
        tabs = ctypes.cast(self._s.table, ctypes.POINTER(_LinkTable))
        # with one subspace: sector 0 = alpha strings, sector 1 = beta strings
        # (only one sector when na == nb); tables are src->dst == same sector.
        want = 0 if (spin == 0 or self.na == self.nb) else 1
        t = tabs[min(want, nt - 1)]
        n = t.nsrc * t.nlink
        dt = np.dtype([("addr", "<u4"), ("op", "<u2"), ("sign", "i1"), ("pad", "u1")])
        buf = (ctypes.c_char * (8 * n)).from_address(t.link)
        arr = np.frombuffer(bytes(buf), dtype=dt).reshape(t.nsrc, t.nlink)
        out = np.empty((t.nsrc, t.nlink, 4), dtype=np.int64)
        out[..., 0] = arr["op"] & 0xff
        out[..., 1] = arr["op"] >> 8
        out[..., 2] = arr["addr"]
        out[..., 3] = arr["sign"]
        return out

    def close(self):
        if self._s is not None:
            self.lib.gas_space_free(ctypes.byref(self._s))
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _pair_matrix(eri, norb):
    eri = np.asarray(eri, dtype=np.float64)
    npair = norb * (norb + 1) // 2
    if eri.shape == (npair, npair):
        return np.ascontiguousarray(eri)
    eri = eri.reshape(norb, norb, norb, norb)
    idx = np.tril_indices(norb)
    return np.ascontiguousarray(eri[idx[0], idx[1]][:, idx[0], idx[1]])


class SigmaPlan:
    """Reference sigma: fci_contract_gas_plan_create/execute
    (pyscf/lib/mcscf/fci_contract_gas.c:2388-2452; Python twin
    pyscf/mcscf/fci_gas.py:571-623).  h2e is the absorbed 4-fold pair matrix."""

    def __init__(self, norb, nelec, h2e):
        self.space = CASSpace(norb, nelec, compress=True)
        self.eri = _pair_matrix(h2e, norb)
        self.gos = np.ascontiguousarray(self.eri + self.eri.T)
        self._plan = ctypes.c_void_p()
        _check(self.space.lib.fci_contract_gas_plan_create(
            ctypes.byref(self._plan), ctypes.byref(self.space._s),
            _ptr(self.eri), _ptr(self.gos)), "fci_contract_gas_plan_create")

    def __call__(self, ci):
        ci = np.ascontiguousarray(np.asarray(ci, dtype=np.float64).reshape(-1))
        out = np.zeros_like(ci)
        _check(self.space.lib.fci_contract_gas_plan_execute(self._plan, _ptr(ci), _ptr(out)),
               "fci_contract_gas_plan_execute")
        return out

    def close(self):
        if self._plan is not None:
            self.space.lib.fci_contract_gas_plan_free(self._plan)
            self._plan = None
            self.space.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def contract_2e(h2e, ci, norb, nelec):
    plan = SigmaPlan(norb, nelec, h2e)
    try:
        return plan(ci).reshape(np.shape(ci))
    finally:
        plan.close()


def make_hdiag(h1e, eri, norb, nelec):
    """fci_make_hdiag_gas (pyscf/lib/mcscf/fci_hdiag_gas.c:678-709)."""
    sp = CASSpace(norb, nelec)
    try:
        h1 = np.ascontiguousarray(h1e, dtype=np.float64)
        e4 = _pair_matrix(eri, norb)
        out = np.empty(sp.ndet)
        _check(sp.lib.fci_make_hdiag_gas(ctypes.byref(sp._s), _ptr(h1), _ptr(e4), _ptr(out)),
               "fci_make_hdiag_gas")
        return out
    finally:
        sp.close()


def make_rdm12s(bra, ket, norb, nelec):
    """fci_rdm_gas_plan_make_rdm12s (pyscf/lib/mcscf/fci_rdm_gas.c:2207-2243).

    dm1[p,q] = <bra|q+ p|ket>, dm2[p,q,r,s] = <bra|p+ r+ s q|ket>
    (conventions stated at pyscf/lib/mcscf/fci_gas.h:260-268)."""
    sp = CASSpace(norb, nelec)
    plan = ctypes.c_void_p()
    try:
        _check(sp.lib.fci_rdm_gas_plan_create(ctypes.byref(plan), ctypes.byref(sp._s)),
               "fci_rdm_gas_plan_create")
        b = np.ascontiguousarray(np.asarray(bra, dtype=np.float64).reshape(-1))
        k = np.ascontiguousarray(np.asarray(ket, dtype=np.float64).reshape(-1))
        n = norb
        d1a = np.zeros((n, n)); d1b = np.zeros((n, n))
        d2aa = np.zeros((n,) * 4); d2ab = np.zeros((n,) * 4); d2bb = np.zeros((n,) * 4)
        _check(sp.lib.fci_rdm_gas_plan_make_rdm12s(plan, _ptr(b), _ptr(k), _ptr(d1a), _ptr(d1b),
                                                   _ptr(d2aa), _ptr(d2ab), _ptr(d2bb)),
               "fci_rdm_gas_plan_make_rdm12s")
        return (d1a, d1b), (d2aa, d2ab, d2bb)
    finally:
        if plan:
            sp.lib.fci_rdm_gas_plan_free(plan)
        sp.close()


def make_rdm12(bra, ket, norb, nelec):
    """Spin-free assembly as in pyscf/mcscf/fci_gas.py:724-733."""
    (d1a, d1b), (d2aa, d2ab, d2bb) = make_rdm12s(bra, ket, norb, nelec)
    dm2 = d2aa + d2bb + d2ab + d2ab.transpose(2, 3, 0, 1)
    return d1a + d1b, dm2


# ---- libcsf (pyscf/lib/csf/csfstring.c) -------------------------------------

def makecsf(detstrs, coupstrs, nspin, twoS, twoMS):
    """FCICSFmakecsf (csfstring.c:86-141): umat[det, csf]."""
    lib = lib_csf()
    detstrs = np.ascontiguousarray(detstrs, dtype=np.uint64)
    coupstrs = np.ascontiguousarray(coupstrs, dtype=np.uint64)
    umat = np.ones((detstrs.size, coupstrs.size))
    lib.FCICSFmakecsf(umat.ctypes.data_as(ctypes.c_void_p), detstrs.ctypes.data_as(ctypes.c_void_p),
                      coupstrs.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(nspin),
                      ctypes.c_size_t(detstrs.size), ctypes.c_size_t(coupstrs.size),
                      ctypes.c_int(twoS), ctypes.c_int(twoMS))
    return umat


def makeS2mat(detstrs, nspin, twoMS):
    """FCICSFmakeS2mat (csfstring.c:144-174)."""
    lib = lib_csf()
    detstrs = np.ascontiguousarray(detstrs, dtype=np.uint64)
    s2 = np.zeros((detstrs.size, detstrs.size))
    lib.FCICSFmakeS2mat(s2.ctypes.data_as(ctypes.c_void_p), detstrs.ctypes.data_as(ctypes.c_void_p),
                        ctypes.c_size_t(detstrs.size), ctypes.c_int(nspin), ctypes.c_int(twoMS))
    return s2


def addrs2str_genealogical(nspin, smult, addrs, gentable):
    """FCICSFaddrs2str (csfstring.c:243-293)."""
    lib = lib_csf()
    addrs = np.ascontiguousarray(addrs, dtype=np.int32)
    gt = np.ascontiguousarray(gentable, dtype=np.int32).ravel()
    strs = np.zeros(addrs.size, dtype=np.int64)
    lib.FCICSFaddrs2str(strs.ctypes.data_as(ctypes.c_void_p), addrs.ctypes.data_as(ctypes.c_void_p),
                        ctypes.c_size_t(addrs.size), gt.ctypes.data_as(ctypes.c_void_p),
                        ctypes.c_int(nspin), ctypes.c_int(smult - 1))
    return strs


def strs2addr_genealogical(nspin, smult, strs, gentable):
    """FCICSFstrs2addr (csfstring.c:192-240)."""
    lib = lib_csf()
    strs = np.ascontiguousarray(strs, dtype=np.int64)
    gt = np.ascontiguousarray(gentable, dtype=np.int32).ravel()
    addrs = np.zeros(strs.size, dtype=np.int32)
    lib.FCICSFstrs2addr(addrs.ctypes.data_as(ctypes.c_void_p), strs.ctypes.data_as(ctypes.c_void_p),
                        ctypes.c_size_t(strs.size), gt.ctypes.data_as(ctypes.c_void_p),
                        ctypes.c_int(nspin), ctypes.c_int(smult - 1))
    return addrs


def hdiag_blocks(hdiag_det_conf, eri_full, astrs, bstrs, norb):
    """FCICSFhdiag (csfstring.c:295-362): (nconf, ndet, ndet) within-config H."""
    lib = lib_csf()
    nconf, ndet = hdiag_det_conf.shape
    out = np.zeros((nconf, ndet, ndet))
    hd = np.ascontiguousarray(hdiag_det_conf, dtype=np.float64)
    eri = np.ascontiguousarray(eri_full, dtype=np.float64)
    a = np.ascontiguousarray(astrs, dtype=np.uint64)
    b = np.ascontiguousarray(bstrs, dtype=np.uint64)
    lib.FCICSFhdiag(out.ctypes.data_as(ctypes.c_void_p), hd.ctypes.data_as(ctypes.c_void_p),
                    eri.ctypes.data_as(ctypes.c_void_p), a.ctypes.data_as(ctypes.c_void_p),
                    b.ctypes.data_as(ctypes.c_void_p), ctypes.c_uint(norb),
                    ctypes.c_size_t(nconf), ctypes.c_size_t(ndet))
    return out
