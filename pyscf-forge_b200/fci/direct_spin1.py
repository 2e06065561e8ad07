"""Determinant-basis FCI core on the GPU: link tables, absorb_h1e, the
determinant diagonal, sigma and density matrices.

These are the PySCF-core entry points the reference's CSF solver calls
(pyscf/csf_fci/csf.py:5-7,66-68,400,445-450; inherited RDMs via csf.py:557),
rebuilt over libcsffci_b200.  Device-level functions (prefix ``dev_``) take
and return torch CUDA tensors; the PySCF-style functions accept numpy or
torch and answer in the caller's type.
"""
import ctypes
import os
from math import comb

import numpy as np
import torch

from .. import _capi
from .._runtime import (device, eri_pair_matrix, like_input, ptr, require_cuda, stream, to_dev,
                        workspace)


def num_strings(norb, nelec):
    return comb(norb, nelec) if 0 <= nelec <= norb else 0


def _unpack_nelec(nelec, spin=None):
    """(neleca, nelecb) from an int or a pair (role of direct_spin1._unpack_nelec)."""
    if isinstance(nelec, (int, np.integer)):
        nelec = int(nelec)
        if spin is None:
            spin = nelec % 2
        na = (nelec + spin) // 2
        return na, nelec - na
    return int(nelec[0]), int(nelec[1])


_LINK_CACHE = {}


def dev_link_table(norb, nelec):
    """Device link table int64[N, nlink] (each element one csffci_link_t)."""
    require_cuda()
    key = (torch.cuda.current_device(), int(norb), int(nelec))
    t = _LINK_CACHE.get(key)
    if t is None:
        n = num_strings(norb, nelec)
        nlink = nelec * (norb - nelec + 1)
        t = torch.empty((n, max(nlink, 1)), dtype=torch.int64, device=device())
        if nlink > 0 and n > 0:
            _capi.call("csffci_link_table", norb, nelec, ptr(t), stream())
        _LINK_CACHE[key] = t
    return t


def decode_link_table(t):
    """int64[N, nlink] device table -> numpy int64[N, nlink, 4] with columns
    (cre, des, addr, sign) -- for inspection and tests."""
    raw = t.cpu().numpy().view(np.uint8).reshape(t.shape[0], t.shape[1], 8)
    addr = raw[..., 0:4].copy().view(np.uint32)[..., 0].astype(np.int64)
    op = raw[..., 4:6].copy().view(np.uint16)[..., 0].astype(np.int64)
    sign = raw[..., 6].view(np.int8).astype(np.int64)
    out = np.stack([op & 0xff, op >> 8, addr, sign], axis=-1)
    return out


def dev_absorb_h1e(h1e, eri4, norb, nelec, fac=1.0):
    """h2e (npair, npair) with h1e folded in (csf.py:445,520)."""
    if not isinstance(nelec, (int, np.integer)):
        nelec = sum(nelec)
    h1 = to_dev(h1e).reshape(norb, norb)
    e4 = to_dev(eri4)
    npair = norb * (norb + 1) // 2
    out = torch.empty((npair, npair), dtype=torch.float64, device=device())
    _capi.call("csffci_absorb_h1e", norb, int(nelec), ptr(h1), ptr(e4), float(fac), ptr(out), stream())
    return out


def dev_make_hdiag(h1a, h1b, eri4, norb, nelec):
    na, nb = nelec
    h1a = to_dev(h1a).reshape(norb, norb)
    h1b = to_dev(h1b).reshape(norb, norb)
    e4 = to_dev(eri4)
    out = torch.empty(num_strings(norb, na) * num_strings(norb, nb), dtype=torch.float64,
                      device=device())
    nbytes = _capi.query("csffci_hdiag_det_workspace", norb, na, nb)
    ws = workspace("hdiag", nbytes)
    _capi.call("csffci_hdiag_det", norb, na, nb, ptr(h1a), ptr(h1b), ptr(e4), ptr(out), ptr(ws),
               nbytes, stream())
    return out


class SigmaPlan:
    """csffci_sigma_plan for one (norb, nelec, h2e): link tables, kernel
    choice and workspace bound once, then executed per vector (the model of
    the reference's fci_contract_gas_plan, pyscf/lib/mcscf/fci_gas.h:244-253).
    Holds references to h2e and the link tables, whose device memory the
    plan borrows; the kernel is fixed at creation (CSFFCI_SIGMA_VARIANT is
    read then).  deterministic: the scatter of CSFFCI_SIGMA_DETERMINISTIC
    (bit-identical reruns, 4 <= norb <= 16)."""

    def __init__(self, h2e, norb, nelec, spin_symmetric=False, deterministic=False):
        require_cuda()
        na, nb = nelec
        self.norb, self.nelec = int(norb), (int(na), int(nb))
        self.h2e = h2e.contiguous()
        self.la = dev_link_table(norb, na)
        self.lb = dev_link_table(norb, nb)
        self.sym = bool(spin_symmetric) and na == nb
        self.deterministic = bool(deterministic)
        flags = _capi.SIGMA_SPIN_SYMMETRIC if self.sym else 0
        if self.deterministic:
            flags |= _capi.SIGMA_DETERMINISTIC
        h = ctypes.c_void_p()
        nbytes = ctypes.c_size_t()
        _capi.call("csffci_sigma_plan_create", self.norb, na, nb, ptr(self.h2e), ptr(self.la), ptr(self.lb),
                   flags, ctypes.byref(h), ctypes.byref(nbytes))
        self._h = h
        self.work_bytes = int(nbytes.value)
        self._bound = None
        self.variant = _capi.query("csffci_sigma_plan_variant", h)

    def __call__(self, ci, out, eta=None, accumulate=False):
        flags = _capi.SIGMA_ACCUMULATE if accumulate else 0
        if eta is not None:
            if not self.sym:
                raise ValueError("the plan was created without the spin-symmetric mode")
            flags |= _capi.SIGMA_SPIN_SYMMETRIC
        if self.work_bytes:
            # the spin-symmetric scratch is the shared stream-ordered sigma
            # workspace (one per device, not one per plan); rebind when it
            # was reallocated
            ws = workspace("sigma", self.work_bytes)
            if ws.data_ptr() != self._bound:
                _capi.call("csffci_sigma_plan_bind", self._h, ptr(ws), ws.numel())
                self._bound = ws.data_ptr()
        _capi.call("csffci_sigma_plan_execute", self._h, ptr(ci), ptr(out), int(eta or 1), flags, stream())
        return out

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        # at interpreter exit the module globals may already be gone
        lib = getattr(_capi, "_LIB", None) if _capi is not None else None
        if h is not None and lib is not None:
            lib.csffci_sigma_plan_destroy(h)


_PLAN_CACHE = {}
_PLAN_CACHE_SIZE = 8


def sigma_plan(h2e, norb, nelec, deterministic=False):
    """The cached SigmaPlan of (device, norb, nelec, h2e tensor, scatter
    mode); the cache keeps the h2e tensor alive, so its address names it,
    and holds at most _PLAN_CACHE_SIZE plans (least recently used dropped
    first)."""
    key = (torch.cuda.current_device(), int(norb), int(nelec[0]), int(nelec[1]), h2e.data_ptr(),
           tuple(h2e.shape), bool(deterministic))
    plan = _PLAN_CACHE.pop(key, None)
    if plan is None or plan.h2e.data_ptr() != h2e.data_ptr():
        plan = SigmaPlan(h2e, norb, nelec, spin_symmetric=nelec[0] == nelec[1], deterministic=deterministic)
    _PLAN_CACHE[key] = plan
    while len(_PLAN_CACHE) > _PLAN_CACHE_SIZE:
        _PLAN_CACHE.pop(next(iter(_PLAN_CACHE)))
    return plan


def dev_contract_2e(h2e, ci, norb, nelec, eta=None, out=None, accumulate=False, deterministic=False):
    """sigma = sum h2e[pq,rs] E_pq E_rs ci on the device.  eta (+1/-1) asserts
    ci = eta ci^T (na == nb) and selects the row-local kernel; deterministic
    selects the order-independent scatter (bit-identical reruns).  Runs
    through the cached sigma plan of (norb, nelec, h2e, scatter mode)."""
    na, nb = nelec
    ci = ci.contiguous()
    if out is None:
        out = torch.empty_like(ci)
        accumulate = False
    h2e = h2e if h2e.is_contiguous() else h2e.contiguous()
    if os.environ.get("CSFFCI_SIGMA_VARIANT") is not None:
        # a kernel named for this call (tests, profiling): an unplanned call
        # reads the variable on every launch
        la = dev_link_table(norb, na)
        lb = dev_link_table(norb, nb)
        flags = _capi.SIGMA_ACCUMULATE if accumulate else 0
        if eta is not None:
            flags |= _capi.SIGMA_SPIN_SYMMETRIC
        if deterministic:
            flags |= _capi.SIGMA_DETERMINISTIC
        nbytes = _capi.query("csffci_sigma_workspace", norb, na, nb, flags)
        ws = workspace("sigma", nbytes) if nbytes else None
        _capi.call("csffci_sigma", norb, na, nb, ptr(h2e), ptr(la), ptr(lb), ptr(ci), ptr(out), flags,
                   int(eta or 1), ptr(ws), nbytes, stream())
        return out
    return sigma_plan(h2e, norb, (na, nb), deterministic)(ci, out, eta=eta, accumulate=accumulate)


def dev_spin_parity(ci, n, rtol=1e-12):
    """+1 / -1 if the (n, n) CI matrix is symmetric / antisymmetric to
    rtol*max|c|, else None (decides the spin-symmetric sigma path)."""
    out = torch.empty(3, dtype=torch.float64, device=ci.device)
    ws = workspace("parity", 148 * 4 * 3 * 8)
    _capi.call("csffci_spin_parity", n, ptr(ci), ptr(out), ptr(ws), ws.numel(), stream())
    a, b, m = out.cpu().numpy()
    if m == 0.0:
        return None
    if a <= rtol * m:
        return 1
    if b <= rtol * m:
        return -1
    return None


def dev_contract_1e(h1a, h1b, ci, norb, nelec, out):
    """out += sum h1a[p,q] Ea_pq ci + h1b[p,q] Eb_pq ci (csf.py:527-528)."""
    na, nb = nelec
    la = dev_link_table(norb, na)
    lb = dev_link_table(norb, nb)
    h1a = to_dev(h1a).reshape(norb, norb)
    h1b = to_dev(h1b).reshape(norb, norb)
    _capi.call("csffci_contract_1e", norb, na, nb, ptr(h1a), ptr(h1b), ptr(la), ptr(lb),
               ptr(ci.contiguous()), ptr(out), stream())
    return out


def dev_rdm12(bra, ket, norb, nelec, with_dm2=True):
    na, nb = nelec
    la = dev_link_table(norb, na)
    lb = dev_link_table(norb, nb)
    dm1 = torch.empty((norb, norb), dtype=torch.float64, device=device())
    dm2 = torch.empty((norb,) * 4, dtype=torch.float64, device=device()) if with_dm2 else None
    nbytes = _capi.query("csffci_rdm12_workspace", norb, na, nb)
    ws = workspace("rdm", nbytes)
    bra = bra.contiguous()
    ket = bra if ket is None else ket.contiguous()
    _capi.call("csffci_rdm12", norb, na, nb, ptr(la), ptr(lb), ptr(bra), ptr(ket), ptr(dm1),
               ptr(dm2), ptr(ws), nbytes, stream())
    return dm1, dm2


def dev_rdm12s(bra, ket, norb, nelec, with_dm2=True):
    """Spin-resolved RDMs on the device: ((dm1a, dm1b), (dm2aa, dm2ab,
    dm2bb)) with dm1s[p,q] = <q+ p>, dm2ab[p,q,r,s] = <p+_a r+_b s_b q_a>
    (conventions of fci_gas.h:260-268; reference twin
    fci_rdm_gas_plan_make_rdm12s, fci_rdm_gas.c:2207-2243)."""
    na, nb = nelec
    la = dev_link_table(norb, na)
    lb = dev_link_table(norb, nb)
    dev = device()
    d1 = [torch.empty((norb, norb), dtype=torch.float64, device=dev) for _ in range(2)]
    d2 = [torch.empty((norb,) * 4, dtype=torch.float64, device=dev) for _ in range(3)] if with_dm2 \
        else [None, None, None]
    nbytes = _capi.query("csffci_rdm12s_workspace", norb, na, nb)
    ws = workspace("rdm12s", nbytes)
    bra = bra.contiguous()
    ket = bra if ket is None else ket.contiguous()
    _capi.call("csffci_rdm12s", norb, na, nb, ptr(la), ptr(lb), ptr(bra), ptr(ket), ptr(d1[0]), ptr(d1[1]),
               ptr(d2[0]), ptr(d2[1]), ptr(d2[2]), ptr(ws), nbytes, stream())
    return tuple(d1), tuple(d2)


# ---------------------------------------------------------------------------
# PySCF-style functions (numpy in/out, or torch when given torch)
# ---------------------------------------------------------------------------

def absorb_h1e(h1e, eri, norb, nelec, fac=1):
    h2e = dev_absorb_h1e(h1e, eri_pair_matrix(eri, norb), norb, nelec, fac)
    return like_input(h2e, eri)


def make_hdiag(h1e, eri, norb, nelec, compress=False):
    nelec = _unpack_nelec(nelec)
    h1 = h1e.detach().cpu().numpy() if isinstance(h1e, torch.Tensor) else np.asarray(h1e)
    if h1.ndim == 3:
        h1a, h1b = h1[0], h1[1]
    else:
        h1a = h1b = h1
    out = dev_make_hdiag(h1a, h1b, eri_pair_matrix(eri, norb), norb, nelec)
    return like_input(out, h1e)


def contract_2e(eri, fcivec, norb, nelec, link_index=None):
    nelec = _unpack_nelec(nelec)
    h2e = to_dev(eri_pair_matrix(eri, norb))
    ci = to_dev(fcivec)
    eta = dev_spin_parity(ci, num_strings(norb, nelec[0])) if nelec[0] == nelec[1] else None
    out = dev_contract_2e(h2e, ci.reshape(-1), norb, nelec, eta=eta)
    return like_input(out.reshape(ci.shape), fcivec)


def contract_1e(f1e, fcivec, norb, nelec, link_index=None):
    nelec = _unpack_nelec(nelec)
    f = f1e.detach().cpu().numpy() if isinstance(f1e, torch.Tensor) else np.asarray(f1e)
    fa, fb = (f[0], f[1]) if f.ndim == 3 else (f, f)
    ci = to_dev(fcivec).reshape(-1)
    out = torch.zeros_like(ci)
    dev_contract_1e(fa, fb, ci, norb, nelec, out)
    return like_input(out.reshape(to_dev(fcivec).shape), fcivec)


def make_rdm1(fcivec, norb, nelec, link_index=None):
    nelec = _unpack_nelec(nelec)
    c = to_dev(fcivec).reshape(-1)
    dm1, _ = dev_rdm12(c, None, norb, nelec, with_dm2=False)
    return like_input(dm1, fcivec)


def make_rdm12(fcivec, norb, nelec, link_index=None, reorder=True):
    nelec = _unpack_nelec(nelec)
    c = to_dev(fcivec).reshape(-1)
    dm1, dm2 = dev_rdm12(c, None, norb, nelec)
    return like_input(dm1, fcivec), like_input(dm2, fcivec)


def trans_rdm1(cibra, ciket, norb, nelec, link_index=None):
    nelec = _unpack_nelec(nelec)
    dm1, _ = dev_rdm12(to_dev(cibra).reshape(-1), to_dev(ciket).reshape(-1), norb, nelec,
                       with_dm2=False)
    return like_input(dm1, cibra)


def trans_rdm12(cibra, ciket, norb, nelec, link_index=None, reorder=True):
    nelec = _unpack_nelec(nelec)
    dm1, dm2 = dev_rdm12(to_dev(cibra).reshape(-1), to_dev(ciket).reshape(-1), norb, nelec)
    return like_input(dm1, cibra), like_input(dm2, cibra)


def make_rdm1s(fcivec, norb, nelec, link_index=None):
    """(dm1a, dm1b) (direct_spin1.make_rdm1s, inherited at csf.py:557)."""
    nelec = _unpack_nelec(nelec)
    (d1a, d1b), _ = dev_rdm12s(to_dev(fcivec).reshape(-1), None, norb, nelec, with_dm2=False)
    return like_input(d1a, fcivec), like_input(d1b, fcivec)


def make_rdm12s(fcivec, norb, nelec, link_index=None, reorder=True):
    """((dm1a, dm1b), (dm2aa, dm2ab, dm2bb)) (direct_spin1.make_rdm12s)."""
    nelec = _unpack_nelec(nelec)
    d1, d2 = dev_rdm12s(to_dev(fcivec).reshape(-1), None, norb, nelec)
    return tuple(like_input(x, fcivec) for x in d1), tuple(like_input(x, fcivec) for x in d2)


def trans_rdm1s(cibra, ciket, norb, nelec, link_index=None):
    nelec = _unpack_nelec(nelec)
    (d1a, d1b), _ = dev_rdm12s(to_dev(cibra).reshape(-1), to_dev(ciket).reshape(-1), norb, nelec,
                               with_dm2=False)
    return like_input(d1a, cibra), like_input(d1b, cibra)


def trans_rdm12s(cibra, ciket, norb, nelec, link_index=None, reorder=True):
    nelec = _unpack_nelec(nelec)
    d1, d2 = dev_rdm12s(to_dev(cibra).reshape(-1), to_dev(ciket).reshape(-1), norb, nelec)
    return tuple(like_input(x, cibra) for x in d1), tuple(like_input(x, cibra) for x in d2)


def energy(h1e, eri, fcivec, norb, nelec, link_index=None):
    h2e = absorb_h1e(h1e, eri, norb, nelec, 0.5)
    ci = to_dev(fcivec).reshape(-1)
    sig = dev_contract_2e(to_dev(h2e), ci, norb, _unpack_nelec(nelec))
    return float(torch.dot(ci, sig))
