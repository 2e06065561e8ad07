"""CSFTransformer on the GPU: genealogical CSF addressing, spin eigenvectors
and the CSF <-> determinant transforms.

Mirrors pyscf/csf_fci/csfstring.py (class CSFTransformer 33-223 and the
module functions it uses).  The masks (csd_mask, econf_det_mask,
econf_csf_mask) and the per-npair spin eigenvector blocks live on the device
and are built once per (norb, neleca, nelecb, smult), as in
_update_spin_cache (csfstring.py:105-115); unlike the reference the spin
eigenvectors are cached instead of being rebuilt on every transform
(csfstring.py:630).
"""
import ctypes
from math import comb

import numpy as np
import torch

from .. import _capi
from .._runtime import device, ptr, require_cuda, stream, to_dev, workspace
from .csdstring import get_csdaddrs_shape, check_csd_mask_size


class ImpossibleCIvecError(RuntimeError):
    """csfstring.py:15-25."""

    def __init__(self, message, ndet=None, ncsf=None, norb=None, neleca=None, nelecb=None):
        self.message = message
        self.ndet = ndet
        self.ncsf = ncsf
        self.norb = norb
        self.neleca = neleca
        self.nelecb = nelecb

    def __str__(self):
        return self.message


class ImpossibleSpinError(ImpossibleCIvecError):
    """csfstring.py:27-31."""

    def __init__(self, message, ndet=None, ncsf=None, norb=None, neleca=None, nelecb=None, smult=None):
        ImpossibleCIvecError.__init__(self, message, ndet=ndet, ncsf=ncsf, norb=norb,
                                      neleca=neleca, nelecb=nelecb)
        self.smult = smult


def csf_gentable(nspin, smult):
    """Genealogical path-count table (csfstring.py:806-849)."""
    assert (smult - 1) % 2 == nspin % 2, "{} {}".format(smult, nspin)
    if smult > nspin + 1:
        return np.zeros((1, 1), dtype=np.int32)
    n0 = (nspin - (smult - 1)) // 2
    n1 = (nspin + (smult - 1)) // 2
    g = np.zeros((n0 + 1, n1 + 1), dtype=np.int64)
    g[n0, n0:] = 1
    for i0 in range(n0, 0, -1):
        row = list(g[i0, i0:])
        row = [sum(row[i1:]) for i1 in range(len(row))]
        row = [row[0]] + row
        g[i0 - 1, i0 - 1:] = row
    return g.astype(np.int32)


def count_csfs(nspin, smult):
    """csfstring.py:851-852 (closed form of the table's corner)."""
    twoS = smult - 1
    if twoS > nspin or (nspin - twoS) % 2:
        return 0
    n0 = (nspin - twoS) // 2
    return comb(nspin, n0) - (comb(nspin, n0 - 1) if n0 > 0 else 0)


def get_csfvec_shape(norb, neleca, nelecb, smult):
    """csfstring.py:858-911: (min_npair, npair_offset, npair_dconf_size,
    npair_sconf_size, npair_csf_size)."""
    s = (smult - 1) / 2
    ms = (neleca - nelecb) / 2
    nless = min(neleca, nelecb)
    if neleca > norb or nelecb > norb or neleca < 0 or nelecb < 0:
        raise ImpossibleCIvecError("({}e+{}e,{}o)".format(neleca, nelecb, norb),
                                   norb=norb, neleca=neleca, nelecb=nelecb)
    if abs(neleca - nelecb) > smult - 1:
        raise ImpossibleSpinError("Impossible quantum numbers: s = {}; ms = {}".format(s, ms),
                                  norb=norb, neleca=neleca, nelecb=nelecb, smult=smult)
    min_npair = max(0, neleca + nelecb - norb)
    pairs = range(min_npair, nless + 1)
    nspins = [neleca + nelecb - 2 * p for p in pairs]
    if (smult - 1) > nspins[0]:
        raise ImpossibleSpinError('Maximum possible 2s+1 = {} for ({}e+{}e,{}o)'.format(
            nspins[0] + 1, neleca, nelecb, norb), norb=norb, neleca=neleca, nelecb=nelecb,
            smult=smult)
    dconf = np.array([comb(norb, p) for p in pairs], dtype=np.int64)
    sconf = np.array([comb(norb - p, ns) for p, ns in zip(pairs, nspins)], dtype=np.int64)
    ncsf = np.array([count_csfs(ns, smult) for ns in nspins], dtype=np.int64)
    sizes = dconf * sconf * ncsf
    offset = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    return min_npair, offset, dconf, sconf, ncsf


def count_all_csfs(norb, neleca, nelecb, smult):
    a, b, c = get_csfvec_shape(norb, neleca, nelecb, smult)[-3:]
    return int(np.sum(a * b * c))


def addrs2str(nspin, smult, addrs):
    """Genealogical coupling strings of addresses (csfstring.c:243-293)."""
    g = csf_gentable(nspin, smult)
    n1 = (nspin + smult - 1) // 2
    out = np.zeros(len(addrs), dtype=np.int64)
    for j, a in enumerate(np.asarray(addrs, dtype=np.int64).tolist()):
        s, i0, i1 = 1, 0, 0
        for ispin in range(nspin):
            if i1 == n1:
                break
            if g[i0, i1 + 1] <= a:
                a -= int(g[i0, i1 + 1])
                i0 += 1
            else:
                s |= 1 << ispin
                i1 += 1
        out[j] = s
    return out


def strs2addr(nspin, smult, strs):
    """Genealogical addresses of coupling strings (csfstring.c:192-240)."""
    g = csf_gentable(nspin, smult)
    n1 = (nspin + smult - 1) // 2
    out = np.zeros(len(strs), dtype=np.int32)
    for j, s in enumerate(np.asarray(strs, dtype=np.int64).tolist()):
        a, i0, i1 = 0, 0, 0
        for ispin in range(nspin):
            if (s >> ispin) & 1:
                i1 += 1
            else:
                if i1 < n1:
                    a += int(g[i0, i1 + 1])
                i0 += 1
        out[j] = a
    return out


def get_spin_evecs(nspin, neleca, nelecb, smult):
    """umat[det, csf] of nspin unpaired electrons (csfstring.py:913-960) as a
    device tensor, bit-identical to FCICSFmakecsf (csfstring.c:86-141)."""
    assert abs(neleca - nelecb) <= smult - 1
    assert abs(neleca - nelecb) <= nspin
    assert abs(neleca - nelecb) % 2 == (smult - 1) % 2
    assert abs(neleca - nelecb) % 2 == nspin % 2
    na = (nspin + neleca - nelecb) // 2
    ndet = comb(nspin, na)
    ncsf = count_csfs(nspin, smult)
    umat = torch.empty((ndet, ncsf), dtype=torch.float64, device=device())
    if ndet * ncsf:
        _capi.call("csffci_spin_evecs", nspin, neleca, nelecb, smult, ptr(umat), stream())
    return umat


def _block_sign(npair, nelecb):
    """csfstring.py:623-627."""
    ncomm = npair * (npair - 1) // 2 + npair * max(0, nelecb - npair)
    return -1.0 if ncomm % 2 else 1.0


class CSFTransformer:
    """GPU counterpart of csfstring.CSFTransformer (csfstring.py:33-223)."""

    def __init__(self, norb, neleca, nelecb, smult, orbsym=None, wfnsym=None, max_memory=None, gas=None):
        require_cuda()
        self._norb = self._neleca = self._nelecb = self._smult = None
        self._orbsym = None
        self.confsym = None
        self._gas = None
        self.confgas = None
        self._symcache = {}
        self.wfnsym = wfnsym
        self.max_memory = max_memory
        self._update_spin_cache(norb, neleca, nelecb, smult)
        self.orbsym = orbsym
        self.gas = gas

    # ---- cache -----------------------------------------------------------
    def _update_spin_cache(self, norb, neleca, nelecb, smult):
        if (self._norb, self._neleca, self._nelecb, self._smult) == (norb, neleca, nelecb, smult):
            return
        check_csd_mask_size(norb, neleca, nelecb)
        min_npair, csf_off, dconf, sconf, ncsf_b = get_csfvec_shape(norb, neleca, nelecb, smult)
        _, csd_off, _, _, spins = get_csdaddrs_shape(norb, neleca, nelecb)
        self._norb, self._neleca, self._nelecb, self._smult = norb, neleca, nelecb, smult
        ndet = comb(norb, neleca) * comb(norb, nelecb)
        self._ncsf = int(np.sum(dconf * sconf * ncsf_b))
        dev = device()
        self.csd_mask = torch.empty(ndet, dtype=torch.int32, device=dev)
        self.econf_det_mask = torch.empty(ndet, dtype=torch.int32, device=dev)
        self.econf_csf_mask = torch.empty(max(self._ncsf, 1), dtype=torch.int32, device=dev)
        _capi.call("csffci_csd_masks", norb, neleca, nelecb, smult, ptr(self.csd_mask),
                   ptr(self.econf_det_mask), ptr(self.econf_csf_mask), stream())
        self.econf_csf_mask = self.econf_csf_mask[:self._ncsf]
        self._blocks = []
        for ip, npair in enumerate(range(min_npair, min(neleca, nelecb) + 1)):
            nspin = neleca + nelecb - 2 * npair
            nc = int(ncsf_b[ip])
            umat = get_spin_evecs(nspin, neleca, nelecb, smult) if nc > 0 else None
            self._blocks.append(dict(npair=npair, nspin=nspin, csd_offset=int(csd_off[ip]),
                                     csf_offset=int(csf_off[ip]), nconf=int(dconf[ip] * sconf[ip]),
                                     ndet=int(spins[ip]), ncsf=nc,
                                     sign=_block_sign(npair, nelecb), umat=umat, zmat=None))
        self._cblocks = None
        self._eta = None
        self._shape_info = (min_npair, csf_off, dconf, sconf, ncsf_b)
        self._symcache = {}
        if self._orbsym is not None:
            self.confsym = make_confsym(norb, neleca, nelecb, self.econf_det_mask, self._orbsym)
        self.confgas = None
        if self._gas is not None:
            self.confgas = make_confgas(norb, neleca, nelecb, self.econf_det_mask, self._gas)

    def _update_symm_cache(self, orbsym):
        """csfstring.py:117-120: configuration irreps for a new orbsym."""
        if orbsym is not None:
            orbsym = np.asarray(orbsym, dtype=np.int64)
        changed = (orbsym is None) != (self._orbsym is None) or (
            orbsym is not None and (orbsym.shape != self._orbsym.shape or np.any(orbsym != self._orbsym)))
        if orbsym is not None and (self.confsym is None or changed):
            self.confsym = make_confsym(self._norb, self._neleca, self._nelecb, self.econf_det_mask, orbsym)
        if changed:
            self._symcache = {}
        if orbsym is None:
            self.confsym = None
        self._orbsym = orbsym

    # ---- GAS restriction ---------------------------------------------------
    @property
    def gas(self):
        """(subspace sizes, spin-free supergroup rows) of a GAS restriction,
        or None (csf_fci.gas.spin_free_supergroups gives this form)."""
        return self._gas

    @gas.setter
    def gas(self, spec):
        if spec is not None:
            orbs, sg = spec
            orbs = tuple(int(n) for n in orbs)
            sg = np.ascontiguousarray(np.asarray(sg, dtype=np.int32).reshape(-1, len(orbs)))
            if sum(orbs) != self._norb:
                raise ValueError("GAS subspaces hold %d orbitals, the space has %d" % (sum(orbs), self._norb))
            spec = (orbs, sg)
        old = self._gas
        same = (old is None and spec is None) or (
            old is not None and spec is not None and old[0] == spec[0] and np.array_equal(old[1], spec[1]))
        if same:
            return
        self._gas = spec
        self._symcache = {}
        self.confgas = None if spec is None else make_confgas(
            self._norb, self._neleca, self._nelecb, self.econf_det_mask, spec)

    def _conf_selected(self):
        """Boolean device mask over configurations: those of irrep wfnsym
        (with point-group symmetry) and inside the GAS restriction (with
        one); None when neither restricts the space."""
        sym = self.wfnsym is not None and self._orbsym is not None
        if not sym and self._gas is None:
            return None
        sel = None
        if sym:
            sel = self.confsym == int(self.wfnsym)
        if self._gas is not None:
            g = self.confgas.to(torch.bool)
            sel = g if sel is None else (sel & g)
        return sel

    def _sym(self):
        """Packing of the CSF vector to the CSFs of the selected
        configurations -- those of irrep wfnsym (csfstring.py:74-88) and,
        with a GAS restriction, inside it: per block the selected
        configurations and their packed offsets.  None when the space is not
        restricted."""
        sym = self.wfnsym is not None and self._orbsym is not None
        if not sym and self._gas is None:
            return None
        key = (int(self.wfnsym) if sym else None, self._gas is not None)
        st = self._symcache.get(key)
        if st is not None:
            return st
        cs = self._conf_selected()
        sel, offs, nsel = [], [], []
        c0 = 0
        packed = 0
        for b in self._blocks:
            nconf = b["nconf"]
            idx = torch.nonzero(cs[c0:c0 + nconf]).reshape(-1).to(torch.int32)
            sel.append(idx.contiguous())
            offs.append(packed)
            nsel.append(int(idx.numel()))
            packed += int(idx.numel()) * b["ncsf"]
            c0 += nconf
        idx_sym = cs[self.econf_csf_mask.long()]
        st = dict(sel=sel, offs=offs, nsel=nsel, ncsf=packed, idx_sym=idx_sym,
                  pos=torch.cumsum(idx_sym.to(torch.int64), 0) - 1)
        self._symcache[key] = st
        return st

    @property
    def idx_sym(self):
        """Boolean device mask over all CSFs: those of the irrep wfnsym (the
        idx_sym of csf_symm.py:77); None without symmetry."""
        st = self._sym()
        return None if st is None else st["idx_sym"]

    def _c_blocks(self, with_zmat=False, packed=True):
        if with_zmat:
            for b in self._blocks:
                if b["ncsf"] and b["nspin"] >= 2 and b["zmat"] is None:
                    npos = b["nspin"] * (b["nspin"] - 1) // 2
                    z = torch.empty((npos, b["ncsf"]), dtype=torch.float64, device=device())
                    _capi.call("csffci_spin_exchange_table", b["nspin"], self._neleca, self._nelecb,
                               self._smult, ptr(b["umat"]), ptr(z), stream())
                    b["zmat"] = z
        arr = (_capi.Block * len(self._blocks))()
        for i, b in enumerate(self._blocks):
            arr[i].csd_offset = b["csd_offset"]
            arr[i].csf_offset = b["csf_offset"]
            arr[i].nconf = b["nconf"]
            arr[i].ndet = b["ndet"]
            arr[i].ncsf = b["ncsf"]
            arr[i].nspin = b["nspin"]
            arr[i].npair = b["npair"]
            arr[i].sign = b["sign"]
            arr[i].umat = b["umat"].data_ptr() if b["umat"] is not None and b["umat"].numel() else None
            arr[i].zmat = b["zmat"].data_ptr() if b["zmat"] is not None else None
        st = self._sym() if packed else None
        if st is not None:
            for i in range(len(self._blocks)):
                arr[i].nconf = st["nsel"][i]
                arr[i].csf_offset = st["offs"][i]
                arr[i].conf_sel = st["sel"][i].data_ptr() if st["nsel"][i] else None
        return arr

    # ---- device transforms ----------------------------------------------
    def dev_det2csf(self, x):
        """x: device (nvec, ndet) -> (nvec, ncsf), no normalisation; with
        point-group symmetry the CSF vector is the packed one (only the
        configurations of the irrep wfnsym are formed)."""
        x = x.reshape(-1, self.ndet).contiguous()
        n = self.ncsf
        out = torch.empty((x.shape[0], n), dtype=torch.float64, device=x.device)
        blocks = self._c_blocks()
        _capi.call("csffci_det2csf", x.shape[0], ptr(x), self.ndet, ptr(out), n,
                   ptr(self.csd_mask), blocks, len(self._blocks), stream())
        return out

    def dev_csf2det(self, x):
        """x: device (nvec, ncsf) -> (nvec, ndet), no normalisation (packed
        CSF vectors with point-group symmetry)."""
        n = self.ncsf
        x = x.reshape(-1, n).contiguous()
        out = torch.empty((x.shape[0], self.ndet), dtype=torch.float64, device=x.device)
        blocks = self._c_blocks()
        _capi.call("csffci_csf2det", x.shape[0], ptr(x), n, ptr(out), self.ndet, self.ndet,
                   ptr(self.csd_mask), blocks, len(self._blocks), stream())
        return out

    def dev_hdiag_csf(self, hdiag_det, eri4, packed=False):
        """CSF diagonal over all CSFs (as make_hdiag_csf returns it,
        csf.py:70-144), or over the packed symmetric CSFs."""
        st = self._sym() if packed else None
        out = torch.empty(self._ncsf if st is None else st["ncsf"], dtype=torch.float64, device=device())
        blocks = self._c_blocks(with_zmat=True, packed=packed)
        _capi.call("csffci_hdiag_csf", self._norb, self._neleca, self._nelecb, ptr(hdiag_det),
                   ptr(eri4), ptr(self.csd_mask), blocks, len(self._blocks), ptr(out), stream())
        return out

    @property
    def spin_parity(self):
        """eta with c[Ia,Ib] = eta c[Ib,Ia] for every determinant vector built
        from CSFs when neleca == nelecb (None otherwise); found once by
        transforming a probe vector."""
        if self._neleca != self._nelecb:
            return None
        if self._eta is None:
            g = torch.Generator(device="cpu").manual_seed(7)
            x = torch.randn(max(self.ncsf, 1), generator=g, dtype=torch.float64)[:self.ncsf].to(device())
            c = self.dev_csf2det(x).reshape(self.ndeta, self.ndetb)
            sym = float(torch.linalg.norm(c - c.T))
            anti = float(torch.linalg.norm(c + c.T))
            self._eta = 1 if sym <= anti else -1
        return self._eta

    # ---- reference-shaped API ------------------------------------------
    def vec_det2csf(self, civec, order='C', normalize=True, return_norm=False):
        """csfstring.py:45-52 / transform_civec_det2csf 341-414."""
        civec, norm = self._transform(civec, order, normalize, reverse=False)
        if return_norm:
            return civec, norm
        return civec

    def vec_csf2det(self, civec, order='C', normalize=True, return_norm=False):
        """csfstring.py:54-60 / transform_civec_csf2det 416-487."""
        civec, norm = self._transform(civec, order, normalize, reverse=True)
        if return_norm:
            return civec, norm
        return civec

    def _transform(self, arr, order, normalize, reverse):
        vec_on_cols = order.upper() == 'F'
        is_torch = isinstance(arr, torch.Tensor)
        is_list = isinstance(arr, list)
        is_tuple = isinstance(arr, tuple)
        ncol_in = self.ncsf if reverse else self.ndet
        if is_list or is_tuple:
            nvec = len(arr)
            is_flat = False
            x = torch.stack([to_dev(a).reshape(-1) for a in arr]) if nvec else None
        else:
            size = arr.numel() if is_torch else np.asarray(arr).size
            if reverse and size == 0:
                return (arr, 0.0)
            if size % ncol_in != 0:
                raise ImpossibleCIvecError(
                    'Impossible CI vector size {0} for system with {1} {2}'.format(
                        size, ncol_in, 'CSFs' if reverse else 'determinants'),
                    ndet=self.ndet, norb=self._norb, neleca=self._neleca, nelecb=self._nelecb)
            nvec = size // ncol_in
            is_flat = len(arr.shape) == 1
            x = to_dev(arr)
        if vec_on_cols:
            x = x.reshape(ncol_in, nvec).T.contiguous()
        else:
            x = x.reshape(nvec, ncol_in)
        y = self.dev_csf2det(x) if reverse else self.dev_det2csf(x)
        norm = torch.linalg.norm(y, dim=1)
        if normalize:
            if reverse:
                y = y / norm[:, None]
            else:
                ok = ~torch.isclose(norm, torch.zeros_like(norm))
                y = torch.where(ok[:, None], y / torch.where(ok, norm, torch.ones_like(norm))[:, None], y)
        if vec_on_cols:
            y = y.T.contiguous()
        if not is_torch:
            y = y.cpu().numpy()
            norm = norm.cpu().numpy()
        if is_flat:
            y = y.reshape(-1)
        elif is_list:
            y = list(y)
        elif is_tuple:
            y = tuple(y)
        if norm.shape[0] == 1:
            norm = norm[0] if not is_torch else norm[0]
            norm = float(norm)
        return y, norm

    def mat_det2csf_confspace(self, mat, confs):
        """transform_opmat_det2csf_pspace (csfstring.py:676-785): an operator
        given over every determinant of the configurations ``confs`` (ordered
        configuration by configuration, determinants ascending within each)
        -> CSF basis over those configurations; returns (op, csf_addrs) with
        csf_addrs sorted."""
        from .csf import _pspace_transform
        return _pspace_transform(self, mat, confs)

    def _pack(self, vec, idx, order, n_full):
        if idx is None:
            return vec
        is_torch = isinstance(vec, torch.Tensor)
        is_seq = isinstance(vec, (list, tuple))
        if is_seq:
            return type(vec)(self._pack(v, idx, order, n_full) for v in vec)
        x = vec if is_torch else np.asarray(vec)
        ix = idx if is_torch and x.is_cuda else (idx.cpu().numpy() if isinstance(idx, torch.Tensor) else idx)
        if is_torch and not x.is_cuda:
            ix = torch.as_tensor(ix)
        if x.ndim == 1:
            return x[ix]
        if order.upper() == 'F':
            return x[ix, :]
        return x.reshape(-1, n_full)[:, ix]

    def _unpack(self, vec, idx, order, n_full):
        if idx is None:
            return vec
        is_torch = isinstance(vec, torch.Tensor)
        if isinstance(vec, (list, tuple)):
            return type(vec)(self._unpack(v, idx, order, n_full) for v in vec)
        x = vec if is_torch else np.asarray(vec)
        if is_torch:
            ix = idx.to(x.device)
            if x.ndim == 1:
                out = torch.zeros(n_full, dtype=x.dtype, device=x.device)
                out[ix] = x
            elif order.upper() == 'F':
                out = torch.zeros((n_full, x.shape[1]), dtype=x.dtype, device=x.device)
                out[ix, :] = x
            else:
                out = torch.zeros((x.shape[0], n_full), dtype=x.dtype, device=x.device)
                out[:, ix] = x
            return out
        ix = idx.cpu().numpy() if isinstance(idx, torch.Tensor) else idx
        if x.ndim == 1:
            out = np.zeros(n_full, dtype=x.dtype)
            out[ix] = x
        elif order.upper() == 'F':
            out = np.zeros((n_full, x.shape[1]), dtype=x.dtype)
            out[ix, :] = x
        else:
            out = np.zeros((x.shape[0], n_full), dtype=x.dtype)
            out[:, ix] = x
        return out

    def pack_csf(self, csfvec, order='C'):
        """csfstring.py:74-79: full CSF vector(s) -> the CSFs of irrep wfnsym."""
        return self._pack(csfvec, self.idx_sym, order, self._ncsf)

    def unpack_csf(self, csfvec, order='C'):
        """csfstring.py:81-86: packed symmetric CSF vector(s) -> full, zeros
        elsewhere."""
        return self._unpack(csfvec, self.idx_sym, order, self._ncsf)

    def _idx_sym_det(self):
        cs = self._conf_selected()
        if cs is None:
            return None
        return cs[self.econf_det_mask.long()]

    def pack_det(self, detvec, order='C'):
        """csfstring.py:88-96: determinant vector(s) -> the determinants whose
        configuration has irrep wfnsym."""
        if isinstance(detvec, (np.ndarray, torch.Tensor)) and tuple(detvec.shape[-2:]) == (self.ndeta, self.ndetb):
            detvec = detvec.reshape(-1, self.ndet)
            if detvec.shape[0] == 1:
                detvec = detvec[0]
        return self._pack(detvec, self._idx_sym_det(), order, self.ndet)

    def unpack_det(self, detvec, order='C'):
        """csfstring.py:98-103."""
        return self._unpack(detvec, self._idx_sym_det(), order, self.ndet)

    # ---- properties (setting one triggers a cache update) ---------------
    @property
    def norb(self):
        return self._norb

    @norb.setter
    def norb(self, x):
        self._update_spin_cache(x, self._neleca, self._nelecb, self._smult)

    @property
    def neleca(self):
        return self._neleca

    @neleca.setter
    def neleca(self, x):
        self._update_spin_cache(self._norb, x, self._nelecb, self._smult)

    @property
    def nelecb(self):
        return self._nelecb

    @nelecb.setter
    def nelecb(self, x):
        self._update_spin_cache(self._norb, self._neleca, x, self._smult)

    @property
    def smult(self):
        return self._smult

    @smult.setter
    def smult(self, x):
        self._update_spin_cache(self._norb, self._neleca, self._nelecb, x)

    @property
    def orbsym(self):
        return self._orbsym

    @orbsym.setter
    def orbsym(self, x):
        self._update_symm_cache(x)

    @property
    def ndeta(self):
        return comb(self._norb, self._neleca)

    @property
    def ndetb(self):
        return comb(self._norb, self._nelecb)

    @property
    def ndet(self):
        return self.ndeta * self.ndetb

    @property
    def ncsf(self):
        """csfstring.py:205-208: the number of CSFs of irrep wfnsym when
        point-group symmetry is set, else of all CSFs."""
        st = self._sym()
        return self._ncsf if st is None else st["ncsf"]

    def print_config(self, printer=print):
        printer('***** CSFTransformer configuration *****')
        printer('norb = {}'.format(self.norb))
        printer('neleca, nelecb = {}, {}'.format(self.neleca, self.nelecb))
        printer('smult = {}'.format(self.smult))
        printer('orbsym = {}'.format(self.orbsym))
        printer('wfnsym = {}'.format(self.wfnsym))
        printer('ndeta, ndetb = {}, {}'.format(self.ndeta, self.ndetb))
        printer('ncsf = {}'.format(self.ncsf))


def gen_strs_irrep(strs, orbsym):
    """Irrep of each occupation string: the XOR of the irreps of its
    occupied orbitals (the direct product in D2h and its subgroups, PySCF
    irrep ids), as direct_spin1_symm._gen_strs_irrep is used at
    csfstring.py:280-285."""
    orbsym = torch.as_tensor(np.asarray(orbsym, dtype=np.int64), device=strs.device)
    out = torch.zeros(strs.shape, dtype=torch.int64, device=strs.device)
    for p in range(orbsym.numel()):
        out ^= ((strs >> p) & 1) * orbsym[p]
    return out


def make_confsym(norb, neleca, nelecb, econf_det_mask, orbsym):
    """csfstring.py:278-290: irrep of every electron configuration (all
    determinants of a configuration share it), as a device int64 tensor
    indexed by configuration."""
    if np.any(np.asarray(orbsym) > 7):
        raise NotImplementedError('High-momentum point groups in Dooh/Coov')
    dev = econf_det_mask.device
    na, nb = comb(norb, neleca), comb(norb, nelecb)
    stra = torch.empty(na, dtype=torch.int64, device=dev)
    _capi.call("csffci_gen_strings", norb, neleca, ptr(stra), stream())
    strb = stra
    if nelecb != neleca:
        strb = torch.empty(nb, dtype=torch.int64, device=dev)
        _capi.call("csffci_gen_strings", norb, nelecb, ptr(strb), stream())
    ia = gen_strs_irrep(stra, orbsym)
    ib = gen_strs_irrep(strb, orbsym)
    detsym = (ia[:, None] ^ ib[None, :]).reshape(-1)
    nconf = int(econf_det_mask.max().item()) + 1 if econf_det_mask.numel() else 0
    confsym = torch.zeros(nconf, dtype=torch.int64, device=dev)
    confsym[econf_det_mask.long()] = detsym
    return confsym


def make_confgas(norb, neleca, nelecb, econf_det_mask, gas):
    """Per configuration, 1 when its total occupation per GAS subspace is one
    of the supergroups of gas = (subspace sizes, supergroup rows), else 0
    (csffci_gas_conf_mask), as a device uint8 tensor indexed by
    configuration."""
    orbs, sg = gas
    dev = econf_det_mask.device
    nconf = int(econf_det_mask.max().item()) + 1 if econf_det_mask.numel() else 0
    out = torch.zeros(max(nconf, 1), dtype=torch.uint8, device=dev)
    norbs = np.ascontiguousarray(orbs, dtype=np.int32)
    rows = np.ascontiguousarray(sg, dtype=np.int32)
    _capi.call("csffci_gas_conf_mask", norb, neleca, nelecb, ptr(econf_det_mask), len(orbs),
               norbs.ctypes.data, rows.shape[0], rows.ctypes.data, ptr(out), stream())
    return out[:nconf]


def make_econf_csf_mask(norb, neleca, nelecb, smult):
    """csfstring.py:789-804 on the device."""
    n = count_all_csfs(norb, neleca, nelecb, smult)
    mask = torch.empty(max(n, 1), dtype=torch.int32, device=device())
    _capi.call("csffci_csd_masks", norb, neleca, nelecb, smult, None, None, ptr(mask), stream())
    return mask[:n]


def transform_civec_det2csf(detarr, norb, neleca, nelecb, smult, csd_mask=None, vec_on_cols=False,
                            do_normalize=True, max_memory=None):
    t = CSFTransformer(norb, neleca, nelecb, smult)
    return t._transform(detarr, 'F' if vec_on_cols else 'C', do_normalize, reverse=False)


def transform_civec_csf2det(csfarr, norb, neleca, nelecb, smult, csd_mask=None, vec_on_cols=False,
                            do_normalize=True, max_memory=None):
    t = CSFTransformer(norb, neleca, nelecb, smult)
    return t._transform(csfarr, 'F' if vec_on_cols else 'C', do_normalize, reverse=True)
