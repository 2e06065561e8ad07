"""CSF-basis FCI solver on the GPU with the API of pyscf.csf_fci.csf.

Mirrors pyscf/csf_fci/csf.py: ``kernel`` (368-497), ``CSFFCISolver``
(499-555), ``FCISolver`` (557-591), ``make_hdiag_csf`` (70-144), ``pspace``
(246-366), ``get_init_guess`` (51-64), including the reading of a
two-component h1e as (alpha, beta) split into charge and spin parts
(13-48).  Every vector operation runs on the device through
libcsffci_b200; results are handed back as numpy arrays when the caller
passed numpy (the PySCF convention) and as torch tensors otherwise.
"""
import time
from math import comb

import numpy as np
import torch

from .. import _capi
from .._runtime import device, eri_pair_matrix, like_input, ptr, require_cuda, stream, to_dev
from ..fci import direct_spin1
from ..fci.davidson import DiagPrecond, davidson, gram
from ..fci.direct_spin1 import _unpack_nelec
from . import gas as _gas
from .csfstring import CSFTransformer, count_all_csfs


def unpack_h1e_ab(h1e):
    """csf.py:28-32."""
    h = h1e.detach().cpu().numpy() if isinstance(h1e, torch.Tensor) else np.asarray(h1e)
    if h.ndim == 3 and h.shape[0] == 2:
        return h[0], h[1]
    return h, h


def unpack_h1e_cs(h1e):
    """csf.py:40-44: charge and spin parts."""
    ha, hb = unpack_h1e_ab(h1e)
    return (ha + hb) / 2.0, (ha - hb) / 2.0


class H2eff:
    """Absorbed two-electron Hamiltonian kept on the device, with the spin
    part of h1e attached (the role of tag_array(h2eff, h1e_s=...) at
    csf.py:518-523)."""

    def __init__(self, h2e, h1e_s=None):
        self.h2e = h2e
        self.h1e_s = None if h1e_s is None or not np.any(h1e_s) else np.asarray(h1e_s)

    def __array__(self, dtype=None, copy=None):
        a = self.h2e.cpu().numpy()
        return a if dtype is None else a.astype(dtype)


def make_hdiag_det(fci, h1e, eri, norb, nelec):
    """csf.py:66-68 (two-component h1e)."""
    ha, hb = unpack_h1e_ab(h1e)
    return direct_spin1.dev_make_hdiag(ha, hb, eri_pair_matrix(eri, norb), norb, _unpack_nelec(nelec))


def make_hdiag_csf(h1e, eri, norb, nelec, transformer, hdiag_det=None, max_memory=None):
    """csf.py:70-144, computed configuration by configuration on the device
    (no (nconf, ndet, ndet) blocks are materialised, so no MemoryError path
    is needed)."""
    eri4 = to_dev(eri_pair_matrix(eri, norb))
    if hdiag_det is None:
        hdiag_det = make_hdiag_det(None, h1e, eri, norb, nelec)
    return transformer.dev_hdiag_csf(to_dev(hdiag_det).reshape(-1), eri4)


def _block_of_conf(transformer):
    """(first configuration, block) table for configuration lookups."""
    out = []
    c0 = 0
    for b in transformer._blocks:
        out.append((c0, b))
        c0 += b["nconf"]
    return out


def _pspace_transform(transformer, mat, confs):
    """transform_opmat_det2csf_pspace (csfstring.py:676-785): U^T mat U with
    U block-diagonal over the configurations, rows = determinants of the
    configurations in CSD order, columns = their CSFs (ascending).  U is
    assembled on the device from the cached spin-eigenvector blocks (one
    slice copy per configuration), so no block leaves the GPU."""
    confs = np.sort(np.asarray(confs, dtype=np.int64))
    table = _block_of_conf(transformer)
    pieces = []
    det_pos = 0
    ncol = 0
    csf_addrs = []
    for conf in confs.tolist():
        c0, b = next((c0, b) for (c0, b) in reversed(table) if c0 <= conf)
        local = conf - c0
        nd, nc = b["ndet"], b["ncsf"]
        if nc > 0:
            pieces.append((det_pos, ncol, b))
            csf_addrs.extend(range(b["csf_offset"] + local * nc, b["csf_offset"] + (local + 1) * nc))
            ncol += nc
        det_pos += nd
    U = torch.zeros((det_pos, ncol), dtype=torch.float64, device=device())
    for r0, k0, b in pieces:
        blk = U[r0:r0 + b["ndet"], k0:k0 + b["ncsf"]]
        blk.copy_(b["umat"])
        blk.mul_(float(b["sign"]))
    h0 = to_dev(mat)
    Ut = U.T.contiguous()
    Wt = gram(Ut, h0)        # (ncsf, ndet) = U^T h0 (h0 symmetric)
    out = gram(Ut, Wt)       # (ncsf, ncsf) = U^T h0 U
    return out, np.asarray(csf_addrs, dtype=np.int64)


def _conf_dets(transformer, confs):
    """Determinant addresses of every configuration in confs (sorted), in
    CSD order within each (ascending determinant address, as asserted at
    csfstring.py:735)."""
    table = _block_of_conf(transformer)
    pieces = []
    for conf in np.sort(np.asarray(confs, dtype=np.int64)).tolist():
        c0, b = next((c0, b) for (c0, b) in reversed(table) if c0 <= conf)
        s = b["csd_offset"] + (conf - c0) * b["ndet"]
        pieces.append(transformer.csd_mask[s:s + b["ndet"]])
    return torch.cat(pieces).contiguous() if pieces else transformer.csd_mask[:0]


def pspace(fci, h1e, eri, norb, nelec, transformer, hdiag_det=None, hdiag_csf=None, npsp=200,
           max_memory=None):
    """csf.py:246-366: the lowest-diagonal CSFs, completed to whole
    configurations, with H built over their determinants by Slater-Condon
    rules and transformed to the CSF basis.  max_memory (MB; default
    fci.max_memory) bounds the p-space matrices as at csf.py:294-303:
    MemoryError when 1.2 * 8 * (npsp_det + npsp_csf)^2 bytes exceed it (here
    the matrices live in device memory, so the budget is the device buffer's,
    not the host process's growth)."""
    if norb > 63:
        raise NotImplementedError('norb > 63')
    if max_memory is None:
        max_memory = getattr(fci, 'max_memory', None)
    neleca, nelecb = _unpack_nelec(nelec)
    eri4 = to_dev(eri_pair_matrix(eri, norb))
    if hdiag_det is None:
        hdiag_det = make_hdiag_det(fci, h1e, eri, norb, nelec)
    hdiag_det = to_dev(hdiag_det).reshape(-1)
    if hdiag_csf is None:
        hdiag_csf = make_hdiag_csf(h1e, eri, norb, nelec, transformer, hdiag_det=hdiag_det)
    hdiag_csf = to_dev(hdiag_csf).reshape(-1)
    npsp = int(npsp)
    # candidates: every CSF, or those of the irrep wfnsym (csf.py:266-271);
    # addresses stay in the full CSF numbering, as the reference returns them
    idx_sym = transformer.idx_sym
    cand = torch.arange(hdiag_csf.numel(), device=hdiag_csf.device)
    if idx_sym is not None:
        cand = cand[idx_sym]
    ncsf = cand.numel()
    if ncsf > npsp:
        csf_addr = cand[torch.argsort(hdiag_csf[cand], stable=True)[:npsp]]
    else:
        csf_addr = cand
    npsp_csf = csf_addr.numel()
    econf = torch.unique(transformer.econf_csf_mask[csf_addr].long()).cpu().numpy()
    det_addr = _conf_dets(transformer, econf)
    n = det_addr.numel()
    mem_h0 = 1.2 * (n + npsp_csf) ** 2.0 * 8 / 1e6
    if max_memory is not None and mem_h0 > max_memory:
        raise MemoryError("pspace_size of {} CSFs -> {} determinants requires {} MB, cf {} MB "
                          "remaining memory".format(npsp_csf, n, mem_h0, max_memory))
    ha, hb = unpack_h1e_ab(h1e)
    h1a, h1b = to_dev(ha), to_dev(hb)
    h0 = torch.empty((n, n), dtype=torch.float64, device=device())
    _capi.call("csffci_pspace_h0", norb, neleca, nelecb, ptr(h1a), ptr(h1b), ptr(eri4),
               ptr(hdiag_det), ptr(det_addr), n, ptr(h0), stream())
    h0c, addr = _pspace_transform(transformer, h0, econf)
    if addr.size > npsp_csf:
        keep = torch.argsort(torch.diagonal(h0c), stable=True)[:npsp_csf].cpu().numpy()
        addr = addr[keep]
        h0c = h0c[torch.as_tensor(keep, device=h0c.device)][:, torch.as_tensor(keep, device=h0c.device)]
    return addr, h0c.cpu().numpy()


def get_init_guess(norb, nelec, nroots, hdiag_csf, transformer):
    """csf.py:51-64: unit vectors on the lowest diagonal CSFs (CSF basis,
    device; the packed symmetric CSF basis when the transformer has a
    point group, from the full diagonal)."""
    hd = to_dev(hdiag_csf).reshape(-1)
    if transformer.idx_sym is not None and hd.numel() != transformer.ncsf:
        hd = transformer.pack_csf(hd)
    ncsf = hd.numel()
    assert ncsf >= nroots, "Can't find {} roots among only {} CSFs".format(nroots, ncsf)
    addr = torch.argsort(hd, stable=True)[:nroots]
    x = torch.zeros((nroots, ncsf), dtype=torch.float64, device=hd.device)
    x[torch.arange(nroots, device=hd.device), addr] = 1.0
    return x


class _Hop:
    """x (k, ncsf) -> H x in the CSF basis:
    csf2det -> sigma (+ spin part of h1e) -> det2csf (csf.py:447-450)."""

    def __init__(self, transformer, h2eff, norb, nelec, deterministic=False):
        self.t = transformer
        self.h2e = h2eff.h2e
        self.h1e_s = h2eff.h1e_s
        self.norb = norb
        self.nelec = nelec
        self.eta = transformer.spin_parity
        self.deterministic = bool(deterministic)
        self.nsigma = 0

    def __call__(self, x):
        x = x.reshape(-1, self.t.ncsf)
        xd = self.t.dev_csf2det(x)
        hx = torch.empty_like(xd)
        for i in range(xd.shape[0]):
            direct_spin1.dev_contract_2e(self.h2e, xd[i], self.norb, self.nelec, eta=self.eta,
                                         out=hx[i], deterministic=self.deterministic)
            if self.h1e_s is not None:
                direct_spin1.dev_contract_1e(self.h1e_s, -self.h1e_s, xd[i], self.norb, self.nelec,
                                             hx[i])
            self.nsigma += 1
        return self.t.dev_det2csf(hx)


def kernel(fci, h1e, eri, norb, nelec, smult=None, idx_sym=None, ci0=None, tol=None, lindep=None,
           max_cycle=None, max_space=None, nroots=None, davidson_only=None, pspace_size=None,
           max_memory=None, orbsym=None, wfnsym=None, ecore=0, transformer=None, **kwargs):
    """csf.py:368-497."""
    require_cuda()
    kwargs.pop('verbose', None)
    if nroots is None:
        nroots = fci.nroots
    if pspace_size is None:
        pspace_size = fci.pspace_size
    if davidson_only is None:
        davidson_only = fci.davidson_only
    if transformer is None:
        transformer = fci.transformer
    nelec = _unpack_nelec(nelec, fci.spin)
    neleca, nelecb = nelec
    t0 = time.perf_counter()
    hdiag_det = make_hdiag_det(fci, h1e, eri, norb, nelec)
    hdiag_csf = make_hdiag_csf(h1e, eri, norb, nelec, transformer, hdiag_det=hdiag_det)
    ncsf_all = count_all_csfs(norb, neleca, nelecb, smult)
    if idx_sym is None:
        idx_sym = transformer.idx_sym
    if idx_sym is None:
        ncsf_sym = ncsf_all
        pos = None
    else:
        # Davidson runs in the packed space of the CSFs of irrep wfnsym
        # (csf.py:391-394, 431-437); pos maps full CSF addresses to it
        idx_sym = to_dev(idx_sym).to(torch.bool)
        ncsf_sym = int(idx_sym.sum().item())
        pos = (torch.cumsum(idx_sym.to(torch.int64), 0) - 1).cpu().numpy()
    assert ncsf_sym > 0, "Can't find {} roots among only 0 CSFs".format(nroots)
    nroots = min(ncsf_sym, nroots)
    na, nb = comb(norb, neleca), comb(norb, nelecb)
    addr, h0 = fci.pspace(h1e, eri, norb, nelec, hdiag_det=hdiag_det, hdiag_csf=hdiag_csf,
                          npsp=max(pspace_size, nroots))
    if pspace_size > 0:
        pw, pv = np.linalg.eigh(h0)
    else:
        pw = pv = None

    if pspace_size >= ncsf_sym and not davidson_only:
        # csf.py:416-429: the p-space is the whole space (exact diagonalisation)
        fci.converged = [True] * nroots if nroots > 1 else True
        if ncsf_sym == 1:
            civec = transformer.dev_csf2det(torch.as_tensor(pv[:, 0].reshape(1, 1), device=device()))
            return pw[0] + ecore, civec.reshape(na, nb)
        order = np.argsort(addr)
        pv_full = np.zeros((ncsf_sym, pv.shape[1]))
        pv_full[addr if pos is None else pos[addr]] = pv
        if nroots > 1:
            civec = transformer.dev_csf2det(torch.as_tensor(pv_full[:, :nroots].T.copy(), device=device()))
            return pw[:nroots] + ecore, [c.reshape(na, nb) for c in civec]
        elif abs(pw[0] - pw[1]) > 1e-12:
            civec = transformer.dev_csf2det(torch.as_tensor(pv_full[:, :1].T.copy(), device=device()))
            return pw[0] + ecore, civec.reshape(na, nb)
        del order

    if pos is None:
        precond = fci.make_precond(hdiag_csf, pw, pv, addr)
    else:
        precond = fci.make_precond(to_dev(hdiag_csf).reshape(-1)[idx_sym], pw, pv, pos[addr])
    h2e = fci.absorb_h1e(h1e, eri, norb, nelec, .5)
    if not isinstance(h2e, H2eff):
        h2e = H2eff(to_dev(eri_pair_matrix(h2e, norb)))
    hop = _Hop(transformer, h2e, norb, nelec, deterministic=getattr(fci, 'deterministic_sigma', False))

    if ci0 is None:
        x0 = get_init_guess(norb, nelec, nroots, hdiag_csf, transformer)
    else:
        if isinstance(ci0, (list, tuple)):
            c = torch.stack([to_dev(v).reshape(-1) for v in ci0])
        else:
            c = to_dev(ci0).reshape(-1, na * nb)
        x0 = transformer.dev_det2csf(c)
        x0 = x0 / torch.linalg.norm(x0, dim=1, keepdim=True)

    if tol is None:
        tol = fci.conv_tol
    if lindep is None:
        lindep = fci.lindep
    if max_cycle is None:
        max_cycle = fci.max_cycle
    if max_space is None:
        max_space = fci.max_space
    tol_residual = getattr(fci, 'conv_tol_residual', None)
    log = print if getattr(fci, "verbose", 0) >= 5 else None
    stats = {}
    conv, e, c = davidson(hop, x0, precond, tol=tol, max_cycle=max_cycle, max_space=max_space,
                          lindep=lindep, nroots=nroots, follow_state=True,
                          tol_residual=tol_residual, log=log, stats=stats)
    fci.converged = conv if nroots > 1 else conv[0]
    fci.nsigma = hop.nsigma
    fci.niter = stats.get("niter", 0)
    fci.kernel_time = time.perf_counter() - t0
    cdet = transformer.dev_csf2det(c)
    cdet = cdet / torch.linalg.norm(cdet, dim=1, keepdim=True)
    if nroots > 1:
        return e + ecore, [ci.reshape(na, nb) for ci in cdet]
    return e[0] + ecore, cdet[0].reshape(na, nb)


class FCIBase:
    """Duck-typed stand-in for direct_spin1.FCISolver (the PySCF base class
    of csf.FCISolver, csf.py:557): solver attributes and the determinant-
    basis operations, all on the GPU."""

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
    stdout = None

    def __init__(self, mol=None):
        self.mol = mol
        self.converged = False
        self.norb = None
        self.nelec = None
        self.eci = None
        self.ci = None

    def check_sanity(self):
        return self

    def absorb_h1e(self, h1e, eri, norb, nelec, fac=1):
        return direct_spin1.absorb_h1e(h1e, eri, norb, nelec, fac)

    def contract_2e(self, eri, fcivec, norb, nelec, link_index=None, **kwargs):
        return direct_spin1.contract_2e(eri, fcivec, norb, nelec, link_index)

    def contract_1e(self, f1e, fcivec, norb, nelec, link_index=None, **kwargs):
        return direct_spin1.contract_1e(f1e, fcivec, norb, nelec, link_index)

    def make_hdiag(self, h1e, eri, norb, nelec, compress=False):
        return direct_spin1.make_hdiag(h1e, eri, norb, nelec)

    def make_precond(self, hdiag, pspaceig=None, pspaceci=None, addr=None):
        return DiagPrecond(to_dev(hdiag).reshape(-1), self.level_shift, pspaceig, pspaceci, addr)

    def make_rdm1(self, fcivec, norb, nelec, link_index=None):
        return direct_spin1.make_rdm1(fcivec, norb, nelec)

    def make_rdm12(self, fcivec, norb, nelec, link_index=None, reorder=True):
        return direct_spin1.make_rdm12(fcivec, norb, nelec)

    def trans_rdm1(self, cibra, ciket, norb, nelec, link_index=None):
        return direct_spin1.trans_rdm1(cibra, ciket, norb, nelec)

    def make_rdm1s(self, fcivec, norb, nelec, link_index=None):
        return direct_spin1.make_rdm1s(fcivec, norb, nelec)

    def make_rdm12s(self, fcivec, norb, nelec, link_index=None, reorder=True):
        return direct_spin1.make_rdm12s(fcivec, norb, nelec)

    def trans_rdm1s(self, cibra, ciket, norb, nelec, link_index=None):
        return direct_spin1.trans_rdm1s(cibra, ciket, norb, nelec)

    def trans_rdm12s(self, cibra, ciket, norb, nelec, link_index=None, reorder=True):
        return direct_spin1.trans_rdm12s(cibra, ciket, norb, nelec)

    def trans_rdm12(self, cibra, ciket, norb, nelec, link_index=None, reorder=True):
        return direct_spin1.trans_rdm12(cibra, ciket, norb, nelec)

    def energy(self, h1e, eri, fcivec, norb, nelec, link_index=None):
        return direct_spin1.energy(h1e, eri, fcivec, norb, nelec)

    def spin_square(self, fcivec, norb, nelec):
        """(<S^2>, 2S+1) per vector (fci.spin_op.spin_square0 semantics)."""
        from .spin_op import spin_square
        if isinstance(fcivec, (list, tuple)):
            res = [spin_square(c, norb, nelec) for c in fcivec]
            return [r[0] for r in res], [r[1] for r in res]
        return spin_square(fcivec, norb, nelec)


class CSFFCISolver:
    """csf.py:499-555.  With gas_orbs set, the CSF space is restricted to the
    configurations a GAS restriction allows (gas_orbs, gas_restr and
    gas_restr_type as the reference's GAS solver takes them,
    pyscf/mcscf/fci_gas.py:778-801; the restriction has to be spin
    complete, see csf_fci.gas)."""
    _keys = {'smult', 'transformer', 'gas_orbs', 'gas_restr', 'gas_restr_type', 'deterministic_sigma'}
    pspace_size = 200
    gas_orbs = None
    gas_restr = None
    gas_restr_type = _gas.GAS_RESTR_SPIN_SUPERGROUP
    # sigma with the deterministic scatter (CSFFCI_SIGMA_DETERMINISTIC,
    # 4 <= norb <= 16): reruns give bit-identical sigma vectors, energies
    # and CI vectors, at the cost of three integer atomics per scattered
    # element (in the host-driven loop and in the device-resident plan)
    deterministic_sigma = False

    def __init__(self, mol=None, smult=None):
        self.smult = smult
        self.transformer = None
        super().__init__(mol)

    def gas_spec(self, norb=None, nelec=None):
        """(subspace sizes, spin-free supergroups) of the GAS restriction for
        (norb, nelec), or None without one."""
        if self.gas_orbs is None:
            return None
        norb = self.norb if norb is None else norb
        nelec = _unpack_nelec(self.nelec if nelec is None else nelec)
        if sum(int(n) for n in self.gas_orbs) != int(norb):
            raise ValueError("sum(gas_orbs) must equal norb")
        return _gas.spin_free_supergroups(self.gas_orbs, nelec, self.gas_restr, self.gas_restr_type)

    def _apply_gas(self):
        self.transformer.gas = self.gas_spec()

    def make_hdiag(self, h1e, eri, norb, nelec, compress=False):
        out = make_hdiag_det(self, h1e, eri, norb, nelec)
        return out if isinstance(h1e, torch.Tensor) else out.cpu().numpy()

    def make_hdiag_csf(self, h1e, eri, norb, nelec, hdiag_det=None, smult=None, max_memory=None):
        self.norb = norb
        self.nelec = nelec
        if smult is not None:
            self.smult = smult
        self.check_transformer_cache()
        out = make_hdiag_csf(h1e, eri, norb, nelec, self.transformer, hdiag_det=hdiag_det)
        return out if isinstance(h1e, torch.Tensor) else out.cpu().numpy()

    def absorb_h1e(self, h1e, eri, norb, nelec, fac=1):
        h1e_c, h1e_s = unpack_h1e_cs(h1e)
        h2e = direct_spin1.dev_absorb_h1e(h1e_c, eri_pair_matrix(eri, norb), norb, nelec, fac)
        return H2eff(h2e, h1e_s)

    def contract_2e(self, eri, fcivec, norb, nelec, link_index=None, out=None, **kwargs):
        """csf.py:521-529.  out (optional, a contiguous float64 torch tensor
        with fcivec's size, on the device or in host memory) receives the
        result, which is then returned: a caller that reuses a pinned host
        buffer gets the result with one DMA copy and no allocation."""
        nelec = _unpack_nelec(nelec)
        if isinstance(eri, H2eff):
            h2e, h1e_s = eri.h2e, eri.h1e_s
        else:
            h2e, h1e_s = to_dev(eri_pair_matrix(eri, norb)), None
        ci = to_dev(fcivec).reshape(-1)
        if out is not None and (not isinstance(out, torch.Tensor) or out.numel() != ci.numel()
                                or out.dtype != torch.float64 or not out.is_contiguous()):
            raise ValueError("out must be a contiguous float64 torch tensor of the CI vector's size")
        eta = None
        if nelec[0] == nelec[1]:
            eta = direct_spin1.dev_spin_parity(ci, comb(norb, nelec[0]))
        dev_out = out.reshape(-1) if out is not None and out.is_cuda else None
        hc = direct_spin1.dev_contract_2e(h2e, ci, norb, nelec, eta=eta, out=dev_out,
                                          deterministic=self.deterministic_sigma)
        if h1e_s is not None:
            direct_spin1.dev_contract_1e(h1e_s, -h1e_s, ci, norb, nelec, hc)
        if out is not None:
            if not out.is_cuda:
                out.reshape(-1).copy_(hc)
            return out
        shape = fcivec.shape if hasattr(fcivec, "shape") else np.shape(fcivec)
        return like_input(hc.reshape(shape), fcivec)

    def pspace(self, h1e, eri, norb, nelec, hdiag_det=None, hdiag_csf=None, npsp=200, **kwargs):
        self.norb = norb
        self.nelec = nelec
        if 'smult' in kwargs:
            self.smult = kwargs.pop('smult')
        self.check_transformer_cache()
        return pspace(self, h1e, eri, norb, nelec, self.transformer, hdiag_det=hdiag_det,
                      hdiag_csf=hdiag_csf, npsp=npsp, max_memory=kwargs.get('max_memory', self.max_memory))

    def log_transformer_cache(self, tverbose=0, **kwargs):
        if len(kwargs):
            self.__dict__.update(kwargs)
            self.check_transformer_cache()
        if self.transformer is None:
            return
        if tverbose >= 10:
            self.transformer.print_config(print)

    def print_transformer_cache(self, **kwargs):
        return self.log_transformer_cache(10, **kwargs)


class FCISolver(CSFFCISolver, FCIBase):
    """csf.py:557-591: Davidson in the CSF basis, ci (and ci0) in the
    determinant basis."""

    def get_init_guess(self, norb, nelec, nroots, hdiag_csf, **kwargs):
        self.norb = norb
        self.nelec = nelec
        self.check_transformer_cache()
        x = get_init_guess(norb, nelec, nroots, hdiag_csf, self.transformer)
        return self.transformer.dev_csf2det(x)

    # One problem small enough that host round trips would dominate its
    # Davidson iterations runs them device-resident instead (the batched
    # solver's plan with one problem: every step on the device, one captured
    # iteration replayed as a CUDA graph).  Larger problems keep the
    # host-driven loop, whose sigma is the single-problem warp-specialised
    # kernel.  Set device_resident = False to always take the host loop.
    device_resident = True
    device_resident_max_ncsf = 2000000
    _DEVICE_KW = {'nroots', 'tol', 'lindep', 'max_cycle', 'max_space', 'pspace_size', 'davidson_only'}

    def _device_resident_ok(self, h1e, eri, norb, nelec, ci0, kwargs):
        if not self.device_resident or ci0 is not None or not set(kwargs) <= self._DEVICE_KW:
            return False
        if not isinstance(h1e, np.ndarray) or h1e.ndim != 2 or isinstance(eri, torch.Tensor):
            return False
        if kwargs.get('davidson_only', self.davidson_only):
            return False
        nroots = kwargs.get('nroots', self.nroots)
        t = self.transformer
        if t is None or t.gas is not None or t.idx_sym is not None or self.gas_orbs is not None:
            return False
        return 4 <= norb <= 16 and 1 <= nroots <= 8 and t.ncsf <= self.device_resident_max_ncsf

    def _kernel_device_resident(self, h1e, eri, norb, nelec, kwargs):
        from ..batched import BatchedCSFSolver, Problem
        nroots = min(int(kwargs.get('nroots', self.nroots)), self.transformer.ncsf)
        tol = kwargs.get('tol', self.conv_tol)
        sol = BatchedCSFSolver(conv_tol=tol, lindep=kwargs.get('lindep', self.lindep),
                               max_cycle=kwargs.get('max_cycle', self.max_cycle),
                               max_space=kwargs.get('max_space', self.max_space), level_shift=self.level_shift,
                               pspace_size=kwargs.get('pspace_size', self.pspace_size),
                               conv_tol_residual=getattr(self, 'conv_tol_residual', None),
                               autotune=False,  # the defaults are the single-problem shapes
                               deterministic=self.deterministic_sigma)
        p = Problem(norb, _unpack_nelec(nelec, self.spin), self.smult, nroots, h1e, eri)
        e, cis, _, conv = sol.kernel([p], with_rdm=False)[0]
        self.phase_s = dict(sol.phase_s)
        self.converged = conv if nroots == 1 else [conv] * nroots
        self.niter = int(sol.niter[0]) if sol.niter is not None else 0
        if nroots > 1:
            return np.asarray(e), cis
        return float(e[0]), cis[0]

    def kernel(self, h1e, eri, norb, nelec, ci0=None, **kwargs):
        kwargs.pop('max_memory', None)
        self.norb = norb
        self.nelec = nelec
        if 'smult' in kwargs:
            self.smult = kwargs.pop('smult')
        self.check_transformer_cache()
        if self._device_resident_ok(h1e, eri, norb, nelec, ci0, kwargs):
            e, c = self._kernel_device_resident(h1e, eri, norb, nelec, kwargs)
            self.eci, self.ci = e, c
            return e, c
        e, c = kernel(self, h1e, eri, norb, nelec, smult=self.smult, idx_sym=None, ci0=ci0,
                      transformer=self.transformer, **kwargs)
        as_torch = isinstance(h1e, torch.Tensor)
        if not as_torch:
            if isinstance(c, list):
                c = [ci.cpu().numpy() for ci in c]
            else:
                c = c.cpu().numpy()
        self.eci, self.ci = e, c
        return e, c

    def check_transformer_cache(self):
        assert isinstance(self.smult, (int, np.integer))
        neleca, nelecb = _unpack_nelec(self.nelec)
        if self.transformer is None:
            self.transformer = CSFTransformer(self.norb, neleca, nelecb, self.smult,
                                              max_memory=self.max_memory)
        else:
            self.transformer.gas = None
            self.transformer._update_spin_cache(self.norb, neleca, nelecb, self.smult)
        self._apply_gas()
