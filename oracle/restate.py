"""ORACLE / TEST INFRASTRUCTURE -- a CPU restatement of the reference's CSF-FCI
path in plain numpy.  It is the checker for the CUDA path and is never
imported by the product code (tests, ``__graft_entry__.smoke`` and the
CPU-baseline arm of ``bench.py`` only).

Each function cites the reference location whose behaviour it restates.
Functions that the reference takes from PySCF core (absent from the
reference tree and from this machine) are restated from the mathematics;
their parity is pinned either through the reference's own GAS C library
(``oracle/gasref.py``; pinned to PySCF direct_spin1 by
pyscf/mcscf/test/test_gasci.py:272-293,765-786) or, for the pspace Slater-
Condon build and the Davidson solver, through brute-force identities
(pyscf/csf_fci/test/test_csf.py:60-132) -- those two are "parity unpinned"
against PySCF itself.
"""
from functools import lru_cache
from math import comb

import numpy as np


# ---------------------------------------------------------------------------
# determinant strings (PySCF cistring semantics; in-repo twin
# pyscf/lib/mcscf/fci_string_gas.c:252-298)
# ---------------------------------------------------------------------------

def num_strings(norb, nelec):
    return comb(norb, nelec) if 0 <= nelec <= norb else 0


@lru_cache(maxsize=None)
def _gen_strings_cached(norb, nelec):
    if nelec == 0:
        return np.zeros(1, dtype=np.int64)
    import itertools
    # ascending integer order == colex order of the occupied sets
    out = [sum(1 << o for o in occ) for occ in itertools.combinations(range(norb), nelec)]
    return np.array(sorted(out), dtype=np.int64)


def gen_strings(norb, nelec):
    return _gen_strings_cached(norb, nelec).copy()


def strs2addr(norb, nelec, strs):
    """Colex rank: sum_i C(p_i, i) over set bits p_1<p_2<..., i=1..nelec
    (fci_string_gas.c:263-276)."""
    strs = np.asarray(strs, dtype=np.int64).reshape(-1)
    addr = np.zeros(strs.size, dtype=np.int64)
    for j, s in enumerate(strs.tolist()):
        a, i, p = 0, 1, 0
        while s:
            if s & 1:
                a += comb(p, i)
                i += 1
            s >>= 1
            p += 1
        addr[j] = a
    return addr


def addrs2str(norb, nelec, addrs):
    return gen_strings(norb, nelec)[np.asarray(addrs, dtype=np.int64)]


def _popcount(x):
    return bin(int(x)).count("1")


def link_table(norb, nelec):
    """[nstr, nlink, 4] (cre p, des q, target addr, sign) with rows ordered as
    fci_string_gas.c:1341-1382: for each occupied q ascending, (q,q) first,
    then every virtual p ascending.  sign = (-1)^(#occupied strictly between
    p and q) (fci_string_gas.c:252-258)."""
    strs = gen_strings(norb, nelec)
    nlink = nelec * (norb - nelec + 1)
    addr_of = {int(s): i for i, s in enumerate(strs.tolist())}
    tab = np.zeros((len(strs), nlink, 4), dtype=np.int64)
    for ia, s in enumerate(strs.tolist()):
        k = 0
        for q in range(norb):
            if not (s >> q) & 1:
                continue
            tab[ia, k] = (q, q, ia, 1)
            k += 1
            for p in range(norb):
                if (s >> p) & 1:
                    continue
                s1 = (s ^ (1 << q)) | (1 << p)
                lo, hi = min(p, q), max(p, q)
                mask = ((1 << hi) - 1) ^ ((1 << (lo + 1)) - 1)
                sign = -1 if _popcount(s & mask) & 1 else 1
                tab[ia, k] = (p, q, addr_of[s1], sign)
                k += 1
    return tab


# ---------------------------------------------------------------------------
# CSD ordering (pyscf/csf_fci/csdstring.py)
# ---------------------------------------------------------------------------

def get_csdaddrs_shape(norb, neleca, nelecb):
    """csdstring.py:233-275."""
    nless = min(neleca, nelecb)
    min_npair = max(0, neleca + nelecb - norb)
    pairs = range(min_npair, nless + 1)
    nspins = [neleca + nelecb - 2 * p for p in pairs]
    dconf = np.array([comb(norb, p) for p in pairs], dtype=np.int64)
    sconf = np.array([comb(norb - p, ns) for p, ns in zip(pairs, nspins)], dtype=np.int64)
    spins = np.array([comb(ns, (ns + neleca - nelecb) // 2) for ns in nspins], dtype=np.int64)
    sizes = dconf * sconf * spins
    offset = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    assert sizes.sum() == comb(norb, neleca) * comb(norb, nelecb)
    return min_npair, offset, dconf, sconf, spins


def csdstrs2ddstrs(norb, dconf_str, sconf_str, spins_str):
    """csfstring.c:48-83 (vectorised over strings)."""
    dconf_str = np.asarray(dconf_str, dtype=np.int64)
    sconf_str = np.asarray(sconf_str, dtype=np.int64)
    spins_str = np.asarray(spins_str, dtype=np.int64)
    n = dconf_str.size
    astr = np.zeros(n, dtype=np.int64)
    bstr = np.zeros(n, dtype=np.int64)
    isorb = np.zeros(n, dtype=np.int64)
    ispin = np.zeros(n, dtype=np.int64)
    for iorb in range(norb):
        bit = np.int64(1) << iorb
        dbl = (dconf_str & bit) != 0
        astr[dbl] |= bit
        bstr[dbl] |= bit
        nd = ~dbl
        occ = nd & (((sconf_str >> isorb) & 1) != 0)
        up = occ & (((spins_str >> ispin) & 1) != 0)
        astr[up] |= bit
        bstr[occ & ~up] |= bit
        ispin[occ] += 1
        isorb[nd] += 1
    return astr, bstr


def make_csd_mask(norb, neleca, nelecb):
    """csdstring.py:28-47: mask[idx_csd] = idx_dd (uint32)."""
    min_npair, offset, dconf, sconf, spins = get_csdaddrs_shape(norb, neleca, nelecb)
    nb = num_strings(norb, nelecb)
    parts = []
    for ip, npair in enumerate(range(min_npair, min(neleca, nelecb) + 1)):
        nspin = neleca + nelecb - 2 * npair
        nup = (nspin + neleca - nelecb) // 2
        d = gen_strings(norb, npair)
        s = gen_strings(norb - npair, nspin)
        u = gen_strings(nspin, nup)
        D, S, U = np.meshgrid(d, s, u, indexing="ij")
        a, b = csdstrs2ddstrs(norb, D.ravel(), S.ravel(), U.ravel())
        parts.append(strs2addr(norb, neleca, a) * nb + strs2addr(norb, nelecb, b))
    return np.concatenate(parts).astype(np.uint32)


def make_econf_det_mask(norb, neleca, nelecb, csd_mask):
    """csdstring.py:49-65."""
    min_npair, offset, dconf, sconf, spins = get_csdaddrs_shape(norb, neleca, nelecb)
    conf_size = dconf * sconf
    parts = []
    iconf = 0
    for ip in range(len(dconf)):
        parts.append(np.repeat(np.arange(iconf, iconf + conf_size[ip]), spins[ip]))
        iconf += conf_size[ip]
    mask_csd = np.concatenate(parts).astype(np.uint32)
    out = np.empty_like(mask_csd)
    out[np.asarray(csd_mask, dtype=np.int64)] = mask_csd
    return out


# ---------------------------------------------------------------------------
# genealogical CSFs (pyscf/csf_fci/csfstring.py, pyscf/lib/csf/csfstring.c)
# ---------------------------------------------------------------------------

def csf_gentable(nspin, smult):
    """csfstring.py:806-849."""
    assert (smult - 1) % 2 == nspin % 2
    if smult > nspin + 1:
        return np.zeros((1, 1), dtype=np.int64)
    n0 = (nspin - (smult - 1)) // 2
    n1 = (nspin + (smult - 1)) // 2
    g = np.zeros((n0 + 1, n1 + 1), dtype=np.int64)
    g[n0, n0:] = 1
    for i0 in range(n0, 0, -1):
        row = list(g[i0, i0:])
        row = [sum(row[i1:]) for i1 in range(len(row))]
        row = [row[0]] + row
        g[i0 - 1, i0 - 1:] = row
    return g


def count_csfs(nspin, smult):
    return int(csf_gentable(nspin, smult)[0, 0])


class ImpossibleCIvecError(RuntimeError):
    pass


class ImpossibleSpinError(ImpossibleCIvecError):
    pass


def get_csfvec_shape(norb, neleca, nelecb, smult):
    """csfstring.py:858-911."""
    nless = min(neleca, nelecb)
    if neleca > norb or nelecb > norb:
        raise ImpossibleCIvecError("({}e+{}e,{}o)".format(neleca, nelecb, norb))
    if abs(neleca - nelecb) > smult - 1:
        raise ImpossibleSpinError("impossible s/ms")
    min_npair = max(0, neleca + nelecb - norb)
    pairs = range(min_npair, nless + 1)
    nspins = [neleca + nelecb - 2 * p for p in pairs]
    if (smult - 1) > nspins[0]:
        raise ImpossibleSpinError("smult too large")
    dconf = np.array([comb(norb, p) for p in pairs], dtype=np.int64)
    sconf = np.array([comb(norb - p, ns) for p, ns in zip(pairs, nspins)], dtype=np.int64)
    ncsf = np.array([count_csfs(ns, smult) for ns in nspins], dtype=np.int64)
    sizes = dconf * sconf * ncsf
    offset = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    return min_npair, offset, dconf, sconf, ncsf


def count_all_csfs(norb, neleca, nelecb, smult):
    _, _, a, b, c = get_csfvec_shape(norb, neleca, nelecb, smult)
    return int(np.sum(a * b * c))


def make_econf_csf_mask(norb, neleca, nelecb, smult):
    """csfstring.py:789-804."""
    min_npair, offset, dconf, sconf, ncsf = get_csfvec_shape(norb, neleca, nelecb, smult)
    parts = []
    iconf = 0
    for ip in range(len(dconf)):
        nconf = dconf[ip] * sconf[ip]
        parts.append(np.repeat(np.arange(iconf, iconf + nconf), ncsf[ip]))
        iconf += nconf
    return np.concatenate(parts).astype(np.uint32)


def strs_irrep(strs, orbsym):
    """Irrep of each occupation string for D2h-subgroup irrep ids: XOR of
    the irreps of the occupied orbitals (the role of
    direct_spin1_symm._gen_strs_irrep at csfstring.py:280-285)."""
    strs = np.asarray(strs, dtype=np.int64)
    out = np.zeros(strs.shape, dtype=np.int64)
    for p, s in enumerate((np.asarray(orbsym, dtype=np.int64) % 10).tolist()):
        out ^= ((strs >> p) & 1) * s
    return out


def make_confsym(norb, neleca, nelecb, econf_det_mask, orbsym):
    """csfstring.py:278-290: irrep of every configuration, read from one
    determinant of it (alpha-string irrep XOR beta-string irrep)."""
    ia = strs_irrep(gen_strings(norb, neleca), orbsym)
    ib = strs_irrep(gen_strings(norb, nelecb), orbsym)
    econf_det_mask = np.asarray(econf_det_mask, dtype=np.int64)
    nconf, addr = np.unique(econf_det_mask, return_index=True)
    nb = ib.size
    return ia[addr // nb] ^ ib[addr % nb]


def gas_allowed_dets(norb, neleca, nelecb, gas_orbs, blocks):
    """Determinants of a GAS space in full-CAS (alpha-major, colex) order:
    those whose (alpha occupation of each subspace, beta occupation of each
    subspace) is a row of the spin-supergroup set D -- the membership rule of
    the reference's GAS space, gas_space_from_blocks
    (pyscf/lib/mcscf/fci_string_gas.c:1683-1704) over the blocks of
    pyscf/mcscf/addons_gas.py:318-428, with subspace g the next gas_orbs[g]
    orbitals."""
    ngas = len(gas_orbs)
    starts = np.concatenate([[0], np.cumsum(gas_orbs)[:-1]]).astype(np.int64)
    masks = [((1 << int(n)) - 1) << int(st) for n, st in zip(gas_orbs, starts)]
    rows = {tuple(int(v) for v in r) for r in np.asarray(blocks)}

    def occ(strs):
        return np.array([[_popcount(int(st) & m) for m in masks] for st in strs], dtype=np.int64)

    oa = occ(gen_strings(norb, neleca))
    ob = occ(gen_strings(norb, nelecb))
    out = np.zeros((oa.shape[0], ob.shape[0]), dtype=bool)
    for i in range(oa.shape[0]):
        for j in range(ob.shape[0]):
            out[i, j] = tuple(oa[i].tolist() + ob[j].tolist()) in rows
    assert len(next(iter(rows))) == 2 * ngas
    return out


def make_confgas(econf_det_mask, allowed_dets):
    """Per configuration, whether its determinants are in the GAS space (for
    a spin-complete set all determinants of a configuration agree)."""
    econf = np.asarray(econf_det_mask, dtype=np.int64).ravel()
    allowed = np.asarray(allowed_dets, dtype=bool).ravel()
    nconf = int(econf.max()) + 1
    hit = np.zeros(nconf, dtype=np.int64)
    tot = np.zeros(nconf, dtype=np.int64)
    np.add.at(hit, econf, allowed.astype(np.int64))
    np.add.at(tot, econf, 1)
    assert np.all((hit == 0) | (hit == tot)), "GAS set is not a union of configurations"
    return hit > 0


def gen_addrs2str(nspin, smult, addrs):
    """csfstring.c:243-293 (coupling string of a genealogical address)."""
    g = csf_gentable(nspin, smult)
    twoS = smult - 1
    n1 = (nspin + twoS) // 2
    out = np.zeros(len(addrs), dtype=np.int64)
    for j, a in enumerate(np.asarray(addrs).tolist()):
        s = 1
        i0 = i1 = 0
        for ispin in range(nspin):
            if i1 == n1:
                break
            elif g[i0, i1 + 1] <= a:
                a -= g[i0, i1 + 1]
                i0 += 1
            else:
                s |= 1 << ispin
                i1 += 1
        assert a == 0
        out[j] = s
    return out


def gen_strs2addr(nspin, smult, strs):
    """csfstring.c:192-240."""
    g = csf_gentable(nspin, smult)
    twoS = smult - 1
    n1 = (nspin + twoS) // 2
    out = np.zeros(len(strs), dtype=np.int64)
    for j, s in enumerate(np.asarray(strs).tolist()):
        a = 0
        i0 = i1 = 0
        for ispin in range(nspin):
            if (s >> ispin) & 1:
                i1 += 1
            else:
                if i1 < n1:
                    a += g[i0, i1 + 1]
                i0 += 1
        out[j] = a
    return out


def makecsf(detstrs, coupstrs, nspin, twoS, twoMS):
    """Clebsch-Gordan coefficients along the coupling path, restating
    csfstring.c:86-141 operation by operation (double arithmetic)."""
    umat = np.empty((len(detstrs), len(coupstrs)))
    for i, d in enumerate(np.asarray(detstrs).tolist()):
        for j, c in enumerate(np.asarray(coupstrs).tolist()):
            t2s = 1
            t2ms = 1 if d & 1 else -1
            num = 1.0
            den = 1.0
            sgn = 1
            osgn = -t2ms
            for ispin in range(1, nspin):
                sup = (c >> ispin) & 1
                msup = (d >> ispin) & 1
                if msup:
                    t2ms += 1
                    osgn *= -1
                else:
                    t2ms -= 1
                    sgn *= osgn
                num *= (t2s + t2ms + 1) if sup == msup else (t2s + 1 - t2ms)
                if num == 0:
                    break
                den *= (t2s + 1)
                if msup and not sup:
                    sgn *= -1
                num /= 2
                t2s += 1 if sup else -1
            umat[i, j] = 0.0 if num == 0 else sgn * np.sqrt(num / den)
    return umat


def get_spin_evecs(nspin, neleca, nelecb, smult):
    """csfstring.py:913-960."""
    na = (nspin + neleca - nelecb) // 2
    ndet = comb(nspin, na)
    ncsf = count_csfs(nspin, smult)
    spinstrs = addrs2str(nspin, na, np.arange(ndet))
    scstrs = gen_addrs2str(nspin, smult, np.arange(ncsf))
    return makecsf(spinstrs, scstrs, nspin, smult - 1, neleca - nelecb)


def _block_sign(npair, nelecb):
    """csfstring.py:623-627 / 762-766."""
    ncomm = npair * (npair - 1) // 2 + npair * max(0, nelecb - npair)
    return -1.0 if ncomm % 2 else 1.0


def transform_det2csf(x, norb, neleca, nelecb, smult, csd_mask=None, reverse=False):
    """_transform_det2csf (csfstring.py:569-674) for arrays (nvec, ndet) or
    (nvec, ncsf) when reverse; no normalisation."""
    if csd_mask is None:
        csd_mask = make_csd_mask(norb, neleca, nelecb)
    csd_mask = np.asarray(csd_mask, dtype=np.int64)
    min_npair, csd_off, dconf, sconf, spins = get_csdaddrs_shape(norb, neleca, nelecb)
    _, csf_off, _, _, ncsf_b = get_csfvec_shape(norb, neleca, nelecb, smult)
    ndet_all = comb(norb, neleca) * comb(norb, nelecb)
    ncsf_all = int(np.sum(dconf * sconf * ncsf_b))
    x = np.atleast_2d(np.asarray(x, dtype=np.float64))
    nrow = x.shape[0]
    out = np.zeros((nrow, ndet_all if reverse else ncsf_all))
    for ip, npair in enumerate(range(min_npair, min(neleca, nelecb) + 1)):
        ncsf = int(ncsf_b[ip])
        if ncsf == 0:
            continue
        nspin = neleca + nelecb - 2 * npair
        nconf = int(dconf[ip] * sconf[ip])
        ndet = int(spins[ip])
        det_addrs = csd_mask[csd_off[ip]:csd_off[ip] + nconf * ndet].reshape(nconf, ndet)
        umat = _block_sign(npair, nelecb) * get_spin_evecs(nspin, neleca, nelecb, smult)
        c0 = int(csf_off[ip])
        if not reverse:
            out[:, c0:c0 + nconf * ncsf] = np.tensordot(x[:, det_addrs], umat, axes=1).reshape(nrow, -1)
        else:
            xin = x[:, c0:c0 + nconf * ncsf].reshape(nrow, nconf, ncsf)
            out[:, det_addrs] = np.tensordot(xin, umat, axes=((2,), (1,)))
    return out


# ---------------------------------------------------------------------------
# integrals, diagonal, absorb_h1e
# ---------------------------------------------------------------------------

def pair_index(p, q):
    hi, lo = max(p, q), min(p, q)
    return hi * (hi + 1) // 2 + lo


def restore1(eri, norb):
    """Full (n,n,n,n) tensor from full / 4-fold (npair,npair) / 8-fold
    storage (the semantics of ao2mo.restore(1, ...))."""
    eri = np.asarray(eri, dtype=np.float64)
    n = norb
    npair = n * (n + 1) // 2
    if eri.size == n ** 4:
        return eri.reshape(n, n, n, n).copy()
    if eri.size == npair * (npair + 1) // 2 and eri.ndim == 1:
        e4 = np.zeros((npair, npair))
        iu = np.tril_indices(npair)
        e4[iu] = eri
        e4 = e4 + e4.T - np.diag(np.diag(e4))
        eri = e4
    eri = eri.reshape(npair, npair)
    idx = np.array([[pair_index(p, q) for q in range(n)] for p in range(n)])
    return eri[idx][:, :, idx]


def restore4(eri, norb):
    e = restore1(eri, norb)
    i, j = np.tril_indices(norb)
    return np.ascontiguousarray(e[i, j][:, i, j])


def absorb_h1e(h1e, eri, norb, nelec, fac=1.0):
    """Fold the one-electron operator into the two-electron one so that
    H = sum_{pq,rs} h2e[pq,rs] E_pq E_rs (restated from the identity
    E_pq = E_pq N / N, with f = h - 1/2 sum_k (pk|kq)); returns the 4-fold
    (npair, npair) matrix scaled by fac.  Role of direct_spin1.absorb_h1e
    called at pyscf/csf_fci/csf.py:445,520."""
    if not isinstance(nelec, (int, np.integer)):
        nelec = sum(nelec)
    h2e = restore1(eri, norb)
    f1e = np.asarray(h1e, dtype=np.float64) - np.einsum("jiik->jk", h2e) * 0.5
    f1e = f1e * (1.0 / (nelec + 1e-100))
    for k in range(norb):
        h2e[k, k, :, :] += f1e
        h2e[:, :, k, k] += f1e
    return restore4(h2e, norb) * fac


def make_hdiag(h1e, eri, norb, nelec):
    """Determinant diagonal (direct_uhf.make_hdiag, called at csf.py:66-68)
    from Slater-Condon rules; h1e may be (2,n,n) = (alpha, beta)."""
    h1e = np.asarray(h1e, dtype=np.float64)
    ha, hb = (h1e[0], h1e[1]) if h1e.ndim == 3 else (h1e, h1e)
    e = restore1(eri, norb)
    J = np.einsum("iijj->ij", e)
    K = np.einsum("ijji->ij", e)
    na, nb = nelec
    sa = gen_strings(norb, na)
    sb = gen_strings(norb, nb)
    occ = lambda strs: (((strs[:, None] >> np.arange(norb)) & 1) != 0).astype(np.float64)
    oa, ob = occ(sa), occ(sb)
    ea = oa @ np.diag(ha) + 0.5 * np.einsum("ai,ij,aj->a", oa, J - K, oa)
    eb = ob @ np.diag(hb) + 0.5 * np.einsum("bi,ij,bj->b", ob, J - K, ob)
    cross = oa @ J @ ob.T
    return (ea[:, None] + eb[None, :] + cross).ravel()


def make_hdiag_csf(h1e, eri, norb, nelec, smult, hdiag_det=None, csd_mask=None):
    """csf.py:70-144 with the within-configuration blocks of
    csfstring.c:295-362 restated."""
    neleca, nelecb = nelec
    if hdiag_det is None:
        hdiag_det = make_hdiag(h1e, eri, norb, nelec)
    if csd_mask is None:
        csd_mask = make_csd_mask(norb, neleca, nelecb)
    csd_mask = np.asarray(csd_mask, dtype=np.int64)
    e = restore1(eri, norb)
    min_npair, csd_off, dconf, sconf, spins = get_csdaddrs_shape(norb, neleca, nelecb)
    _, csf_off, _, _, ncsf_b = get_csfvec_shape(norb, neleca, nelecb, smult)
    nb_all = num_strings(norb, nelecb)
    ncsf_all = int(np.sum(dconf * sconf * ncsf_b))
    out = np.zeros(ncsf_all)
    for ip, npair in enumerate(range(min_npair, min(neleca, nelecb) + 1)):
        ncsf = int(ncsf_b[ip])
        if ncsf == 0:
            continue
        nconf = int(dconf[ip] * sconf[ip])
        ndet = int(spins[ip])
        det_addr = csd_mask[csd_off[ip]:csd_off[ip] + nconf * ndet].reshape(nconf, ndet)
        c0 = int(csf_off[ip])
        if ndet == 1:
            out[c0:c0 + nconf] = hdiag_det[det_addr.ravel()]
            continue
        sa = addrs2str(norb, neleca, det_addr // nb_all)
        sb = addrs2str(norb, nelecb, det_addr % nb_all)
        H = np.zeros((nconf, ndet, ndet))
        for c in range(nconf):
            for x in range(ndet):
                H[c, x, x] = hdiag_det[det_addr[c, x]]
                for y in range(ndet):
                    if x == y:
                        continue
                    exc = int(sa[c, x]) ^ int(sa[c, y])
                    if _popcount(exc) != 2:
                        continue
                    somo = int(sa[c, x]) ^ int(sb[c, x])
                    p = (exc & -exc).bit_length() - 1
                    q = exc.bit_length() - 1
                    between = somo & (((1 << q) - 1) ^ ((1 << (p + 1)) - 1))
                    sgn = -1.0 if _popcount(between) & 1 else 1.0
                    H[c, x, y] = sgn * e[p, q, q, p]
        nspin = neleca + nelecb - 2 * npair
        U = get_spin_evecs(nspin, neleca, nelecb, smult)
        out[c0:c0 + nconf * ncsf] = np.einsum("cxy,xk,yk->ck", H, U, U).ravel()
    return out


# ---------------------------------------------------------------------------
# sigma, contract_1e, RDMs  (direct_spin1 semantics through link tables)
# ---------------------------------------------------------------------------

def _t_vectors(ci, norb, nelec, packed):
    """T[pq, J] = <J|E_pq|c> summed over both spins.  packed=True folds
    (p,q) and (q,p) into the triangular pair index (what a symmetric h2e
    needs); packed=False keeps all norb^2 ordered pairs."""
    na, nb = nelec
    la, lb = link_table(norb, na), link_table(norb, nb)
    Na, Nb = len(la), len(lb)
    c = np.asarray(ci, dtype=np.float64).reshape(Na, Nb)
    npq = norb * (norb + 1) // 2 if packed else norb * norb
    T = np.zeros((npq, Na, Nb))
    for ja in range(Na):
        for (a, i, ia, s) in la[ja]:
            idx = pair_index(a, i) if packed else i * norb + a
            T[idx, ja, :] += s * c[ia, :]
    for jb in range(Nb):
        for (a, i, ib, s) in lb[jb]:
            idx = pair_index(a, i) if packed else i * norb + a
            T[idx, :, jb] += s * c[:, ib]
    return T


def contract_2e(h2e, ci, norb, nelec):
    """sigma = sum_{pq,rs} h2e[pq,rs] E_pq E_rs c with h2e the absorbed
    4-fold pair matrix (role of direct_spin1.contract_2e at csf.py:449,526;
    pinned to the reference GAS sigma fci_contract_gas.c:2388-2452)."""
    na, nb = nelec
    la, lb = link_table(norb, na), link_table(norb, nb)
    Na, Nb = len(la), len(lb)
    h2e = restore4(h2e, norb)
    D = _t_vectors(ci, norb, nelec, packed=True)
    V = np.tensordot(h2e, D, axes=1)
    sig = np.zeros((Na, Nb))
    for ja in range(Na):
        for (a, i, ia, s) in la[ja]:
            sig[ia, :] += s * V[pair_index(a, i), ja, :]
    for jb in range(Nb):
        for (a, i, ib, s) in lb[jb]:
            sig[:, ib] += s * V[pair_index(a, i), :, jb]
    return sig.reshape(np.shape(ci))


def contract_1e_ab(h1a, h1b, ci, norb, nelec):
    """sum_pq h1a[p,q] Ea_pq c + h1b[p,q] Eb_pq c (direct_uhf.contract_1e as
    called at csf.py:527-528)."""
    na, nb = nelec
    la, lb = link_table(norb, na), link_table(norb, nb)
    Na, Nb = len(la), len(lb)
    c = np.asarray(ci, dtype=np.float64).reshape(Na, Nb)
    out = np.zeros((Na, Nb))
    for ja in range(Na):
        for (a, i, ia, s) in la[ja]:
            out[ia, :] += s * h1a[a, i] * c[ja, :]
    for jb in range(Nb):
        for (a, i, ib, s) in lb[jb]:
            out[:, ib] += s * h1b[a, i] * c[:, jb]
    return out.reshape(np.shape(ci))


def make_rdm12(bra, ket, norb, nelec):
    """dm1[p,q] = <bra|q+ p|ket>, dm2[p,q,r,s] = <bra|p+ r+ s q|ket>
    (conventions of pyscf/lib/mcscf/fci_gas.h:260-268), from
    <E_pq E_rs> = sum_J <bra|E_pq|J><J|E_rs|ket>."""
    Tb = _t_vectors(bra, norb, nelec, packed=False).reshape(norb, norb, -1)
    Tk = _t_vectors(ket, norb, nelec, packed=False).reshape(norb, norb, -1)
    # Tb[q,p,J] = <J|E_qp|bra> = <bra|E_pq|J>
    ee = np.einsum("qpJ,rsJ->pqrs", Tb, Tk)
    bra_v = np.asarray(bra).reshape(-1)
    dm1 = np.einsum("pqJ,J->qp", Tk, bra_v)  # <bra|E_pq|ket> placed at [q,p]
    dm2 = ee.copy()
    for q in range(norb):
        dm2[:, q, q, :] -= dm1.T  # delta_qr <E_ps> = dm1[s,p]
    return dm1, dm2


# ---------------------------------------------------------------------------
# pspace (csf.py:246-366) -- Slater-Condon restated (parity unpinned vs PySCF
# libfci; checked against brute force as in test_csf.py:125-132)
# ---------------------------------------------------------------------------

def _sc_element(e, ha, hb, a1, b1, a2, b2, norb):
    """<a1 b1|H|a2 b2> for distinct determinants (Slater-Condon)."""
    da = a1 ^ a2
    db = b1 ^ b2
    na_exc = _popcount(da) // 2
    nb_exc = _popcount(db) // 2
    if na_exc + nb_exc > 2:
        return 0.0

    def single(s_from, s_to):
        q = (s_from & ~s_to).bit_length() - 1  # annihilated
        p = (s_to & ~s_from).bit_length() - 1  # created
        lo, hi = min(p, q), max(p, q)
        mask = ((1 << hi) - 1) ^ ((1 << (lo + 1)) - 1)
        sgn = -1.0 if _popcount(s_from & mask) & 1 else 1.0
        return p, q, sgn

    occ = lambda s: [i for i in range(norb) if (s >> i) & 1]
    if na_exc == 1 and nb_exc == 0:
        p, q, sg = single(a2, a1)
        v = ha[p, q]
        for k in occ(a2):
            v += e[p, q, k, k] - e[p, k, k, q]
        for k in occ(b2):
            v += e[p, q, k, k]
        return sg * v
    if nb_exc == 1 and na_exc == 0:
        p, q, sg = single(b2, b1)
        v = hb[p, q]
        for k in occ(b2):
            v += e[p, q, k, k] - e[p, k, k, q]
        for k in occ(a2):
            v += e[p, q, k, k]
        return sg * v
    if na_exc == 1 and nb_exc == 1:
        p, q, s1 = single(a2, a1)
        r, s, s2 = single(b2, b1)
        return s1 * s2 * e[p, q, r, s]

    def double(s_from, s_to):
        qs = occ(s_from & ~s_to)
        ps = occ(s_to & ~s_from)
        # |to> = a+_p1 a+_p2 a_q2 a_q1 |from> phase computed stepwise
        q1, q2 = qs
        p1, p2 = ps
        st = s_from
        sgn = 1.0
        for (cre, des) in ((p1, q1), (p2, q2)):
            lo, hi = min(cre, des), max(cre, des)
            mask = ((1 << hi) - 1) ^ ((1 << (lo + 1)) - 1)
            if _popcount(st & mask) & 1:
                sgn = -sgn
            st = (st ^ (1 << des)) | (1 << cre)
        return p1, q1, p2, q2, sgn

    if na_exc == 2 or nb_exc == 2:
        s_from, s_to = (a2, a1) if na_exc == 2 else (b2, b1)
        p1, q1, p2, q2, sg = double(s_from, s_to)
        return sg * (e[p1, q1, p2, q2] - e[p1, q2, p2, q1])
    return 0.0


def pspace_h0_det(h1e, eri, norb, nelec, det_addr):
    """Full (symmetric) det-basis H among det_addr (role of
    libfci.FCIpspace_h0tril_uhf + hermi_triu, csf.py:313-326)."""
    h1e = np.asarray(h1e, dtype=np.float64)
    ha, hb = (h1e[0], h1e[1]) if h1e.ndim == 3 else (h1e, h1e)
    e = restore1(eri, norb)
    na, nb = nelec
    Nb = num_strings(norb, nb)
    sa = gen_strings(norb, na)
    sb = gen_strings(norb, nb)
    det_addr = np.asarray(det_addr, dtype=np.int64)
    hd = make_hdiag(h1e, eri, norb, nelec)
    n = len(det_addr)
    h0 = np.zeros((n, n))
    for i in range(n):
        ai, bi = divmod(int(det_addr[i]), Nb)
        h0[i, i] = hd[det_addr[i]]
        for j in range(i):
            aj, bj = divmod(int(det_addr[j]), Nb)
            v = _sc_element(e, ha, hb, int(sa[ai]), int(sb[bi]), int(sa[aj]), int(sb[bj]), norb)
            h0[i, j] = h0[j, i] = v
    return h0


# ---------------------------------------------------------------------------
# spin
# ---------------------------------------------------------------------------

def spin_square(ci, norb, nelec):
    """<S^2> and 2S+1 of a det-basis vector, from S^2 = Sz^2 + Sz + S- S+
    with S+ = sum_p a+_{p,alpha} a_{p,beta} (role of spin_op.spin_square0)."""
    na, nb = nelec
    c = np.asarray(ci, dtype=np.float64).reshape(num_strings(norb, na), num_strings(norb, nb))
    sz = 0.5 * (na - nb)
    if nb == 0:
        ss = sz * sz + sz
    else:
        sa = gen_strings(norb, na); sb = gen_strings(norb, nb)
        sa1 = gen_strings(norb, na + 1); sb1 = gen_strings(norb, nb - 1)
        addr_a1 = {int(s): i for i, s in enumerate(sa1.tolist())}
        addr_b1 = {int(s): i for i, s in enumerate(sb1.tolist())}
        sp = np.zeros((len(sa1), len(sb1)))
        for ia, a in enumerate(sa.tolist()):
            for ib, b in enumerate(sb.tolist()):
                v = c[ia, ib]
                if v == 0.0:
                    continue
                for p in range(norb):
                    if (b >> p) & 1 and not (a >> p) & 1:
                        # a+_{p a} a_{p b} |a b> ; ordering A'B': move a_pb past
                        # the remaining beta creators below p and the alpha string
                        sgn_b = (-1) ** _popcount(b & ((1 << p) - 1))
                        sgn_a = (-1) ** _popcount(a & ((1 << p) - 1))
                        sgn_pass = (-1) ** (_popcount(a))  # a_pb moves past all alpha creators
                        sgn = sgn_a * sgn_b * sgn_pass
                        sp[addr_a1[a | (1 << p)], addr_b1[b ^ (1 << p)]] += sgn * v
        ss = sz * sz + sz + float(np.sum(sp * sp))
    s = np.sqrt(ss + 0.25) - 0.5
    return ss, 2 * s + 1
