"""GAS-restricted CSF spaces.

The reference restricts its determinant GAS solver (pyscf/mcscf/fci_gas.py)
through a canonical set of spin-supergroups (pyscf/mcscf/addons_gas.py:
318-700): rows (alpha occupation of each GAS subspace, beta occupation of
each subspace).  When that set is spin complete (addons_gas.py:782-798:
every alpha/beta split of every retained total-occupation row is present),
the determinant space is a union of whole electron configurations, so on the
CSF basis the restriction is a filter on configurations: a configuration is
kept when its total occupation per subspace is one of the spin-free
supergroups.  The 'supergroup', 'cumulative-occ' and 'ras' restriction types
are spin complete by construction; a 'spin-supergroup' set has to be.

This module restates the reference's normalisation of the four restriction
types (same canonical row order, same validation), and reduces a restriction
to (subspace sizes, spin-free supergroups) for the device filter
(csffci_gas_conf_mask).
"""
from functools import lru_cache
from math import comb

import numpy as np

from ..fci.direct_spin1 import _unpack_nelec

GAS_RESTR_SPIN_SUPERGROUP = "spin-supergroup"
GAS_RESTR_SUPERGROUP = "supergroup"
GAS_RESTR_CUMULATIVE_OCC = "cumulative-occ"
GAS_RESTR_RAS = "ras"

# limits of the reference's C kernels (addons_gas.py:33-38)
GAS_MAX_ORB = 63
GAS_MAX_LOCAL_ORB = 31
GAS_MAX_NGAS = 15
# limits of the device filter (csffci_gas_conf_mask): 6-bit occupations of
# at most 10 subspaces packed into one 64-bit key, 1024 supergroups
GAS_DEVICE_MAX_NGAS = 10
GAS_DEVICE_MAX_SUPERGROUPS = 1024


def _is_int(v):
    return isinstance(v, (int, np.integer)) and not isinstance(v, (bool, np.bool_))


def _exact_int_array(values, label):
    """Integer array; floats and booleans are rejected (addons_gas.py:78-89)."""
    arr = np.asarray(values, dtype=object)
    if not all(_is_int(v) for v in arr.flat):
        raise TypeError("%s must contain integers" % label)
    return np.asarray(arr.astype(np.int64), dtype=np.int64)


def _int_vector(values, label, length=None):
    arr = _exact_int_array(values, label)
    if arr.ndim != 1 or (length is not None and arr.size != length):
        shape = "(%d,)" % length if length is not None else "one-dimensional"
        raise ValueError("%s must be %s" % (label, shape))
    return tuple(int(v) for v in arr)


def _canonical_rows(values, ncol, label):
    """Non-empty, unique, lexicographically sorted integer rows."""
    arr = _exact_int_array(values, label)
    if arr.ndim != 2 or arr.shape[1] != int(ncol):
        raise ValueError("%s must have shape (nrow, %d)" % (label, int(ncol)))
    if arr.shape[0] == 0:
        raise ValueError("%s must contain at least one row" % label)
    return np.ascontiguousarray(np.unique(arr, axis=0), dtype=np.int32)


def _check_orbs(gas_orbs, allow_empty=False):
    lo = 0 if allow_empty else 1
    if len(gas_orbs) == 0 or len(gas_orbs) > GAS_MAX_NGAS:
        raise ValueError("number of GAS spaces exceeds C kernel limit")
    if any(n < lo or n > GAS_MAX_LOCAL_ORB for n in gas_orbs):
        raise ValueError("each GAS space must have %d..31 orbitals" % lo)
    if sum(gas_orbs) <= 0:
        raise ValueError("at least one active orbital is required")
    if sum(gas_orbs) > GAS_MAX_ORB:
        raise ValueError("total active orbitals exceed 63")


def blocks_from_supergroups(gas_orbs, nelec, supergroups):
    """All alpha/beta splits of spin-free supergroup rows, as canonical
    spin-supergroup rows (alpha occupations, beta occupations); the role of
    addons_gas.blocks_from_supergroups (addons_gas.py:360-428)."""
    gas_orbs = _int_vector(gas_orbs, "gas_orbs")
    _check_orbs(gas_orbs)
    na, nb = _unpack_nelec(nelec)
    if na < 0 or nb < 0 or na > sum(gas_orbs) or nb > sum(gas_orbs):
        raise ValueError("invalid alpha/beta electron count")
    ngas = len(gas_orbs)
    sg = _canonical_rows(supergroups, ngas, "supergroups")
    cap = 2 * np.asarray(gas_orbs)
    if np.any(sg < 0):
        raise ValueError("supergroup occupations must be non-negative")
    if np.any(sg > cap):
        raise ValueError("supergroup occupation exceeds local GAS capacity")
    if np.any(sg.sum(axis=1) != na + nb):
        raise ValueError("every supergroup must sum to the requested electron count")
    rows = []
    for tot in sg:
        # alpha occupation of subspace g ranges over [max(0, n_g - norb_g), min(norb_g, n_g)]
        lo = [max(0, int(t) - n) for t, n in zip(tot, gas_orbs)]
        hi = [min(n, int(t)) for t, n in zip(tot, gas_orbs)]
        alpha = [0] * ngas

        def split(g, left):
            if g == ngas:
                if left == 0:
                    rows.append(alpha + [int(t) - a for t, a in zip(tot, alpha)])
                return
            rest_lo, rest_hi = sum(lo[g + 1:]), sum(hi[g + 1:])
            for a in range(max(lo[g], left - rest_hi), min(hi[g], left - rest_lo) + 1):
                alpha[g] = a
                split(g + 1, left - a)

        split(0, na)
    if not rows:
        raise ValueError("supergroups generate no legal spin-supergroups")
    return _canonical_rows(rows, 2 * ngas, "spin-supergroups")


def supergroups_from_cumulative_occ(gas_orbs, nelec, bounds, allow_empty=False):
    """Spin-free supergroups whose running occupation after subspace g lies
    in [bounds[g][0], bounds[g][1]] (addons_gas.py:431-524)."""
    gas_orbs = _int_vector(gas_orbs, "gas_orbs")
    _check_orbs(gas_orbs, allow_empty)
    na, nb = _unpack_nelec(nelec)
    ntot = na + nb
    if na < 0 or nb < 0 or na > sum(gas_orbs) or nb > sum(gas_orbs):
        raise ValueError("invalid alpha/beta electron count")
    ngas = len(gas_orbs)
    b = _exact_int_array(bounds, "cumulative occupation bounds")
    if b.ndim != 2 or b.shape != (ngas, 2):
        raise ValueError("cumulative occupation bounds must have shape (%d, 2)" % ngas)
    lower, upper = b[:, 0], b[:, 1]
    if np.any(lower < 0):
        raise ValueError("cumulative occupations must be non-negative")
    if np.any(lower > upper):
        raise ValueError("cumulative minimum exceeds maximum")
    if np.any(lower[1:] < lower[:-1]) or np.any(upper[1:] < upper[:-1]):
        raise ValueError("cumulative bounds must be non-decreasing")
    if np.any(upper > 2 * np.cumsum(gas_orbs)):
        raise ValueError("cumulative occupation exceeds orbital capacity")
    if np.any(upper > ntot):
        raise ValueError("cumulative occupation exceeds active electrons")
    if int(lower[-1]) != ntot or int(upper[-1]) != ntot:
        raise ValueError("the final cumulative bound must equal the active electron count")
    cap = [2 * n for n in gas_orbs]
    cap_after = [sum(cap[g + 1:]) for g in range(ngas)]

    def occ_range(g, run):
        return (max(0, int(lower[g]) - run, ntot - run - cap_after[g]),
                min(cap[g], int(upper[g]) - run, ntot - run))

    @lru_cache(maxsize=None)
    def reachable(g, run):
        if g == ngas:
            return run == ntot
        lo, hi = occ_range(g, run)
        return any(reachable(g + 1, run + k) for k in range(lo, hi + 1))

    rows, cur = [], [0] * ngas

    def walk(g, run):
        if g == ngas:
            if run == ntot:
                rows.append(list(cur))
            return
        lo, hi = occ_range(g, run)
        for k in range(lo, hi + 1):
            if reachable(g + 1, run + k):
                cur[g] = k
                walk(g + 1, run + k)

    walk(0, 0)
    if not rows:
        raise ValueError("cumulative bounds generate no legal supergroups")
    return _canonical_rows(rows, ngas, "supergroups")


def _ras_bounds(gas_orbs, nelec, gas_restr):
    """RAS1/RAS2/RAS3 with hole and particle limits as cumulative bounds
    (addons_gas.py:535-609)."""
    from collections.abc import Mapping
    if not isinstance(gas_restr, Mapping):
        raise TypeError("ras gas_restr must be a mapping with max_holes and max_particles")
    keys = set(gas_restr)
    if keys != {"max_holes", "max_particles"}:
        missing = {"max_holes", "max_particles"} - keys
        if missing:
            raise ValueError("missing RAS restriction keys: %s" % ", ".join(sorted(missing)))
        raise ValueError("unknown RAS restriction keys: %s" %
                         ", ".join(sorted(keys - {"max_holes", "max_particles"})))
    mh, mp = gas_restr["max_holes"], gas_restr["max_particles"]
    if not _is_int(mh):
        raise TypeError("max_holes must be an integer")
    if not _is_int(mp):
        raise TypeError("max_particles must be an integer")
    mh, mp = int(mh), int(mp)
    if mh < 0 or mp < 0:
        raise ValueError("RAS hole and particle limits must be non-negative")
    n1, n2, n3 = gas_orbs
    if mh > 2 * n1:
        raise ValueError("max_holes exceeds the RAS1 electron capacity")
    if mp > 2 * n3:
        raise ValueError("max_particles exceeds the RAS3 electron capacity")
    ntot = sum(_unpack_nelec(nelec))
    b = np.array([[max(0, 2 * n1 - mh), min(2 * n1, ntot)],
                  [max(0, ntot - mp), min(2 * (n1 + n2), ntot)],
                  [ntot, ntot]], dtype=np.int64)
    b[1, 0] = max(b[1, 0], b[0, 0])
    return b


def normalize_gas_spec(gas_orbs, nelec, gas_restr=None, gas_restr_type=GAS_RESTR_SPIN_SUPERGROUP):
    """(kernel subspace sizes, canonical spin-supergroup rows) of one public
    GAS specification, as addons_gas.normalize_gas_spec (addons_gas.py:
    653-700): empty RAS spaces are dropped from the kernel subspaces."""
    if not isinstance(gas_restr_type, str):
        raise TypeError("gas_restr_type must be a string")
    types = (GAS_RESTR_SPIN_SUPERGROUP, GAS_RESTR_SUPERGROUP, GAS_RESTR_CUMULATIVE_OCC, GAS_RESTR_RAS)
    if gas_restr_type not in types:
        raise NotImplementedError("unsupported gas_restr_type %r; supported types: %s" %
                                  (gas_restr_type, ", ".join(sorted(types))))
    user_orbs = _int_vector(gas_orbs, "gas_orbs", 3 if gas_restr_type == GAS_RESTR_RAS else None)
    na, nb = _unpack_nelec(nelec)
    if gas_restr is None:
        if gas_restr_type != GAS_RESTR_SPIN_SUPERGROUP:
            raise ValueError("gas_restr is required for gas_restr_type %r" % gas_restr_type)
        if len(user_orbs) != 1:
            raise ValueError("gas_restr is required for multi-space GAS")
        _check_orbs(user_orbs)
        return user_orbs, np.asarray([[na, nb]], dtype=np.int32)
    if gas_restr_type == GAS_RESTR_SPIN_SUPERGROUP:
        _check_orbs(user_orbs)
        return user_orbs, _canonical_rows(gas_restr, 2 * len(user_orbs), "spin-supergroups")
    if gas_restr_type == GAS_RESTR_SUPERGROUP:
        return user_orbs, blocks_from_supergroups(user_orbs, (na, nb), gas_restr)
    if gas_restr_type == GAS_RESTR_CUMULATIVE_OCC:
        sg = supergroups_from_cumulative_occ(user_orbs, (na, nb), gas_restr)
        return user_orbs, blocks_from_supergroups(user_orbs, (na, nb), sg)
    bounds = _ras_bounds(user_orbs, (na, nb), gas_restr)
    sg = supergroups_from_cumulative_occ(user_orbs, (na, nb), bounds, allow_empty=True)
    keep = np.asarray(user_orbs) > 0
    korbs = tuple(int(n) for n in np.asarray(user_orbs)[keep])
    ksg = _canonical_rows(sg[:, keep], len(korbs), "supergroups")
    return korbs, blocks_from_supergroups(korbs, (na, nb), ksg)


def is_spin_complete(gas_orbs, nelec, blocks):
    """Every alpha/beta split of every retained total-occupation row present
    (addons_gas.py:782-798)."""
    gas_orbs = _int_vector(gas_orbs, "gas_orbs")
    ngas = len(gas_orbs)
    blocks = _canonical_rows(blocks, 2 * ngas, "spin-supergroups")
    sg = np.unique(blocks[:, :ngas] + blocks[:, ngas:], axis=0)
    full = blocks_from_supergroups(gas_orbs, nelec, sg)
    return {tuple(r) for r in blocks.tolist()} == {tuple(r) for r in full.tolist()}


def spin_free_supergroups(gas_orbs, nelec, gas_restr=None, gas_restr_type=GAS_RESTR_SPIN_SUPERGROUP):
    """(kernel subspace sizes, spin-free supergroup rows) of a restriction
    that the CSF basis can represent; ValueError for a spin-supergroup set
    that is not spin complete (its determinant space mixes spin states)."""
    korbs, blocks = normalize_gas_spec(gas_orbs, nelec, gas_restr, gas_restr_type)
    ngas = len(korbs)
    if not is_spin_complete(korbs, nelec, blocks):
        raise ValueError("the spin-supergroup set is not spin complete: a CSF basis cannot represent it "
                         "(add every alpha/beta split of each total-occupation row)")
    sg = np.unique(blocks[:, :ngas] + blocks[:, ngas:], axis=0).astype(np.int32)
    return korbs, sg


def gas_ndet(gas_orbs, nelec, blocks):
    """Determinants of a spin-supergroup set: sum over rows of the products of
    the per-subspace string counts."""
    na, nb = _unpack_nelec(nelec)
    ngas = len(gas_orbs)
    tot = 0
    for r in np.asarray(blocks):
        a = 1
        for g in range(ngas):
            a *= comb(gas_orbs[g], int(r[g])) * comb(gas_orbs[g], int(r[ngas + g]))
        tot += a
    return tot


__all__ = ["GAS_RESTR_SPIN_SUPERGROUP", "GAS_RESTR_SUPERGROUP", "GAS_RESTR_CUMULATIVE_OCC", "GAS_RESTR_RAS",
           "normalize_gas_spec", "blocks_from_supergroups", "supergroups_from_cumulative_occ",
           "is_spin_complete", "spin_free_supergroups", "gas_ndet"]
