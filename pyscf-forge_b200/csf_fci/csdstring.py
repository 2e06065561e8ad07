"""Configuration-spin-determinant (CSD) ordering: shape bookkeeping on the
host, the permutation itself on the device.

Mirrors pyscf/csf_fci/csdstring.py.  The CSD order runs, slowest to
fastest, over the number of electron pairs, the doubly-occupied
configuration, the singly-occupied configuration in the remaining
orbitals and the up-spin pattern of the unpaired electrons, each in
colex order (csdstring.py:10-14).
"""
from math import comb

import numpy as np
import torch

from .. import _capi
from .._runtime import device, ptr, stream


def check_csd_mask_size(norb, neleca, nelecb):
    """csdstring.py:16-26: determinant addressing is 32-bit."""
    mask_size = comb(norb, neleca) * comb(norb, nelecb)
    assert mask_size <= 2 ** 32, "{:.2f} billion determinants; more than {:.2f} billion not supported".format(
        mask_size / 1e9, 2 ** 32 / 1e9)
    return mask_size


def get_csdaddrs_shape(norb, neleca, nelecb):
    """csdstring.py:233-275: (min_npair, npair_offset, npair_dconf_size,
    npair_sconf_size, npair_spins_size)."""
    nless = min(neleca, nelecb)
    min_npair = max(0, neleca + nelecb - norb)
    pairs = range(min_npair, nless + 1)
    nspins = [neleca + nelecb - 2 * p for p in pairs]
    dconf = np.array([comb(norb, p) for p in pairs], dtype=np.int64)
    sconf = np.array([comb(norb - p, ns) for p, ns in zip(pairs, nspins)], dtype=np.int64)
    spins = np.array([comb(ns, (ns + neleca - nelecb) // 2) for ns in nspins], dtype=np.int64)
    sizes = dconf * sconf * spins
    offset = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    assert int(sizes.sum()) == comb(norb, neleca) * comb(norb, nelecb)
    return min_npair, offset, dconf, sconf, spins


def make_csd_mask(norb, neleca, nelecb):
    """csdstring.py:28-47 on the device: mask[idx_csd] = idx_det (uint32,
    held in an int32 tensor)."""
    check_csd_mask_size(norb, neleca, nelecb)
    n = comb(norb, neleca) * comb(norb, nelecb)
    mask = torch.empty(n, dtype=torch.int32, device=device())
    _capi.call("csffci_csd_masks", norb, neleca, nelecb, 0, ptr(mask), None, None, stream())
    return mask


def make_econf_det_mask(norb, neleca, nelecb, csd_mask=None):
    """csdstring.py:49-65 on the device."""
    n = comb(norb, neleca) * comb(norb, nelecb)
    mask = torch.empty(n, dtype=torch.int32, device=device())
    _capi.call("csffci_csd_masks", norb, neleca, nelecb, 0, None, ptr(mask), None, stream())
    return mask
