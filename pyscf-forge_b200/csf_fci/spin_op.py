"""Spin ladder operators on determinant CI vectors, on the GPU
(pyscf/csf_fci/spin_op.py:1-151): ``contract_sladder`` / ``contract_sdown``
/ ``contract_sup`` apply S- or S+ (csffci_spin_ladder), ``mdown`` / ``mup``
rotate a spin-pure vector between its M_S = S microstate and another one,
``spin_square`` gives <S^2> from S^2 = S-S+ + Sz + Sz^2.  numpy in, numpy
out; torch CUDA tensors in, torch tensors out.
"""
from math import comb

import numpy as np
import torch

from .. import _capi
from .._runtime import like_input, ptr, stream, to_dev
from ..fci.direct_spin1 import _unpack_nelec


def norm_sdown(smult, nelec):
    """spin_op.py:12-15: |S- |S, M>| for the M of nelec."""
    s2 = smult - 1
    m2 = nelec[0] - nelec[1]
    return np.sqrt((s2 - m2 + 2) * (s2 + m2) / 4)


def norm_sup(smult, nelec):
    """spin_op.py:17-20: |S+ |S, M>|."""
    s2 = smult - 1
    m2 = nelec[0] - nelec[1]
    return np.sqrt((s2 - m2) * (s2 + m2 + 2) / 4)


def dev_contract_sladder(ci, norb, nelec, op=-1):
    """S+ (op=1) or S- (op=-1) on a device vector; returns the device
    (C(norb,na+op), C(norb,nb-op)) vector."""
    neleca, nelecb = _unpack_nelec(nelec)
    c = to_dev(ci).reshape(-1).contiguous()
    assert c.numel() == comb(norb, neleca) * comb(norb, nelecb)
    out = torch.empty((comb(norb, neleca + op), comb(norb, nelecb - op)), dtype=torch.float64, device=c.device)
    _capi.call("csffci_spin_ladder", norb, neleca, nelecb, op, ptr(c), ptr(out), stream())
    return out


def contract_sladder(fcivec, norb, nelec, op=-1):
    """spin_op.py:22-68: S+ or S- on fcivec; changes neleca - nelecb without
    changing <S^2>.  The vacuum of the operator gives a (0, 0) array."""
    neleca, nelecb = _unpack_nelec(nelec)
    assert op in (-1, 1), 'op = -1 or 1'
    if ((op == -1 and (neleca == 0 or nelecb == norb)) or (op == 1 and (neleca == norb or nelecb == 0))):
        if isinstance(fcivec, torch.Tensor):
            return torch.zeros((0, 0), dtype=torch.float64, device=fcivec.device)
        return np.zeros((0, 0))
    out = dev_contract_sladder(fcivec, norb, (neleca, nelecb), op)
    return out if isinstance(fcivec, torch.Tensor) else out.cpu().numpy()


def contract_sdown(ci, norb, nelec):
    return contract_sladder(ci, norb, nelec, op=-1)


def contract_sup(ci, norb, nelec):
    return contract_sladder(ci, norb, nelec, op=1)


def as_list(ci0):
    if isinstance(ci0, (np.ndarray, torch.Tensor)) and ci0.ndim == 2:
        return [ci0]
    return list(ci0)


def like_ci0(ci1, ci0):
    if isinstance(ci0, (np.ndarray, torch.Tensor)) and ci0.ndim == 2:
        return ci1[0]
    if isinstance(ci1[0], torch.Tensor):
        return torch.stack(ci1, dim=0)
    return np.stack(ci1, axis=0)


def mdown(ci0, norb, nelec, smult):
    """spin_op.py:84-115: M_S = S vector(s) -> the same state(s) with the
    electron numbers nelec."""
    ci1 = as_list(ci0)
    neleca, nelecb = _unpack_nelec(nelec)
    for i in range(len(ci1)):
        for j in range(((smult - 1) - (neleca - nelecb)) // 2, 0, -1):
            ci1[i] = contract_sdown(ci1[i], norb, (neleca + j, nelecb - j))
            ci1[i] = ci1[i] / norm_sdown(smult, (neleca + j, nelecb - j))
    return like_ci0(ci1, ci0)


def mup(ci0, norb, nelec, smult):
    """spin_op.py:117-145: vector(s) with electron numbers nelec -> the
    M_S = S microstate."""
    ci1 = as_list(ci0)
    neleca, nelecb = _unpack_nelec(nelec)
    for i in range(len(ci1)):
        for j in range(((smult - 1) - (neleca - nelecb)) // 2):
            ci1[i] = contract_sup(ci1[i], norb, (neleca + j, nelecb - j))
            ci1[i] = ci1[i] / norm_sup(smult, (neleca + j, nelecb - j))
    return like_ci0(ci1, ci0)


def spin_square(fcivec, norb, nelec):
    """(<S^2>, 2S+1) of a determinant vector, unnormalised as
    fci.spin_op.spin_square0 returns it: <S^2> = |S+ c|^2 + (Sz + Sz^2)|c|^2."""
    neleca, nelecb = _unpack_nelec(nelec)
    c = to_dev(fcivec).reshape(-1)
    sz = 0.5 * (neleca - nelecb)
    ss = (sz + sz * sz) * float(torch.dot(c, c))
    if neleca < norb and nelecb > 0:
        sp = dev_contract_sladder(c, norb, (neleca, nelecb), op=1)
        ss += float(torch.dot(sp.reshape(-1), sp.reshape(-1)))
    s = np.sqrt(ss + .25) - .5
    return ss, s * 2 + 1
