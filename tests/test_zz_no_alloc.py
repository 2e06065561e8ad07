"""GPU: the allocation-free determinant diagonal (csffci_hdiag_det_noalloc).

Some callers cannot call cudaMalloc, for example a program whose device
memory belongs to another allocator with a fixed budget.  They also have no
buffer to lend as a workspace, so the library offers a diagonal that keeps
its scratch in a fixed array of its own.  This file checks, through the C
ABI, that it gives the same diagonal as csffci_hdiag_det on two calls in a
row (the shared scratch keeps the previous call's contents), and that a
space too large for the fixed array is refused with an error.  The file
sorts last so that a run stopping at the first failure has already run
every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

import restate as R
from conftest import seeded_integrals

pytestmark = pytest.mark.gpu


def _diag_both(norb, nelec, seed):
    from pyscf_forge_b200 import _capi
    from pyscf_forge_b200._runtime import ptr, stream
    from math import comb
    h1, eri = seeded_integrals(norb, 2 * norb, seed=seed)
    ha = torch.as_tensor(h1, device="cuda")
    hb = torch.as_tensor(h1 + 0.01 * np.eye(norb), device="cuda")
    e4 = torch.as_tensor(R.restore4(eri, norb), device="cuda")
    n = comb(norb, nelec[0]) * comb(norb, nelec[1])
    ref = torch.empty(n, dtype=torch.float64, device="cuda")
    nbytes = _capi.query("csffci_hdiag_det_workspace", norb, nelec[0], nelec[1])
    ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    _capi.call("csffci_hdiag_det", norb, nelec[0], nelec[1], ptr(ha), ptr(hb), ptr(e4), ptr(ref),
               ptr(ws), nbytes, stream())
    got = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
    _capi.call("csffci_hdiag_det_noalloc", norb, nelec[0], nelec[1], ptr(ha), ptr(hb), ptr(e4),
               ptr(got), stream())
    torch.cuda.synchronize()
    return got.cpu().numpy(), ref.cpu().numpy()


def test_noalloc_diagonal_matches_workspace_version_twice():
    # two calls in a row with different sizes and integrals: the second
    # sees whatever the first left in the shared scratch
    for norb, nelec, seed in ((12, (6, 6), 1), (10, (6, 3), 2), (16, (8, 8), 3)):
        got, ref = _diag_both(norb, nelec, seed)
        # same kernels and arithmetic as csffci_hdiag_det: tolerance 1e-12
        np.testing.assert_allclose(got, ref, atol=1e-12, rtol=0)


def test_noalloc_rejects_spaces_beyond_the_fixed_scratch():
    from pyscf_forge_b200 import _capi
    lib = _capi.load()
    dummy = ctypes.c_void_p(0)
    st = lib.csffci_hdiag_det_noalloc(18, 9, 9, dummy, dummy, dummy, dummy, None)
    assert st == _capi.CSFFCI_ERR_MEMORY
    assert b"scratch" in lib.csffci_last_error()
