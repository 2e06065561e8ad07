"""CPU: the deterministic sigma scatter (CSFFCI_SIGMA_DETERMINISTIC).

det_add3 (pyscf-forge_b200/csrc/sigma_rr_kernel.cuh) splits each scattered
contribution x into three integer digits, x = d2 2^6 + d1 2^-37 + d0 2^-80,
and adds each digit to its own int64 plane; k_det_finish (csrc/sigma.cu)
forms sigma from the digit sums.  Restated here with numpy float64 (the
same IEEE operations: rint, fma-free exact steps) and Python integers:
the split is exact up to the rounding of d0, the digits stay within 2^42,
the plane sums do not depend on the order of the contributions, and the
formed value is within one rounding of the exact sum.  Also the C-ABI
checks of the flag (no compute call)."""
import ctypes
import math
import random
from fractions import Fraction

import numpy as np
import pytest


def _split(x):
    """det_add3's digits of x (the two remainders are exact, so the fma of
    the kernel and the plain subtraction here give the same values)."""
    x = np.float64(x)
    h2 = np.rint(x * np.float64(2.0 ** -6))
    r1 = x - h2 * np.float64(64.0)
    h1 = np.rint(r1 * np.float64(2.0 ** 37))
    r0 = r1 - h1 * np.float64(2.0 ** -37)
    h0 = np.rint(r0 * np.float64(2.0 ** 80))
    return int(h0), int(h1), int(h2)


def _value(w0, w1, w2):
    """k_det_finish's value of the digit sums (each term exact, fixed order)."""
    return (np.float64(w2) * np.float64(64.0) + np.float64(w1) * np.float64(2.0 ** -37)) \
        + np.float64(w0) * np.float64(2.0 ** -80)


def _contributions(rng, n):
    mags = rng.choice([1e-300, 1e-30, 1e-12, 1e-3, 0.7, 3.0, 1e3, 1e9, 2.0 ** 47])
    return [float(v) for v in rng.standard_normal(n) * mags]


def test_split_is_exact_and_bounded():
    rng = np.random.default_rng(3)
    for x in _contributions(rng, 2000) + [0.0, -0.0, 2.0 ** 47 - 1, -(2.0 ** 47), 5e-324]:
        d0, d1, d2 = _split(x)
        assert max(abs(d0), abs(d1), abs(d2)) <= 2 ** 42
        back = Fraction(d2) * 64 + Fraction(d1, 2 ** 37) + Fraction(d0, 2 ** 80)
        # only d0 rounds: the error is at most half a unit of 2^-80
        assert abs(back - Fraction(x)) <= Fraction(1, 2 ** 81)


def test_plane_sums_are_order_independent():
    rng = np.random.default_rng(4)
    for trial in range(30):
        xs = _contributions(rng, 150)
        digits = [_split(x) for x in xs]
        sums = [tuple(sum(d[k] for d in digits) for k in range(3))]
        for _ in range(5):
            random.Random(trial).shuffle(digits)
            # int64 wrap-around sums, as the integer atomics form them
            w = [0, 0, 0]
            for d in digits:
                for k in range(3):
                    w[k] = (w[k] + d[k] + 2 ** 63) % 2 ** 64 - 2 ** 63
            sums.append(tuple(w))
        assert len(set(sums)) == 1
        w0, w1, w2 = sums[0]
        assert max(abs(w0), abs(w1), abs(w2)) < 2 ** 53  # exact conversion to double
        v = _value(w0, w1, w2)
        exact = math.fsum(xs)
        # three roundings of the fixed-order sum (plus 2^-80 per contribution)
        assert abs(v - exact) <= 4 * np.spacing(max(abs(exact), 1e-300)) + 150 * 2.0 ** -80


def test_symmetric_finish_adds_digits_first():
    """S[a][b] + eta S[b][a] on the digit sums (integer add) equals the
    exact sum of both entries' contributions, for eta = +1 and -1."""
    rng = np.random.default_rng(5)
    for eta in (1, -1):
        xa, xb = _contributions(rng, 70), _contributions(rng, 70)
        da = [sum(_split(x)[k] for x in xa) for k in range(3)]
        db = [sum(_split(x)[k] for x in xb) for k in range(3)]
        v = _value(*[da[k] + eta * db[k] for k in range(3)])
        exact = math.fsum(xa + [eta * x for x in xb])
        assert abs(v - exact) <= 4 * np.spacing(max(abs(exact), 1e-300)) + 140 * 2.0 ** -80


def test_plan_flag_checks():
    """csffci_sigma_plan_create with CSFFCI_SIGMA_DETERMINISTIC: the digit
    planes as workspace and the warp-specialised kernel inside 4..16
    orbitals; refused outside it and with the reference kernel.  create
    only records the borrowed pointers, so placeholders do here."""
    from math import comb
    from pyscf_forge_b200 import _capi
    lib = _capi.load()
    dummy = ctypes.c_void_p(16)
    det = _capi.SIGMA_DETERMINISTIC
    for norb, nelec, extra in ((12, (6, 6), _capi.SIGMA_SPIN_SYMMETRIC), (10, (5, 4), 0), (16, (3, 2), 0),
                               (4, (2, 1), 0)):
        h = ctypes.c_void_p()
        nbytes = ctypes.c_size_t()
        st = lib.csffci_sigma_plan_create(norb, nelec[0], nelec[1], dummy, dummy, dummy, det | extra,
                                          ctypes.byref(h), ctypes.byref(nbytes))
        assert st == 0, lib.csffci_last_error()
        assert nbytes.value == 3 * 8 * comb(norb, nelec[0]) * comb(norb, nelec[1])
        assert lib.csffci_sigma_plan_variant(h) == 4
        lib.csffci_sigma_plan_destroy(h)
        assert lib.csffci_sigma_workspace(norb, nelec[0], nelec[1], det) == nbytes.value
    for norb, flags in ((3, det), (17, det), (12, det | _capi.SIGMA_REFERENCE_KERNEL)):
        h = ctypes.c_void_p()
        st = lib.csffci_sigma_plan_create(norb, 3, 3, dummy, dummy, dummy, flags, ctypes.byref(h), None)
        assert st == _capi.CSFFCI_ERR_INVALID
        assert b"deterministic" in lib.csffci_last_error()
