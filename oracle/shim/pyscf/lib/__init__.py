import ctypes
import os
import sys

import numpy as np

from pyscf.lib import logger, param, numpy_helper  # noqa: F401
from pyscf.lib.numpy_helper import tag_array, hermi_triu  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE = os.path.abspath(os.path.join(_HERE, "..", "..", ".."))
if _ORACLE not in sys.path:
    sys.path.insert(0, _ORACLE)
import gasref  # noqa: E402,F401
import restate  # noqa: E402


class _FakeLibfci:
    """libfci.FCIpspace_h0tril_uhf restated (Slater-Condon)."""

    def FCIpspace_h0tril_uhf(self, h0, h1a, h1b, g2aa, g2ab, g2bb, stra, strb, norb, npsp):
        norb = norb.value
        np_ = npsp.value
        as_arr = lambda p, shape, dt: np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(dt)), shape=shape)
        H0 = as_arr(h0, (np_, np_), ctypes.c_double)
        ha = as_arr(h1a, (norb, norb), ctypes.c_double).copy()
        hb = as_arr(h1b, (norb, norb), ctypes.c_double).copy()
        e = as_arr(g2aa, (norb,) * 4, ctypes.c_double).copy()
        sa = as_arr(stra, (np_,), ctypes.c_int64).copy()
        sb = as_arr(strb, (np_,), ctypes.c_int64).copy()
        for i in range(np_):
            for j in range(i):
                H0[i, j] = restate._sc_element(e, ha, hb, int(sa[i]), int(sb[i]), int(sa[j]), int(sb[j]), norb)


def load_library(name):
    if name == "libcsf":
        return gasref.lib_csf()
    if name == "libfci_gas":
        return ctypes.CDLL(os.path.join(gasref.REF_DIR, "libfci_gas.so"))
    if name == "libfci":
        return _FakeLibfci()
    raise OSError(name)


class StreamObject:
    verbose = 0
    stdout = sys.stdout

    def __init__(self, *a, **k):
        pass


def current_memory():
    return (0.0, 0.0)


def fp(a):
    a = np.asarray(a).ravel()
    return float(np.dot(np.cos(np.arange(a.size)), a))




def davidson1(*a, **k):
    raise NotImplementedError("the stand-in drives Davidson through FCISolver.eig")


def take_2d(a, idx, idy):
    """a[idx][:, idy] as a new array (role of lib.take_2d)."""
    return np.asarray(a)[np.ix_(np.asarray(idx), np.asarray(idy))].copy()


def takebak_2d(out, a, idx, idy):
    """out[idx[:, None], idy] += a (role of lib.takebak_2d)."""
    out[np.ix_(np.asarray(idx), np.asarray(idy))] += a
    return out


def isinteger(obj):
    """Integer scalars (Python or numpy), not bool (role of lib.isinteger)."""
    return isinstance(obj, (int, np.integer)) and not isinstance(obj, (bool, np.bool_))


def with_doc(doc):
    """Decorator setting __doc__ (role of lib.with_doc)."""
    def deco(fn):
        fn.__doc__ = doc
        return fn
    return deco
