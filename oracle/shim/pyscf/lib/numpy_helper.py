import numpy as np


class _Tagged(np.ndarray):
    pass


def tag_array(a, **kw):
    t = np.asarray(a).view(_Tagged)
    t.__dict__.update(kw)
    return t


def transpose(a, inplace=False):
    return np.ascontiguousarray(np.asarray(a).T)


def hermi_triu(h):
    """Fill the upper triangle from the lower one."""
    h = np.array(h)
    iu = np.triu_indices(h.shape[0], 1)
    h[iu] = h.T[iu]
    return h
