import numpy as np
from pyscf.lib import restate


def num_strings(norb, nelec):
    return restate.num_strings(norb, nelec)


def addrs2str(norb, nelec, addrs):
    return restate.addrs2str(norb, nelec, np.asarray(addrs, dtype=np.int64).reshape(-1))


def addr2str(norb, nelec, addr):
    return int(restate.gen_strings(norb, nelec)[int(addr)])


def strs2addr(norb, nelec, strs):
    return restate.strs2addr(norb, nelec, strs)


def gen_strings4orblist(orb_list, nelec):
    return restate.gen_strings(len(list(orb_list)), nelec)
