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


def _sign_above(p, string0):
    """(-1)^(occupied orbitals above p): the sign of a+_p / a_p on a string
    (PySCF's cre_sign / des_sign convention)."""
    return -1 if bin(int(string0) >> (p + 1)).count('1') % 2 else 1


def gen_cre_str_index(orb_list, nelec):
    """(nstr, norb-nelec, 4) rows (p, 0, address of p+ |str>, sign) for the
    unoccupied p of each string (role of cistring.gen_cre_str_index)."""
    orbs = list(orb_list)
    norb = len(orbs)
    strs = restate.gen_strings(norb, nelec)
    tgt = {int(s): i for i, s in enumerate(restate.gen_strings(norb, nelec + 1).tolist())}
    out = np.zeros((len(strs), norb - nelec, 4), dtype=np.int32)
    for k, s in enumerate(strs.tolist()):
        j = 0
        for p in orbs:
            if not (s >> p) & 1:
                out[k, j] = (p, 0, tgt[s | (1 << p)], _sign_above(p, s))
                j += 1
    return out


def gen_des_str_index(orb_list, nelec):
    """(nstr, nelec, 4) rows (0, p, address of a_p |str>, sign) for the
    occupied p of each string (role of cistring.gen_des_str_index)."""
    orbs = list(orb_list)
    norb = len(orbs)
    strs = restate.gen_strings(norb, nelec)
    tgt = {int(s): i for i, s in enumerate(restate.gen_strings(norb, nelec - 1).tolist())}
    out = np.zeros((len(strs), nelec, 4), dtype=np.int32)
    for k, s in enumerate(strs.tolist()):
        j = 0
        for p in orbs:
            if (s >> p) & 1:
                out[k, j] = (0, p, tgt[s ^ (1 << p)], _sign_above(p, s))
                j += 1
    return out


def make_strings(orb_list, nelec):
    """Occupation strings of nelec electrons in orb_list (role of
    cistring.make_strings)."""
    return gen_strings4orblist(orb_list, nelec)
