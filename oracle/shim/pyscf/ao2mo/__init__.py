from pyscf.lib import restate


def restore(sym, eri, norb):
    if sym == 1:
        return restate.restore1(eri, norb)
    if sym == 4:
        return restate.restore4(eri, norb)
    raise NotImplementedError(sym)
