from pyscf.lib import restate


def spin_square0(ci, norb, nelec):
    return restate.spin_square(ci, norb, nelec)
