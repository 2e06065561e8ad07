"""pyscf.fci.addons pieces used by the reference's csf_fci/spin_op.py."""
from pyscf.fci.direct_spin1 import _unpack_nelec  # noqa: F401
