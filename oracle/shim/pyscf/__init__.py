"""ORACLE / TEST INFRASTRUCTURE: a minimal stand-in for the parts of PySCF
core that the reference's pyscf/csf_fci/{csf,csfstring,csdstring}.py import,
so that those reference files run unmodified in the build container to
generate golden fixtures (tests/golden/make_golden.py).  PySCF core is not
installed there.  Every numerical routine below delegates either to the
reference's own C (oracle/_ref via oracle/gasref.py) or to the numpy
restatement in oracle/restate.py.  The reference's csf_fci package is found
through a second path entry pointing at the reference checkout.
"""
import os as _os
__path__.append(_os.path.join(_os.environ.get("CSF_REF_ROOT", "/root/reference"), "pyscf"))
from pyscf import lib, ao2mo  # noqa: E402
from pyscf import __config__  # noqa: E402
