"""CPU: the C-ABI library loads and exports every symbol include/*.h declares
(no compute calls without a GPU)."""
import ctypes
import glob
import os
import re

from conftest import ROOT


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"\b(csffci_\w+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol():
    from pyscf_forge_b200 import _capi
    lib = _capi.load()
    declared = _declared()
    assert declared, "no declarations parsed"
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    # every declared entry point has a ctypes signature in the binding
    assert declared <= set(_capi.exported_symbols()), sorted(declared - set(_capi.exported_symbols()))
    assert lib.csffci_abi_version() == 1


def test_struct_layouts():
    from pyscf_forge_b200 import _capi
    assert ctypes.sizeof(_capi.LinkEntry) == 8
    assert ctypes.sizeof(_capi.Block) == 72


def test_struct_layouts_match_header(tmp_path):
    """sizeof/offsetof of every descriptor struct of include/csffci_b200.h,
    compiled by the host C compiler, equal the ctypes mirrors."""
    import shutil
    import subprocess
    import pytest
    from pyscf_forge_b200 import _capi
    cc = shutil.which("gcc") or shutil.which("cc")
    cuda_inc = "/usr/local/cuda/include"
    if cc is None or not os.path.exists(os.path.join(cuda_inc, "cuda_runtime.h")):
        pytest.skip("no host C compiler or CUDA headers")
    structs = {"csffci_link_t": _capi.LinkEntry, "csffci_block_t": _capi.Block,
               "csffci_sigma_job_t": _capi.SigmaJob, "csffci_transform_job_t": _capi.TransformJob,
               "csffci_zero_job_t": _capi.ZeroJob, "csffci_dot_t": _capi.Dot,
               "csffci_combine_t": _capi.Combine, "csffci_precond_t": _capi.Precond,
               "csffci_batch_problem_t": _capi.BatchProblem, "csffci_batch_options_t": _capi.BatchOptions}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "csffci_b200.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append('printf("%s %%zu\\n", sizeof(%s));' % (cname, cname))
        for f in py._fields_:
            lines.append('printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (cname, f[0], cname, f[0]))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), "-I", cuda_inc, str(src), "-o", str(exe)],
                   check=True)
    out = dict(l.split() for l in subprocess.run([str(exe)], check=True, capture_output=True,
                                                   text=True).stdout.splitlines())
    for cname, py in structs.items():
        assert int(out[cname]) == ctypes.sizeof(py), cname
        for f in py._fields_:
            assert int(out[cname + "." + f[0]]) == getattr(py, f[0]).offset, (cname, f[0])


def test_binding_argument_counts_match_header():
    """Every ctypes signature has as many arguments as the header's
    declaration (a miscounted binding would shift every later argument)."""
    from pyscf_forge_b200 import _capi
    decl = {}
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        for name, params in re.findall(r"\b(csffci_\w+)\s*\(([^;{]*?)\)\s*;", txt, flags=re.S):
            params = params.strip()
            decl[name] = 0 if params in ("", "void") else params.count(",") + 1
    assert decl
    for name, (args, _) in _capi._SIGS.items():
        assert name in decl, name
        assert len(args) == decl[name], (name, len(args), decl[name])
