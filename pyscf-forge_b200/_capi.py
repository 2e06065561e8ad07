"""ctypes binding of libcsffci_b200.so (declared in include/csffci_b200.h).

The library is the only compute path: if it cannot be loaded, every entry
point of this package raises.  There is no CPU fallback.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcsffci_b200.so")

CSFFCI_OK = 0
CSFFCI_ERR_INVALID = -1
CSFFCI_ERR_MEMORY = -2
CSFFCI_ERR_CUDA = -3
CSFFCI_ERR_TIMEOUT = -4

SIGMA_ACCUMULATE = 1
SIGMA_SPIN_SYMMETRIC = 2
SIGMA_REFERENCE_KERNEL = 4
SIGMA_DETERMINISTIC = 8
SIGMA_JOB_DETERMINISTIC = 1


class LinkEntry(ctypes.Structure):
    """csffci_link_t: byte layout of the raw gas_link_entry_t
    (pyscf/lib/mcscf/fci_gas.h:94-105)."""
    _fields_ = [("addr", ctypes.c_uint32), ("op", ctypes.c_uint16),
                ("sign", ctypes.c_int8), ("pad", ctypes.c_uint8)]


class Block(ctypes.Structure):
    """csffci_block_t: one npair block of the CSF <-> determinant map."""
    _fields_ = [("csd_offset", ctypes.c_int64), ("csf_offset", ctypes.c_int64),
                ("nconf", ctypes.c_int64), ("ndet", ctypes.c_int32), ("ncsf", ctypes.c_int32),
                ("nspin", ctypes.c_int32), ("npair", ctypes.c_int32), ("sign", ctypes.c_double),
                ("umat", ctypes.c_void_p), ("zmat", ctypes.c_void_p), ("conf_sel", ctypes.c_void_p)]


class SigmaJob(ctypes.Structure):
    """csffci_sigma_job_t."""
    _fields_ = [("h2e", ctypes.c_void_p), ("link_a", ctypes.c_void_p), ("link_b", ctypes.c_void_p),
                ("ci", ctypes.c_void_p), ("sigma", ctypes.c_void_p), ("scratch", ctypes.c_void_p),
                ("neleca", ctypes.c_int32), ("nelecb", ctypes.c_int32), ("sym", ctypes.c_int32),
                ("eta", ctypes.c_int32), ("live", ctypes.c_void_p), ("live_index", ctypes.c_int32),
                ("flags", ctypes.c_int32), ("Na", ctypes.c_int64), ("Nb", ctypes.c_int64),
                ("unit_begin", ctypes.c_int64), ("nunits", ctypes.c_int64),
                ("tile_begin", ctypes.c_int64), ("elem_begin", ctypes.c_int64),
                ("nla", ctypes.c_int32), ("nlb", ctypes.c_int32)]


class TransformJob(ctypes.Structure):
    """csffci_transform_job_t."""
    _fields_ = [("x", ctypes.c_void_p), ("y", ctypes.c_void_p), ("mask", ctypes.c_void_p),
                ("umat", ctypes.c_void_p), ("ldx", ctypes.c_int64), ("ldy", ctypes.c_int64),
                ("csd_offset", ctypes.c_int64), ("csf_offset", ctypes.c_int64), ("nconf", ctypes.c_int64),
                ("ndet", ctypes.c_int32), ("ncsf", ctypes.c_int32), ("nvec", ctypes.c_int32),
                ("pad", ctypes.c_int32), ("sign", ctypes.c_double), ("live", ctypes.c_void_p),
                ("tile_begin", ctypes.c_int64)]


class ZeroJob(ctypes.Structure):
    """csffci_zero_job_t."""
    _fields_ = [("y", ctypes.c_void_p), ("ld", ctypes.c_int64), ("n", ctypes.c_int64),
                ("nvec", ctypes.c_int64), ("elem_begin", ctypes.c_int64)]


class Dot(ctypes.Structure):
    """csffci_dot_t."""
    _fields_ = [("x", ctypes.c_void_p), ("y", ctypes.c_void_p), ("hdiag", ctypes.c_void_p),
                ("n", ctypes.c_int64), ("e_shift", ctypes.c_double), ("out_index", ctypes.c_int64)]


class Combine(ctypes.Structure):
    """csffci_combine_t."""
    _fields_ = [("y", ctypes.c_void_p), ("x", ctypes.c_void_p), ("coef", ctypes.c_void_p),
                ("n", ctypes.c_int64), ("ldx", ctypes.c_int64), ("ldy", ctypes.c_int64),
                ("ny", ctypes.c_int32), ("nx", ctypes.c_int32), ("ldc", ctypes.c_int32),
                ("pad", ctypes.c_int32), ("beta", ctypes.c_double), ("scale", ctypes.c_double),
                ("unit_begin", ctypes.c_int64)]


class Precond(ctypes.Structure):
    """csffci_precond_t."""
    _fields_ = [("r", ctypes.c_void_p), ("x", ctypes.c_void_p), ("hdiag", ctypes.c_void_p),
                ("t", ctypes.c_void_p), ("ab", ctypes.c_void_p), ("n", ctypes.c_int64),
                ("e_shift", ctypes.c_double), ("unit_begin", ctypes.c_int64)]


class BatchProblem(ctypes.Structure):
    """csffci_batch_problem_t."""
    _fields_ = [("norb", ctypes.c_int32), ("neleca", ctypes.c_int32), ("nelecb", ctypes.c_int32),
                ("nroots", ctypes.c_int32), ("eta", ctypes.c_int32), ("nblocks", ctypes.c_int32),
                ("blocks", ctypes.c_void_p), ("csd_mask", ctypes.c_void_p), ("ncsf", ctypes.c_int64),
                ("h2e", ctypes.c_void_p), ("link_a", ctypes.c_void_p), ("link_b", ctypes.c_void_p),
                ("hdiag", ctypes.c_void_p), ("x0", ctypes.c_void_p)]


class BatchOptions(ctypes.Structure):
    """csffci_batch_options_t."""
    _fields_ = [("conv_tol", ctypes.c_double), ("conv_tol_residual", ctypes.c_double),
                ("lindep", ctypes.c_double), ("level_shift", ctypes.c_double),
                ("max_space", ctypes.c_int32), ("max_cycle", ctypes.c_int32),
                ("check_every", ctypes.c_int32), ("use_graph", ctypes.c_int32),
                ("autotune", ctypes.c_int32), ("deterministic", ctypes.c_int32)]


assert ctypes.sizeof(LinkEntry) == 8
assert ctypes.sizeof(Block) == 72
assert ctypes.sizeof(SigmaJob) == 136
assert ctypes.sizeof(TransformJob) == 112
assert ctypes.sizeof(BatchProblem) == 88
assert ctypes.sizeof(BatchOptions) == 56
assert ctypes.sizeof(ZeroJob) == 40
assert ctypes.sizeof(Dot) == 48
assert ctypes.sizeof(Combine) == 88
assert ctypes.sizeof(Precond) == 64

_i = ctypes.c_int
_i64 = ctypes.c_int64
_sz = ctypes.c_size_t
_d = ctypes.c_double
_p = ctypes.c_void_p

_SIGS = {
    "csffci_abi_version": ([], _i),
    "csffci_last_error": ([], ctypes.c_char_p),
    "csffci_profile_enable": ([_i], _i),
    "csffci_profile_report": ([ctypes.c_char_p, _sz], _i),
    "csffci_fp64_peak": ([_i, _i, ctypes.POINTER(_d), _p], _i),
    "csffci_gen_strings": ([_i, _i, _p, _p], _i),
    "csffci_link_table": ([_i, _i, _p, _p], _i),
    "csffci_gas_conf_mask": ([_i, _i, _i, _p, _i, _p, _i, _p, _p, _p], _i),
    "csffci_csd_masks": ([_i, _i, _i, _i, _p, _p, _p, _p], _i),
    "csffci_spin_evecs": ([_i, _i, _i, _i, _p, _p], _i),
    "csffci_spin_exchange_table": ([_i, _i, _i, _i, _p, _p, _p], _i),
    "csffci_det2csf": ([_i, _p, _i64, _p, _i64, _p, _p, _i, _p], _i),
    "csffci_csf2det": ([_i, _p, _i64, _p, _i64, _i64, _p, _p, _i, _p], _i),
    "csffci_absorb_h1e": ([_i, _i, _p, _p, _d, _p, _p], _i),
    "csffci_hdiag_det_workspace": ([_i, _i, _i], _sz),
    "csffci_hdiag_det": ([_i, _i, _i, _p, _p, _p, _p, _p, _sz, _p], _i),
    "csffci_hdiag_det_noalloc": ([_i, _i, _i, _p, _p, _p, _p, _p], _i),
    "csffci_hdiag_csf": ([_i, _i, _i, _p, _p, _p, _p, _i, _p, _p], _i),
    "csffci_pspace_h0": ([_i, _i, _i, _p, _p, _p, _p, _p, _i, _p, _p], _i),
    "csffci_sigma_workspace": ([_i, _i, _i, _i], _sz),
    "csffci_spin_parity": ([_i64, _p, _p, _p, _sz, _p], _i),
    "csffci_sigma": ([_i, _i, _i, _p, _p, _p, _p, _p, _i, _i, _p, _sz, _p], _i),
    "csffci_contract_1e": ([_i, _i, _i, _p, _p, _p, _p, _p, _p, _p], _i),
    "csffci_rdm12_workspace": ([_i, _i, _i], _sz),
    "csffci_rdm12": ([_i, _i, _i, _p, _p, _p, _p, _p, _p, _p, _sz, _p], _i),
    "csffci_rdm12s_workspace": ([_i, _i, _i], _sz),
    "csffci_rdm12s": ([_i, _i, _i] + [_p] * 10 + [_sz, _p], _i),
    "csffci_gram_workspace": ([_i, _i, _i64], _sz),
    "csffci_gram": ([_i, _p, _i64, _i, _p, _i64, _i64, _p, _p, _sz, _p], _i),
    "csffci_combine": ([_i, _p, _i64, _d, _i, _p, _i64, _p, _i64, _p], _i),
    "csffci_precond_workspace": ([], _sz),
    "csffci_precond": ([_i64, _p, _p, _p, _d, _d, _i, _d, _p, _p, _p], _i),
    "csffci_precond_dots": ([_i64, _p, _p, _p, _d, _d, _p, _p, _p], _i),
    "csffci_sigma_plan_create": ([_i, _i, _i, _p, _p, _p, _i, ctypes.POINTER(_p), ctypes.POINTER(_sz)], _i),
    "csffci_sigma_plan_bind": ([_p, _p, _sz], _i),
    "csffci_sigma_plan_execute": ([_p, _p, _p, _i, _i, _p], _i),
    "csffci_sigma_plan_variant": ([_p], _i),
    "csffci_sigma_plan_destroy": ([_p], None),
    "csffci_sigma_batch_workspace": ([_i], _sz),
    "csffci_sigma_batch": ([_i, _i, _p, _p, _sz, _p], _i),
    "csffci_transform_batch": ([_i, _i, _p, _i, _p, _p, _sz, _p], _i),
    "csffci_dots_batch": ([_i, _p, _p, _p, _sz, _p], _i),
    "csffci_combine_batch": ([_i, _p, _p, _sz, _p], _i),
    "csffci_precond_batch": ([_i, _p, _p, _sz, _p], _i),
    "csffci_spin_ladder": ([_i, _i, _i, _i, _p, _p, _p], _i),
    "csffci_batch_plan_create": ([_i, _p, _p, ctypes.POINTER(_p), ctypes.POINTER(_sz)], _i),
    "csffci_batch_plan_bind": ([_p, _p, _sz, _p], _i),
    "csffci_batch_plan_run": ([_p, _p, ctypes.POINTER(_i)], _i),
    "csffci_batch_plan_max_roots": ([_p], _i),
    "csffci_batch_plan_tile_variants": ([_p, _p, _p, _i], _i),
    "csffci_batch_plan_results": ([_p, _p, _p, _p, _p, _p], _i),
    "csffci_batch_plan_to_det": ([_p, _p], _i),
    "csffci_batch_plan_vectors": ([_p, _i, ctypes.POINTER(_p), ctypes.POINTER(_p)], _i),
    "csffci_batch_plan_destroy": ([_p], None),
}

_LIB = None


class CSFFCIError(RuntimeError):
    def __init__(self, name, status, message):
        super().__init__("%s failed (status %d): %s" % (name, status, message))
        self.status = status


def exported_symbols():
    return sorted(_SIGS)


def load():
    """Load (building first if the sources are newer and nvcc exists)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    try:
        from . import build as _build
        if not _build.up_to_date():
            _build.build()
    except Exception:  # no nvcc on this machine: use the shipped library
        pass
    if not os.path.exists(LIB_PATH):
        raise ImportError("libcsffci_b200.so is missing (%s); build it with "
                          "python pyscf-forge_b200/build.py" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, (args, res) in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _LIB = lib
    return lib


def call(name, *args):
    lib = load()
    st = getattr(lib, name)(*args)
    if st != CSFFCI_OK:
        msg = lib.csffci_last_error().decode(errors="replace")
        if st == CSFFCI_ERR_MEMORY:
            raise MemoryError("%s: %s" % (name, msg))
        raise CSFFCIError(name, st, msg)
    return st


def query(name, *args):
    return getattr(load(), name)(*args)


def profile_enable(on=True):
    call("csffci_profile_enable", 1 if on else 0)


def profile_report():
    """{kernel: (launches, total_ms)} recorded since profile_enable(True)."""
    buf = ctypes.create_string_buffer(1 << 16)
    call("csffci_profile_report", buf, len(buf))
    out = {}
    for line in buf.value.decode().splitlines():
        name, cnt, ms = line.split()
        out[name] = (int(cnt), float(ms))
    return out


def fp64_peak(kind=0, iters=20000, stream=None):
    """Measured FP64 TFLOP/s on the current device (kind 0: DMMA at 16 warps
    per SM, 1: DFMA, 2: DMMA at 17 warps per SM)."""
    out = ctypes.c_double(0.0)
    call("csffci_fp64_peak", int(kind), int(iters), ctypes.byref(out), stream)
    return out.value
