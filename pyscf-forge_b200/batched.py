"""Many independent CSF-FCI problems solved in lockstep on one GPU.

``BatchedCSFSolver.kernel(problems)`` runs the Davidson iterations of every
problem of a batch together: each iteration issues a fixed number of
launches for the whole batch (batched det<->CSF transforms, one persistent
sigma launch per orbital count over every (problem, vector) job, batched dot
products, linear combinations and preconditioning), with three host
synchronisations per iteration for the small subspace eigenproblems.
Problems may differ in norb, electron numbers, spin and number of roots.
Problems whose CSF space fits the p-space are diagonalised exactly, as the
reference does (pyscf/csf_fci/csf.py:416-429).  RDMs of every root come from
the adjoint kernel (csffci_rdm12).

``solve_plain(problems)`` is the one-problem-at-a-time form through the
public FCISolver API, for comparison.  ``make_uneven_batch`` generates the
seeded uneven batch of the benchmark configuration.

No counterpart in the reference, which solves one problem per call.
"""
import ctypes
import time
from math import comb

import numpy as np
import torch

from . import _capi
from ._runtime import device, eri_pair_matrix, ptr, stream, to_dev, workspace
from .csf_fci.csf import FCISolver, pspace as csf_pspace
from .csf_fci.csfstring import CSFTransformer, ImpossibleCIvecError, get_csfvec_shape, count_all_csfs
from .fci import direct_spin1 as D


class Problem:
    """One CI problem: integrals (h1 (n,n), eri any PySCF layout), norb,
    (neleca, nelecb), 2S+1 and the number of roots."""

    def __init__(self, norb, nelec, smult, nroots, h1, eri):
        self.norb = int(norb)
        self.nelec = (int(nelec[0]), int(nelec[1]))
        self.smult = int(smult)
        self.nroots = int(nroots)
        self.h1 = np.asarray(h1, dtype=np.float64)
        self.eri = np.asarray(eri, dtype=np.float64)


def _seeded_integrals(norb, rank, seed):
    rng = np.random.default_rng(seed)
    h1 = rng.normal(0.0, 0.3, (norb, norb))
    h1 = 0.5 * (h1 + h1.T)
    np.fill_diagonal(h1, np.linspace(-2.0, 0.5, norb))
    L = rng.normal(0.0, 0.2, (rank, norb * norb)).reshape(rank, norb, norb)
    L = 0.5 * (L + L.transpose(0, 2, 1))
    eri = 0.5 * np.einsum("xpq,xrs->pqrs", L, L)
    return h1, eri


def make_uneven_batch(nprob=128, seed0=1000, norb_lo=6, norb_hi=12):
    """Seeded uneven batch: problem i uses seed seed0+i; norb ~ U{lo..hi};
    N electrons = 2*ceil(norb/2) + U{-2..2} (MS = 0 for even N, 1/2 for
    odd); S ~ U{0,1,2} (+1/2 for odd N), redrawn when impossible; nroots ~
    U{1..4} capped at the number of CSFs; integrals rank 2*norb."""
    out = []
    for i in range(nprob):
        rng = np.random.default_rng(seed0 + i)
        norb = int(rng.integers(norb_lo, norb_hi + 1))
        ntot = 2 * ((norb + 1) // 2) + int(rng.integers(-2, 3))
        ntot = max(2, min(ntot, 2 * norb - 2))
        ms2 = ntot % 2
        na, nb = (ntot + ms2) // 2, (ntot - ms2) // 2
        while True:
            s2 = ms2 + 2 * int(rng.integers(0, 3))
            try:
                ncsf = count_all_csfs(norb, na, nb, s2 + 1)
            except ImpossibleCIvecError:
                continue
            if ncsf > 0:
                break
        nroots = min(int(rng.integers(1, 5)), ncsf)
        h1, eri = _seeded_integrals(norb, 2 * norb, seed0 + i)
        out.append(Problem(norb, (na, nb), s2 + 1, nroots, h1, eri))
    return out


def solve_plain(problems, with_rdm=True, phases=None, **solver_attrs):
    """One problem at a time through the public FCISolver API.  phases (a
    dict, optional) accumulates the wall time of the solver's phases and of
    the RDMs."""
    out = []
    for p in problems:
        sol = FCISolver(None, smult=p.smult)
        sol.nroots = p.nroots
        for k, v in solver_attrs.items():
            setattr(sol, k, v)
        t0 = time.perf_counter()
        e, ci = sol.kernel(p.h1, p.eri, p.norb, p.nelec)
        t1 = time.perf_counter()
        cis = ci if isinstance(ci, list) else [ci]
        rdms = [sol.make_rdm12(c, p.norb, p.nelec) for c in cis] if with_rdm else None
        if phases is not None:
            for k, v in getattr(sol, "phase_s", {"kernel": t1 - t0}).items():
                phases[k] = phases.get(k, 0.0) + v
            phases["rdm"] = phases.get("rdm", 0.0) + time.perf_counter() - t1
        out.append((np.atleast_1d(e), cis, rdms))
    return out


_TRANSFORMERS = {}


def _transformer(norb, na, nb, smult):
    key = (torch.cuda.current_device(), norb, na, nb, smult)
    t = _TRANSFORMERS.get(key)
    if t is None:
        t = CSFTransformer(norb, na, nb, smult)
        _TRANSFORMERS[key] = t
    return t


def _transform_jobs(t, src, ld_src, dst, ld_dst, nvec):
    """Descriptors of the blocks of transformer ``t`` for vectors at device
    addresses src (rows of ld_src doubles) -> dst (rows of ld_dst)."""
    jobs = []
    for b in t._blocks:
        if b["ncsf"] == 0 or b["nconf"] == 0:
            continue
        j = _capi.TransformJob()
        j.x, j.y = src, dst
        j.mask = t.csd_mask.data_ptr()
        j.umat = b["umat"].data_ptr()
        j.ldx, j.ldy = ld_src, ld_dst
        j.csd_offset, j.csf_offset, j.nconf = b["csd_offset"], b["csf_offset"], b["nconf"]
        j.ndet, j.ncsf, j.nvec, j.sign = b["ndet"], b["ncsf"], nvec, b["sign"]
        jobs.append(j)
    return jobs


def _launch_transform(reverse, jobs, zjobs):
    if not jobs and not zjobs:
        return
    ja = (_capi.TransformJob * max(len(jobs), 1))(*jobs)
    za = (_capi.ZeroJob * max(len(zjobs), 1))(*zjobs)
    nbytes = len(jobs) * ctypes.sizeof(_capi.TransformJob) + len(zjobs) * ctypes.sizeof(_capi.ZeroJob)
    ws = workspace("batch_transform", nbytes)
    _capi.call("csffci_transform_batch", int(reverse), len(jobs), ja, len(zjobs), za, ptr(ws), nbytes,
               stream())


def _launch_sigma(jobs_by_norb):
    for norb, jobs in jobs_by_norb.items():
        arr = (_capi.SigmaJob * len(jobs))(*jobs)
        nbytes = _capi.query("csffci_sigma_batch_workspace", len(jobs))
        ws = workspace("batch_sigma", nbytes)
        _capi.call("csffci_sigma_batch", norb, len(jobs), arr, ptr(ws), nbytes, stream())


def _sigma_job(h2e, la, lb, ci, sigma, scratch, nelec, eta, deterministic=False):
    j = _capi.SigmaJob()
    j.h2e, j.link_a, j.link_b = h2e.data_ptr(), la.data_ptr(), lb.data_ptr()
    j.ci, j.sigma, j.scratch = ci, sigma, scratch
    j.neleca, j.nelecb = nelec
    j.sym = 1 if eta is not None else 0
    j.eta = eta if eta is not None else 1
    j.flags = _capi.SIGMA_JOB_DETERMINISTIC if deterministic else 0
    return j


def sigma_many(items, deterministic=False):
    """sigma = sum h2e[pq,rs] E_pq E_rs ci for many independent problems in
    one launch per orbital count (csffci_sigma_batch).  items: sequence of
    (h2e (npair,npair) device, ci (na*nb) device, norb, (neleca, nelecb),
    eta or None); eta asserts ci = eta ci^T (neleca == nelecb).
    deterministic: the order-independent scatter (4 <= norb <= 16; each job
    then takes three int64 digit planes of scratch).  Returns the list of
    sigma vectors."""
    jobs, outs, keep = {}, [], []
    for h2e, ci, norb, nelec, eta in items:
        nelec = (int(nelec[0]), int(nelec[1]))
        ci = ci.reshape(-1).contiguous()
        out = torch.empty_like(ci)
        if deterministic:
            scr = torch.empty(3 * ci.numel(), dtype=torch.int64, device=ci.device)
        else:
            scr = torch.empty_like(ci) if eta is not None else None
        la = D.dev_link_table(norb, nelec[0])
        lb = D.dev_link_table(norb, nelec[1])
        keep += [ci, scr]
        jobs.setdefault(int(norb), []).append(
            _sigma_job(h2e, la, lb, ci.data_ptr(), out.data_ptr(), 0 if scr is None else scr.data_ptr(),
                       nelec, eta, deterministic))
        outs.append(out)
    _launch_sigma(jobs)
    torch.cuda.current_stream().synchronize()
    return outs


def transform_many(items, reverse):
    """Batched det<->CSF transforms (csffci_transform_batch): items is a
    sequence of (CSFTransformer, x (nvec, n) device); reverse=False maps
    determinants to CSFs, True maps CSFs to determinants.  No
    normalisation."""
    jobs, zjobs, outs, keep = [], [], [], []
    for t, x in items:
        nin, nout = (t.ncsf, t.ndet) if reverse else (t.ndet, t.ncsf)
        x = x.reshape(-1, nin).contiguous()
        y = torch.empty((x.shape[0], nout), dtype=torch.float64, device=x.device)
        keep.append(x)
        if reverse:
            z = _capi.ZeroJob()
            z.y, z.ld, z.n, z.nvec = y.data_ptr(), nout, nout, x.shape[0]
            zjobs.append(z)
        jobs += _transform_jobs(t, x.data_ptr(), nin, y.data_ptr(), nout, x.shape[0])
        outs.append(y)
    _launch_transform(reverse, jobs, zjobs)
    torch.cuda.current_stream().synchronize()
    return outs


class _State:
    pass


def _call_batch(name, structs, *args):
    """Marshal a list of ctypes structures and call a batched entry point
    whose descriptor table goes to a cached workspace."""
    n = len(structs)
    if n == 0:
        return
    arr = (type(structs[0]) * n)(*structs)
    nbytes = ctypes.sizeof(arr) + 256
    ws = workspace("batch_" + name, nbytes)
    return arr, ws, nbytes


class BatchedCSFSolver:
    """Lockstep batched CSF-basis Davidson (see the module docstring)."""

    def __init__(self, conv_tol=1e-10, lindep=1e-14, max_cycle=100, max_space=12, level_shift=1e-3,
                 pspace_size=200, conv_tol_residual=None, engine="device", check_every=4, use_graph=True,
                 autotune=True, deterministic=False):
        self.conv_tol = conv_tol
        self.lindep = lindep
        self.max_cycle = max_cycle
        self.max_space = max_space
        self.level_shift = level_shift
        self.pspace_size = pspace_size
        self.conv_tol_residual = conv_tol_residual
        # "device": every Davidson step on the device (csffci_batch_plan_*,
        # one captured iteration replayed as a CUDA graph); "host": the
        # subspace algebra on the host between batched launches
        self.engine = engine
        self.check_every = check_every
        self.use_graph = use_graph
        self.autotune = autotune
        # sigma with the deterministic scatter (4 <= norb <= 16, device
        # engine): every reduction of the plan then runs in a fixed order and
        # a rerun gives the same bits
        self.deterministic = deterministic
        self.iterations = 0
        self.niter = None
        self.tile_variants = None

    # ---- batched primitives ------------------------------------------------
    def _dots(self, dots, nout):
        out = torch.empty(max(nout, 1), dtype=torch.float64, device=device())
        if dots:
            arr = (_capi.Dot * len(dots))(*dots)
            ws = workspace("batch_dots", ctypes.sizeof(arr))
            _capi.call("csffci_dots_batch", len(dots), arr, ptr(out), ptr(ws), ctypes.sizeof(arr), stream())
        return out

    def _combine(self, ops):
        if not ops:
            return
        arr = (_capi.Combine * len(ops))(*ops)
        ws = workspace("batch_combine", ctypes.sizeof(arr))
        _capi.call("csffci_combine_batch", len(ops), arr, ptr(ws), ctypes.sizeof(arr), stream())

    def _precond(self, ops):
        if not ops:
            return
        arr = (_capi.Precond * len(ops))(*ops)
        ws = workspace("batch_precond", ctypes.sizeof(arr))
        _capi.call("csffci_precond_batch", len(ops), arr, ptr(ws), ctypes.sizeof(arr), stream())

    def _transform(self, reverse, jobs, zjobs):
        _launch_transform(reverse, jobs, zjobs)

    def _sigma(self, jobs_by_norb):
        _launch_sigma(jobs_by_norb)

    @staticmethod
    def _coef(mats):
        """Upload several small host matrices at once; returns device base
        tensor and the element offset of each."""
        offs, flat = [], []
        o = 0
        for m in mats:
            m = np.ascontiguousarray(m, dtype=np.float64).ravel()
            offs.append(o)
            flat.append(m)
            o += m.size
        buf = torch.as_tensor(np.concatenate(flat) if flat else np.zeros(1), device=device())
        return buf, offs

    def _transform_jobs(self, S, src, ld_src, dst, ld_dst, nvec, reverse):
        return _transform_jobs(S.t, src, ld_src, dst, ld_dst, nvec)

    # ---- solve -------------------------------------------------------------
    def _mark(self, name):
        """Wall time of the phase that just ended (device synchronised)."""
        torch.cuda.synchronize()
        t = time.perf_counter()
        self.phase_s[name] = self.phase_s.get(name, 0.0) + t - self._t
        self._t = t

    def kernel(self, problems, with_rdm=True):
        dev = device()
        self.phase_s = {}
        torch.cuda.synchronize()
        self._t = time.perf_counter()
        states = []
        exact = []
        for ip, p in enumerate(problems):
            S = _State()
            S.ip = ip
            S.p = p
            S.norb = p.norb
            S.nelec = p.nelec
            na, nb = p.nelec
            S.t = _transformer(p.norb, na, nb, p.smult)
            S.n = S.t.ncsf
            S.ndet = S.t.ndet
            S.k = min(p.nroots, S.n)
            eri4 = eri_pair_matrix(p.eri, p.norb)
            S.eri4 = to_dev(eri4)
            S.h2e = D.dev_absorb_h1e(p.h1, eri4, p.norb, p.nelec, 0.5)
            S.hd = D.dev_make_hdiag(p.h1, p.h1, eri4, p.norb, p.nelec)
            S.hc = S.t.dev_hdiag_csf(S.hd, S.eri4)
            S.la = D.dev_link_table(p.norb, na)
            S.lb = D.dev_link_table(p.norb, nb)
            S.eta = S.t.spin_parity if na == nb else None
            if S.n <= self.pspace_size:
                exact.append(S)
            else:
                states.append(S)
        self._mark("setup")
        for S in exact:
            addr, h0 = csf_pspace(None, S.p.h1, S.p.eri, S.norb, S.nelec, S.t, hdiag_det=S.hd,
                                  hdiag_csf=S.hc, npsp=S.n)
            w, v = np.linalg.eigh(h0)
            full = np.zeros((S.k, S.n))
            full[:, addr] = v[:, :S.k].T
            S.X = torch.as_tensor(full, device=dev)
            S.e = w[:S.k]
            S.conv = [True] * S.k
        if self.engine == "device":
            self._mark("exact_pspace")
            self._device_davidson(states)
            self._mark("davidson")
        elif self.engine == "host":
            if self.deterministic:
                raise ValueError("the deterministic scatter runs with engine='device'")
            self._davidson(states)
        else:
            raise ValueError("engine must be 'device' or 'host'")
        allS = sorted(exact + states, key=lambda s: s.ip)
        out = self._finish(allS, with_rdm)
        self._mark("finish_rdm")
        return out

    def _device_davidson(self, states):
        """All problems through one csffci_batch plan: tables built once,
        iterations replayed on the device until every problem finished."""
        if not states:
            return
        dev = device()
        n = len(states)
        probs = (_capi.BatchProblem * n)()
        keep = []
        for i, S in enumerate(states):
            q = probs[i]
            q.norb, q.neleca, q.nelecb, q.nroots = S.norb, S.nelec[0], S.nelec[1], S.k
            q.eta = int(S.eta) if S.eta is not None else 0
            blocks = S.t._c_blocks()
            keep.append(blocks)
            q.nblocks = len(blocks)
            q.blocks = ctypes.addressof(blocks)
            q.csd_mask = S.t.csd_mask.data_ptr()
            q.ncsf = S.n
            q.h2e, q.link_a, q.link_b = S.h2e.data_ptr(), S.la.data_ptr(), S.lb.data_ptr()
            q.hdiag = S.hc.data_ptr()
            x0 = torch.zeros((S.k, S.n), dtype=torch.float64, device=dev)
            x0[torch.arange(S.k, device=dev), torch.argsort(S.hc, stable=True)[:S.k]] = 1.0
            keep.append(x0)
            q.x0 = x0.data_ptr()
        opt = _capi.BatchOptions(float(self.conv_tol), float(self.conv_tol_residual or 0.0), float(self.lindep),
                                 float(self.level_shift), int(self.max_space), int(self.max_cycle),
                                 int(self.check_every), 1 if self.use_graph else 0, 1 if self.autotune else 0,
                                 1 if self.deterministic else 0)
        plan = ctypes.c_void_p()
        nbytes = ctypes.c_size_t()
        _capi.call("csffci_batch_plan_create", n, probs, ctypes.byref(opt), ctypes.byref(plan), ctypes.byref(nbytes))
        try:
            arena = torch.empty(nbytes.value // 8 + 64, dtype=torch.float64, device=dev)
            base = (-arena.data_ptr()) % 256 // 8
            arena_ptr = arena.data_ptr() + 8 * base
            _capi.call("csffci_batch_plan_bind", plan, arena_ptr, nbytes.value, stream())
            it = ctypes.c_int()
            _capi.call("csffci_batch_plan_run", plan, stream(), ctypes.byref(it))
            self.iterations = it.value
            kb = _capi.query("csffci_batch_plan_max_roots", plan)
            e = np.empty(n * kb)
            conv = np.zeros(n * kb, dtype=np.int32)
            niter = np.zeros(n, dtype=np.int32)
            nfound = np.zeros(n, dtype=np.int32)
            _capi.call("csffci_batch_plan_results", plan, e.ctypes.data, conv.ctypes.data, niter.ctypes.data,
                       nfound.ctypes.data, stream())
            vn = np.zeros(32, dtype=np.int32)
            vv = np.zeros(32, dtype=np.int32)
            ng = _capi.query("csffci_batch_plan_tile_variants", plan, vn.ctypes.data, vv.ctypes.data, 32)
            self.tile_variants = {int(vn[g]): int(vv[g]) for g in range(min(ng, 32))}
            _capi.call("csffci_batch_plan_to_det", plan, stream())
            self.niter = niter
            for i, S in enumerate(states):
                kk = int(nfound[i])
                S.e = e[i * kb:i * kb + kk].copy()
                S.conv = [bool(c) for c in conv[i * kb:i * kb + kk]]
                csf, det = ctypes.c_void_p(), ctypes.c_void_p()
                _capi.call("csffci_batch_plan_vectors", plan, i, ctypes.byref(csf), ctypes.byref(det))
                oc = (csf.value - arena.data_ptr()) // 8
                od = (det.value - arena.data_ptr()) // 8
                S.X = arena[oc:oc + kk * S.n].view(kk, S.n).clone()
                S.cdet_ready = arena[od:od + kk * S.ndet].view(kk, S.ndet).clone()
        finally:
            _capi.query("csffci_batch_plan_destroy", plan)

    def _davidson(self, states):
        if not states:
            return
        dev = device()
        tol = self.conv_tol
        toloose = np.sqrt(tol) if self.conv_tol_residual is None else self.conv_tol_residual
        for S in states:
            S.space = self.max_space + S.k
            S.V = torch.empty((S.space + S.k, S.n), dtype=torch.float64, device=dev)
            S.AV = torch.empty_like(S.V)
            S.X = torch.empty((S.k, S.n), dtype=torch.float64, device=dev)
            S.AX = torch.empty_like(S.X)
            S.R = torch.empty_like(S.X)
            S.T = torch.zeros((S.k, S.n), dtype=torch.float64, device=dev)
            S.T[torch.arange(S.k, device=dev), torch.argsort(S.hc, stable=True)[:S.k]] = 1.0
            S.kT = S.k
            S.h = np.zeros((S.space + S.k, S.space + S.k))
            S.m = 0
            S.e = None
            S.e_prev = None
            S.x_prev = None
            S.conv = [False] * S.k
            S.done = False
        for it in range(self.max_cycle):
            act = [S for S in states if not S.done and S.kT > 0]
            if not act:
                break
            self.iterations = it + 1
            # (a) project the new vectors off V twice, then orthonormalise them
            # the corrections are not normalised by the preconditioner: their
            # squared norms are taken in the first pass so that the
            # linear-dependence cut below is relative (as for normalised
            # corrections in the one-problem solver)
            for ipass in range(2):
                dots, nout = [], 0
                for S in act:
                    if ipass == 0:
                        S.nbase = nout
                        for i in range(S.kT):
                            d = _capi.Dot()
                            d.x, d.y, d.hdiag = S.T[i].data_ptr(), S.T[i].data_ptr(), None
                            d.n, d.out_index = S.n, nout + i
                            dots.append(d)
                        nout += S.kT
                    S.obase = nout
                    if S.m == 0:
                        continue
                    for i in range(S.kT):
                        for j in range(S.m):
                            d = _capi.Dot()
                            d.x, d.y, d.hdiag = S.V[j].data_ptr(), S.T[i].data_ptr(), None
                            d.n, d.out_index = S.n, nout + i * S.m + j
                            dots.append(d)
                    nout += S.kT * S.m
                if dots:
                    out = self._dots(dots, nout)
                    if ipass == 0:
                        tn_dev = out
                    ops = []
                    for S in act:
                        if S.m == 0:
                            continue
                        o = _capi.Combine()
                        o.y, o.x = S.T.data_ptr(), S.V.data_ptr()
                        o.coef = out.data_ptr() + 8 * S.obase
                        o.n, o.ldx, o.ldy = S.n, S.n, S.n
                        o.ny, o.nx, o.ldc = S.kT, S.m, S.m
                        o.beta, o.scale = 1.0, -1.0
                        ops.append(o)
                    self._combine(ops)
            dots, nout = [], 0
            for S in act:
                S.gbase = nout
                for i in range(S.kT):
                    for j in range(S.kT):
                        d = _capi.Dot()
                        d.x, d.y, d.hdiag = S.T[i].data_ptr(), S.T[j].data_ptr(), None
                        d.n, d.out_index = S.n, nout + i * S.kT + j
                        dots.append(d)
                nout += S.kT * S.kT
            G = self._dots(dots, nout).cpu().numpy()
            tn = tn_dev.cpu().numpy()
            mats, owners = [], []
            for S in act:
                g = G[S.gbase:S.gbase + S.kT * S.kT].reshape(S.kT, S.kT)
                sc = 1.0 / np.sqrt(np.maximum(tn[S.nbase:S.nbase + S.kT], 1e-300))
                g = g * sc[:, None] * sc[None, :]
                w, q = np.linalg.eigh(0.5 * (g + g.T))
                keep = w > max(self.lindep, 1e-14 * max(w.max(), 0.0))
                c = (q[:, keep] / np.sqrt(w[keep])).T * sc[None, :]  # rows: orthonormal combos
                nkeep = int(keep.sum())
                if S.m + nkeep > S.space + S.k:
                    nkeep = S.space + S.k - S.m
                    c = c[-nkeep:] if nkeep > 0 else c[:0]
                S.knew = nkeep
                if nkeep == 0:
                    S.done = True
                    continue
                mats.append(c)
                owners.append(S)
            act = owners
            if not act:
                break
            cbuf, offs = self._coef(mats)
            ops = []
            for S, off in zip(act, offs):
                o = _capi.Combine()
                o.y = S.V[S.m].data_ptr()
                o.x = S.T.data_ptr()
                o.coef = cbuf.data_ptr() + 8 * off
                o.n, o.ldx, o.ldy = S.n, S.n, S.n
                o.ny, o.nx, o.ldc = S.knew, S.kT, S.kT
                o.beta, o.scale = 0.0, 1.0
                ops.append(o)
            self._combine(ops)
            # (b) H on the new vectors: CSF -> det, sigma, det -> CSF
            nd = sum(S.knew * S.ndet for S in act)
            dbuf = torch.empty(3 * nd, dtype=torch.float64, device=dev)
            o = 0
            fwd, zj, rev = [], [], []
            sjobs = {}
            for S in act:
                S.m_old = S.m
                cdet = dbuf[o:o + S.knew * S.ndet]
                sdet = dbuf[nd + o:nd + o + S.knew * S.ndet]
                sc = dbuf[2 * nd + o:2 * nd + o + S.knew * S.ndet]
                o += S.knew * S.ndet
                z = _capi.ZeroJob()
                z.y, z.ld, z.n, z.nvec = cdet.data_ptr(), S.ndet, S.ndet, S.knew
                zj.append(z)
                rev += self._transform_jobs(S, S.V[S.m].data_ptr(), S.n, cdet.data_ptr(), S.ndet, S.knew, True)
                for v in range(S.knew):
                    off = 8 * v * S.ndet
                    sjobs.setdefault(S.norb, []).append(
                        _sigma_job(S.h2e, S.la, S.lb, cdet.data_ptr() + off, sdet.data_ptr() + off,
                                   sc.data_ptr() + off, S.nelec, S.eta))
                fwd += self._transform_jobs(S, sdet.data_ptr(), S.ndet, S.AV[S.m].data_ptr(), S.n, S.knew, False)
                S.m += S.knew
            self._transform(True, rev, zj)
            self._sigma(sjobs)
            self._transform(False, fwd, [])
            del dbuf
            # (c) subspace matrices and Ritz pairs
            dots, nout = [], 0
            for S in act:
                S.hbase = nout
                for i in range(S.m):
                    for jj in range(S.m_old, S.m):
                        d = _capi.Dot()
                        d.x, d.y, d.hdiag = S.V[i].data_ptr(), S.AV[jj].data_ptr(), None
                        d.n, d.out_index = S.n, nout
                        nout += 1
                        dots.append(d)
            Hb = self._dots(dots, nout).cpu().numpy()
            cx, cr = [], []
            for S in act:
                kn = S.m - S.m_old
                blk = Hb[S.hbase:S.hbase + S.m * kn].reshape(S.m, kn)
                S.h[:S.m, S.m_old:S.m] = blk
                S.h[S.m_old:S.m, :S.m] = blk.T
                w, c = np.linalg.eigh(S.h[:S.m, :S.m])
                kk = min(S.k, S.m)
                if S.x_prev is not None and any(S.conv):
                    ov = np.abs(S.x_prev[:, :S.m] @ c)
                    idx = []
                    for i in range(ov.shape[0]):
                        order = np.argsort(-ov[i])
                        jsel = next(j for j in order if j not in idx)
                        idx.append(jsel)
                    idx = sorted(idx, key=lambda j: w[j])[:kk]
                else:
                    idx = list(range(kk))
                S.e_prev = S.e
                S.e = w[idx]
                S.cc = np.ascontiguousarray(c[:, idx].T)
                S.kk = kk
                cx.append(S.cc)
                cr.append(-S.e[:, None] * S.cc)
            cbuf, offs = self._coef(cx + cr)
            ops1, ops2 = [], []
            for i, S in enumerate(act):
                for tgt, src in ((S.X, S.V), (S.AX, S.AV), (S.R, S.AV)):
                    o = _capi.Combine()
                    o.y, o.x = tgt.data_ptr(), src.data_ptr()
                    o.coef = cbuf.data_ptr() + 8 * offs[i]
                    o.n, o.ldx, o.ldy = S.n, S.n, S.n
                    o.ny, o.nx, o.ldc = S.kk, S.m, S.m
                    o.beta, o.scale = 0.0, 1.0
                    ops1.append(o)
                o = _capi.Combine()
                o.y, o.x = S.R.data_ptr(), S.V.data_ptr()
                o.coef = cbuf.data_ptr() + 8 * offs[len(act) + i]
                o.n, o.ldx, o.ldy = S.n, S.n, S.n
                o.ny, o.nx, o.ldc = S.kk, S.m, S.m
                o.beta, o.scale = 1.0, 1.0
                ops2.append(o)
            self._combine(ops1)
            self._combine(ops2)
            dots, nout = [], 0
            for S in act:
                S.rbase = nout
                for i in range(S.kk):
                    d = _capi.Dot()
                    d.x, d.y, d.hdiag = S.R[i].data_ptr(), S.R[i].data_ptr(), None
                    d.n, d.out_index = S.n, nout
                    nout += 1
                    dots.append(d)
            rn = np.sqrt(np.maximum(self._dots(dots, nout).cpu().numpy(), 0.0))
            # (d) convergence, preconditioned corrections, restarts
            wdots, nout = [], 0
            pre = []
            for S in act:
                r = rn[S.rbase:S.rbase + S.kk]
                if S.e_prev is not None and len(S.e_prev) == len(S.e):
                    de = S.e - S.e_prev
                else:
                    de = np.full(S.kk, np.inf)
                S.conv = [bool(abs(de[i]) < tol and r[i] < toloose) for i in range(S.kk)]
                S.x_prev = np.zeros((S.kk, S.space + S.k))
                S.x_prev[:, :S.m] = S.cc
                if all(S.conv) and S.kk == S.k:
                    S.done = True
                    S.kT = 0
                    continue
                todo = [i for i in range(S.kk) if not S.conv[i]]
                S.kT = len(todo)
                for row, i in enumerate(todo):
                    es = float(S.e[i]) - self.level_shift
                    for which, (x, y) in enumerate(((S.X[i], S.R[i]), (S.X[i], S.X[i]))):
                        d = _capi.Dot()
                        d.x, d.y, d.hdiag = x.data_ptr(), y.data_ptr(), S.hc.data_ptr()
                        d.n, d.e_shift, d.out_index = S.n, es, nout + which
                        wdots.append(d)
                    q = _capi.Precond()
                    q.r, q.x, q.hdiag = S.R[i].data_ptr(), S.X[i].data_ptr(), S.hc.data_ptr()
                    q.t = S.T[row].data_ptr()
                    q.n, q.e_shift = S.n, es
                    pre.append((q, nout))  # ab patched to a device address below
                    nout += 2
                if S.m + S.kT > S.space:
                    S.restart = True
                else:
                    S.restart = False
            ab = self._dots(wdots, nout)
            for q, idx in pre:
                q.ab = ab.data_ptr() + 8 * idx
            self._precond([q for q, _ in pre])
            ops = []
            eye_mats, eye_states = [], []
            for S in act:
                if not S.done and S.restart:
                    eye_mats.append(np.eye(S.kk))
                    eye_states.append(S)
            if eye_states:
                cbuf, offs = self._coef(eye_mats)
                for S, off in zip(eye_states, offs):
                    for tgt, src in ((S.V, S.X), (S.AV, S.AX)):
                        o = _capi.Combine()
                        o.y, o.x = tgt.data_ptr(), src.data_ptr()
                        o.coef = cbuf.data_ptr() + 8 * off
                        o.n, o.ldx, o.ldy = S.n, S.n, S.n
                        o.ny, o.nx, o.ldc = S.kk, S.kk, S.kk
                        o.beta, o.scale = 0.0, 1.0
                        ops.append(o)
                self._combine(ops)
                for S in eye_states:
                    S.m = S.kk
                    S.h[:] = 0.0
                    S.h[np.arange(S.kk), np.arange(S.kk)] = S.e
                    S.x_prev = np.zeros((S.kk, S.space + S.k))
                    S.x_prev[:, :S.kk] = np.eye(S.kk)
        for S in states:
            S.X = S.X[:len(S.e)]

    def _finish(self, allS, with_rdm):
        dev = device()
        # all eigenvectors to the determinant basis in one batched launch
        nd = sum(S.X.shape[0] * S.ndet for S in allS if getattr(S, "cdet_ready", None) is None)
        dbuf = torch.empty(max(nd, 1), dtype=torch.float64, device=dev)
        o = 0
        jobs, zj = [], []
        for S in allS:
            if getattr(S, "cdet_ready", None) is not None:
                S.cdet = S.cdet_ready
                continue
            S.Xc = S.X.contiguous()
            S.cdet = dbuf[o:o + S.Xc.shape[0] * S.ndet].view(S.Xc.shape[0], S.ndet)
            o += S.Xc.shape[0] * S.ndet
            z = _capi.ZeroJob()
            z.y, z.ld, z.n, z.nvec = S.cdet.data_ptr(), S.ndet, S.ndet, S.Xc.shape[0]
            zj.append(z)
            jobs += self._transform_jobs(S, S.Xc.data_ptr(), S.n, S.cdet.data_ptr(), S.ndet, S.Xc.shape[0], True)
        self._transform(True, jobs, zj)
        results = []
        for S in allS:
            na, nb = comb(S.norb, S.nelec[0]), comb(S.norb, S.nelec[1])
            cis = []
            rdms = []
            for i in range(S.cdet.shape[0]):
                c = S.cdet[i]
                c = c / torch.linalg.vector_norm(c)
                if with_rdm:
                    d1, d2 = D.dev_rdm12(c, None, S.norb, S.nelec)
                    rdms.append((d1, d2))
                cis.append(c.reshape(na, nb))
            results.append((np.asarray(S.e), [c.cpu().numpy() for c in cis],
                            [(d1.cpu().numpy(), d2.cpu().numpy()) for d1, d2 in rdms] if with_rdm else None,
                            all(S.conv)))
        return results
