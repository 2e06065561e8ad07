"""Benchmark: CAS(16,16) singlet FP64 sigma throughput on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one sigma = sum_{pq,rs} h2e[pq,rs] E_pq E_rs c over the full
CAS(16,16) (8,8) determinant space (165,636,900 determinants, 1.33 GB per
vector), c a singlet vector produced from random CSFs (exactly what the
Davidson loop of the CSF solver feeds to sigma).  Integrals: seeded
synthetic h1/eri of rank 32 (no molecular data available offline).

Our arm: ``value`` = sigma/s with c resident in HBM (inputs 1.33 GB >> the
126 MB L2, so every step streams from HBM; no flush needed); ``e2e`` = the
same through the public API (FCISolver.contract_2e on a pinned host vector,
host->device copy of c and device->host copy of sigma inside the timed
region).  ``roofline`` reports the sigma kernel against HBM with the
algorithmic bytes 8*ndet*2*(nlink_a+nlink_b) per launch.  N>1: independent
replicas, one per GPU (the path does not shard); value is the sum.

``rdm`` (same line, rank 0 at N=1): device time of the adjoint (RDM) kernel
at CAS(16,16) (one root) and CAS(14,14) (two roots state-averaged).

``batched`` (same line, rank 0 at N=1): solves+RDMs/s of 128 seeded uneven
problems through the device-resident batched solver, next to the plain
one-problem-at-a-time GPU form on the same problems (run_batched), and the
batched det<->CSF transform throughput on their spaces.

``solves`` (same line, rank 0 at N=1): the single-problem configurations
C0-C2 end to end, beside the reference solver's timings and energies
(run_solves).

Reference arm: the reference's own CPU sigma (pyscf/lib/mcscf GAS library
with one subspace, built into oracle/_ref) on all host cores.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NORB, NELEC, RANK = 16, (8, 8), 32
WORKLOAD = "CAS(16,16) (8,8) singlet FP64 sigma"
METRIC = "CAS(16,16) FP64 sigma/s"
# smaller singlet cases of the same kernel, for profiling captures
WORKLOADS = {"cas16": (16, (8, 8), 32), "cas14": (14, (7, 7), 28), "cas12": (12, (6, 6), 24),
             "cas16_5e5e": (16, (5, 5), 32)}


# DRAM bytes (read + write) per sigma launch, by (workload, kernel), from
# one ncu capture of the dram byte counters on the full-size launch; None
# for what was not captured
TRAFFIC = {("cas16", "k_sigma_rr"): 26934597120 + 13410886400,
           ("cas16", "k_sigma_ws"): 33107436032 + 16856211456,
           ("cas16", "k_sigma_wsr"): 39177203456 + 19706565376}


def seeded_integrals(norb, rank, seed=0):
    import numpy as np
    rng = np.random.default_rng(seed)
    h1 = rng.normal(0.0, 0.3, (norb, norb))
    h1 = 0.5 * (h1 + h1.T)
    np.fill_diagonal(h1, np.linspace(-2.0, 0.5, norb))
    L = rng.normal(0.0, 0.2, (rank, norb * norb)).reshape(rank, norb, norb)
    L = 0.5 * (L + L.transpose(0, 2, 1))
    eri = 0.5 * np.einsum("xpq,xrs->pqrs", L, L)
    return h1, eri


def max_over_ranks(x, world, device="cuda"):
    """The largest of a per-rank time over all ranks (every rank returns it):
    multi-GPU numbers are reported for the slowest replica."""
    if world <= 1:
        return float(x)
    import torch
    tt = torch.tensor([float(x)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
    return float(tt.item())


def algorithmic(norb, nelec):
    from math import comb
    na, nb = nelec
    ndet = comb(norb, na) * comb(norb, nb)
    nla = na * (norb - na + 1)
    nlb = nb * (norb - nb + 1)
    npair = norb * (norb + 1) // 2
    return ndet, 8.0 * ndet * 2 * (nla + nlb), 2.0 * ndet * npair ** 2


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        import statistics
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _cpu_info():
    cores = len(os.sched_getaffinity(0))
    cpu_model = ""
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                cpu_model = ln.split(":", 1)[1].strip()
                break
    except Exception:
        pass
    return cores, cpu_model


def reference_sigma_plan(norb, nelec, h2e):
    """The reference's own CPU sigma (fci_contract_gas_plan_create/execute,
    pyscf/lib/mcscf/fci_contract_gas.c:2388-2452, one GAS subspace = the
    full CAS) on all host threads.  Used only as the timed CPU baseline and
    as the checker of the timed GPU output, never on the measured path."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import gasref
    cores, _ = _cpu_info()
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    return gasref.SigmaPlan(norb, nelec, h2e)


def bench_config(world):
    """The workload both arms report (the same dict, so that the two lines
    describe the same configuration)."""
    ndet = algorithmic(NORB, NELEC)[0]
    return {"workload": WORKLOAD, "norb": NORB, "nelec": list(NELEC), "eri_rank": RANK, "ndet": ndet,
            "vector": "normalised singlet-symmetric CI vector (c = c^T), seeded",
            "l2": "inputs 1.33 GB >> 126 MB L2 (no flush needed)",
            "parallelism": "replicas%d" % world}


def run_reference(args, rank_env):
    """Reference arm: the reference's own CPU sigma on the benchmark's
    workload, on all host threads of rank 0.  One full CAS(16,16) sigma
    takes tens of seconds, so the arm times as many whole sigmas as fit in
    about 90 s (at least one, at most --steps) and reports that count as
    ``steps``; no warm-up is needed for a CPU library call (the plan is
    built before the timed loop)."""
    import numpy as np
    rank, world = rank_env
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import restate as R
    from math import comb
    h1, eri = seeded_integrals(NORB, RANK)
    h2e = R.absorb_h1e(h1, eri, NORB, NELEC, 0.5)
    plan = reference_sigma_plan(NORB, NELEC, h2e)
    n = comb(NORB, NELEC[0])
    c = np.random.default_rng(1).normal(size=(n, n))
    c += c.T
    c /= np.linalg.norm(c)
    budget = 90.0
    nsig, t0 = 0, time.perf_counter()
    while True:
        plan(c)
        nsig += 1
        el = time.perf_counter() - t0
        if nsig >= max(1, args.steps) or el + el / nsig > budget:
            break
    plan.close()
    value = nsig / el
    cores, cpu_model = _cpu_info()
    sample = "%d full CAS(16,16) (8,8) sigma(s) in %.1f s on %d threads (%s)" % (nsig, el, cores, cpu_model)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "sigma/s",
            "n_gpus": world, "steps": nsig, "warmup": 0, "requested_steps": args.steps,
            "requested_warmup": args.warmup, "ms_per_step": 1000.0 * el / nsig, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(world),
            "cpu_baseline": {"value": value, "unit": "sigma/s", "cores": cores, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "sigma/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank_env):
    import numpy as np
    import torch
    rank, world = rank_env
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    import pyscf_forge_b200 as P
    from pyscf_forge_b200 import _capi
    from pyscf_forge_b200.fci import direct_spin1 as D
    from pyscf_forge_b200.csf_fci.csfstring import CSFTransformer
    sys.path.insert(0, os.path.join(ROOT, "oracle"))

    NORB, NELEC, RANK = WORKLOADS[args.workload]
    h1, eri = seeded_integrals(NORB, RANK)
    sol = P.csf_solver(None, smult=1)
    sol.norb, sol.nelec = NORB, NELEC
    sol.check_transformer_cache()
    t = sol.transformer
    h2eff = sol.absorb_h1e(h1, eri, NORB, NELEC, 0.5)
    g = torch.Generator(device="cpu").manual_seed(1 + rank)
    x = torch.randn(t.ncsf, generator=g, dtype=torch.float64).cuda()
    c = t.dev_csf2det(x)[0]
    c /= torch.linalg.norm(c)
    eta = t.spin_parity
    del x
    out = torch.empty_like(c)
    ndet, B, F = algorithmic(NORB, NELEC)

    def step():
        D.dev_contract_2e(h2eff.h2e, c, NORB, NELEC, eta=eta, out=out)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    barrier()
    _capi.profile_enable(True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        barrier()
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        barrier()
    prof = _capi.profile_report()
    _capi.profile_enable(False)
    ms = e0.elapsed_time(e1) / args.steps
    ms = max_over_ranks(ms, world)
    value = world * 1000.0 / ms
    kname = next((k for k in ("k_sigma_wsr", "k_sigma_wsr_bulk", "k_sigma_ws", "k_sigma_rr", "k_sigma")
                  if k in prof), "k_sigma_rr")
    k_cnt, k_ms = prof.get(kname, (0, 0.0))
    traffic = TRAFFIC.get((args.workload, kname))
    k_avg_ms = k_ms / max(k_cnt, 1)
    launches = sum(v[0] for v in prof.values())

    if args.no_e2e:
        print(json.dumps({"workload": args.workload, "ms_per_step": ms, "kernel_ms": k_avg_ms}), flush=True)
        return
    # end-to-end through the public API: pinned host vector in, sigma into a
    # reused pinned host buffer (out=); both copies are inside the timed loop
    ch = torch.empty(ndet, dtype=torch.float64).pin_memory()
    ch.copy_(c.cpu())  # contract_2e detects the singlet symmetry of ch on the device
    res = torch.empty(ndet, dtype=torch.float64).pin_memory()
    e2e_steps = max(1, min(args.steps, 3))
    sol.contract_2e(h2eff, ch, NORB, NELEC, out=res)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        sol.contract_2e(h2eff, ch, NORB, NELEC, out=res)
    barrier()
    e2e_ms = (time.perf_counter() - t0) * 1000.0 / e2e_steps
    e2e_ms = max_over_ranks(e2e_ms, world)
    # the public-API result must equal the device step
    step()
    torch.cuda.synchronize()
    err = float((res.to(out.device) - out).abs().max())
    assert err < 1e-9, err

    hbm, src = peaks()
    achieved = B / (k_avg_ms * 1e-3) / 1e9
    dmma = _capi.fp64_peak(0)
    line = {"metric": METRIC, "value": value, "unit": "sigma/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded rank-32 integrals, random singlet CSF vector)",
            "config": bench_config(world),
            "e2e": {"value": world * 1000.0 / e2e_ms, "unit": "sigma/s",
                    "h2d_bytes_per_step": ndet * 8, "d2h_bytes_per_step": ndet * 8,
                    "note": "FCISolver.contract_2e, pinned host vector in, pinned host buffer out (out=)"},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": traffic,
                         "kernel": kname,
                         "algorithmic_bytes": B,
                         "flops": F, "tflops": F / (k_avg_ms * 1e-3) / 1e12,
                         "flops_formed": F / 2, "dmma_peak_tflops": dmma,
                         "frac_dmma": (F / 2) / (k_avg_ms * 1e-3) / 1e12 / dmma,
                         "dmma_note": "singlet lower triangle forms F/2; DMMA peak measured live "
                                      "(register-only m8n8k4 loop, csffci_fp64_peak)",
                         "peak_note": "hbm_gbs %s (MEASURED_PEAKS.json)" % src},
            "clocks": clk.summary()}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # one full reference sigma on the host, on the very vector the timed
        # loop used: the measured CPU baseline, and the check of the timed
        # output against the reference
        h2e_np = h2eff.h2e.cpu().numpy()
        c_np = c.cpu().numpy()
        plan = reference_sigma_plan(NORB, NELEC, h2e_np)
        t0 = time.perf_counter()
        ref = plan(c_np)
        t_ref = time.perf_counter() - t0
        plan.close()
        ref_d = torch.as_tensor(ref, device=out.device)
        del ref, c_np
        line["max_abs_err_vs_reference"] = float((out - ref_d).abs().max())
        line["max_abs_sigma"] = float(ref_d.abs().max())
        del ref_d
        cores, cpu_model = _cpu_info()
        line["cpu_baseline"] = {"value": 1.0 / t_ref, "unit": "sigma/s", "cores": cores, "kind": "reference",
                                "sample": "1 full CAS(16,16) (8,8) sigma of the benchmark's own vector in "
                                          "%.1f s on %d threads (%s)" % (t_ref, cores, cpu_model)}
    if rank == 0 and world == 1 and not args.no_rdm:
        line["rdm"] = run_rdm(dmma)
    if rank == 0 and world == 1 and not args.no_batched:
        line["batched"] = run_batched(args.batch)
        line["batched"]["transforms"] = run_batch_transforms()
        line["solves"] = run_solves()
    if rank == 0 and world == 1 and not args.no_c4:
        line["c4"] = run_c4(ref_check=not args.no_cpu_baseline)
    if rank == 0 and world == 1 and not args.no_rdm:
        line["transforms"] = run_transforms()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_rdm(dmma_peak, cases=None):
    """The adjoint (RDM) kernel on the sizes of the large configurations,
    device-timed: the CAS(16,16) singlet 2-RDM of one root, and the
    state-averaged 1-/2-RDMs of two CAS(14,14) (7,7) roots (the backward of
    the differentiable state-averaged energy).  Vectors are random unit
    vectors of those spaces (the kernel's cost does not depend on them)."""
    import torch
    from math import comb
    from pyscf_forge_b200.fci import direct_spin1 as D
    out = {}
    for tag, norb, nelec, nroots in (("cas16_singlet_1root", 16, (8, 8), 1), ("cas14_sa2", 14, (7, 7), 2)):
        if cases and tag not in cases:
            continue
        n = comb(norb, nelec[0]) * comb(norb, nelec[1])
        g = torch.Generator(device="cuda").manual_seed(3)
        cs = [torch.randn(n, dtype=torch.float64, device="cuda", generator=g) for _ in range(nroots)]
        cs = [c / torch.linalg.norm(c) for c in cs]
        D.dev_rdm12(cs[0], None, norb, nelec)  # warm-up (workspace)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        dm1 = dm2 = None
        for c in cs:
            d1, d2 = D.dev_rdm12(c, None, norb, nelec)
            dm1 = d1 / nroots if dm1 is None else dm1 + d1 / nroots
            dm2 = d2 / nroots if dm2 is None else dm2 + d2 / nroots
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        flops = nroots * 2.0 * n * norb ** 4
        out[tag] = {"ms": ms, "determinants": n, "roots": nroots,
                    "gram_tflops": flops / (ms * 1e-3) / 1e12,
                    "frac_dmma": flops / (ms * 1e-3) / 1e12 / dmma_peak,
                    "trace_dm1": float(torch.trace(dm1))}
    out["note"] = ("adjoint = transition-density / RDM kernel: T slabs <J|E_pq|c> built in shared memory, "
                   "Gram on FP64 DMMA (bra == ket: symmetric half), 1-RDM from the Gram; flops counted "
                   "as the dense 2*ndet*norb^4")
    return out


def run_transforms(workload="cas16", nvecs=(1, 4), reps=5):
    """The det<->CSF transforms (csffci_det2csf / csffci_csf2det: per npair
    block a GEMM with the csd_mask gather or scatter fused into it) on the
    singlet space of a workload, device-timed, with the fraction of the HBM
    roofline on the compulsory bytes 8*(ndet+ncsf) + 4*ndet per vector."""
    import torch
    from pyscf_forge_b200 import _capi
    from pyscf_forge_b200.csf_fci.csfstring import CSFTransformer
    norb, nelec, _ = WORKLOADS[workload]
    t = CSFTransformer(norb, nelec[0], nelec[1], 1)
    hbm, src = peaks()
    out = {"workload": "%s singlet (ndet %d, ncsf %d)" % (workload, t.ndet, t.ncsf)}
    for nv in nvecs:
        g = torch.Generator(device="cpu").manual_seed(7)
        x = torch.randn(nv, t.ncsf, generator=g, dtype=torch.float64).cuda()
        d = t.dev_csf2det(x)
        torch.cuda.synchronize()
        for name, fn, arg in (("csf2det", t.dev_csf2det, x), ("det2csf", t.dev_det2csf, d)):
            fn(arg)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                fn(arg)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            _capi.profile_enable(True)
            fn(arg)
            prof = _capi.profile_report()
            _capi.profile_enable(False)
            byts = nv * (8.0 * (t.ndet + t.ncsf) + 4.0 * t.ndet)
            out["%s_nvec%d" % (name, nv)] = {"ms": ms, "GBps": byts / (ms * 1e-3) / 1e9,
                                             "frac_hbm": byts / (ms * 1e-3) / 1e9 / hbm,
                                             "kernel_ms": {k: round(v[1], 3) for k, v in prof.items()}}
        del x, d
    out["peak_note"] = "hbm_gbs %s" % src
    return out


C4_MAX_SPACE = 40
C4_MAX_CYCLE = 300


def run_c4(ref_check=True):
    """The large configuration: CAS(16,16) (8,8) singlet, 4 roots
    state-averaged with equal weights.  The solve is FCISolver.kernel (the
    reference's kernel, pyscf/csf_fci/csf.py:368-497: CSF diagonal,
    p-space, Olsen preconditioner, Davidson on hop = csf2det . sigma .
    det2csf) reached through the differentiable energy; the backward of the
    state-averaged energy then runs the 1-/2-RDM kernel on every root.
    Reported: solve and backward seconds, Davidson iterations and sigmas,
    the device memory peak, device time per kernel, and the checks
      * |H c_k - E_k c_k| of every root (the library's sigma),
      * tr dm1 = N and sum_pr dm2[p,p,r,r] = N(N-1) of the averaged RDMs,
      * E_SA = sum h1 * dE/dh1 + sum eri * dE/deri (H is linear in h1, eri),
      * with ref_check, <c_0|H|c_0> and |H c_0 - E_0 c_0| with the
        reference's own CPU sigma on the host."""
    import numpy as np
    import torch
    from pyscf_forge_b200 import _capi
    from pyscf_forge_b200.autograd import csf_fci_energy
    from pyscf_forge_b200.csf_fci.csf import FCISolver
    from pyscf_forge_b200.fci import direct_spin1 as D
    norb, nelec, rank, nroots = 16, (8, 8), 32, 4
    h1, eri = seeded_integrals(norb, rank)
    h1t = torch.tensor(h1, requires_grad=True)
    erit = torch.tensor(eri, requires_grad=True)
    sol = FCISolver(None, smult=1)
    # the seeded integrals are weakly diagonally dominant (as the batched
    # configuration's, see run_batched): a larger subspace than the
    # reference's default 12 is what converges four roots
    sol.max_space = C4_MAX_SPACE
    sol.max_cycle = C4_MAX_CYCLE
    torch.cuda.synchronize()
    torch.cuda.reset_peak_memory_stats()
    _capi.profile_enable(True)
    t0 = time.perf_counter()
    E = csf_fci_energy(h1t, erit, norb, nelec, smult=1, nroots=nroots, solver=sol)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    w = torch.full((nroots,), 1.0 / nroots, dtype=torch.float64)
    e_sa = (w * E).sum()
    e_sa.backward()
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    prof = _capi.profile_report()
    _capi.profile_enable(False)
    peak = torch.cuda.max_memory_allocated()
    gh1, geri = h1t.grad.numpy(), erit.grad.numpy()
    n = sum(nelec)
    dm1 = gh1.T
    dm2 = 2.0 * geri
    out = {"workload": "CAS(16,16) (8,8) singlet, %d roots state-averaged (equal weights), "
                       "seeded rank-32 integrals" % nroots,
           "energies": [float(x) for x in E.detach()], "e_sa": float(e_sa.detach()),
           "solver": "conv_tol 1e-10, max_space %d, max_cycle %d" % (C4_MAX_SPACE, C4_MAX_CYCLE),
           "converged": [bool(x) for x in np.atleast_1d(sol.converged)],
           "solve_s": t1 - t0, "rdm_backward_s": t2 - t1, "sigmas": int(getattr(sol, "nsigma", 0)),
           "davidson_iterations": int(getattr(sol, "niter", 0)),
           "device_peak_gb": peak / 1e9, "hbm_budget_gb": 180.0,
           "trace_dm1_minus_n": float(np.trace(dm1) - n),
           "trace_dm2_minus_n_n1": float(np.einsum("pprr->", dm2) - n * (n - 1)),
           "energy_from_gradients_minus_e_sa": float(np.sum(h1 * gh1) + np.sum(eri * geri) - float(e_sa.detach())),
           "kernel_ms": {k: round(v[1], 3) for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])},
           "kernel_launches": {k: v[0] for k, v in prof.items()}}
    h2e = sol.absorb_h1e(h1, eri, norb, nelec, 0.5).h2e
    res = []
    for k, c in enumerate(sol.ci):
        c = c.reshape(-1)
        hc = D.dev_contract_2e(h2e, c, norb, nelec)
        res.append(float(torch.linalg.norm(hc - float(E[k].detach()) * c)))
        del hc
    out["residual_norms"] = res
    if ref_check:
        import restate as R
        c0 = sol.ci[0].reshape(-1).cpu().numpy()
        plan = reference_sigma_plan(norb, nelec, R.absorb_h1e(h1, eri, norb, nelec, 0.5))
        hc0 = plan(c0)
        plan.close()
        e0 = float(np.dot(c0, hc0) / np.dot(c0, c0))
        out["reference_check_root0"] = {
            "rayleigh_quotient_minus_e0": e0 - float(E[0].detach()),
            "residual_norm": float(np.linalg.norm(hc0 - float(E[0].detach()) * c0)),
            "note": "the reference's CPU sigma (libfci_gas, one GAS subspace) applied to root 0"}
    return out


SOLVE_CONFIGS = {"C0": (8, (4, 4), 1, 1, 16), "C1": (12, (6, 6), 1, 3, 24), "C2": (14, (7, 7), 3, 2, 28)}


def run_solves():
    """The single-problem configurations C0 (norb 8 (4,4) singlet, 1 root),
    C1 (norb 12 (6,6) singlet, 3 roots) and C2 (norb 14 (7,7) triplet, 2
    roots), seeded integrals of rank 16/24/28: a fresh FCISolver.kernel plus
    make_rdm12 of every root, end to end (host integrals in, host energies,
    CI vectors and RDMs out), timed on the second of two runs.  Settings are
    those of the reference timing (conv_tol 1e-10, max_cycle 400,
    max_space 30).  Beside each: the reference's own csf.py kernel +
    make_rdm12 on the same problem (tests/golden/ref_solves_c0_c2.jsonl,
    made by oracle/time_reference_solves.py in the build container on 8
    threads: a reported baseline from another host) and the energy
    difference from it."""
    import numpy as np
    import torch
    import pyscf_forge_b200 as P
    ref = {}
    path = os.path.join(ROOT, "tests", "golden", "ref_solves_c0_c2.jsonl")
    if os.path.exists(path):
        for l in open(path):
            d = json.loads(l)
            ref[d["config"]] = d
    out = {}
    for tag, (norb, nelec, smult, nroots, rank) in SOLVE_CONFIGS.items():
        h1, eri = seeded_integrals(norb, rank)
        for _ in range(2):
            sol = P.csf_solver(None, smult=smult)
            sol.nroots, sol.conv_tol, sol.max_cycle, sol.max_space = nroots, 1e-10, 400, 30
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e, ci = sol.kernel(h1, eri, norb, nelec)
            cis = ci if isinstance(ci, list) else [ci]
            rdms = [sol.make_rdm12(c, norb, nelec) for c in cis]
            torch.cuda.synchronize()
            t = time.perf_counter() - t0
        e = np.atleast_1d(np.asarray(e, dtype=float))
        row = {"seconds": t, "solves_rdms_per_s": 1.0 / t, "energies": [float(x) for x in e],
               "converged": [bool(x) for x in np.atleast_1d(sol.converged)],
               "trace_dm1_minus_n": max(abs(float(np.trace(r[0])) - sum(nelec)) for r in rdms)}
        if tag in ref:
            r = ref[tag]
            row["max_abs_dE_vs_reference"] = float(np.max(np.abs(e - np.asarray(r["energies"]))))
            rs = r["solve_s"] + r["rdm_s"]
            row["reference_cpu"] = {"seconds": rs, "threads": r["threads"],
                                    "note": "reference csf.py kernel + make_rdm12 on the stand-in, build "
                                            "container, not this host"}
            row["speedup_vs_reference_cpu"] = rs / t
        out[tag] = row
    return out


def run_batch_transforms(reps=3):
    """The batched det<->CSF transforms (csffci_transform_batch, one launch
    over every problem) on the CSF spaces of the 128-problem batch, one
    vector per root, device-timed per launch (k_transform_batch), with the
    fraction of the HBM roofline on the compulsory bytes 8*(ndet+ncsf) +
    4*ndet per vector."""
    import numpy as np
    import torch
    from pyscf_forge_b200 import _capi
    from pyscf_forge_b200 import batched as Bt
    from pyscf_forge_b200.csf_fci.csfstring import CSFTransformer
    hbm, src = peaks()
    g = torch.Generator(device="cpu").manual_seed(11)
    items, nbytes = [], 0
    for p in Bt.make_uneven_batch(128):
        t = CSFTransformer(p.norb, p.nelec[0], p.nelec[1], p.smult)
        x = torch.randn(p.nroots, t.ncsf, generator=g, dtype=torch.float64).cuda()
        items.append((t, x))
        nbytes += p.nroots * (8 * (t.ndet + t.ncsf) + 4 * t.ndet)
    dets = Bt.transform_many(items, reverse=True)
    back = [(t, d) for (t, _), d in zip(items, dets)]
    out = {"workload": "C3 batch spaces, one vector per root (%d vectors)" % sum(x.shape[0] for _, x in items),
           "algorithmic_bytes": nbytes}
    for name, its, rev in (("csf2det", items, True), ("det2csf", back, False)):
        Bt.transform_many(its, reverse=rev)
        _capi.profile_enable(True)
        for _ in range(reps):
            Bt.transform_many(its, reverse=rev)
        prof = _capi.profile_report()
        _capi.profile_enable(False)
        n, tot = prof.get("k_transform_batch", (0, 0.0))
        ms = tot / max(n, 1)
        out[name] = {"kernel_ms": round(ms, 4), "GBps": nbytes / ms / 1e6, "frac_hbm": nbytes / ms / 1e6 / hbm}
    err = max(float((y - x).abs().max()) for (_, x), y in zip(items, Bt.transform_many(back, reverse=False)))
    out["round_trip_max_abs_err"] = err
    out["peak_note"] = "hbm_gbs %s" % src
    return out


def run_batched(nprob):
    """Batched uneven solves: nprob seeded problems (norb 6..12, 1-4 roots,
    several spins), energies and 1-/2-RDMs of every root, through the
    device-resident batched solver (one captured Davidson iteration replayed
    for all problems) and through the plain one-problem-at-a-time GPU form
    (FCISolver.kernel + make_rdm12 per problem).  Both are end to end: host
    integrals in, host energies / CI vectors / RDMs out.  Solver settings
    are conv_tol 1e-10 (residual sqrt(conv_tol)), level shift 1e-3,
    max_cycle 400 and max_space 30: with the reference's max_space 12 one
    of these problems does not converge in 400 iterations, in the
    reference's iteration as in ours (weakly diagonally dominant seeded
    integrals and a 5 mEh gap above its second root).  Energies are compared
    with the reference's own solver on the stand-in
    (tests/golden/c3_batch128.npz, same settings), whose CPU time per
    problem, measured where the fixture was made, is reported beside."""
    import numpy as np
    import torch
    from pyscf_forge_b200 import batched as Bt
    probs = Bt.make_uneven_batch(nprob)
    kw = dict(conv_tol=1e-10, max_cycle=400, max_space=30)
    Bt.BatchedCSFSolver(**kw).kernel(probs)  # warm-up: transformers, autotuner
    Bt.solve_plain(probs[:8], **kw)
    torch.cuda.synchronize()
    from pyscf_forge_b200 import _capi
    sol = Bt.BatchedCSFSolver(**kw)
    _capi.profile_enable(True)
    t0 = time.perf_counter()
    rb = sol.kernel(probs)
    torch.cuda.synchronize()
    tb = time.perf_counter() - t0
    prof = _capi.profile_report()
    _capi.profile_enable(False)
    plain_phases = {}
    t0 = time.perf_counter()
    rp = Bt.solve_plain(probs, phases=plain_phases, **kw)
    torch.cuda.synchronize()
    tp = time.perf_counter() - t0
    de = max(float(np.max(np.abs(a[0] - b[0]))) for a, b in zip(rb, rp))
    conv = [bool(np.all(a[3])) for a in rb]
    de_conv = max([float(np.max(np.abs(a[0] - b[0]))) for a, b, c in zip(rb, rp, conv) if c] or [0.0])
    nroots = sum(len(a[0]) for a in rb)
    ref = {}
    gpath = os.path.join(ROOT, "tests", "golden", "c3_batch128.npz")
    if nprob == 128 and os.path.exists(gpath):
        g = np.load(gpath)
        dref = max(float(np.max(np.abs(np.asarray(a[0]) - g["energies"][i, :len(a[0])])))
                   for i, a in enumerate(rb))
        ref = {"max_abs_dE_vs_reference": dref,
               "reference_cpu": {"solves_per_s": 128.0 / float(g["wall_seconds"]),
                                 "cpu_seconds_solve_plus_rdm": float(np.sum(g["seconds"][:, 1])),
                                 "workers": int(g["workers"]),
                                 "note": "the reference's csf.py kernel + make_rdm12 on the PySCF stand-in "
                                         "(reference C sigma/RDMs), one problem per worker process, one "
                                         "thread each; measured in the build container where the fixture "
                                         "was made, not on this host"}}
    return {"metric": "batched solves+RDMs/s", "value": nprob / tb, "unit": "solves/s",
            "plain_value": nprob / tp, "speedup_vs_plain": tp / tb, "seconds": tb, "plain_seconds": tp,
            "problems": nprob, "roots": nroots, "converged_problems": int(sum(bool(a[3]) for a in rb)),
            "iterations": sol.iterations, "phase_s": {k: round(v, 4) for k, v in sol.phase_s.items()},
            "plain_phase_s": {k: round(v, 4) for k, v in plain_phases.items()},
            "kernel_ms": {k: round(v[1], 2) for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])[:12]},
            "max_abs_dE_vs_plain": de,
            "max_abs_dE_vs_plain_converged": de_conv,
            "tile_variants": {str(k): v for k, v in (sol.tile_variants or {}).items()},
            **ref,
            "config": {"workload": "%d uneven problems, norb 6..12, nelec within +-2 of half filling, "
                                   "S in {0,1,2}, 1-4 roots, seeded rank-2*norb integrals" % nprob,
                       "solver": "conv_tol 1e-10, max_cycle 400, max_space 30",
                       "plain": "FCISolver.kernel + make_rdm12 per root, one problem at a time",
                       "e2e": "host integrals in, host energies/CI/RDMs out (both forms)"}}


def run_batch_sigma(norbs, variants, steps=3):
    """Per-launch time of the batched sigma (csffci_sigma_batch) of the C3
    problems of the given orbital counts, one job per root with a seeded
    random vector (symmetrised for equal electron counts, as the solver's
    vectors are), for each sigma kernel variant (CSFFCI_SIGMA_VARIANT)."""
    import numpy as np
    import torch
    from math import comb
    from pyscf_forge_b200 import _capi
    from pyscf_forge_b200 import batched as Bt
    from pyscf_forge_b200.fci import direct_spin1 as D
    from pyscf_forge_b200._runtime import eri_pair_matrix
    rng = np.random.default_rng(1)
    items = []
    for p in Bt.make_uneven_batch(128):
        if p.norb not in norbs:
            continue
        na, nb = comb(p.norb, p.nelec[0]), comb(p.norb, p.nelec[1])
        h2e = D.dev_absorb_h1e(p.h1, eri_pair_matrix(p.eri, p.norb), p.norb, p.nelec, 0.5)
        eta = (-1 if p.smult == 3 else 1) if p.nelec[0] == p.nelec[1] else None
        for _ in range(p.nroots):
            c = rng.standard_normal((na, nb))
            if eta is not None:
                c = c + eta * c.T
            items.append((h2e, torch.as_tensor(c.ravel(), device="cuda"), p.norb, p.nelec, eta))
    old = os.environ.get("CSFFCI_SIGMA_VARIANT")
    out = {"workload": "C3 batch, norb %s: %d jobs (one per root)" % (sorted(norbs), len(items)), "variants": {}}
    ref = None
    try:
        for v in variants:
            os.environ["CSFFCI_SIGMA_VARIANT"] = str(v)
            res = Bt.sigma_many(items)  # warm-up (and the result to compare)
            if ref is None:
                ref = [r.clone() for r in res]
            err = max(float((a - b).abs().max()) for a, b in zip(res, ref))
            _capi.profile_enable(True)
            for _ in range(steps):
                Bt.sigma_many(items)
            prof = _capi.profile_report()
            _capi.profile_enable(False)
            out["variants"][str(v)] = {"max_abs_diff_vs_first": err,
                                       "ms_per_launch": {k: round(t[1] / t[0], 3) for k, t in sorted(prof.items())
                                                         if "sigma" in k}}
    finally:
        if old is None:
            os.environ.pop("CSFFCI_SIGMA_VARIANT", None)
        else:
            os.environ["CSFFCI_SIGMA_VARIANT"] = old
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="cas16", choices=sorted(WORKLOADS),
                    help="cas16 is the benchmark; the smaller ones exist for profiling captures")
    ap.add_argument("--no-e2e", action="store_true", help="time the device loop only (profiling)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-solves measurement")
    ap.add_argument("--no-rdm", action="store_true", help="skip the RDM (adjoint) timing")
    ap.add_argument("--no-c4", action="store_true", help="skip the CAS(16,16) 4-root solve + RDM backward")
    ap.add_argument("--c4-only", action="store_true", help="only the CAS(16,16) 4-root solve + RDM backward")
    ap.add_argument("--c4-max-cycle", type=int, default=None, help="Davidson iterations of the C4 solve")
    ap.add_argument("--transforms-only", action="store_true",
                    help="only the det<->CSF transform timing of --workload (profiling captures)")
    ap.add_argument("--rdm-only", default="", help="only the RDM timing of these cases "
                    "(cas16_singlet_1root,cas14_sa2), for profiling captures")
    ap.add_argument("--batch", type=int, default=128, help="problems in the batched-solves measurement")
    ap.add_argument("--batch-sigma-only", default="", help="only the batched sigma launches of the C3 "
                    "problems of these orbital counts (e.g. 10,11,12), per kernel variant")
    ap.add_argument("--sigma-variants", default="0,1,2,3,4,7", help="variants for --batch-sigma-only")
    args = ap.parse_args()
    global C4_MAX_CYCLE
    if args.c4_max_cycle:
        C4_MAX_CYCLE = args.c4_max_cycle
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference(args, (rank, world))
        return
    if args.transforms_only:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        if rank == 0:
            print(json.dumps(run_transforms(args.workload)), flush=True)
        return
    if args.c4_only:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        if rank == 0:
            print(json.dumps(run_c4(ref_check=not args.no_cpu_baseline)), flush=True)
        return
    if args.batch_sigma_only:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        if rank == 0:
            print(json.dumps(run_batch_sigma({int(x) for x in args.batch_sigma_only.split(",")},
                                             [int(x) for x in args.sigma_variants.split(",")])), flush=True)
        return
    if args.rdm_only:
        # the adjoint timing alone (profiling captures of the RDM kernels)
        import torch
        from pyscf_forge_b200 import _capi
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        if rank == 0:
            print(json.dumps(run_rdm(_capi.fp64_peak(0), args.rdm_only.split(","))), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, (rank, world))
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
