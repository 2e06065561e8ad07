// Pieces shared by the warp-specialised sigma kernels (sigma_ws.cu: one MMA
// warp per m-tile of 8 rows; sigma_wsr.cu: 16-row MMA warps with the
// registers re-split between the roles): the named-barrier helpers, the row
// setup both roles run, and the mover role (copies, beta gather, beta
// scatter) over a ring of three D/V and link stages.
//
// Barrier ids (the protocol of both kernels, restated on the CPU in
// tests/test_ws_protocol.py):
//   1+s  "D of the tile in stage s is gathered": movers arrive, MMA warps wait
//   4+s  "V of the tile in stage s is written":  MMA warps arrive, movers wait
//   7    movers among themselves
//   8    MMA warps among themselves (every MMA warp has read D before V
//        overwrites it)
//   9    every thread: row boundaries (the row setup both roles share)
#pragma once
#include "sigma_rr_kernel.cuh"

namespace csffci {

__device__ __forceinline__ void ws_bar_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(nthreads) : "memory");
}

__device__ __forceinline__ void ws_bar_arrive(int id, int nthreads) {
  asm volatile("bar.arrive %0, %1;\n" ::"r"(id), "r"(nthreads) : "memory");
}

__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// m8n8k4 FP64 MMA accumulating into (c0, c1): A row g col t, B row t col g
__device__ __forceinline__ void ws_dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

constexpr int WS_NB = 16;     // columns per tile
constexpr int WS_STAGES = 3;  // ring of D/V and link buffers

// ---- bulk copies of the alpha rows (global -> shared on this GPU, no
//      multicast), completed on one mbarrier per stage ----------------------
__device__ __forceinline__ unsigned ws_smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void ws_mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(ws_smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void ws_mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// one arrival that also announces the bytes the stage's copies will deliver
__device__ __forceinline__ void ws_mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(ws_smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool ws_mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(ws_smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// src and dst 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void ws_bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   ws_smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(ws_smem_addr(bar))
               : "memory");
}

// generic-proxy accesses of shared memory before this point are ordered
// before later async-proxy (bulk copy) accesses
__device__ __forceinline__ void ws_fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// try_wait polls allowed before a stage's copies count as lost
constexpr long long WS_MBAR_POLLS = 1ll << 22;

// The shared state of the row Ja a CTA works on.
struct WSShared {
  double* Dbuf;
  csffci_link_t* Lbuf;
  double* crow;
  RRAlpha* al;
  int* zl;
  unsigned* pneg;
  int* zf;
  RRRow* srow;
  long long* apoff;  // per pair row: Ka*Nb of its alpha link in row Ja, -1 without one
  unsigned long long* mbar;  // one mbarrier per stage (bulk alpha-row copies)
  csffci_sigma_job_t* job;   // job-table kernels: the current unit's job ...
  int* jst;                  // ... its index in the table and whether it is live
};

// One step of the grid-stride loop: row unit ru and, from g.split_from on
// (the last, partial round of the grid), which of two tile ranges of it.
struct WSUnit {
  long long ru;
  int part, parts;
};

__device__ __forceinline__ WSUnit ws_unit(const RRArgs& g, long long u) {
  WSUnit r;
  r.ru = u;
  r.part = 0;
  r.parts = 1;
  if (u >= g.split_from) {  // two tile ranges per row unit
    const long long k = u - g.split_from;
    r.ru = g.split_from + (k >> 1);
    r.part = (int)(k & 1);
    r.parts = 2;
  }
  return r;
}

// Job-table kernels: thread 0 finds the job that owns row unit ru (units
// only grow along a CTA's loop, so the search goes forward from the last
// job) and copies it to shared memory; both roles call this with the same
// ru and return the same answer: whether the job is live (a gated job, whose
// problem has no new vector this iteration, is skipped as a whole).
template <int NTH>
__device__ __forceinline__ bool ws_batch_job(const RRArgs& g, const WSShared& S, long long ru, int tid) {
  ws_bar_sync(9, NTH);  // every thread is done with the previous unit's job record
  if (tid == 0) {
    int j = S.jst[0] < 0 ? 0 : S.jst[0];
    while (j + 1 < g.njobs && g.jobs[j + 1].unit_begin <= ru) ++j;
    if (j != S.jst[0]) {
      *S.job = g.jobs[j];
      S.jst[0] = j;
    }
    const csffci_sigma_job_t& J = *S.job;
    S.jst[1] = J.live == nullptr || J.live_index < *J.live;
  }
  ws_bar_sync(9, NTH);
  return S.jst[1] != 0;
}

// Row setup shared by both roles (every thread of the CTA calls it with the
// same arguments, and it synchronises the CTA on barrier 9): the alpha links
// of row Ja, the rows without one, the sign masks of this row (in half par
// of pneg) and the copy of c row Ja.  Returns false (for every thread) when
// the spin-symmetric unit has no second row.  lu is the job's own row unit;
// a unit of the last, partial round of the grid (parts == 2) is one of two
// tile ranges [c0, c0 + nchunk) of it, so that the last round spreads over
// every SM.
template <int NTH, int NB>
__device__ __forceinline__ bool ws_row_setup(const RRArgs& g, const WSShared& S, const csffci_sigma_job_t& sjob,
                                             long long lu, int part, int parts, int w, int par, int tid,
                                             int warp, int lane) {
  const long long Nb = sjob.Nb;
  const int nla = sjob.nla, npair = g.npair, ds = g.ds;
  long long ja = lu;
  if (sjob.sym && w == 1) {
    ja = sjob.Na - 1 - lu;
    if (ja <= lu) return false;
  }
  unsigned* const pcur = S.pneg + par * npair;
  ws_bar_sync(9, NTH);  // the previous row is fully consumed
  if (tid == 0) {
    S.srow->ja = ja;
    S.srow->jend = sjob.sym ? ja + 1 : Nb;
    const int nt = (int)((S.srow->jend + NB - 1) / NB);
    S.srow->c0 = parts == 2 && part ? nt / 2 : 0;
    S.srow->nchunk = parts == 2 && !part ? nt / 2 : nt - S.srow->c0;
    S.srow->pc = par * npair;
  }
  for (int r = tid; r < npair; r += NTH) {
    pcur[r] = 0u;
    S.zf[r] = 1;
    S.apoff[r] = -1;
  }
  ws_bar_sync(9, NTH);
  for (int l = tid; l < nla; l += NTH) {
    const uint2 e = rr_link(&sjob.link_a[ja * nla + l]);
    const int pr = rr_lpair(e);
    RRAlpha a;
    a.off = (long long)e.x * Nb;
    a.drow = pr * ds;
    a.neg = rr_lneg(e);
    S.al[l] = a;
    pcur[pr] = a.neg;
    S.zf[pr] = 0;
    S.apoff[pr] = a.off;
  }
  for (long long i = tid; i < Nb; i += NTH) cp_async8(&S.crow[i], &sjob.ci[ja * Nb + i]);
  cp_async_commit();
  ws_bar_sync(9, NTH);
  if (warp == 0) {
    int n = 0;
    for (int base = 0; base < npair; base += 32) {
      const int r = base + lane;
      const bool z = r < npair && S.zf[r];
      const unsigned bal = __ballot_sync(0xffffffffu, z);
      if (z) S.zl[n + __popc(bal & ((1u << lane) - 1u))] = r * ds;
      n += __popc(bal);
    }
    if (lane == 0) S.srow->nzero = n;
  }
  return true;
}

// The mover role of a warp-specialised sigma kernel: NMOV warps (the last
// ones of the CTA, mtid = their thread index among the movers).  For tile c
// of a row: issue the copies of tile c (alpha rows of c, beta link rows,
// zero rows), finish the beta gather of tile c-1, and scatter V of tile
// c-2 through the beta links.  RU links per thread and pass are handled
// together, every load of the pass issued before the dependent ones (a
// mover is often the only warp of the role on its scheduler, so this
// instruction-level parallelism is its way to hide latency).
template <int NTH, int NMOV, int RU, bool BATCH, bool DET = false>
__device__ __forceinline__ void ws_mover_role(const RRArgs& g, const WSShared& S, int tid, int warp, int lane,
                                              int mtid, int mwarp) {
  constexpr int NB = WS_NB;
  constexpr int MTH = NMOV * 32;   // mover threads
  constexpr int MPASS = MTH / NB;  // link rows per mover pass (threads over the NB columns)
  const int ds = g.ds, LS = g.ls;
  const size_t dsz = (size_t)g.nd_rows * ds, lsz = (size_t)NB * LS;
  const int jl = mtid % NB, ml = mtid / NB;
  int par = 0;
  unsigned mphase = 0;  // parity to wait for next, per stage (bulk copies)
  for (long long u = blockIdx.x; u < g.total_units; u += gridDim.x) {
    const WSUnit un = ws_unit(g, u);
    if (BATCH && !ws_batch_job<NTH>(g, S, un.ru, tid)) continue;
    const csffci_sigma_job_t& sjob = BATCH ? *S.job : g.job0;
    const long long lu = un.ru - sjob.unit_begin;
    for (int w = 0; w < (sjob.sym ? 2 : 1); ++w) {
      if (!ws_row_setup<NTH, NB>(g, S, sjob, lu, un.part, un.parts, w, par, tid, warp, lane)) break;
      par ^= 1;
      cp_async_wait_all();
      ws_bar_sync(9, NTH);
      const RRRow& srow = *S.srow;
      const int nch = srow.nchunk, c0 = srow.c0;  // local tiles c, global tiles c0 + c
      const long long jend = srow.jend, ja = srow.ja, Nb = sjob.Nb;
      const int nla = sjob.nla, nlb = sjob.nlb, nz = srow.nzero;
      const unsigned* pc = S.pneg + srow.pc;
      const bool SYM = sjob.sym != 0;
      // the deterministic scatter writes the digit planes in scratch, whose
      // planes are Na*Nb apart (a job table's) or g.det_stride (one problem)
      double* const out = (SYM || DET) ? sjob.scratch : sjob.sigma;
      const long long dstr = BATCH ? sjob.Na * sjob.Nb : g.det_stride;
      for (int c = 0; c <= nch + 1; ++c) {
        // every mover has finished step c-1 (its scatter read the stage
        // that the copies below refill)
        ws_bar_sync(7, MTH);
        if (c < nch) {
          // copies of tile c into stage c % 3 (its last tile, c-3, was
          // scattered at step c-1): alpha rows of c, beta links, zero rows
          const int s = c % WS_STAGES;
          double* Dd = S.Dbuf + s * dsz;
          csffci_link_t* Ld = S.Lbuf + s * lsz;
          const long long j1 = (long long)(c0 + c) * NB;
          const int nc = (int)min((long long)NB, jend - j1);
          if (g.bulk) {
            // one mover warp hands the alpha rows of tile c to the bulk-copy
            // engine: row l is c[Ka_l][j1 .. j1+nc) rounded up to an even
            // count (16-byte size; the extra column is in bounds because Nb
            // is even and only lands in a column the scatters skip)
            if (mwarp == 0) {
              const unsigned rowbytes = (unsigned)((nc + 1) & ~1) * 8u;
              if (lane == 0) {
                ws_fence_proxy_async();
                ws_mbar_expect_tx(&S.mbar[s], rowbytes * (unsigned)nla);
              }
              __syncwarp();
              for (int l = lane; l < nla; l += 32) {
                const RRAlpha a = S.al[l];
                ws_bulk_g2s(&Dd[a.drow], sjob.ci + a.off + j1, rowbytes, &S.mbar[s]);
              }
            }
          } else if (jl < nc) {
            const double* src = sjob.ci + j1 + jl;
            for (int l0 = ml; l0 < nla; l0 += RU * MPASS) {
              RRAlpha a[RU];
#pragma unroll
              for (int k = 0; k < RU; ++k) a[k] = S.al[min(l0 + k * MPASS, nla - 1)];
#pragma unroll
              for (int k = 0; k < RU; ++k)
                if (l0 + k * MPASS < nla) cp_async8(&Dd[a[k].drow + jl], src + a[k].off);
            }
          }
          const csffci_link_t* lsrc = sjob.link_b + j1 * nlb;
          for (int jb = mwarp; jb < nc; jb += NMOV)
            for (int m = lane; m < nlb; m += 32) cp_async8(&Ld[jb * LS + m], &lsrc[(long long)jb * nlb + m]);
          cp_async_commit();
          const int zr = lane / (NB / 2), zc = 2 * (lane % (NB / 2));
          for (int i = mwarp * 4 + zr; i < nz; i += NMOV * 4)
            *reinterpret_cast<double2*>(&Dd[S.zl[i] + zc]) = make_double2(0.0, 0.0);
        }
        if (c >= 1 && c - 1 < nch) {
          // gather of tile c-1: its copies have landed (the newest group,
          // tile c, may still be in flight)
          if (c < nch) cp_async_wait_one();
          else cp_async_wait_all();
          const int s = (c - 1) % WS_STAGES;
          if (g.bulk) {
            // the alpha rows of tile c-1 have landed (bounded wait: a stage
            // whose copies never complete poisons this row's sigma with NaN
            // and the kernel goes on, so that no barrier is left waiting)
            const unsigned parity = (mphase >> s) & 1u;
            long long polls = 0;
            while (!ws_mbar_try_wait(&S.mbar[s], parity))
              if (++polls > WS_MBAR_POLLS) {
                if (mtid == 0) atomicAdd(&(SYM ? sjob.scratch : sjob.sigma)[ja * Nb], __longlong_as_double(0x7ff8000000000000ll));
                break;
              }
            mphase ^= 1u << s;
          }
          ws_bar_sync(7, MTH);
          double* D = S.Dbuf + s * dsz;
          const csffci_link_t* Lt = S.Lbuf + s * lsz;
          const int ncol = (int)min((long long)NB, jend - (long long)(c0 + c - 1) * NB);
          if (jl < ncol)
            for (int m0 = ml; m0 < nlb; m0 += RU * MPASS) {
              // distinct links of a column have distinct pairs, so the
              // read-modify-writes of a pass do not overlap
              uint2 e[RU];
              double v[RU], d[RU];
              unsigned f[RU];
#pragma unroll
              for (int k = 0; k < RU; ++k) {
                const int m = m0 + k * MPASS;
                e[k] = m < nlb ? rr_link(&Lt[jl * LS + m]) : make_uint2(0u, 0u);
              }
#pragma unroll
              for (int k = 0; k < RU; ++k) {
                v[k] = S.crow[e[k].x];
                f[k] = rr_lneg(e[k]) ^ pc[rr_lpair(e[k])];
                d[k] = D[rr_lpair(e[k]) * ds + jl];
              }
#pragma unroll
              for (int k = 0; k < RU; ++k)
                if (m0 + k * MPASS < nlb) D[rr_lpair(e[k]) * ds + jl] = d[k] + rr_flip(v[k], f[k]);
            }
          if (g.bulk) ws_fence_proxy_async();
          ws_bar_arrive(1 + s, NTH);  // D of tile c-1 is gathered
        }
        if (c >= 2) {
          // scatter of tile c-2
          const int s = (c - 2) % WS_STAGES;
          ws_bar_sync(4 + s, NTH);  // V of tile c-2 is written
          const double* D = S.Dbuf + s * dsz;
          const csffci_link_t* Lt = S.Lbuf + s * lsz;
          const long long j0 = (long long)(c0 + c - 2) * NB;
          const int ncol = (int)min((long long)NB, jend - j0);
          if (jl < ncol) {
            double* const orow = out + ja * Nb;
            for (int m0 = ml; m0 < nlb; m0 += RU * MPASS) {
              uint2 e[RU];
              double v[RU];
#pragma unroll
              for (int k = 0; k < RU; ++k) {
                const int m = m0 + k * MPASS;
                e[k] = m < nlb ? rr_link(&Lt[jl * LS + m]) : make_uint2(0u, 0u);
              }
#pragma unroll
              for (int k = 0; k < RU; ++k) v[k] = D[rr_lpair(e[k]) * ds + jl];
#pragma unroll
              for (int k = 0; k < RU; ++k)
                if (m0 + k * MPASS < nlb) ws_out_add<DET>(&orow[e[k].x], rr_flip(v[k], rr_lneg(e[k])), dstr);
            }
          }
        }
      }
    }
  }
}

// Shared-memory carve-up of a warp-specialised kernel (same layout for both
// kernels; extra_bytes are appended for a kernel's own buffers and their
// offset returned in *extra_off).  Returns 0 when it does not fit.
size_t ws_layout(RRArgs& g, int npair, int rows_multiple, long long max_nb, int max_nla, int max_nlb,
                 size_t extra_bytes, unsigned* extra_off);

// The grid strides over the row units, so with nru units and a grid of G
// CTAs the last round has nru % G units and leaves the other SMs idle for
// a whole unit.  Those units are cut in two tile ranges each: the last
// round then spreads over twice as many CTAs.  The earlier units stay whole
// (every unit reloads its row of c, so cutting them all would double that).
inline void ws_split_last_round(RRArgs& g, long long grid) {
  const long long nru = g.total_units;
  const long long tail = grid > 0 ? nru % grid : 0;
  if (nru <= grid || tail == 0) return;
  g.split_from = nru - tail;
  g.parts = 2;  // ws_row_setup cuts these units in two
  g.total_units = g.split_from + tail * 2;
}

// whether the alpha rows of one problem can go through the bulk-copy
// engine: 16-byte aligned rows of c (ci 16-byte aligned, Nb even)
inline bool ws_bulk_ok(const csffci_sigma_job_t& J) {
  return ((uintptr_t)J.ci & 15u) == 0 && (J.Nb & 1) == 0;
}

}  // namespace csffci
