// Register-resident sigma kernel template (k_sigma_rr) and its launcher,
// shared by the tile-shape variant translation units sigma_rr_v*.cu; the
// algorithm and layouts are described in sigma_rr.cu.
#pragma once
#include <stdlib.h>
#include <string.h>

#include "batch_internal.cuh"
#include "common.cuh"
#include "profile.cuh"

namespace csffci {

__device__ __forceinline__ void cp_async8(void* s, const void* gsrc) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gsrc) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

struct RRArgs {
  const csffci_sigma_job_t* jobs;  // device array (njobs > 1) ...
  csffci_sigma_job_t job0;         // ... or the single job by value
  int njobs;
  long long total_units;
  int npair, ds, ls, nd_rows;
  unsigned off_d, off_l, off_crow, off_al, off_zl, off_pn, off_zf;
  unsigned off_ap;     // warp-specialised kernels: per-pair alpha offsets
  unsigned off_extra;  // register-split kernel: tail partial sums
  unsigned off_mbar;   // warp-specialised kernels: one mbarrier per stage
  int bulk;            // warp-specialised kernels: alpha rows by bulk copy
  int parts;           // warp-specialised kernels: parts of each row unit from split_from on
  long long split_from;  // warp-specialised kernels: first row unit cut into parts
  long long det_stride;  // deterministic mode: elements between the digit planes (0: FP64 atomics)
};

// Deterministic scatter: x = d2 2^6 + d1 2^-37 + d0 2^-80 with integer
// digits |d_k| <= 2^42 (for |x| < 2^48; larger x up to 2^55 only widens
// d2), each added to its own int64 plane by an integer atomic.  Integer
// addition is associative, so the plane sums do not depend on the order of
// the contributions.  Every step is exact except the rounding of d0 (below
// 2^-80), which depends on x alone: x - 64 h2 and r1 - 2^-37 h1 are exactly
// representable (the remainder keeps the low bits of x), so fma returns
// them without rounding.
__device__ __forceinline__ void det_add3(double* p, long long stride, double x) {
  const double h2 = rint(x * 0x1p-6);
  const double r1 = fma(-h2, 0x1p6, x);
  const double h1 = rint(r1 * 0x1p37);
  const double r0 = fma(-h1, 0x1p-37, r1);
  const double h0 = rint(r0 * 0x1p80);
  unsigned long long* w = reinterpret_cast<unsigned long long*>(p);
  atomicAdd(w, (unsigned long long)(long long)h0);
  atomicAdd(w + stride, (unsigned long long)(long long)h1);
  atomicAdd(w + 2 * stride, (unsigned long long)(long long)h2);
}

// one scattered contribution: an FP64 atomic, or the three digit atomics
template <bool DET>
__device__ __forceinline__ void ws_out_add(double* p, double x, long long stride) {
  if (DET) det_add3(p, stride, x);
  else atomicAdd(p, x);
}

// Alpha link of the current row Ja as the tile loops use it: the offset
// Ka*Nb of its row of c (copies) and of sigma (alpha scatter), the offset
// of its pair row in the D tile, and its sign as a mask on the high word.
struct RRAlpha {
  long long off;
  int drow;
  unsigned neg;
};

// x with its sign flipped where the mask (0 or 0x80000000) is set
__device__ __forceinline__ double rr_flip(double x, unsigned mask) {
  return __hiloint2double(__double2hiint(x) ^ (int)mask, __double2loint(x));
}

// state of the row Ja a CTA is working on (uniform over the CTA)
struct RRRow {
  long long ja, jend;
  int nchunk, nzero, pc;
  int c0;  // warp-specialised kernels: first tile of the row's part
};

// link entry as two words: addr, then op | sign << 16 | pair << 24 (the
// pair index hi*(hi+1)/2+lo is written by csffci_link_table)
__device__ __forceinline__ uint2 rr_link(const csffci_link_t* p) { return *reinterpret_cast<const uint2*>(p); }
__device__ __forceinline__ int rr_lpair(uint2 w) { return (int)(w.y >> 24); }
__device__ __forceinline__ unsigned rr_lneg(uint2 w) { return (w.y << 8) & 0x80000000u; }

// m16n8k4 FP64 MMA: A 16x4 (a0: row g, a1: row g+8; col t), B 4x8 (row t,
// col g), C 16x8 (c0,c1: row g, cols 2t,2t+1; c2,c3: row g+8), g = lane/4,
// t = lane%4.
__device__ __forceinline__ void rr_dmma16(double (&c)[4], double a0, double a1, double b) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(b));
}

__device__ __forceinline__ void rr_dmma8(double (&c)[4], double a0, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(c[0]), "+d"(c[1])
      : "d"(a0), "d"(b));
}

// KS k-steps of 4 (npair rounded up to a multiple of 4); MT m-tiles of MW
// (8 or 16) output rows; NT n-tiles of 8 columns per tile.
// CTAs per SM the register allocation is sized for: the (16, 4) and (8, 4)
// shapes keep every register they need (one CTA per SM); the two-n-tile
// shapes cap registers so that small orbital counts, whose CTAs have few
// warps, run two or three CTAs per SM.
template <int MT, int MW, int NT>
constexpr int rr_min_blocks() {
  return NT == 2 ? (MW == 16 ? (MT <= 5 ? 3 : MT <= 6 ? 2 : 1) : (MT <= 10 ? 2 : 1)) : 1;
}

// Warps of a CTA.  Warp w runs on scheduler w mod 4 of the SM, and each
// scheduler has its own FP64 MMA pipe, so the MMA phase lasts as long as the
// busiest scheduler's share.  One warp per m-tile leaves that share uneven
// when MT mod 4 is 1 or 2 (17 m-tiles: 5, 4, 4, 4 warps); there the last
// m-tiles are split along their n-tiles over SF warps each, which fills the
// CTA to a multiple of four warps with equal MMA counts per scheduler.  Only
// one-CTA-per-SM shapes are split (with several CTAs per SM the warps of the
// CTAs interleave over the schedulers), and the warps per scheduler, hence
// the register budget, do not change.
template <int MT, int MW, int NT>
struct RRLayout {
  static constexpr int q = MT / 4, r = MT % 4;
  static constexpr bool split = rr_min_blocks<MT, MW, NT>() == 1 && q >= 1 && (r == 1 || r == 2);
  static constexpr int SF = !split ? 1 : (r == 1 ? (NT >= 4 ? 4 : NT) : (NT >= 2 ? 2 : 1));
  static constexpr int NW = split ? 4 * q + r * SF : MT;
  static constexpr int NTS = NT / SF;  // n-tiles of a warp on a split m-tile
};

template <int KS, int MT, int MW, int NT, bool BATCH>
__global__ void __launch_bounds__(RRLayout<MT, MW, NT>::NW * 32, (rr_min_blocks<MT, MW, NT>()))
    k_sigma_rr(RRArgs g) {
  using L = RRLayout<MT, MW, NT>;
  constexpr int NW = L::NW;
  constexpr int NTH = NW * 32;
  constexpr int NB = 8 * NT;
  constexpr int MPW = 32 / NB;       // link rows per warp pass (lanes over NB columns)
  constexpr int ZPW = 64 / NB;       // zero rows per warp pass (16-byte stores)
  extern __shared__ __align__(16) unsigned char smraw[];
  double* Dbuf = (double*)(smraw + g.off_d);
  csffci_link_t* Lbuf = (csffci_link_t*)(smraw + g.off_l);
  double* crow = (double*)(smraw + g.off_crow);
  RRAlpha* al = (RRAlpha*)(smraw + g.off_al);
  int* zl = (int*)(smraw + g.off_zl);             // D-row offsets of the rows without an alpha link
  unsigned* pneg = (unsigned*)(smraw + g.off_pn);  // [2][npair] alpha sign masks of two rows
  int* zf = (int*)(smraw + g.off_zf);             // 1 where a pair row has no alpha link

  __shared__ csffci_sigma_job_t sjob_s;
  __shared__ int sjob_idx, sjob_live;
  __shared__ RRRow srow;
  // the single-problem launch reads its job from the parameter bank
  const csffci_sigma_job_t& sjob = BATCH ? sjob_s : g.job0;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  // this warp's m-tile and, on a split m-tile, its first n-tile
  const bool part = L::split && warp >= 4 * L::q;
  const int mt = part ? 4 * L::q + (warp - 4 * L::q) / L::SF : warp;
  const int t0 = part ? ((warp - 4 * L::q) % L::SF) * L::NTS : 0;
  const int ds = g.ds, LS = g.ls, npair = g.npair;
  const int ndr = g.nd_rows;
  const size_t dsz = (size_t)ndr * ds, lsz = (size_t)NB * LS;

  // h2e rows MW*mt+g (and +8), columns 4s+t of the current job, resident in
  // registers; each column carries the alpha sign of its pair row in the
  // current row Ja (A' = h2e diag(s), so that the alpha rows of the D tile
  // are copied without their signs)
  double a0f[KS], a1f[MW == 16 ? KS : 1];
  // rows past npair are k rows of the MMA that nothing else writes
  for (int i = tid; i < (ndr - npair) * ds; i += NTH) {
    Dbuf[npair * ds + i] = 0.0;
    Dbuf[dsz + npair * ds + i] = 0.0;
  }
  int cur = -1;
  bool fresh = true;  // a0f holds h2e without signs
  int par = 0;        // which half of pneg holds the current row's signs
  __shared__ int sjob_loaded;
  if (BATCH && tid == 0) sjob_loaded = -1;

  for (long long u = blockIdx.x; u < g.total_units; u += gridDim.x) {
    if (BATCH) {
      __syncthreads();  // everything of the previous unit is consumed
      if (tid == 0) {
        int j = sjob_loaded < 0 ? 0 : sjob_loaded;
        while (j + 1 < g.njobs && g.jobs[j + 1].unit_begin <= u) ++j;
        if (j != sjob_loaded) {
          sjob_s = g.jobs[j];
          sjob_loaded = j;
        }
        sjob_idx = j;
        sjob_live = sjob_s.live == nullptr || sjob_s.live_index < *sjob_s.live;
      }
      __syncthreads();
      if (!sjob_live) continue;  // a gated job: uniform over the block
    }
    if ((BATCH ? sjob_idx : 0) != cur) {
      cur = BATCH ? sjob_idx : 0;
      const double* h2e = sjob.h2e;
      const int r0 = mt * MW + gq, r1 = r0 + 8;
#pragma unroll
      for (int s = 0; s < KS; ++s) {
        const int c = 4 * s + tq;
        a0f[s] = (r0 < npair && c < npair) ? h2e[(long long)r0 * npair + c] : 0.0;
        if (MW == 16) a1f[s] = (r1 < npair && c < npair) ? h2e[(long long)r1 * npair + c] : 0.0;
      }
      fresh = true;
    }
    const long long lu = u - sjob.unit_begin;
    for (int w = 0; w < (sjob.sym ? 2 : 1); ++w) {
      {
        // row setup; the tile loop below keeps almost nothing in registers
        // across the MMA (the A fragments fill the register budget at 16
        // orbitals) and reads the row's state back from shared memory
        const long long Nb = sjob.Nb;
        const int nla = sjob.nla;
        long long ja = lu;
        if (sjob.sym && w == 1) {
          ja = sjob.Na - 1 - lu;
          if (ja <= lu) break;
        }
        unsigned* const pcur = pneg + par * npair;
        const unsigned* const pold = pneg + (par ^ 1) * npair;
        __syncthreads();  // the previous row is fully consumed
        if (tid == 0) {
          srow.ja = ja;
          srow.jend = sjob.sym ? ja + 1 : Nb;
          srow.nchunk = (int)((srow.jend + NB - 1) / NB);
          srow.pc = par * npair;
        }
        for (int r = tid; r < npair; r += NTH) {
          pcur[r] = 0u;
          zf[r] = 1;
        }
        __syncthreads();
        for (int l = tid; l < nla; l += NTH) {
          const uint2 e = rr_link(&sjob.link_a[ja * nla + l]);
          const int pr = rr_lpair(e);
          RRAlpha a;
          a.off = (long long)e.x * Nb;
          a.drow = pr * ds;
          a.neg = rr_lneg(e);
          al[l] = a;
          pcur[pr] = a.neg;
          zf[pr] = 0;
        }
        for (long long i = tid; i < Nb; i += NTH) cp_async8(&crow[i], &sjob.ci[ja * Nb + i]);
        __syncthreads();
        // the rows without an alpha link, compacted by warp 0
        if (warp == 0) {
          int n = 0;
          for (int base = 0; base < npair; base += 32) {
            const int r = base + lane;
            const bool z = r < npair && zf[r];
            const unsigned bal = __ballot_sync(0xffffffffu, z);
            if (z) zl[n + __popc(bal & ((1u << lane) - 1u))] = r * ds;
            n += __popc(bal);
          }
          if (lane == 0) srow.nzero = n;
        }
        // sign columns of A: flip where this row's alpha sign differs from
        // the one the registers carry
#pragma unroll
        for (int s = 0; s < KS; ++s) {
          const int c = 4 * s + tq;
          if (c < npair && ((fresh ? 0u : pold[c]) ^ pcur[c])) {
            a0f[s] = -a0f[s];
            if (MW == 16) a1f[s] = -a1f[s];
          }
        }
        fresh = false;
        par ^= 1;
        __syncthreads();
      }
      // copies of one tile: alpha rows of c (unsigned), beta links; zero rows
      auto issue = [&](int bb, long long j1) {
        double* Dd = Dbuf + bb * dsz;
        csffci_link_t* Ld = Lbuf + bb * lsz;
        const int nc = (int)min((long long)NB, srow.jend - j1);
        const int jl = lane % NB;
        if (jl < nc) {
          const double* src = sjob.ci + j1 + jl;
          for (int l = warp * MPW + lane / NB; l < sjob.nla; l += NW * MPW) {
            const RRAlpha a = al[l];
            cp_async8(&Dd[a.drow + jl], src + a.off);
          }
        }
        const int nlb = sjob.nlb;
        const csffci_link_t* lsrc = sjob.link_b + j1 * nlb;
        for (int jb = warp; jb < nc; jb += NW)
          for (int m = lane; m < nlb; m += 32) cp_async8(&Ld[jb * LS + m], &lsrc[(long long)jb * nlb + m]);
        cp_async_commit();
        // (the buffer being filled is idle: its last reads, the scatters two
        // tiles back, ended before the barrier that opened this tile)
        const int zr = lane / (NB / 2), zc = 2 * (lane % (NB / 2));
        for (int i = warp * ZPW + zr; i < srow.nzero; i += NW * ZPW)
          *reinterpret_cast<double2*>(&Dd[zl[i] + zc]) = make_double2(0.0, 0.0);
      };
      issue(0, 0);
      for (int ch = 0; ch < srow.nchunk; ++ch) {
        const int b = ch & 1;
        cp_async_wait_all();
        __syncthreads();
        {
          // beta gather D[pq][Jb] += sign s(pq) c[Ja][Kb] (the alpha sign s
          // of the pair row is undone by A')
          double* D = Dbuf + b * dsz;
          const csffci_link_t* Lt = Lbuf + b * lsz;
          const unsigned* pc = pneg + srow.pc;
          const int ncol = (int)min((long long)NB, srow.jend - (long long)ch * NB);
          const int jl = lane % NB, nlb = sjob.nlb;
          if (jl < ncol)
            for (int m = warp * MPW + lane / NB; m < nlb; m += NW * MPW) {
              const uint2 e = rr_link(&Lt[jl * LS + m]);
              const int pr = rr_lpair(e);
              D[pr * ds + jl] += rr_flip(crow[e.x], rr_lneg(e) ^ pc[pr]);
            }
        }
        __syncthreads();
        if (ch + 1 < srow.nchunk) issue(b ^ 1, (long long)(ch + 1) * NB);
        // V = A' D on the FP64 tensor cores
        double acc[NT][4];
#pragma unroll
        for (int t = 0; t < NT; ++t) acc[t][0] = acc[t][1] = acc[t][2] = acc[t][3] = 0.0;
        {
          const double* Db = Dbuf + b * dsz + tq * ds + gq + 8 * t0;
          if (!part) {
#pragma unroll
            for (int s = 0; s < KS; ++s) {
              if (MW == 16) {
#pragma unroll
                for (int t = 0; t < NT; ++t) rr_dmma16(acc[t], a0f[s], a1f[s], Db[4 * s * ds + 8 * t]);
              } else {
#pragma unroll
                for (int t = 0; t < NT; ++t) rr_dmma8(acc[t], a0f[s], Db[4 * s * ds + 8 * t]);
              }
            }
          } else {
#pragma unroll
            for (int s = 0; s < KS; ++s) {
              if (MW == 16) {
#pragma unroll
                for (int t = 0; t < L::NTS; ++t) rr_dmma16(acc[t], a0f[s], a1f[s], Db[4 * s * ds + 8 * t]);
              } else {
#pragma unroll
                for (int t = 0; t < L::NTS; ++t) rr_dmma8(acc[t], a0f[s], Db[4 * s * ds + 8 * t]);
              }
            }
          }
        }
        __syncthreads();
        {
          const int r0 = mt * MW + gq, r1 = r0 + 8;
          const int ntw = part ? L::NTS : NT;
          double* V = Dbuf + b * dsz + 8 * t0 + 2 * tq;
#pragma unroll
          for (int t = 0; t < NT; ++t) {
            if (t < ntw) {
              if (r0 < npair) {
                V[r0 * ds + 8 * t] = acc[t][0];
                V[r0 * ds + 8 * t + 1] = acc[t][1];
              }
              if (MW == 16 && r1 < npair) {
                V[r1 * ds + 8 * t] = acc[t][2];
                V[r1 * ds + 8 * t + 1] = acc[t][3];
              }
            }
          }
        }
        __syncthreads();
        {
          const double* D = Dbuf + b * dsz;
          const csffci_link_t* Lt = Lbuf + b * lsz;
          const long long j0 = (long long)ch * NB, ja = srow.ja;
          const int ncol = (int)min((long long)NB, srow.jend - j0);
          const int jl = lane % NB, ml = lane / NB;
          const bool SYM = sjob.sym != 0;
          double* const out = SYM ? sjob.scratch : sjob.sigma;
          if (jl < ncol) {
            // row-local scatter through the beta links of each column
            double* const orow = out + ja * sjob.Nb;
            const int nlb = sjob.nlb;
            for (int m = warp * MPW + ml; m < nlb; m += NW * MPW) {
              const uint2 e = rr_link(&Lt[jl * LS + m]);
              atomicAdd(&orow[e.x], rr_flip(D[rr_lpair(e) * ds + jl], rr_lneg(e)));
            }
            // alpha scatter sigma[Ka][Jb] through the links of Ja (coalesced
            // over Jb); in the spin-symmetric mode only Jb < Ja
            const long long J = j0 + jl;
            if (!SYM || J < ja) {
              double* const ocol = out + J;
              const int nla = sjob.nla;
              for (int l = warp * MPW + ml; l < nla; l += NW * MPW) {
                const RRAlpha a = al[l];
                atomicAdd(&ocol[a.off], rr_flip(D[a.drow + jl], a.neg));
              }
            }
          }
        }
      }
    }
  }
}

inline int norb_of_npair(int npair) {
  int n = 0;
  while (n * (n + 1) / 2 < npair) ++n;
  return n <= 16 ? n : 0;
}

template <int KS, int MT, int MW, int NT>
static int launch_rr(RRArgs& g, size_t smem, cudaStream_t stream) {
  constexpr int NW = RRLayout<MT, MW, NT>::NW;
  auto kern = g.jobs ? k_sigma_rr<KS, MT, MW, NT, true> : k_sigma_rr<KS, MT, MW, NT, false>;
  CSF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev = 0, nsm = 148, per_sm = 1;
  CSF_CUDA(cudaGetDevice(&dev));
  CSF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  CSF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NW * 32, smem));
  if (per_sm < 1) {
    set_error("sigma: register-resident kernel does not fit on an SM (smem %zu)", smem);
    return CSFFCI_ERR_INVALID;
  }
  long long grid = (long long)nsm * per_sm;
  if (grid > g.total_units) grid = g.total_units;
  if (grid < 1) return CSFFCI_OK;
  static const char* names[17] = {"k_sigma_rr",     "k_sigma_rr",     "k_sigma_rr",     "k_sigma_rr",
                                  "k_sigma_rr_n4",  "k_sigma_rr_n5",  "k_sigma_rr_n6",  "k_sigma_rr_n7",
                                  "k_sigma_rr_n8",  "k_sigma_rr_n9",  "k_sigma_rr_n10", "k_sigma_rr_n11",
                                  "k_sigma_rr_n12", "k_sigma_rr_n13", "k_sigma_rr_n14", "k_sigma_rr_n15",
                                  "k_sigma_rr_n16"};
  ProfScope ps(g.jobs ? names[norb_of_npair(g.npair)] : "k_sigma_rr", stream);
  kern<<<(int)grid, NW * 32, smem, stream>>>(g);
  return check_launch("sigma (register-resident)");
}

// tile-shape variants: (rows per warp, n-tiles of 8 columns)
constexpr int RR_NVARIANT = 4;
// the warp-specialised kernel (sigma_ws.cu), 4..16 orbitals, one problem
// or a job table: one MMA warp per 8 rows (variant 4) or, up to 12
// orbitals, per 16 rows in CTAs of 8 warps (variant 7)
constexpr int RR_VARIANT_WS = 4;
constexpr int RR_VARIANT_WS16 = 7;
bool sigma_ws_supported(int norb);
bool sigma_ws16_supported(int norb);
int sigma_ws_launch(int norb, int njobs, const csffci_sigma_job_t* jobs_dev, const csffci_sigma_job_t& job0,
                    long long total_units, long long max_nb, int max_nla, int max_nlb, cudaStream_t stream,
                    int mw, long long det_stride = 0);
// the warp-specialised kernel with registers re-split between the roles
// (sigma_wsr.cu), one problem at 16 orbitals
constexpr int RR_VARIANT_WSR = 5;
// the same with the alpha rows moved by the bulk-copy engine
constexpr int RR_VARIANT_WSR_BULK = 6;
bool sigma_wsr_supported(int norb);
int sigma_wsr_launch(int norb, const csffci_sigma_job_t& job0, long long total_units, long long max_nb,
                     int max_nla, int max_nlb, cudaStream_t stream, bool bulk);
bool rr_variant_valid(int norb, int v);
// the variants a job table may run: the tile shapes and the warp-specialised kernel
bool batch_variant_valid(int norb, int v);
int rr_default_variant(int norb);
int sigma_rr_launch(int norb, int njobs, const csffci_sigma_job_t* jobs_dev, const csffci_sigma_job_t& job0,
                    long long total_units, long long max_nb, int max_nla, int max_nlb, cudaStream_t stream,
                    int variant, long long det_stride = 0);
int rr_dispatch_v0(int norb, RRArgs& g, size_t smem, cudaStream_t stream);  // (16, 4)
int rr_dispatch_v1(int norb, RRArgs& g, size_t smem, cudaStream_t stream);  // (8, 4)
int rr_dispatch_v2(int norb, RRArgs& g, size_t smem, cudaStream_t stream);  // (16, 2)
int rr_dispatch_v3(int norb, RRArgs& g, size_t smem, cudaStream_t stream);  // (8, 2)

}  // namespace csffci
