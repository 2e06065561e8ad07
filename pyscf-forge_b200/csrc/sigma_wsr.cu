// Warp-specialised sigma kernel with the registers re-split between the
// warp roles (tile variant 5), for one problem at 16 orbitals (npair = 136 =
// 8 x 16 + 8 rows of V = A' D).
//
// k_sigma_ws (sigma_ws.cu) gives every MMA warp one m-tile of 8 rows: at 16
// orbitals that is 17 MMA warps, 5 of them on one of the SM's four
// schedulers (each scheduler owns one FP64 tensor pipe), every warp reading
// the whole D tile for 8 rows of output, and 3 mover warps.  Here the CTA
// has 16 warps (four warpgroups) and the register file is re-split at the
// start of the kernel with setmaxnreg:
//
//   warps 0-7    (warpgroups 0, 1) "big" MMA warps: rows 16b..16b+15 with
//                m16n8k4, A' fragments of 16 rows x 136 columns in registers
//                (REG_BIG per thread); each B fragment read from shared
//                memory now feeds 16 rows, so the B traffic halves;
//   warps 8-11   (warpgroup 2) "tail" MMA warps: rows 128..135 split over
//                the two n-tiles and the two halves of K (17 m8n8k4 per
//                tile each); the K halves are summed through a small
//                double-buffered shared array;
//   warps 12-15  (warpgroup 3) movers, the role of sigma_ws.cuh.
//
// Warp w issues on scheduler w mod 4, so every scheduler carries two big
// warps, one tail warp and one mover: 2 x 136 + 17 = 289 m8n8k4-equivalents
// of MMA per 16-column tile on each tensor pipe (against 340 on the busiest
// pipe of k_sigma_ws), and four movers instead of three.
//
// Registers: launched with 128 per thread (512 threads = the whole register
// file); warpgroups 0-1 raise theirs to REG_BIG, warpgroup 2 lowers to
// REG_TAIL and warpgroup 3 to REG_MOV, with 2*128*REG_BIG + 128*REG_TAIL +
// 128*REG_MOV = 512*128.  setmaxnreg.inc waits until the registers it asks
// for are free, so the launcher checks that the kernel really was given 128
// registers per thread before launching it (with fewer, the raise would
// wait for registers that never come).
//
// The barrier protocol is that of sigma_ws.cuh (ids 1..9); the tail warps'
// K-half sums are ordered by barrier 8: the second half writes its partial
// before barrier 8 of the tile, the first half reads it after.
#include <stdlib.h>

#include "sigma_ws.cuh"

namespace csffci {

constexpr int WSR_NBIG = 8;   // MMA warps of 16 rows
constexpr int WSR_NTAIL = 4;  // MMA warps of the last 8 rows
constexpr int WSR_NMOV = 4;   // movers
constexpr int WSR_NW = WSR_NBIG + WSR_NTAIL + WSR_NMOV;
constexpr int WSR_NTH = WSR_NW * 32;
constexpr int WSR_NMMA = (WSR_NBIG + WSR_NTAIL) * 32;
constexpr int WSR_REG_LAUNCH = 128;
constexpr int WSR_REG_BIG = 176;
constexpr int WSR_REG_TAIL = 104;
constexpr int WSR_REG_MOV = 56;
constexpr int WSR_RU = 3;  // mover links per pass: 8 link rows per pass x 3 = 24 divides 72
static_assert(2 * 128 * WSR_REG_BIG + 128 * WSR_REG_TAIL + 128 * WSR_REG_MOV <= WSR_NTH * WSR_REG_LAUNCH,
              "the re-split registers fit in the launch's allocation");
static_assert(WSR_REG_BIG % 8 == 0 && WSR_REG_TAIL % 8 == 0 && WSR_REG_MOV % 8 == 0 && WSR_REG_MOV >= 24,
              "setmaxnreg counts are multiples of 8 in [24, 256]");
static_assert(WSR_NTH * WSR_REG_LAUNCH == 65536, "the launch takes the whole register file");

template <int N>
__device__ __forceinline__ void wsr_reg_inc() {
  asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" ::"n"(N));
}
template <int N>
__device__ __forceinline__ void wsr_reg_dec() {
  asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" ::"n"(N));
}

// KS k-steps of 4 (KS = 34 at 16 orbitals), KH = KS/2 per tail K half
template <int KS>
__global__ void __launch_bounds__(WSR_NTH, 1) k_sigma_wsr(RRArgs g) {
  static_assert(KS % 2 == 0, "the tail warps split K in two equal halves");
  constexpr int NB = WS_NB;
  constexpr int KH = KS / 2;
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ RRRow srow;
  WSShared S;
  S.Dbuf = (double*)(smraw + g.off_d);
  S.Lbuf = (csffci_link_t*)(smraw + g.off_l);
  S.crow = (double*)(smraw + g.off_crow);
  S.al = (RRAlpha*)(smraw + g.off_al);
  S.zl = (int*)(smraw + g.off_zl);
  S.pneg = (unsigned*)(smraw + g.off_pn);
  S.zf = (int*)(smraw + g.off_zf);
  S.srow = &srow;
  S.apoff = (long long*)(smraw + g.off_ap);
  S.mbar = (unsigned long long*)(smraw + g.off_mbar);
  S.job = nullptr;  // one problem: the job is g.job0
  S.jst = nullptr;
  // tail partial sums: [tile parity][n-tile][64 doubles]
  double* const Pbuf = (double*)(smraw + g.off_extra);
  const csffci_sigma_job_t& sjob = g.job0;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (g.bulk && tid == 0) {
    for (int s = 0; s < WS_STAGES; ++s) ws_mbar_init(&S.mbar[s], 1);
    ws_mbar_init_fence();  // the row setup's barriers order it before every use
  }
  const int ds = g.ds, npair = g.npair;
  const int ndr = g.nd_rows;
  const size_t dsz = (size_t)ndr * ds;
  for (int i = tid; i < (ndr - npair) * ds; i += WSR_NTH)
    for (int s = 0; s < WS_STAGES; ++s) S.Dbuf[s * dsz + npair * ds + i] = 0.0;

  if (warp < WSR_NBIG) {
    // ---- big MMA warps: 16 rows each, m16n8k4 ----
    wsr_reg_inc<WSR_REG_BIG>();
    const int gq = lane >> 2, tq = lane & 3;
    const int r0 = 16 * warp + gq, r1 = r0 + 8;
    double a0[KS], a1[KS];
#pragma unroll
    for (int k = 0; k < KS; ++k) {
      const int c = 4 * k + tq;
      a0[k] = (r0 < npair && c < npair) ? sjob.h2e[(long long)r0 * npair + c] : 0.0;
      a1[k] = (r1 < npair && c < npair) ? sjob.h2e[(long long)r1 * npair + c] : 0.0;
    }
    bool fresh = true;
    int par = 0;
    for (long long u = blockIdx.x; u < g.total_units; u += gridDim.x) {
      const WSUnit un = ws_unit(g, u);
      const long long lu = un.ru - sjob.unit_begin;
      for (int w = 0; w < (sjob.sym ? 2 : 1); ++w) {
        if (!ws_row_setup<WSR_NTH, NB>(g, S, sjob, lu, un.part, un.parts, w, par, tid, warp, lane)) break;
        {
          // sign columns of A where this row's alpha sign differs from the
          // one the registers carry
          const unsigned* pcur = S.pneg + par * npair;
          const unsigned* pold = S.pneg + (par ^ 1) * npair;
#pragma unroll
          for (int k = 0; k < KS; ++k) {
            const int c = 4 * k + tq;
            if (c < npair && ((fresh ? 0u : pold[c]) ^ pcur[c])) {
              a0[k] = -a0[k];
              a1[k] = -a1[k];
            }
          }
        }
        fresh = false;
        cp_async_wait_all();  // this thread's part of the c row
        ws_bar_sync(9, WSR_NTH);
        const int nch = srow.nchunk;
        par ^= 1;
        for (int c = 0; c < nch; ++c) {
          const int s = c % WS_STAGES;
          ws_bar_sync(1 + s, WSR_NTH);  // D of tile c is gathered
          double acc[2][4];
#pragma unroll
          for (int j = 0; j < 2; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0;
          const double* Db = S.Dbuf + s * dsz + tq * ds + gq;
#pragma unroll
          for (int k = 0; k < KS; ++k) {
            const double b0 = Db[4 * k * ds], b1 = Db[4 * k * ds + 8];
            rr_dmma16(acc[0], a0[k], a1[k], b0);
            rr_dmma16(acc[1], a0[k], a1[k], b1);
          }
          ws_bar_sync(8, WSR_NMMA);  // every MMA warp has read D of tile c
          double* V = S.Dbuf + s * dsz + 2 * tq;
          if (r0 < npair) {
            V[r0 * ds + 0] = acc[0][0];
            V[r0 * ds + 1] = acc[0][1];
            V[r0 * ds + 8] = acc[1][0];
            V[r0 * ds + 9] = acc[1][1];
          }
          if (r1 < npair) {
            V[r1 * ds + 0] = acc[0][2];
            V[r1 * ds + 1] = acc[0][3];
            V[r1 * ds + 8] = acc[1][2];
            V[r1 * ds + 9] = acc[1][3];
          }
          if (g.bulk) ws_fence_proxy_async();  // V before the stage's next bulk copy
          ws_bar_arrive(4 + s, WSR_NTH);  // V of tile c is written
          // alpha scatter of this lane's two pair rows from the accumulators
          // (J < Ja in the spin-symmetric mode, whose column Ja is left to
          // the transpose)
          double* const obase = sjob.sym ? sjob.scratch : sjob.sigma;
          const int alim = (int)(sjob.sym ? srow.ja : sjob.Nb);
          const int J = (srow.c0 + c) * NB + 2 * tq;
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int r = h ? r1 : r0;
            const long long aoff = r < npair ? S.apoff[r] : -1;
            if (aoff >= 0) {
              double* const abase = obase + aoff;
              const unsigned aneg = S.pneg[srow.pc + r];
              if (J < alim) atomicAdd(abase + J, rr_flip(acc[0][2 * h], aneg));
              if (J + 1 < alim) atomicAdd(abase + J + 1, rr_flip(acc[0][2 * h + 1], aneg));
              if (J + 8 < alim) atomicAdd(abase + J + 8, rr_flip(acc[1][2 * h], aneg));
              if (J + 9 < alim) atomicAdd(abase + J + 9, rr_flip(acc[1][2 * h + 1], aneg));
            }
          }
        }
      }
    }
  } else if (warp < WSR_NBIG + WSR_NTAIL) {
    // ---- tail MMA warps: rows 128..135, one n-tile and one K half each ----
    wsr_reg_dec<WSR_REG_TAIL>();
    const int gq = lane >> 2, tq = lane & 3;
    const int tw = warp - WSR_NBIG;
    const int nt = tw & 1, kh = tw >> 1;
    const int kb = kh ? KH : 0;
    const int rt = 16 * WSR_NBIG + gq;
    double at[KH];
#pragma unroll
    for (int k = 0; k < KH; ++k) {
      const int c = 4 * (kb + k) + tq;
      at[k] = (rt < npair && c < npair) ? sjob.h2e[(long long)rt * npair + c] : 0.0;
    }
    bool fresh = true;
    int par = 0;
    int tpar = 0;  // parity of the tile count (Pbuf half)
    for (long long u = blockIdx.x; u < g.total_units; u += gridDim.x) {
      const WSUnit un = ws_unit(g, u);
      const long long lu = un.ru - sjob.unit_begin;
      for (int w = 0; w < (sjob.sym ? 2 : 1); ++w) {
        if (!ws_row_setup<WSR_NTH, NB>(g, S, sjob, lu, un.part, un.parts, w, par, tid, warp, lane)) break;
        {
          const unsigned* pcur = S.pneg + par * npair;
          const unsigned* pold = S.pneg + (par ^ 1) * npair;
#pragma unroll
          for (int k = 0; k < KH; ++k) {
            const int c = 4 * (kb + k) + tq;
            if (c < npair && ((fresh ? 0u : pold[c]) ^ pcur[c])) at[k] = -at[k];
          }
        }
        fresh = false;
        cp_async_wait_all();
        ws_bar_sync(9, WSR_NTH);
        const int nch = srow.nchunk;
        par ^= 1;
        for (int c = 0; c < nch; ++c) {
          const int s = c % WS_STAGES;
          ws_bar_sync(1 + s, WSR_NTH);  // D of tile c is gathered
          double acc0 = 0.0, acc1 = 0.0;
          const double* Db = S.Dbuf + s * dsz + (4 * kb + tq) * ds + gq + 8 * nt;
#pragma unroll
          for (int k = 0; k < KH; ++k) ws_dmma(acc0, acc1, at[k], Db[4 * k * ds]);
          double* const P = Pbuf + (tpar * 2 + nt) * 64 + 2 * lane;
          if (kh) {
            P[0] = acc0;
            P[1] = acc1;
          }
          ws_bar_sync(8, WSR_NMMA);  // D of tile c read by every MMA warp; partials written
          if (!kh) {
            acc0 += P[0];
            acc1 += P[1];
            if (rt < npair) {
              double* V = S.Dbuf + s * dsz + rt * ds + 8 * nt + 2 * tq;
              V[0] = acc0;
              V[1] = acc1;
            }
          }
          if (g.bulk) ws_fence_proxy_async();
          ws_bar_arrive(4 + s, WSR_NTH);  // V of tile c is written
          if (!kh) {
            const long long aoff = rt < npair ? S.apoff[rt] : -1;
            if (aoff >= 0) {
              double* const abase = (sjob.sym ? sjob.scratch : sjob.sigma) + aoff;
              const unsigned aneg = S.pneg[srow.pc + rt];
              const int alim = (int)(sjob.sym ? srow.ja : sjob.Nb);
              const int J = (srow.c0 + c) * NB + 8 * nt + 2 * tq;
              if (J < alim) atomicAdd(abase + J, rr_flip(acc0, aneg));
              if (J + 1 < alim) atomicAdd(abase + J + 1, rr_flip(acc1, aneg));
            }
          }
          tpar ^= 1;
        }
      }
    }
  } else {
    wsr_reg_dec<WSR_REG_MOV>();
    const int mw = warp - WSR_NBIG - WSR_NTAIL;
    ws_mover_role<WSR_NTH, WSR_NMOV, WSR_RU, false, false>(g, S, tid, warp, lane, mw * 32 + lane, mw);
  }
}

bool sigma_wsr_supported(int norb) { return norb == 16; }

int sigma_wsr_launch(int norb, const csffci_sigma_job_t& job0, long long total_units, long long max_nb,
                     int max_nla, int max_nlb, cudaStream_t stream, bool bulk) {
  if (!sigma_wsr_supported(norb)) {
    set_error("sigma: the register-split warp-specialised variant covers norb 16, not %d", norb);
    return CSFFCI_ERR_INVALID;
  }
  const int npair = norb * (norb + 1) / 2;
  constexpr int KS = 34;
  if ((npair + 3) / 4 != KS || npair > 16 * WSR_NBIG + 8) {
    set_error("sigma: register-split kernel built for 136 pair rows, not %d", npair);
    return CSFFCI_ERR_INVALID;
  }
  RRArgs g;
  memset(&g, 0, sizeof(g));
  g.jobs = nullptr;
  g.job0 = job0;
  g.njobs = 1;
  g.parts = 1;
  g.split_from = total_units;
  g.total_units = total_units;
  unsigned extra = 0;
  const size_t smem = ws_layout(g, npair, 8, max_nb, max_nla, max_nlb, 4 * 64 * sizeof(double), &extra);
  if (smem == 0) {
    set_error("sigma: register-split tiles exceed shared memory (norb %d)", norb);
    return CSFFCI_ERR_INVALID;
  }
  g.off_extra = extra;
  g.bulk = bulk && ws_bulk_ok(job0) ? 1 : 0;
  auto kern = k_sigma_wsr<KS>;
  // setmaxnreg re-splits the registers the launch allocated (128 per
  // thread); with any other count the raise of warpgroups 0-1 could not be
  // met, so refuse rather than launch
  cudaFuncAttributes fa;
  CSF_CUDA(cudaFuncGetAttributes(&fa, kern));
  if (fa.numRegs != WSR_REG_LAUNCH) {
    set_error("sigma: register-split kernel compiled to %d registers per thread, not %d", fa.numRegs,
              WSR_REG_LAUNCH);
    return CSFFCI_ERR_INVALID;
  }
  CSF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev = 0, nsm = 148, per_sm = 0;
  CSF_CUDA(cudaGetDevice(&dev));
  CSF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  CSF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, WSR_NTH, smem));
  if (per_sm != 1) {
    set_error("sigma: register-split kernel needs exactly one CTA per SM (got %d)", per_sm);
    return CSFFCI_ERR_INVALID;
  }
  long long grid = nsm;
  ws_split_last_round(g, grid);
  if (grid > g.total_units) grid = g.total_units;
  if (grid < 1) return CSFFCI_OK;
  ProfScope ps(g.bulk ? "k_sigma_wsr_bulk" : "k_sigma_wsr", stream);
  kern<<<(int)grid, WSR_NTH, smem, stream>>>(g);
  return check_launch("sigma (register-split warp-specialised)");
}

}  // namespace csffci
