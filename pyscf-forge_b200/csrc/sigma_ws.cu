// Warp-specialised variant of the register-resident sigma kernel, 4..16
// orbitals: tile variant 4 (one MMA warp per 8 rows) and, up to 12 orbitals,
// variant 7 (one MMA warp per 16 rows, m16n8k4, in CTAs of 8 warps).  Either
// runs one problem or a job table of many (BATCH: each unit's job is looked
// up between two barrier-9 syncs, gated jobs are skipped by both roles); the
// form with 8-row warps also has the deterministic scatter (DET: integer
// digit planes instead of FP64 atomics, det_add3), for one problem or a job
// table.
//
// k_sigma_rr runs the gather, MMA and scatter phases of a tile one after the
// other, separated by block barriers, so the FP64 tensor pipe idles while
// the gather/scatter phases run.  Here the warps of a CTA have two roles:
//
//   MMA warps    own m-tiles of V = A' D as in k_sigma_rr (A' = h2e with the
//                alpha signs of the current row, in registers); per tile they
//                only run the MMA and write V over the tile's D rows.
//   mover warps  for tile c: issue the copies of tile c, finish the gather of
//                tile c-1 (beta links) and scatter V of tile c-2 through the
//                beta links; the alpha scatter of V runs on the MMA warps,
//                from their accumulators.
//
// Tiles are 16 columns wide (two n-tiles of 8); the D/V and link buffers
// form a ring of three stages.  The two roles hand stages to each other
// with named barriers: for stage s, barrier 1+s means "D of the tile in s is
// gathered" (movers arrive, MMA warps wait) and barrier 4+s means "V of the
// tile in s is written" (MMA warps arrive, movers wait).  Barrier 7 orders
// the movers among themselves (their copies have landed before any gathers)
// and barrier 8 the MMA warps (every MMA warp has read D before V overwrites
// it).  A role reaches tile c+3 of a stage only after the other role has
// finished tile c, so a barrier id is never used by two tiles at once.
// Barrier 9 (all threads) separates the rows Ja, whose setup both roles
// share; the two roles run separate loops, so that the registers of the A
// fragments are not held in the movers' code.
//
// The CTA has a multiple of four warps, so every scheduler gets the same
// number; at 16 orbitals that is 17 MMA warps and 3 movers, 5 warps per
// scheduler: the register budget of k_sigma_rr, which the A fragments need.
// Up to 12 orbitals the fragments are small enough for two CTAs per SM.
#include <stdlib.h>

#include "sigma_ws.cuh"

namespace csffci {

// MMA warps: one per m-tile of 8 rows, the last m-tiles split over two warps
// (one n-tile each) when MT mod 4 is 1 or 2; movers fill the CTA to a
// multiple of four warps with at least two.
template <int MT, int MW = 8>
struct WSLayout {
  static constexpr int q = MT / 4, r = MT % 4;
  // splitting balances the MMA units over the schedulers; it is skipped
  // where it would leave fewer than three movers (17 m-tiles: 18 MMA warps
  // and 2 movers against 17 and 3), the movers being the limit there
  static constexpr bool split0 = q >= 1 && (r == 1 || r == 2);
  static constexpr int NWM0 = split0 ? 4 * q + 2 * r : MT;
  static constexpr bool split = MW == 8 && split0 && 4 * ((NWM0 + 2 + 3) / 4) - NWM0 >= 3;
  static constexpr int NWM = split ? NWM0 : MT;
  // 16-row MMA warps (up to 12 orbitals): at least three movers
  static constexpr int NTOT = MW == 8 ? 4 * ((NWM + 2 + 3) / 4) : 4 * ((NWM + 3 + 3) / 4);
  static constexpr int NMOV = NTOT - NWM;
};

constexpr int WS_RU = 4;      // links a mover thread handles together (loads in flight)

template <int KS, int MT, int MW, bool BATCH, int MINB, bool DET = false>
__global__ void __launch_bounds__(WSLayout<MT, MW>::NTOT * 32, MINB) k_sigma_ws(RRArgs g) {
  using L = WSLayout<MT, MW>;
  constexpr int NB = WS_NB;
  constexpr int NTH = L::NTOT * 32;
  constexpr int NWM = L::NWM, NMOV = L::NMOV;
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
  __shared__ csffci_sigma_job_t sjob_s;
  __shared__ int jst[2];
  S.job = &sjob_s;
  S.jst = jst;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (BATCH && tid == 0) jst[0] = -1;  // ordered before its first use by barrier 9
  if (g.bulk && tid == 0) {
    for (int s = 0; s < WS_STAGES; ++s) ws_mbar_init(&S.mbar[s], 1);
    ws_mbar_init_fence();  // the row setup's barriers order it before every use
  }
  const int ds = g.ds, npair = g.npair;
  const int ndr = g.nd_rows;
  const size_t dsz = (size_t)ndr * ds;
  for (int i = tid; i < (ndr - npair) * ds; i += NTH)
    for (int s = 0; s < WS_STAGES; ++s) S.Dbuf[s * dsz + npair * ds + i] = 0.0;

  if (warp < NWM) {
    // ---- MMA warps: own the A fragments; per tile only the MMA and V ----
    const int gq = lane >> 2, tq = lane & 3;
    const bool part = L::split && warp >= 4 * L::q;
    const int mt = part ? 4 * L::q + (warp - 4 * L::q) / 2 : warp;
    const int t0 = part ? (warp - 4 * L::q) % 2 : 0;
    double a0f[KS], a1f[MW == 16 ? KS : 1];
    // h2e rows MW mt + g (and + 8) of the job, columns 4k + t (without signs)
    auto load_a = [&](const double* h2e) {
      const int r0 = mt * MW + gq, r1 = r0 + 8;
#pragma unroll
      for (int k = 0; k < KS; ++k) {
        const int c = 4 * k + tq;
        a0f[k] = (r0 < npair && c < npair) ? h2e[(long long)r0 * npair + c] : 0.0;
        if (MW == 16) a1f[k] = (r1 < npair && c < npair) ? h2e[(long long)r1 * npair + c] : 0.0;
      }
    };
    if (!BATCH) load_a(g.job0.h2e);
    int cur = -1;       // job table index whose h2e the registers hold
    bool fresh = true;  // a0f holds h2e without signs
    int par = 0;
    for (long long u = blockIdx.x; u < g.total_units; u += gridDim.x) {
      const WSUnit un = ws_unit(g, u);
      if (BATCH) {
        if (!ws_batch_job<NTH>(g, S, un.ru, tid)) continue;
        if (jst[0] != cur) {
          cur = jst[0];
          load_a(sjob_s.h2e);
          fresh = true;
        }
      }
      const csffci_sigma_job_t& sjob = BATCH ? sjob_s : g.job0;
      const long long lu = un.ru - sjob.unit_begin;
      for (int w = 0; w < (sjob.sym ? 2 : 1); ++w) {
        if (!ws_row_setup<NTH, NB>(g, S, sjob, lu, un.part, un.parts, w, par, tid, warp, lane)) break;
        {
          // sign columns of A where this row's alpha sign differs from the
          // one the registers carry
          const unsigned* pcur = S.pneg + par * npair;
          const unsigned* pold = S.pneg + (par ^ 1) * npair;
#pragma unroll
          for (int k = 0; k < KS; ++k) {
            const int c = 4 * k + tq;
            if (c < npair && ((fresh ? 0u : pold[c]) ^ pcur[c])) {
              a0f[k] = -a0f[k];
              if (MW == 16) a1f[k] = -a1f[k];
            }
          }
        }
        fresh = false;
        cp_async_wait_all();  // this thread's part of the c row
        ws_bar_sync(9, NTH);
        const int nch = srow.nchunk;
        par ^= 1;
        for (int c = 0; c < nch; ++c) {
          const int s = c % WS_STAGES;
          ws_bar_sync(1 + s, NTH);  // D of tile c is gathered
          if constexpr (MW == 16) {
            // rows r0 = 16 mt + g and r1 = r0 + 8, both n-tiles (m16n8k4)
            double acc[2][4];
#pragma unroll
            for (int t = 0; t < 2; ++t) acc[t][0] = acc[t][1] = acc[t][2] = acc[t][3] = 0.0;
            const double* Db = S.Dbuf + s * dsz + tq * ds + gq;
#pragma unroll
            for (int k = 0; k < KS; ++k) {
              rr_dmma16(acc[0], a0f[k], a1f[k], Db[4 * k * ds]);
              rr_dmma16(acc[1], a0f[k], a1f[k], Db[4 * k * ds + 8]);
            }
            ws_bar_sync(8, NWM * 32);  // every MMA warp has read D of tile c
            const int r0 = mt * 16 + gq, r1 = r0 + 8;
#pragma unroll
            for (int t = 0; t < 2; ++t) {
              if (r0 < npair) {
                double* V = S.Dbuf + s * dsz + r0 * ds + 8 * t + 2 * tq;
                V[0] = acc[t][0];
                V[1] = acc[t][1];
              }
              if (r1 < npair) {
                double* V = S.Dbuf + s * dsz + r1 * ds + 8 * t + 2 * tq;
                V[0] = acc[t][2];
                V[1] = acc[t][3];
              }
            }
            ws_bar_arrive(4 + s, NTH);  // V of tile c is written
            // the alpha scatter of this lane's two pair rows (as below)
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
#pragma unroll
                for (int t = 0; t < 2; ++t) {
                  if (J + 8 * t < alim) ws_out_add<DET>(abase + J + 8 * t, rr_flip(acc[t][2 * h], aneg), g.det_stride);
                  if (J + 8 * t + 1 < alim)
                    ws_out_add<DET>(abase + J + 8 * t + 1, rr_flip(acc[t][2 * h + 1], aneg), g.det_stride);
                }
              }
            }
            continue;
          }
          double acc[2][2];
          acc[0][0] = acc[0][1] = acc[1][0] = acc[1][1] = 0.0;
          const double* Db = S.Dbuf + s * dsz + tq * ds + gq + 8 * t0;
          if (!part) {
#pragma unroll
            for (int k = 0; k < KS; ++k) {
              ws_dmma(acc[0][0], acc[0][1], a0f[k], Db[4 * k * ds]);
              ws_dmma(acc[1][0], acc[1][1], a0f[k], Db[4 * k * ds + 8]);
            }
          } else {
#pragma unroll
            for (int k = 0; k < KS; ++k) ws_dmma(acc[0][0], acc[0][1], a0f[k], Db[4 * k * ds]);
          }
          ws_bar_sync(8, NWM * 32);  // every MMA warp has read D of tile c
          const int r0 = mt * 8 + gq;
          if (r0 < npair) {
            double* V = S.Dbuf + s * dsz + r0 * ds + 8 * t0 + 2 * tq;
            V[0] = acc[0][0];
            V[1] = acc[0][1];
            if (!part) {
              V[8] = acc[1][0];
              V[9] = acc[1][1];
            }
          }
          ws_bar_arrive(4 + s, NTH);  // V of tile c is written
          // the alpha scatter of this lane's pair row, from its own
          // accumulators: sigma[Ka][J] += sign V[pq][J] for J < lim (J < Ja
          // in the spin-symmetric mode, where column Ja is left to the
          // transpose); the row's alpha link is re-read here so that nothing
          // of it stays in registers across the MMA
          const long long aoff = r0 < npair ? S.apoff[r0] : -1;
          if (aoff >= 0) {
            double* const abase = ((sjob.sym || DET) ? sjob.scratch : sjob.sigma) + aoff;
            const long long dstr = BATCH ? sjob.Na * sjob.Nb : g.det_stride;
            const unsigned aneg = S.pneg[srow.pc + r0];
            const int alim = (int)(sjob.sym ? srow.ja : sjob.Nb);
            const int J = (srow.c0 + c) * NB + 8 * t0 + 2 * tq;
            if (J < alim) ws_out_add<DET>(abase + J, rr_flip(acc[0][0], aneg), dstr);
            if (J + 1 < alim) ws_out_add<DET>(abase + J + 1, rr_flip(acc[0][1], aneg), dstr);
            if (!part) {
              if (J + 8 < alim) ws_out_add<DET>(abase + J + 8, rr_flip(acc[1][0], aneg), dstr);
              if (J + 9 < alim) ws_out_add<DET>(abase + J + 9, rr_flip(acc[1][1], aneg), dstr);
            }
          }
        }
      }
    }
  } else {
    ws_mover_role<NTH, NMOV, WS_RU, BATCH, DET>(g, S, tid, warp, lane, tid - NWM * 32, warp - NWM);
  }
}

bool sigma_ws_supported(int norb) { return norb >= 4 && norb <= 16; }
bool sigma_ws16_supported(int norb) { return norb >= 8 && norb <= 12; }

// CTAs per SM the registers are sized for: below 13 orbitals the A
// fragments are small enough for two CTAs per SM, so that one CTA's row
// setup (barrier 9) overlaps the other's tiles
constexpr int ws_min_blocks(int norb) { return norb <= 12 ? 2 : 1; }

template <int KS, int MT, int NORB, int MW>
static int launch_ws(RRArgs& g, size_t smem, cudaStream_t stream) {
  constexpr int NTH = WSLayout<MT, MW>::NTOT * 32;
  // 16-row MMA warps: 8-warp CTAs, two per SM
  constexpr int MINB = MW == 16 ? 2 : ws_min_blocks(NORB);
  // the deterministic scatter: one problem, 8-row MMA warps only
  auto kern = g.jobs ? ((MW == 8 && g.det_stride) ? k_sigma_ws<KS, MT, MW, true, MINB, MW == 8>
                                                  : k_sigma_ws<KS, MT, MW, true, MINB>)
                     : ((MW == 8 && g.det_stride) ? k_sigma_ws<KS, MT, MW, false, MINB, MW == 8>
                                                  : k_sigma_ws<KS, MT, MW, false, MINB>);
  CSF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev = 0, nsm = 148, per_sm = 0;
  CSF_CUDA(cudaGetDevice(&dev));
  CSF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  CSF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NTH, smem));
  if (per_sm < 1) {
    set_error("sigma: warp-specialised kernel does not fit on an SM (smem %zu)", smem);
    return CSFFCI_ERR_INVALID;
  }
  long long grid = (long long)nsm * per_sm;
  ws_split_last_round(g, grid);
  if (grid > g.total_units) grid = g.total_units;
  if (grid < 1) return CSFFCI_OK;
  static const char* names8[17] = {"", "", "", "", "k_sigma_ws_n4", "k_sigma_ws_n5", "k_sigma_ws_n6",
                                   "k_sigma_ws_n7", "k_sigma_ws_n8", "k_sigma_ws_n9",
                                   "k_sigma_ws_n10", "k_sigma_ws_n11", "k_sigma_ws_n12", "k_sigma_ws_n13",
                                   "k_sigma_ws_n14", "k_sigma_ws_n15", "k_sigma_ws_n16"};
  static const char* names16[13] = {"", "", "", "", "", "", "", "", "k_sigma_ws16_n8", "k_sigma_ws16_n9",
                                    "k_sigma_ws16_n10", "k_sigma_ws16_n11", "k_sigma_ws16_n12"};
  const char* name = MW == 16 ? (g.jobs ? names16[NORB <= 12 ? NORB : 0] : "k_sigma_ws16")
                              : (g.jobs ? names8[NORB] : g.det_stride ? "k_sigma_ws_det" : "k_sigma_ws");
  ProfScope ps(name, stream);
  kern<<<(int)grid, NTH, smem, stream>>>(g);
  return check_launch("sigma (warp-specialised)");
}

size_t ws_layout(RRArgs& g, int npair, int rows_multiple, long long max_nb, int max_nla, int max_nlb,
                 size_t extra_bytes, unsigned* extra_off) {
  const int ks = (npair + 3) / 4;
  g.npair = npair;
  g.ds = WS_NB + 4;  // = 4 (mod 16): conflict-free B-fragment loads
  g.ls = max_nlb | 1;
  const int rows_w = ((npair + rows_multiple - 1) / rows_multiple) * rows_multiple;
  g.nd_rows = 4 * ks > rows_w ? 4 * ks : rows_w;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 15) & ~(size_t)15;
    return (unsigned)o;
  };
  g.off_d = take((size_t)WS_STAGES * g.nd_rows * g.ds * sizeof(double));
  g.off_l = take((size_t)WS_STAGES * WS_NB * g.ls * sizeof(csffci_link_t));
  g.off_crow = take((size_t)max_nb * sizeof(double));
  g.off_al = take((size_t)(max_nla > 0 ? max_nla : 1) * sizeof(RRAlpha));
  g.off_zl = take((size_t)npair * sizeof(int));
  g.off_pn = take((size_t)2 * npair * sizeof(unsigned));
  g.off_zf = take((size_t)npair * sizeof(int));
  g.off_ap = take((size_t)npair * sizeof(long long));  // per-pair alpha offsets
  g.off_mbar = take((size_t)WS_STAGES * sizeof(unsigned long long));
  if (extra_bytes) {
    const unsigned o = take(extra_bytes);
    if (extra_off) *extra_off = o;
  }
  return off > 227 * 1024 - 256 ? 0 : off;
}

int sigma_ws_launch(int norb, int njobs, const csffci_sigma_job_t* jobs_dev, const csffci_sigma_job_t& job0,
                    long long total_units, long long max_nb, int max_nla, int max_nlb, cudaStream_t stream,
                    int mw, long long det_stride) {
  if (!(mw == 8 ? sigma_ws_supported(norb) : sigma_ws16_supported(norb))) {
    set_error("sigma: no warp-specialised kernel with %d-row MMA warps for norb %d", mw, norb);
    return CSFFCI_ERR_INVALID;
  }
  if (det_stride && mw != 8) {
    set_error("sigma: the deterministic scatter runs with 8-row MMA warps");
    return CSFFCI_ERR_INVALID;
  }
  const int npair = norb * (norb + 1) / 2;
  RRArgs g;
  memset(&g, 0, sizeof(g));
  g.jobs = jobs_dev;
  g.job0 = job0;
  g.njobs = jobs_dev ? njobs : 1;
  g.parts = 1;
  g.split_from = total_units;
  g.total_units = total_units;
  g.det_stride = det_stride;
  const size_t smem = ws_layout(g, npair, mw, max_nb, max_nla, max_nlb, 0, nullptr);
  if (smem == 0) {
    set_error("sigma: warp-specialised tiles exceed shared memory (norb %d)", norb);
    return CSFFCI_ERR_INVALID;
  }
  if (mw == 16) {
    switch (norb) {  // KS = ceil(npair / 4), MT = ceil(npair / 16)
      case 8: return launch_ws<9, 3, 8, 16>(g, smem, stream);
      case 9: return launch_ws<12, 3, 9, 16>(g, smem, stream);
      case 10: return launch_ws<14, 4, 10, 16>(g, smem, stream);
      case 11: return launch_ws<17, 5, 11, 16>(g, smem, stream);
      default: return launch_ws<20, 5, 12, 16>(g, smem, stream);
    }
  }
  switch (norb) {  // KS = ceil(npair / 4), MT = ceil(npair / 8)
    case 4: return launch_ws<3, 2, 4, 8>(g, smem, stream);
    case 5: return launch_ws<4, 2, 5, 8>(g, smem, stream);
    case 6: return launch_ws<6, 3, 6, 8>(g, smem, stream);
    case 7: return launch_ws<7, 4, 7, 8>(g, smem, stream);
    case 8: return launch_ws<9, 5, 8, 8>(g, smem, stream);
    case 9: return launch_ws<12, 6, 9, 8>(g, smem, stream);
    case 10: return launch_ws<14, 7, 10, 8>(g, smem, stream);
    case 11: return launch_ws<17, 9, 11, 8>(g, smem, stream);
    case 12: return launch_ws<20, 10, 12, 8>(g, smem, stream);
    case 13: return launch_ws<23, 12, 13, 8>(g, smem, stream);
    case 14: return launch_ws<27, 14, 14, 8>(g, smem, stream);
    case 15: return launch_ws<30, 15, 15, 8>(g, smem, stream);
    default: return launch_ws<34, 17, 16, 8>(g, smem, stream);
  }
}

}  // namespace csffci
