// Warp-specialised variant of the register-resident sigma kernel (tile
// variant 4), for one problem at 13..16 orbitals.
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
#include <stdlib.h>

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

// MMA warps: one per m-tile of 8 rows, the last m-tiles split over two warps
// (one n-tile each) when MT mod 4 is 1 or 2; movers fill the CTA to a
// multiple of four warps with at least two.
template <int MT>
struct WSLayout {
  static constexpr int q = MT / 4, r = MT % 4;
  // splitting balances the MMA units over the schedulers; it is skipped
  // where it would leave fewer than three movers (17 m-tiles: 18 MMA warps
  // and 2 movers against 17 and 3), the movers being the limit there
  static constexpr bool split0 = q >= 1 && (r == 1 || r == 2);
  static constexpr int NWM0 = split0 ? 4 * q + 2 * r : MT;
  static constexpr bool split = split0 && 4 * ((NWM0 + 2 + 3) / 4) - NWM0 >= 3;
  static constexpr int NWM = split ? NWM0 : MT;
  static constexpr int NTOT = 4 * ((NWM + 2 + 3) / 4);
  static constexpr int NMOV = NTOT - NWM;
};

constexpr int WS_NB = 16;     // columns per tile
constexpr int WS_STAGES = 3;  // ring of D/V and link buffers
constexpr int WS_RU = 4;      // links a mover thread handles together (loads in flight)

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
};

// Row setup shared by both roles (every thread of the CTA calls it with the
// same arguments, and it synchronises the CTA on barrier 9): the alpha links
// of row Ja, the rows without one, the sign masks of this row (in half par
// of pneg) and the copy of c row Ja.  Returns false (for every thread) when
// the spin-symmetric unit has no second row.
template <int NTH, int NB>
__device__ __forceinline__ bool ws_row_setup(const RRArgs& g, const WSShared& S, long long lu, int w, int par,
                                             int tid, int warp, int lane) {
  const csffci_sigma_job_t& sjob = g.job0;
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
    S.srow->nchunk = (int)((S.srow->jend + NB - 1) / NB);
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

template <int KS, int MT>
__global__ void __launch_bounds__(WSLayout<MT>::NTOT * 32, 1) k_sigma_ws(RRArgs g) {
  using L = WSLayout<MT>;
  constexpr int NB = WS_NB;
  constexpr int NTH = L::NTOT * 32;
  constexpr int NWM = L::NWM, NMOV = L::NMOV;
  constexpr int MTH = NMOV * 32;   // mover threads
  constexpr int MPASS = MTH / NB;  // link rows per mover pass (threads over the NB columns)
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
  const csffci_sigma_job_t& sjob = g.job0;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ds = g.ds, LS = g.ls, npair = g.npair;
  const int ndr = g.nd_rows;
  const size_t dsz = (size_t)ndr * ds, lsz = (size_t)NB * LS;
  for (int i = tid; i < (ndr - npair) * ds; i += NTH)
    for (int s = 0; s < WS_STAGES; ++s) S.Dbuf[s * dsz + npair * ds + i] = 0.0;

  if (warp < NWM) {
    // ---- MMA warps: own the A fragments; per tile only the MMA and V ----
    const int gq = lane >> 2, tq = lane & 3;
    const bool part = L::split && warp >= 4 * L::q;
    const int mt = part ? 4 * L::q + (warp - 4 * L::q) / 2 : warp;
    const int t0 = part ? (warp - 4 * L::q) % 2 : 0;
    double a0f[KS];
    {
      const int r0 = mt * 8 + gq;
#pragma unroll
      for (int k = 0; k < KS; ++k) {
        const int c = 4 * k + tq;
        a0f[k] = (r0 < npair && c < npair) ? sjob.h2e[(long long)r0 * npair + c] : 0.0;
      }
    }
    bool fresh = true;
    int par = 0;
    for (long long u = blockIdx.x; u < g.total_units; u += gridDim.x) {
      const long long lu = u - sjob.unit_begin;
      for (int w = 0; w < (sjob.sym ? 2 : 1); ++w) {
        if (!ws_row_setup<NTH, NB>(g, S, lu, w, par, tid, warp, lane)) break;
        {
          // sign columns of A where this row's alpha sign differs from the
          // one the registers carry
          const unsigned* pcur = S.pneg + par * npair;
          const unsigned* pold = S.pneg + (par ^ 1) * npair;
#pragma unroll
          for (int k = 0; k < KS; ++k) {
            const int c = 4 * k + tq;
            if (c < npair && ((fresh ? 0u : pold[c]) ^ pcur[c])) a0f[k] = -a0f[k];
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
            double* const abase = (sjob.sym ? sjob.scratch : sjob.sigma) + aoff;
            const unsigned aneg = S.pneg[srow.pc + r0];
            const int alim = (int)(sjob.sym ? srow.ja : sjob.Nb);
            const int J = c * NB + 8 * t0 + 2 * tq;
            if (J < alim) atomicAdd(abase + J, rr_flip(acc[0][0], aneg));
            if (J + 1 < alim) atomicAdd(abase + J + 1, rr_flip(acc[0][1], aneg));
            if (!part) {
              if (J + 8 < alim) atomicAdd(abase + J + 8, rr_flip(acc[1][0], aneg));
              if (J + 9 < alim) atomicAdd(abase + J + 9, rr_flip(acc[1][1], aneg));
            }
          }
        }
      }
    }
  } else {
    // ---- movers: copies, beta gather, scatters ----
    const int mtid = tid - NWM * 32;
    const int mwarp = warp - NWM;
    const int jl = mtid % NB, ml = mtid / NB;
    int par = 0;
    for (long long u = blockIdx.x; u < g.total_units; u += gridDim.x) {
      const long long lu = u - sjob.unit_begin;
      for (int w = 0; w < (sjob.sym ? 2 : 1); ++w) {
        if (!ws_row_setup<NTH, NB>(g, S, lu, w, par, tid, warp, lane)) break;
        par ^= 1;
        cp_async_wait_all();
        ws_bar_sync(9, NTH);
        const int nch = srow.nchunk;
        const long long jend = srow.jend, ja = srow.ja, Nb = sjob.Nb;
        const int nla = sjob.nla, nlb = sjob.nlb, nz = srow.nzero;
        const unsigned* pc = S.pneg + srow.pc;
        const bool SYM = sjob.sym != 0;
        double* const out = SYM ? sjob.scratch : sjob.sigma;
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
            const long long j1 = (long long)c * NB;
            const int nc = (int)min((long long)NB, jend - j1);
            if (jl < nc) {
              const double* src = sjob.ci + j1 + jl;
              for (int l0 = ml; l0 < nla; l0 += WS_RU * MPASS) {
                RRAlpha a[WS_RU];
#pragma unroll
                for (int k = 0; k < WS_RU; ++k) a[k] = S.al[min(l0 + k * MPASS, nla - 1)];
#pragma unroll
                for (int k = 0; k < WS_RU; ++k)
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
            ws_bar_sync(7, MTH);
            const int s = (c - 1) % WS_STAGES;
            double* D = S.Dbuf + s * dsz;
            const csffci_link_t* Lt = S.Lbuf + s * lsz;
            const int ncol = (int)min((long long)NB, jend - (long long)(c - 1) * NB);
            if (jl < ncol)
              for (int m0 = ml; m0 < nlb; m0 += WS_RU * MPASS) {
                // WS_RU links per pass, every load of the pass issued before
                // the dependent ones (distinct links of a column have
                // distinct pairs, so the read-modify-writes do not overlap)
                uint2 e[WS_RU];
                double v[WS_RU], d[WS_RU];
                unsigned f[WS_RU];
#pragma unroll
                for (int k = 0; k < WS_RU; ++k) {
                  const int m = m0 + k * MPASS;
                  e[k] = m < nlb ? rr_link(&Lt[jl * LS + m]) : make_uint2(0u, 0u);
                }
#pragma unroll
                for (int k = 0; k < WS_RU; ++k) {
                  v[k] = S.crow[e[k].x];
                  f[k] = rr_lneg(e[k]) ^ pc[rr_lpair(e[k])];
                  d[k] = D[rr_lpair(e[k]) * ds + jl];
                }
#pragma unroll
                for (int k = 0; k < WS_RU; ++k)
                  if (m0 + k * MPASS < nlb) D[rr_lpair(e[k]) * ds + jl] = d[k] + rr_flip(v[k], f[k]);
              }
            ws_bar_arrive(1 + s, NTH);  // D of tile c-1 is gathered
          }
          if (c >= 2) {
            // scatter of tile c-2
            const int s = (c - 2) % WS_STAGES;
            ws_bar_sync(4 + s, NTH);  // V of tile c-2 is written
            const double* D = S.Dbuf + s * dsz;
            const csffci_link_t* Lt = S.Lbuf + s * lsz;
            const long long j0 = (long long)(c - 2) * NB;
            const int ncol = (int)min((long long)NB, jend - j0);
            if (jl < ncol) {
              double* const orow = out + ja * Nb;
              for (int m0 = ml; m0 < nlb; m0 += WS_RU * MPASS) {
                uint2 e[WS_RU];
                double v[WS_RU];
#pragma unroll
                for (int k = 0; k < WS_RU; ++k) {
                  const int m = m0 + k * MPASS;
                  e[k] = m < nlb ? rr_link(&Lt[jl * LS + m]) : make_uint2(0u, 0u);
                }
#pragma unroll
                for (int k = 0; k < WS_RU; ++k) v[k] = D[rr_lpair(e[k]) * ds + jl];
#pragma unroll
                for (int k = 0; k < WS_RU; ++k)
                  if (m0 + k * MPASS < nlb) atomicAdd(&orow[e[k].x], rr_flip(v[k], rr_lneg(e[k])));
              }
            }
          }
        }
      }
    }
  }
}

bool sigma_ws_supported(int norb) { return norb >= 13 && norb <= 16; }

template <int KS, int MT>
static int launch_ws(RRArgs& g, size_t smem, cudaStream_t stream) {
  constexpr int NTH = WSLayout<MT>::NTOT * 32;
  auto kern = k_sigma_ws<KS, MT>;
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
  if (grid > g.total_units) grid = g.total_units;
  if (grid < 1) return CSFFCI_OK;
  ProfScope ps("k_sigma_ws", stream);
  kern<<<(int)grid, NTH, smem, stream>>>(g);
  return check_launch("sigma (warp-specialised)");
}

int sigma_ws_launch(int norb, const csffci_sigma_job_t& job0, long long total_units, long long max_nb,
                    int max_nla, int max_nlb, cudaStream_t stream) {
  if (!sigma_ws_supported(norb)) {
    set_error("sigma: the warp-specialised variant covers norb 13..16, not %d", norb);
    return CSFFCI_ERR_INVALID;
  }
  const int npair = norb * (norb + 1) / 2;
  const int ks = (npair + 3) / 4;
  RRArgs g;
  memset(&g, 0, sizeof(g));
  g.jobs = nullptr;
  g.job0 = job0;
  g.njobs = 1;
  g.total_units = total_units;
  g.npair = npair;
  g.ds = WS_NB + 4;  // = 4 (mod 16): conflict-free B-fragment loads
  g.ls = max_nlb | 1;
  const int rows_w = ((npair + 7) / 8) * 8;
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
  const size_t smem = off;
  if (smem > 227 * 1024 - 256) {
    set_error("sigma: warp-specialised tiles of %zu bytes exceed shared memory", smem);
    return CSFFCI_ERR_INVALID;
  }
  switch (norb) {
    case 13: return launch_ws<23, 12>(g, smem, stream);
    case 14: return launch_ws<27, 14>(g, smem, stream);
    case 15: return launch_ws<30, 15>(g, smem, stream);
    default: return launch_ws<34, 17>(g, smem, stream);
  }
}

}  // namespace csffci
