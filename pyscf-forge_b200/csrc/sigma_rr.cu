// sigma with h2e held in registers ("register-resident" kernel), for
// 8 <= norb <= 16.
//
// Warp w owns the output rows 8w..8w+7 of V = h2e . D for the whole kernel,
// so its A fragments (h2e[8w + lane/4][4s + lane%4], s < npad/4) are loaded
// once into registers and shared memory is left for the tiles:
//   D[2][npad][ds]      double-buffered gather tile (cp.async prefetch of
//                       the next tile's alpha rows behind the current MMA)
//   L[2][NB][LS]        the beta link rows of the tile's NB columns
//   crow[Nb]            row Ja of c (the beta gathers read it)
// One CTA owns a row Ja (and, in the spin-symmetric mode, the pair of rows
// u and Na-1-u so that all units cost the same).
//
// Spin-symmetric mode (na == nb, c = eta c^T): only tiles with Jb <= Ja are
// formed (half the GEMM).  A tile's V[pq][Jb] is scattered twice:
//   row-local      s[Ja][Kb] += sign V   (beta links of Jb)
//   transposed     s[Jb][Ka] += eta sign V (alpha links of Ja, Jb < Ja)
// and sigma = s + eta s^T afterwards (csffci_sigma).  General mode: all Jb,
// row-local beta scatter and the alpha scatter sigma[Ka][Jb] += sign V.
// Shared-memory layouts are chosen bank-conflict free for the 32-lane
// accesses: ds = 8 (mod 16) doubles for the m8n8k4 B fragments, LS odd for
// the column-wise link reads.
#include <stdlib.h>

#include "common.cuh"
#include "profile.cuh"
#include "sigma_rr.cuh"

namespace csffci {

__device__ __forceinline__ void cp_async8(void* s, const void* gsrc) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gsrc) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

__device__ __forceinline__ int rr_pair(const csffci_link_t& e) {
  int p = e.op & 0xff, q = e.op >> 8;
  int hi = p > q ? p : q, lo = p > q ? q : p;
  return hi * (hi + 1) / 2 + lo;
}

struct RRArgs {
  const double* h2e;
  const csffci_link_t* la;
  const csffci_link_t* lb;
  const double* ci;
  double* out;
  long long Na, Nb, nunits;
  int npair, ds, ls, nla, nlb, nd_rows;
  unsigned off_d, off_l, off_crow, off_las, off_rowsrc, off_zrow;
};


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

// KS k-steps of 4 (npair rounded up to a multiple of 4); NW warps owning MW
// (8 or 16) output rows each; NT n-tiles of 8 columns per tile.
template <int KS, int NW, int MW, int NT, bool SYM>
__global__ void __launch_bounds__(NW * 32, 1) k_sigma_rr(RRArgs g) {
  constexpr int NTH = NW * 32;
  constexpr int NB = 8 * NT;
  extern __shared__ __align__(16) unsigned char smraw[];
  double* Dbuf = (double*)(smraw + g.off_d);
  csffci_link_t* Lbuf = (csffci_link_t*)(smraw + g.off_l);
  double* crow = (double*)(smraw + g.off_crow);
  csffci_link_t* las = (csffci_link_t*)(smraw + g.off_las);
  int* rowsrc = (int*)(smraw + g.off_rowsrc);  // alpha link of a pair row, -1 if none
  int* zrow = (int*)(smraw + g.off_zrow);      // [0] = count, then the rows without one

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  const long long Nb = g.Nb;
  const int ds = g.ds, LS = g.ls, nla = g.nla, nlb = g.nlb, npair = g.npair;
  const int ndr = g.nd_rows;
  const size_t dsz = (size_t)ndr * ds, lsz = (size_t)NB * LS;

  // h2e rows MW*w+g (and MW*w+8+g), columns 4s+t, resident for the kernel
  double a0f[KS], a1f[MW == 16 ? KS : 1];
  {
    const int r0 = warp * MW + gq, r1 = r0 + 8;
#pragma unroll
    for (int s = 0; s < KS; ++s) {
      const int c = 4 * s + tq;
      a0f[s] = (r0 < npair && c < npair) ? g.h2e[(long long)r0 * npair + c] : 0.0;
      if (MW == 16) a1f[s] = (r1 < npair && c < npair) ? g.h2e[(long long)r1 * npair + c] : 0.0;
    }
  }
  // rows past npair are k rows of the MMA that nothing else writes
  for (int i = tid; i < (ndr - npair) * ds; i += NTH) {
    Dbuf[npair * ds + i] = 0.0;
    Dbuf[dsz + npair * ds + i] = 0.0;
  }

  for (long long u = blockIdx.x; u < g.nunits; u += gridDim.x) {
    for (int w = 0; w < (SYM ? 2 : 1); ++w) {
      long long ja = u;
      if (SYM && w == 1) {
        ja = g.Na - 1 - u;
        if (ja <= u) break;
      }
      const long long jend = SYM ? ja + 1 : Nb;
      const int nchunk = (int)((jend + NB - 1) / NB);
      __syncthreads();  // the previous row is fully consumed
      for (int r = tid; r < ndr; r += NTH) rowsrc[r] = -1;
      __syncthreads();
      for (int l = tid; l < nla; l += NTH) {
        csffci_link_t e = g.la[ja * nla + l];
        las[l] = e;
        rowsrc[rr_pair(e)] = l;
      }
      __syncthreads();
      if (tid == 0) {
        // rows to reset each tile: first those without an alpha link (zeroed),
        // then the alpha rows with a negative sign (negated)
        int n = 0;
        for (int r = 0; r < npair; ++r)
          if (rowsrc[r] < 0) zrow[2 + n++] = r;
        zrow[0] = n;
        for (int r = 0; r < npair; ++r)
          if (rowsrc[r] >= 0 && las[rowsrc[r]].sign < 0) zrow[2 + n++] = r;
        zrow[1] = n;
      }
      for (long long i = tid; i < Nb; i += NTH) cp_async8(&crow[i], &g.ci[ja * Nb + i]);
      {
        double* D = Dbuf;
        csffci_link_t* L = Lbuf;
        const int ncol = (int)min((long long)NB, jend);
        for (int idx = tid; idx < nla * NB; idx += NTH) {
          const int l = idx / NB, jb = idx - l * NB;
          if (jb < ncol) {
            const csffci_link_t e = las[l];
            cp_async8(&D[rr_pair(e) * ds + jb], &g.ci[(long long)e.addr * Nb + jb]);
          }
        }
        for (int idx = tid; idx < ncol * nlb; idx += NTH) {
          const int jb = idx / nlb, m = idx - jb * nlb;
          cp_async8(&L[jb * LS + m], &g.lb[idx]);
        }
        cp_async_commit();
      }
      for (int ch = 0; ch < nchunk; ++ch) {
        const int b = ch & 1;
        const long long j0 = (long long)ch * NB;
        const int ncol = (int)min((long long)NB, jend - j0);
        double* D = Dbuf + b * dsz;
        csffci_link_t* L = Lbuf + b * lsz;
        cp_async_wait_all();
        __syncthreads();
        // rows without an alpha link start from zero; alpha rows with a
        // negative sign are negated (the copies brought the raw values)
        const int nz = zrow[0], nfix = zrow[1];
        for (int idx = tid; idx < nfix * NB; idx += NTH) {
          const int i = idx / NB, jb = idx - i * NB;
          double* p = &D[zrow[2 + i] * ds + jb];
          *p = i < nz ? 0.0 : -*p;
        }
        __syncthreads();
        for (int idx = tid; idx < nlb * NB; idx += NTH) {
          const int m = idx / NB, jb = idx - m * NB;
          if (jb < ncol) {
            const csffci_link_t e = L[jb * LS + m];
            D[rr_pair(e) * ds + jb] += e.sign * crow[e.addr];
          }
        }
        __syncthreads();
        if (ch + 1 < nchunk) {
          double* D2 = Dbuf + (b ^ 1) * dsz;
          csffci_link_t* L2 = Lbuf + (b ^ 1) * lsz;
          const long long j1 = j0 + NB;
          const int ncol2 = (int)min((long long)NB, jend - j1);
          for (int idx = tid; idx < nla * NB; idx += NTH) {
            const int l = idx / NB, jb = idx - l * NB;
            if (jb < ncol2) {
              const csffci_link_t e = las[l];
              cp_async8(&D2[rr_pair(e) * ds + jb], &g.ci[(long long)e.addr * Nb + j1 + jb]);
            }
          }
          const csffci_link_t* src = g.lb + j1 * nlb;
          for (int idx = tid; idx < ncol2 * nlb; idx += NTH) {
            const int jb = idx / nlb, m = idx - jb * nlb;
            cp_async8(&L2[jb * LS + m], &src[idx]);
          }
          cp_async_commit();
        }
        // V = H D on the FP64 tensor cores
        double acc[NT][4];
#pragma unroll
        for (int t = 0; t < NT; ++t) acc[t][0] = acc[t][1] = acc[t][2] = acc[t][3] = 0.0;
        const double* Db = D + tq * ds + gq;
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
        __syncthreads();
        {
          const int r0 = warp * MW + gq, r1 = r0 + 8;
#pragma unroll
          for (int t = 0; t < NT; ++t) {
            if (r0 < npair) {
              D[r0 * ds + 8 * t + 2 * tq] = acc[t][0];
              D[r0 * ds + 8 * t + 2 * tq + 1] = acc[t][1];
            }
            if (MW == 16 && r1 < npair) {
              D[r1 * ds + 8 * t + 2 * tq] = acc[t][2];
              D[r1 * ds + 8 * t + 2 * tq + 1] = acc[t][3];
            }
          }
        }
        __syncthreads();
        // row-local scatter through the beta links of each column
        for (int idx = tid; idx < nlb * NB; idx += NTH) {
          const int m = idx / NB, jb = idx - m * NB;
          if (jb < ncol) {
            const csffci_link_t e = L[jb * LS + m];
            atomicAdd(&g.out[ja * Nb + e.addr], e.sign * D[rr_pair(e) * ds + jb]);
          }
        }
        // alpha scatter sigma[Ka][Jb] through the links of Ja (coalesced over
        // Jb); in the spin-symmetric mode only Jb < Ja
        for (int idx = tid; idx < nla * NB; idx += NTH) {
          const int l = idx / NB, jb = idx - l * NB;
          const long long J = j0 + jb;
          if (jb < ncol && (!SYM || J < ja)) {
            const csffci_link_t e = las[l];
            atomicAdd(&g.out[(long long)e.addr * Nb + J], e.sign * D[rr_pair(e) * ds + jb]);
          }
        }
      }
    }
  }
}

template <int KS, int NW, int MW, int NT, bool SYM>
static int launch_rr(RRArgs& g, size_t smem, cudaStream_t stream) {
  auto kern = k_sigma_rr<KS, NW, MW, NT, SYM>;
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
  if (grid > g.nunits) grid = g.nunits;
  ProfScope ps("k_sigma_rr", stream);
  kern<<<(int)grid, NW * 32, smem, stream>>>(g);
  return check_launch("sigma (register-resident)");
}

bool sigma_rr_supported(int norb) { return norb >= 8 && norb <= 16; }

// (rows per warp, n-tiles): 16-row warps halve the B-fragment traffic but
// need 2*KS + 4*NT doubles of registers per lane; with 9 warps (norb 15,16)
// an SMSP holds 3 warps, i.e. at most 168 registers, so those sizes use
// either 8-row warps or two n-tiles.  CSFFCI_SIGMA_MW overrides (8 or 16).
static int rr_rows_per_warp(int norb) {
  const char* env = getenv("CSFFCI_SIGMA_MW");
  if (env && atoi(env) == 8) return 8;
  if (env && atoi(env) == 16) return 16;
  return norb >= 15 ? 8 : 16;
}

int sigma_rr_run(int norb, int neleca, int nelecb, const double* h2e, const csffci_link_t* la,
                 const csffci_link_t* lb, const double* ci, double* out, bool sym, double eta,
                 cudaStream_t stream) {
  (void)eta;  // the caller forms sigma = s + eta s^T
  const int npair = norb * (norb + 1) / 2;
  const int ks = (npair + 3) / 4;
  const int mw = rr_rows_per_warp(norb);
  const int nt = (mw == 16 && norb >= 15) ? 2 : 4;
  const int nb = 8 * nt;
  RRArgs g;
  g.h2e = h2e;
  g.la = la;
  g.lb = lb;
  g.ci = ci;
  g.out = out;
  g.Na = (long long)host_binom(norb, neleca);
  g.Nb = (long long)host_binom(norb, nelecb);
  g.npair = npair;
  g.nla = neleca * (norb - neleca + 1);
  g.nlb = nelecb * (norb - nelecb + 1);
  g.ds = nb + 8;     // = 8 (mod 16)
  g.ls = g.nlb | 1;  // odd stride
  g.nd_rows = 4 * ks > ((npair + mw - 1) / mw) * mw ? 4 * ks : ((npair + mw - 1) / mw) * mw;
  g.nunits = sym ? (g.Na + 1) / 2 : g.Na;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 15) & ~(size_t)15;
    return (unsigned)o;
  };
  g.off_d = take((size_t)2 * g.nd_rows * g.ds * sizeof(double));
  g.off_l = take((size_t)2 * nb * g.ls * sizeof(csffci_link_t));
  g.off_crow = take((size_t)g.Nb * sizeof(double));
  g.off_las = take((size_t)(g.nla > 0 ? g.nla : 1) * sizeof(csffci_link_t));
  g.off_rowsrc = take((size_t)g.nd_rows * sizeof(int));
  g.off_zrow = take((size_t)(npair + 2) * sizeof(int));
  const size_t smem = off;
  if (smem > 227 * 1024) {
    set_error("sigma: tile of %zu bytes exceeds shared memory", smem);
    return CSFFCI_ERR_INVALID;
  }
#define RR_LAUNCH(K, W, M, T) \
  return sym ? launch_rr<K, W, M, T, true>(g, smem, stream) : launch_rr<K, W, M, T, false>(g, smem, stream)
  switch (norb) {
    case 8: RR_LAUNCH(9, 3, 16, 4);
    case 9: RR_LAUNCH(12, 3, 16, 4);
    case 10: RR_LAUNCH(14, 4, 16, 4);
    case 11: RR_LAUNCH(17, 5, 16, 4);
    case 12: RR_LAUNCH(20, 5, 16, 4);
    case 13: RR_LAUNCH(23, 6, 16, 4);
    case 14: RR_LAUNCH(27, 7, 16, 4);
    case 15:
      if (mw == 16) RR_LAUNCH(30, 8, 16, 2);
      RR_LAUNCH(30, 15, 8, 4);
    case 16:
      if (mw == 16) RR_LAUNCH(34, 9, 16, 2);
      RR_LAUNCH(34, 17, 8, 4);
    default:
      set_error("sigma: no register-resident instance for norb=%d", norb);
      return CSFFCI_ERR_INVALID;
  }
#undef RR_LAUNCH
}

}  // namespace csffci
