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
#include "common.cuh"
#include "profile.cuh"
#include "sigma_rr.cuh"

namespace csffci {

__device__ __forceinline__ void rr_dmma(double& c0, double& c1, double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(c0), "+d"(c1)
      : "d"(a), "d"(b));
}

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
  int npair, ds, ls, nla, nlb;
  double eta;
  unsigned off_d, off_l, off_crow, off_las, off_rowsrc;
};

constexpr int RR_NT = 4, RR_NB = 32;

template <int KS, bool SYM>
__global__ void __launch_bounds__(KS * 16, 1) k_sigma_rr(RRArgs g) {
  constexpr int NPAD = KS * 4;
  constexpr int NTH = KS * 16;
  constexpr int NT = RR_NT, NB = RR_NB;
  extern __shared__ __align__(16) unsigned char smraw[];
  double* Dbuf = (double*)(smraw + g.off_d);
  csffci_link_t* Lbuf = (csffci_link_t*)(smraw + g.off_l);
  double* crow = (double*)(smraw + g.off_crow);
  csffci_link_t* las = (csffci_link_t*)(smraw + g.off_las);
  int* rowsrc = (int*)(smraw + g.off_rowsrc);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long Nb = g.Nb;
  const int ds = g.ds, LS = g.ls, nla = g.nla, nlb = g.nlb;
  const size_t dsz = (size_t)NPAD * ds, lsz = (size_t)NB * LS;

  double afrag[KS];
  {
    const int r = warp * 8 + (lane >> 2);
#pragma unroll
    for (int s = 0; s < KS; ++s) {
      const int c = 4 * s + (lane & 3);
      afrag[s] = (r < g.npair && c < g.npair) ? g.h2e[(long long)r * g.npair + c] : 0.0;
    }
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
      for (int r = tid; r < NPAD; r += NTH) rowsrc[r] = -1;
      __syncthreads();
      for (int l = tid; l < nla; l += NTH) {
        csffci_link_t e = g.la[ja * nla + l];
        las[l] = e;
        rowsrc[rr_pair(e)] = l;
      }
      __syncthreads();
      for (long long i = tid; i < Nb; i += NTH) cp_async8(&crow[i], &g.ci[ja * Nb + i]);
      // first tile of the row (committed together with crow)
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
        // signs of the alpha rows; zero the other rows and the unused columns
        for (int idx = tid; idx < NPAD * NB; idx += NTH) {
          const int r = idx / NB, jb = idx - r * NB;
          const int l = rowsrc[r];
          double v = 0.0;
          if (l >= 0 && jb < ncol) v = las[l].sign * D[r * ds + jb];
          D[r * ds + jb] = v;
        }
        __syncthreads();
        // + beta links of every column, read from the cached row of c
        for (int idx = tid; idx < nlb * NB; idx += NTH) {
          const int m = idx / NB, jb = idx - m * NB;
          if (jb < ncol) {
            const csffci_link_t e = L[jb * LS + m];
            D[rr_pair(e) * ds + jb] += e.sign * crow[e.addr];
          }
        }
        __syncthreads();
        // prefetch the next tile of this row into the other buffer
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
        // V = H . D on the FP64 tensor cores (A fragments in registers)
        double acc[NT][2];
#pragma unroll
        for (int t = 0; t < NT; ++t) acc[t][0] = acc[t][1] = 0.0;
        const double* Db = D + (lane & 3) * ds + (lane >> 2);
#pragma unroll
        for (int s = 0; s < KS; ++s) {
#pragma unroll
          for (int t = 0; t < NT; ++t) rr_dmma(acc[t][0], acc[t][1], afrag[s], Db[4 * s * ds + 8 * t]);
        }
        __syncthreads();
        {
          double* dst = D + (warp * 8 + (lane >> 2)) * ds + 2 * (lane & 3);
#pragma unroll
          for (int t = 0; t < NT; ++t) {
            dst[8 * t] = acc[t][0];
            dst[8 * t + 1] = acc[t][1];
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
        // transposed (SYM) or alpha (general) scatter through the links of Ja
        for (int idx = tid; idx < nla * NB; idx += NTH) {
          const int l = idx / NB, jb = idx - l * NB;
          const long long J = j0 + jb;
          if (jb < ncol) {
            const csffci_link_t e = las[l];
            const double v = e.sign * D[rr_pair(e) * ds + jb];
            if (SYM) {
              if (J < ja) atomicAdd(&g.out[J * Nb + e.addr], g.eta * v);
            } else {
              atomicAdd(&g.out[(long long)e.addr * Nb + J], v);
            }
          }
        }
      }
    }
  }
}

template <int KS, bool SYM>
static int launch_rr(RRArgs& g, size_t smem, cudaStream_t stream) {
  auto kern = k_sigma_rr<KS, SYM>;
  CSF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev = 0, nsm = 148, per_sm = 1;
  CSF_CUDA(cudaGetDevice(&dev));
  CSF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  CSF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, KS * 16, smem));
  if (per_sm < 1) {
    set_error("sigma: register-resident kernel does not fit on an SM (smem %zu)", smem);
    return CSFFCI_ERR_INVALID;
  }
  long long grid = (long long)nsm * per_sm;
  if (grid > g.nunits) grid = g.nunits;
  ProfScope ps("k_sigma_rr", stream);
  kern<<<(int)grid, KS * 16, smem, stream>>>(g);
  return check_launch("sigma (register-resident)");
}

bool sigma_rr_supported(int norb) { return norb >= 8 && norb <= 16; }

int sigma_rr_run(int norb, int neleca, int nelecb, const double* h2e, const csffci_link_t* la,
                 const csffci_link_t* lb, const double* ci, double* out, bool sym, double eta,
                 cudaStream_t stream) {
  const int npair = norb * (norb + 1) / 2;
  const int npad = (npair + 7) & ~7;
  const int ks = npad / 4;
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
  g.ds = RR_NB + 8;  // 40 = 8 (mod 16)
  g.ls = g.nlb | 1;  // odd stride
  g.eta = eta;
  g.nunits = sym ? (g.Na + 1) / 2 : g.Na;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 15) & ~(size_t)15;
    return (unsigned)o;
  };
  g.off_d = take((size_t)2 * npad * g.ds * sizeof(double));
  g.off_l = take((size_t)2 * RR_NB * g.ls * sizeof(csffci_link_t));
  g.off_crow = take((size_t)g.Nb * sizeof(double));
  g.off_las = take((size_t)(g.nla > 0 ? g.nla : 1) * sizeof(csffci_link_t));
  g.off_rowsrc = take((size_t)npad * sizeof(int));
  const size_t smem = off;
  if (smem > 227 * 1024) {
    set_error("sigma: tile of %zu bytes exceeds shared memory", smem);
    return CSFFCI_ERR_INVALID;
  }
#define RR_CASE(K)                                                                  \
  case K:                                                                           \
    return sym ? launch_rr<K, true>(g, smem, stream) : launch_rr<K, false>(g, smem, stream);
  switch (ks) {
    RR_CASE(10)
    RR_CASE(12)
    RR_CASE(14)
    RR_CASE(18)
    RR_CASE(20)
    RR_CASE(24)
    RR_CASE(28)
    RR_CASE(30)
    RR_CASE(34)
    default:
      set_error("sigma: no register-resident instance for norb=%d", norb);
      return CSFFCI_ERR_INVALID;
  }
#undef RR_CASE
}

}  // namespace csffci
