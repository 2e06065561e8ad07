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

__device__ __forceinline__ int rr_pair(const csffci_link_t& e) {
  int p = e.op & 0xff, q = e.op >> 8;
  int hi = p > q ? p : q, lo = p > q ? q : p;
  return hi * (hi + 1) / 2 + lo;
}

struct RRArgs {
  const csffci_sigma_job_t* jobs;  // device array (njobs > 1) ...
  csffci_sigma_job_t job0;         // ... or the single job by value
  int njobs;
  long long total_units;
  int npair, ds, ls, nd_rows;
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
// CTAs per SM the register allocation is sized for: the (16, 4) and (8, 4)
// shapes keep every register they need (one CTA per SM); the two-n-tile
// shapes cap registers so that small orbital counts, whose CTAs have few
// warps, run two or three CTAs per SM.
template <int NW, int MW, int NT>
constexpr int rr_min_blocks() {
  return NT == 2 ? (MW == 16 ? (NW <= 5 ? 3 : NW <= 6 ? 2 : 1) : (NW <= 10 ? 2 : 1)) : 1;
}

template <int KS, int NW, int MW, int NT, bool BATCH>
__global__ void __launch_bounds__(NW * 32, (rr_min_blocks<NW, MW, NT>())) k_sigma_rr(RRArgs g) {
  constexpr int NTH = NW * 32;
  constexpr int NB = 8 * NT;
  extern __shared__ __align__(16) unsigned char smraw[];
  double* Dbuf = (double*)(smraw + g.off_d);
  csffci_link_t* Lbuf = (csffci_link_t*)(smraw + g.off_l);
  double* crow = (double*)(smraw + g.off_crow);
  csffci_link_t* las = (csffci_link_t*)(smraw + g.off_las);
  int* rowsrc = (int*)(smraw + g.off_rowsrc);  // alpha link of a pair row, -1 if none
  int* zrow = (int*)(smraw + g.off_zrow);      // [0] = count, then the rows without one

  __shared__ csffci_sigma_job_t sjob_s;
  __shared__ int sjob_idx, sjob_live;
  // the single-problem launch reads its job from the parameter bank
  const csffci_sigma_job_t& sjob = BATCH ? sjob_s : g.job0;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  const int ds = g.ds, LS = g.ls, npair = g.npair;
  const int ndr = g.nd_rows;
  const size_t dsz = (size_t)ndr * ds, lsz = (size_t)NB * LS;

  // h2e rows MW*w+g (and MW*w+8+g), columns 4s+t of the current job,
  // resident in registers until the CTA moves to another job
  double a0f[KS], a1f[MW == 16 ? KS : 1];
  // rows past npair are k rows of the MMA that nothing else writes
  for (int i = tid; i < (ndr - npair) * ds; i += NTH) {
    Dbuf[npair * ds + i] = 0.0;
    Dbuf[dsz + npair * ds + i] = 0.0;
  }
  int cur = -1;
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
      const int r0 = warp * MW + gq, r1 = r0 + 8;
#pragma unroll
      for (int s = 0; s < KS; ++s) {
        const int c = 4 * s + tq;
        a0f[s] = (r0 < npair && c < npair) ? h2e[(long long)r0 * npair + c] : 0.0;
        if (MW == 16) a1f[s] = (r1 < npair && c < npair) ? h2e[(long long)r1 * npair + c] : 0.0;
      }
    }
    const long long Nb = sjob.Nb;
    const int nla = sjob.nla, nlb = sjob.nlb;
    const bool SYM = sjob.sym != 0;
    double* const out = SYM ? sjob.scratch : sjob.sigma;
    const long long lu = u - sjob.unit_begin;
    for (int w = 0; w < (SYM ? 2 : 1); ++w) {
      long long ja = lu;
      if (SYM && w == 1) {
        ja = sjob.Na - 1 - lu;
        if (ja <= lu) break;
      }
      const long long jend = SYM ? ja + 1 : Nb;
      const int nchunk = (int)((jend + NB - 1) / NB);
      __syncthreads();  // the previous row is fully consumed
      for (int r = tid; r < ndr; r += NTH) rowsrc[r] = -1;
      __syncthreads();
      for (int l = tid; l < nla; l += NTH) {
        csffci_link_t e = sjob.link_a[ja * nla + l];
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
      for (long long i = tid; i < Nb; i += NTH) cp_async8(&crow[i], &sjob.ci[ja * Nb + i]);
      {
        double* D = Dbuf;
        csffci_link_t* L = Lbuf;
        const int ncol = (int)min((long long)NB, jend);
        for (int idx = tid; idx < nla * NB; idx += NTH) {
          const int l = idx / NB, jb = idx - l * NB;
          if (jb < ncol) {
            const csffci_link_t e = las[l];
            cp_async8(&D[rr_pair(e) * ds + jb], &sjob.ci[(long long)e.addr * Nb + jb]);
          }
        }
        for (int idx = tid; idx < ncol * nlb; idx += NTH) {
          const int jb = idx / nlb, m = idx - jb * nlb;
          cp_async8(&L[jb * LS + m], &sjob.link_b[idx]);
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
              cp_async8(&D2[rr_pair(e) * ds + jb], &sjob.ci[(long long)e.addr * Nb + j1 + jb]);
            }
          }
          const csffci_link_t* src = sjob.link_b + j1 * nlb;
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
            atomicAdd(&out[ja * Nb + e.addr], e.sign * D[rr_pair(e) * ds + jb]);
          }
        }
        // alpha scatter sigma[Ka][Jb] through the links of Ja (coalesced over
        // Jb); in the spin-symmetric mode only Jb < Ja
        for (int idx = tid; idx < nla * NB; idx += NTH) {
          const int l = idx / NB, jb = idx - l * NB;
          const long long J = j0 + jb;
          if (jb < ncol && (!SYM || J < ja)) {
            const csffci_link_t e = las[l];
            atomicAdd(&out[(long long)e.addr * Nb + J], e.sign * D[rr_pair(e) * ds + jb]);
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

template <int KS, int NW, int MW, int NT>
static int launch_rr(RRArgs& g, size_t smem, cudaStream_t stream) {
  auto kern = g.jobs ? k_sigma_rr<KS, NW, MW, NT, true> : k_sigma_rr<KS, NW, MW, NT, false>;
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
bool rr_variant_valid(int norb, int v);
int rr_default_variant(int norb);
int sigma_rr_launch(int norb, int njobs, const csffci_sigma_job_t* jobs_dev, const csffci_sigma_job_t& job0,
                    long long total_units, long long max_nb, int max_nla, int max_nlb, cudaStream_t stream,
                    int variant);
int rr_dispatch_v0(int norb, RRArgs& g, size_t smem, cudaStream_t stream);  // (16, 4)
int rr_dispatch_v1(int norb, RRArgs& g, size_t smem, cudaStream_t stream);  // (8, 4)
int rr_dispatch_v2(int norb, RRArgs& g, size_t smem, cudaStream_t stream);  // (16, 2)
int rr_dispatch_v3(int norb, RRArgs& g, size_t smem, cudaStream_t stream);  // (8, 2)

}  // namespace csffci
