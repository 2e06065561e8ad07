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
#include <string.h>

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
template <int KS, int NW, int MW, int NT, bool BATCH>
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

  __shared__ csffci_sigma_job_t sjob_s;
  __shared__ int sjob_idx;
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

  for (long long u = blockIdx.x; u < g.total_units; u += gridDim.x) {
    if (BATCH) {
      __syncthreads();  // everything of the previous unit is consumed
      if (tid == 0) {
        int j = cur < 0 ? 0 : cur;
        while (j + 1 < g.njobs && g.jobs[j + 1].unit_begin <= u) ++j;
        if (j != cur) sjob_s = g.jobs[j];
        sjob_idx = j;
      }
      __syncthreads();
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

template <int KS, int NW, int MW, int NT>
static int launch_rr(RRArgs& g, size_t smem, cudaStream_t stream) {
  auto kern = g.njobs > 1 ? k_sigma_rr<KS, NW, MW, NT, true> : k_sigma_rr<KS, NW, MW, NT, false>;
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
  ProfScope ps("k_sigma_rr", stream);
  kern<<<(int)grid, NW * 32, smem, stream>>>(g);
  return check_launch("sigma (register-resident)");
}

bool sigma_rr_supported(int norb) { return norb >= 4 && norb <= 16; }

// (rows per warp, n-tiles): 16-row warps halve the B-fragment traffic but
// need 2*KS + 4*NT doubles of registers per lane; with 9 warps (norb 15,16)
// an SMSP holds 3 warps, i.e. at most 168 registers, so those sizes use
// 8-row warps (CSFFCI_SIGMA_MW=16 selects 16-row warps with two n-tiles).
static int rr_rows_per_warp(int norb) {
  const char* env = getenv("CSFFCI_SIGMA_MW");
  if (env && atoi(env) == 8) return 8;
  if (env && atoi(env) == 16) return 16;
  return norb >= 15 ? 8 : 16;
}

// fill the bookkeeping fields of the jobs; returns the largest Nb, nla, nlb
static void rr_prepare(int norb, int njobs, csffci_sigma_job_t* jobs, long long* total_units,
                       long long* max_nb, int* max_nla, int* max_nlb) {
  long long u = 0, t = 0, e = 0;
  *max_nb = 0;
  *max_nla = *max_nlb = 0;
  for (int i = 0; i < njobs; ++i) {
    csffci_sigma_job_t& J = jobs[i];
    J.Na = (long long)host_binom(norb, J.neleca);
    J.Nb = (long long)host_binom(norb, J.nelecb);
    J.nla = J.neleca * (norb - J.neleca + 1);
    J.nlb = J.nelecb * (norb - J.nelecb + 1);
    J.nunits = J.sym ? (J.Na + 1) / 2 : J.Na;
    J.unit_begin = u;
    u += J.nunits;
    J.tile_begin = t;
    t += J.sym ? ((J.Na + 31) / 32) * ((J.Na + 31) / 32) : 0;
    J.elem_begin = e;
    e += J.Na * J.Nb;
    if (J.Nb > *max_nb) *max_nb = J.Nb;
    if (J.nla > *max_nla) *max_nla = J.nla;
    if (J.nlb > *max_nlb) *max_nlb = J.nlb;
  }
  *total_units = u;
}

int sigma_rr_launch(int norb, int njobs, const csffci_sigma_job_t* jobs_dev,
                    const csffci_sigma_job_t& job0, long long total_units, long long max_nb,
                    int max_nla, int max_nlb, cudaStream_t stream) {
  const int npair = norb * (norb + 1) / 2;
  const int ks = (npair + 3) / 4;
  const int mw = rr_rows_per_warp(norb);
  const int nt = (mw == 16 && norb >= 15) ? 2 : 4;
  const int nb = 8 * nt;
  RRArgs g;
  g.jobs = jobs_dev;
  g.job0 = job0;
  g.njobs = njobs;
  g.total_units = total_units;
  g.npair = npair;
  g.ds = nb + 8;          // = 8 (mod 16)
  g.ls = max_nlb | 1;     // odd stride
  const int rows_w = ((npair + mw - 1) / mw) * mw;
  g.nd_rows = 4 * ks > rows_w ? 4 * ks : rows_w;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 15) & ~(size_t)15;
    return (unsigned)o;
  };
  g.off_d = take((size_t)2 * g.nd_rows * g.ds * sizeof(double));
  g.off_l = take((size_t)2 * nb * g.ls * sizeof(csffci_link_t));
  g.off_crow = take((size_t)max_nb * sizeof(double));
  g.off_las = take((size_t)(max_nla > 0 ? max_nla : 1) * sizeof(csffci_link_t));
  g.off_rowsrc = take((size_t)g.nd_rows * sizeof(int));
  g.off_zrow = take((size_t)(npair + 2) * sizeof(int));
  const size_t smem = off;
  if (smem > 227 * 1024 - 256) {
    set_error("sigma: tile of %zu bytes exceeds shared memory", smem);
    return CSFFCI_ERR_INVALID;
  }
#define RR_LAUNCH(K, W, M, T) return launch_rr<K, W, M, T>(g, smem, stream)
  switch (norb) {
    case 4: RR_LAUNCH(3, 1, 16, 4);
    case 5: RR_LAUNCH(4, 1, 16, 4);
    case 6: RR_LAUNCH(6, 2, 16, 4);
    case 7: RR_LAUNCH(7, 2, 16, 4);
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

int sigma_rr_run(int norb, int neleca, int nelecb, const double* h2e, const csffci_link_t* la,
                 const csffci_link_t* lb, const double* ci, double* out, bool sym, double eta,
                 cudaStream_t stream) {
  csffci_sigma_job_t J;
  memset(&J, 0, sizeof(J));
  J.h2e = h2e;
  J.link_a = la;
  J.link_b = lb;
  J.ci = ci;
  J.sigma = out;
  J.scratch = out;
  J.neleca = neleca;
  J.nelecb = nelecb;
  J.sym = sym ? 1 : 0;
  J.eta = eta < 0 ? -1 : 1;
  long long total, maxnb;
  int mla, mlb;
  rr_prepare(norb, 1, &J, &total, &maxnb, &mla, &mlb);
  return sigma_rr_launch(norb, 1, nullptr, J, total, maxnb, mla, mlb, stream);
}

// ---- batch: zero the outputs, run the jobs, form sigma = S + eta S^T -----
__global__ void k_batch_zero(const csffci_sigma_job_t* jobs, int njobs, long long total) {
  int j = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    while (j + 1 < njobs && jobs[j + 1].elem_begin <= i) ++j;
    const csffci_sigma_job_t& J = jobs[j];
    (J.sym ? J.scratch : J.sigma)[i - J.elem_begin] = 0.0;
  }
}

__global__ void k_batch_sym_add(const csffci_sigma_job_t* jobs, int njobs, long long total_tiles) {
  __shared__ double tile[32][33];
  int j = 0;
  for (long long t = blockIdx.x; t < total_tiles; t += gridDim.x) {
    while (j + 1 < njobs && (jobs[j + 1].tile_begin <= t || jobs[j + 1].Na == 0)) {
      if (jobs[j + 1].tile_begin > t) break;
      ++j;
    }
    while (!jobs[j].sym) ++j;  // non-symmetric jobs own no tiles
    const csffci_sigma_job_t& J = jobs[j];
    const long long n = J.Na;
    const long long ntile = (n + 31) / 32;
    const long long lt = t - J.tile_begin;
    const long long ti = lt / ntile, tj = lt - ti * ntile;
    const double* s = J.scratch;
    const double eta = (double)J.eta;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      long long row = tj * 32 + r, col = ti * 32 + threadIdx.x;
      tile[r][threadIdx.x] = (row < n && col < n) ? s[row * n + col] : 0.0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      long long row = ti * 32 + r, col = tj * 32 + threadIdx.x;
      if (row < n && col < n) J.sigma[row * n + col] = s[row * n + col] + eta * tile[threadIdx.x][r];
    }
    __syncthreads();
  }
}

}  // namespace csffci

using namespace csffci;

extern "C" {

size_t csffci_sigma_batch_workspace(int njobs) {
  return (size_t)(njobs > 0 ? njobs : 1) * sizeof(csffci_sigma_job_t);
}

int csffci_sigma_batch(int norb, int njobs, csffci_sigma_job_t* jobs, void* work, size_t work_bytes,
                       cudaStream_t stream) {
  CSF_REQUIRE(norb >= 4 && norb <= 16, "sigma_batch: norb=%d outside [4,16]", norb);
  CSF_REQUIRE(njobs >= 0 && (njobs == 0 || jobs != nullptr), "sigma_batch: bad job list");
  if (njobs == 0) return CSFFCI_OK;
  for (int i = 0; i < njobs; ++i) {
    const csffci_sigma_job_t& J = jobs[i];
    CSF_REQUIRE(J.neleca >= 0 && J.nelecb >= 0 && J.neleca <= norb && J.nelecb <= norb,
                "sigma_batch: job %d has bad nelec (%d,%d)", i, J.neleca, J.nelecb);
    CSF_REQUIRE(!J.sym || (J.neleca == J.nelecb && J.scratch != nullptr && (J.eta == 1 || J.eta == -1)),
                "sigma_batch: job %d: spin-symmetric mode needs neleca == nelecb, eta = +-1 and scratch", i);
    CSF_REQUIRE(J.h2e && J.link_a && J.link_b && J.ci && J.sigma, "sigma_batch: job %d has a NULL pointer", i);
  }
  if (work == nullptr || work_bytes < csffci_sigma_batch_workspace(njobs)) {
    set_error("sigma_batch: workspace of %zu bytes < %zu required", work_bytes,
              csffci_sigma_batch_workspace(njobs));
    return CSFFCI_ERR_MEMORY;
  }
  long long total, maxnb;
  int mla, mlb;
  rr_prepare(norb, njobs, jobs, &total, &maxnb, &mla, &mlb);
  long long nelem = jobs[njobs - 1].elem_begin + jobs[njobs - 1].Na * jobs[njobs - 1].Nb;
  long long ntiles = 0;
  for (int i = 0; i < njobs; ++i)
    if (jobs[i].sym) ntiles = jobs[i].tile_begin + ((jobs[i].Na + 31) / 32) * ((jobs[i].Na + 31) / 32);
  csffci_sigma_job_t* dj = (csffci_sigma_job_t*)work;
  CSF_CUDA(cudaMemcpyAsync(dj, jobs, njobs * sizeof(csffci_sigma_job_t), cudaMemcpyHostToDevice, stream));
  k_batch_zero<<<grid_for(nelem, 256, 148 * 16), 256, 0, stream>>>(dj, njobs, nelem);
  int st = check_launch("sigma_batch zero");
  if (st) return st;
  st = njobs > 1 ? sigma_rr_launch(norb, njobs, dj, jobs[0], total, maxnb, mla, mlb, stream)
                 : sigma_rr_launch(norb, 1, nullptr, jobs[0], total, maxnb, mla, mlb, stream);
  if (st) return st;
  if (ntiles > 0) {
    dim3 blk(32, 8);
    ProfScope ps("k_batch_sym_add", stream);
    k_batch_sym_add<<<grid_for(ntiles, 1, 148 * 16), blk, 0, stream>>>(dj, njobs, ntiles);
    return check_launch("sigma_batch symmetric add");
  }
  return CSFFCI_OK;
}

}  // extern "C"
