// sigma = sum_{pq,rs} h2e[pq][rs] E_pq E_rs c  (the direct_spin1 contraction
// the reference calls at pyscf/csf_fci/csf.py:449 through CSFFCISolver.
// contract_2e, csf.py:525-529).
//
// Per tile (one alpha string Ja x NB consecutive beta strings):
//   D[pq][jb] = sum_{alpha links of Ja} s c[Ia][Jb] + sum_{beta links of Jb} s c[Ja][Ib]
//   V = h2e . D                                  (FP64 DMMA, m8n8k4)
//   sigma[Ka][Jb] += s V[pq][jb]  for alpha links (E_pq Ja = s Ka)
//   sigma[Ja][Kb] += s V[pq][jb]  for beta links  (E_pq Jb = s Kb)
// Gather and scatter use the same link rows because h2e is symmetric.
// h2e stays resident in shared memory (persistent CTAs, one per SM) when
// it fits (norb <= 16).  In the spin-symmetric mode (na == nb and
// c = eta c^T, true for every vector produced from CSFs with MS = 0) only
// the beta scatter is done and sigma = s + eta s^T, which removes every
// cross-row update.
#include "common.cuh"
#include "profile.cuh"
#include <new>

#include "sigma_rr.cuh"

namespace csffci {

__device__ __forceinline__ void dmma884(double& c0, double& c1, double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(c0), "+d"(c1)
      : "d"(a), "d"(b));
}

struct SigmaArgs {
  const double* h2e;
  const csffci_link_t* la;
  const csffci_link_t* lb;
  const double* ci;
  double* out;
  long long Na, Nb;
  int norb, npair, npad, hstride, dstride;
  int nla, nlb;
  int alpha_scatter;
  long long nchunk, nitems;
};

__device__ __forceinline__ int link_pair(const csffci_link_t& e) {
  return pair_index(e.op & 0xff, e.op >> 8);
}

template <int NT, bool HSMEM>
__global__ void k_sigma(SigmaArgs g) {
  extern __shared__ __align__(16) double smem[];
  constexpr int NB = 8 * NT;
  double* Hs = smem;
  double* Ds = smem + (HSMEM ? (size_t)g.npad * g.hstride : 0);
  int* rowsrc = (int*)(Ds + (size_t)g.npad * g.dstride);
  csffci_link_t* las = (csffci_link_t*)(rowsrc + ((g.npad + 1) & ~1));

  const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, warp = tid >> 5;
  const long long Nb = g.Nb;

  if (HSMEM) {
    for (int i = tid; i < g.npad * g.npad; i += nth) {
      int r = i / g.npad, c = i - r * g.npad;
      Hs[r * g.hstride + c] = (r < g.npair && c < g.npair) ? g.h2e[(long long)r * g.npair + c] : 0.0;
    }
  }
  const long long G = gridDim.x;
  const long long it0 = g.nitems * blockIdx.x / G, it1 = g.nitems * (blockIdx.x + 1) / G;
  long long cur_ja = -1;
  const int m0 = warp * 8;

  for (long long it = it0; it < it1; ++it) {
    const long long ja = it / g.nchunk;
    const long long j0 = (it - ja * g.nchunk) * NB;
    __syncthreads();
    if (ja != cur_ja) {
      for (int r = tid; r < g.npad; r += nth) rowsrc[r] = -1;
      __syncthreads();
      for (int l = tid; l < g.nla; l += nth) {
        csffci_link_t e = g.la[ja * g.nla + l];
        las[l] = e;
        rowsrc[link_pair(e)] = l;
      }
      __syncthreads();
      cur_ja = ja;
    }
    // D rows from the alpha links of Ja (zero where Ja has no link)
    for (int idx = tid; idx < g.npad * NB; idx += nth) {
      int r = idx / NB, jb = idx - r * NB;
      int l = rowsrc[r];
      double v = 0.0;
      if (l >= 0 && j0 + jb < Nb) {
        csffci_link_t e = las[l];
        v = e.sign * __ldg(&g.ci[(long long)e.addr * Nb + j0 + jb]);
      }
      Ds[r * g.dstride + jb] = v;
    }
    __syncthreads();
    // + beta links of each Jb (distinct pairs per column: no conflicts)
    for (int idx = tid; idx < NB * g.nlb; idx += nth) {
      int jb = idx / g.nlb, m = idx - jb * g.nlb;
      if (j0 + jb < Nb) {
        csffci_link_t e = g.lb[(j0 + jb) * g.nlb + m];
        Ds[link_pair(e) * g.dstride + jb] += e.sign * __ldg(&g.ci[ja * Nb + e.addr]);
      }
    }
    __syncthreads();
    // V = H . D on the FP64 tensor cores; warp w owns rows 8w..8w+7
    double acc[NT][2];
#pragma unroll
    for (int t = 0; t < NT; ++t) acc[t][0] = acc[t][1] = 0.0;
    const int arow = m0 + (lane >> 2);
    for (int k0 = 0; k0 < g.npad; k0 += 4) {
      const int kr = k0 + (lane & 3);
      double a;
      if (HSMEM) {
        a = Hs[arow * g.hstride + kr];
      } else {
        a = (arow < g.npair && kr < g.npair) ? __ldg(&g.h2e[(long long)arow * g.npair + kr]) : 0.0;
      }
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        double b = Ds[kr * g.dstride + 8 * t + (lane >> 2)];
        dmma884(acc[t][0], acc[t][1], a, b);
      }
    }
    __syncthreads();
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      double* dst = Ds + arow * g.dstride + 8 * t + 2 * (lane & 3);
      dst[0] = acc[t][0];
      dst[1] = acc[t][1];
    }
    __syncthreads();
    if (g.alpha_scatter) {
      for (int idx = tid; idx < g.nla * NB; idx += nth) {
        int l = idx / NB, jb = idx - l * NB;
        if (j0 + jb < Nb) {
          csffci_link_t e = las[l];
          atomicAdd(&g.out[(long long)e.addr * Nb + j0 + jb], e.sign * Ds[link_pair(e) * g.dstride + jb]);
        }
      }
    }
    for (int idx = tid; idx < NB * g.nlb; idx += nth) {
      int jb = idx / g.nlb, m = idx - jb * g.nlb;
      if (j0 + jb < Nb) {
        csffci_link_t e = g.lb[(j0 + jb) * g.nlb + m];
        atomicAdd(&g.out[ja * Nb + e.addr], e.sign * Ds[link_pair(e) * g.dstride + jb]);
      }
    }
  }
}

// out[a][b] (+)= s[a][b] + eta * s[b][a]   (square n x n)
__global__ void k_sym_add(const double* __restrict__ s, double* out, long long n, double eta,
                          int accumulate) {
  __shared__ double tile[32][33];
  long long ntile = (n + 31) / 32;
  for (long long t = blockIdx.x; t < ntile * ntile; t += gridDim.x) {
    long long ti = t / ntile, tj = t - ti * ntile;
    // load s[tj block rows][ti block cols] transposed
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      long long row = tj * 32 + r, col = ti * 32 + threadIdx.x;
      tile[r][threadIdx.x] = (row < n && col < n) ? s[row * n + col] : 0.0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      long long row = ti * 32 + r, col = tj * 32 + threadIdx.x;
      if (row < n && col < n) {
        double v = s[row * n + col] + eta * tile[threadIdx.x][r];
        out[row * n + col] = accumulate ? out[row * n + col] + v : v;
      }
    }
    __syncthreads();
  }
}

// The deterministic mode's sigma from its three int64 digit planes w[k][i]
// (weights 2^-80, 2^-37, 2^6, see det_add3): out[i] (+)= the value of the
// digit sums.  Spin-symmetric: out[a][b] (+)= value(S[a][b] + eta S[b][a]),
// the digits of the two entries added as integers first (exact; the
// transpose is staged through a shared tile as in k_sym_add).  The three
// converted terms are exact (|digit sum| < 2^53) and are added in a fixed
// order, so the result depends on the digit sums alone.
__device__ __forceinline__ double det_value(long long w0, long long w1, long long w2) {
  return ((double)w2 * 0x1p6 + (double)w1 * 0x1p-37) + (double)w0 * 0x1p-80;
}

__global__ void k_det_finish(const long long* __restrict__ w, double* out, long long n, int accumulate) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double v = det_value(w[i], w[n + i], w[2 * n + i]);
    out[i] = accumulate ? out[i] + v : v;
  }
}

__global__ void k_det_finish_sym(const long long* __restrict__ w, double* out, long long na, int eta,
                                 int accumulate) {
  __shared__ long long tile[3][32][33];
  const long long n = na * na;
  const long long ntile = (na + 31) / 32;
  for (long long t = blockIdx.x; t < ntile * ntile; t += gridDim.x) {
    const long long ti = t / ntile, tj = t - ti * ntile;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      const long long row = tj * 32 + r, col = ti * 32 + threadIdx.x;
      const bool in = row < na && col < na;
#pragma unroll
      for (int k = 0; k < 3; ++k) tile[k][r][threadIdx.x] = in ? w[k * n + row * na + col] : 0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      const long long row = ti * 32 + r, col = tj * 32 + threadIdx.x;
      if (row < na && col < na) {
        long long d[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          // two's complement wrap-around: the exact integer sum (mod 2^64)
          const unsigned long long a = (unsigned long long)w[k * n + row * na + col];
          const unsigned long long b = (unsigned long long)tile[k][threadIdx.x][r];
          d[k] = (long long)(eta > 0 ? a + b : a - b);
        }
        const double v = det_value(d[0], d[1], d[2]);
        out[row * na + col] = accumulate ? out[row * na + col] + v : v;
      }
    }
    __syncthreads();
  }
}

// per-block maxima of |c - c^T|, |c + c^T|, |c| over a square n x n matrix
__global__ void k_parity_part(const double* __restrict__ c, long long n, double* part) {
  __shared__ double s0[256], s1[256], s2[256];
  double a = 0.0, b = 0.0, m = 0.0;
  long long tot = n * n;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot;
       i += (long long)gridDim.x * blockDim.x) {
    long long r = i / n, q = i - r * n;
    if (q > r) continue;
    double x = c[i], y = c[q * n + r];
    a = fmax(a, fabs(x - y));
    b = fmax(b, fabs(x + y));
    m = fmax(m, fmax(fabs(x), fabs(y)));
  }
  s0[threadIdx.x] = a;
  s1[threadIdx.x] = b;
  s2[threadIdx.x] = m;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      s0[threadIdx.x] = fmax(s0[threadIdx.x], s0[threadIdx.x + w]);
      s1[threadIdx.x] = fmax(s1[threadIdx.x], s1[threadIdx.x + w]);
      s2[threadIdx.x] = fmax(s2[threadIdx.x], s2[threadIdx.x + w]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x] = s0[0];
    part[3 * blockIdx.x + 1] = s1[0];
    part[3 * blockIdx.x + 2] = s2[0];
  }
}

__global__ void k_parity_final(const double* part, int np, double* out3) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double a = 0, b = 0, m = 0;
    for (int i = 0; i < np; ++i) {
      a = fmax(a, part[3 * i]);
      b = fmax(b, part[3 * i + 1]);
      m = fmax(m, part[3 * i + 2]);
    }
    out3[0] = a;
    out3[1] = b;
    out3[2] = m;
  }
}

struct SigmaConfig {
  int npad, hstride, dstride, nt, threads;
  bool hsmem;
  size_t smem;
};

static int pick_stride(int base, int want_mod16a, int want_mod16b) {
  int s = base;
  while ((s % 16) != want_mod16a && (s % 16) != want_mod16b) ++s;
  return s;
}

static SigmaConfig sigma_config(int norb, int nla) {
  SigmaConfig c;
  int npair = norb * (norb + 1) / 2;
  c.npad = (npair + 7) & ~7;
  c.threads = 4 * c.npad;
  c.hstride = pick_stride(c.npad, 4, 12);
  const size_t limit = 227 * 1024;
  size_t links = (size_t)((c.npad + 1) & ~1) * 4 + (size_t)nla * 8 + 64;
  c.hsmem = false;
  c.nt = 2;
  for (int nt : {8, 4, 2}) {
    int ds = pick_stride(8 * nt, 8, 8);
    size_t need = (size_t)c.npad * c.hstride * 8 + (size_t)c.npad * ds * 8 + links;
    if (need <= limit) {
      c.hsmem = true;
      c.nt = nt;
      c.dstride = ds;
      c.smem = need;
      return c;
    }
  }
  for (int nt : {8, 4, 2}) {
    int ds = pick_stride(8 * nt, 8, 8);
    size_t need = (size_t)c.npad * ds * 8 + links;
    if (need <= limit) {
      c.nt = nt;
      c.dstride = ds;
      c.smem = need;
      return c;
    }
  }
  c.nt = 0;
  return c;
}

template <int NT, bool HS>
static int launch_sigma(const SigmaConfig& c, SigmaArgs& g, int grid, cudaStream_t stream) {
  auto kern = k_sigma<NT, HS>;
  CSF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c.smem));
  ProfScope ps("k_sigma", stream);
  kern<<<grid, c.threads, c.smem, stream>>>(g);
  return check_launch("sigma");
}

}  // namespace csffci

using namespace csffci;

extern "C" {

int csffci_spin_parity(int64_t n, const double* c, double* out3, void* work, size_t work_bytes,
                       cudaStream_t stream) {
  CSF_REQUIRE(n >= 0 && out3 != nullptr, "spin_parity: bad arguments");
  const int np = 148 * 4;
  if (work == nullptr || work_bytes < (size_t)(3 * np) * sizeof(double)) {
    set_error("spin_parity: workspace of %zu bytes < %zu required", work_bytes,
              (size_t)(3 * np) * sizeof(double));
    return CSFFCI_ERR_MEMORY;
  }
  k_parity_part<<<np, 256, 0, stream>>>(c, n, (double*)work);
  int st = check_launch("spin_parity");
  if (st) return st;
  k_parity_final<<<1, 32, 0, stream>>>((double*)work, np, out3);
  return check_launch("spin_parity final");
}

size_t csffci_sigma_workspace(int norb, int neleca, int nelecb, int flags) {
  if (flags & CSFFCI_SIGMA_DETERMINISTIC)  // three int64 digit planes (they hold s in the symmetric mode)
    return (size_t)(host_binom(norb, neleca) * host_binom(norb, nelecb)) * 3 * sizeof(long long);
  if (flags & CSFFCI_SIGMA_SPIN_SYMMETRIC)
    return (size_t)(host_binom(norb, neleca) * host_binom(norb, nelecb)) * sizeof(double);
  return 0;
}

}  // extern "C"

namespace csffci {
// csffci_sigma with an explicit kernel choice: variant -1 is the default
// for one problem (sigma_rr_single_variant), -2 the shared-memory-h2e
// kernel (as CSFFCI_SIGMA_REFERENCE_KERNEL), anything else a variant of the
// register-resident family (sigma_rr.cu)
static int sigma_exec(int norb, int neleca, int nelecb, const double* h2e, const csffci_link_t* link_a,
                      const csffci_link_t* link_b, const double* ci, double* sigma, int flags, int eta,
                      void* work, size_t work_bytes, int variant, cudaStream_t stream) {
  CSF_REQUIRE(norb >= 1 && norb <= 22, "sigma: norb=%d outside [1,22]", norb);
  CSF_REQUIRE(neleca >= 0 && nelecb >= 0 && neleca <= norb && nelecb <= norb,
              "sigma: bad nelec (%d,%d)", neleca, nelecb);
  const bool sym = (flags & CSFFCI_SIGMA_SPIN_SYMMETRIC) != 0;
  const bool accumulate = (flags & CSFFCI_SIGMA_ACCUMULATE) != 0;
  CSF_REQUIRE(!sym || neleca == nelecb, "sigma: spin-symmetric mode needs neleca == nelecb");
  CSF_REQUIRE(!sym || eta == 1 || eta == -1, "sigma: eta must be +1 or -1");
  long long Na = (long long)host_binom(norb, neleca), Nb = (long long)host_binom(norb, nelecb);
  long long ndet = Na * Nb;
  int nla = neleca * (norb - neleca + 1), nlb = nelecb * (norb - nelecb + 1);
  if (flags & CSFFCI_SIGMA_DETERMINISTIC) {
    CSF_REQUIRE(!(flags & CSFFCI_SIGMA_REFERENCE_KERNEL),
                "sigma: the deterministic mode runs the warp-specialised kernel, not the reference kernel");
    CSF_REQUIRE(norb >= 4 && norb <= 16, "sigma: the deterministic mode covers 4 <= norb <= 16, not %d", norb);
    const size_t need = csffci_sigma_workspace(norb, neleca, nelecb, flags);
    if (work == nullptr || work_bytes < need) {
      set_error("sigma: workspace of %zu bytes < %zu required", work_bytes, need);
      return CSFFCI_ERR_MEMORY;
    }
    if (ndet == 0) return CSFFCI_OK;
    CSF_CUDA(cudaMemsetAsync(work, 0, need, stream));
    int st = sigma_rr_run(norb, neleca, nelecb, h2e, link_a, link_b, ci, (double*)work, sym, (double)eta,
                          stream, -1, ndet);
    if (st) return st;
    ProfScope ps("k_det_finish", stream);
    if (sym) {
      dim3 blk(32, 8);
      const long long tiles = ((Na + 31) / 32) * ((Na + 31) / 32);
      k_det_finish_sym<<<grid_for(tiles, 1, 148 * 16), blk, 0, stream>>>((const long long*)work, sigma, Na, eta,
                                                                        accumulate ? 1 : 0);
    } else {
      k_det_finish<<<grid_for(ndet, 256, 148 * 16), 256, 0, stream>>>((const long long*)work, sigma, ndet,
                                                                      accumulate ? 1 : 0);
    }
    return check_launch("sigma deterministic finish");
  }
  double* target = sigma;
  if (sym) {
    size_t need = csffci_sigma_workspace(norb, neleca, nelecb, flags);
    if (work == nullptr || work_bytes < need) {
      set_error("sigma: workspace of %zu bytes < %zu required", work_bytes, need);
      return CSFFCI_ERR_MEMORY;
    }
    target = (double*)work;
  }
  if (sym || !accumulate) CSF_CUDA(cudaMemsetAsync(target, 0, ndet * sizeof(double), stream));
  if (ndet == 0) return CSFFCI_OK;

  if (sigma_rr_supported(norb) && !(flags & CSFFCI_SIGMA_REFERENCE_KERNEL) && variant != -2) {
    int st = sigma_rr_run(norb, neleca, nelecb, h2e, link_a, link_b, ci, target, sym, (double)eta, stream,
                          variant);
    if (st) return st;
    if (sym) {
      dim3 blk(32, 8);
      ProfScope ps("k_sym_add", stream);
      long long tiles = ((Na + 31) / 32) * ((Na + 31) / 32);
      k_sym_add<<<grid_for(tiles, 1, 148 * 16), blk, 0, stream>>>(target, sigma, Na, (double)eta,
                                                                 accumulate ? 1 : 0);
      return check_launch("sigma symmetric add");
    }
    return CSFFCI_OK;
  }
  SigmaConfig c = sigma_config(norb, nla);
  CSF_REQUIRE(c.nt > 0, "sigma: no tile configuration fits shared memory for norb=%d", norb);
  SigmaArgs g;
  g.h2e = h2e;
  g.la = link_a;
  g.lb = link_b;
  g.ci = ci;
  g.out = target;
  g.Na = Na;
  g.Nb = Nb;
  g.norb = norb;
  g.npair = norb * (norb + 1) / 2;
  g.npad = c.npad;
  g.hstride = c.hstride;
  g.dstride = c.dstride;
  g.nla = nla;
  g.nlb = nlb;
  g.alpha_scatter = sym ? 0 : 1;
  int NB = 8 * c.nt;
  g.nchunk = (Nb + NB - 1) / NB;
  g.nitems = Na * g.nchunk;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  int per_sm = 1;
  if (c.smem * 2 <= 227 * 1024 && c.threads * 2 <= 2048) per_sm = 2;
  long long grid = (long long)nsm * per_sm;
  if (grid > g.nitems) grid = g.nitems;
  int st;
  if (c.hsmem) {
    switch (c.nt) {
      case 8: st = launch_sigma<8, true>(c, g, (int)grid, stream); break;
      case 4: st = launch_sigma<4, true>(c, g, (int)grid, stream); break;
      default: st = launch_sigma<2, true>(c, g, (int)grid, stream); break;
    }
  } else {
    switch (c.nt) {
      case 8: st = launch_sigma<8, false>(c, g, (int)grid, stream); break;
      case 4: st = launch_sigma<4, false>(c, g, (int)grid, stream); break;
      default: st = launch_sigma<2, false>(c, g, (int)grid, stream); break;
    }
  }
  if (st) return st;
  if (sym) {
    dim3 blk(32, 8);
    ProfScope ps("k_sym_add", stream);
    long long tiles = ((Na + 31) / 32) * ((Na + 31) / 32);
    k_sym_add<<<grid_for(tiles, 1, 148 * 16), blk, 0, stream>>>(target, sigma, Na, (double)eta,
                                                               accumulate ? 1 : 0);
    return check_launch("sigma symmetric add");
  }
  return CSFFCI_OK;
}
}  // namespace csffci

// ---- sigma plan: the per-problem state of csffci_sigma bound once ------
struct csffci_sigma_plan {
  int norb, neleca, nelecb, flags, variant;
  const double* h2e;
  const csffci_link_t* link_a;
  const csffci_link_t* link_b;
  size_t work_bytes;
  void* work;
};

extern "C" {

int csffci_sigma(int norb, int neleca, int nelecb, const double* h2e, const csffci_link_t* link_a,
                 const csffci_link_t* link_b, const double* ci, double* sigma, int flags, int eta,
                 void* work, size_t work_bytes, cudaStream_t stream) {
  return sigma_exec(norb, neleca, nelecb, h2e, link_a, link_b, ci, sigma, flags, eta, work, work_bytes, -1,
                    stream);
}

int csffci_sigma_plan_create(int norb, int neleca, int nelecb, const double* h2e, const csffci_link_t* link_a,
                             const csffci_link_t* link_b, int flags, csffci_sigma_plan_t** plan,
                             size_t* work_bytes) {
  CSF_REQUIRE(plan != nullptr, "sigma_plan_create: plan is NULL");
  *plan = nullptr;
  CSF_REQUIRE(norb >= 1 && norb <= 22, "sigma_plan_create: norb=%d outside [1,22]", norb);
  CSF_REQUIRE(neleca >= 0 && nelecb >= 0 && neleca <= norb && nelecb <= norb,
              "sigma_plan_create: bad nelec (%d,%d)", neleca, nelecb);
  CSF_REQUIRE(h2e != nullptr && link_a != nullptr && link_b != nullptr,
              "sigma_plan_create: h2e and the link tables are required");
  CSF_REQUIRE((flags & ~(CSFFCI_SIGMA_SPIN_SYMMETRIC | CSFFCI_SIGMA_REFERENCE_KERNEL |
                         CSFFCI_SIGMA_DETERMINISTIC)) == 0,
              "sigma_plan_create: flags may hold SPIN_SYMMETRIC, REFERENCE_KERNEL and DETERMINISTIC only");
  CSF_REQUIRE(!(flags & CSFFCI_SIGMA_DETERMINISTIC) ||
                  (norb >= 4 && norb <= 16 && !(flags & CSFFCI_SIGMA_REFERENCE_KERNEL)),
              "sigma_plan_create: the deterministic mode covers 4 <= norb <= 16 (warp-specialised kernel)");
  CSF_REQUIRE(!(flags & CSFFCI_SIGMA_SPIN_SYMMETRIC) || neleca == nelecb,
              "sigma_plan_create: the spin-symmetric mode needs neleca == nelecb");
  csffci_sigma_plan_t* p = new (std::nothrow) csffci_sigma_plan_t;
  if (!p) {
    set_error("sigma_plan_create: out of host memory");
    return CSFFCI_ERR_MEMORY;
  }
  p->norb = norb;
  p->neleca = neleca;
  p->nelecb = nelecb;
  p->flags = flags;
  p->h2e = h2e;
  p->link_a = link_a;
  p->link_b = link_b;
  p->variant = (flags & CSFFCI_SIGMA_REFERENCE_KERNEL) || !sigma_rr_supported(norb)
                   ? -2
                   : sigma_rr_single_variant(norb);
  if (p->variant < 0 && p->variant != -2) p->variant = rr_default_variant(norb);
  if (flags & CSFFCI_SIGMA_DETERMINISTIC) p->variant = 4;  // the warp-specialised kernel
  p->work_bytes = csffci_sigma_workspace(norb, neleca, nelecb, flags);
  p->work = nullptr;
  if (work_bytes) *work_bytes = p->work_bytes;
  *plan = p;
  return CSFFCI_OK;
}

int csffci_sigma_plan_bind(csffci_sigma_plan_t* plan, void* work, size_t work_bytes) {
  CSF_REQUIRE(plan != nullptr, "sigma_plan_bind: plan is NULL");
  if (plan->work_bytes && (work == nullptr || work_bytes < plan->work_bytes)) {
    set_error("sigma_plan_bind: workspace of %zu bytes < %zu required", work_bytes, plan->work_bytes);
    return CSFFCI_ERR_MEMORY;
  }
  plan->work = work;
  return CSFFCI_OK;
}

int csffci_sigma_plan_execute(const csffci_sigma_plan_t* plan, const double* ci, double* sigma, int eta,
                              int flags, cudaStream_t stream) {
  CSF_REQUIRE(plan != nullptr, "sigma_plan_execute: plan is NULL");
  CSF_REQUIRE((flags & ~(CSFFCI_SIGMA_ACCUMULATE | CSFFCI_SIGMA_SPIN_SYMMETRIC)) == 0,
              "sigma_plan_execute: flags may hold ACCUMULATE and SPIN_SYMMETRIC only");
  CSF_REQUIRE(!(flags & CSFFCI_SIGMA_SPIN_SYMMETRIC) || (plan->flags & CSFFCI_SIGMA_SPIN_SYMMETRIC),
              "sigma_plan_execute: the plan was created without the spin-symmetric mode");
  CSF_REQUIRE(!plan->work_bytes || plan->work != nullptr, "sigma_plan_execute: the plan has no workspace bound");
  return sigma_exec(plan->norb, plan->neleca, plan->nelecb, plan->h2e, plan->link_a, plan->link_b, ci, sigma,
                    flags | (plan->flags & (CSFFCI_SIGMA_REFERENCE_KERNEL | CSFFCI_SIGMA_DETERMINISTIC)), eta,
                    plan->work, plan->work_bytes,
                    plan->variant, stream);
}

int csffci_sigma_plan_variant(const csffci_sigma_plan_t* plan) {
  CSF_REQUIRE(plan != nullptr, "sigma_plan_variant: plan is NULL");
  return plan->variant;
}

void csffci_sigma_plan_destroy(csffci_sigma_plan_t* plan) { delete plan; }

}  // extern "C"
