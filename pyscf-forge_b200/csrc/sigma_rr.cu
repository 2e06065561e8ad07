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
// Shared-memory layouts are chosen bank-conflict free for the regular
// accesses: ds = 4 (mod 16) doubles, so that the B-fragment loads of a half
// warp (rows 4s+t, t = 0..3, columns g) fall in 16 distinct banks (measured
// 5 % faster at norb 12 than 8 (mod 16)), LS odd for the column-wise link
// reads.
#include <stdlib.h>
#include <string.h>

#include <map>
#include <mutex>
#include <vector>

#include "sigma_rr.cuh"
#include "sigma_rr_kernel.cuh"

namespace csffci {

bool sigma_rr_supported(int norb) { return norb >= 4 && norb <= 16; }

// the tile loops read link entries as 8-byte words and copy 8-byte elements
static bool rr_aligned8(const void* p) { return ((uintptr_t)p & 7u) == 0; }

// Tile shapes (rows per warp, n-tiles of 8 columns): 16-row warps halve
// the B-fragment traffic but need 2*KS + 4*NT doubles of registers per lane;
// with 9 warps (norb 15,16) an SMSP holds 3 warps, i.e. at most 168
// registers, so those sizes have no (16, 4) instance.  Where the
// warp-specialised kernel is not the default (rr_default_variant), the
// fastest shapes measured on B200 for one singlet/doublet problem are
// (16, 2) up to norb 10 and at 13, (8, 2) for 11-12, (8, 4) from 14 (the
// two-n-tile shapes run 2-3 CTAs per SM at small norb); CSFFCI_SIGMA_VARIANT
// overrides the choice and the batched solver's autotuner picks per orbital
// count.
static const int kVariantShape[RR_NVARIANT][2] = {{16, 4}, {8, 4}, {16, 2}, {8, 2}};

bool rr_variant_valid(int norb, int v) { return v >= 0 && v < RR_NVARIANT && !(v == 0 && norb >= 15); }

bool batch_variant_valid(int norb, int v) {
  return rr_variant_valid(norb, v) || (v == RR_VARIANT_WS && sigma_ws_supported(norb)) ||
         (v == RR_VARIANT_WS16 && sigma_ws16_supported(norb));
}

// one problem: the register-split kernel at 16 orbitals, else the job-table
// default (CSFFCI_SIGMA_VARIANT may name any variant)
int sigma_rr_single_variant(int norb) {
  const char* env = getenv("CSFFCI_SIGMA_VARIANT");
  if (env) {
    const int v = atoi(env);
    if (batch_variant_valid(norb, v)) return v;
    if ((v == RR_VARIANT_WSR || v == RR_VARIANT_WSR_BULK) && sigma_wsr_supported(norb)) return v;
    if (rr_variant_valid(norb, v)) return v;
  }
  // measured on B200 (one problem), best tile shape -> k_sigma_ws: 10
  // orbitals (5,5) singlet 0.044 -> 0.042 ms, 11 (6,5) 0.191 -> 0.167 ms,
  // 12 (6,6) singlet 0.444 -> 0.349 ms, 12 (7,6) 0.572 -> 0.507 ms, 14
  // singlet 7.61 -> 6.31 ms, 15: 31.1 -> 25.8 ms, 16: 148.8 -> 129.5 ms and
  // 116 ms (k_sigma_wsr, registers re-split between the roles); at 13 the
  // warp-specialised kernel is no faster, at 9 and below the tile shapes
  // are faster
  if (sigma_wsr_supported(norb)) return RR_VARIANT_WSR;
  return rr_default_variant(norb);
}

// job tables (and one problem below 16 orbitals): the warp-specialised
// kernel at 10..12 and 14..16 orbitals (the C3 batch of 128 problems: norb
// 12 jobs 24.6 -> 23.2 ms per launch, norb 11 4.40 -> 3.99 ms, norb 10
// 0.89 -> 0.85 ms against the best tile shape); the batched solver's
// autotuner times every variant on its own job tables
int rr_default_variant(int norb) {
  const char* env = getenv("CSFFCI_SIGMA_VARIANT");
  if (env) {
    const int v = atoi(env);
    if (batch_variant_valid(norb, v)) return v;
  }
  if (norb >= 10 && norb != 13 && sigma_ws_supported(norb)) return RR_VARIANT_WS;
  return norb <= 10 || norb == 13 ? 2 : norb <= 12 ? 3 : 1;
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
                    int max_nla, int max_nlb, cudaStream_t stream, int variant, long long det_stride) {
  const int npair = norb * (norb + 1) / 2;
  const int ks = (npair + 3) / 4;
  if (det_stride)  // the deterministic scatter exists in the warp-specialised kernel only
    return sigma_ws_launch(norb, njobs, jobs_dev, job0, total_units, max_nb, max_nla, max_nlb, stream, 8,
                           det_stride);
  if (variant < 0 && !jobs_dev) variant = sigma_rr_single_variant(norb);
  if (variant < 0) variant = rr_default_variant(norb);
  if (variant == RR_VARIANT_WS || variant == RR_VARIANT_WS16)
    return sigma_ws_launch(norb, njobs, jobs_dev, job0, total_units, max_nb, max_nla, max_nlb, stream,
                           variant == RR_VARIANT_WS16 ? 16 : 8);
  if (variant == RR_VARIANT_WSR || variant == RR_VARIANT_WSR_BULK) {
    if (jobs_dev) {
      set_error("sigma: the register-split variant takes one problem, not a job table");
      return CSFFCI_ERR_INVALID;
    }
    return sigma_wsr_launch(norb, job0, total_units, max_nb, max_nla, max_nlb, stream,
                            variant == RR_VARIANT_WSR_BULK);
  }
  if (!rr_variant_valid(norb, variant)) {
    set_error("sigma: tile variant %d is not available for norb=%d", variant, norb);
    return CSFFCI_ERR_INVALID;
  }
  const int mw = kVariantShape[variant][0];
  const int nt = kVariantShape[variant][1];
  const int nb = 8 * nt;
  RRArgs g;
  memset(&g, 0, sizeof(g));
  g.jobs = jobs_dev;
  g.job0 = job0;
  g.njobs = njobs;
  g.total_units = total_units;
  g.npair = npair;
  g.ds = nb + 4;  // = 4 (mod 16): a half warp's B-fragment loads hit distinct banks
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
  g.off_al = take((size_t)(max_nla > 0 ? max_nla : 1) * sizeof(RRAlpha));
  g.off_zl = take((size_t)npair * sizeof(int));
  g.off_pn = take((size_t)2 * npair * sizeof(unsigned));
  g.off_zf = take((size_t)npair * sizeof(int));
  const size_t smem = off;
  if (smem > 227 * 1024 - 256) {
    set_error("sigma: tile of %zu bytes exceeds shared memory", smem);
    return CSFFCI_ERR_INVALID;
  }
switch (variant) {
    case 0: return rr_dispatch_v0(norb, g, smem, stream);
    case 1: return rr_dispatch_v1(norb, g, smem, stream);
    case 2: return rr_dispatch_v2(norb, g, smem, stream);
    default: return rr_dispatch_v3(norb, g, smem, stream);
  }
}

int sigma_rr_run(int norb, int neleca, int nelecb, const double* h2e, const csffci_link_t* la,
                 const csffci_link_t* lb, const double* ci, double* out, bool sym, double eta,
                 cudaStream_t stream, int variant, long long det_stride) {
  CSF_REQUIRE(rr_aligned8(la) && rr_aligned8(lb) && rr_aligned8(ci) && rr_aligned8(out),
              "sigma: link tables and vectors must be 8-byte aligned");
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
  return sigma_rr_launch(norb, 1, nullptr, J, total, maxnb, mla, mlb, stream, variant, det_stride);
}

// ---- batch: zero the outputs, run the jobs, form sigma = S + eta S^T -----
__device__ __forceinline__ bool job_live(const csffci_sigma_job_t& J) {
  return J.live == nullptr || J.live_index < *J.live;
}

__global__ void k_batch_zero(const csffci_sigma_job_t* jobs, int njobs, long long total) {
  int j = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    while (j + 1 < njobs && jobs[j + 1].elem_begin <= i) ++j;
    const csffci_sigma_job_t& J = jobs[j];
    if (!job_live(J)) continue;
    const long long li = i - J.elem_begin;
    if (J.flags & CSFFCI_SIGMA_JOB_DETERMINISTIC) {  // the three digit planes
      long long* w = reinterpret_cast<long long*>(J.scratch);
      const long long nd = J.Na * J.Nb;
      w[li] = w[nd + li] = w[2 * nd + li] = 0;
    } else {
      (J.sym ? J.scratch : J.sigma)[li] = 0.0;
    }
  }
}

// the digit planes of a deterministic job -> sigma (k_det_finish's value;
// general jobs elementwise here, spin-symmetric ones by k_batch_det_sym)
__device__ __forceinline__ double batch_det_value(long long w0, long long w1, long long w2) {
  return ((double)w2 * 0x1p6 + (double)w1 * 0x1p-37) + (double)w0 * 0x1p-80;
}

__global__ void k_batch_det_finish(const csffci_sigma_job_t* jobs, int njobs, long long total) {
  int j = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    while (j + 1 < njobs && jobs[j + 1].elem_begin <= i) ++j;
    const csffci_sigma_job_t& J = jobs[j];
    if (J.sym || !job_live(J)) continue;
    const long long li = i - J.elem_begin, nd = J.Na * J.Nb;
    const long long* w = reinterpret_cast<const long long*>(J.scratch);
    J.sigma[li] = batch_det_value(w[li], w[nd + li], w[2 * nd + li]);
  }
}

// sigma = S + eta S^T of spin-symmetric deterministic jobs, the digit words
// of the two entries added as integers before the conversion
__global__ void k_batch_det_sym(const csffci_sigma_job_t* jobs, int njobs, long long total_tiles) {
  __shared__ long long tile[3][32][33];
  int j = 0;
  for (long long t = blockIdx.x; t < total_tiles; t += gridDim.x) {
    while (j + 1 < njobs && jobs[j + 1].tile_begin <= t) ++j;
    while (!jobs[j].sym) ++j;  // general jobs own no tiles
    const csffci_sigma_job_t& J = jobs[j];
    if (!job_live(J)) continue;  // uniform over the block (one tile per block)
    const long long n = J.Na, nd = n * n;
    const long long ntile = (n + 31) / 32;
    const long long lt = t - J.tile_begin;
    const long long ti = lt / ntile, tj = lt - ti * ntile;
    const long long* w = reinterpret_cast<const long long*>(J.scratch);
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      const long long row = tj * 32 + r, col = ti * 32 + threadIdx.x;
      const bool in = row < n && col < n;
#pragma unroll
      for (int k = 0; k < 3; ++k) tile[k][r][threadIdx.x] = in ? w[k * nd + row * n + col] : 0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      const long long row = ti * 32 + r, col = tj * 32 + threadIdx.x;
      if (row < n && col < n) {
        long long d[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const unsigned long long a = (unsigned long long)w[k * nd + row * n + col];
          const unsigned long long b = (unsigned long long)tile[k][threadIdx.x][r];
          d[k] = (long long)(J.eta > 0 ? a + b : a - b);
        }
        J.sigma[row * n + col] = batch_det_value(d[0], d[1], d[2]);
      }
    }
    __syncthreads();
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
    if (!job_live(J)) continue;  // uniform over the block (one tile per block)
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

int sigma_batch_prepare(int norb, int njobs, csffci_sigma_job_t* jobs, SigmaBatchInfo* info) {
  CSF_REQUIRE(norb >= 4 && norb <= 16, "sigma_batch: norb=%d outside [4,16]", norb);
  CSF_REQUIRE(njobs > 0 && jobs != nullptr, "sigma_batch: bad job list");
  for (int i = 0; i < njobs; ++i) {
    const csffci_sigma_job_t& J = jobs[i];
    CSF_REQUIRE(J.neleca >= 0 && J.nelecb >= 0 && J.neleca <= norb && J.nelecb <= norb,
                "sigma_batch: job %d has bad nelec (%d,%d)", i, J.neleca, J.nelecb);
    CSF_REQUIRE(!J.sym || (J.neleca == J.nelecb && J.scratch != nullptr && (J.eta == 1 || J.eta == -1)),
                "sigma_batch: job %d: spin-symmetric mode needs neleca == nelecb, eta = +-1 and scratch", i);
    CSF_REQUIRE(J.h2e && J.link_a && J.link_b && J.ci && J.sigma, "sigma_batch: job %d has a NULL pointer", i);
    CSF_REQUIRE(rr_aligned8(J.link_a) && rr_aligned8(J.link_b) && rr_aligned8(J.ci) && rr_aligned8(J.sigma) &&
                    rr_aligned8(J.scratch),
                "sigma_batch: job %d has a pointer that is not 8-byte aligned", i);
    CSF_REQUIRE((J.flags & ~CSFFCI_SIGMA_JOB_DETERMINISTIC) == 0 &&
                    (J.flags & CSFFCI_SIGMA_JOB_DETERMINISTIC) == (jobs[0].flags & CSFFCI_SIGMA_JOB_DETERMINISTIC),
                "sigma_batch: job %d: flags must be 0 or DETERMINISTIC, the same for every job", i);
    CSF_REQUIRE(!(J.flags & CSFFCI_SIGMA_JOB_DETERMINISTIC) || (J.scratch != nullptr && sigma_ws_supported(norb)),
                "sigma_batch: job %d: the deterministic scatter needs scratch (3*ndet int64) and 4 <= norb <= 16",
                i);
  }
  info->norb = norb;
  info->njobs = njobs;
  rr_prepare(norb, njobs, jobs, &info->total_units, &info->max_nb, &info->max_nla, &info->max_nlb);
  info->nelem = jobs[njobs - 1].elem_begin + jobs[njobs - 1].Na * jobs[njobs - 1].Nb;
  info->ntiles = 0;
  for (int i = 0; i < njobs; ++i)
    if (jobs[i].sym) info->ntiles = jobs[i].tile_begin + ((jobs[i].Na + 31) / 32) * ((jobs[i].Na + 31) / 32);
  info->job0 = jobs[0];
  info->det = (jobs[0].flags & CSFFCI_SIGMA_JOB_DETERMINISTIC) ? 1 : 0;
  if (info->det) info->variant = RR_VARIANT_WS;  // the only kernel with the deterministic scatter
  return CSFFCI_OK;
}

int sigma_batch_launch(const SigmaBatchInfo& info, const csffci_sigma_job_t* dj, cudaStream_t stream) {
  const int njobs = info.njobs;
  if (njobs == 0) return CSFFCI_OK;
  k_batch_zero<<<grid_for(info.nelem, 256, 148 * 16), 256, 0, stream>>>(dj, njobs, info.nelem);
  int st = check_launch("sigma_batch zero");
  if (st) return st;
  // a gated single job goes through the job-table kernel (the by-value
  // form cannot see the gate)
  const bool table = njobs > 1 || info.job0.live != nullptr;
  if (info.det) {
    // the job table's form of the deterministic kernel (each job's planes
    // are its own Na*Nb apart), then sigma from the planes
    st = sigma_rr_launch(info.norb, njobs, dj, info.job0, info.total_units, info.max_nb, info.max_nla,
                         info.max_nlb, stream, RR_VARIANT_WS, 1);
    if (st) return st;
    {
      ProfScope ps("k_batch_det_finish", stream);
      k_batch_det_finish<<<grid_for(info.nelem, 256, 148 * 16), 256, 0, stream>>>(dj, njobs, info.nelem);
    }
    st = check_launch("sigma_batch deterministic finish");
    if (st || info.ntiles == 0) return st;
    dim3 blk(32, 8);
    ProfScope ps("k_batch_det_sym", stream);
    k_batch_det_sym<<<grid_for(info.ntiles, 1, 148 * 16), blk, 0, stream>>>(dj, njobs, info.ntiles);
    return check_launch("sigma_batch deterministic symmetric finish");
  }
  st = table ? sigma_rr_launch(info.norb, njobs, dj, info.job0, info.total_units, info.max_nb,
                               info.max_nla, info.max_nlb, stream, info.variant)
             : sigma_rr_launch(info.norb, 1, nullptr, info.job0, info.total_units, info.max_nb,
                               info.max_nla, info.max_nlb, stream, info.variant);
  if (st) return st;
  if (info.ntiles > 0) {
    dim3 blk(32, 8);
    ProfScope ps("k_batch_sym_add", stream);
    k_batch_sym_add<<<grid_for(info.ntiles, 1, 148 * 16), blk, 0, stream>>>(dj, njobs, info.ntiles);
    return check_launch("sigma_batch symmetric add");
  }
  return CSFFCI_OK;
}

// ---- autotuner: the fastest tile variant per (norb, job-shape signature),
//      timed on the caller's job table and cached for the process ---------
static std::mutex g_tune_mu;
static std::map<std::pair<int, unsigned long long>, int> g_tune_cache;

static unsigned long long job_signature(const csffci_sigma_job_t* jobs, int njobs) {
  unsigned long long h = 1469598103934665603ull;  // FNV-1a
  auto mix = [&](unsigned long long v) {
    h ^= v;
    h *= 1099511628211ull;
  };
  mix((unsigned long long)njobs);
  for (int i = 0; i < njobs; ++i)
    mix(((unsigned long long)jobs[i].neleca << 16) | ((unsigned long long)jobs[i].nelecb << 8) |
        (unsigned long long)jobs[i].sym);
  return h;
}

int sigma_batch_tune(SigmaBatchInfo& info, const csffci_sigma_job_t* jobs_host, const csffci_sigma_job_t* dj,
                     cudaStream_t stream) {
  if (info.det) return CSFFCI_OK;  // one kernel has the deterministic scatter: nothing to choose
  const auto key = std::make_pair(info.norb, job_signature(jobs_host, info.njobs));
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      info.variant = it->second;
      return CSFFCI_OK;
    }
  }
  cudaEvent_t a, b;
  CSF_CUDA(cudaEventCreate(&a));
  CSF_CUDA(cudaEventCreate(&b));
  int best = rr_default_variant(info.norb);
  float best_ms = 1e30f;
  for (int v = 0; v <= RR_VARIANT_WS16; ++v) {
    if (!batch_variant_valid(info.norb, v)) continue;
    SigmaBatchInfo t = info;
    t.variant = v;
    if (sigma_batch_launch(t, dj, stream) != CSFFCI_OK) continue;  // e.g. shared memory too small
    cudaEventRecord(a, stream);
    int st = sigma_batch_launch(t, dj, stream);
    if (st == CSFFCI_OK) st = sigma_batch_launch(t, dj, stream);
    cudaEventRecord(b, stream);
    if (cudaEventSynchronize(b) != cudaSuccess || st != CSFFCI_OK) continue;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    if (ms < best_ms) {
      best_ms = ms;
      best = v;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  info.variant = best;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache[key] = best;
  return CSFFCI_OK;
}

}  // namespace csffci

using namespace csffci;

extern "C" {

size_t csffci_sigma_batch_workspace(int njobs) {
  return (size_t)(njobs > 0 ? njobs : 1) * sizeof(csffci_sigma_job_t);
}

int csffci_sigma_batch(int norb, int njobs, csffci_sigma_job_t* jobs, void* work, size_t work_bytes,
                       cudaStream_t stream) {
  CSF_REQUIRE(njobs >= 0 && (njobs == 0 || jobs != nullptr), "sigma_batch: bad job list");
  if (njobs == 0) return CSFFCI_OK;
  if (work == nullptr || work_bytes < csffci_sigma_batch_workspace(njobs)) {
    set_error("sigma_batch: workspace of %zu bytes < %zu required", work_bytes,
              csffci_sigma_batch_workspace(njobs));
    return CSFFCI_ERR_MEMORY;
  }
  SigmaBatchInfo info;
  int st = sigma_batch_prepare(norb, njobs, jobs, &info);
  if (st) return st;
  csffci_sigma_job_t* dj = (csffci_sigma_job_t*)work;
  CSF_CUDA(cudaMemcpyAsync(dj, jobs, njobs * sizeof(csffci_sigma_job_t), cudaMemcpyHostToDevice, stream));
  return sigma_batch_launch(info, dj, stream);
}

}  // extern "C"
