// Batched kernels for many independent CI problems solved in lockstep: one
// launch per operation covers every problem of the batch (descriptor
// tables in device memory), so the launch count of a Davidson iteration does
// not grow with the number of problems.
//
//   csffci_transform_batch  det <-> CSF block GEMMs of many (problem, block)
//   csffci_dots_batch       dot products x.y or x.(P y), P = 1/(hdiag-(e-shift))
//   csffci_combine_batch    y = beta y + scale * coef . X   (subspace algebra)
//   csffci_precond_batch    t = (r - e1 x) P with e1 = ab[0]/ab[1] read on device
// Every reduction runs in a fixed order (one block per dot product).
#include "common.cuh"
#include "profile.cuh"
#include "batch_internal.cuh"

namespace csffci {

// ---------------------------------------------------------------------------
// transforms
// ---------------------------------------------------------------------------
constexpr int BT_M = 32, BT_N = 32, BT_K = 16;

__device__ __forceinline__ int find_job(const int64_t* begin, int njobs, int64_t u, int hint) {
  int j = hint;
  while (j + 1 < njobs && begin[j + 1] <= u) ++j;
  return j;
}

// Blocks with few CSFs (ncsf <= BR_MAX_NCSF) and few determinants per
// configuration are most of the determinants below 13 orbitals (norb 12,
// (6,6): 92 % of them in blocks of 6..70 determinants and 2..14 CSFs), and
// a 32 x 32 output tile would leave most of its columns empty there.  Such
// a job is cut into units of 256 (vector, configuration) rows instead, one
// row per thread: the row's determinants are gathered through its mask
// row and contracted with umat (read as warp-uniform loads: every thread
// of a unit is in the same job) into NC register sums.  The sums run over
// k in increasing order with fma, as the tile path's do, so both paths give
// the same bits.
constexpr int BR_ROWS = 256, BR_MAX_NCSF = 16, BR_MAX_NDET = 256;

__host__ __device__ inline bool row_job(const csffci_transform_job_t& J) {
  return J.ncsf <= BR_MAX_NCSF && J.ndet <= BR_MAX_NDET;
}

template <int NC>
__device__ __forceinline__ void transform_row(const csffci_transform_job_t& J, int64_t vec, int64_t conf,
                                              int reverse) {
  const int nd = J.ndet, nc = J.ncsf;
  const uint32_t* mk = J.mask + J.csd_offset + conf * nd;
  if (!reverse) {
    double acc[NC];
#pragma unroll
    for (int k = 0; k < NC; ++k) acc[k] = 0.0;
    const double* xv = J.x + vec * J.ldx;
    for (int d = 0; d < nd; ++d) {
      const double v = xv[mk[d]];
      const double* u = J.umat + (int64_t)d * nc;
#pragma unroll
      for (int k = 0; k < NC; ++k)
        if (k < nc) acc[k] = fma(v, u[k], acc[k]);
    }
    double* yo = J.y + vec * J.ldy + J.csf_offset + conf * nc;
#pragma unroll
    for (int k = 0; k < NC; ++k)
      if (k < nc) yo[k] = J.sign * acc[k];
  } else {
    double cin[NC];
    const double* xi = J.x + vec * J.ldx + J.csf_offset + conf * nc;
#pragma unroll
    for (int k = 0; k < NC; ++k) cin[k] = k < nc ? xi[k] : 0.0;
    double* yv = J.y + vec * J.ldy;
    for (int d = 0; d < nd; ++d) {
      const double* u = J.umat + (int64_t)d * nc;
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < NC; ++k)
        if (k < nc) acc = fma(cin[k], u[k], acc);
      yv[mk[d]] = J.sign * acc;
    }
  }
}

// One tile = 32 (vec, conf) rows x 32 output columns of one job, or, for a
// row job, 256 rows.
__global__ void __launch_bounds__(256) k_transform_batch(const csffci_transform_job_t* jobs, int njobs,
                                                         int64_t total_tiles, int reverse) {
  __shared__ double As[BT_K][BT_M + 1];
  __shared__ double Bs[BT_K][BT_N + 1];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  int j = 0;
  for (int64_t tile = blockIdx.x; tile < total_tiles; tile += gridDim.x) {
    while (j + 1 < njobs && jobs[j + 1].tile_begin <= tile) ++j;
    const csffci_transform_job_t& J = jobs[j];
    const int nv = J.live ? min(J.nvec, *J.live) : J.nvec;
    const int64_t M = (int64_t)nv * J.nconf;
    const int64_t lt = tile - J.tile_begin;
    if (row_job(J)) {
      const int64_t m = lt * BR_ROWS + tid;
      if (m < M) {
        const csffci_transform_job_t Jr = J;  // in registers: the stores below cannot alias it
        const int64_t vec = m / Jr.nconf, conf = m - vec * Jr.nconf;
        if (Jr.ncsf <= 2) transform_row<2>(Jr, vec, conf, reverse);
        else if (Jr.ncsf <= 4) transform_row<4>(Jr, vec, conf, reverse);
        else if (Jr.ncsf <= 8) transform_row<8>(Jr, vec, conf, reverse);
        else transform_row<BR_MAX_NCSF>(Jr, vec, conf, reverse);
      }
      continue;
    }
    const int N = reverse ? J.ndet : J.ncsf;
    const int K = reverse ? J.ncsf : J.ndet;
    const int ntn = (N + BT_N - 1) / BT_N;
    const int64_t m0 = (lt / ntn) * BT_M;
    const int n0 = (int)(lt % ntn) * BT_N;
    if (m0 >= M) continue;  // rows of vectors that are not live (uniform per block)
    double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
    for (int k0 = 0; k0 < K; k0 += BT_K) {
      for (int e = tid; e < BT_M * BT_K; e += 256) {
        const int row = e / BT_K, kk = e - row * BT_K;
        const int64_t m = m0 + row;
        double v = 0.0;
        if (m < M && k0 + kk < K) {
          const int64_t vec = m / J.nconf, conf = m - vec * J.nconf;
          if (!reverse) {
            const uint32_t d = J.mask[J.csd_offset + conf * J.ndet + k0 + kk];
            v = J.x[vec * J.ldx + d];
          } else {
            v = J.x[vec * J.ldx + J.csf_offset + conf * J.ncsf + k0 + kk];
          }
        }
        As[kk][row] = v;
      }
      for (int e = tid; e < BT_N * BT_K; e += 256) {
        double v = 0.0;
        if (!reverse) {
          const int kk = e / BT_N, col = e - kk * BT_N;
          if (k0 + kk < K && n0 + col < N) v = J.umat[(int64_t)(k0 + kk) * J.ncsf + n0 + col];
          Bs[kk][col] = v;
        } else {
          const int col = e / BT_K, kk = e - col * BT_K;
          if (k0 + kk < K && n0 + col < N) v = J.umat[(int64_t)(n0 + col) * J.ncsf + k0 + kk];
          Bs[kk][col] = v;
        }
      }
      __syncthreads();
#pragma unroll
      for (int kk = 0; kk < BT_K; ++kk) {
        const double a0 = As[kk][ty * 2], a1 = As[kk][ty * 2 + 1];
        const double b0 = Bs[kk][tx * 2], b1 = Bs[kk][tx * 2 + 1];
        acc[0][0] = fma(a0, b0, acc[0][0]);
        acc[0][1] = fma(a0, b1, acc[0][1]);
        acc[1][0] = fma(a1, b0, acc[1][0]);
        acc[1][1] = fma(a1, b1, acc[1][1]);
      }
      __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      const int64_t m = m0 + ty * 2 + a;
      if (m >= M) continue;
      const int64_t vec = m / J.nconf, conf = m - vec * J.nconf;
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const int n = n0 + tx * 2 + b;
        if (n >= N) continue;
        const double v = J.sign * acc[a][b];
        if (!reverse) {
          J.y[vec * J.ldy + J.csf_offset + conf * J.ncsf + n] = v;
        } else {
          J.y[vec * J.ldy + J.mask[J.csd_offset + conf * J.ndet + n]] = v;
        }
      }
    }
  }
}

// zero the determinant vectors of reverse jobs (blocks without CSFs must
// read as zero); one entry per (vector, det) of each zero job
__global__ void k_zero_batch(const csffci_zero_job_t* jobs, int njobs, int64_t total) {
  int j = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    while (j + 1 < njobs && jobs[j + 1].elem_begin <= i) ++j;
    const csffci_zero_job_t& J = jobs[j];
    const int64_t li = i - J.elem_begin;
    const int64_t v = li / J.n;
    J.y[v * J.ld + (li - v * J.n)] = 0.0;
  }
}

// ---------------------------------------------------------------------------
// dots: one block per dot product, fixed-order tree reduction
// ---------------------------------------------------------------------------
__device__ __forceinline__ double pinv(double h, double es) {
  double v = 1.0 / (h - es);
  if (fabs(v) > 1e8) v = 1e8;
  return v;
}

__global__ void __launch_bounds__(256) k_dots_batch(const csffci_dot_t* dots, int ndots, double* out) {
  __shared__ double red[256];
  for (int d = blockIdx.x; d < ndots; d += gridDim.x) {
    const csffci_dot_t D = dots[d];
    double acc = 0.0;
    if (D.hdiag) {
      for (int64_t k = threadIdx.x; k < D.n; k += blockDim.x)
        acc = fma(D.x[k] * pinv(D.hdiag[k], D.e_shift), D.y[k], acc);
    } else {
      for (int64_t k = threadIdx.x; k < D.n; k += blockDim.x) acc = fma(D.x[k], D.y[k], acc);
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
      if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[D.out_index] = red[0];
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// combine: y[r][k] = beta*y[r][k] + scale * sum_i coef[r*ldc + i] * x[i][k]
// ---------------------------------------------------------------------------
__global__ void k_combine_batch(const csffci_combine_t* ops, int nops, int64_t total_units) {
  int j = 0;
  for (int64_t u = blockIdx.x; u < total_units; u += gridDim.x) {
    while (j + 1 < nops && ops[j + 1].unit_begin <= u) ++j;
    const csffci_combine_t& O = ops[j];
    const int64_t k = (u - O.unit_begin) * blockDim.x + threadIdx.x;
    if (k >= O.n) continue;
    for (int r = 0; r < O.ny; ++r) {
      double acc = 0.0;
      for (int i = 0; i < O.nx; ++i) acc = fma(O.coef[r * O.ldc + i], O.x[i * O.ldx + k], acc);
      double* yp = O.y + r * O.ldy + k;
      *yp = (O.beta == 0.0 ? 0.0 : O.beta * *yp) + O.scale * acc;
    }
  }
}

// ---------------------------------------------------------------------------
// precond: t = (r - e1 x) P, e1 = ab[0] / ab[1] (0 when ab is NULL)
// ---------------------------------------------------------------------------
__global__ void k_precond_batch(const csffci_precond_t* ops, int nops, int64_t total_units) {
  int j = 0;
  for (int64_t u = blockIdx.x; u < total_units; u += gridDim.x) {
    while (j + 1 < nops && ops[j + 1].unit_begin <= u) ++j;
    const csffci_precond_t& O = ops[j];
    const int64_t k = (u - O.unit_begin) * blockDim.x + threadIdx.x;
    if (k >= O.n) continue;
    double e1 = 0.0;
    if (O.ab) {
      const double b = O.ab[1];
      e1 = b != 0.0 ? O.ab[0] / b : 0.0;
    }
    O.t[k] = (O.r[k] - e1 * O.x[k]) * pinv(O.hdiag[k], O.e_shift);
  }
}

int transform_batch_prepare(int reverse, int njobs, csffci_transform_job_t* jobs, int64_t* total_tiles) {
  int64_t tiles = 0;
  for (int i = 0; i < njobs; ++i) {
    csffci_transform_job_t& J = jobs[i];
    CSF_REQUIRE(J.x && J.y && J.mask && J.umat && J.ncsf > 0 && J.ndet > 0, "transform_batch: job %d incomplete", i);
    J.tile_begin = tiles;
    const int64_t M = (int64_t)J.nvec * J.nconf;
    const int N = reverse ? J.ndet : J.ncsf;
    tiles += row_job(J) ? (M + BR_ROWS - 1) / BR_ROWS : ((M + BT_M - 1) / BT_M) * ((N + BT_N - 1) / BT_N);
  }
  *total_tiles = tiles;
  return CSFFCI_OK;
}

int transform_batch_launch(int reverse, const csffci_transform_job_t* jobs_dev, int njobs, int64_t tiles,
                           cudaStream_t stream) {
  if (tiles == 0 || njobs == 0) return CSFFCI_OK;
  ProfScope ps("k_transform_batch", stream);
  k_transform_batch<<<grid_for(tiles, 1, 148 * 8), 256, 0, stream>>>(jobs_dev, njobs, tiles, reverse);
  return check_launch("transform_batch");
}

}  // namespace csffci

using namespace csffci;

extern "C" {

int csffci_transform_batch(int reverse, int njobs, csffci_transform_job_t* jobs, int nzero,
                           csffci_zero_job_t* zjobs, void* work, size_t work_bytes,
                           cudaStream_t stream) {
  CSF_REQUIRE(njobs >= 0 && nzero >= 0, "transform_batch: bad counts");
  const size_t need = (size_t)njobs * sizeof(csffci_transform_job_t) + (size_t)nzero * sizeof(csffci_zero_job_t);
  if (need == 0) return CSFFCI_OK;
  if (work == nullptr || work_bytes < need) {
    set_error("transform_batch: workspace of %zu bytes < %zu required", work_bytes, need);
    return CSFFCI_ERR_MEMORY;
  }
  int64_t tiles = 0;
  int st = transform_batch_prepare(reverse, njobs, jobs, &tiles);
  if (st) return st;
  int64_t zelem = 0;
  for (int i = 0; i < nzero; ++i) {
    zjobs[i].elem_begin = zelem;
    zelem += zjobs[i].nvec * zjobs[i].n;
  }
  char* w = (char*)work;
  csffci_transform_job_t* dj = (csffci_transform_job_t*)w;
  csffci_zero_job_t* dz = (csffci_zero_job_t*)(w + (size_t)njobs * sizeof(csffci_transform_job_t));
  if (njobs) CSF_CUDA(cudaMemcpyAsync(dj, jobs, njobs * sizeof(*jobs), cudaMemcpyHostToDevice, stream));
  if (nzero) {
    CSF_CUDA(cudaMemcpyAsync(dz, zjobs, nzero * sizeof(*zjobs), cudaMemcpyHostToDevice, stream));
    k_zero_batch<<<grid_for(zelem, 256, 148 * 16), 256, 0, stream>>>(dz, nzero, zelem);
    st = check_launch("transform_batch zero");
    if (st) return st;
  }
  return transform_batch_launch(reverse, dj, njobs, tiles, stream);
}

int csffci_dots_batch(int ndots, const csffci_dot_t* dots, double* out, void* work, size_t work_bytes,
                      cudaStream_t stream) {
  CSF_REQUIRE(ndots >= 0, "dots_batch: bad count");
  if (ndots == 0) return CSFFCI_OK;
  const size_t need = (size_t)ndots * sizeof(csffci_dot_t);
  if (work == nullptr || work_bytes < need) {
    set_error("dots_batch: workspace of %zu bytes < %zu required", work_bytes, need);
    return CSFFCI_ERR_MEMORY;
  }
  CSF_CUDA(cudaMemcpyAsync(work, dots, need, cudaMemcpyHostToDevice, stream));
  k_dots_batch<<<grid_for(ndots, 1, 148 * 16), 256, 0, stream>>>((const csffci_dot_t*)work, ndots, out);
  return check_launch("dots_batch");
}

int csffci_combine_batch(int nops, csffci_combine_t* ops, void* work, size_t work_bytes,
                         cudaStream_t stream) {
  CSF_REQUIRE(nops >= 0, "combine_batch: bad count");
  if (nops == 0) return CSFFCI_OK;
  const size_t need = (size_t)nops * sizeof(csffci_combine_t);
  if (work == nullptr || work_bytes < need) {
    set_error("combine_batch: workspace of %zu bytes < %zu required", work_bytes, need);
    return CSFFCI_ERR_MEMORY;
  }
  int64_t units = 0;
  for (int i = 0; i < nops; ++i) {
    ops[i].unit_begin = units;
    units += (ops[i].n + 255) / 256;
  }
  CSF_CUDA(cudaMemcpyAsync(work, ops, need, cudaMemcpyHostToDevice, stream));
  if (units == 0) return CSFFCI_OK;
  k_combine_batch<<<grid_for(units, 1, 148 * 32), 256, 0, stream>>>((const csffci_combine_t*)work, nops, units);
  return check_launch("combine_batch");
}

int csffci_precond_batch(int nops, csffci_precond_t* ops, void* work, size_t work_bytes,
                         cudaStream_t stream) {
  CSF_REQUIRE(nops >= 0, "precond_batch: bad count");
  if (nops == 0) return CSFFCI_OK;
  const size_t need = (size_t)nops * sizeof(csffci_precond_t);
  if (work == nullptr || work_bytes < need) {
    set_error("precond_batch: workspace of %zu bytes < %zu required", work_bytes, need);
    return CSFFCI_ERR_MEMORY;
  }
  int64_t units = 0;
  for (int i = 0; i < nops; ++i) {
    ops[i].unit_begin = units;
    units += (ops[i].n + 255) / 256;
  }
  CSF_CUDA(cudaMemcpyAsync(work, ops, need, cudaMemcpyHostToDevice, stream));
  if (units == 0) return CSFFCI_OK;
  k_precond_batch<<<grid_for(units, 1, 148 * 32), 256, 0, stream>>>((const csffci_precond_t*)work, nops, units);
  return check_launch("precond_batch");
}

}  // extern "C"
