// Davidson update kernels: subspace expansion/contraction (combine) and the
// diagonal / Olsen preconditioner.  The Gram blocks come from csffci_gram
// (rdm.cu).  All reductions are done in a fixed order (per-block partials,
// then one ordered pass) so results are bit-reproducible run to run.
#include "common.cuh"
#include "profile.cuh"

namespace csffci {

// y[r][k] = beta*y[r][k] + sum_i coef[r][i] x[i][k]: rows of y in groups of
// CB_RG held in registers, x read once per group (coalesced over k, the
// loop over i unrolled so that several loads are in flight); each output is
// beta*y first, then the terms in ascending i (a fixed order)
constexpr int CB_RG = 4;
__global__ void k_combine(int ny, double* y, int64_t ldy, double beta, int nx,
                          const double* __restrict__ x, int64_t ldx, const double* __restrict__ coef,
                          int64_t n) {
  extern __shared__ double cs[];  // coef rows padded with zeros to a multiple of CB_RG
  const int nyp = (ny + CB_RG - 1) / CB_RG * CB_RG;
  for (int i = threadIdx.x; i < nx * nyp; i += blockDim.x) cs[i] = i < nx * ny ? coef[i] : 0.0;
  __syncthreads();
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    for (int r0 = 0; r0 < ny; r0 += CB_RG) {
      double acc[CB_RG];
#pragma unroll
      for (int rr = 0; rr < CB_RG; ++rr)
        acc[rr] = (r0 + rr < ny && beta != 0.0) ? beta * y[(int64_t)(r0 + rr) * ldy + k] : 0.0;
      const double* c0 = cs + (int64_t)r0 * nx;
#pragma unroll 8
      for (int i = 0; i < nx; ++i) {
        const double xv = x[(int64_t)i * ldx + k];
#pragma unroll
        for (int rr = 0; rr < CB_RG; ++rr) acc[rr] = fma(c0[rr * nx + i], xv, acc[rr]);
      }
#pragma unroll
      for (int rr = 0; rr < CB_RG; ++rr)
        if (r0 + rr < ny) y[(int64_t)(r0 + rr) * ldy + k] = acc[rr];
    }
  }
}

// 1/(hdiag - (e - shift)) with the magnitude capped at 1e8 (cap value +1e8,
// as the p-space preconditioner the reference uses through fci.make_precond)
__device__ __forceinline__ double precond_inv(double h, double e, double shift) {
  double v = 1.0 / (h - (e - shift));
  if (fabs(v) > 1e8) v = 1e8;
  return v;
}

// per-block partial sums of x.(r*hinv) and x.(x*hinv)
__global__ void k_precond_dots(int64_t n, const double* __restrict__ r, const double* __restrict__ x,
                               const double* __restrict__ hd, double e, double shift, double* part) {
  __shared__ double s0[256], s1[256];
  double a = 0.0, b = 0.0;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    double hi = precond_inv(hd[k], e, shift);
    a = fma(x[k] * hi, r[k], a);
    b = fma(x[k] * hi, x[k], b);
  }
  s0[threadIdx.x] = a;
  s1[threadIdx.x] = b;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      s0[threadIdx.x] += s0[threadIdx.x + w];
      s1[threadIdx.x] += s1[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s0[0];
    part[2 * blockIdx.x + 1] = s1[0];
  }
}

__global__ void k_precond_sum(const double* part, int npart, double* out2) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int i = 0; i < npart; ++i) {
      a += part[2 * i];
      b += part[2 * i + 1];
    }
    out2[0] = a;
    out2[1] = b;
  }
}

__global__ void k_precond_apply(int64_t n, const double* __restrict__ r, const double* __restrict__ x,
                                const double* __restrict__ hd, double e, double shift, int mode,
                                double e1_given, const double* part, int npart, double* t) {
  __shared__ double e1s;
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    if (mode == 1) {
      for (int i = 0; i < npart; ++i) {
        a += part[2 * i];
        b += part[2 * i + 1];
      }
    }
    e1s = mode == 2 ? e1_given : ((mode == 1 && b != 0.0) ? a / b : 0.0);
  }
  __syncthreads();
  const double e1 = e1s;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x)
    t[k] = (r[k] - e1 * x[k]) * precond_inv(hd[k], e, shift);
}

}  // namespace csffci

using namespace csffci;

extern "C" {

int csffci_combine(int ny, double* y, int64_t ldy, double beta, int nx, const double* x,
                   int64_t ldx, const double* coef, int64_t n, cudaStream_t stream) {
  CSF_REQUIRE(ny >= 0 && nx >= 0 && n >= 0 && nx * ((ny + CB_RG - 1) / CB_RG * CB_RG) <= 4096,
              "combine: bad sizes");
  if (ny == 0 || n == 0) return CSFFCI_OK;
  size_t sm = (size_t)nx * ((ny + CB_RG - 1) / CB_RG * CB_RG) * sizeof(double);
  {
    ProfScope ps_("k_combine", stream);
    k_combine<<<grid_for(n, 256, 148 * 8), 256, sm, stream>>>(ny, y, ldy, beta, nx, x, ldx, coef, n);
  }
  return check_launch("combine");
}

size_t csffci_precond_workspace(void) { return (2 * 148 * 4 + 2) * sizeof(double); }

int csffci_precond_dots(int64_t n, const double* r, const double* x, const double* hdiag, double e,
                        double shift, double* out2, double* work, cudaStream_t stream) {
  CSF_REQUIRE(n >= 0 && work != nullptr && out2 != nullptr, "precond_dots: bad arguments");
  int nblk = grid_for(n > 0 ? n : 1, 256, 148 * 4);
  {
    ProfScope ps_("k_precond_dots", stream);
    k_precond_dots<<<nblk, 256, 0, stream>>>(n, r, x, hdiag, e, shift, work);
  }
  int st = check_launch("precond dots");
  if (st) return st;
  k_precond_sum<<<1, 32, 0, stream>>>(work, nblk, out2);
  return check_launch("precond dots sum");
}

int csffci_precond(int64_t n, const double* r, const double* x, const double* hdiag, double e,
                   double shift, int mode, double e1, double* t, double* work,
                   cudaStream_t stream) {
  CSF_REQUIRE(n >= 0 && work != nullptr && mode >= 0 && mode <= 2, "precond: bad arguments");
  if (n == 0) return CSFFCI_OK;
  int nblk = grid_for(n, 256, 148 * 4);
  if (mode == 1) {
    {
      ProfScope ps_("k_precond_dots", stream);
      k_precond_dots<<<nblk, 256, 0, stream>>>(n, r, x, hdiag, e, shift, work);
    }
    int st = check_launch("precond dots");
    if (st) return st;
  }
  {
    ProfScope ps_("k_precond_apply", stream);
    k_precond_apply<<<grid_for(n, 256, 148 * 8), 256, 0, stream>>>(n, r, x, hdiag, e, shift, mode, e1,
                                                                  work, nblk, t);
  }
  return check_launch("precond");
}

}  // extern "C"
