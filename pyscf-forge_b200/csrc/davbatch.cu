// Device-resident lockstep Davidson-Liu for a batch of independent CSF-FCI
// problems (csffci_batch_plan_*).
//
// Every step of an iteration runs on the device for all problems at once,
// driven by a per-problem state record (subspace size, number of new
// vectors, convergence flags, Ritz values) that the kernels read and write,
// so an iteration is a fixed launch sequence with no host synchronisation
// and is captured once as a CUDA graph and replayed:
//
//   k_db_proj<0>   partial dots T.V and |T|^2 over 1024-element chunks
//   k_db_sproj<0>  reduce -> projection coefficients
//   k_db_proj<1>   T -= coef.V, partial dots T.V        (second projection)
//   k_db_sproj<1>
//   k_db_proj<2>   T -= coef.V, partial Gram T.T
//   k_db_sproj<2>  orthonormal combinations (Jacobi on the small Gram)
//   k_db_new       W = c.T, V[m..] = W
//   CSF -> det (batched block GEMMs), sigma per orbital count (gated
//   persistent job table), det -> CSF into AW
//   k_db_hv        AV[m..] = AW, partial dots V.AW
//   k_db_sritz     subspace matrix update, Jacobi eigensolver, root
//                  selection (overlap following once a root converged)
//   k_db_ritz      X = cc.V, AX = cc.AV, R = AX - e X, partial |R|^2 and
//                  the Olsen dots x.P r, x.P x
//   k_db_sconv     convergence, correction bookkeeping, restart decision
//   k_db_pre       T = (R - e1 X) P  (Olsen correction over the diagonal),
//                  restart copies V[:k] = X, AV[:k] = AX
//
// The per-problem algorithm is that of the one-problem solver (role of
// pyscf lib.davidson1 via fci.eig at pyscf/csf_fci/csf.py:487-490, with the
// diagonal Olsen preconditioner of fci.make_precond, csf.py:433).  Every
// reduction runs in a fixed order (chunk partials summed in unit order), so
// a batch is bit-reproducible up to the atomic scatter of sigma.  No
// counterpart in the reference, which solves one problem per call.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "batch_internal.cuh"
#include "common.cuh"
#include "profile.cuh"
#include "sigma_rr_kernel.cuh"

namespace csffci {

constexpr int DB_KMAX = 8;     // roots per problem
constexpr int DB_CAPMAX = 64;  // subspace capacity max_space + 2*nroots
constexpr int DB_NT = 256;     // threads of the streaming kernels
constexpr int DB_EPT = 4;      // elements per thread
constexpr int DB_CH = DB_NT * DB_EPT;
constexpr int DB_NW = DB_NT / 32;
constexpr int DB_ST = 128;  // threads of the small per-problem kernels

struct DBProb {
  int64_t n;
  int32_t k, cap, space, unit0, nunits, pad;
  double *V, *AV, *X, *AX, *R, *T, *W, *AW;
  const double* hdiag;
  double *h, *coef, *cc, *xprev;
  double *qprev, *dprev;  // eigenvectors (cap x cap) and eigenvalues of the last subspace matrix
};

struct DBState {
  int32_t m, m_old, kT, knew, kk, done, restart, niter, any_conv, have_e, kk_prev;
  int32_t mq;  // size of the basis qprev/dprev diagonalise (0: none)
  int32_t todo[DB_KMAX];
  int32_t conv[DB_KMAX];
  double e[DB_KMAX], e_prev[DB_KMAX], rnorm[DB_KMAX], e1[DB_KMAX], es[DB_KMAX], tnorm[DB_KMAX];
};

struct DBArgs {
  const DBProb* prob;
  DBState* st;
  const int32_t* unit_prob;
  double* partial;
  int nslot, capb, kb, nprob;
  long long nunits;
  double tol, toloose, lindep, shift;
  int* count;
};

__device__ __forceinline__ double db_pinv(double h, double es) {
  double v = 1.0 / (h - es);
  if (fabs(v) > 1e8) v = 1e8;
  return v;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// slot of dot (row i, column j) and of the per-row extras
__device__ __forceinline__ int slot_dot(const DBArgs& a, int i, int j) { return i * a.capb + j; }
__device__ __forceinline__ int slot_x(const DBArgs& a, int which, int i) {
  return a.kb * a.capb + which * a.kb + i;
}

// the warp partials of slots [0, nslot) of this block -> partial[u]
__device__ __forceinline__ void db_flush(const DBArgs& a, long long u, const double* red) {
  __syncthreads();
  for (int s = threadIdx.x; s < a.nslot; s += DB_NT) {
    double v = 0.0;
#pragma unroll
    for (int w = 0; w < DB_NW; ++w) v += red[w * a.nslot + s];
    a.partial[u * a.nslot + s] = v;
  }
}

// ---------------------------------------------------------------------------
// streaming kernels: one unit = one 1024-element chunk of one problem; KM
// is the largest root count of the batch (register arrays)
// ---------------------------------------------------------------------------
template <int KM, int PASS>
__global__ void __launch_bounds__(DB_NT) k_db_proj(DBArgs a) {
  extern __shared__ double red[];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (long long u = blockIdx.x; u < a.nunits; u += gridDim.x) {
    const int p = a.unit_prob[u];
    const DBState& S = a.st[p];
    const int kT = S.kT;
    if (S.done || kT == 0) continue;
    const DBProb& P = a.prob[p];
    const int m = S.m;
    const int64_t n = P.n;
    const int64_t e0 = (int64_t)(u - P.unit0) * DB_CH + tid;
    double t[KM][DB_EPT];
#pragma unroll
    for (int i = 0; i < KM; ++i)
#pragma unroll
      for (int q = 0; q < DB_EPT; ++q) {
        const int64_t e = e0 + q * DB_NT;
        t[i][q] = (i < kT && e < n) ? P.T[i * n + e] : 0.0;
      }
    if (PASS >= 1 && m > 0) {
      for (int j = 0; j < m; ++j) {
        double v[DB_EPT];
#pragma unroll
        for (int q = 0; q < DB_EPT; ++q) {
          const int64_t e = e0 + q * DB_NT;
          v[q] = e < n ? P.V[j * n + e] : 0.0;
        }
#pragma unroll
        for (int i = 0; i < KM; ++i) {
          if (i < kT) {
            const double c = P.coef[i * P.cap + j];
#pragma unroll
            for (int q = 0; q < DB_EPT; ++q) t[i][q] = fma(-c, v[q], t[i][q]);
          }
        }
      }
#pragma unroll
      for (int i = 0; i < KM; ++i)
        if (i < kT)
#pragma unroll
          for (int q = 0; q < DB_EPT; ++q) {
            const int64_t e = e0 + q * DB_NT;
            if (e < n) P.T[i * n + e] = t[i][q];
          }
    }
    __syncthreads();  // red of the previous unit is flushed
    if (PASS <= 1) {
      for (int j = 0; j < m; ++j) {
        double v[DB_EPT];
#pragma unroll
        for (int q = 0; q < DB_EPT; ++q) {
          const int64_t e = e0 + q * DB_NT;
          v[q] = e < n ? P.V[j * n + e] : 0.0;
        }
#pragma unroll
        for (int i = 0; i < KM; ++i) {
          if (i < kT) {
            double s = 0.0;
#pragma unroll
            for (int q = 0; q < DB_EPT; ++q) s = fma(t[i][q], v[q], s);
            s = warp_sum(s);
            if (lane == 0) red[w * a.nslot + slot_dot(a, i, j)] = s;
          }
        }
      }
      if (PASS == 0) {
#pragma unroll
        for (int i = 0; i < KM; ++i) {
          if (i < kT) {
            double s = 0.0;
#pragma unroll
            for (int q = 0; q < DB_EPT; ++q) s = fma(t[i][q], t[i][q], s);
            s = warp_sum(s);
            if (lane == 0) red[w * a.nslot + slot_x(a, 0, i)] = s;
          }
        }
      }
    } else {
#pragma unroll
      for (int i = 0; i < KM; ++i)
#pragma unroll
        for (int i2 = 0; i2 <= i; ++i2) {
          if (i < kT) {
            double s = 0.0;
#pragma unroll
            for (int q = 0; q < DB_EPT; ++q) s = fma(t[i][q], t[i2][q], s);
            s = warp_sum(s);
            if (lane == 0) red[w * a.nslot + slot_dot(a, i, i2)] = s;
          }
        }
    }
    db_flush(a, u, red);
  }
}

// W = corth . T (knew rows), V[m_old + r] = W[r]
template <int KM>
__global__ void __launch_bounds__(DB_NT) k_db_new(DBArgs a) {
  const int tid = threadIdx.x;
  for (long long u = blockIdx.x; u < a.nunits; u += gridDim.x) {
    const int p = a.unit_prob[u];
    const DBState& S = a.st[p];
    if (S.done || S.knew == 0) continue;
    const DBProb& P = a.prob[p];
    const int kT = S.kT, knew = S.knew, m0 = S.m_old;
    const int64_t n = P.n;
    const int64_t e0 = (int64_t)(u - P.unit0) * DB_CH + tid;
#pragma unroll
    for (int q = 0; q < DB_EPT; ++q) {
      const int64_t e = e0 + q * DB_NT;
      if (e >= n) continue;
      double t[KM];
#pragma unroll
      for (int i = 0; i < KM; ++i) t[i] = i < kT ? P.T[i * n + e] : 0.0;
      for (int r = 0; r < knew; ++r) {
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < KM; ++i)
          if (i < kT) s = fma(P.coef[r * P.cap + i], t[i], s);
        P.W[r * n + e] = s;
        P.V[(m0 + r) * n + e] = s;
      }
    }
  }
}

// AV[m_old + r] = AW[r]; partial dots V[j] . AW[r], j < m_old + knew
template <int KM>
__global__ void __launch_bounds__(DB_NT) k_db_hv(DBArgs a) {
  extern __shared__ double red[];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (long long u = blockIdx.x; u < a.nunits; u += gridDim.x) {
    const int p = a.unit_prob[u];
    const DBState& S = a.st[p];
    if (S.done || S.knew == 0) continue;
    const DBProb& P = a.prob[p];
    const int knew = S.knew, m0 = S.m_old, m = m0 + knew;
    const int64_t n = P.n;
    const int64_t e0 = (int64_t)(u - P.unit0) * DB_CH + tid;
    double y[KM][DB_EPT];
#pragma unroll
    for (int r = 0; r < KM; ++r)
#pragma unroll
      for (int q = 0; q < DB_EPT; ++q) {
        const int64_t e = e0 + q * DB_NT;
        double v = 0.0;
        if (r < knew && e < n) {
          v = P.AW[r * n + e];
          P.AV[(m0 + r) * n + e] = v;
        }
        y[r][q] = v;
      }
    __syncthreads();
    for (int j = 0; j < m; ++j) {
      double v[DB_EPT];
#pragma unroll
      for (int q = 0; q < DB_EPT; ++q) {
        const int64_t e = e0 + q * DB_NT;
        v[q] = e < n ? P.V[j * n + e] : 0.0;
      }
#pragma unroll
      for (int r = 0; r < KM; ++r) {
        if (r < knew) {
          double s = 0.0;
#pragma unroll
          for (int q = 0; q < DB_EPT; ++q) s = fma(y[r][q], v[q], s);
          s = warp_sum(s);
          if (lane == 0) red[w * a.nslot + slot_dot(a, r, j)] = s;
        }
      }
    }
    db_flush(a, u, red);
  }
}

// X = cc.V, AX = cc.AV, R = AX - e X; partial |R|^2, x.P r, x.P x
template <int KM>
__global__ void __launch_bounds__(DB_NT) k_db_ritz(DBArgs a) {
  extern __shared__ double red[];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (long long u = blockIdx.x; u < a.nunits; u += gridDim.x) {
    const int p = a.unit_prob[u];
    const DBState& S = a.st[p];
    if (S.done || S.knew == 0) continue;
    const DBProb& P = a.prob[p];
    const int kk = S.kk, m = S.m;
    const int64_t n = P.n;
    const int64_t e0 = (int64_t)(u - P.unit0) * DB_CH + tid;
    double x[KM][DB_EPT], ax[KM][DB_EPT];
#pragma unroll
    for (int i = 0; i < KM; ++i)
#pragma unroll
      for (int q = 0; q < DB_EPT; ++q) x[i][q] = ax[i][q] = 0.0;
    for (int j = 0; j < m; ++j) {
      double v[DB_EPT], av[DB_EPT];
#pragma unroll
      for (int q = 0; q < DB_EPT; ++q) {
        const int64_t e = e0 + q * DB_NT;
        v[q] = e < n ? P.V[j * n + e] : 0.0;
        av[q] = e < n ? P.AV[j * n + e] : 0.0;
      }
#pragma unroll
      for (int i = 0; i < KM; ++i) {
        if (i < kk) {
          const double c = P.cc[i * P.cap + j];
#pragma unroll
          for (int q = 0; q < DB_EPT; ++q) {
            x[i][q] = fma(c, v[q], x[i][q]);
            ax[i][q] = fma(c, av[q], ax[i][q]);
          }
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < KM; ++i) {
      if (i < kk) {
        const double ei = S.e[i];
        const double es = ei - a.shift;
        double rr = 0.0, xpr = 0.0, xpx = 0.0;
#pragma unroll
        for (int q = 0; q < DB_EPT; ++q) {
          const int64_t e = e0 + q * DB_NT;
          if (e < n) {
            const double r = fma(-ei, x[i][q], ax[i][q]);
            P.X[i * n + e] = x[i][q];
            P.AX[i * n + e] = ax[i][q];
            P.R[i * n + e] = r;
            const double pw = db_pinv(P.hdiag[e], es);
            rr = fma(r, r, rr);
            xpr = fma(x[i][q] * pw, r, xpr);
            xpx = fma(x[i][q] * pw, x[i][q], xpx);
          }
        }
        rr = warp_sum(rr);
        xpr = warp_sum(xpr);
        xpx = warp_sum(xpx);
        if (lane == 0) {
          red[w * a.nslot + slot_x(a, 0, i)] = rr;
          red[w * a.nslot + slot_x(a, 1, i)] = xpr;
          red[w * a.nslot + slot_x(a, 2, i)] = xpx;
        }
      }
    }
    db_flush(a, u, red);
  }
}

// T[row] = (R[i] - e1 X[i]) P for the unconverged roots; restart copies
__global__ void __launch_bounds__(DB_NT) k_db_pre(DBArgs a) {
  const int tid = threadIdx.x;
  for (long long u = blockIdx.x; u < a.nunits; u += gridDim.x) {
    const int p = a.unit_prob[u];
    const DBState& S = a.st[p];
    if (S.done) continue;
    const DBProb& P = a.prob[p];
    const int kT = S.kT, kk = S.kk;
    const int64_t n = P.n;
    const int64_t e0 = (int64_t)(u - P.unit0) * DB_CH + tid;
#pragma unroll
    for (int q = 0; q < DB_EPT; ++q) {
      const int64_t e = e0 + q * DB_NT;
      if (e >= n) continue;
      const double hd = P.hdiag[e];
      for (int row = 0; row < kT; ++row) {
        const int i = S.todo[row];
        P.T[row * n + e] = (P.R[i * n + e] - S.e1[row] * P.X[i * n + e]) * db_pinv(hd, S.es[row]);
      }
      if (S.restart) {
        for (int i = 0; i < kk; ++i) {
          P.V[i * n + e] = P.X[i * n + e];
          P.AV[i * n + e] = P.AX[i * n + e];
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// small per-problem kernels (one block of DB_ST threads per problem)
// ---------------------------------------------------------------------------
__device__ double db_reduce_slot(const DBArgs& a, const DBProb& P, int s) {
  double v = 0.0;
  const double* src = a.partial + (long long)P.unit0 * a.nslot + s;
  for (int u = 0; u < P.nunits; ++u) v += src[(long long)u * a.nslot];
  return v;
}

// Cyclic Jacobi eigensolver for the symmetric n x n matrix A (shared
// memory, leading dimension ld), round-robin parallel ordering: each step
// rotates n/2 disjoint pairs (Golub & Van Loan, Matrix Computations,
// sections 8.5.2 and 8.5.5).  On return diag(A) holds the eigenvalues and
// the columns of Q the eigenvectors; w/perm give them in ascending order.
__device__ void db_jacobi(double* A, double* Q, int n, int ld, double* rot, double* w, int* perm,
                          double* redbuf, bool qinit = false) {
  const int tid = threadIdx.x, nt = blockDim.x;
  if (!qinit)  // else Q holds a starting basis the rotations are applied to
    for (int i = tid; i < n * ld; i += nt) Q[i] = ((i / ld) == (i % ld)) ? 1.0 : 0.0;
  const int nn = n + (n & 1);
  const int np = nn / 2;
  __syncthreads();
  for (int sweep = 0; sweep < 60 && n > 1; ++sweep) {
    // convergence: off-diagonal Frobenius norm vs the diagonal
    double off = 0.0, dia = 0.0;
    for (int i = tid; i < n * n; i += nt) {
      const int r = i / n, c = i % n;
      const double v = A[r * ld + c];
      if (r == c)
        dia += v * v;
      else
        off += v * v;
    }
    redbuf[tid] = off;
    redbuf[nt + tid] = dia;
    __syncthreads();
    if (tid == 0) {
      double so = 0.0, sd = 0.0;
      for (int i = 0; i < nt; ++i) {
        so += redbuf[i];
        sd += redbuf[nt + i];
      }
      redbuf[2 * nt] = so;
      redbuf[2 * nt + 1] = sd;
    }
    __syncthreads();
    const double so = redbuf[2 * nt], sd = redbuf[2 * nt + 1];
    __syncthreads();
    if (so == 0.0 || so <= 1e-32 * sd) break;
    for (int step = 0; step < nn - 1; ++step) {
      for (int t = tid; t < np; t += nt) {
        int pp = t == 0 ? 0 : ((t - 1 + step) % (nn - 1)) + 1;
        int qq = ((nn - 2 - t + step) % (nn - 1)) + 1;
        if (pp > qq) {
          const int x = pp;
          pp = qq;
          qq = x;
        }
        double c = 1.0, s = 0.0;
        if (qq < n) {
          const double apq = A[pp * ld + qq];
          const double app = A[pp * ld + pp], aqq = A[qq * ld + qq];
          if (fabs(apq) <= 1e-18 * sqrt(fabs(app * aqq)) || fabs(apq) < 1e-300) {
            // negligible against the diagonal: set to zero (only this
            // pair's thread touches these two entries in this step)
            A[pp * ld + qq] = 0.0;
            A[qq * ld + pp] = 0.0;
          } else {
            const double tau = (aqq - app) / (2.0 * apq);
            const double tt = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = 1.0 / sqrt(1.0 + tt * tt);
            s = tt * c;
          }
        }
        rot[4 * t + 0] = pp;
        rot[4 * t + 1] = qq;
        rot[4 * t + 2] = c;
        rot[4 * t + 3] = s;
      }
      __syncthreads();
      // rows p, q of A <- J^T A
      for (int i = tid; i < np * n; i += nt) {
        const int t = i / n, col = i % n;
        const int pp = (int)rot[4 * t], qq = (int)rot[4 * t + 1];
        const double c = rot[4 * t + 2], s = rot[4 * t + 3];
        if (qq >= n || s == 0.0) continue;
        const double ap = A[pp * ld + col], aq = A[qq * ld + col];
        A[pp * ld + col] = c * ap - s * aq;
        A[qq * ld + col] = s * ap + c * aq;
      }
      __syncthreads();
      // columns p, q of A <- A J, and of Q <- Q J
      for (int i = tid; i < np * n; i += nt) {
        const int t = i / n, row = i % n;
        const int pp = (int)rot[4 * t], qq = (int)rot[4 * t + 1];
        const double c = rot[4 * t + 2], s = rot[4 * t + 3];
        if (qq >= n || s == 0.0) continue;
        const double ap = A[row * ld + pp], aq = A[row * ld + qq];
        A[row * ld + pp] = c * ap - s * aq;
        A[row * ld + qq] = s * ap + c * aq;
        const double qp = Q[row * ld + pp], qv = Q[row * ld + qq];
        Q[row * ld + pp] = c * qp - s * qv;
        Q[row * ld + qq] = s * qp + c * qv;
      }
      __syncthreads();
    }
  }
  // ascending order (ties by index)
  for (int i = tid; i < n; i += nt) {
    const double di = A[i * ld + i];
    int r = 0;
    for (int j = 0; j < n; ++j) {
      const double dj = A[j * ld + j];
      r += (dj < di) || (dj == di && j < i);
    }
    perm[r] = i;
    w[r] = di;
  }
  __syncthreads();
}

// orthonormal combinations of the projected corrections; the Gram matrix
// is scaled by the norms before projection so that the linear-dependence
// cut is relative
__device__ void db_orth(const DBArgs& a, const DBProb& P, DBState& S, int kT) {
  const int tid = threadIdx.x;
  __shared__ double G[DB_KMAX * DB_KMAX], Q[DB_KMAX * DB_KMAX], rot[4 * DB_KMAX], w[DB_KMAX];
  __shared__ double sc[DB_KMAX], redbuf[2 * DB_ST + 2];
  __shared__ int perm[DB_KMAX];
  for (int i = tid; i < kT; i += DB_ST) sc[i] = 1.0 / sqrt(fmax(S.tnorm[i], 1e-300));
  __syncthreads();
  for (int idx = tid; idx < kT * kT; idx += DB_ST) {
    const int i = idx / kT, i2 = idx % kT;
    if (i2 <= i) {
      const double v = db_reduce_slot(a, P, slot_dot(a, i, i2)) * sc[i] * sc[i2];
      G[i * DB_KMAX + i2] = v;
      G[i2 * DB_KMAX + i] = v;
    }
  }
  __syncthreads();
  db_jacobi(G, Q, kT, DB_KMAX, rot, w, perm, redbuf);
  if (tid == 0) {
    double wmax = 0.0;
    for (int i = 0; i < kT; ++i) wmax = fmax(wmax, w[i]);
    const double cut = fmax(a.lindep, 1e-14 * wmax);
    int first = 0;
    while (first < kT && !(w[first] > cut)) ++first;
    int nkeep = kT - first;
    if (S.m + nkeep > P.cap) {
      nkeep = P.cap - S.m;
      if (nkeep < 0) nkeep = 0;
      first = kT - nkeep;
    }
    for (int r = 0; r < nkeep; ++r) {
      const int col = perm[first + r];
      const double f = 1.0 / sqrt(w[first + r]);
      for (int i = 0; i < kT; ++i) P.coef[r * P.cap + i] = Q[i * DB_KMAX + col] * f * sc[i];
    }
    S.knew = nkeep;
    S.m_old = S.m;
    if (nkeep == 0) S.done = 1;
  }
}

template <int PASS>
__global__ void __launch_bounds__(DB_ST) k_db_sproj(DBArgs a) {
  const int p = blockIdx.x, tid = threadIdx.x;
  DBState& S = a.st[p];
  if (S.done || S.kT == 0) return;
  const DBProb& P = a.prob[p];
  const int kT = S.kT, m = S.m;
  if constexpr (PASS <= 1) {
    for (int idx = tid; idx < kT * m; idx += DB_ST) {
      const int i = idx / m, j = idx % m;
      P.coef[i * P.cap + j] = db_reduce_slot(a, P, slot_dot(a, i, j));
    }
    if (PASS == 0)
      for (int i = tid; i < kT; i += DB_ST) S.tnorm[i] = db_reduce_slot(a, P, slot_x(a, 0, i));
  } else {
    db_orth(a, P, S, kT);
  }
}

__global__ void __launch_bounds__(DB_ST) k_db_sritz(DBArgs a) {
  extern __shared__ double sm[];
  const int p = blockIdx.x, tid = threadIdx.x;
  DBState& S = a.st[p];
  if (S.done || S.knew == 0) return;
  const DBProb& P = a.prob[p];
  const int cap = P.cap, ld = a.capb;
  const int knew = S.knew, m0 = S.m_old, m = m0 + knew;
  double* A = sm;
  double* Q = A + ld * ld;
  double* rot = Q + ld * ld;
  double* w = rot + 2 * ld + 4;
  double* ov = w + ld;
  double* redbuf = ov + DB_KMAX * ld;
  int* perm = (int*)(redbuf + 2 * DB_ST + 2);
  __shared__ int idx_s[DB_KMAX];
  // new columns of the subspace matrix; the square of new rows and columns
  // takes the symmetric part of its two computed halves
  for (int idx = tid; idx < knew * m; idx += DB_ST) {
    const int r = idx / m, j = idx % m;
    const double v = db_reduce_slot(a, P, slot_dot(a, r, j));
    if (j < m0) {
      P.h[j * cap + m0 + r] = v;
      P.h[(m0 + r) * cap + j] = v;
    } else {
      const int r2 = j - m0;
      P.h[(m0 + r) * cap + j] = 0.5 * (v + db_reduce_slot(a, P, slot_dot(a, r2, m0 + r)));
    }
  }
  __syncthreads();
  // Warm start: the first m0 basis vectors were diagonalised at the last
  // iteration (eigenvectors qprev, eigenvalues dprev; after a restart the
  // identity and the Ritz values).  In the basis diag(qprev, I) the matrix
  // is diag(dprev) bordered by the new rows and columns, which the Jacobi
  // sweeps then clear in a few sweeps instead of diagonalising from scratch
  // (the off-diagonal entries dropped there are below the Jacobi tolerance
  // of the last solve).  Both border halves sum in the same order, so A
  // stays exactly symmetric.
  const bool warm = S.mq == m0 && m0 > 0;
  for (int idx = tid; idx < m * m; idx += DB_ST) {
    const int i = idx / m, j = idx % m;
    double v;
    if (!warm || (i >= m0 && j >= m0)) {
      v = P.h[i * cap + j];
    } else if (i < m0 && j < m0) {
      v = i == j ? P.dprev[i] : 0.0;
    } else {
      const int r = i < m0 ? i : j, c = i < m0 ? j : i;  // qprev column r, new column c
      v = 0.0;
      for (int l = 0; l < m0; ++l) v = fma(P.qprev[l * cap + r], P.h[l * cap + c], v);
    }
    A[i * ld + j] = v;
    if (warm) Q[i * ld + j] = (i < m0 && j < m0) ? P.qprev[i * cap + j] : (i == j ? 1.0 : 0.0);
  }
  __syncthreads();
  db_jacobi(A, Q, m, ld, rot, w, perm, redbuf, warm);
  // the eigenpairs of this basis, for the next iteration's warm start
  for (int idx = tid; idx < m * m; idx += DB_ST) {
    const int i = idx / m, j = idx % m;
    P.qprev[i * cap + j] = Q[i * ld + j];
  }
  for (int i = tid; i < m; i += DB_ST) P.dprev[i] = A[i * ld + i];
  const int kk = m < P.k ? m : P.k;
  const bool follow = S.have_e && S.any_conv;
  if (follow) {
    for (int idx = tid; idx < S.kk_prev * m; idx += DB_ST) {
      const int i = idx / m, j = idx % m;
      double s = 0.0;
      for (int l = 0; l < m; ++l) s = fma(P.xprev[i * cap + l], Q[l * ld + perm[j]], s);
      ov[i * ld + j] = fabs(s);
    }
  }
  __syncthreads();
  if (tid == 0) {
    int sel[DB_KMAX];
    int nsel = 0;
    if (follow) {
      // for each previous root the unused Ritz vector of largest overlap,
      // then the chosen ones by energy
      for (int i = 0; i < S.kk_prev; ++i) {
        int best = -1;
        double bv = -1.0;
        for (int j = 0; j < m; ++j) {
          bool used = false;
          for (int t = 0; t < nsel; ++t) used |= sel[t] == j;
          if (!used && ov[i * ld + j] > bv) {
            bv = ov[i * ld + j];
            best = j;
          }
        }
        if (best >= 0) sel[nsel++] = best;
      }
      for (int i = 1; i < nsel; ++i)
        for (int j = i; j > 0 && sel[j] < sel[j - 1]; --j) {
          const int x = sel[j];
          sel[j] = sel[j - 1];
          sel[j - 1] = x;
        }
      if (nsel > kk) nsel = kk;
    }
    if (nsel < kk) {
      nsel = kk;
      for (int i = 0; i < kk; ++i) sel[i] = i;
    }
    for (int i = 0; i < DB_KMAX; ++i) S.e_prev[i] = S.e[i];
    S.kk_prev = S.have_e ? S.kk : 0;
    for (int i = 0; i < kk; ++i) {
      idx_s[i] = sel[i];
      S.e[i] = w[sel[i]];
    }
    S.kk = kk;
    S.m = m;
  }
  __syncthreads();
  for (int idx = tid; idx < kk * cap; idx += DB_ST) {
    const int i = idx / cap, j = idx % cap;
    P.cc[i * cap + j] = j < m ? Q[j * ld + perm[idx_s[i]]] : 0.0;
  }
}

__global__ void __launch_bounds__(DB_ST) k_db_sconv(DBArgs a) {
  const int p = blockIdx.x, tid = threadIdx.x;
  DBState& S = a.st[p];
  if (S.done || S.knew == 0) return;
  const DBProb& P = a.prob[p];
  const int kk = S.kk, cap = P.cap;
  __shared__ double rr[DB_KMAX], xpr[DB_KMAX], xpx[DB_KMAX];
  __shared__ int restart_s, done_s;
  for (int idx = tid; idx < 3 * kk; idx += DB_ST) {
    const int which = idx / kk, i = idx % kk;
    const double v = db_reduce_slot(a, P, slot_x(a, which, i));
    (which == 0 ? rr : which == 1 ? xpr : xpx)[i] = v;
  }
  __syncthreads();
  if (tid == 0) {
    const bool have_prev = S.have_e && S.kk_prev == kk;
    bool all = true, any = false;
    for (int i = 0; i < kk; ++i) {
      S.rnorm[i] = sqrt(fmax(rr[i], 0.0));
      const double de = have_prev ? S.e[i] - S.e_prev[i] : INFINITY;
      const bool c = fabs(de) < a.tol && S.rnorm[i] < a.toloose;
      S.conv[i] = c;
      all &= c;
      any |= c;
    }
    S.any_conv = any;
    S.have_e = 1;
    S.niter += 1;
    int kT = 0;
    if (all && kk == P.k) {
      S.done = 1;
    } else {
      for (int i = 0; i < kk; ++i) {
        if (S.conv[i]) continue;
        S.todo[kT] = i;
        S.e1[kT] = xpx[i] != 0.0 ? xpr[i] / xpx[i] : 0.0;
        S.es[kT] = S.e[i] - a.shift;
        ++kT;
      }
    }
    if (kT == 0) S.done = 1;  // nothing left to correct
    S.kT = kT;
    S.knew = 0;  // set again by the next orthonormalisation
    S.restart = !S.done && (S.m + kT > P.space);
    if (S.restart) S.m = kk;
    S.mq = S.restart ? kk : S.m;  // the basis the stored eigenpairs belong to
    restart_s = S.restart;
    done_s = S.done;
  }
  __syncthreads();
  if (done_s) return;
  // the previous Ritz coefficients for root following (identity after a
  // restart, whose basis is the Ritz vectors themselves) and, on restart,
  // the subspace matrix diag(e)
  const int restart = restart_s;
  for (int idx = tid; idx < kk * cap; idx += DB_ST) {
    const int i = idx / cap, j = idx % cap;
    P.xprev[idx] = restart ? (i == j ? 1.0 : 0.0) : P.cc[idx];
  }
  if (restart) {
    // the basis is the Ritz vectors: h = diag(e), eigenvectors the identity
    for (int idx = tid; idx < cap * cap; idx += DB_ST) {
      const int i = idx / cap, j = idx % cap;
      P.h[idx] = (i == j && i < kk) ? S.e[i] : 0.0;
      P.qprev[idx] = (i == j && i < kk) ? 1.0 : 0.0;
    }
    for (int i = tid; i < kk; i += DB_ST) P.dprev[i] = S.e[i];
  }
}

__global__ void k_db_init(DBArgs a, const double* const* x0) {
  const int p = blockIdx.x;
  DBState& S = a.st[p];
  const DBProb& P = a.prob[p];
  for (int64_t i = threadIdx.x; i < (int64_t)P.k * P.n; i += blockDim.x) P.T[i] = x0[p][i];
  if (threadIdx.x == 0) {
    memset(&S, 0, sizeof(S));
    S.kT = P.k;
  }
}

__global__ void k_db_count(DBArgs a) {
  __shared__ int c;
  if (threadIdx.x == 0) c = 0;
  __syncthreads();
  int mine = 0;
  for (int p = threadIdx.x; p < a.nprob; p += blockDim.x) mine += a.st[p].done ? 0 : 1;
  atomicAdd(&c, mine);
  __syncthreads();
  if (threadIdx.x == 0) *a.count = c;
}

}  // namespace csffci

using namespace csffci;

struct csffci_batch_plan {
  int nprob = 0, kb = 0, capb = 0, nslot = 0;
  long long nunits = 0;
  csffci_batch_options_t opt{};
  std::vector<csffci_batch_problem_t> in;
  std::vector<std::vector<csffci_block_t>> blocks;
  std::vector<DBProb> prob;
  std::vector<int64_t> ndet;
  std::vector<int64_t> off_cdet;  // byte offsets of the det buffers
  std::vector<int32_t> unit_prob;
  // sigma groups by orbital count
  std::vector<int> group_norb;
  std::vector<std::vector<csffci_sigma_job_t>> group_jobs;
  std::vector<SigmaBatchInfo> group_info;
  std::vector<csffci_sigma_job_t*> group_dev;
  std::vector<csffci_transform_job_t> jrev, jfwd, jdet;
  int64_t trev = 0, tfwd = 0, tdet = 0;
  csffci_transform_job_t *drev = nullptr, *dfwd = nullptr, *ddet = nullptr;
  csffci_sigma_job_t* dtune = nullptr;
  size_t arena_bytes = 0;
  char* arena = nullptr;
  DBArgs args{};
  double** dx0 = nullptr;
  int* hcount = nullptr;
  size_t smem_stream = 0, smem_ritz = 0;
  bool bound = false;
  cudaStream_t cap_stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int iterations = 0;
};

namespace {

size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

template <int KM>
int enqueue_iteration_km(csffci_batch_plan_t* P, cudaStream_t s) {
  const DBArgs& a = P->args;
  const int gs = grid_for(a.nunits, 1, 148 * 8);
  const int np = P->nprob;
  int st;
#define DB_CHECK(what)                 \
  if ((st = check_launch(what)) != 0) \
    return st;
  // one profiler scope per launch (timed only while profiling is enabled)
#define DB_LAUNCH(name, what, ...)  \
  {                                 \
    ProfScope ps_(name, s);         \
    __VA_ARGS__;                    \
  }                                 \
  DB_CHECK(what)
  DB_LAUNCH("k_db_proj", "batch solver: projection 0", (k_db_proj<KM, 0><<<gs, DB_NT, P->smem_stream, s>>>(a)));
  DB_LAUNCH("k_db_sproj", "batch solver: projection 0 reduce", (k_db_sproj<0><<<np, DB_ST, 0, s>>>(a)));
  DB_LAUNCH("k_db_proj", "batch solver: projection 1", (k_db_proj<KM, 1><<<gs, DB_NT, P->smem_stream, s>>>(a)));
  DB_LAUNCH("k_db_sproj", "batch solver: projection 1 reduce", (k_db_sproj<1><<<np, DB_ST, 0, s>>>(a)));
  DB_LAUNCH("k_db_proj", "batch solver: projection 2", (k_db_proj<KM, 2><<<gs, DB_NT, P->smem_stream, s>>>(a)));
  DB_LAUNCH("k_db_sproj", "batch solver: orthonormalisation", (k_db_sproj<2><<<np, DB_ST, 0, s>>>(a)));
  DB_LAUNCH("k_db_new", "batch solver: new vectors", (k_db_new<KM><<<gs, DB_NT, 0, s>>>(a)));
  if ((st = transform_batch_launch(1, P->drev, (int)P->jrev.size(), P->trev, s)) != 0) return st;
  for (size_t g = 0; g < P->group_info.size(); ++g)
    if ((st = sigma_batch_launch(P->group_info[g], P->group_dev[g], s)) != 0) return st;
  if ((st = transform_batch_launch(0, P->dfwd, (int)P->jfwd.size(), P->tfwd, s)) != 0) return st;
  DB_LAUNCH("k_db_hv", "batch solver: H v", (k_db_hv<KM><<<gs, DB_NT, P->smem_stream, s>>>(a)));
  DB_LAUNCH("k_db_sritz", "batch solver: subspace eigenproblem", (k_db_sritz<<<np, DB_ST, P->smem_ritz, s>>>(a)));
  DB_LAUNCH("k_db_ritz", "batch solver: Ritz vectors", (k_db_ritz<KM><<<gs, DB_NT, P->smem_stream, s>>>(a)));
  DB_LAUNCH("k_db_sconv", "batch solver: convergence", (k_db_sconv<<<np, DB_ST, 0, s>>>(a)));
  DB_LAUNCH("k_db_pre", "batch solver: preconditioner", (k_db_pre<<<gs, DB_NT, 0, s>>>(a)));
#undef DB_LAUNCH
#undef DB_CHECK
  return CSFFCI_OK;
}

int enqueue_iteration(csffci_batch_plan_t* P, cudaStream_t s) {
  return P->kb <= 4 ? enqueue_iteration_km<4>(P, s) : enqueue_iteration_km<DB_KMAX>(P, s);
}

template <int KM>
int set_stream_smem(int bytes) {
  CSF_CUDA(cudaFuncSetAttribute(k_db_proj<KM, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  CSF_CUDA(cudaFuncSetAttribute(k_db_proj<KM, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  CSF_CUDA(cudaFuncSetAttribute(k_db_proj<KM, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  CSF_CUDA(cudaFuncSetAttribute(k_db_hv<KM>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  CSF_CUDA(cudaFuncSetAttribute(k_db_ritz<KM>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  return CSFFCI_OK;
}

}  // namespace

extern "C" {

int csffci_batch_plan_create(int nprob, const csffci_batch_problem_t* probs, const csffci_batch_options_t* opt,
                             csffci_batch_plan_t** plan, size_t* arena_bytes) {
  CSF_REQUIRE(plan && arena_bytes && opt, "batch_plan_create: NULL argument");
  *plan = nullptr;
  CSF_REQUIRE(nprob > 0 && probs, "batch_plan_create: empty batch");
  CSF_REQUIRE(opt->max_space >= 1 && opt->max_cycle >= 0, "batch_plan_create: bad options");
  for (int i = 0; i < nprob && opt->deterministic; ++i)
    CSF_REQUIRE(probs[i].norb >= 4 && probs[i].norb <= 16,
                "batch_plan_create: the deterministic scatter covers 4 <= norb <= 16, not %d", probs[i].norb);
  auto* P = new csffci_batch_plan();
  P->nprob = nprob;
  P->opt = *opt;
  if (P->opt.check_every < 1) P->opt.check_every = 1;
  P->in.assign(probs, probs + nprob);
  P->blocks.resize(nprob);
  P->prob.resize(nprob);
  P->ndet.resize(nprob);
  int kb = 1, capb = 1;
  long long nunits = 0;
  for (int i = 0; i < nprob; ++i) {
    const csffci_batch_problem_t& q = probs[i];
    if (!(q.norb >= 4 && q.norb <= 16 && q.neleca >= 0 && q.nelecb >= 0 && q.neleca <= q.norb &&
          q.nelecb <= q.norb && q.nroots >= 1 && q.nroots <= DB_KMAX && q.ncsf >= q.nroots &&
          q.nblocks >= 0 && (q.nblocks == 0 || q.blocks) && q.csd_mask && q.h2e && q.link_a && q.link_b &&
          q.hdiag && q.x0 && (q.eta == 0 || ((q.eta == 1 || q.eta == -1) && q.neleca == q.nelecb)))) {
      delete P;
      set_error("batch_plan_create: problem %d is invalid (norb 4..16, 1..%d roots <= ncsf, eta 0 or +-1 "
                "with neleca == nelecb, device pointers set)",
                i, DB_KMAX);
      return CSFFCI_ERR_INVALID;
    }
    const int cap = opt->max_space + 2 * q.nroots;
    if (cap > DB_CAPMAX) {
      delete P;
      set_error("batch_plan_create: max_space + 2*nroots = %d exceeds %d", cap, DB_CAPMAX);
      return CSFFCI_ERR_INVALID;
    }
    for (int b = 0; b < q.nblocks; ++b)
      if (q.blocks[b].conf_sel != nullptr) {
        delete P;
        set_error("batch_plan_create: problem %d: point-group-restricted CSF blocks are not supported", i);
        return CSFFCI_ERR_INVALID;
      }
    P->blocks[i].assign(q.blocks, q.blocks + q.nblocks);
    DBProb& d = P->prob[i];
    memset(&d, 0, sizeof(d));
    d.n = q.ncsf;
    d.k = q.nroots;
    d.cap = cap;
    d.space = opt->max_space + q.nroots;
    d.unit0 = (int32_t)nunits;
    d.nunits = (int32_t)((q.ncsf + DB_CH - 1) / DB_CH);
    d.hdiag = q.hdiag;
    nunits += d.nunits;
    P->ndet[i] = (int64_t)host_binom(q.norb, q.neleca) * (int64_t)host_binom(q.norb, q.nelecb);
    if (q.nroots > kb) kb = q.nroots;
    if (cap > capb) capb = cap;
  }
  P->kb = kb;
  P->capb = capb;
  P->nslot = kb * capb + 3 * kb;
  P->nunits = nunits;
  // arena: per-problem vectors, then the tables (offsets until bind)
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += al(bytes);
    return o;
  };
  std::vector<size_t> o_vec(nprob), o_det(nprob), o_small(nprob);
  for (int i = 0; i < nprob; ++i) {
    const DBProb& d = P->prob[i];
    o_vec[i] = take(sizeof(double) * (size_t)d.n * (2 * d.cap + 6 * d.k));
    // det buffers: k vectors, k sigmas, and per root the spin-symmetric
    // scratch (ndet doubles) or, with the deterministic scatter, the three
    // int64 digit planes (3 ndet)
    const int nscr = opt->deterministic ? 3 : (probs[i].eta ? 1 : 0);
    o_det[i] = take(sizeof(double) * (size_t)P->ndet[i] * d.k * (2 + nscr));
    o_small[i] = take(sizeof(double) * (2 * (size_t)d.cap * d.cap + 3 * (size_t)d.k * d.cap + d.cap));
  }
  const size_t o_partial = take(sizeof(double) * (size_t)nunits * P->nslot);
  const size_t o_prob = take(sizeof(DBProb) * nprob);
  const size_t o_state = take(sizeof(DBState) * nprob);
  const size_t o_units = take(sizeof(int32_t) * nunits);
  const size_t o_x0 = take(sizeof(double*) * nprob);
  const size_t o_count = take(sizeof(int));
  // sigma groups (one job per problem and root) and transform jobs
  std::vector<int> norbs;
  for (int i = 0; i < nprob; ++i) {
    bool seen = false;
    for (int v : norbs) seen |= v == probs[i].norb;
    if (!seen) norbs.push_back(probs[i].norb);
  }
  P->group_norb = norbs;
  std::vector<size_t> o_group(norbs.size());
  size_t max_group = 1;
  for (size_t g = 0; g < norbs.size(); ++g) {
    size_t nj = 0;
    for (int i = 0; i < nprob; ++i)
      if (probs[i].norb == norbs[g]) nj += probs[i].nroots;
    o_group[g] = take(sizeof(csffci_sigma_job_t) * nj);
    if (nj > max_group) max_group = nj;
  }
  const size_t o_tune = take(sizeof(csffci_sigma_job_t) * max_group);  // ungated copy for the autotuner
  size_t ntj = 0;
  for (int i = 0; i < nprob; ++i)
    for (int b = 0; b < probs[i].nblocks; ++b)
      if (probs[i].blocks[b].ncsf > 0 && probs[i].blocks[b].nconf > 0) ++ntj;
  const size_t o_rev = take(sizeof(csffci_transform_job_t) * (ntj ? ntj : 1));
  const size_t o_fwd = take(sizeof(csffci_transform_job_t) * (ntj ? ntj : 1));
  const size_t o_det_jobs = take(sizeof(csffci_transform_job_t) * (ntj ? ntj : 1));
  P->arena_bytes = off;
  for (int i = 0; i < nprob; ++i) {
    DBProb& d = P->prob[i];
    d.V = (double*)o_vec[i];
    d.h = (double*)o_small[i];
  }
  P->off_cdet.assign(o_det.begin(), o_det.end());
  P->args.partial = (double*)o_partial;
  P->args.prob = (const DBProb*)o_prob;
  P->args.st = (DBState*)o_state;
  P->args.unit_prob = (const int32_t*)o_units;
  P->dx0 = (double**)o_x0;
  P->args.count = (int*)o_count;
  P->group_dev.resize(norbs.size());
  for (size_t g = 0; g < norbs.size(); ++g) P->group_dev[g] = (csffci_sigma_job_t*)o_group[g];
  P->drev = (csffci_transform_job_t*)o_rev;
  P->dfwd = (csffci_transform_job_t*)o_fwd;
  P->ddet = (csffci_transform_job_t*)o_det_jobs;
  P->dtune = (csffci_sigma_job_t*)o_tune;
  *plan = P;
  *arena_bytes = P->arena_bytes;
  return CSFFCI_OK;
}

int csffci_batch_plan_bind(csffci_batch_plan_t* P, void* arena, size_t arena_bytes, cudaStream_t stream) {
  CSF_REQUIRE(P && !P->bound, "batch_plan_bind: plan missing or already bound");
  CSF_REQUIRE(arena && arena_bytes >= P->arena_bytes && ((uintptr_t)arena & 255) == 0,
              "batch_plan_bind: arena of %zu bytes (need %zu, 256-byte aligned)", arena_bytes, P->arena_bytes);
  char* base = (char*)arena;
  P->arena = base;
  auto rel = [&](const void* o) { return base + (size_t)(uintptr_t)o; };
  const int nprob = P->nprob;
  for (int i = 0; i < nprob; ++i) {
    DBProb& d = P->prob[i];
    double* v = (double*)rel(d.V);
    double* sm = (double*)rel(d.h);
    const size_t n = (size_t)d.n;
    d.V = v;
    d.AV = v + (size_t)d.cap * n;
    d.X = d.AV + (size_t)d.cap * n;
    d.AX = d.X + (size_t)d.k * n;
    d.R = d.AX + (size_t)d.k * n;
    d.T = d.R + (size_t)d.k * n;
    d.W = d.T + (size_t)d.k * n;
    d.AW = d.W + (size_t)d.k * n;
    d.h = sm;
    d.coef = sm + (size_t)d.cap * d.cap;
    d.cc = d.coef + (size_t)d.k * d.cap;
    d.xprev = d.cc + (size_t)d.k * d.cap;
    d.qprev = d.xprev + (size_t)d.k * d.cap;
    d.dprev = d.qprev + (size_t)d.cap * d.cap;
  }
  P->args.partial = (double*)rel(P->args.partial);
  P->args.prob = (const DBProb*)rel(P->args.prob);
  P->args.st = (DBState*)rel(P->args.st);
  P->args.unit_prob = (const int32_t*)rel(P->args.unit_prob);
  P->dx0 = (double**)rel(P->dx0);
  P->args.count = (int*)rel(P->args.count);
  for (auto& g : P->group_dev) g = (csffci_sigma_job_t*)rel(g);
  P->drev = (csffci_transform_job_t*)rel(P->drev);
  P->dfwd = (csffci_transform_job_t*)rel(P->dfwd);
  P->ddet = (csffci_transform_job_t*)rel(P->ddet);
  P->dtune = (csffci_sigma_job_t*)rel(P->dtune);
  P->args.nslot = P->nslot;
  P->args.capb = P->capb;
  P->args.kb = P->kb;
  P->args.nprob = nprob;
  P->args.nunits = P->nunits;
  P->args.tol = P->opt.conv_tol;
  P->args.toloose = P->opt.conv_tol_residual > 0 ? P->opt.conv_tol_residual : sqrt(P->opt.conv_tol);
  P->args.lindep = P->opt.lindep;
  P->args.shift = P->opt.level_shift;
  P->unit_prob.resize(P->nunits);
  for (int i = 0; i < nprob; ++i)
    for (int u = 0; u < P->prob[i].nunits; ++u) P->unit_prob[P->prob[i].unit0 + u] = i;
  // sigma job tables: job (problem i, root v) gated by knew of problem i
  P->group_jobs.assign(P->group_norb.size(), {});
  P->group_info.assign(P->group_norb.size(), SigmaBatchInfo());
  DBState* st = P->args.st;
  for (size_t g = 0; g < P->group_norb.size(); ++g) {
    for (int i = 0; i < nprob; ++i) {
      const csffci_batch_problem_t& q = P->in[i];
      if (q.norb != P->group_norb[g]) continue;
      double* det = (double*)(base + P->off_cdet[i]);
      const size_t nd = (size_t)P->ndet[i];
      for (int v = 0; v < q.nroots; ++v) {
        csffci_sigma_job_t J;
        memset(&J, 0, sizeof(J));
        J.h2e = q.h2e;
        J.link_a = q.link_a;
        J.link_b = q.link_b;
        J.ci = det + (size_t)v * nd;
        J.sigma = det + (size_t)(q.nroots + v) * nd;
        if (P->opt.deterministic) {
          J.scratch = det + (size_t)(2 * q.nroots + 3 * v) * nd;
          J.flags = CSFFCI_SIGMA_JOB_DETERMINISTIC;
        } else {
          J.scratch = q.eta ? det + (size_t)(2 * q.nroots + v) * nd : nullptr;
        }
        J.neleca = q.neleca;
        J.nelecb = q.nelecb;
        J.sym = q.eta ? 1 : 0;
        J.eta = q.eta ? q.eta : 1;
        J.live = &st[i].knew;
        J.live_index = v;
        P->group_jobs[g].push_back(J);
      }
    }
    int stt = sigma_batch_prepare(P->group_norb[g], (int)P->group_jobs[g].size(), P->group_jobs[g].data(),
                                  &P->group_info[g]);
    if (stt) return stt;
  }
  // transform tables: W -> cdet (gated by knew), sdet -> AW (gated by
  // knew), X -> cdet (gated by kk, for the final vectors)
  P->jrev.clear();
  P->jfwd.clear();
  P->jdet.clear();
  for (int i = 0; i < nprob; ++i) {
    const csffci_batch_problem_t& q = P->in[i];
    const DBProb& d = P->prob[i];
    double* det = (double*)(base + P->off_cdet[i]);
    const int64_t nd = P->ndet[i];
    for (const csffci_block_t& b : P->blocks[i]) {
      if (b.ncsf <= 0 || b.nconf <= 0) continue;
      csffci_transform_job_t J;
      memset(&J, 0, sizeof(J));
      J.mask = q.csd_mask;
      J.umat = b.umat;
      J.csd_offset = b.csd_offset;
      J.csf_offset = b.csf_offset;
      J.nconf = b.nconf;
      J.ndet = b.ndet;
      J.ncsf = b.ncsf;
      J.nvec = q.nroots;
      J.sign = b.sign;
      csffci_transform_job_t r = J, f = J, x = J;
      r.x = d.W;
      r.ldx = d.n;
      r.y = det;
      r.ldy = nd;
      r.live = &st[i].knew;
      f.x = det + (size_t)q.nroots * nd;
      f.ldx = nd;
      f.y = d.AW;
      f.ldy = d.n;
      f.live = &st[i].knew;
      x.x = d.X;
      x.ldx = d.n;
      x.y = det;
      x.ldy = nd;
      x.live = &st[i].kk;
      P->jrev.push_back(r);
      P->jfwd.push_back(f);
      P->jdet.push_back(x);
    }
  }
  int stt = transform_batch_prepare(1, (int)P->jrev.size(), P->jrev.data(), &P->trev);
  if (!stt) stt = transform_batch_prepare(0, (int)P->jfwd.size(), P->jfwd.data(), &P->tfwd);
  if (!stt) stt = transform_batch_prepare(1, (int)P->jdet.size(), P->jdet.data(), &P->tdet);
  if (stt) return stt;
  // uploads
  std::vector<const double*> x0(nprob);
  for (int i = 0; i < nprob; ++i) x0[i] = P->in[i].x0;
  CSF_CUDA(cudaMemcpyAsync((void*)P->args.prob, P->prob.data(), sizeof(DBProb) * nprob, cudaMemcpyHostToDevice,
                           stream));
  CSF_CUDA(cudaMemcpyAsync((void*)P->args.unit_prob, P->unit_prob.data(), sizeof(int32_t) * P->nunits,
                           cudaMemcpyHostToDevice, stream));
  CSF_CUDA(cudaMemcpyAsync(P->dx0, x0.data(), sizeof(double*) * nprob, cudaMemcpyHostToDevice, stream));
  for (size_t g = 0; g < P->group_jobs.size(); ++g)
    CSF_CUDA(cudaMemcpyAsync(P->group_dev[g], P->group_jobs[g].data(),
                             sizeof(csffci_sigma_job_t) * P->group_jobs[g].size(), cudaMemcpyHostToDevice, stream));
  if (!P->jrev.empty()) {
    const size_t nb = sizeof(csffci_transform_job_t) * P->jrev.size();
    CSF_CUDA(cudaMemcpyAsync(P->drev, P->jrev.data(), nb, cudaMemcpyHostToDevice, stream));
    CSF_CUDA(cudaMemcpyAsync(P->dfwd, P->jfwd.data(), nb, cudaMemcpyHostToDevice, stream));
    CSF_CUDA(cudaMemcpyAsync(P->ddet, P->jdet.data(), nb, cudaMemcpyHostToDevice, stream));
  }
  // determinant vectors read as zero outside the CSF blocks: clear once
  for (int i = 0; i < nprob; ++i)
    CSF_CUDA(cudaMemsetAsync(base + P->off_cdet[i], 0,
                             sizeof(double) * (size_t)P->ndet[i] * P->in[i].nroots, stream));
  // autotuner: every tile variant timed on each group's jobs (ungated
  // copy; the outputs are scratch at this point)
  if (P->opt.autotune) {
    for (size_t g = 0; g < P->group_jobs.size(); ++g) {
      std::vector<csffci_sigma_job_t> ung = P->group_jobs[g];
      for (auto& J : ung) J.live = nullptr;
      CSF_CUDA(cudaMemcpyAsync(P->dtune, ung.data(), sizeof(csffci_sigma_job_t) * ung.size(),
                               cudaMemcpyHostToDevice, stream));
      SigmaBatchInfo t = P->group_info[g];
      t.job0.live = nullptr;
      int stt2 = sigma_batch_tune(t, ung.data(), P->dtune, stream);
      if (stt2) return stt2;
      P->group_info[g].variant = t.variant;
      CSF_CUDA(cudaStreamSynchronize(stream));  // ung is released below
    }
  }
  k_db_init<<<nprob, 256, 0, stream>>>(P->args, (const double* const*)P->dx0);
  int st2 = check_launch("batch solver: init");
  if (st2) return st2;
  // shared memory of the streaming and subspace kernels
  P->smem_stream = sizeof(double) * DB_NW * P->nslot;
  P->smem_ritz = sizeof(double) * (2 * P->capb * P->capb + 2 * P->capb + 4 + P->capb + DB_KMAX * P->capb +
                                   2 * DB_ST + 2) +
                 sizeof(int) * P->capb;
  if (P->smem_stream > 48 * 1024) {
    st2 = P->kb <= 4 ? set_stream_smem<4>((int)P->smem_stream) : set_stream_smem<DB_KMAX>((int)P->smem_stream);
    if (st2) return st2;
  }
  if (P->smem_ritz > 48 * 1024)
    CSF_CUDA(cudaFuncSetAttribute(k_db_sritz, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P->smem_ritz));
  CSF_CUDA(cudaMallocHost(&P->hcount, sizeof(int)));
  CSF_CUDA(cudaStreamSynchronize(stream));
  P->bound = true;
  return CSFFCI_OK;
}

int csffci_batch_plan_run(csffci_batch_plan_t* P, cudaStream_t stream, int* iterations) {
  CSF_REQUIRE(P && P->bound, "batch_plan_run: plan not bound");
  int it = 0, st = 0;
  const int maxc = P->opt.max_cycle;
  if (maxc > 0 && P->opt.use_graph && !P->exec) {
    // first iteration eagerly (sets kernel attributes, validates the
    // launch sequence), then one iteration captured as a graph
    if ((st = enqueue_iteration(P, stream)) != 0) return st;
    ++it;
    if (!P->cap_stream) CSF_CUDA(cudaStreamCreateWithFlags(&P->cap_stream, cudaStreamNonBlocking));
    CSF_CUDA(cudaStreamSynchronize(stream));
    CSF_CUDA(cudaStreamBeginCapture(P->cap_stream, cudaStreamCaptureModeRelaxed));
    st = enqueue_iteration(P, P->cap_stream);
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(P->cap_stream, &g);
    if (st) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    CSF_CUDA(ce);
    P->graph = g;
    CSF_CUDA(cudaGraphInstantiate(&P->exec, P->graph, 0));
  }
  while (it < maxc) {
    int n = P->opt.check_every;
    if (n > maxc - it) n = maxc - it;
    for (int r = 0; r < n; ++r) {
      if (P->exec) {
        CSF_CUDA(cudaGraphLaunch(P->exec, stream));
      } else if ((st = enqueue_iteration(P, stream)) != 0) {
        return st;
      }
    }
    it += n;
    k_db_count<<<1, 256, 0, stream>>>(P->args);
    if ((st = check_launch("batch solver: count")) != 0) return st;
    CSF_CUDA(cudaMemcpyAsync(P->hcount, P->args.count, sizeof(int), cudaMemcpyDeviceToHost, stream));
    CSF_CUDA(cudaStreamSynchronize(stream));
    if (*P->hcount == 0) break;
  }
  P->iterations = it;
  if (iterations) *iterations = it;
  return CSFFCI_OK;
}

int csffci_batch_plan_max_roots(const csffci_batch_plan_t* P) { return P ? P->kb : 0; }

int csffci_batch_plan_tile_variants(const csffci_batch_plan_t* P, int32_t* norb, int32_t* variant, int cap) {
  if (!P) return 0;
  const int n = (int)P->group_norb.size();
  for (int g = 0; g < n && g < cap; ++g) {
    if (norb) norb[g] = P->group_norb[g];
    if (variant)
      variant[g] = (g < (int)P->group_info.size() && P->group_info[g].variant >= 0)
                       ? P->group_info[g].variant
                       : rr_default_variant(P->group_norb[g]);
  }
  return n;
}

int csffci_batch_plan_results(csffci_batch_plan_t* P, double* energies, int32_t* converged, int32_t* niter,
                              int32_t* nfound, cudaStream_t stream) {
  CSF_REQUIRE(P && P->bound, "batch_plan_results: plan not bound");
  std::vector<DBState> st(P->nprob);
  CSF_CUDA(cudaMemcpyAsync(st.data(), P->args.st, sizeof(DBState) * P->nprob, cudaMemcpyDeviceToHost, stream));
  CSF_CUDA(cudaStreamSynchronize(stream));
  const int kb = P->kb;
  for (int i = 0; i < P->nprob; ++i) {
    for (int r = 0; r < kb; ++r) {
      const bool have = r < st[i].kk;
      if (energies) energies[i * kb + r] = have ? st[i].e[r] : NAN;
      if (converged) converged[i * kb + r] = have ? st[i].conv[r] : 0;
    }
    if (niter) niter[i] = st[i].niter;
    if (nfound) nfound[i] = st[i].kk;
  }
  return CSFFCI_OK;
}

int csffci_batch_plan_to_det(csffci_batch_plan_t* P, cudaStream_t stream) {
  CSF_REQUIRE(P && P->bound, "batch_plan_to_det: plan not bound");
  for (int i = 0; i < P->nprob; ++i)
    CSF_CUDA(cudaMemsetAsync(P->arena + P->off_cdet[i], 0, sizeof(double) * (size_t)P->ndet[i] * P->in[i].nroots,
                             stream));
  return transform_batch_launch(1, P->ddet, (int)P->jdet.size(), P->tdet, stream);
}

int csffci_batch_plan_vectors(const csffci_batch_plan_t* P, int iprob, const double** csf, const double** det) {
  CSF_REQUIRE(P && P->bound && iprob >= 0 && iprob < P->nprob, "batch_plan_vectors: bad problem index");
  if (csf) *csf = P->prob[iprob].X;
  if (det) *det = (const double*)(P->arena + P->off_cdet[iprob]);
  return CSFFCI_OK;
}

void csffci_batch_plan_destroy(csffci_batch_plan_t* P) {
  if (!P) return;
  if (P->exec) cudaGraphExecDestroy(P->exec);
  if (P->graph) cudaGraphDestroy(P->graph);
  if (P->cap_stream) cudaStreamDestroy(P->cap_stream);
  if (P->hcount) cudaFreeHost(P->hcount);
  delete P;
}

}  // extern "C"
