// Reduced density matrices as the adjoint of sigma, and the split-K Gram
// kernel they share with the Davidson update.
//
//   T[pq][J] = <J|E_pq|c>  (gathered through the link tables of J, the same
//   way sigma builds D, but over all norb^2 ordered pairs)
//   <bra|E_pq E_rs|ket> = sum_J Tb[qp][J] Tk[rs][J]            (Gram GEMM)
//   dm1[p][q] = <bra|E_qp|ket>,  dm2[p][q][r][s] = <E_pq E_rs> - d_qr <E_ps>
// (conventions of pyscf/lib/mcscf/fci_gas.h:260-268).  The determinant
// space is processed in slabs that fit the caller's workspace, so D(pq,J)
// is never materialised for the whole space.
#include <utility>

#include "common.cuh"
#include "profile.cuh"

namespace csffci {

// ---------------------------------------------------------------------------
// skinny Gram for the Davidson projections: out[i][j] = sum_k X[i][k] Y[j][k]
// with at most GS_MAXY vectors on one side (the new corrections or the Ritz
// vectors) and at most GS_MAXX on the other (the subspace).  Each block
// streams k-chunks of GS_NT*KT elements: the chunk of the narrow side stays
// in registers while every row of the wide side is read once (coalesced,
// KT loads per thread), so the kernel moves (nx + ny) * n * 8 bytes and is
// bound by HBM bandwidth.  Per-warp sums accumulate in shared memory in a
// fixed order; the block partials are summed over the blocks in a fixed
// order as well, so results are bit-reproducible.
// ---------------------------------------------------------------------------
constexpr int GS_NT = 256, GS_MAXX = 64, GS_MAXY = 4;

template <int NY, int KT>
__global__ void __launch_bounds__(GS_NT) k_gram_skinny(int nx, const double* __restrict__ x, int64_t ldx, int ny,
                                                       const double* __restrict__ y, int64_t ldy, int64_t n,
                                                       double* part) {
  __shared__ double wsum[GS_NT / 32][GS_MAXX][NY];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int e = lane; e < GS_MAXX * NY; e += 32) (&wsum[warp][0][0])[e] = 0.0;
  __syncwarp();
  constexpr int KC = GS_NT * KT;
  for (int64_t k0 = (int64_t)blockIdx.x * KC; k0 < n; k0 += (int64_t)gridDim.x * KC) {
    double yv[NY][KT];
#pragma unroll
    for (int q = 0; q < KT; ++q) {
      const int64_t k = k0 + tid + (int64_t)q * GS_NT;
#pragma unroll
      for (int j = 0; j < NY; ++j) yv[j][q] = (j < ny && k < n) ? y[(int64_t)j * ldy + k] : 0.0;
    }
    for (int i = 0; i < nx; ++i) {
      const double* xi = x + (int64_t)i * ldx;
      double sj[NY];
#pragma unroll
      for (int j = 0; j < NY; ++j) sj[j] = 0.0;
#pragma unroll
      for (int q = 0; q < KT; ++q) {
        const int64_t k = k0 + tid + (int64_t)q * GS_NT;
        const double xv = k < n ? xi[k] : 0.0;
#pragma unroll
        for (int j = 0; j < NY; ++j) sj[j] = fma(xv, yv[j][q], sj[j]);
      }
#pragma unroll
      for (int j = 0; j < NY; ++j) {
        double v = sj[j];
#pragma unroll
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        sj[j] = v;
      }
      if (lane == 0) {
#pragma unroll
        for (int j = 0; j < NY; ++j) wsum[warp][i][j] += sj[j];
      }
    }
  }
  __syncthreads();
  for (int e = tid; e < nx * NY; e += GS_NT) {
    const int i = e / NY, j = e - i * NY;
    double v = 0.0;
#pragma unroll
    for (int w = 0; w < GS_NT / 32; ++w) v += wsum[w][i][j];
    part[(int64_t)blockIdx.x * nx * NY + e] = v;
  }
}

// out[i][j] (or out[j][i] when transposed) = sum over the blocks of part
__global__ void k_gram_skinny_reduce(int nx, int ny, int ystride, int nblk, const double* part, double* out,
                                     int transposed) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nx * ny; e += gridDim.x * blockDim.x) {
    const int i = e / ny, j = e - i * ny;
    double v = 0.0;
    for (int b = 0; b < nblk; ++b) v += part[((int64_t)b * nx + i) * ystride + j];
    if (transposed)
      out[(int64_t)j * nx + i] = v;
    else
      out[e] = v;
  }
}

static int gram_skinny_ystride(int ny) { return ny <= 1 ? 1 : ny <= 2 ? 2 : 4; }

static int gram_skinny_blocks(int64_t n, int ny) {
  const int kt = ny <= 2 ? 16 : 8;
  int64_t nb = (n + GS_NT * kt - 1) / (GS_NT * kt);
  if (nb > 148 * 4) nb = 148 * 4;
  return (int)(nb < 1 ? 1 : nb);
}

static bool gram_skinny_fits(int nx, int ny) {
  return (ny <= GS_MAXY && nx <= GS_MAXX) || (nx <= GS_MAXY && ny <= GS_MAXX);
}

static size_t gram_skinny_workspace(int nx, int ny, int64_t n) {
  if (!(ny <= GS_MAXY && nx <= GS_MAXX)) std::swap(nx, ny);
  return (size_t)gram_skinny_blocks(n, ny) * nx * gram_skinny_ystride(ny) * sizeof(double);
}

static int gram_skinny_run(int nx, const double* x, int64_t ldx, int ny, const double* y, int64_t ldy, int64_t n,
                           double* out, double* part, cudaStream_t stream) {
  int transposed = 0;
  if (!(ny <= GS_MAXY && nx <= GS_MAXX)) {
    std::swap(nx, ny);
    std::swap(x, y);
    std::swap(ldx, ldy);
    transposed = 1;
  }
  const int nblk = gram_skinny_blocks(n, ny);
  const int ys = gram_skinny_ystride(ny);
  {
    ProfScope ps_("k_gram_skinny", stream);
    if (ys == 1)
      k_gram_skinny<1, 16><<<nblk, GS_NT, 0, stream>>>(nx, x, ldx, ny, y, ldy, n, part);
    else if (ys == 2)
      k_gram_skinny<2, 16><<<nblk, GS_NT, 0, stream>>>(nx, x, ldx, ny, y, ldy, n, part);
    else
      k_gram_skinny<4, 8><<<nblk, GS_NT, 0, stream>>>(nx, x, ldx, ny, y, ldy, n, part);
  }
  int st = check_launch("gram (skinny)");
  if (st) return st;
  k_gram_skinny_reduce<<<grid_for(nx * ny, 128), 128, 0, stream>>>(nx, ny, ys, nblk, part, out, transposed);
  return check_launch("gram (skinny) reduce");
}

// ---------------------------------------------------------------------------
// split-K Gram: part[split][i][j] = sum_{k in split} X[i][k] Y[j][k]
// then out[i][j] (+)= sum_split part[split][i][j] in a fixed order.
// ---------------------------------------------------------------------------
constexpr int GT = 32, GK = 32;

__global__ void __launch_bounds__(256) k_gram_part(int nx, const double* __restrict__ x, int64_t ldx,
                                                   int ny, const double* __restrict__ y, int64_t ldy,
                                                   int64_t n, int64_t kchunk, int nsplit,
                                                   double* part) {
  __shared__ double Xs[GK][GT + 1];
  __shared__ double Ys[GK][GT + 1];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int tiles_i = (nx + GT - 1) / GT, tiles_j = (ny + GT - 1) / GT;
  const int64_t ntask = (int64_t)tiles_i * tiles_j * nsplit;
  for (int64_t task = blockIdx.x; task < ntask; task += gridDim.x) {
    int split = (int)(task % nsplit);
    int64_t tt = task / nsplit;
    int ti = (int)(tt / tiles_j), tj = (int)(tt % tiles_j);
    int64_t k_begin = split * kchunk, k_end = k_begin + kchunk;
    if (k_end > n) k_end = n;
    double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
    for (int64_t k0 = k_begin; k0 < k_end; k0 += GK) {
      for (int e = tid; e < GT * GK; e += 256) {
        int r = e / GK, kk = e - r * GK;
        int gi = ti * GT + r, gj = tj * GT + r;
        int64_t k = k0 + kk;
        Xs[kk][r] = (gi < nx && k < k_end) ? x[(int64_t)gi * ldx + k] : 0.0;
        Ys[kk][r] = (gj < ny && k < k_end) ? y[(int64_t)gj * ldy + k] : 0.0;
      }
      __syncthreads();
#pragma unroll 8
      for (int kk = 0; kk < GK; ++kk) {
        double a0 = Xs[kk][ty], a1 = Xs[kk][ty + 16];
        double b0 = Ys[kk][tx], b1 = Ys[kk][tx + 16];
        acc[0][0] = fma(a0, b0, acc[0][0]);
        acc[0][1] = fma(a0, b1, acc[0][1]);
        acc[1][0] = fma(a1, b0, acc[1][0]);
        acc[1][1] = fma(a1, b1, acc[1][1]);
      }
      __syncthreads();
    }
    double* P = part + (int64_t)split * nx * ny;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        int gi = ti * GT + ty + 16 * a, gj = tj * GT + tx + 16 * b;
        if (gi < nx && gj < ny) P[(int64_t)gi * ny + gj] = acc[a][b];
      }
  }
}

__global__ void k_gram_reduce(int nxy, int nsplit, const double* part, double* out, int accumulate) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nxy; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int p = 0; p < nsplit; ++p) s += part[(int64_t)p * nxy + i];
    out[i] = accumulate ? out[i] + s : s;
  }
}

static int gram_nsplit(int nx, int ny, int64_t n) {
  int tiles = ((nx + GT - 1) / GT) * ((ny + GT - 1) / GT);
  int64_t want = (148 * 4 + tiles - 1) / tiles;
  int64_t maxs = (n + 4095) / 4096;
  if (want > maxs) want = maxs;
  if (want < 1) want = 1;
  if (want > 1024) want = 1024;
  return (int)want;
}

size_t gram_workspace(int nx, int ny, int64_t n) {
  return (size_t)gram_nsplit(nx, ny, n) * nx * ny * sizeof(double);
}

int gram_run(int nx, const double* x, int64_t ldx, int ny, const double* y, int64_t ldy, int64_t n,
             double* out, int accumulate, double* part, cudaStream_t stream) {
  int nsplit = gram_nsplit(nx, ny, n);
  int64_t kchunk = (n + nsplit - 1) / nsplit;
  kchunk = (kchunk + GK - 1) / GK * GK;
  nsplit = (int)((n + kchunk - 1) / kchunk);
  if (nsplit < 1) nsplit = 1;
  int tiles = ((nx + GT - 1) / GT) * ((ny + GT - 1) / GT);
  {
    ProfScope ps_("k_gram_part", stream);
    k_gram_part<<<grid_for((int64_t)tiles * nsplit, 1, 148 * 8), 256, 0, stream>>>(
        nx, x, ldx, ny, y, ldy, n, kchunk, nsplit, part);
  }
  int st = check_launch("gram");
  if (st) return st;
  k_gram_reduce<<<grid_for(nx * ny, 256), 256, 0, stream>>>(nx * ny, nsplit, part, out, accumulate);
  return check_launch("gram reduce");
}

// ---------------------------------------------------------------------------
// FP64 tensor-core Gram for the RDM contraction G = X Y^T (nx, ny ~ norb^2,
// K = determinants of a slab): 64x64 tiles, 8 warps of 32x16 (m8n8k4 DMMA),
// K staged through shared memory in 16-wide chunks (double-buffered
// cp.async), split-K partials reduced in a fixed order.  With sym (X == Y)
// only the tiles on and above the diagonal are formed and the reduction
// mirrors the rest.
// ---------------------------------------------------------------------------
constexpr int GD_T = 64, GD_KC = 16, GD_LD = 20;  // LD = 4 (mod 16): conflict-free fragment loads

__device__ __forceinline__ void gd_dmma(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void gd_cp8(double* s, const double* g) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(g) : "memory");
}

__device__ __forceinline__ void gd_stage(double* As, double* Bs, const double* x, int64_t ldx, int nx,
                                         const double* y, int64_t ldy, int ny, int i0, int j0, int64_t k0,
                                         int64_t k_end) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int r = 0; r < (GD_T * GD_KC) / 256; ++r) {
    const int e = tid + 256 * r;
    const int row = e / GD_KC, kk = e - row * GD_KC;
    const int64_t k = k0 + kk;
    double* da = &As[row * GD_LD + kk];
    double* db = &Bs[row * GD_LD + kk];
    if (i0 + row < nx && k < k_end)
      gd_cp8(da, &x[(int64_t)(i0 + row) * ldx + k]);
    else
      *da = 0.0;
    if (j0 + row < ny && k < k_end)
      gd_cp8(db, &y[(int64_t)(j0 + row) * ldy + k]);
    else
      *db = 0.0;
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}

__global__ void __launch_bounds__(256) k_gram_dmma(int nx, const double* __restrict__ x, int64_t ldx, int ny,
                                                   const double* __restrict__ y, int64_t ldy, int64_t n,
                                                   int64_t kchunk, int nsplit, int sym, double* part) {
  __shared__ __align__(16) double As[2][GD_T * GD_LD];
  __shared__ __align__(16) double Bs[2][GD_T * GD_LD];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  const int wi = warp & 1, wj = warp >> 1;
  const int tiles_i = (nx + GD_T - 1) / GD_T, tiles_j = (ny + GD_T - 1) / GD_T;
  const int npairs = sym ? tiles_i * (tiles_i + 1) / 2 : tiles_i * tiles_j;
  const int64_t ntask = (int64_t)npairs * nsplit;
  for (int64_t task = blockIdx.x; task < ntask; task += gridDim.x) {
    const int split = (int)(task % nsplit);
    int tp = (int)(task / nsplit), ti, tj;
    if (sym) {  // (ti, tj) with ti <= tj, row-major over the upper triangle
      ti = 0;
      while (tp >= tiles_i - ti) {
        tp -= tiles_i - ti;
        ++ti;
      }
      tj = ti + tp;
    } else {
      ti = tp / tiles_j;
      tj = tp - ti * tiles_j;
    }
    const int i0 = ti * GD_T, j0 = tj * GD_T;
    const int64_t k_begin = (int64_t)split * kchunk;
    const int64_t k_end = min(n, k_begin + kchunk);
    const int nkc = (int)((k_end - k_begin + GD_KC - 1) / GD_KC);
    double acc[4][2][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    __syncthreads();  // the buffers of the previous task are consumed
    if (nkc > 0) gd_stage(As[0], Bs[0], x, ldx, nx, y, ldy, ny, i0, j0, k_begin, k_end);
    for (int c = 0; c < nkc; ++c) {
      const int b = c & 1;
      if (c + 1 < nkc) {
        gd_stage(As[b ^ 1], Bs[b ^ 1], x, ldx, nx, y, ldy, ny, i0, j0, k_begin + (int64_t)(c + 1) * GD_KC,
                 k_end);
        asm volatile("cp.async.wait_group 1;\n" ::: "memory");
      } else {
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
      }
      __syncthreads();
      const double* Ab = As[b] + (wi * 32 + gq) * GD_LD + tq;
      const double* Bb = Bs[b] + (wj * 16 + gq) * GD_LD + tq;
#pragma unroll
      for (int s4 = 0; s4 < GD_KC / 4; ++s4) {
        double av[4], bv[2];
#pragma unroll
        for (int a = 0; a < 4; ++a) av[a] = Ab[a * 8 * GD_LD + 4 * s4];
#pragma unroll
        for (int bb = 0; bb < 2; ++bb) bv[bb] = Bb[bb * 8 * GD_LD + 4 * s4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int bb = 0; bb < 2; ++bb) gd_dmma(acc[a][bb], av[a], bv[bb]);
      }
      __syncthreads();  // buffer b is free for the chunk after next
    }
    double* P = part + (int64_t)split * nx * ny;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int i = i0 + wi * 32 + a * 8 + gq;
      if (i >= nx) continue;
#pragma unroll
      for (int bb = 0; bb < 2; ++bb) {
        const int j = j0 + wj * 16 + bb * 8 + 2 * tq;
        if (j < ny) P[(int64_t)i * ny + j] = acc[a][bb][0];
        if (j + 1 < ny) P[(int64_t)i * ny + j + 1] = acc[a][bb][1];
      }
    }
  }
}

// out[i][j] (+)= sum_split part[split][i][j]; with sym the tiles below the
// diagonal read the transposed entry of their mirror tile
__global__ void k_gram_reduce_sym(int nx, int ny, int nsplit, const double* part, double* out, int accumulate,
                                  int sym) {
  const int nxy = nx * ny;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nxy; t += gridDim.x * blockDim.x) {
    const int i = t / ny, j = t - i * ny;
    const int src = (sym && i / GD_T > j / GD_T) ? j * ny + i : t;
    double s = 0.0;
    for (int p = 0; p < nsplit; ++p) s += part[(int64_t)p * nxy + src];
    out[t] = accumulate ? out[t] + s : s;
  }
}

static int gram_dmma_nsplit(int nx, int ny, int64_t n) {
  const int ti = (nx + GD_T - 1) / GD_T, tj = (ny + GD_T - 1) / GD_T;
  const int tiles = ti * tj;
  int64_t want = (148 * 3 + tiles - 1) / tiles;
  int64_t maxs = (n + 1023) / 1024;
  if (want > maxs) want = maxs;
  if (want < 1) want = 1;
  if (want > 256) want = 256;
  return (int)want;
}

size_t gram_dmma_workspace(int nx, int ny, int64_t n) {
  return (size_t)gram_dmma_nsplit(nx, ny, n) * nx * ny * sizeof(double);
}

int gram_dmma_run(int nx, const double* x, int64_t ldx, int ny, const double* y, int64_t ldy, int64_t n,
                  double* out, int accumulate, double* part, cudaStream_t stream) {
  const int sym = (x == y && ldx == ldy && nx == ny) ? 1 : 0;
  int nsplit = gram_dmma_nsplit(nx, ny, n);
  int64_t kchunk = (n + nsplit - 1) / nsplit;
  kchunk = (kchunk + GD_KC - 1) / GD_KC * GD_KC;
  nsplit = (int)((n + kchunk - 1) / kchunk);
  if (nsplit < 1) nsplit = 1;
  const int ti = (nx + GD_T - 1) / GD_T, tj = (ny + GD_T - 1) / GD_T;
  const int npairs = sym ? ti * (ti + 1) / 2 : ti * tj;
  {
    ProfScope ps("k_gram_dmma", stream);
    k_gram_dmma<<<grid_for((int64_t)npairs * nsplit, 1, 148 * 4), 256, 0, stream>>>(nx, x, ldx, ny, y, ldy, n,
                                                                                   kchunk, nsplit, sym, part);
  }
  int st = check_launch("gram (tensor cores)");
  if (st) return st;
  k_gram_reduce_sym<<<grid_for(nx * ny, 256), 256, 0, stream>>>(nx, ny, nsplit, part, out, accumulate, sym);
  return check_launch("gram reduce");
}

// ---------------------------------------------------------------------------
// T slab: T[pq][j] for determinants J = J0 + j, j < S, pq = p*norb + q
// ---------------------------------------------------------------------------
// T slab built 32 determinants per block in shared memory: the alpha
// and/or beta link contributions of each determinant are added into a
// zeroed (n^2, 32) tile, which is then written out row by row (coalesced,
// each T element written once; no separate zeroing pass and no scattered
// read-modify-write in global memory).  spin: 0 alpha, 1 beta, 2 both.
constexpr int TT_J = 32, TT_LD = 33;

__global__ void __launch_bounds__(256) k_tslab_tile(int norb, long long Nb, int nla, int nlb,
                                                    const csffci_link_t* __restrict__ la,
                                                    const csffci_link_t* __restrict__ lb,
                                                    const double* __restrict__ c, long long J0, long long S,
                                                    int spin, double* __restrict__ T) {
  extern __shared__ double tile[];  // [n^2][TT_LD]
  const int n2 = norb * norb;
  const long long nblk = (S + TT_J - 1) / TT_J;
  for (long long blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
    const long long j0 = blk * TT_J;
    const int nj = (int)min((long long)TT_J, S - j0);
    __syncthreads();  // the previous tile is written out
    for (int i = threadIdx.x; i < n2 * TT_LD; i += blockDim.x) tile[i] = 0.0;
    __syncthreads();
    if (spin != 1) {
      for (int idx = threadIdx.x; idx < nla * TT_J; idx += blockDim.x) {
        const int l = idx / TT_J, t = idx - l * TT_J;
        if (t >= nj) continue;
        const long long J = J0 + j0 + t, ja = J / Nb, jb = J - ja * Nb;
        const csffci_link_t e = la[ja * nla + l];
        const int a = e.op & 0xff, i = e.op >> 8;
        tile[(i * norb + a) * TT_LD + t] += e.sign * c[(long long)e.addr * Nb + jb];
      }
      __syncthreads();
    }
    if (spin != 0) {
      for (int idx = threadIdx.x; idx < nlb * TT_J; idx += blockDim.x) {
        const int l = idx / TT_J, t = idx - l * TT_J;
        if (t >= nj) continue;
        const long long J = J0 + j0 + t, ja = J / Nb, jb = J - ja * Nb;
        const csffci_link_t e = lb[jb * nlb + l];
        const int a = e.op & 0xff, i = e.op >> 8;
        tile[(i * norb + a) * TT_LD + t] += e.sign * c[ja * Nb + e.addr];
      }
      __syncthreads();
    }
    for (int idx = threadIdx.x; idx < n2 * TT_J; idx += blockDim.x) {
      const int pq = idx / TT_J, t = idx - pq * TT_J;
      if (t < nj) T[(long long)pq * S + j0 + t] = tile[pq * TT_LD + t];
    }
  }
}

static int tslab_tile_launch(int norb, long long Nb, int nla, int nlb, const csffci_link_t* la,
                             const csffci_link_t* lb, const double* c, long long J0, long long s, int spin,
                             double* T, cudaStream_t stream) {
  const size_t smem = (size_t)norb * norb * TT_LD * sizeof(double);
  if (smem > 48 * 1024) CSF_CUDA(cudaFuncSetAttribute(k_tslab_tile, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                      (int)smem));
  ProfScope ps("k_tslab_tile", stream);
  k_tslab_tile<<<grid_for((s + TT_J - 1) / TT_J, 1, 148 * 4), 256, smem, stream>>>(norb, Nb, nla, nlb, la, lb, c,
                                                                                   J0, s, spin, T);
  return check_launch("rdm T slab");
}

__global__ void k_rdm_assemble(int norb, const double* __restrict__ G, const double* __restrict__ d1,
                               double* dm2) {
  const int n = norb, n2 = n * n;
  long long tot = (long long)n2 * n2;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    int p = (int)(t / ((long long)n * n2));
    int q = (int)((t / n2) % n);
    int r = (int)((t / n) % n);
    int s = (int)(t % n);
    double v = G[(long long)(q * n + p) * n2 + r * n + s];
    if (q == r) v -= d1[s * n + p];
    dm2[t] = v;
  }
}

// spin-resolved assembly: dm2[p][q][r][s] = G[(qp)][(rs)] - d_qr d1[p][s]
// (same-spin blocks) or G[(qp)][(rs)] (alpha-beta block, d1 == NULL)
__global__ void k_rdm_assemble_s(int norb, const double* __restrict__ G, const double* __restrict__ d1,
                                 double* dm2) {
  const int n = norb, n2 = n * n;
  long long tot = (long long)n2 * n2;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    int p = (int)(t / ((long long)n * n2));
    int q = (int)((t / n2) % n);
    int r = (int)((t / n) % n);
    int s = (int)(t % n);
    double v = G[(long long)(q * n + p) * n2 + r * n + s];
    if (d1 && q == r) v -= d1[p * n + s];
    dm2[t] = v;
  }
}

// <E_xy> from the Gram of the 2-RDM: sum_r <E_xy E_rr> = <E_xy N> = N <E_xy>
// (bra and ket both have N electrons of the spin the Gram is taken over),
// so d1t[x][y] = (1/N) sum_r G[(y,x)][(r,r)] without another pass over T
__global__ void k_d1_from_gram(int norb, const double* __restrict__ G, double inv_n, double* d1t) {
  const int n = norb, n2 = n * n;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += gridDim.x * blockDim.x) {
    const int x = t / n, y = t - x * n;
    const double* row = G + (long long)(y * n + x) * n2;
    double acc = 0.0;
    for (int r = 0; r < n; ++r) acc += row[r * n + r];
    d1t[t] = acc * inv_n;
  }
}

__global__ void k_transpose_small(int n, const double* in, double* out) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n * n; t += gridDim.x * blockDim.x) {
    int i = t / n, j = t - i * n;
    out[j * n + i] = in[t];
  }
}

}  // namespace csffci

using namespace csffci;

extern "C" {

int csffci_gram(int nx, const double* x, int64_t ldx, int ny, const double* y, int64_t ldy,
                int64_t n, double* out, void* work, size_t work_bytes, cudaStream_t stream) {
  CSF_REQUIRE(nx >= 0 && ny >= 0 && n >= 0, "gram: bad sizes");
  if (nx == 0 || ny == 0) return CSFFCI_OK;
  size_t need = csffci_gram_workspace(nx, ny, n);
  if (work == nullptr || work_bytes < need) {
    set_error("gram: workspace of %zu bytes < %zu required", work_bytes, need);
    return CSFFCI_ERR_MEMORY;
  }
  if (gram_skinny_fits(nx, ny)) return gram_skinny_run(nx, x, ldx, ny, y, ldy, n, out, (double*)work, stream);
  return gram_run(nx, x, ldx, ny, y, ldy, n, out, 0, (double*)work, stream);
}

size_t csffci_gram_workspace(int nx, int ny, int64_t n) {
  return gram_skinny_fits(nx, ny) ? gram_skinny_workspace(nx, ny, n) : gram_workspace(nx, ny, n);
}

size_t csffci_rdm12_workspace(int norb, int neleca, int nelecb) {
  long long ndet = (long long)(host_binom(norb, neleca) * host_binom(norb, nelecb));
  long long n2 = (long long)norb * norb;
  long long S = ndet < (1ll << 18) ? ndet : (1ll << 18);
  if (S < 1) S = 1;
  size_t t = (size_t)(2 * S * n2) * sizeof(double);
  size_t g = (size_t)(n2 * n2 + 2 * n2) * sizeof(double);
  size_t part = gram_workspace((int)n2, (int)n2, S);
  size_t partd = gram_dmma_workspace((int)n2, (int)n2, S);
  size_t part1 = gram_workspace(1, (int)n2, S);
  if (partd > part) part = partd;
  return t + g + (part > part1 ? part : part1) + 1024;
}

int csffci_rdm12(int norb, int neleca, int nelecb, const csffci_link_t* link_a,
                 const csffci_link_t* link_b, const double* bra, const double* ket, double* dm1,
                 double* dm2, void* work, size_t work_bytes, cudaStream_t stream) {
  CSF_REQUIRE(norb >= 1 && norb <= 22, "rdm12: norb=%d outside [1,22]", norb);
  long long Na = (long long)host_binom(norb, neleca), Nb = (long long)host_binom(norb, nelecb);
  long long ndet = Na * Nb;
  int n2 = norb * norb;
  int nla = neleca * (norb - neleca + 1), nlb = nelecb * (norb - nelecb + 1);
  size_t need = csffci_rdm12_workspace(norb, neleca, nelecb);
  if (work == nullptr || work_bytes < need) {
    set_error("rdm12: workspace of %zu bytes < %zu required", work_bytes, need);
    return CSFFCI_ERR_MEMORY;
  }
  long long S = ndet < (1ll << 18) ? ndet : (1ll << 18);
  double* Tk = (double*)work;
  double* Tb = Tk + (size_t)S * n2;
  double* G = Tb + (size_t)S * n2;
  double* d1t = G + (size_t)n2 * n2;
  double* part = d1t + 2 * (size_t)n2;
  const bool same = (bra == ket);
  int st;
  for (long long J0 = 0; J0 < ndet; J0 += S) {
    long long s = (ndet - J0 < S) ? ndet - J0 : S;
    const int accumulate = J0 > 0;
    for (int which = 0; which < (same ? 1 : 2); ++which) {
      double* T = which == 0 ? Tk : Tb;
      const double* c = which == 0 ? ket : bra;
      if ((st = tslab_tile_launch(norb, Nb, nla, nlb, link_a, link_b, c, J0, s, 2, T, stream))) return st;
    }
    const double* TB = same ? Tk : Tb;
    if (dm2) {
      if ((st = gram_dmma_run(n2, TB, s, n2, Tk, s, s, G, accumulate, part, stream))) return st;
    } else {
      // d1t[qp] = sum_J bra_J Tk[qp][J]  -> dm1[p][q] after the transpose
      if ((st = gram_run(1, bra + J0, s, n2, Tk, s, s, d1t, accumulate, part, stream))) return st;
    }
  }
  if (dm2) {
    const int ne = neleca + nelecb;
    k_d1_from_gram<<<grid_for(n2, 256), 256, 0, stream>>>(norb, G, ne > 0 ? 1.0 / ne : 0.0, d1t);
    if ((st = check_launch("rdm1 from the Gram"))) return st;
  }
  k_transpose_small<<<grid_for(n2, 256), 256, 0, stream>>>(norb, d1t, dm1);
  if ((st = check_launch("rdm1 transpose"))) return st;
  if (dm2) {
    k_rdm_assemble<<<grid_for((long long)n2 * n2, 256, 148 * 8), 256, 0, stream>>>(norb, G, dm1, dm2);
    return check_launch("rdm2 assemble");
  }
  return CSFFCI_OK;
}

static long long rdm12s_slab(long long ndet) {
  long long S = ndet < (1ll << 17) ? ndet : (1ll << 17);
  return S < 1 ? 1 : S;
}

size_t csffci_rdm12s_workspace(int norb, int neleca, int nelecb) {
  long long ndet = (long long)(host_binom(norb, neleca) * host_binom(norb, nelecb));
  long long n2 = (long long)norb * norb;
  long long S = rdm12s_slab(ndet);
  size_t t = (size_t)(4 * S * n2) * sizeof(double);
  size_t g = (size_t)(3 * n2 * n2 + 4 * n2) * sizeof(double);
  size_t part = gram_workspace((int)n2, (int)n2, S);
  size_t partd = gram_dmma_workspace((int)n2, (int)n2, S);
  size_t part1 = gram_workspace(1, (int)n2, S);
  if (partd > part) part = partd;
  return t + g + (part > part1 ? part : part1) + 1024;
}

int csffci_rdm12s(int norb, int neleca, int nelecb, const csffci_link_t* link_a,
                  const csffci_link_t* link_b, const double* bra, const double* ket, double* dm1a,
                  double* dm1b, double* dm2aa, double* dm2ab, double* dm2bb, void* work,
                  size_t work_bytes, cudaStream_t stream) {
  CSF_REQUIRE(norb >= 1 && norb <= 22, "rdm12s: norb=%d outside [1,22]", norb);
  CSF_REQUIRE(dm1a && dm1b && bra && ket, "rdm12s: NULL argument");
  CSF_REQUIRE((dm2aa == nullptr) == (dm2ab == nullptr) && (dm2ab == nullptr) == (dm2bb == nullptr),
              "rdm12s: the three 2-RDM blocks are all given or all NULL");
  long long Na = (long long)host_binom(norb, neleca), Nb = (long long)host_binom(norb, nelecb);
  long long ndet = Na * Nb;
  int n2 = norb * norb;
  int nla = neleca * (norb - neleca + 1), nlb = nelecb * (norb - nelecb + 1);
  size_t need = csffci_rdm12s_workspace(norb, neleca, nelecb);
  if (work == nullptr || work_bytes < need) {
    set_error("rdm12s: workspace of %zu bytes < %zu required", work_bytes, need);
    return CSFFCI_ERR_MEMORY;
  }
  const long long S = rdm12s_slab(ndet);
  double* Tka = (double*)work;  // <J|E^alpha_pq|ket>
  double* Tkb = Tka + (size_t)S * n2;
  double* Tba = Tkb + (size_t)S * n2;  // the same for bra
  double* Tbb = Tba + (size_t)S * n2;
  double* Gaa = Tbb + (size_t)S * n2;
  double* Gab = Gaa + (size_t)n2 * n2;
  double* Gbb = Gab + (size_t)n2 * n2;
  double* d1at = Gbb + (size_t)n2 * n2;
  double* d1bt = d1at + n2;
  double* part = d1bt + 2 * (size_t)n2;
  const bool same = (bra == ket);
  const bool two = dm2aa != nullptr;
  int st;
  for (long long J0 = 0; J0 < ndet; J0 += S) {
    const long long s = (ndet - J0 < S) ? ndet - J0 : S;
    const int accumulate = J0 > 0;
    for (int which = 0; which < (same ? 1 : 2); ++which) {
      const double* c = which == 0 ? ket : bra;
      double* Ta = which == 0 ? Tka : Tba;
      double* Tb = which == 0 ? Tkb : Tbb;
      if ((st = tslab_tile_launch(norb, Nb, nla, nlb, link_a, link_b, c, J0, s, 0, Ta, stream))) return st;
      if ((st = tslab_tile_launch(norb, Nb, nla, nlb, link_a, link_b, c, J0, s, 1, Tb, stream))) return st;
    }
    const double* BA = same ? Tka : Tba;
    const double* BB = same ? Tkb : Tbb;
    if (two) {
      if ((st = gram_dmma_run(n2, BA, s, n2, Tka, s, s, Gaa, accumulate, part, stream))) return st;
      if ((st = gram_dmma_run(n2, BA, s, n2, Tkb, s, s, Gab, accumulate, part, stream))) return st;
      if ((st = gram_dmma_run(n2, BB, s, n2, Tkb, s, s, Gbb, accumulate, part, stream))) return st;
    } else {
      if ((st = gram_run(1, bra + J0, s, n2, Tka, s, s, d1at, accumulate, part, stream))) return st;
      if ((st = gram_run(1, bra + J0, s, n2, Tkb, s, s, d1bt, accumulate, part, stream))) return st;
    }
  }
  if (two) {
    // same-spin Grams: sum_r <E^s_xy E^s_rr> = N_s <E^s_xy>
    k_d1_from_gram<<<grid_for(n2, 256), 256, 0, stream>>>(norb, Gaa, neleca > 0 ? 1.0 / neleca : 0.0, d1at);
    if ((st = check_launch("rdm1a from the Gram"))) return st;
    k_d1_from_gram<<<grid_for(n2, 256), 256, 0, stream>>>(norb, Gbb, nelecb > 0 ? 1.0 / nelecb : 0.0, d1bt);
    if ((st = check_launch("rdm1b from the Gram"))) return st;
  }
  k_transpose_small<<<grid_for(n2, 256), 256, 0, stream>>>(norb, d1at, dm1a);
  if ((st = check_launch("rdm1a transpose"))) return st;
  k_transpose_small<<<grid_for(n2, 256), 256, 0, stream>>>(norb, d1bt, dm1b);
  if ((st = check_launch("rdm1b transpose"))) return st;
  if (two) {
    const int g = grid_for((long long)n2 * n2, 256, 148 * 8);
    // same-spin: <p+ r+ s q> = <E_pq E_rs> - d_qr <p+ s> = ... - d_qr dm1[s][p]
    k_rdm_assemble_s<<<g, 256, 0, stream>>>(norb, Gaa, d1at, dm2aa);
    if ((st = check_launch("rdm2aa assemble"))) return st;
    k_rdm_assemble_s<<<g, 256, 0, stream>>>(norb, Gab, nullptr, dm2ab);
    if ((st = check_launch("rdm2ab assemble"))) return st;
    k_rdm_assemble_s<<<g, 256, 0, stream>>>(norb, Gbb, d1bt, dm2bb);
    return check_launch("rdm2bb assemble");
  }
  return CSFFCI_OK;
}

}  // extern "C"
