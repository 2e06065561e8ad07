// det <-> CSF transforms and the CSF diagonal.
//
// Per npair block the reference gathers x[:, csd_mask block] into a
// (nvec*nconf, ndet) matrix, multiplies it by +-umat and scatters into the CSF
// vector (pyscf/csf_fci/csfstring.py:641-658).  Here each block is one tiled
// FP64 GEMM whose A-operand loader performs the csd_mask gather (det->CSF)
// and whose store performs the csd_mask scatter (CSF->det); csd_mask is a
// permutation, so the scatter has no conflicts.  HBM-bound: every CI element
// is read once and written once per call.
#include "common.cuh"
#include "profile.cuh"

namespace csffci {

enum { MODE_DET2CSF = 0, MODE_CSF2DET = 1 };

struct BlockGemmArgs {
  const double* x;
  double* y;
  int64_t ldx, ldy;
  const uint32_t* mask;
  const double* umat;
  int64_t csd_off, csf_off, nconf;
  const int32_t* conf_sel;  // selected configurations (point-group symmetry) or NULL
  int ndet, ncsf;
  int nvec;
  double sign;
};

constexpr int TBM = 64, TBN = 64, TBK = 16;

template <int MODE>
__global__ void __launch_bounds__(256) k_block_gemm(BlockGemmArgs g) {
  __shared__ double As[TBK][TBM + 1];
  __shared__ double Bs[TBK][TBN + 1];
  const int64_t M = (int64_t)g.nvec * g.nconf;
  const int N = (MODE == MODE_DET2CSF) ? g.ncsf : g.ndet;
  const int K = (MODE == MODE_DET2CSF) ? g.ndet : g.ncsf;
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int64_t ntile_m = (M + TBM - 1) / TBM;
  const int ntile_n = (N + TBN - 1) / TBN;
  for (int64_t tile = blockIdx.x; tile < ntile_m * ntile_n; tile += gridDim.x) {
    const int64_t m0 = (tile / ntile_n) * TBM;
    const int n0 = (int)(tile % ntile_n) * TBN;
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
    for (int k0 = 0; k0 < K; k0 += TBK) {
      // A tile: 64 rows x 16 k; thread loads (row = tid/16 + 16*r, k = tid%16)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        int row = ty + 16 * r;
        int kk = tx;
        int64_t m = m0 + row;
        double v = 0.0;
        if (m < M && k0 + kk < K) {
          int64_t vec = m / g.nconf, conf = m - vec * g.nconf;
          if (MODE == MODE_DET2CSF) {
            const int64_t cf = g.conf_sel ? g.conf_sel[conf] : conf;
            uint32_t d = g.mask[g.csd_off + cf * g.ndet + k0 + kk];
            v = g.x[vec * g.ldx + d];
          } else {
            v = g.x[vec * g.ldx + g.csf_off + conf * g.ncsf + k0 + kk];
          }
        }
        As[kk][row] = v;
      }
      // B tile: 16 k x 64 n
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        double v = 0.0;
        if (MODE == MODE_DET2CSF) {
          int kk = ty, col = tx + 16 * r;
          if (k0 + kk < K && n0 + col < N) v = g.umat[(int64_t)(k0 + kk) * g.ncsf + n0 + col];
          Bs[kk][col] = v;
        } else {
          int kk = tx, col = ty + 16 * r;
          if (k0 + kk < K && n0 + col < N) v = g.umat[(int64_t)(n0 + col) * g.ncsf + k0 + kk];
          Bs[kk][col] = v;
        }
      }
      __syncthreads();
#pragma unroll
      for (int kk = 0; kk < TBK; ++kk) {
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
      }
      __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int64_t m = m0 + ty * 4 + i;
      if (m >= M) continue;
      int64_t vec = m / g.nconf, conf = m - vec * g.nconf;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int n = n0 + tx * 4 + j;
        if (n >= N) continue;
        double v = g.sign * acc[i][j];
        if (MODE == MODE_DET2CSF) {
          g.y[vec * g.ldy + g.csf_off + conf * g.ncsf + n] = v;
        } else {
          const int64_t cf = g.conf_sel ? g.conf_sel[conf] : conf;
          uint32_t d = g.mask[g.csd_off + cf * g.ndet + n];
          g.y[vec * g.ldy + d] = v;
        }
      }
    }
  }
}

// Blocks with few determinants and CSFs per configuration (at CAS(16,16)
// the npair >= 3 blocks: at most 252 determinants and 42 CSFs, 98 % of the
// configurations and 70 % of the determinants) make poor 64x64 GEMM tiles:
// N = ncsf and K = ndet are far below the tile, so most of the tile's work
// is padding.  Here one thread takes one (vector, configuration): the
// block's umat sits in shared memory (every thread of a warp reads the same
// element, a broadcast), and the configuration's gathered determinant
// values (det->CSF) or its CSF coefficients (CSF->det) meet it in
// registers.  The sums run over the determinants (det->CSF) or the CSFs
// (CSF->det) in ascending order with the same fused multiply-adds as the
// GEMM path, so both give the same bits.
constexpr int SMALL_MAX_NCSF = 48;
constexpr size_t SMALL_MAX_UMAT_BYTES = 96 * 1024;

template <int MODE, int NC>
__global__ void __launch_bounds__(256) k_block_small(BlockGemmArgs g) {
  extern __shared__ double Us[];  // umat [ndet][ncsf]
  const int nd = g.ndet, nc = g.ncsf;
  for (int i = threadIdx.x; i < nd * nc; i += blockDim.x) Us[i] = g.umat[i];
  __syncthreads();
  const int64_t M = (int64_t)g.nvec * g.nconf;
  for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < M;
       m += (int64_t)gridDim.x * blockDim.x) {
    const int64_t vec = m / g.nconf, conf = m - vec * g.nconf;
    const int64_t cf = g.conf_sel ? g.conf_sel[conf] : conf;
    const uint32_t* mk = g.mask + g.csd_off + cf * nd;
    if (MODE == MODE_DET2CSF) {
      double acc[NC];
#pragma unroll
      for (int k = 0; k < NC; ++k) acc[k] = 0.0;
      const double* xv = g.x + vec * g.ldx;
      for (int x = 0; x < nd; ++x) {
        const double v = xv[mk[x]];
        const double* u = Us + x * nc;
#pragma unroll
        for (int k = 0; k < NC; ++k)
          if (k < nc) acc[k] = fma(v, u[k], acc[k]);
      }
      double* yo = g.y + vec * g.ldy + g.csf_off + conf * nc;
#pragma unroll
      for (int k = 0; k < NC; ++k)
        if (k < nc) yo[k] = g.sign * acc[k];
    } else {
      double cin[NC];
      const double* xi = g.x + vec * g.ldx + g.csf_off + conf * nc;
#pragma unroll
      for (int k = 0; k < NC; ++k) cin[k] = k < nc ? xi[k] : 0.0;
      double* yv = g.y + vec * g.ldy;
      for (int x = 0; x < nd; ++x) {
        const double* u = Us + x * nc;
        double sacc = 0.0;
#pragma unroll
        for (int k = 0; k < NC; ++k)
          if (k < nc) sacc = fma(cin[k], u[k], sacc);
        yv[mk[x]] = g.sign * sacc;
      }
    }
  }
}

// profiler names per npair block (kernel timing by block)
static const char* block_kernel_name(bool small, int npair) {
  static const char* sm[9] = {"k_block_small_np0", "k_block_small_np1", "k_block_small_np2", "k_block_small_np3",
                              "k_block_small_np4", "k_block_small_np5", "k_block_small_np6", "k_block_small_np7",
                              "k_block_small_np8+"};
  static const char* gm[9] = {"k_block_gemm_np0", "k_block_gemm_np1", "k_block_gemm_np2", "k_block_gemm_np3",
                              "k_block_gemm_np4", "k_block_gemm_np5", "k_block_gemm_np6", "k_block_gemm_np7",
                              "k_block_gemm_np8+"};
  const int i = npair < 0 ? 0 : npair > 8 ? 8 : npair;
  return small ? sm[i] : gm[i];
}

template <int MODE, int NC>
static int launch_small(const BlockGemmArgs& g, cudaStream_t stream, int npair) {
  const size_t smem = (size_t)g.ndet * g.ncsf * sizeof(double);
  auto kern = k_block_small<MODE, NC>;
  if (smem > 48 * 1024) CSF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t M = (int64_t)g.nvec * g.nconf;
  {
    ProfScope ps_(block_kernel_name(true, npair), stream);
    kern<<<grid_for(M, 256, 148 * 8), 256, smem, stream>>>(g);
  }
  return check_launch("det/csf transform (small blocks)");
}

template <int MODE>
static int run_small(const BlockGemmArgs& g, cudaStream_t stream, int npair) {
  if (g.ncsf <= 2) return launch_small<MODE, 2>(g, stream, npair);
  if (g.ncsf <= 8) return launch_small<MODE, 8>(g, stream, npair);
  if (g.ncsf <= 16) return launch_small<MODE, 16>(g, stream, npair);
  if (g.ncsf <= 32) return launch_small<MODE, 32>(g, stream, npair);
  return launch_small<MODE, SMALL_MAX_NCSF>(g, stream, npair);
}

static bool small_block(const csffci_block_t& B) {
  return B.ncsf <= SMALL_MAX_NCSF && (size_t)B.ndet * B.ncsf * sizeof(double) <= SMALL_MAX_UMAT_BYTES &&
         B.ndet <= 256;
}

// det -> CSF blocks with few (vector, configuration) rows and a long K (at
// CAS(16,16) npair 0: 1 configuration x 12870 determinants x 1430 CSFs, and
// npair 1: 240 x 3432 x 429): the 64 x 64 GEMM tiles leave most SMs idle
// and walk K alone.  Here a CTA takes 16 rows x 32 CSF columns and its 8
// warps split K: the rows' gathered determinant values are staged in shared
// memory a chunk of K at a time (coalesced mask reads, independent
// gathers), each lane keeps the 16 sums of its column, and the 8 warp
// partials are added in a fixed order at the end.
constexpr int TK_M = 16, TK_N = 32, TK_KC = 512, TK_W = 8;

constexpr size_t TK_SMEM = (size_t)TK_M * TK_KC * sizeof(double);  // 64 KB (dynamic)
static_assert((size_t)TK_W * TK_M * (TK_N + 1) * sizeof(double) <= TK_SMEM, "the partials reuse the chunk buffer");

__global__ void __launch_bounds__(TK_W * 32) k_block_tallk(BlockGemmArgs g) {
  extern __shared__ double tk_smem[];
  double (*Xs)[TK_KC] = reinterpret_cast<double (*)[TK_KC]>(tk_smem);              // gathered chunk
  double (*Ps)[TK_M][TK_N + 1] = reinterpret_cast<double (*)[TK_M][TK_N + 1]>(tk_smem);  // warp partials
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t M = (int64_t)g.nvec * g.nconf;
  const int N = g.ncsf, K = g.ndet;
  const int ntn = (N + TK_N - 1) / TK_N;
  const int64_t ntiles = ((M + TK_M - 1) / TK_M) * ntn;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t m0 = (tile / ntn) * TK_M;
    const int n0 = (int)(tile % ntn) * TK_N;
    const int n = n0 + lane;
    double acc[TK_M];
#pragma unroll
    for (int i = 0; i < TK_M; ++i) acc[i] = 0.0;
    for (int k0 = 0; k0 < K; k0 += TK_KC) {
      const int kc = min(TK_KC, K - k0);
      __syncthreads();  // the previous chunk is consumed
      for (int e = tid; e < TK_M * TK_KC; e += TK_W * 32) {
        const int r = e / TK_KC, kk = e - r * TK_KC;
        const int64_t m = m0 + r;
        double v = 0.0;
        if (m < M && kk < kc) {
          const int64_t vec = m / g.nconf, conf = m - vec * g.nconf;
          const int64_t cf = g.conf_sel ? g.conf_sel[conf] : conf;
          v = g.x[vec * g.ldx + g.mask[g.csd_off + cf * g.ndet + k0 + kk]];
        }
        Xs[r][kk] = v;
      }
      __syncthreads();
      const int kw = (kc + TK_W - 1) / TK_W;  // k per warp in this chunk
      const int kb = warp * kw, ke = min(kc, kb + kw);
      if (n < N)
        for (int kk = kb; kk < ke; ++kk) {
          const double u = g.umat[(int64_t)(k0 + kk) * N + n];
#pragma unroll
          for (int i = 0; i < TK_M; ++i) acc[i] = fma(Xs[i][kk], u, acc[i]);
        }
    }
    __syncthreads();  // every warp is done with the last chunk (Ps overlays Xs)
#pragma unroll
    for (int i = 0; i < TK_M; ++i) Ps[warp][i][lane] = acc[i];
    __syncthreads();
    for (int e = tid; e < TK_M * TK_N; e += TK_W * 32) {
      const int i = e / TK_N, j = e - i * TK_N;
      const int64_t m = m0 + i;
      if (m >= M || n0 + j >= N) continue;
      double v = 0.0;
#pragma unroll
      for (int w = 0; w < TK_W; ++w) v += Ps[w][i][j];
      const int64_t vec = m / g.nconf, conf = m - vec * g.nconf;
      g.y[vec * g.ldy + g.csf_off + conf * N + n0 + j] = g.sign * v;
    }
  }
}

__global__ void k_zero_rows(double* y, int64_t ldy, int nvec, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)nvec * n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t v = i / n;
    y[v * ldy + (i - v * n)] = 0.0;
  }
}

template <int MODE>
static int run_blocks(int nvec, const double* x, int64_t ldx, double* y, int64_t ldy,
                      const uint32_t* mask, const csffci_block_t* blocks, int nblock,
                      cudaStream_t stream) {
  for (int b = 0; b < nblock; ++b) {
    const csffci_block_t& B = blocks[b];
    if (B.ncsf == 0 || B.nconf == 0) continue;
    CSF_REQUIRE(B.umat != nullptr, "transform: block %d has no umat", b);
    BlockGemmArgs g;
    g.x = x;
    g.y = y;
    g.ldx = ldx;
    g.ldy = ldy;
    g.mask = mask;
    g.umat = B.umat;
    g.csd_off = B.csd_offset;
    g.csf_off = B.csf_offset;
    g.nconf = B.nconf;
    g.conf_sel = B.conf_sel;
    g.ndet = B.ndet;
    g.ncsf = B.ncsf;
    g.nvec = nvec;
    g.sign = B.sign;
    if (small_block(B)) {
      const int st = run_small<MODE>(g, stream, B.npair);
      if (st) return st;
      continue;
    }
    int64_t M = (int64_t)nvec * B.nconf;
    int N = (MODE == MODE_DET2CSF) ? B.ncsf : B.ndet;
    int64_t tiles = ((M + TBM - 1) / TBM) * ((N + TBN - 1) / TBN);
    if (MODE == MODE_DET2CSF && tiles < 2 * 148 && B.ndet >= 4 * TK_KC) {
      // few GEMM tiles over a long K: the K-split kernel
      const int64_t tk = ((M + TK_M - 1) / TK_M) * ((N + TK_N - 1) / TK_N);
      CSF_CUDA(cudaFuncSetAttribute(k_block_tallk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TK_SMEM));
      {
        ProfScope ps_(block_kernel_name(false, B.npair), stream);
        k_block_tallk<<<grid_for(tk, 1, 148 * 3), TK_W * 32, TK_SMEM, stream>>>(g);
      }
      const int st = check_launch("det->CSF transform (long K)");
      if (st) return st;
      continue;
    }
    {
      ProfScope ps_(block_kernel_name(false, B.npair), stream);
      k_block_gemm<MODE><<<grid_for(tiles, 1, 148 * 8), 256, 0, stream>>>(g);
    }
    int st = check_launch("det/csf transform");
    if (st) return st;
  }
  return CSFFCI_OK;
}

// ---------------------------------------------------------------------------
// CSF diagonal: per configuration c and CSF k
//   hdiag_csf[c,k] = sum_x U[x,k]^2 hdiag_det[x] + sum_{a<b} K(S_a,S_b) Z[ab,k]
// which equals sum_xy U[x,k] H_xy U[y,k] over the within-configuration block
// of pyscf/lib/csf/csfstring.c:295-362 (H_xy = (-1)^(somos between)
// (pq|qp) for two dets that differ by exchanging the spins of SOMOs p,q);
// K(p,q) = (pq|qp) = eri[pq][pq].
// ---------------------------------------------------------------------------

struct HdiagCsfArgs {
  const double* hd;
  const double* eri;
  const uint32_t* mask;
  const double* umat;
  const double* zmat;
  double* out;
  int64_t csd_off, csf_off, nconf, sconf;
  const int32_t* conf_sel;
  int ndet, ncsf, nspin, npair, norb, npair_orb;
};

__global__ void k_hdiag_csf(HdiagCsfArgs g) {
  const int64_t n = g.nconf * g.ncsf;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t ic = i / g.ncsf;  // position in the (packed) CSF vector
    const int k = (int)(i - ic * g.ncsf);
    const int64_t conf = g.conf_sel ? g.conf_sel[ic] : ic;  // configuration within the block
    double acc = 0.0;
    const uint32_t* m = g.mask + g.csd_off + conf * g.ndet;
    for (int x = 0; x < g.ndet; ++x) {
      double u = g.umat[(int64_t)x * g.ncsf + k];
      acc = fma(u * u, g.hd[m[x]], acc);
    }
    if (g.nspin >= 2) {
      int64_t dc = conf / g.sconf, sc = conf - dc * g.sconf;
      unsigned long long dstr = str_unrank(g.norb, g.npair, (unsigned long long)dc);
      unsigned long long sstr = str_unrank(g.norb - g.npair, g.nspin, (unsigned long long)sc);
      int somo[64];
      int ns = 0, isorb = 0;
      for (int iorb = 0; iorb < g.norb; ++iorb) {
        if ((dstr >> iorb) & 1ull) continue;
        if ((sstr >> isorb) & 1ull) somo[ns++] = iorb;
        ++isorb;
      }
      int ab = 0;
      for (int b = 1; b < ns; ++b)
        for (int a = 0; a < b; ++a, ++ab) {
          int pq = pair_index(somo[a], somo[b]);
          acc = fma(g.eri[(int64_t)pq * g.npair_orb + pq], g.zmat[(int64_t)ab * g.ncsf + k], acc);
        }
    }
    g.out[g.csf_off + ic * g.ncsf + k] = acc;
  }
}

}  // namespace csffci

using namespace csffci;

extern "C" {

int csffci_det2csf(int nvec, const double* x_det, int64_t ld_det, double* x_csf, int64_t ld_csf,
                   const uint32_t* csd_mask, const csffci_block_t* blocks, int nblock,
                   cudaStream_t stream) {
  CSF_REQUIRE(nvec >= 0 && blocks != nullptr && nblock >= 0, "det2csf: bad arguments");
  if (nvec == 0) return CSFFCI_OK;
  return run_blocks<MODE_DET2CSF>(nvec, x_det, ld_det, x_csf, ld_csf, csd_mask, blocks, nblock,
                                  stream);
}

int csffci_csf2det(int nvec, const double* x_csf, int64_t ld_csf, double* x_det, int64_t ld_det,
                   int64_t ndet, const uint32_t* csd_mask, const csffci_block_t* blocks,
                   int nblock, cudaStream_t stream) {
  CSF_REQUIRE(nvec >= 0 && blocks != nullptr && nblock >= 0, "csf2det: bad arguments");
  if (nvec == 0) return CSFFCI_OK;
  // determinants of blocks without CSFs (and every other one, for
  // simplicity of the contract) start from zero
  bool full = true;
  for (int b = 0; b < nblock; ++b)
    if ((blocks[b].ncsf == 0 && blocks[b].nconf > 0) || blocks[b].conf_sel != nullptr) full = false;
  if (!full) {
    {
      ProfScope ps_("k_zero_rows", stream);
      k_zero_rows<<<grid_for((int64_t)nvec * ndet, 256, 148 * 16), 256, 0, stream>>>(x_det, ld_det,
                                                                                       nvec, ndet);
    }
    int st = check_launch("csf2det zero");
    if (st) return st;
  }
  return run_blocks<MODE_CSF2DET>(nvec, x_csf, ld_csf, x_det, ld_det, csd_mask, blocks, nblock,
                                  stream);
}

int csffci_hdiag_csf(int norb, int neleca, int nelecb, const double* hdiag_det, const double* eri,
                     const uint32_t* csd_mask, const csffci_block_t* blocks, int nblock,
                     double* hdiag_csf, cudaStream_t stream) {
  CSF_REQUIRE(norb >= 0 && norb <= 63 && blocks != nullptr, "hdiag_csf: bad arguments");
  int npair_orb = norb * (norb + 1) / 2;
  for (int b = 0; b < nblock; ++b) {
    const csffci_block_t& B = blocks[b];
    if (B.ncsf == 0 || B.nconf == 0) continue;
    CSF_REQUIRE(B.umat != nullptr, "hdiag_csf: block %d has no umat", b);
    CSF_REQUIRE(B.nspin < 2 || B.zmat != nullptr, "hdiag_csf: block %d has no zmat", b);
    HdiagCsfArgs g;
    g.hd = hdiag_det;
    g.eri = eri;
    g.mask = csd_mask;
    g.umat = B.umat;
    g.zmat = B.zmat;
    g.out = hdiag_csf;
    g.csd_off = B.csd_offset;
    g.csf_off = B.csf_offset;
    g.nconf = B.nconf;
    g.conf_sel = B.conf_sel;
    g.sconf = (int64_t)host_binom(norb - B.npair, B.nspin);
    g.ndet = B.ndet;
    g.ncsf = B.ncsf;
    g.nspin = B.nspin;
    g.npair = B.npair;
    g.norb = norb;
    g.npair_orb = npair_orb;
    {
      ProfScope ps_("k_hdiag_csf", stream);
      k_hdiag_csf<<<grid_for(B.nconf * B.ncsf, 128, 148 * 32), 128, 0, stream>>>(g);
    }
    int st = check_launch("hdiag_csf");
    if (st) return st;
  }
  return CSFFCI_OK;
}

}  // extern "C"
