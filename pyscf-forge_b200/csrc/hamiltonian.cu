// Hamiltonian building blocks: absorb_h1e, the determinant diagonal, the
// p-space Slater-Condon block and the one-electron contraction.
#include <mutex>

#include "common.cuh"
#include "profile.cuh"

namespace csffci {

// f(j,k) = (h1e[j][k] - 1/2 sum_i (ji|ik)) / nelec, evaluated on the fly
__device__ __forceinline__ double absorb_f(int norb, int npair, const double* h1e,
                                           const double* eri, double inv_n, int j, int k) {
  double s = 0.0;
  for (int i = 0; i < norb; ++i) s += eri[(int64_t)pair_index(j, i) * npair + pair_index(i, k)];
  return (h1e[j * norb + k] - 0.5 * s) * inv_n;
}

__device__ __forceinline__ void unpair(int pq, int* p, int* q) {
  int h = (int)((sqrt(8.0 * pq + 1.0) - 1.0) * 0.5);
  while (h * (h + 1) / 2 > pq) --h;
  while ((h + 1) * (h + 2) / 2 <= pq) ++h;
  *p = h;
  *q = pq - h * (h + 1) / 2;
}

// h2e[pq][rs] = fac*(eri[pq][rs] + delta_pq f[r][s] + delta_rs f[p][q]),
// pair (p,q) with p >= q
__global__ void k_absorb_h2e(int norb, int npair, const double* h1e, const double* eri,
                             double inv_n, double fac, double* h2e) {
  int64_t n = (int64_t)npair * npair;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    int pq = (int)(t / npair), rs = (int)(t - (int64_t)pq * npair);
    int p, q, r, s;
    unpair(pq, &p, &q);
    unpair(rs, &r, &s);
    double v = eri[t];
    if (p == q) v += absorb_f(norb, npair, h1e, eri, inv_n, r, s);
    if (r == s) v += absorb_f(norb, npair, h1e, eri, inv_n, p, q);
    h2e[t] = v * fac;
  }
}

// per-string pieces of the determinant diagonal:
//   e1[I] = sum_{i in I} h[i][i] + 1/2 sum_{i,j in I} (J_ij - K_ij)
//   jv[I][q] = sum_{i in I} J_iq          (only for the alpha strings)
// with J_ij = (ii|jj) = eri[ii][jj], K_ij = (ij|ji) = eri[ij][ij].
__global__ void k_string_energy(int norb, int nelec, int npair, unsigned long long nstr,
                                const double* h, const double* eri, double* e1, double* jv,
                                uint64_t* strs_out) {
  for (unsigned long long I = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; I < nstr;
       I += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned long long s = str_unrank(norb, nelec, I);
    if (strs_out) strs_out[I] = s;
    double e = 0.0;
    for (int i = 0; i < norb; ++i) {
      if (!((s >> i) & 1ull)) continue;
      e += h[i * norb + i];
      int ii = pair_index(i, i);
      for (int j = 0; j < norb; ++j) {
        if (!((s >> j) & 1ull)) continue;
        int jj = pair_index(j, j), ij = pair_index(i, j);
        e += 0.5 * (eri[(int64_t)ii * npair + jj] - eri[(int64_t)ij * npair + ij]);
      }
    }
    e1[I] = e;
    if (jv) {
      for (int q = 0; q < norb; ++q) {
        int qq = pair_index(q, q);
        double acc = 0.0;
        for (int i = 0; i < norb; ++i)
          if ((s >> i) & 1ull) acc += eri[(int64_t)pair_index(i, i) * npair + qq];
        jv[I * norb + q] = acc;
      }
    }
  }
}

__global__ void k_hdiag_det(int norb, unsigned long long Na, unsigned long long Nb,
                            const double* __restrict__ ea, const double* __restrict__ eb,
                            const double* __restrict__ ja, const uint64_t* __restrict__ sb,
                            double* hdiag) {
  unsigned long long n = Na * Nb;
  for (unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; t < n;
       t += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned long long ia = t / Nb, ib = t - ia * Nb;
    unsigned long long s = sb[ib];
    const double* j = ja + ia * norb;
    double v = ea[ia] + eb[ib];
    while (s) {
      int q = __ffsll((long long)s) - 1;
      s &= s - 1;
      v += j[q];
    }
    hdiag[t] = v;
  }
}

// ---------------------------------------------------------------------------
// Slater-Condon matrix elements <a1 b1|H|a2 b2> for distinct determinants
// ---------------------------------------------------------------------------
__device__ __forceinline__ double eri_at(const double* eri, int npair, int p, int q, int r, int s) {
  return eri[(int64_t)pair_index(p, q) * npair + pair_index(r, s)];
}

__device__ __forceinline__ int between_sign(unsigned long long s, int p, int q) {
  int hi = p > q ? p : q, lo = p > q ? q : p;
  unsigned long long mask = (1ull << hi) - (1ull << (lo + 1));
  return (__popcll(s & mask) & 1) ? -1 : 1;
}

__device__ double sc_element(int norb, int npair, const double* ha, const double* hb,
                             const double* eri, unsigned long long a1, unsigned long long b1,
                             unsigned long long a2, unsigned long long b2) {
  unsigned long long da = a1 ^ a2, db = b1 ^ b2;
  int nxa = __popcll(da) / 2, nxb = __popcll(db) / 2;
  if (nxa + nxb > 2) return 0.0;
  if (nxa + nxb == 1) {
    bool alpha = nxa == 1;
    unsigned long long sf = alpha ? a2 : b2, st = alpha ? a1 : b1, so = alpha ? b2 : a2;
    const double* h = alpha ? ha : hb;
    int q = __ffsll((long long)(sf & ~st)) - 1;
    int p = __ffsll((long long)(st & ~sf)) - 1;
    double v = h[p * norb + q];
    unsigned long long k = sf;
    while (k) {
      int kk = __ffsll((long long)k) - 1;
      k &= k - 1;
      v += eri_at(eri, npair, p, q, kk, kk) - eri_at(eri, npair, p, kk, kk, q);
    }
    k = so;
    while (k) {
      int kk = __ffsll((long long)k) - 1;
      k &= k - 1;
      v += eri_at(eri, npair, p, q, kk, kk);
    }
    return between_sign(sf, p, q) * v;
  }
  if (nxa == 1 && nxb == 1) {
    int q = __ffsll((long long)(a2 & ~a1)) - 1, p = __ffsll((long long)(a1 & ~a2)) - 1;
    int s = __ffsll((long long)(b2 & ~b1)) - 1, r = __ffsll((long long)(b1 & ~b2)) - 1;
    return between_sign(a2, p, q) * between_sign(b2, r, s) * eri_at(eri, npair, p, q, r, s);
  }
  // double excitation within one spin
  unsigned long long sf = nxa == 2 ? a2 : b2, st = nxa == 2 ? a1 : b1;
  unsigned long long qs = sf & ~st, ps = st & ~sf;
  int q1 = __ffsll((long long)qs) - 1;
  int q2 = 63 - __clzll((long long)qs);
  int p1 = __ffsll((long long)ps) - 1;
  int p2 = 63 - __clzll((long long)ps);
  int sgn = between_sign(sf, p1, q1);
  unsigned long long mid = (sf ^ (1ull << q1)) | (1ull << p1);
  sgn *= between_sign(mid, p2, q2);
  return sgn * (eri_at(eri, npair, p1, q1, p2, q2) - eri_at(eri, npair, p1, q2, p2, q1));
}

__global__ void k_pspace_h0(int norb, int npair, unsigned long long Nb, const double* ha,
                            const double* hb, const double* eri, const double* hd,
                            const uint32_t* addr, int neleca, int nelecb, int n, double* h0) {
  int64_t tot = (int64_t)n * n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot;
       t += (int64_t)gridDim.x * blockDim.x) {
    int i = (int)(t / n), j = (int)(t - (int64_t)i * n);
    double v;
    if (i == j) {
      v = hd[addr[i]];
    } else {
      unsigned long long ai = addr[i] / Nb, bi = addr[i] - ai * Nb;
      unsigned long long aj = addr[j] / Nb, bj = addr[j] - aj * Nb;
      v = sc_element(norb, npair, ha, hb, eri, str_unrank(norb, neleca, ai),
                     str_unrank(norb, nelecb, bi), str_unrank(norb, neleca, aj),
                     str_unrank(norb, nelecb, bj));
    }
    h0[t] = v;
  }
}

// sigma[K] += sum over links of K: s * h[i][a] * c[target]  (gather form of
// sum_pq h_pq E_pq c; one thread owns one output element)
__global__ void k_contract_1e(int norb, unsigned long long Na, unsigned long long Nb, int nla,
                              int nlb, const double* __restrict__ ha, const double* __restrict__ hb,
                              const csffci_link_t* __restrict__ la,
                              const csffci_link_t* __restrict__ lb, const double* __restrict__ ci,
                              double* sigma) {
  unsigned long long n = Na * Nb;
  for (unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; t < n;
       t += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned long long ka = t / Nb, kb = t - ka * Nb;
    double acc = 0.0;
    const csffci_link_t* L = la + ka * nla;
    for (int l = 0; l < nla; ++l) {
      csffci_link_t e = L[l];
      int a = e.op & 0xff, i = e.op >> 8;
      acc += e.sign * ha[i * norb + a] * ci[(unsigned long long)e.addr * Nb + kb];
    }
    L = lb + kb * nlb;
    for (int l = 0; l < nlb; ++l) {
      csffci_link_t e = L[l];
      int a = e.op & 0xff, i = e.op >> 8;
      acc += e.sign * hb[i * norb + a] * ci[ka * Nb + e.addr];
    }
    sigma[t] += acc;
  }
}

}  // namespace csffci

using namespace csffci;

extern "C" {

int csffci_absorb_h1e(int norb, int nelec, const double* h1e, const double* eri, double fac,
                      double* h2e, cudaStream_t stream) {
  CSF_REQUIRE(norb >= 1 && norb <= 63, "absorb_h1e: bad norb %d", norb);
  CSF_REQUIRE(h2e != eri, "absorb_h1e: h2e must not alias eri");
  int npair = norb * (norb + 1) / 2;
  k_absorb_h2e<<<grid_for((int64_t)npair * npair, 128), 128, 0, stream>>>(
      norb, npair, h1e, eri, 1.0 / (nelec + 1e-100), fac, h2e);
  return check_launch("absorb_h1e");
}

size_t csffci_hdiag_det_workspace(int norb, int neleca, int nelecb) {
  unsigned long long Na = host_binom(norb, neleca), Nb = host_binom(norb, nelecb);
  return (size_t)(Na * (norb + 1) + Nb) * sizeof(double) + (size_t)Nb * sizeof(uint64_t) + 256;
}

int csffci_hdiag_det(int norb, int neleca, int nelecb, const double* h1a, const double* h1b,
                     const double* eri, double* hdiag, void* work, size_t work_bytes,
                     cudaStream_t stream) {
  CSF_REQUIRE(norb >= 1 && norb <= 63 && neleca >= 0 && nelecb >= 0 && neleca <= norb &&
                  nelecb <= norb,
              "hdiag_det: bad (norb=%d, nelec=(%d,%d))", norb, neleca, nelecb);
  size_t need = csffci_hdiag_det_workspace(norb, neleca, nelecb);
  if (work == nullptr || work_bytes < need) {
    set_error("hdiag_det: workspace of %zu bytes < %zu required", work_bytes, need);
    return CSFFCI_ERR_MEMORY;
  }
  int npair = norb * (norb + 1) / 2;
  unsigned long long Na = host_binom(norb, neleca), Nb = host_binom(norb, nelecb);
  double* ea = (double*)work;
  double* ja = ea + Na;
  double* eb = ja + Na * norb;
  uint64_t* sb = (uint64_t*)(eb + Nb);
  k_string_energy<<<grid_for((long long)Na, 128), 128, 0, stream>>>(norb, neleca, npair, Na, h1a,
                                                                    eri, ea, ja, nullptr);
  int st = check_launch("hdiag_det alpha strings");
  if (st) return st;
  k_string_energy<<<grid_for((long long)Nb, 128), 128, 0, stream>>>(norb, nelecb, npair, Nb, h1b,
                                                                    eri, eb, nullptr, sb);
  st = check_launch("hdiag_det beta strings");
  if (st) return st;
  {
    ProfScope ps_("k_hdiag_det", stream);
    k_hdiag_det<<<grid_for((long long)(Na * Nb), 256, 148 * 32), 256, 0, stream>>>(norb, Na, Nb, ea,
                                                                                    eb, ja, sb, hdiag);
  }
  return check_launch("hdiag_det");
}

int csffci_pspace_h0(int norb, int neleca, int nelecb, const double* h1a, const double* h1b,
                     const double* eri, const double* hdiag_det, const uint32_t* det_addr, int n,
                     double* h0, cudaStream_t stream) {
  CSF_REQUIRE(norb >= 1 && norb <= 63 && n >= 0, "pspace_h0: bad arguments");
  if (n == 0) return CSFFCI_OK;
  int npair = norb * (norb + 1) / 2;
  unsigned long long Nb = host_binom(norb, nelecb);
  {
    ProfScope ps_("k_pspace_h0", stream);
    k_pspace_h0<<<grid_for((long long)n * n, 128, 148 * 32), 128, 0, stream>>>(
        norb, npair, Nb, h1a, h1b, eri, hdiag_det, det_addr, neleca, nelecb, n, h0);
  }
  return check_launch("pspace_h0");
}

int csffci_contract_1e(int norb, int neleca, int nelecb, const double* h1a, const double* h1b,
                       const csffci_link_t* link_a, const csffci_link_t* link_b, const double* ci,
                       double* sigma, cudaStream_t stream) {
  CSF_REQUIRE(norb >= 1 && norb <= 63, "contract_1e: bad norb %d", norb);
  unsigned long long Na = host_binom(norb, neleca), Nb = host_binom(norb, nelecb);
  int nla = neleca * (norb - neleca + 1), nlb = nelecb * (norb - nelecb + 1);
  k_contract_1e<<<grid_for((long long)(Na * Nb), 256, 148 * 32), 256, 0, stream>>>(
      norb, Na, Nb, nla, nlb, h1a, h1b, link_a, link_b, ci, sigma);
  return check_launch("contract_1e");
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Determinant diagonal without any allocation and without a caller
// workspace.
//
// Some callers cannot call cudaMalloc: a host program whose device memory
// is owned entirely by another allocator (a framework's caching pool with a
// fixed budget, where a raw cudaMalloc would grow memory behind its back),
// or a latency-sensitive loop where cudaMalloc/cudaFree would synchronise
// the device.  Such callers also have no spare buffer to hand over as the
// workspace that csffci_hdiag_det needs.  This variant keeps that
// workspace in a fixed array that is part of the library image instead.
//
// The array below is CSFFCI_HDIAG_NOALLOC_MAX_DOUBLES doubles (2 MiB).  Every
// GPU that loads the library holds it until the process exits.  It fits the
// per-string tables of up to norb = 16 at half filling: Na*(norb+1) + Nb
// doubles plus Nb 64-bit strings.  Larger spaces are rejected.
// ---------------------------------------------------------------------------
static __device__ __align__(256) double g_hdiag_noalloc_scratch[CSFFCI_HDIAG_NOALLOC_MAX_DOUBLES];

namespace csffci {
namespace {
std::mutex g_noalloc_mutex;
// device address of the array per device ordinal, valid for the context
// whose unique id is g_noalloc_ctx[dev] (0: not looked up yet)
void* g_noalloc_ptr[256] = {nullptr};
unsigned long long g_noalloc_ctx[256] = {0};

// Unique id of the calling thread's current context (cuCtxGetId, reached
// through the runtime's driver entry points so that libcuda is not linked);
// 0 when it cannot be had.  Context ids are never reused within a process,
// so an id that differs from the cached one means the cached address
// belongs to a context that no longer is current (a cudaDeviceReset, or a
// context created by another library).
unsigned long long current_context_id() {
  typedef int (*get_current_fn)(void**);
  typedef int (*get_id_fn)(void*, unsigned long long*);
  static get_current_fn get_current = nullptr;
  static get_id_fn get_id = nullptr;
  static bool resolved = false;
  if (!resolved) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = (get_current_fn)f;
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = (get_id_fn)f;
    resolved = true;
  }
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != 0 || ctx == nullptr || get_id(ctx, &id) != 0) return 0;
  return id;
}
}  // namespace
}  // namespace csffci

extern "C" int csffci_hdiag_det_noalloc(int norb, int neleca, int nelecb, const double* h1a,
                                        const double* h1b, const double* eri, double* hdiag,
                                        cudaStream_t stream) {
  CSF_REQUIRE(norb >= 1 && norb <= 63 && neleca >= 0 && nelecb >= 0 && neleca <= norb &&
                  nelecb <= norb,
              "hdiag_det_noalloc: bad (norb=%d, nelec=(%d,%d))", norb, neleca, nelecb);
  const unsigned long long Na = host_binom(norb, neleca), Nb = host_binom(norb, nelecb);
  const unsigned long long need = Na * (unsigned long long)(norb + 1) + 2ull * Nb;
  if (need > (unsigned long long)CSFFCI_HDIAG_NOALLOC_MAX_DOUBLES) {
    set_error("hdiag_det_noalloc: (norb=%d, nelec=(%d,%d)) needs %llu doubles of scratch, more "
              "than the fixed %d; use csffci_hdiag_det with a workspace",
              norb, neleca, nelecb, need, CSFFCI_HDIAG_NOALLOC_MAX_DOUBLES);
    return CSFFCI_ERR_MEMORY;
  }
  // The symbol's name is a host-side stand-in, not a device address: look
  // the address up once per device and context, with that device current.
  int dev = 0;
  CSF_CUDA(cudaGetDevice(&dev));
  CSF_REQUIRE(dev >= 0 && dev < 256, "hdiag_det_noalloc: device ordinal %d out of range", dev);
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    const unsigned long long ctx = current_context_id();
    if (g_noalloc_ptr[dev] == nullptr || ctx == 0 || ctx != g_noalloc_ctx[dev]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_hdiag_noalloc_scratch);
      if (e != cudaSuccess || p == nullptr) {
        set_error("hdiag_det_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev,
                  cudaGetErrorString(e));
        return CSFFCI_ERR_CUDA;
      }
      g_noalloc_ptr[dev] = p;
      g_noalloc_ctx[dev] = current_context_id();
    }
    base = g_noalloc_ptr[dev];
  }
  // Every entry of the scratch that the kernels read is written first by the
  // same call (ea, ja, eb and the beta strings), so nothing needs clearing.
  const int npair = norb * (norb + 1) / 2;
  double* ea = (double*)base;
  double* ja = ea + Na;
  double* eb = ja + Na * norb;
  uint64_t* sb = (uint64_t*)(eb + Nb);
  k_string_energy<<<grid_for((long long)Na, 128), 128, 0, stream>>>(norb, neleca, npair, Na, h1a,
                                                                    eri, ea, ja, nullptr);
  int st = check_launch("hdiag_det_noalloc alpha strings");
  if (st) return st;
  k_string_energy<<<grid_for((long long)Nb, 128), 128, 0, stream>>>(norb, nelecb, npair, Nb, h1b,
                                                                    eri, eb, nullptr, sb);
  st = check_launch("hdiag_det_noalloc beta strings");
  if (st) return st;
  k_hdiag_det<<<grid_for((long long)(Na * Nb), 256, 148 * 32), 256, 0, stream>>>(norb, Na, Nb, ea,
                                                                                  eb, ja, sb, hdiag);
  return check_launch("hdiag_det_noalloc");
}
