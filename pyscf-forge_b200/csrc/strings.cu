// Integer addressing kernels: determinant strings, link tables, the CSD
// (configuration-spin-determinant) permutation, configuration masks and the
// genealogical spin eigenvectors.  All results are bit-exact with the
// reference (see the citations on each kernel).
#include <algorithm>
#include <vector>
#include <string.h>

#include <string>
#include <vector>

#include "common.cuh"

namespace csffci {

static thread_local std::string g_last_error;

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("%s: launch failed: %s", what, cudaGetErrorString(e));
    return CSFFCI_ERR_CUDA;
  }
  return CSFFCI_OK;
}

// ---------------------------------------------------------------------------
// strings and link tables
// ---------------------------------------------------------------------------

__global__ void k_gen_strings(int norb, int nelec, unsigned long long n, uint64_t* out) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x)
    out[i] = str_unrank(norb, nelec, i);
}

// Byte 7 of an entry: the pair index hi*(hi+1)/2+lo of (p, q), the row of
// the four-fold h2e that the sigma tile loops address directly (it fits a
// byte up to 22 orbitals; 0 above).
__device__ __forceinline__ uint8_t link_pair_byte(int p, int q) {
  const int hi = p > q ? p : q, lo = p > q ? q : p;
  const int pr = hi * (hi + 1) / 2 + lo;
  return (uint8_t)(pr < 256 ? pr : 0);
}

// One thread per source string; entries in the order of
// pyscf/lib/mcscf/fci_string_gas.c:1341-1382: for each occupied q
// ascending, (q,q) first, then each virtual p ascending.  Sign of
// a+_p a_q |s> is (-1)^(occupied orbitals strictly between p and q)
// (fci_string_gas.c:252-258).
__global__ void k_link_table(int norb, int nelec, unsigned long long nstr, int nlink,
                             csffci_link_t* link) {
  for (unsigned long long ia = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
       ia < nstr; ia += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned long long s = str_unrank(norb, nelec, ia);
    unsigned long long full = (norb == 64) ? ~0ull : ((1ull << norb) - 1ull);
    csffci_link_t* row = link + ia * (unsigned long long)nlink;
    int k = 0;
    unsigned long long occ = s;
    while (occ) {
      int q = __ffsll((long long)occ) - 1;
      occ &= occ - 1;
      csffci_link_t e;
      e.addr = (uint32_t)ia;
      e.op = (uint16_t)(q | (q << 8));
      e.sign = 1;
      e.pad = link_pair_byte(q, q);
      row[k++] = e;
      unsigned long long vir = (~s) & full;
      while (vir) {
        int p = __ffsll((long long)vir) - 1;
        vir &= vir - 1;
        unsigned long long s1 = (s ^ (1ull << q)) | (1ull << p);
        int hi = p > q ? p : q, lo = p > q ? q : p;
        unsigned long long mask = (1ull << hi) - (1ull << (lo + 1));
        e.addr = (uint32_t)str_rank(s1);
        e.op = (uint16_t)(p | (q << 8));
        e.sign = (int8_t)(1 - 2 * (__popcll(s & mask) & 1));
        e.pad = link_pair_byte(p, q);
        row[k++] = e;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// GAS configuration filter
// ---------------------------------------------------------------------------

// The spin-free supergroups of a GAS restriction as sorted 64-bit keys
// (6 bits of total occupation per subspace, subspace g at bit 6g) and the
// orbital mask of each subspace (consecutive orbitals in subspace order).
constexpr int kGasMaxSpaces = 10;
constexpr int kGasMaxKeys = 1024;
struct GasKeys {
  int ngas, nkey;
  unsigned long long orbmask[kGasMaxSpaces];
  unsigned long long key[kGasMaxKeys];
};

// conf_ok[econf_det_mask[I]] = 1 when the total occupation per subspace of
// determinant I (alpha + beta) is one of the supergroups; every determinant
// of a configuration has the same occupations, so the writes of one
// configuration agree.
__global__ void k_gas_conf(int norb, int neleca, int nelecb, unsigned long long nb, unsigned long long ndet,
                           const uint32_t* __restrict__ econf_det_mask, GasKeys K, uint8_t* conf_ok) {
  __shared__ unsigned long long skey[kGasMaxKeys];
  for (int i = threadIdx.x; i < K.nkey; i += blockDim.x) skey[i] = K.key[i];
  __syncthreads();
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < ndet;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long ia = i / nb, ib = i - ia * nb;
    const unsigned long long sa = str_unrank(norb, neleca, ia), sb = str_unrank(norb, nelecb, ib);
    unsigned long long key = 0;
    for (int g = 0; g < K.ngas; ++g)
      key |= (unsigned long long)(__popcll(sa & K.orbmask[g]) + __popcll(sb & K.orbmask[g])) << (6 * g);
    int lo = 0, hi = K.nkey - 1;
    bool ok = false;
    while (lo <= hi) {
      const int mid = (lo + hi) >> 1;
      const unsigned long long v = skey[mid];
      if (v == key) {
        ok = true;
        break;
      }
      if (v < key) lo = mid + 1;
      else hi = mid - 1;
    }
    conf_ok[econf_det_mask[i]] = ok ? 1 : 0;
  }
}

// ---------------------------------------------------------------------------
// CSD masks
// ---------------------------------------------------------------------------

struct CsdBlocks {
  int nblock;
  int norb, neleca, nelecb;
  long long csd_off[34];
  long long conf_off[34];
  long long csf_off[34];
  long long sconf[34];
  long long spins[34];
  long long ncsf[34];
  int npair[34];
  int nspin[34];
  int nup[34];
  long long ndet_total;
  long long ncsf_total;
};

static int build_csd_blocks(int norb, int na, int nb, int smult, CsdBlocks* B) {
  memset(B, 0, sizeof(*B));
  B->norb = norb;
  B->neleca = na;
  B->nelecb = nb;
  int nless = na < nb ? na : nb;
  int min_npair = na + nb - norb > 0 ? na + nb - norb : 0;
  long long off = 0, coff = 0, foff = 0;
  int ib = 0;
  for (int npair = min_npair; npair <= nless; ++npair, ++ib) {
    int nspin = na + nb - 2 * npair;
    int nup = (nspin + na - nb) / 2;
    long long dconf = (long long)host_binom(norb, npair);
    long long sconf = (long long)host_binom(norb - npair, nspin);
    long long spins = (long long)host_binom(nspin, nup);
    long long ncsf = 0;
    if (smult > 0) {
      // number of genealogical couplings of nspin spins to 2S = smult-1
      int twoS = smult - 1;
      if (twoS <= nspin && ((nspin - twoS) % 2 == 0)) {
        int n0 = (nspin - twoS) / 2;
        ncsf = (long long)host_binom(nspin, n0) - (n0 > 0 ? (long long)host_binom(nspin, n0 - 1) : 0);
      }
    }
    B->csd_off[ib] = off;
    B->conf_off[ib] = coff;
    B->csf_off[ib] = foff;
    B->sconf[ib] = sconf;
    B->spins[ib] = spins;
    B->ncsf[ib] = ncsf;
    B->npair[ib] = npair;
    B->nspin[ib] = nspin;
    B->nup[ib] = nup;
    off += dconf * sconf * spins;
    coff += dconf * sconf;
    foff += dconf * sconf * ncsf;
  }
  B->nblock = ib;
  B->ndet_total = off;
  B->ncsf_total = foff;
  return 0;
}

// Spread the nspin unpaired/paired pattern over the orbitals
// (csdstrs2ddstrs, pyscf/lib/csf/csfstring.c:48-83).
__device__ __forceinline__ void csd_to_dd(int norb, unsigned long long dstr, unsigned long long sstr,
                                          unsigned long long ustr, unsigned long long* a,
                                          unsigned long long* b) {
  unsigned long long as = 0, bs = 0;
  int isorb = 0, ispin = 0;
  for (int iorb = 0; iorb < norb; ++iorb) {
    unsigned long long bit = 1ull << iorb;
    if (dstr & bit) {
      as |= bit;
      bs |= bit;
    } else {
      if ((sstr >> isorb) & 1ull) {
        if ((ustr >> ispin) & 1ull) as |= bit; else bs |= bit;
        ++ispin;
      }
      ++isorb;
    }
  }
  *a = as;
  *b = bs;
}

__global__ void k_csd_masks(CsdBlocks B, unsigned long long nb_strings, uint32_t* csd_mask,
                            uint32_t* econf_det_mask) {
  unsigned long long n = (unsigned long long)B.ndet_total;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    int b = 0;
    while (b + 1 < B.nblock && (unsigned long long)B.csd_off[b + 1] <= i) ++b;
    unsigned long long local = i - (unsigned long long)B.csd_off[b];
    unsigned long long ss = (unsigned long long)(B.sconf[b] * B.spins[b]);
    unsigned long long dc = local / ss;
    unsigned long long rem = local - dc * ss;
    unsigned long long sc = rem / (unsigned long long)B.spins[b];
    unsigned long long sp = rem - sc * (unsigned long long)B.spins[b];
    int npair = B.npair[b], nspin = B.nspin[b];
    unsigned long long dstr = str_unrank(B.norb, npair, dc);
    unsigned long long sstr = str_unrank(B.norb - npair, nspin, sc);
    unsigned long long ustr = str_unrank(nspin, B.nup[b], sp);
    unsigned long long a, bb;
    csd_to_dd(B.norb, dstr, sstr, ustr, &a, &bb);
    unsigned long long dd = str_rank(a) * nb_strings + str_rank(bb);
    if (csd_mask) csd_mask[i] = (uint32_t)dd;
    if (econf_det_mask)
      econf_det_mask[dd] = (uint32_t)((unsigned long long)B.conf_off[b] + dc * (unsigned long long)B.sconf[b] + sc);
  }
}

__global__ void k_econf_csf(CsdBlocks B, uint32_t* econf_csf_mask) {
  unsigned long long n = (unsigned long long)B.ncsf_total;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    int b = 0;
    while (b + 1 < B.nblock && (unsigned long long)B.csf_off[b + 1] <= i) ++b;
    while (B.ncsf[b] == 0) ++b;  // empty blocks have no CSFs at all
    unsigned long long local = i - (unsigned long long)B.csf_off[b];
    econf_csf_mask[i] = (uint32_t)((unsigned long long)B.conf_off[b] + local / (unsigned long long)B.ncsf[b]);
  }
}

// ---------------------------------------------------------------------------
// genealogical couplings and Clebsch-Gordan spin eigenvectors
// ---------------------------------------------------------------------------

struct GenTable {
  int nspin, n0, n1;
  int g[17 * 33];  // (n0+1) x (n1+1), n0 <= 16, n1 <= 32
};

// csf_gentable (pyscf/csf_fci/csfstring.py:806-849)
static int build_gentable(int nspin, int smult, GenTable* T) {
  memset(T, 0, sizeof(*T));
  int twoS = smult - 1;
  T->nspin = nspin;
  if (twoS > nspin) {
    T->n0 = 0;
    T->n1 = 0;
    return 0;
  }
  int n0 = (nspin - twoS) / 2, n1 = (nspin + twoS) / 2;
  if (n0 > 16 || n1 > 32) return -1;
  T->n0 = n0;
  T->n1 = n1;
  int W = n1 + 1;
  std::vector<long long> g((n0 + 1) * W, 0);
  for (int i1 = n0; i1 <= n1; ++i1) g[n0 * W + i1] = 1;
  for (int i0 = n0; i0 >= 1; --i0) {
    int len = n1 + 1 - i0;
    std::vector<long long> row(len + 1);
    for (int j = 0; j < len; ++j) {
      long long s = 0;
      for (int t = j; t < len; ++t) s += g[i0 * W + i0 + t];
      row[j + 1] = s;
    }
    row[0] = row[1];
    for (int j = 0; j <= len; ++j) g[(i0 - 1) * W + i0 - 1 + j] = row[j];
  }
  for (int i = 0; i < (n0 + 1) * W; ++i) {
    if (g[i] > 0x7fffffffLL) return -1;
    T->g[i] = (int)g[i];
  }
  return 0;
}

// FCICSFaddrs2str (csfstring.c:243-293)
__device__ __forceinline__ unsigned long long gen_unrank(const GenTable& T, long long a) {
  unsigned long long s = 1ull;
  int i0 = 0, i1 = 0;
  int W = T.n1 + 1;
  for (int ispin = 0; ispin < T.nspin; ++ispin) {
    if (i1 == T.n1) break;
    int g = T.g[i0 * W + i1 + 1];
    if (g <= a) {
      a -= g;
      ++i0;
    } else {
      s |= 1ull << ispin;
      ++i1;
    }
  }
  return s;
}

// FCICSFmakecsf (csfstring.c:86-141), same double arithmetic in the same
// order so that every coefficient is bit-identical.
__global__ void k_spin_evecs(GenTable T, int na_s, unsigned long long ndet,
                             unsigned long long ncsf, double* umat) {
  unsigned long long n = ndet * ncsf;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned long long idet = i / ncsf, icoup = i - idet * ncsf;
    unsigned long long det = str_unrank(T.nspin, na_s, idet);
    unsigned long long coup = gen_unrank(T, (long long)icoup);
    int t2s = 1;
    int t2ms = (det & 1ull) ? 1 : -1;
    double num = 1, den = 1;
    int sgn = 1;
    int osgn = -t2ms;
    for (int ispin = 1; ispin < T.nspin; ++ispin) {
      unsigned long long sup = (1ull << ispin) & coup;
      unsigned long long msup = (1ull << ispin) & det;
      if (msup) {
        t2ms++;
        osgn *= -1;
      } else {
        t2ms--;
        sgn *= osgn;
      }
      num *= (sup == msup) ? t2s + t2ms + 1 : t2s + 1 - t2ms;
      if (num == 0) break;
      den *= (t2s + 1);
      if (msup && !sup) sgn *= -1;
      num /= 2;
      if (sup) t2s++; else t2s--;
    }
    umat[i] = (num == 0) ? 0.0 : sgn * sqrt((double)num / den);
  }
}

// zmat[ab][k] = (-1)^(b-a-1) sum_{x: bit a != bit b} U[x][k] U[swap_ab(x)][k]
// The rows x are the colex-ordered spin strings with na_s up spins, walked
// in order with Gosper's next-combination step.
__global__ void k_spin_exchange(int nspin, int na_s, unsigned long long ndet,
                                unsigned long long ncsf, const double* __restrict__ umat,
                                double* zmat) {
  int npos = nspin * (nspin - 1) / 2;
  unsigned long long n = (unsigned long long)npos * ncsf;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned long long ab = i / ncsf, k = i - ab * ncsf;
    int b = 1;
    while ((unsigned long long)((b + 1) * b / 2) <= ab) ++b;
    int a = (int)(ab - (unsigned long long)(b * (b - 1) / 2));
    unsigned long long swap = (1ull << a) | (1ull << b);
    unsigned long long s = (na_s == 0) ? 0ull : ((1ull << na_s) - 1ull);
    double acc = 0.0;
    for (unsigned long long x = 0; x < ndet; ++x) {
      unsigned long long bits = s & swap;
      if (bits != 0ull && bits != swap) {
        unsigned long long y = str_rank(s ^ swap);
        acc += umat[x * ncsf + k] * umat[y * ncsf + k];
      }
      if (s != 0ull) {  // Gosper: next larger integer with the same popcount
        unsigned long long c = s & (0ull - s);
        unsigned long long r = s + c;
        s = (((r ^ s) >> 2) / c) | r;
      }
    }
    zmat[i] = ((b - a - 1) & 1) ? -acc : acc;
  }
}

}  // namespace csffci

using namespace csffci;

extern "C" {

int csffci_abi_version(void) { return 1; }

const char* csffci_last_error(void) { return g_last_error.c_str(); }

int csffci_gen_strings(int norb, int nelec, uint64_t* strs, cudaStream_t stream) {
  CSF_REQUIRE(norb >= 0 && norb <= 63 && nelec >= 0 && nelec <= norb,
              "gen_strings: bad (norb=%d, nelec=%d)", norb, nelec);
  unsigned long long n = host_binom(norb, nelec);
  k_gen_strings<<<grid_for((long long)n, 256), 256, 0, stream>>>(norb, nelec, n, strs);
  return check_launch("gen_strings");
}

int csffci_link_table(int norb, int nelec, csffci_link_t* link, cudaStream_t stream) {
  CSF_REQUIRE(norb >= 1 && norb <= 63 && nelec >= 0 && nelec <= norb,
              "link_table: bad (norb=%d, nelec=%d)", norb, nelec);
  unsigned long long n = host_binom(norb, nelec);
  if (n > 0xffffffffull) {
    set_error("link_table: %llu strings exceed 32-bit addressing", n);
    return CSFFCI_ERR_INVALID;
  }
  int nlink = nelec * (norb - nelec + 1);
  if (nlink == 0) return CSFFCI_OK;
  k_link_table<<<grid_for((long long)n, 128), 128, 0, stream>>>(norb, nelec, n, nlink, link);
  return check_launch("link_table");
}

int csffci_gas_conf_mask(int norb, int neleca, int nelecb, const uint32_t* econf_det_mask, int ngas,
                         const int32_t* gas_norb, int nsupergroup, const int32_t* supergroups, uint8_t* conf_ok,
                         cudaStream_t stream) {
  CSF_REQUIRE(norb >= 1 && norb <= 63 && neleca >= 0 && nelecb >= 0 && neleca <= norb && nelecb <= norb,
              "gas_conf_mask: bad (norb=%d, nelec=(%d,%d))", norb, neleca, nelecb);
  CSF_REQUIRE(econf_det_mask && conf_ok && gas_norb && supergroups, "gas_conf_mask: NULL pointer");
  CSF_REQUIRE(ngas >= 1 && ngas <= kGasMaxSpaces, "gas_conf_mask: ngas=%d outside [1,%d]", ngas, kGasMaxSpaces);
  CSF_REQUIRE(nsupergroup >= 1 && nsupergroup <= kGasMaxKeys, "gas_conf_mask: %d supergroups outside [1,%d]",
              nsupergroup, kGasMaxKeys);
  GasKeys K;
  K.ngas = ngas;
  int start = 0;
  for (int g = 0; g < ngas; ++g) {
    CSF_REQUIRE(gas_norb[g] >= 1 && start + gas_norb[g] <= norb, "gas_conf_mask: subspace %d does not fit", g);
    K.orbmask[g] = (gas_norb[g] == 64 ? ~0ull : ((1ull << gas_norb[g]) - 1ull)) << start;
    start += gas_norb[g];
  }
  CSF_REQUIRE(start == norb, "gas_conf_mask: subspaces hold %d of %d orbitals", start, norb);
  std::vector<unsigned long long> keys((size_t)nsupergroup);
  for (int r = 0; r < nsupergroup; ++r) {
    unsigned long long k = 0;
    for (int g = 0; g < ngas; ++g) {
      const int n = supergroups[(size_t)r * ngas + g];
      CSF_REQUIRE(n >= 0 && n <= 2 * gas_norb[g], "gas_conf_mask: occupation %d of subspace %d", n, g);
      k |= (unsigned long long)n << (6 * g);
    }
    keys[(size_t)r] = k;
  }
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  K.nkey = (int)keys.size();
  for (int i = 0; i < K.nkey; ++i) K.key[i] = keys[(size_t)i];
  const unsigned long long na = host_binom(norb, neleca), nb = host_binom(norb, nelecb);
  const unsigned long long ndet = na * nb;
  CSF_REQUIRE(ndet <= 0xffffffffull, "gas_conf_mask: %llu determinants exceed uint32 addressing", ndet);
  if (ndet == 0) return CSFFCI_OK;
  k_gas_conf<<<grid_for((long long)ndet, 256, 148 * 16), 256, 0, stream>>>(norb, neleca, nelecb, nb, ndet,
                                                                            econf_det_mask, K, conf_ok);
  return check_launch("gas_conf_mask");
}

int csffci_csd_masks(int norb, int neleca, int nelecb, int smult, uint32_t* csd_mask,
                     uint32_t* econf_det_mask, uint32_t* econf_csf_mask, cudaStream_t stream) {
  CSF_REQUIRE(norb >= 0 && norb <= 63 && neleca >= 0 && nelecb >= 0 && neleca <= norb &&
                  nelecb <= norb,
              "csd_masks: bad (norb=%d, nelec=(%d,%d))", norb, neleca, nelecb);
  CsdBlocks B;
  build_csd_blocks(norb, neleca, nelecb, smult, &B);
  CSF_REQUIRE(B.nblock <= 34, "csd_masks: too many npair blocks");
  unsigned long long ndet = host_binom(norb, neleca) * host_binom(norb, nelecb);
  CSF_REQUIRE(ndet <= 0xffffffffull, "csd_masks: %llu determinants exceed uint32 addressing", ndet);
  if (csd_mask || econf_det_mask) {
    k_csd_masks<<<grid_for((long long)ndet, 256, 148 * 64), 256, 0, stream>>>(
        B, host_binom(norb, nelecb), csd_mask, econf_det_mask);
    int st = check_launch("csd_masks");
    if (st) return st;
  }
  if (econf_csf_mask && B.ncsf_total > 0) {
    k_econf_csf<<<grid_for(B.ncsf_total, 256, 148 * 64), 256, 0, stream>>>(B, econf_csf_mask);
    return check_launch("econf_csf_mask");
  }
  return CSFFCI_OK;
}

int csffci_spin_evecs(int nspin, int neleca, int nelecb, int smult, double* umat,
                      cudaStream_t stream) {
  int twoMS = neleca - nelecb;
  CSF_REQUIRE(nspin >= 0 && nspin <= 32, "spin_evecs: nspin=%d outside [0,32]", nspin);
  CSF_REQUIRE(abs(twoMS) <= smult - 1 && abs(twoMS) <= nspin && ((twoMS - (smult - 1)) % 2 == 0) &&
                  ((twoMS - nspin) % 2 == 0),
              "spin_evecs: impossible (nspin=%d, 2MS=%d, smult=%d)", nspin, twoMS, smult);
  GenTable T;
  CSF_REQUIRE(build_gentable(nspin, smult, &T) == 0, "spin_evecs: coupling table too large");
  int na_s = (nspin + twoMS) / 2;
  unsigned long long ndet = host_binom(nspin, na_s);
  unsigned long long ncsf = (smult - 1 > nspin) ? 0 : (unsigned long long)T.g[0];
  if (ndet * ncsf == 0) return CSFFCI_OK;
  k_spin_evecs<<<grid_for((long long)(ndet * ncsf), 256, 148 * 64), 256, 0, stream>>>(T, na_s, ndet, ncsf, umat);
  return check_launch("spin_evecs");
}

int csffci_spin_exchange_table(int nspin, int neleca, int nelecb, int smult,
                               const double* umat, double* zmat, cudaStream_t stream) {
  int twoMS = neleca - nelecb;
  CSF_REQUIRE(nspin >= 0 && nspin <= 32, "spin_exchange_table: nspin=%d outside [0,32]", nspin);
  CSF_REQUIRE(abs(twoMS) <= nspin && ((twoMS - nspin) % 2 == 0),
              "spin_exchange_table: impossible (nspin=%d, 2MS=%d)", nspin, twoMS);
  GenTable T;
  CSF_REQUIRE(build_gentable(nspin, smult, &T) == 0, "spin_exchange_table: coupling table too large");
  int na_s = (nspin + twoMS) / 2;
  unsigned long long ndet = host_binom(nspin, na_s);
  unsigned long long ncsf = (smult - 1 > nspin) ? 0 : (unsigned long long)T.g[0];
  unsigned long long npos = (unsigned long long)(nspin * (nspin - 1) / 2);
  if (npos * ncsf == 0) return CSFFCI_OK;
  k_spin_exchange<<<grid_for((long long)(npos * ncsf), 128, 148 * 64), 128, 0, stream>>>(
      nspin, na_s, ndet, ncsf, umat, zmat);
  return check_launch("spin_exchange_table");
}

}  // extern "C"
