// Shared helpers for the CSF-FCI sm_100a kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdarg.h>
#include <stdio.h>

#include "../../include/csffci_b200.h"

namespace csffci {

// ---------------------------------------------------------------------------
// error reporting: every entry point returns a status and leaves a message
// retrievable through csffci_last_error() (thread-local).
// ---------------------------------------------------------------------------
void set_error(const char* fmt, ...);
int check_launch(const char* what);

#define CSF_REQUIRE(cond, ...)                                 \
  do {                                                         \
    if (!(cond)) {                                             \
      ::csffci::set_error(__VA_ARGS__);                        \
      return CSFFCI_ERR_INVALID;                               \
    }                                                          \
  } while (0)

#define CSF_CUDA(call)                                                        \
  do {                                                                        \
    cudaError_t _e = (call);                                                  \
    if (_e != cudaSuccess) {                                                  \
      ::csffci::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,          \
                          cudaGetErrorString(_e));                            \
      return CSFFCI_ERR_CUDA;                                                 \
    }                                                                         \
  } while (0)

// ---------------------------------------------------------------------------
// binomial coefficients C(n,k), n,k < 64, built at compile time into
// constant memory (C(63,31) < 2^63).
// ---------------------------------------------------------------------------
struct BinomTable {
  unsigned long long v[64][64];
  constexpr BinomTable() : v{} {
    for (int n = 0; n < 64; ++n) {
      v[n][0] = 1ull;
      for (int k = 1; k <= n; ++k) v[n][k] = v[n - 1][k - 1] + (k <= n - 1 ? v[n - 1][k] : 0ull);
    }
  }
};

// one copy per translation unit (no relocatable device code needed)
static __constant__ BinomTable c_binom = BinomTable{};
static constexpr BinomTable h_binom_table{};

inline unsigned long long host_binom(int n, int k) {
  return (k < 0 || n < 0 || k > n) ? 0ull : h_binom_table.v[n][k];
}

__device__ __forceinline__ unsigned long long binom(int n, int k) {
  return (k < 0 || n < 0 || k > n) ? 0ull : c_binom.v[n][k];
}

// Colex rank of an occupation bit string: sum_i C(p_i, i), i = 1..nelec over
// set bits p_1 < p_2 < ... (the ascending-integer order PySCF uses for
// determinant strings).
__device__ __forceinline__ unsigned long long str_rank(unsigned long long s) {
  unsigned long long a = 0;
  int i = 1;
  while (s) {
    int p = __ffsll((long long)s) - 1;
    a += c_binom.v[p][i];
    ++i;
    s &= s - 1;
  }
  return a;
}

// Inverse of str_rank for strings of nelec set bits among norb.
__device__ __forceinline__ unsigned long long str_unrank(int norb, int nelec,
                                                         unsigned long long a) {
  unsigned long long s = 0;
  int e = nelec;
  for (int p = norb - 1; p >= 0 && e > 0; --p) {
    unsigned long long c = c_binom.v[p][e];
    if (c <= a) {
      s |= 1ull << p;
      a -= c;
      --e;
    }
  }
  return s;
}

__host__ __device__ inline int pair_index(int p, int q) {
  int hi = p > q ? p : q, lo = p > q ? q : p;
  return hi * (hi + 1) / 2 + lo;
}

inline int grid_for(long long n, int block, int cap = 148 * 32) {
  long long g = (n + block - 1) / block;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

}  // namespace csffci
