// Spin ladder operators on determinant CI vectors: S- = sum_i b+_i a_i and
// S+ = sum_i a+_i b_i (contract_sladder, pyscf/csf_fci/spin_op.py:22-68).
//
// Gather form: one thread per output determinant (Ka, Kb) sums, over the
// orbitals i that the operator can have moved, the sign-weighted source
// element c[Ia, Ib], with Ia, Ib the strings before the move.  The sign of
// a+_i / a_i on a string is (-1)^(occupied orbitals above i) (the
// cre_sign/des_sign convention of the reference's string tables), times
// (-1)^(neleca-1) (S-) or (-1)^neleca (S+) for moving the beta operator past
// the alpha string.  No atomics; every output element is written once.
#include "common.cuh"
#include "profile.cuh"

namespace csffci {

__global__ void k_spin_ladder(int norb, int na_out, int nb_out, int op, const double* __restrict__ ci,
                              long long nb_in, double* __restrict__ out, long long Na_out,
                              long long Nb_out, double fac) {
  const long long n = Na_out * Nb_out;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long ka = idx / Nb_out, kb = idx - ka * Nb_out;
    const unsigned long long Ka = str_unrank(norb, na_out, (unsigned long long)ka);
    const unsigned long long Kb = str_unrank(norb, nb_out, (unsigned long long)kb);
    double acc = 0.0;
    for (int i = 0; i < norb; ++i) {
      const unsigned long long bit = 1ull << i;
      unsigned long long Ia, Ib;
      if (op < 0) {  // S-: alpha i was occupied, beta i was empty
        if ((Ka & bit) || !(Kb & bit)) continue;
        Ia = Ka | bit;
        Ib = Kb ^ bit;
      } else {  // S+: alpha i was empty, beta i was occupied
        if (!(Ka & bit) || (Kb & bit)) continue;
        Ia = Ka ^ bit;
        Ib = Kb | bit;
      }
      const int above = __popcll(Ka >> (i + 1)) + __popcll(Kb >> (i + 1));
      const double v = ci[(long long)str_rank(Ia) * nb_in + (long long)str_rank(Ib)];
      acc += (above & 1) ? -v : v;
    }
    out[idx] = fac * acc;
  }
}

}  // namespace csffci

using namespace csffci;

extern "C" {

int csffci_spin_ladder(int norb, int neleca, int nelecb, int op, const double* ci, double* out,
                       cudaStream_t stream) {
  CSF_REQUIRE(norb >= 1 && norb <= 63 && (op == 1 || op == -1), "spin_ladder: bad norb/op");
  const int na_out = neleca + op, nb_out = nelecb - op;
  CSF_REQUIRE(neleca >= 0 && nelecb >= 0 && neleca <= norb && nelecb <= norb && na_out >= 0 &&
                  nb_out >= 0 && na_out <= norb && nb_out <= norb,
              "spin_ladder: (%d,%d) has no image under S%c in %d orbitals", neleca, nelecb,
              op < 0 ? '-' : '+', norb);
  CSF_REQUIRE(ci != nullptr && out != nullptr, "spin_ladder: NULL vector");
  const long long Na_out = (long long)host_binom(norb, na_out);
  const long long Nb_out = (long long)host_binom(norb, nb_out);
  const long long nb_in = (long long)host_binom(norb, nelecb);
  const int ncomm = op < 0 ? neleca - 1 : neleca;
  const double fac = (ncomm & 1) ? -1.0 : 1.0;
  ProfScope ps("k_spin_ladder", stream);
  k_spin_ladder<<<grid_for(Na_out * Nb_out, 256, 148 * 16), 256, 0, stream>>>(
      norb, na_out, nb_out, op, ci, nb_in, out, Na_out, Nb_out, fac);
  return check_launch("spin_ladder");
}

}  // extern "C"
