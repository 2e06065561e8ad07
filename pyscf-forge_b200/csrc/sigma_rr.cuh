// Register-resident sigma kernel (sigma_rr.cu), used by csffci_sigma for
// 4 <= norb <= 16.
#pragma once
#include "common.cuh"

namespace csffci {
bool sigma_rr_supported(int norb);
int sigma_rr_run(int norb, int neleca, int nelecb, const double* h2e, const csffci_link_t* la,
                 const csffci_link_t* lb, const double* ci, double* out, bool sym, double eta,
                 cudaStream_t stream);
}  // namespace csffci
