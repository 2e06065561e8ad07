// Register-resident sigma kernel (sigma_rr.cu), used by csffci_sigma for
// 4 <= norb <= 16.
#pragma once
#include "common.cuh"

namespace csffci {
bool sigma_rr_supported(int norb);
// variant: tile variant of the register-resident family (0..3), 4, 5, 6 or
// 7 for the warp-specialised kernels, -1 for the default of one problem;
// det_stride != 0 runs the deterministic scatter into three int64 digit
// planes det_stride elements apart, out pointing at the first
int sigma_rr_run(int norb, int neleca, int nelecb, const double* h2e, const csffci_link_t* la,
                 const csffci_link_t* lb, const double* ci, double* out, bool sym, double eta,
                 cudaStream_t stream, int variant = -1, long long det_stride = 0);
// the kernel variant one problem of norb orbitals runs by default
// (CSFFCI_SIGMA_VARIANT overrides it)
int sigma_rr_single_variant(int norb);
// the register-resident tile variant of norb orbitals (0..3)
int rr_default_variant(int norb);
}  // namespace csffci
