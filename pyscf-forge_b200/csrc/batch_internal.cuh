// Launch pieces of the batched kernels shared by the one-call batch entry
// points and the device-resident batched solver, which prepares its job
// tables once and replays the launches (CUDA graph) every iteration.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "csffci_b200.h"

namespace csffci {

// transform jobs: fill tile_begin, return the total tile count
int transform_batch_prepare(int reverse, int njobs, csffci_transform_job_t* jobs, int64_t* total_tiles);
int transform_batch_launch(int reverse, const csffci_transform_job_t* jobs_dev, int njobs, int64_t tiles,
                           cudaStream_t stream);

// sigma jobs of one orbital count: bookkeeping, then the zero / sigma /
// symmetric-add launches over a device copy of the table
struct SigmaBatchInfo {
  int norb = 0, njobs = 0;
  long long total_units = 0, max_nb = 0, nelem = 0, ntiles = 0;
  int max_nla = 0, max_nlb = 0;
  int variant = -1;  // tile shape of the sigma kernel (-1: default for norb)
  int det = 0;       // the jobs use the deterministic scatter (CSFFCI_SIGMA_JOB_DETERMINISTIC)
  csffci_sigma_job_t job0{};
};
int sigma_batch_prepare(int norb, int njobs, csffci_sigma_job_t* jobs, SigmaBatchInfo* info);
int sigma_batch_launch(const SigmaBatchInfo& info, const csffci_sigma_job_t* jobs_dev, cudaStream_t stream);
// time every tile variant on the (ungated) device job table and set
// info.variant to the fastest; cached per (norb, job shapes).  The sigma
// outputs of the jobs are overwritten.
int sigma_batch_tune(SigmaBatchInfo& info, const csffci_sigma_job_t* jobs_host, const csffci_sigma_job_t* jobs_dev,
                     cudaStream_t stream);

}  // namespace csffci
