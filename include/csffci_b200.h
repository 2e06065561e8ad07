/*
 * csffci_b200.h -- C ABI of the B200 CSF-basis FCI engine (libcsffci_b200.so).
 *
 * Every function takes DEVICE pointers (caller-owned buffers, e.g. from
 * torch), explicit sizes and a cudaStream_t, launches asynchronously on that
 * stream and returns CSFFCI_OK or a negative status; the text of the last
 * error on the calling host thread is returned by csffci_last_error().
 * Functions are re-entrant across streams as long as their output and
 * workspace buffers are distinct.  Nothing allocates device memory except
 * where a function says so; workspaces are passed in.
 *
 * Layouts (all row-major):
 *   determinant CI vector  f64[Na][Nb]      alpha-major, strings in ascending
 *                                           integer (colex) order
 *   CSF CI vector          f64[ncsf]        npair -> doubly-occupied config ->
 *                                           singly-occupied config -> genealogical
 *                                           coupling (pyscf/csf_fci/csdstring.py:10-14,
 *                                           pyscf/csf_fci/csfstring.py:806-849)
 *   two-electron integrals f64[npair][npair] four-fold pair matrix, pair index
 *                                           hi*(hi+1)/2+lo (pyscf/lib/mcscf/fci_gas.h:171-176)
 *   link table             csffci_link_t[N][nlink], row order of
 *                                           pyscf/lib/mcscf/fci_string_gas.c:1341-1382
 */
#ifndef CSFFCI_B200_H
#define CSFFCI_B200_H

#include <stdint.h>
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  CSFFCI_OK = 0,
  CSFFCI_ERR_INVALID = -1, /* bad argument (same meaning as GAS_ERR_INVALID, fci_gas.h:38-42) */
  CSFFCI_ERR_MEMORY = -2,  /* workspace too small (GAS_ERR_MEMORY) */
  CSFFCI_ERR_CUDA = -3,    /* a CUDA runtime call failed */
  CSFFCI_ERR_TIMEOUT = -4  /* a bounded device-side wait gave up */
};

/* One spin-string excitation a+_cre a_des |I> = sign |addr>; byte layout of
 * gas_link_entry_t in raw format (pyscf/lib/mcscf/fci_gas.h:94-105):
 * op = cre | des << 8.  pad (the padding byte there) holds the pair index
 * hi*(hi+1)/2+lo of (cre, des), written by csffci_link_table for norb <= 22;
 * the sigma kernels read it, so the tables they are given come from
 * csffci_link_table, 8-byte aligned. */
typedef struct {
  uint32_t addr;
  uint16_t op;
  int8_t sign;
  uint8_t pad;
} csffci_link_t;

/* One npair block of the CSF <-> determinant map (the loop body of
 * _transform_det2csf, pyscf/csf_fci/csfstring.py:596-659). umat is a device
 * pointer to f64[ndet][ncsf] (the spin eigenvectors of the block, without
 * the block sign). */
typedef struct {
  int64_t csd_offset;  /* first CSD (and det) index of the block            */
  int64_t csf_offset;  /* first CSF index of the block                      */
  int64_t nconf;       /* configurations in the block                       */
  int32_t ndet;        /* spin determinants per configuration               */
  int32_t ncsf;        /* CSFs per configuration (0: block dropped)         */
  int32_t nspin;       /* unpaired electrons                                */
  int32_t npair;       /* doubly occupied orbitals                          */
  double sign;         /* (-1)^ncomm, csfstring.py:623-627                  */
  const double* umat;  /* device f64[ndet][ncsf]                            */
  const double* zmat;  /* device f64[nspin*(nspin-1)/2][ncsf] exchange
                          expectation table for hdiag_csf (may be NULL for
                          transforms)                                        */
  const int32_t* conf_sel; /* NULL: all configurations of the block.  Else
                          device int32[nconf]: the block's configurations
                          (indices within the block, ascending) that belong
                          to the wavefunction's point-group irrep; nconf and
                          csf_offset then count in the packed CSF vector of
                          the symmetric solver (csf_symm.py:25-107,
                          csfstring.py:74-103 pack_csf/unpack_csf).         */
} csffci_block_t;

int csffci_abi_version(void);
const char* csffci_last_error(void);

/* Per-kernel CUDA-event timing on the calling host thread (off by default).
 * enable(1) clears previous records; report() synchronises the recorded
 * events and writes "kernel count total_ms" lines into buf.  No counterpart
 * in the reference (its timing is logger checkpoints, csf.py:387-491). */
int csffci_profile_enable(int on);
int csffci_profile_report(char* buf, size_t len);
/* FP64 throughput of a register-only loop on the current device (kind 0:
 * DMMA m8n8k4 at 16 warps per SM, kind 1: DFMA, kind 2: DMMA at 17 warps per
 * SM, one CTA of 544 threads, which loads one of the four schedulers with 5
 * warps), in TFLOP/s; synchronises the stream.  Kind 0 is the FP64 roofline
 * denominator for the sigma kernel.  No counterpart in the reference. */
int csffci_fp64_peak(int kind, int iters, double* tflops, cudaStream_t stream);

/* ---- strings and link tables (PySCF cistring; reference twin
 *      pyscf/lib/mcscf/fci_string_gas.c:263-298, 1304-1427) ------------- */

/* strs[i] = i-th occupation string of nelec electrons in norb orbitals. */
int csffci_gen_strings(int norb, int nelec, uint64_t* strs, cudaStream_t stream);

/* link[I][k], nlink = nelec*(norb-nelec+1); bit-exact with the raw
 * fill_link_table of fci_string_gas.c:1304-1427. */
int csffci_link_table(int norb, int nelec, csffci_link_t* link, cudaStream_t stream);

/* ---- CSD / configuration masks (csdstring.py:28-65, csfstring.py:789-804,
 *      csfstring.c:13-83) ----------------------------------------------- */

/* csd_mask[idx_csd] = idx_det; econf_det_mask[idx_det] = configuration;
 * econf_csf_mask[idx_csf] = configuration (any output may be NULL). */
int csffci_csd_masks(int norb, int neleca, int nelecb, int smult,
                     uint32_t* csd_mask, uint32_t* econf_det_mask,
                     uint32_t* econf_csf_mask, cudaStream_t stream);

/* conf_ok[c] = 1 for the configurations c whose total occupation per GAS
 * subspace (alpha + beta electrons in the gas_norb[g] consecutive orbitals of
 * subspace g) is one of the nsupergroup rows of supergroups (int32
 * [nsupergroup][ngas], host memory); 0 otherwise.  econf_det_mask (device,
 * from csffci_csd_masks) maps determinants to configurations; conf_ok is a
 * device array over the configurations.  This is the configuration form of
 * a spin-complete GAS restriction (the reference's spin-supergroup set D,
 * pyscf/mcscf/addons_gas.py:318-428, 782-798).  ngas <= 10, nsupergroup
 * <= 1024. */
int csffci_gas_conf_mask(int norb, int neleca, int nelecb, const uint32_t* econf_det_mask, int ngas,
                         const int32_t* gas_norb, int nsupergroup, const int32_t* supergroups,
                         uint8_t* conf_ok, cudaStream_t stream);

/* ---- genealogical spin couplings (csfstring.py:806-960, csfstring.c:86-293) */

/* umat[det][csf] for nspin unpaired electrons, 2MS = neleca-nelecb, 2S+1 =
 * smult; bit-exact with FCICSFmakecsf (csfstring.c:86-141). */
int csffci_spin_evecs(int nspin, int neleca, int nelecb, int smult, double* umat,
                      cudaStream_t stream);

/* zmat[(a,b)][csf] = sum_x umat[x][csf] umat[swap_ab(x)][csf] (-1)^(b-a-1):
 * the expectation value, per CSF, of the signed spin exchange of unpaired
 * positions a<b; used by csffci_hdiag_csf in place of the per-configuration
 * blocks built by FCICSFhdiag (csfstring.c:295-362). */
int csffci_spin_exchange_table(int nspin, int neleca, int nelecb, int smult,
                               const double* umat, double* zmat, cudaStream_t stream);

/* ---- det <-> CSF transforms, batched over nvec vectors
 *      (transform_civec_det2csf / _csf2det, csfstring.py:341-487,569-674) */
int csffci_det2csf(int nvec, const double* x_det, int64_t ld_det, double* x_csf,
                   int64_t ld_csf, const uint32_t* csd_mask,
                   const csffci_block_t* blocks, int nblock, cudaStream_t stream);
/* x_det is fully overwritten (determinants of dropped blocks are zero). */
int csffci_csf2det(int nvec, const double* x_csf, int64_t ld_csf, double* x_det,
                   int64_t ld_det, int64_t ndet, const uint32_t* csd_mask,
                   const csffci_block_t* blocks, int nblock, cudaStream_t stream);

/* ---- Hamiltonian pieces ------------------------------------------------ */

/* h2e[pq][rs] = fac*(eri[pq][rs] + delta_{p=q} f[r,s] + delta_{r=s} f[p,q]),
 * f = (h1e - 1/2 sum_k (pk|kq)) / nelec.  Replaces direct_spin1.absorb_h1e
 * called at csf.py:445,520. */
int csffci_absorb_h1e(int norb, int nelec, const double* h1e, const double* eri,
                      double fac, double* h2e, cudaStream_t stream);

/* Determinant diagonal with (alpha, beta) one-electron parts; replaces
 * direct_uhf.make_hdiag at csf.py:66-68 (reference twin
 * fci_hdiag_gas.c:678-709).  work: >= csffci_hdiag_det_workspace() bytes. */
size_t csffci_hdiag_det_workspace(int norb, int neleca, int nelecb);
int csffci_hdiag_det(int norb, int neleca, int nelecb, const double* h1a,
                     const double* h1b, const double* eri, double* hdiag,
                     void* work, size_t work_bytes, cudaStream_t stream);

/* Same result as csffci_hdiag_det, but allocates nothing and takes no
 * workspace: for callers that cannot call cudaMalloc (device memory owned by
 * another allocator with a fixed budget, or loops where an allocation would
 * synchronise the device) and so have no buffer to lend.  No counterpart in
 * the reference.  Its scratch is a fixed array of
 * CSFFCI_HDIAG_NOALLOC_MAX_DOUBLES doubles (2 MiB) inside the library,
 * held by every GPU that loads it until exit; spaces needing more
 * (Na*(norb+1) + 2*Nb doubles; up to norb = 16 at half filling fits) are
 * rejected with CSFFCI_ERR_MEMORY.  The first call on a device looks up
 * the array's device address, so make that first call before any stream
 * capture; the address is kept per device and context, and the first call
 * in a new context (after cudaDeviceReset, or under another context made
 * current) looks it up again.  All calls share the array: calls that
 * overlap on the GPU (other streams, other host threads) race and must be
 * serialised by the caller. */
#define CSFFCI_HDIAG_NOALLOC_MAX_DOUBLES (1 << 18)
int csffci_hdiag_det_noalloc(int norb, int neleca, int nelecb, const double* h1a,
                             const double* h1b, const double* eri, double* hdiag,
                             cudaStream_t stream);

/* CSF diagonal computed per configuration on the fly (make_hdiag_csf,
 * csf.py:70-144, which materialises (nconf,ndet,ndet) blocks instead).
 * blocks[i].zmat must be set (csffci_spin_exchange_table). */
int csffci_hdiag_csf(int norb, int neleca, int nelecb, const double* hdiag_det,
                     const double* eri, const uint32_t* csd_mask,
                     const csffci_block_t* blocks, int nblock, double* hdiag_csf,
                     cudaStream_t stream);

/* Slater-Condon H among n determinants (full symmetric matrix, diagonal
 * from hdiag_det); replaces libfci.FCIpspace_h0tril_uhf + hermi_triu at
 * csf.py:313-326. */
int csffci_pspace_h0(int norb, int neleca, int nelecb, const double* h1a,
                     const double* h1b, const double* eri, const double* hdiag_det,
                     const uint32_t* det_addr, int n, double* h0, cudaStream_t stream);

/* ---- sigma (direct_spin1.contract_2e at csf.py:449,525-529; reference twin
 *      fci_contract_gas_plan_execute, fci_contract_gas.c:2423-2452) ------- */

enum {
  CSFFCI_SIGMA_ACCUMULATE = 1, /* add into sigma instead of overwriting */
  CSFFCI_SIGMA_SPIN_SYMMETRIC = 2, /* ci == eta * ci^T (na == nb): only the
                                      Jb <= Ja half of the contraction is
                                      formed, then sigma = s + eta * s^T */
  CSFFCI_SIGMA_REFERENCE_KERNEL = 4, /* force the simple shared-memory-h2e
                                        kernel (used to cross-check) */
  CSFFCI_SIGMA_DETERMINISTIC = 8 /* bit-identical reruns (4 <= norb <= 16):
                                    every scattered contribution is split
                                    into three fixed-point digits (weights
                                    2^-80, 2^-37, 2^6) added by 64-bit
                                    integer atomics, whose order does not
                                    change the sums; sigma is formed from
                                    the digit sums afterwards.  Workspace:
                                    3 * ndet int64; contributions must stay
                                    below 2^55 in magnitude.  No counterpart
                                    in the reference (its CPU sigma runs in
                                    a fixed order per thread count). */
};

size_t csffci_sigma_workspace(int norb, int neleca, int nelecb, int flags);
/* out3 = (max|c - c^T|, max|c + c^T|, max|c|) of a square n x n CI matrix
 * (device); decides whether CSFFCI_SIGMA_SPIN_SYMMETRIC applies.  work:
 * 148*4*3 doubles.  No counterpart in the reference. */
int csffci_spin_parity(int64_t n, const double* c, double* out3, void* work,
                       size_t work_bytes, cudaStream_t stream);
/* sigma = sum_{pq,rs} h2e[pq][rs] E_pq E_rs ci.  eta (+1/-1) is used only
 * with CSFFCI_SIGMA_SPIN_SYMMETRIC. */
int csffci_sigma(int norb, int neleca, int nelecb, const double* h2e,
                 const csffci_link_t* link_a, const csffci_link_t* link_b,
                 const double* ci, double* sigma, int flags, int eta, void* work,
                 size_t work_bytes, cudaStream_t stream);

/* Sigma plan: the state of csffci_sigma for one problem bound once, the
 * model of the reference's contraction plan (fci_contract_gas_plan_create /
 * _execute / _free, pyscf/lib/mcscf/fci_gas.h:244-253,
 * fci_contract_gas.c:2388-2452).  create borrows h2e and the link tables
 * (device pointers that must outlive the plan; their contents are read at
 * every execute), fixes the sigma kernel for (norb, neleca, nelecb) and
 * returns the workspace the plan needs (the spin-symmetric scratch when
 * flags holds CSFFCI_SIGMA_SPIN_SYMMETRIC, the three digit planes with
 * CSFFCI_SIGMA_DETERMINISTIC; flags may also hold
 * CSFFCI_SIGMA_REFERENCE_KERNEL).  bind hands that workspace over (caller
 * owned, for the life of the plan).  execute computes sigma from ci on the
 * stream, with flags ACCUMULATE and/or SPIN_SYMMETRIC (the latter only
 * when the plan was created with it; eta = +1/-1 as in csffci_sigma); it
 * allocates nothing and synchronises nothing, so it can be replayed from
 * a captured graph.  One plan must not be executed concurrently on two
 * streams (they would share the workspace), as a GAS plan must not be
 * executed by two host threads at once (fci_gas.h:276-292). */
typedef struct csffci_sigma_plan csffci_sigma_plan_t;
int csffci_sigma_plan_create(int norb, int neleca, int nelecb, const double* h2e,
                             const csffci_link_t* link_a, const csffci_link_t* link_b, int flags,
                             csffci_sigma_plan_t** plan, size_t* work_bytes);
int csffci_sigma_plan_bind(csffci_sigma_plan_t* plan, void* work, size_t work_bytes);
int csffci_sigma_plan_execute(const csffci_sigma_plan_t* plan, const double* ci, double* sigma, int eta,
                              int flags, cudaStream_t stream);
/* the kernel the plan runs: 0..3 register-resident tile variants, 4, 5
 * and 7 the warp-specialised kernels, -2 the shared-memory-h2e kernel */
int csffci_sigma_plan_variant(const csffci_sigma_plan_t* plan);
void csffci_sigma_plan_destroy(csffci_sigma_plan_t* plan);

/* One sigma of a batch (csffci_sigma_batch).  The caller fills the first
 * block; the library fills the rest.  sym = 1 asserts neleca == nelecb and
 * ci = eta ci^T (the spin-symmetric kernel) and needs scratch (ndet
 * doubles); otherwise scratch may be NULL.  flags may hold
 * CSFFCI_SIGMA_JOB_DETERMINISTIC (the scatter of CSFFCI_SIGMA_DETERMINISTIC,
 * 4 <= norb <= 16; scratch then holds the three int64 digit planes, 3 *
 * ndet elements, in either mode); all jobs of one call share it.  live
 * (device, may be NULL) gates the job at run time: it runs only when
 * live_index < *live (used by the device-resident batched solver, whose
 * number of new vectors per problem changes from one iteration to the
 * next). */
enum { CSFFCI_SIGMA_JOB_DETERMINISTIC = 1 };
typedef struct {
  const double* h2e;
  const csffci_link_t* link_a;
  const csffci_link_t* link_b;
  const double* ci;
  double* sigma;
  double* scratch;
  int32_t neleca, nelecb, sym, eta;
  const int32_t* live;
  int32_t live_index, flags;
  /* filled by the library */
  int64_t Na, Nb, unit_begin, nunits, tile_begin, elem_begin;
  int32_t nla, nlb;
} csffci_sigma_job_t;

/* Many sigmas of one orbital count in one persistent launch (role of
 * csf.py:449 applied to every vector of every problem of a batch; no
 * counterpart in the reference, which solves one problem at a time).  Jobs
 * may differ in h2e, electron numbers, spin mode and vectors.  jobs is a
 * host array (updated in place with the bookkeeping fields); work holds the
 * device copy of the job table: csffci_sigma_batch_workspace(njobs)
 * bytes.  Every sigma is overwritten. */
size_t csffci_sigma_batch_workspace(int njobs);
int csffci_sigma_batch(int norb, int njobs, csffci_sigma_job_t* jobs, void* work,
                       size_t work_bytes, cudaStream_t stream);

/* sigma += sum_pq h1a[p,q] Ea_pq ci + h1b[p,q] Eb_pq ci (direct_uhf.contract_1e
 * as used for the spin part of h1e at csf.py:527-528). */
int csffci_contract_1e(int norb, int neleca, int nelecb, const double* h1a,
                       const double* h1b, const csffci_link_t* link_a,
                       const csffci_link_t* link_b, const double* ci, double* sigma,
                       cudaStream_t stream);

/* ---- spin ladder operators (contract_sladder,
 *      pyscf/csf_fci/spin_op.py:22-68) ------------------------------------ */

/* out = S- ci (op = -1: an alpha electron becomes beta) or S+ ci (op = +1)
 * for a determinant vector of (neleca, nelecb) electrons; out is the
 * (C(norb, neleca+op), C(norb, nelecb-op)) vector, fully overwritten, with
 * the sign convention of the reference's spin_op.py.  mup/mdown and
 * <S^2> (spin_square) are built on it. */
int csffci_spin_ladder(int norb, int neleca, int nelecb, int op, const double* ci, double* out,
                       cudaStream_t stream);

/* ---- density matrices (direct_spin1.make_rdm12/trans_rdm12, inherited at
 *      csf.py:557; reference twin fci_rdm_gas_plan_make_rdm12s,
 *      fci_rdm_gas.c:2207-2243, assembled as fci_gas.py:724-733) --------- */

size_t csffci_rdm12_workspace(int norb, int neleca, int nelecb);
/* dm1[p][q] = <bra|q+ p|ket>, dm2[p][q][r][s] = <bra|p+ r+ s q|ket>
 * (fci_gas.h:260-268).  dm2 may be NULL (1-RDM only). */
int csffci_rdm12(int norb, int neleca, int nelecb, const csffci_link_t* link_a,
                 const csffci_link_t* link_b, const double* bra, const double* ket,
                 double* dm1, double* dm2, void* work, size_t work_bytes,
                 cudaStream_t stream);

/* Spin-resolved RDMs (make_rdm12s / trans_rdm12s, inherited at csf.py:557;
 * reference twin fci_rdm_gas_plan_make_rdm12s, fci_rdm_gas.c:2207-2243):
 * dm1s[p][q] = <bra|q+ p|ket> per spin, dm2aa[p][q][r][s] = <p+_a r+_a s_a q_a>,
 * dm2ab = <p+_a r+_b s_b q_a>, dm2bb = <p+_b r+_b s_b q_b>.  The three 2-RDM
 * blocks are all given or all NULL (1-RDMs only). */
size_t csffci_rdm12s_workspace(int norb, int neleca, int nelecb);
int csffci_rdm12s(int norb, int neleca, int nelecb, const csffci_link_t* link_a,
                  const csffci_link_t* link_b, const double* bra, const double* ket, double* dm1a,
                  double* dm1b, double* dm2aa, double* dm2ab, double* dm2bb, void* work,
                  size_t work_bytes, cudaStream_t stream);

/* ---- Davidson update (role of pyscf lib.davidson1 via fci.eig at
 *      csf.py:487-490) --------------------------------------------------- */

/* out[i][j] = sum_k x[i][k] y[j][k]  (nx x ny Gram block, vectors of
 * length n with leading dimensions ldx, ldy); split over the length with a
 * fixed-order final reduction (bit-reproducible). */
size_t csffci_gram_workspace(int nx, int ny, int64_t n);
int csffci_gram(int nx, const double* x, int64_t ldx, int ny, const double* y,
                int64_t ldy, int64_t n, double* out, void* work, size_t work_bytes,
                cudaStream_t stream);
/* y[r][:] = beta*y[r][:] + sum_i coef[r][i] x[i][:], r < ny, i < nx
 * (coef is a device f64[ny][nx]). */
int csffci_combine(int ny, double* y, int64_t ldy, double beta, int nx,
                   const double* x, int64_t ldx, const double* coef, int64_t n,
                   cudaStream_t stream);
/* Davidson/Olsen correction vector for one root (Davidson-Liu with
 * Olsen's correction, J. Olsen, P. Jorgensen, J. Simons, CPL 169, 463
 * (1990); the reference obtains it from fci.make_precond, csf.py:433):
 *   t = (r - e1 x) * P,  P = 1/(hdiag - (e - shift)) with |P| capped at 1e8
 * mode 0: e1 = 0;  mode 1: e1 = (x.P r)/(x.P x) over the diagonal P;
 * mode 2: e1 given (the caller folds an exact p-space block into it).
 * work: csffci_precond_workspace() bytes. */
size_t csffci_precond_workspace(void);
int csffci_precond(int64_t n, const double* r, const double* x, const double* hdiag,
                   double e, double shift, int mode, double e1, double* t, double* work,
                   cudaStream_t stream);
/* out2[0] = x.(P r), out2[1] = x.(P x) over the diagonal P (device). */
int csffci_precond_dots(int64_t n, const double* r, const double* x, const double* hdiag,
                        double e, double shift, double* out2, double* work,
                        cudaStream_t stream);

/* ---- batched forms for many independent problems (no counterpart in the
 *      reference, which solves one problem at a time; used by the lockstep
 *      batched solver).  Descriptor arrays are host arrays; the library
 *      fills their bookkeeping fields, copies them into work and launches
 *      one kernel per call. ------------------------------------------------ */

/* one npair block of one problem's transform over nvec vectors; live
 * (device, may be NULL) caps the vector count at run time to *live */
typedef struct {
  const double* x;
  double* y;
  const uint32_t* mask;
  const double* umat;
  int64_t ldx, ldy, csd_offset, csf_offset, nconf;
  int32_t ndet, ncsf, nvec, pad;
  double sign;
  const int32_t* live;
  int64_t tile_begin; /* filled by the library */
} csffci_transform_job_t;

/* nvec rows of n determinants (leading dimension ld) to zero before a
 * reverse (CSF -> det) transform */
typedef struct {
  double* y;
  int64_t ld, n, nvec;
  int64_t elem_begin; /* filled by the library */
} csffci_zero_job_t;

/* reverse = 0: det -> CSF; 1: CSF -> det (zero jobs run first).  work:
 * njobs*sizeof(csffci_transform_job_t) + nzero*sizeof(csffci_zero_job_t). */
int csffci_transform_batch(int reverse, int njobs, csffci_transform_job_t* jobs, int nzero,
                           csffci_zero_job_t* zjobs, void* work, size_t work_bytes,
                           cudaStream_t stream);

/* out[out_index] = sum_k x[k] y[k] (* P[k] when hdiag != NULL, P = the
 * capped 1/(hdiag - e_shift)); one block per dot, fixed-order reduction.
 * work: ndots*sizeof(csffci_dot_t). */
typedef struct {
  const double* x;
  const double* y;
  const double* hdiag;
  int64_t n;
  double e_shift;
  int64_t out_index;
} csffci_dot_t;
int csffci_dots_batch(int ndots, const csffci_dot_t* dots, double* out, void* work,
                      size_t work_bytes, cudaStream_t stream);

/* y[r][:] = beta*y[r][:] + scale * sum_i coef[r*ldc+i] x[i][:], r < ny, i < nx
 * (coef in device memory).  work: nops*sizeof(csffci_combine_t). */
typedef struct {
  double* y;
  const double* x;
  const double* coef;
  int64_t n, ldx, ldy;
  int32_t ny, nx, ldc, pad;
  double beta, scale;
  int64_t unit_begin; /* filled by the library */
} csffci_combine_t;
int csffci_combine_batch(int nops, csffci_combine_t* ops, void* work, size_t work_bytes,
                         cudaStream_t stream);

/* t = (r - e1 x) * P, P = capped 1/(hdiag - e_shift), e1 = ab[0]/ab[1] read
 * on the device (ab = the two weighted dots x.P r and x.P x; NULL: e1 = 0).
 * work: nops*sizeof(csffci_precond_t). */
typedef struct {
  const double* r;
  const double* x;
  const double* hdiag;
  double* t;
  const double* ab;
  int64_t n;
  double e_shift;
  int64_t unit_begin; /* filled by the library */
} csffci_precond_t;
int csffci_precond_batch(int nops, csffci_precond_t* ops, void* work, size_t work_bytes,
                         cudaStream_t stream);

/* ---- device-resident batched solver (no counterpart in the reference;
 *      each problem follows the one-problem Davidson of csf.py:487-490
 *      with the diagonal Olsen preconditioner of csf.py:433) -------------
 *
 * A plan holds many independent problems (any norb in 4..16, electron
 * numbers, spin and 1..8 roots each).  Every Davidson step of every
 * problem runs on the device, driven by per-problem state records, so one
 * iteration is a fixed launch sequence without host synchronisation; it is
 * captured once as a CUDA graph (use_graph) and replayed, with the host
 * reading the number of unfinished problems every check_every iterations.
 *
 *   create  -> arena_bytes; bind(arena) -> tables uploaded, state reset
 *              (and, with autotune, the sigma tile shape timed per norb);
 *   run     -> iterations; results -> energies / flags (host);
 *   to_det  -> Ritz vectors in the determinant basis; vectors -> pointers;
 *   destroy. */
typedef struct {
  int32_t norb, neleca, nelecb, nroots;
  int32_t eta;     /* 0: general sigma; +1/-1: CSF vectors satisfy
                      c = eta c^T (neleca == nelecb), spin-symmetric sigma */
  int32_t nblocks; /* CSF blocks of the transformer (csffci_det2csf)       */
  const csffci_block_t* blocks; /* host array; umat device pointers        */
  const uint32_t* csd_mask;     /* device, ndet entries                    */
  int64_t ncsf;
  const double* h2e;            /* device absorbed (npair x npair)          */
  const csffci_link_t* link_a;  /* device link tables                       */
  const csffci_link_t* link_b;
  const double* hdiag;          /* device CSF-basis diagonal (ncsf)         */
  const double* x0;             /* device initial vectors (nroots x ncsf)   */
} csffci_batch_problem_t;

typedef struct {
  double conv_tol;          /* |dE| of every root                            */
  double conv_tol_residual; /* |r| of every root (<= 0: sqrt(conv_tol))      */
  double lindep;            /* relative linear-dependence cut of corrections */
  double level_shift;       /* preconditioner shift                          */
  int32_t max_space;        /* subspace size before restart (+ nroots)       */
  int32_t max_cycle;        /* iteration limit                               */
  int32_t check_every;      /* iterations between completion checks          */
  int32_t use_graph;        /* replay one captured iteration                 */
  int32_t autotune;         /* time the sigma tile variants at bind time     */
  int32_t deterministic;    /* sigma with the deterministic scatter (4..16
                               orbitals): bit-identical reruns            */
} csffci_batch_options_t;

typedef struct csffci_batch_plan csffci_batch_plan_t;

int csffci_batch_plan_create(int nprob, const csffci_batch_problem_t* probs,
                             const csffci_batch_options_t* opt, csffci_batch_plan_t** plan,
                             size_t* arena_bytes);
/* arena: device memory of arena_bytes, 256-byte aligned, owned by the caller
 * for the life of the plan */
int csffci_batch_plan_bind(csffci_batch_plan_t* plan, void* arena, size_t arena_bytes,
                           cudaStream_t stream);
int csffci_batch_plan_run(csffci_batch_plan_t* plan, cudaStream_t stream, int* iterations);
/* largest nroots of the batch: the row length of the result arrays */
int csffci_batch_plan_max_roots(const csffci_batch_plan_t* plan);
/* the sigma tile variant used per orbital count (autotuner or default):
 * fills up to cap entries, returns the number of orbital counts */
int csffci_batch_plan_tile_variants(const csffci_batch_plan_t* plan, int32_t* norb,
                                    int32_t* variant, int cap);
/* host arrays: energies/converged [nprob][max_roots] (NaN / 0 past the
 * roots found), niter/nfound [nprob]; any may be NULL */
int csffci_batch_plan_results(csffci_batch_plan_t* plan, double* energies, int32_t* converged,
                              int32_t* niter, int32_t* nfound, cudaStream_t stream);
/* Ritz vectors of every problem to the determinant basis (in the arena) */
int csffci_batch_plan_to_det(csffci_batch_plan_t* plan, cudaStream_t stream);
/* device addresses of problem iprob's CSF Ritz vectors (nroots x ncsf) and
 * determinant vectors (nroots x ndet, valid after to_det) */
int csffci_batch_plan_vectors(const csffci_batch_plan_t* plan, int iprob, const double** csf,
                              const double** det);
void csffci_batch_plan_destroy(csffci_batch_plan_t* plan);

#ifdef __cplusplus
}
#endif
#endif /* CSFFCI_B200_H */
