/*
 * libkspace — B200 (sm_100a) k-space hot path for LatticeQM.jl, C ABI.
 *
 * Reached from Julia as `multimode=:cuda` on the existing k-loop routines.
 * All array arguments are plain pointers in the caller's memory, laid out as
 * Julia stores them: column-major, ComplexF64 as interleaved (re, im) double
 * pairs, lattice keys as Int64 (d entries per key), fractional k-points.
 * The `_dev` entry points take device pointers instead of host pointers and
 * perform no host<->device copies of those arrays.
 *
 * Every function returns LQM_OK (0) or a negative status; the message of the
 * last failure is lqm_last_error(ctx).  A context owns one CUDA stream and is
 * not thread-safe; distinct contexts are independent.  No entry point falls
 * back to a CPU implementation: a context cannot be created without a
 * visible CUDA device.
 *
 * Reference paths are relative to the LatticeQM.jl source tree.
 */
#ifndef LQM_KSPACE_H
#define LQM_KSPACE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LQM_OK 0
#define LQM_EINVAL (-1)   /* invalid argument (sizes, NaN/Inf input, non-Hermitian keys) */
#define LQM_ECUDA (-2)    /* CUDA runtime error, or no usable device */
#define LQM_ENOMEM (-3)   /* device allocation failed */
#define LQM_ETIMEOUT (-4) /* a device wait exceeded the context timeout */
#define LQM_ENOCONV (-5)  /* SCF did not converge and the caller asked for an error */
#define LQM_EDEVICE (-6)  /* a device-side check failed (e.g. no sign change for mu) */

#define LQM_COMM_ID_BYTES 128 /* size of a communicator id (an NCCL unique id) */

typedef struct lqm_ctx lqm_ctx;
typedef struct lqm_hops lqm_hops;

/* Callback once per SCF iteration: mirrors `log_callback(iter, ϵ, residual, info)`
 * with info = (ϵkin, ϵband, ϵH, ϵF, μ), src/modules/Meanfield/selfconsistent.jl:172-182,296-302.
 * A non-zero return value stops the iteration. */
typedef int (*lqm_scf_log_cb)(int64_t iter, double energy, double residual, double ekin, double eband,
                              double eH, double eF, double mu, void* user);

/* Context: device selection, one stream, workspace.  New entry point (the
 * reference selects executors in src/modules/Parallel/Parallel.jl:85-109). */
int lqm_ctx_create(int device, lqm_ctx** out);
int lqm_ctx_destroy(lqm_ctx* ctx);
const char* lqm_last_error(const lqm_ctx* ctx);
/* Host-side wait limit for device work, seconds (default 600): a call whose
 * device work runs longer returns LQM_ETIMEOUT (the work itself finishes on the
 * context's stream and later calls queue behind it).  lqm_bandmatrix[_dev],
 * lqm_densitymatrix[_dev] and lqm_bands_dos_rho[_dev] apply it before their
 * copies into caller memory; other entry points copy first, and a copy into
 * pageable memory waits for the device work without a limit.
 * After LQM_ETIMEOUT, copies into the caller's output buffers may still be queued
 * on the context's stream (at once for page-locked buffers): those buffers may
 * still be written until the stream drains.  They are safe to reuse or free once
 * a later call on the same context has returned LQM_OK (its work queues behind
 * the earlier copies) or after lqm_ctx_destroy. */
int lqm_ctx_set_timeout(lqm_ctx* ctx, double seconds);
/* Eigensolver path selection: orders n >= n_min use the batched blocked path
 * (panel reduction + batched GEMMs); 0 (default) selects it from n = 224 on.
 * No reference counterpart (the reference always calls LAPACK zheevr). */
int lqm_ctx_set_blocked_min_n(lqm_ctx* ctx, int64_t n_min);
/* Reduction of the blocked path: 1 two-stage (dense -> band of half-bandwidth 16 by
 * panel QRs and GEMM updates, band -> tridiagonal by bulge chasing, two-level
 * back-transformation), 0 the one-stage panel reduction (LAPACK zhetrd/zlatrd
 * form, one Hermitian mat-vec per column), -1 (default) by order.  Replaces no
 * reference call: the reference's LAPACK zheevr (src/modules/Eigen/Eigen.jl:22-23)
 * reduces in one stage; zheevr_2stage is LAPACK's two-stage form of the same solve.
 * By default the blocked path (n >= 224) takes the two-stage form for passes that
 * return no eigenvectors (bands; rho, which forms only the columns it needs): on
 * B200 1.8x faster for eigenvalue-only passes at n = 1324 and not slower for rho;
 * passes that return all eigenvectors keep the one-stage form. */
int lqm_ctx_set_two_stage(lqm_ctx* ctx, int mode);
/* Device-side wait limit of the bulge chase (the two-stage reduction's stage 2):
 * the polls of a warp's progress word before a wait gives up (0, the default: about
 * 2^26 polls, well over a second of waiting).  On expiry the kernel records an error,
 * every warp stops, and the call returns LQM_EDEVICE at its next wait on the stream;
 * the context then serves later calls.  A small limit makes the waits run out on
 * purpose (a test of that path; no fault is involved).  No reference counterpart. */
int lqm_ctx_set_device_wait_limit(lqm_ctx* ctx, int64_t polls);
/* SCF acceleration of lqm_scf_hf on this context: 0 (default) linear damped
 * mixing, 1..8 Anderson (Type-II) acceleration with that history depth
 * (src/modules/Meanfield/fixedpoint.jl:39-194,201-231: acceleration=:anderson,
 * anderson_depth), including its Hermitian projection of each iterate. */
int lqm_ctx_set_scf_acceleration(lqm_ctx* ctx, int anderson_depth);
/* SCF residual of lqm_scf_hf on this context: 0 (default) the relative density
 * change ||rho1 - rho0|| / ||rho1|| (fixedpoint.jl:150-156), 1 the commutator
 * norm ||[H_MF[rho0], rho0]||_F over the SCF's k-points with weights 1/nk
 * (src/modules/Meanfield/selfconsistent.jl:399-405, residual_norm=:commutator). */
int lqm_ctx_set_scf_residual(lqm_ctx* ctx, int mode);
/* Terms of the HartreeFock functional used by lqm_scf_hf and lqm_hartreefock_eval
 * on this context, HartreeFock(h, v; hartree, fock) (src/modules/Meanfield/hartreefock.jl:143-175):
 * nonzero switches the Hartree / Fock field on (both on by default). */
int lqm_ctx_set_scf_terms(lqm_ctx* ctx, int hartree, int fock);
/* ExchangeKernel(j, siteof, flavorof) of the J-augmented functional
 * (src/modules/Meanfield/hartreefock.jl:24-76,298-381) for the following SCF and
 * functional evaluations on this context: j is a site-space Hops given on the
 * host (keys d x nJ, blocks ns x ns x nJ complex, column-major; the zero key
 * present, its diagonal zero); siteof/flavorof (length n, 0-based) map each
 * orbital to its site and flavor, every pair once.  ns = 0 removes the kernel.
 * The exchange energy eJ enters the double counting (E = eband - eH - eF - eJ);
 * lqm_ctx_scf_exchange_energy returns the last SCF's eJ. */
int lqm_ctx_set_scf_exchange(lqm_ctx* ctx, int64_t ns, int64_t nJ, int32_t d, const int64_t* jkeys,
                             const double* jblocks, int64_t n, const int64_t* siteof, const int64_t* flavorof);
int lqm_ctx_scf_exchange_energy(const lqm_ctx* ctx, double* eJ);
/* Block size (threads, a multiple of 32 up to 512; 0 restores the built-in rule)
 * of the one-CTA eigensolver for order n on this context.  No reference
 * counterpart (a device launch parameter). */
int lqm_ctx_set_eigh_threads(lqm_ctx* ctx, int64_t n, int nt);
/* Autotuner of that block size for H's order (below the blocked path): every
 * candidate (the block sizes 32, 64, 128, 256, 384 and 512 from half the
 * built-in rule's size up to four times it, or 512, whose shared-memory plan
 * fits) runs the eigen pass on the nk sample k-points (rho_k at mu = 0, T = 0.01
 * when want_rho, else eigenvectors), warmed up once and timed once with CUDA
 * events; the fastest becomes the context's block size for n (the sample should
 * span several waves of CTAs, e.g. the production k-grid, or it times latency
 * rather than throughput).  best_nt/best_ms
 * receive the choice, cand_nt/cand_ms (up to ncand_max, may be NULL) every
 * candidate, *ncand their number.  Block sizes differ in rounding, so a choice is
 * meant to be made once and reused.  For an order on the blocked path the
 * reduction is tuned instead: candidates 0 (one-stage) and 1 (two-stage), timed the
 * same way for the sample's pass kind (rho_k when want_rho, else all eigenvectors);
 * the faster is kept for that order and kind unless lqm_ctx_set_two_stage fixed the
 * reduction (then LQM_EINVAL).  No reference counterpart. */
int lqm_autotune_eigh(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, int want_rho, int* best_nt,
                      double* best_ms, int64_t ncand_max, int* cand_nt, double* cand_ms, int64_t* ncand);
/* Milliseconds of device time of the last call's kernels (CUDA events). */
int lqm_ctx_last_kernel_ms(const lqm_ctx* ctx, double* ms);

/* Device-time statistics since the last reset: eigh_ms / eigh_launches cover
 * the per-k eigensolver kernel, launches counts every kernel this library
 * launched.  The reset also sets what is recorded: enable_timing 0 = nothing,
 * 1 = CUDA-event timing of the eigensolver launches, 2 = that plus the
 * per-phase SM cycle counters of lqm_ctx_phase_cycles (clock reads inside the
 * kernel, so a profiling mode, not a timing one). */
int lqm_ctx_reset_stats(lqm_ctx* ctx, int enable_timing);
int lqm_ctx_stats(const lqm_ctx* ctx, double* eigh_ms, int64_t* eigh_launches, int64_t* launches);
/* The same statistics per kernel class: 0 = the eigensolver passes (as above),
 * 1 = the one-stage blocked reduction's lower-triangle mat-vec, each launch timed
 * with CUDA events, with its algorithmic bytes (the lower triangle of the trailing
 * block read once per column and k-point, 16 B per element); 2 = the two-stage
 * path's stage-2 back-transformation (applying the bulge-chasing reflectors to the
 * needed eigenvector columns), timed the same way, with its algorithmic flops in
 * the last argument (8 n (n-1) per column and k-point).
 * No reference counterpart (profiling). */
int lqm_ctx_kernel_stats(const lqm_ctx* ctx, int kernel_class, double* ms, int64_t* launches,
                         double* algorithmic_bytes);
/* SM cycles spent by the eigensolver kernel per stage, summed over CTAs while
 * the phase counters are enabled (lqm_ctx_reset_stats(ctx, 2)): [0] Bloch
 * sum, [1] Householder, [2] divide and conquer, [3] bands +
 * back-transformation, [4] end-of-k barrier, [5..12] the divide
 * and conquer merge steps (z/sort, deflation, secular roots, Gu-Eisenstat z,
 * vectors/rotations/values, ranks, update, copy back), [13..15] the
 * Householder steps (trailing pass, mat-vec reduction, next column and
 * reflector).  New (profiling). */
int lqm_ctx_phase_cycles(lqm_ctx* ctx, double* cycles /* [16] */);

/* ---- k-point sharding over several GPUs, one process (and one context) per GPU.
 * Replaces the reference's DistributedExec k-loops (src/modules/Parallel/Parallel.jl:
 * 275-287 pmap over k-chunks, 415-467 the streaming fold of per-worker partial rho).
 * Rank 0 makes an id with lqm_comm_unique_id and hands its LQM_COMM_ID_BYTES bytes to
 * the other ranks (MPI, a TCP store, Distributed.jl); every rank then calls
 * lqm_ctx_set_comm(ctx, nranks, rank, id) on its own context and device (collective:
 * it returns once all ranks have joined, or LQM_ETIMEOUT after the context's wait
 * limit).  With nranks > 1 set, these entry points shard the k list they are given:
 * every rank passes the SAME full list (and weights) and processes its contiguous
 * share lqm_shard_range(nk, nranks, rank):
 *   lqm_densitymatrix[_dev], lqm_bands_dos_rho[_dev]: rho_L and the band energy are
 *     summed over the ranks (NCCL all-reduce); bands are gathered on every rank;
 *   lqm_bandmatrix[_dev]: bands (and U) gathered on every rank;
 *   lqm_chemicalpotential, lqm_dos: the bands gathered, then the same mu / DOS on every
 *     rank as on one GPU;
 *   lqm_scf_hf: per iteration the eigen pass and rho on the shard, bands gathered for
 *     mu, rho / band energy / commutator summed; mixing replicated (no graph replay).
 * Every rank must make the same calls in the same order.  Other entry points ignore
 * the communicator.  NCCL is loaded at run time (libnccl.so.2, or the path in
 * LQM_NCCL_LIB); each NCCL call is polled with the context's wait limit, and a
 * failed or timed-out collective aborts the communicator (the context continues
 * unsharded).  nranks = 1 with id == NULL removes the communicator (nranks = 1 with
 * an id makes a one-rank communicator: the same code path, whose collectives are
 * copies). */
int lqm_comm_unique_id(char* id_out /* LQM_COMM_ID_BYTES */);
int lqm_ctx_set_comm(lqm_ctx* ctx, int nranks, int rank, const char* id);
int lqm_ctx_comm(const lqm_ctx* ctx, int* nranks, int* rank);
/* The share [k0, k1) of a k list of nk points that rank `rank` of nranks processes:
 * k0 = floor(rank nk / nranks), k1 = floor((rank + 1) nk / nranks).  Host only. */
int lqm_shard_range(int64_t nk, int nranks, int rank, int64_t* k0, int64_t* k1);

/* Upload a dense Hops (src/modules/TightBinding/types.jl:54-60, DenseHops):
 * keys d x nR (Int64), blocks n x n x nR column-major ComplexF64 in the same
 * key order.  The key order is the Bloch-sum order (types.jl:18-25). */
int lqm_hops_upload_dense(lqm_ctx* ctx, int64_t n, int64_t nR, int32_t d, const int64_t* keys,
                          const double* blocks, lqm_hops** out);
/* Upload a SparseHops (types.jl:60; the form `autoconversion` gives every Hops
 * with n > MAX_DENSE = 500, types.jl:102-103,272): per key a Julia
 * SparseMatrixCSC with 1-based Int64 colptr (n+1), rowval and ComplexF64 nzval.
 * nnz[r] is the length of rowval[r] (nzval[r] holds 2*nnz[r] doubles), i.e.
 * Julia's length(m.rowval); the call reads only the colptr[r][n]-1 entries that
 * colptr addresses and rejects a colptr that does not start at 1, decreases, or
 * ends beyond nnz[r], rows outside 1..n and non-finite values (LQM_EINVAL).
 * Only the stored entries are copied to the device; the dense blocks are built
 * there (repeated entries are summed in storage order). */
int lqm_hops_upload_csc(lqm_ctx* ctx, int64_t n, int64_t nR, int32_t d, const int64_t* keys,
                        const int64_t* const* colptr, const int64_t* const* rowval,
                        const double* const* nzval, const int64_t* nnz, lqm_hops** out);
/* Release a Hops.  With a context, first waits (within the context's limit) for
 * the work queued on its stream, which may still read the blocks; on LQM_ETIMEOUT
 * nothing is released and h stays valid, to be freed by a later call.  With
 * ctx == NULL the buffer is freed directly (cudaFree waits for the device). */
int lqm_hops_free(lqm_ctx* ctx, lqm_hops* h);
int lqm_hops_dims(const lqm_hops* h, int64_t* n, int64_t* nR, int32_t* d);

/* Batched Bloch sum H(k) = Σ_R H_R e^{i2πk·R}, replaces `fouriersum!`
 * (src/modules/TightBinding/types.jl:18-25) over a k list: Hk is n x n x nk. */
int lqm_bloch(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, double* Hk);
int lqm_bloch_dev(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* d_ks, double* d_Hk);

/* Bands (and optionally eigenvectors) on a k list, replaces `bandmatrix`
 * without projectors (src/modules/Spectrum/bands.jl:164-227; per-k eigen of
 * `Hermitian(H(k))`, upper triangle, src/modules/Eigen/Eigen.jl:22-23,32).
 * bands: n x nk ascending per column; U: n x n x nk (may be NULL).
 * `precision` (here and in the eigen-pass entry points below): 0 = FP64, the only
 * form built; any other value returns LQM_EINVAL. */
int lqm_bandmatrix(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, int want_vectors,
                   int precision, double* bands, double* U);
int lqm_bandmatrix_dev(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* d_ks, int want_vectors,
                       int precision, double* d_bands, double* d_U);

/* ρ_L = Σ_k w_k e^{-i2πk·L} U f(ε-μ;T) U^H for the nL given keys and the band
 * energy Σ_k w_k Σ_n f ε; replaces `getdensitymatrix!` + `densitymatrix_kpoint!`
 * (src/modules/Operators/densitymatrix.jl:28-49,107-145).  w == NULL means
 * uniform 1/nk (densitymatrix.jl:17-20).  rho: n x n x nL, overwritten. */
int lqm_densitymatrix(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, const double* w,
                      double mu, double T, int64_t nL, const int64_t* Lkeys, double* rho, double* eband,
                      int precision);
int lqm_densitymatrix_dev(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* d_ks,
                          const double* d_w, double mu, double T, int64_t nL, const int64_t* Lkeys,
                          double* d_rho, double* eband, int precision);

/* Chemical potential from the bands of H on a k list, replaces
 * `chemicalpotential(H, ks, filling; T)` (src/modules/Spectrum/chemicalpotential.jl:6-46,53-66):
 * T == 0 midpoint of order statistics, T > 0 float bisection of the filling
 * on [min ε, max ε].  w == NULL: unweighted mean (chemicalpotential.jl:76). */
int lqm_chemicalpotential(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, const double* w,
                          double filling, double T, double* mu);
/* Same on precomputed device bands (n x nk). */
int lqm_chemicalpotential_bands_dev(lqm_ctx* ctx, int64_t n, int64_t nk, const double* d_bands,
                                    const double* d_w, double filling, double T, double* mu);

/* Lorentzian DOS, replaces `getdos!`/`dos_compute!` (src/modules/Spectrum/dos.jl:185-188,202-223):
 * DOS(ω) = Σ_k w_k Σ_n Im[1/(ω - iΓ - ε)], divided by nk when w == NULL. */
int lqm_dos(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, const double* w, int64_t nw,
            const double* omegas, double gamma, double* dos);
int lqm_dos_bands_dev(lqm_ctx* ctx, int64_t n, int64_t nk, const double* d_bands, const double* d_w,
                      int64_t nw, const double* d_omegas, double gamma, double* d_dos);

/* Bands, DOS and ρ_L from ONE eigen pass over the k list: the outputs of
 * `bandmatrix` + `getdos` + `getdensitymatrix!` on the same H and ks
 * (src/modules/Spectrum/bands.jl:164-227, src/modules/Spectrum/dos.jl:202-223,
 * src/modules/Operators/densitymatrix.jl:28-49,130-145), which the reference
 * computes with three separate k-loops.  w == NULL: uniform 1/nk for ρ and
 * the unweighted DOS normalisation.  bands: n x nk; rho: n x n x nL; dos: nw. */
int lqm_bands_dos_rho(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, const double* w, double mu,
                      double T, int64_t nL, const int64_t* Lkeys, double* rho, double* eband, int64_t nw,
                      const double* omegas, double gamma, double* dos, double* bands, int precision);
int lqm_bands_dos_rho_dev(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* d_ks, const double* d_w,
                          double mu, double T, int64_t nL, const int64_t* Lkeys, double* d_rho, double* eband,
                          int64_t nw, const double* d_omegas, double gamma, double* d_dos, double* d_bands,
                          int precision);

/* lqm_bands_dos_rho_dev for several models of uneven order on the same k list, with
 * ONE eigensolver launch for all of them: the batched form of the per-model loop of
 * `bandmatrix` / `getdos` / `getdensitymatrix!` (src/modules/Spectrum/bands.jl:164-204,
 * dos.jl:202-223, densitymatrix.jl:28-49), which the reference runs model by model.
 * Each model's k-points go to CTA sub-teams of that model's one-CTA block size
 * (several teams per CTA on named barriers), so small orders fill the SMs as large
 * ones drain.  Models: 1..4, all below the blocked eigensolver's switch; arrays of
 * nmodels entries (H, nL, Lkeys, d_rho, d_omegas, d_dos, d_bands; eband receives
 * nmodels values); d_w NULL means 1/nk. */
int lqm_bands_dos_rho_multi_dev(lqm_ctx* ctx, int nmodels, const lqm_hops* const* H, int64_t nk,
                                const double* d_ks, const double* d_w, double mu, double T, const int64_t* nL,
                                const int64_t* const* Lkeys, double* const* d_rho, double* eband, int64_t nw,
                                const double* const* d_omegas, double gamma, double* const* d_dos,
                                double* const* d_bands);

/* Hartree-Fock SCF with linear mixing, device-resident, replaces
 * `solvehartreefock` (src/modules/Meanfield/selfconsistent.jl:19,256-336,366-381;
 * functional hartreefock.jl:143-289,392-410; mixing fixedpoint.jl:39-194).
 * rho_inout: n x n x nL for the keys Lkeys (initial guess in, converged out).
 * out_scalars[9] = {E_GS, mu, eH, eF, eband, ekin, residual, converged, iterations}. */
int lqm_scf_hf(lqm_ctx* ctx, const lqm_hops* h, const lqm_hops* v, int64_t nk, const double* ks,
               const double* w, double filling, double T, double beta, double tol, int64_t maxiter,
               int64_t nL, const int64_t* Lkeys, double* rho_inout, lqm_scf_log_cb cb, void* cb_user,
               double* out_scalars);

/* Allocation-free eigen pass.  No counterpart in the reference: it exists for
 * callers that cannot allocate device memory, e.g. a host whose device memory
 * is owned by another allocator (a Julia CUDA.jl pool, a framework's caching
 * allocator) that must not see foreign cudaMalloc/cudaFree, or a
 * latency-sensitive loop that cannot afford their implicit device-wide
 * synchronisation.  Same computation as lqm_bandmatrix_dev (bands n x nk; U
 * n x n x nk when d_U is not NULL) with every array a caller-owned device
 * pointer and H given as device keys (d x nR Int64) and blocks (n x n x nR
 * ComplexF64), launched on `stream` (a cudaStream_t; NULL = legacy default).
 * Scratch comes from a fixed 64 MiB device array inside the library (held on
 * every GPU that loads it until exit); n <= 1024, within the one-CTA
 * shared-memory plan (about 470), and one k-point's scratch must fit; other
 * orders return LQM_EINVAL.  The first call on a device resolves
 * that array's address and should come before any stream capture.  Calls that
 * overlap on the GPU share the array and race.  Returns LQM_OK, LQM_EINVAL
 * (sizes/pointers) or LQM_ECUDA (launch/runtime error); it does not wait for
 * the kernels to finish. */
int lqm_bandmatrix_noalloc(void* stream, int64_t n, int64_t nR, int32_t d, const int64_t* d_keys,
                           const double* d_blocks, int64_t nk, const double* d_ks, double* d_bands, double* d_U);

/* bandmatrix(H, ks, projectors...) with band expectation values
 * (src/modules/Spectrum/bands.jl:52-60,107-112,164-227): bands (n x nk) and
 * obs[i + n*(j + nk*p)] = Re <u_i(k_j)| P_p(k_j) |u_i(k_j)> for the nproj
 * operators P_p(k) = sum_R P_p,R e^{+i2pi k.R} (device Hops of order n; a
 * k-independent matrix is a Hops with the single key 0).  nproj = 0 gives
 * the bands only. */
int lqm_bandmatrix_obs(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, int64_t nproj,
                       const lqm_hops* const* P, double* bands, double* obs);

/* Site-resolved density (src/modules/Spectrum/dos.jl:20-52): n_i = 1/nk sum_k
 * sum_{eps_j(k) <= mu} |U_ij(k)|^2, written to n_out (n doubles). */
int lqm_density(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, double mu, double* n_out);
/* Local density of states (src/modules/Spectrum/dos.jl:56-98): n_i = 1/(nk pi)
 * sum_k sum_j |U_ij|^2 (1/nw) sum_w gamma / ((w - eps_j)^2 + gamma^2).  Every
 * k-point contributes the frequency average once (the reference's per-k
 * routine divides its running accumulator by nw at each k-point; the two
 * agree for nw = 1, the ldos(H, ks, frequency) form). */
int lqm_ldos(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, int64_t nw, const double* omegas,
             double gamma, double* n_out);
/* Fermi-surface density, fermisurfacedensity_fromdata(bands, energies[, obs]; broadening)
 * of src/modules/Spectrum/fermisurface.jl on the bands of a k list:
 * density[e + nE k] = sum_b (1/pi) w_bk g^2 / (g^2 + (eps_bk - E_e)^2), w = weights
 * (n x nk, e.g. band expectation values) or 1 when NULL; g = broadening, or for
 * broadening <= 0 the reference's :auto (mean over bands of the band's standard
 * deviation over k, divided by sqrt(nk)); *broadening_used receives g. */
int lqm_fermisurface(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, int64_t nE,
                     const double* energies, double broadening, const double* weights, double* density,
                     double* broadening_used);

/* Berry curvature plaquette phases, berry(H, NX, NY, bandindices)
 * (src/modules/Spectrum/berry.jl:48-82,107-155): eigenvectors of the nb bands
 * `bands` (0-based) on k = (i/(NX-1), j/(NY-1)) + 1.34e-8, link variables
 * det(S^H S')/|det|, and F[i + (NX-1) j] = arg(plaquette product)/(2 pi) for
 * the (NX-1) x (NY-1) plaquettes.  Two-dimensional Hops only. */
int lqm_berry(lqm_ctx* ctx, const lqm_hops* H, int64_t NX, int64_t NY, int64_t nb, const int64_t* bands, double* F);
/* Berry flux of several band manifolds on one state grid: flux[s] = sum of the
 * plaquette phases of lqm_berry over the bands set_bands[set_ptr[s] .. set_ptr[s+1])
 * (0-based; set_ptr has nsets + 1 entries).  Single-band sets give getcherns
 * (src/modules/Spectrum/berry.jl:378-382), the sets {0..n-1} the gap Chern numbers
 * of gapcherns (:470-487) before rounding.  One eigen pass over the NX x NY grid. */
/* Abelian Berry curvature along a k-path, berryalongpath(H, kpoints)
 * (src/modules/Spectrum/berry.jl:170-238): the path (2 x N, N >= 2) padded at both
 * ends and shifted by 1.34e-6 |k_2 - k_1| (1, 1/sqrt 2); per point the plaquette of
 * the four corners k +- (neighbour differences)/2 and their rotations by +-pi/2;
 * out[i + n j] = the plaquette phase of band i at point j (n x N). */
int lqm_berry_path(lqm_ctx* ctx, const lqm_hops* H, int64_t N, const double* kpoints, double* out);
/* Wilson loops over the statesgrid of bands `bands` (0-based, nb <= 8): the loops of
 * WilsonSlice1D in Wilson2D (src/modules/Spectrum/berry.jl:258-268,312-367) on the
 * periodic grid of the first NX-1 x NY-1 points; dir 1: one loop along k_y per k_x
 * (NX - 1 loops), dir 2: along k_x per k_y (NY - 1 loops).  Per loop the product of the
 * polar factors (U V^H of the SVD) of the link overlaps S_a^H S_b and its eigenphases
 * angle/(2 pi) in ascending order: en[loop nb + m]; U (may be NULL) receives the
 * eigenvectors (nb x nb per loop, complex, in the order of en; normalised, phase
 * arbitrary). */
int lqm_wilson(lqm_ctx* ctx, const lqm_hops* H, int64_t NX, int64_t NY, int64_t nb, const int64_t* bands, int dir,
               double* en, double* U);
/* WilsonWannier2D(H, NX, NY, bandindices) (src/modules/Spectrum/berry.jl:274-301): the
 * states of every point rotated by the eigenvectors of the Wilson loop through it (loops
 * along k_y for p1, along k_x for p2, based at that point), then per band the mean over
 * the other direction of the abelian Wilson loops of the rotated band: p1[nb], p2[nb].
 * The same grid and band limit (nb <= 8) as lqm_wilson. */
int lqm_wilson_wannier(lqm_ctx* ctx, const lqm_hops* H, int64_t NX, int64_t NY, int64_t nb, const int64_t* bands,
                       double* p1, double* p2);
int lqm_berry_flux(lqm_ctx* ctx, const lqm_hops* H, int64_t NX, int64_t NY, int64_t nsets, const int64_t* set_ptr,
                   const int64_t* set_bands, double* flux);

/* The HartreeFock functional hf(rho) (src/modules/Meanfield/hartreefock.jl:184-228,
 * 247-289,298-410): hMF = h - v .* rho (Fock) + the Hartree diagonal (+ the
 * exchange fields of the context's ExchangeKernel), with the context's terms.
 * rho: n x n x nL for keys Lkeys (d x nL, the zero key present).  hmf_out
 * receives hMF at the nM keys Mkeys (zero blocks for keys outside hMF's key set
 * keys(h) + keys(v) + exchange keys present in rho); energies = {eH, eF, eJ}. */
int lqm_hartreefock_eval(lqm_ctx* ctx, const lqm_hops* h, const lqm_hops* v, int64_t nL, const int64_t* Lkeys,
                         const double* rho, int64_t nM, const int64_t* Mkeys, double* hmf_out, double* energies);

/* Commutator norm ||[H, rho]||_F = sqrt(sum_k w_k ||H(k) rho(k) - rho(k) H(k)||_F^2),
 * commutator_kspace_norm (src/modules/Meanfield/selfconsistent.jl:130-166);
 * w NULL means 1/nk.  H and rho are Hops of the same order and key dimension
 * (their key sets may differ). */
int lqm_commutator_norm(lqm_ctx* ctx, const lqm_hops* H, const lqm_hops* rho, int64_t nk, const double* ks,
                        const double* w, double* out);

/* Partial spectrum, the `format=:sparse, num_bands` path of bandmatrix and
 * getdensitymatrix! (src/modules/Eigen/eigen_sparse_krylovkit.jl:44-88,
 * src/modules/Operators/densitymatrix.jl:100-104,131-147): per k the
 * num_bands eigenpairs nearest sigma (which = 0, the reference's :LM
 * shift-invert default, sigma defaulting to 1e-8 there), the smallest (1, :SR)
 * or the largest (2, :LR), in ascending order.  Computed by the dense
 * eigensolver and a window selection (on a tie in distance the lower
 * eigenvalue is taken).  bands: num_bands x nk; U: n x num_bands x nk.
 * lqm_densitymatrix_partial is lqm_densitymatrix with rho_k = U_w f U_w^H
 * over the selected states only. */
int lqm_bandmatrix_partial(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, int64_t num_bands,
                           double sigma, int which, int want_vectors, double* bands, double* U);
int lqm_densitymatrix_partial(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, const double* w,
                              double mu, double T, int64_t num_bands, double sigma, int which, int64_t nL,
                              const int64_t* Lkeys, double* rho, double* eband);

/* Nambu (BdG) Hamiltonians: a Hops of order 2d, electron block first, as
 * BdGOperator.h builds it (src/modules/Superconductivity/types.jl:36-97).
 * lqm_bdg_densitymatrix: getdensitymatrix!(rho::BdGOperator, H::BdGOperator, ks,
 * kweights, mu) (src/modules/Superconductivity/green.jl:38-54): rho_L of H - mu tau_z
 * at mu = 0 (n x n x nL, n = 2d) and *energy = <H - mu N> = (band sum)/2 +
 * (Re tr h_e[0] - d mu)/2.  lqm_bdg_filling: Spectrum.filling(H::BdGOperator, ks, mu;
 * T) (src/modules/Superconductivity/operators.jl:117-122), the electron trace of
 * rho_0 over d.  lqm_bdg_chemicalpotential: Spectrum.chemicalpotential(H::BdGOperator,
 * ks, target; T, mu_lo, mu_hi) (operators.jl:139-155), float bisection of the
 * filling on the bracket from the electron-sector bands (one eigen pass with
 * vectors per step).  w NULL means 1/nk.  H is not modified. */
int lqm_bdg_densitymatrix(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, const double* w, double mu,
                          double T, int64_t nL, const int64_t* Lkeys, double* rho, double* energy);
int lqm_bdg_filling(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, const double* w, double mu,
                    double T, double* out);
int lqm_bdg_chemicalpotential(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, const double* w,
                              double filling, double T, double mu_lo, double mu_hi, double* out);

/* Hartree-Fock with pairing on Nambu density matrices: solvehartreefock with
 * HartreeFock(h::BdGOperator, v) = HartreeFockBDG (src/modules/Superconductivity/
 * hartreefock.jl:5-159) in the SCF loop of src/modules/Meanfield/selfconsistent.jl:256-336
 * with the BdG chemical potential and density matrix (operators.jl:139-155,
 * green.jl:38-54).  h, v: the electron-sector Hops (order d); rho_inout: the Nambu
 * density matrix, order 2d, nL keys (closed under L -> -L, the zero key present);
 * k-weights 1/nk; the context's SCF acceleration (linear or Anderson), residual
 * (relative density change or ||[HB, rho0]||) and Hartree/Fock switches (no
 * exchange kernel).  out[10] = {E, mu, eH, eF, eband, ekin,
 * residual, converged, iterations, eP} with E = eband - (eH + eF + eP). */
int lqm_scf_hf_bdg(lqm_ctx* ctx, const lqm_hops* h, const lqm_hops* v, int64_t nk, const double* ks,
                   double filling, double T, double beta, double tol, int64_t maxiter, int64_t nL,
                   const int64_t* Lkeys, double* rho_inout, lqm_scf_log_cb cb, void* cb_user, double* out);

/* Kubo current-current correlator, opticalconductivity(frequencies, H, J1, J2,
 * ks; mu, Gamma, T) (src/modules/LinearResponse/opticalconductivity.jl:101-127
 * with kubo! of src/modules/LinearResponse/kubo.jl:11-26):
 *   chi(w) = -(i/nk) sum_k sum_{i != j} (f_i - f_j) (U^H J1 U)_ij (U^H J2^H U)_ji
 *            / ((e_i - e_j) - (w + i Gamma)),
 * f = fermidirac(e; T, mu).  J1 and J2 are Hops of H's order and key dimension
 * (the current operators of getcurrentoperators, src/modules/Operators/current.jl:20-37).
 * chi receives nw complex values (interleaved re, im).  nw <= 524280.
 * Passing the same handle for J1 and J2 computes U^H J U once. */
int lqm_opticalconductivity(lqm_ctx* ctx, const lqm_hops* H, const lqm_hops* J1, const lqm_hops* J2, int64_t nk,
                            const double* ks, int64_t nw, const double* omegas, double mu, double gamma, double T,
                            double* chi);

/* ---- Reverse-mode derivatives (no reference counterpart: the reference has
 * no derivatives; the forward maps are lqm_densitymatrix and lqm_bandmatrix).
 *
 * Density response at fixed mu and T.  Gbar: nL blocks (2*n*n doubles each,
 * keys Lkeys, d x nL) holding dLoss/d rho_L; output Hbar: one block per key
 * of H (H's key order) such that dLoss = Re sum_R <Hbar_R, dH_R> for every
 * Hermitian-consistent perturbation (dH_{-R} = dH_R^H), <A,B> = sum conj(A) B:
 *   Hbar_R = sum_k e^{-i2pi k.R} w_k U [F o (U^H B_k U)] U^H,
 *   B_k = sum_L e^{+i2pi k.L} Gbar_L,
 *   F_ij = (f_i - f_j)/(eps_i - eps_j), f'((eps_i+eps_j)/2) for |eps_i - eps_j| <= 1e-6 T.
 * w == NULL: uniform weights 1/nk.  The gradient of the grand potential
 * -T sum_k w_k sum_j log(1 + e^{-(eps_j - mu)/T}) with respect to H_R is rho_R
 * itself (lqm_densitymatrix). */
int lqm_densitymatrix_vjp(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, const double* w,
                          double mu, double T, int64_t nL, const int64_t* Lkeys, const double* Gbar,
                          double* Hbar);
/* Band cotangent: eps_bar (n x nk, dLoss/d eps) -> Hbar_R = sum_k e^{-i2pi k.R} U diag(eps_bar_k) U^H. */
int lqm_bands_vjp(lqm_ctx* ctx, const lqm_hops* H, int64_t nk, const double* ks, const double* eps_bar,
                  double* Hbar);

/* Derivatives of the converged Hartree-Fock SCF with respect to the hopping
 * blocks of h (the functional of src/modules/Meanfield/hartreefock.jl:143-289,392-410
 * at the fixed point of src/modules/Meanfield/selfconsistent.jl:256-336).  Inputs:
 * h, v and the converged rho (keys Lkeys, with its chemical potential mu, e.g. from
 * lqm_scf_hf with the same k-points, weights (NULL: 1/nk), T and the context's
 * Hartree/Fock switches; no exchange kernel).  Outputs:
 *   out[5] = {F, Omega_band, N, adjoint residual, adjoint iterations}: the free
 *     energy F = Omega_band + mu N - (eH + eF) of hMF = hf(rho),
 *     Omega_band = -T sum_k w_k sum_j log(1 + e^{-(eps_j - mu)/T}) (T = 0: the sum of
 *     eps_j - mu below mu), N = sum_k w_k sum_j f_j;
 *   dF_dh (may be NULL): dF/dh_R for the keys of h (n x n x nR(h)), which at
 *     self-consistency is the density matrix of hMF at those keys (Hellmann-Feynman);
 *   dL_dh (with eps_bar): for a loss L of the mean-field bands eps(hMF) with band
 *     cotangent eps_bar (n x nk, dL/d eps_jk), the total derivative dL/dh_R through
 *     the fixed point, including the chemical potential's response at T > 0: the
 *     implicit-function adjoint solved by the damped iteration of the SCF's linear
 *     mixing (beta) until its relative change is below tol or maxiter iterations.
 * Pairing: dL = Re sum_R <dL_dh_R, dh_R>, <A, B> = sum conj(A) B, for every
 * Hermitian-consistent perturbation of h.  No reference counterpart (the reference
 * has no derivatives). */
int lqm_scf_hf_gradient(lqm_ctx* ctx, const lqm_hops* h, const lqm_hops* v, int64_t nk, const double* ks,
                        const double* w, double T, double mu, int64_t nL, const int64_t* Lkeys, const double* rho,
                        const double* eps_bar, double beta, double tol, int64_t maxiter, double* dF_dh,
                        double* dL_dh, double* out);

#ifdef __cplusplus
}
#endif
#endif /* LQM_KSPACE_H */
