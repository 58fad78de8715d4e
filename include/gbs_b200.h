/* gbs_b200.h -- C ABI of libgbs_b200.so: batched permanents, hafnians, loop
 * hafnians and torontonians on NVIDIA B200 (sm_100a).
 *
 * Drop-in for the reference's host API (chaofanzhougit/GBSKernels core/host_api.cu)
 * and the entry points its Python binding calls (bindings/gbskernels_ext.cpp).
 *
 * Conventions (identical to the reference):
 *   - complex matrices are interleaved (re, im) binary64 pairs, row-major, batch
 *     contiguous: the memory of a numpy complex128 (B, d, d) array (the reference
 *     types these pointers cuDoubleComplex*, which has the same layout);
 *   - `n` is the matrix side for perm, the MODE count for tor (matrices 2n x 2n),
 *     `N` the matrix side for haf / lhaf;
 *   - every function returns 0 on success or a nonzero code (a cudaError_t value
 *     or cudaErrorInvalidValue = 1 for bad arguments); gbs_last_error() describes
 *     the last failure of the calling thread;
 *   - the caller owns host buffers; the library owns device and pinned buffers.
 *   - a torontonian off the physical domain (I - O_S not positive definite) or an
 *     uncertifiable element yields NaN values (and +inf bounds), never an error.
 */
#ifndef GBS_B200_H
#define GBS_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gbs_session gbs_session;

int gbs_version(void);
const char* gbs_last_error(void);

/* ---- one-shot uniform batches: H2D -> launch -> D2H ------------------------
 * reference: core/host_api.cu:153-230 (gbs_perm_host ... gbs_tor_dd_host)     */
int gbs_perm_host(const double* mats, int n, int batch, double* out);
int gbs_perm_dd_host(const double* mats, int n, int batch, double* out);
int gbs_haf_host(const double* mats, int N, int batch, double* out);
int gbs_haf_dd_host(const double* mats, int N, int batch, double* out);
/* odd N is evaluated as lhaf(A (+) [1]) (gbskernels/__init__.py:190-200) */
int gbs_lhaf_host(const double* mats, int N, int batch, double* out);
int gbs_lhaf_dd_host(const double* mats, int N, int batch, double* out);
int gbs_tor_host(const double* mats, int n, int batch, double* out);
int gbs_tor_dd_host(const double* mats, int n, int batch, double* out);

/* ---- fp64 value + sum|term| (precision="auto" indicator) -------------------
 * reference: core/host_api.cu:235-246 (gbs_*_kappa_host)                       */
int gbs_perm_kappa_host(const double* mats, int n, int batch, double* out, double* absnorm);
int gbs_haf_kappa_host(const double* mats, int N, int batch, double* out, double* absnorm);
int gbs_lhaf_kappa_host(const double* mats, int N, int batch, double* out, double* absnorm);
int gbs_tor_kappa_host(const double* mats, int n, int batch, double* out, double* absnorm);

/* ---- certified tier: fp64 value (bit-identical to the fp64 tier) + a rigorous
 * bound |value - exact| <= bound, carried in directed rounding.  Uncertifiable or
 * off-domain elements return NaN with bound +inf; non-finite input is rejected.
 * reference: core/host_api.cu:248-262 (gbs_*_certified_host)                     */
int gbs_perm_certified_host(const double* mats, int n, int batch, double* out, double* bound);
int gbs_haf_certified_host(const double* mats, int N, int batch, double* out, double* bound);
int gbs_lhaf_certified_host(const double* mats, int N, int batch, double* out, double* bound);
int gbs_tor_certified_host(const double* mats, int n, int batch, double* out, double* bound);
/* certified double-double permanent: the double-double Glynn walk of
 * gbs_perm_dd_host (the value equals it before the final rounding to binary64)
 * in ball arithmetic; the rung of the certified ladder above
 * gbs_perm_certified_host.  reference: core/host_api.cu:263-265
 * (gbs_perm_dd_certified_host), kernels core/certified_dd.cu:124-328.            */
int gbs_perm_dd_certified_host(const double* mats, int n, int batch, double* out, double* bound);
/* certified double-double hafnian / loop hafnian: the double-double power trace of
 * gbs_haf_dd_host / gbs_lhaf_dd_host (the value equals it before the rounding to
 * binary64) with an a-priori radius from double-word operation bounds and the
 * powers of |C|, to N = 32 (the reference stops at 16).
 * reference: core/host_api.cu:266-268 (gbs_haf_dd_certified_host), kernel
 * core/certified_dd.cu:216-328; the loop hafnian rung is this library's own.      */
int gbs_haf_dd_certified_host(const double* mats, int N, int batch, double* out, double* bound);
int gbs_lhaf_dd_certified_host(const double* mats, int N, int batch, double* out, double* bound);
/* certified double-double torontonian (real O, 24 modes batched): the value is
 * computed in double-word arithmetic (returned rounded to binary64) and the bound
 * is rigorous; the rung of the certified ladder above gbs_tor_certified_host.
 * reference counterpart: the certified-dd rung of gbskernels/__init__.py:410-425
 * (its batched dd-certified kernels cover perm / haf, core/host_api.cu:263-268).  */
int gbs_tor_dd_certified_host(const double* mats, int n, int batch, double* out, double* bound);

/* ---- single-large torontonian ----------------------------------------------
 * reference: core/host_api.cu:270-298 (gbs_tor_recursive_single_host) and :300-352
 * (gbs_tor_single_certified_host); bindings/gbskernels_ext.cpp:46-47.
 * O: real (2n x 2n) row-major binary64 (NOT complex), n <= 32.  One torontonian
 * split into at least 2^g prefix work items across the GPU (g in [0, n], the
 * reference's `groups`; the planner may split further).  Off the physical domain
 * (a non-SPD minor of I - O) *out is NaN and *bound +inf.  The certified bound is
 * rigorous: |*out - tor(O)| <= *bound.                                          */
int gbs_tor_recursive_single_host(const double* O, int n, int g, double* out);
int gbs_tor_single_certified_host(const double* O, int n, int g, double* out, double* bound);
/* reference: core/host_api.cu:354-405 (gbs_tor_single_ddcertified_host): the same
 * single-large evaluation in double-word with a rigorous bound.                  */
int gbs_tor_single_ddcertified_host(const double* O, int n, int g, double* out, double* bound);

/* ---- repeated-row loop hafnian (finite-difference sieve) ----------------------
 * reference: core/host_api.cu:409-432 (gbs_lhaf_repeated_host),
 * bindings/gbskernels_ext.cpp:49; algorithm cpu_ref/repeated.py:64-122.
 * A: M x M complex base matrix; gamma: M complex loop weights (NULL = zeros, the
 * ordinary hafnian of the expansion); reps: batch x M non-negative counts; out:
 * batch complex values lhaf(A repeated by reps[b]).  Caps: M <= 32, N = sum(reps[b])
 * <= 64, prod(reps[b][i] + 1) <= 2^40.  A non-symmetric A enters as its symmetric
 * part (A + A^T)/2, the only part x^T A x sees.  The sieve's device buffers stay
 * allocated on each device between calls (grown only); calls are serialised.      */
int gbs_lhaf_repeated_host(const double* A, const double* gamma, int M, const int* reps, int batch, double* out);
/* certified sieve: values bit-identical to gbs_lhaf_repeated_host and a rigorous
 * bound per pattern (bound[b] >= |out[b] - lhaf|); non-finite input is rejected, an
 * uncertifiable pattern returns NaN with bound +inf.
 * reference: core/host_api.cu:434-458 (gbs_lhaf_repeated_cert_host), kernel
 * core/repeated.cu:158-340.                                                       */
int gbs_lhaf_repeated_cert_host(const double* A, const double* gamma, int M, const int* reps, int batch, double* out,
                                double* bound);
const char* gbs_lhaf_repeated_last_error(void);

/* ---- resident sampler chain (on-device conditional draw) ---------------------
 * reference: core/sampler_session.cu:106-137 (gbs_sampler_sample), kernels
 * core/sampler_gather.cu:20-57 and core/sampler_draw.cu:15-47.
 * h_Ak: the M reduced A-matrices (A_k: 2k x 2k complex, row-major) concatenated,
 * A_k starting at complex element h_off[k-1]; ak_total complex elements in all.
 * Per mode k = 1..M the conditional submatrices A_k[idx, idx] of every draw are
 * gathered on the device, their hafnians evaluated by the work-item kernel and the
 * count drawn by inverse CDF of clip(Re haf, 0) * h_invfac[j] (one Philox4_32_10
 * uniform per draw and mode, subsequence = draw index); h_out: num_draws x M counts.
 * Draws that share a prefix (the counts of the modes before k) share their
 * conditional hafnians, which are evaluated once per distinct prefix.
 * Requires 2 M cutoff <= 32 (maxn is accepted for the reference's signature).  The
 * chain's device buffers stay allocated on each device between calls (grown only);
 * calls are serialised.                                                            */
int gbs_sampler_sample(const double* h_Ak, int ak_total, const int* h_off, int M, int num_draws, int cutoff,
                       int maxn, const double* h_invfac, unsigned long long seed, int* h_out);
/* the conditional weights Re haf(A_k[idx, idx]) of mode k for the prefixes in
 * h_state (num_draws x M counts; columns < k-1 used): h_w is num_draws x (cutoff+1).
 * No reference counterpart (a parity hook for the gather and hafnian steps).       */
int gbs_sampler_conditional_weights(const double* h_Ak, int ak_total, const int* h_off, int M, int k,
                                    const int* h_state, int num_draws, int cutoff, double* h_w);
const char* gbs_sampler_last_error(void);
/* prefix sharing of gbs_sampler_sample on (1, the default) or off (0: every draw's
 * conditionals evaluated separately); the samples are identical either way.
 * Process-wide.  No reference counterpart.                                        */
int gbs_sampler_set_dedup(int on);

/* ---- auto tier on the device ----------------------------------------------
 * reference: gbskernels/__init__.py:272-297 (_gpu_auto_batched) whose fp64 pass is
 * gbs_*_kappa_host and whose rerun is gbs_*_dd_host; here both run in the library.
 * func: 0 perm, 1 haf, 2 lhaf, 3 tor.  dim = matrix side (tor: 2n).  Elements
 * with kappa = absnorm/|value| >= kappa_max are re-evaluated in double-double.
 * tier_out[i]: 0 = fp64 value kept, 1 = double-double rerun.                    */
int gbs_auto_host(int func, const double* mats, int dim, int batch, double kappa_max, double* out,
                  double* kappa, int* tier_out);

/* ---- certified tier with the rtol ladder --------------------------------------
 * reference: the certified ladder of gbskernels/__init__.py:374-478 (_certified_single
 * / _certified_batched), whose GPU rungs are gbs_*_certified_host and
 * gbs_*_dd_certified_host; here the whole ladder is one call.  func: 0 perm, 1 haf,
 * 2 lhaf, 3 tor; dim = matrix side (tor: 2n).  The binary64 certificate first;
 * elements whose bound does not prove |error| / |value| <= rtol, or is not finite,
 * are re-evaluated by the certified double-double rung.  tier_out[i]: 3 certified
 * binary64, 4 certified double-double, -1 neither rung certifies it (the
 * reference's mpmath rung is CPU-only and has no counterpart).  rtol < 0: no
 * ladder (-1 marks a non-finite binary64 certificate).  Non-finite input returns
 * cudaErrorInvalidValue.  A complex torontonian has the binary64 rung only (its
 * certificate comes from ball arithmetic through the subset LU).                 */
int gbs_certified_ladder_host(int func, const double* mats, int dim, int batch, double rtol, double* out,
                              double* bound, int* tier_out);

/* ---- resident sessions -------------------------------------------------------
 * reference: core/host_api.cu:521-658 (gbs_session_open ... gbs_dev_free)
 * func: 0 perm, 1 haf, 2 lhaf, 3 tor; prec: 0 fp64, 1 dd.  dim = matrix side.  */
int gbs_session_open(gbs_session** out);
int gbs_session_close(gbs_session* s);
size_t gbs_session_reallocs(const gbs_session* s);
int gbs_session_evaluate(gbs_session* s, int func, int prec, const double* mats, int dim, int batch,
                         double* out);
/* Device-resident output: the (B,) complex results are scattered in request order
 * on the device into a fresh buffer (no host round trip of the results), owned by
 * the caller and released with gbs_dev_free.                                     */
int gbs_session_evaluate_resident(gbs_session* s, int func, int prec, const double* mats, int dim,
                                  int batch, double** d_result);
int gbs_dev_to_host(const double* d_result, double* h_out, int n);
int gbs_dev_free(double* d_result);
/* Resident output for every tier: *d_block = [B complex values][B doubles aux]
 * [B int32 status] in request order (status 0 ok, value NaN otherwise; released
 * with gbs_dev_free).  tier: 0 fp64, 1 dd, 2 fp64 + sum|term| in aux, 3 certified
 * (aux = rigorous bound), 4 certified double-double (perm, tor), -1 auto (fp64 +
 * indicator, kappa >= 1e8 rerun in dd on the device; aux = kappa).
 * reference counterpart: the resident path of core/host_api.cu:600-658 is fp64 /
 * dd only (bindings/gbskernels_ext.cpp:209-228); the other tiers are this
 * library's own.                                                                  */
int gbs_session_evaluate_resident_tier(gbs_session* s, int func, int tier, const double* mats, int dim,
                                       int batch, double** d_block);
/* Ragged / mixed batch (as gbs_queue_evaluate), resident: a block as above.
 * reference: gbskernels/__init__.py:856-908 refuses ragged resident batches (no
 * device scatter there); this one scatters on the device.                        */
int gbs_queue_evaluate_resident(gbs_session* s, int B, const int* funcs, const int* tiers, const int* dims,
                                const long long* offsets, const double* mats, int mode, double** d_block);
/* bytes from device memory (a resident block's aux / status parts) to the host */
int gbs_dev_copy_to_host(const void* d, void* h, size_t bytes);
/* the CUDA device that owns device memory d (DLPack export of resident results) */
int gbs_dev_device(const void* d, int* device);

/* ---- ragged, mixed-function, mixed-tier batches ----------------------------
 * reference: gbskernels/__init__.py:813-852 (Workspace._ragged: one launch per
 * size bucket).  mode 0: ONE persistent launch over a device work queue holding
 * every instance (functions, sizes and tiers mixed); mode 1: one launch per
 * (function, tier, size) bucket.  offsets[i] is in complex elements into `mats`.
 * tiers[i]: 0 fp64, 1 dd, 2 fp64 + sum|term| (aux[i]), 3 certified (aux[i] = bound).
 * status[i]: 0 ok, 1 torontonian off the physical domain, 2 uncertifiable.       */
int gbs_queue_evaluate(gbs_session* s, int batch, const int* funcs, const int* tiers, const int* dims,
                       const long long* offsets, const double* mats, int mode, double* out, double* aux,
                       int* status);
/* as gbs_queue_evaluate, with one host pointer per matrix (mats[i]: dims[i]^2
 * complex, row-major) instead of a packed buffer: each matrix is copied once,
 * straight into the session's pinned staging buffer.  No reference counterpart
 * (the reference stacks each size bucket with np.stack, gbskernels/__init__.py:822-833). */
int gbs_queue_evaluate_ptrs(gbs_session* s, int batch, const int* funcs, const int* tiers, const int* dims,
                            const double* const* mats, int mode, double* out, double* aux, int* status);
/* auto tier over a ragged / mixed batch (tiers are implied): fp64 + indicator for
 * every request in one launch, kappa >= kappa_max reruns in double-double in one
 * more; tier_out[i] 0 fp64, 1 dd; kappa[i] = sum|term| / |value|.
 * reference: gbskernels/__init__.py:799-812 (Workspace auto, per size bucket).    */
int gbs_queue_evaluate_auto(gbs_session* s, int batch, const int* funcs, const int* dims, const long long* offsets,
                            const double* mats, double kappa_max, double* out, double* kappa, int* tier_out,
                            int* status);
/* device-resident plan: validate, cut and upload once; run many times on `stream`
 * (a cudaStream_t, or NULL for the session stream); read results back.  Used for
 * timing with inputs resident in HBM and by servers that re-run a fixed batch.   */
int gbs_queue_prepare(gbs_session* s, int batch, const int* funcs, const int* tiers, const int* dims,
                      const long long* offsets, const double* mats, int mode);
int gbs_queue_run(gbs_session* s, void* stream);
int gbs_queue_read(gbs_session* s, void* stream, double* out, double* aux, int* status);
/* kernel time (CUDA events), launches and work items of the session's last call */
int gbs_session_last_stats(const gbs_session* s, double* kernel_ms, int* launches, long long* items);
/* gbs_queue_run captures a prepared plan's launch sequence (queue resets + one
 * launch per group) into a CUDA graph on its second run and replays the graph
 * afterwards; enable = 0 turns that off for the session.  No reference counterpart
 * (the reference launches each size bucket directly).                           */
int gbs_session_set_graphs(gbs_session* s, int enable);
/* Autotuner hooks (process-wide).  split = log2 of the work per item for
 * (func, tier, evaluated side): haf / lhaf subsets per item, perm Gray steps per
 * lane, tor prefix leaves per item (double-double: subsets per lane); -1 = the
 * planner's default.  warps = block size of per-size launches (0 = default).  The
 * binary64 tiers share one entry.  No reference counterpart.                     */
int gbs_set_split(int func, int tier, int dim, int split, int warps);
int gbs_get_split(int func, int tier, int dim, int* split, int* warps);

/* ---- continuous-batching server (chain-rule sampler queries) -----------------
 * No reference counterpart (the reference's resident sampler session,
 * core/sampler_session.cu:68-128, runs one fixed chain; it serves no requests).
 * A scheduler thread owns `n_slots` sessions (one stream each); requests that
 * arrive while batches run are admitted into the next free slot up to
 * `budget_bytes` of workspace per batch; up to n_slots batches overlap on the GPU.
 * tier: 0 fp64, 1 dd, 2 auto (fp64 + indicator, device double-double rerun when
 * kappa >= 1e8), 3 certified.  Resident states (M x M complex + optional M loop
 * weights) stay in HBM; a state request's matrix state[idx][:, idx] is gathered on
 * the device (core/sampler_gather.cu:20-57 is the reference's gather).           */
typedef struct gbs_server gbs_server;
int gbs_server_open(int n_slots, long long budget_bytes, int max_batch, gbs_server** out);
int gbs_server_close(gbs_server* sv);
int gbs_server_add_state(gbs_server* sv, const double* A, const double* gamma, int M, int* state_id);
int gbs_server_submit(gbs_server* sv, int func, int tier, int dim, const double* mat, long long* ticket);
int gbs_server_submit_state(gbs_server* sv, int func, int tier, int state, int n_idx, const int* idx,
                            int use_gamma, long long* ticket);
/* non-blocking; when *done: out[2] value, aux = kappa (auto) / bound (certified),
 * tier_used 0 fp64 / 1 dd / 3 certified, latency_s = completion - submission      */
int gbs_server_poll(gbs_server* sv, long long ticket, int* done, double* out, double* aux, int* status,
                    int* tier_used, double* latency_s);
int gbs_server_drain(gbs_server* sv, double timeout_s);
int gbs_server_stats(gbs_server* sv, long long* completed, long long* batches, long long* pending);

/* ---- hafnian without allocation ---------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device memory
 * while they evaluate (their memory belongs to another allocator, or an allocation
 * would stall a latency-critical loop): d_mats (batch x N x N complex) and d_out
 * (batch complex) are device pointers the caller owns; every scratch buffer lives
 * in a fixed 4 MiB __device__ array in the library (held by each GPU that loads it
 * until exit).  Limits: N <= 32, batch <= 16384, at most 49152 work items
 * (batch x 2^(N/2 - split), split = 7 unless gbs_set_split tuned (haf, fp64, N):
 * batch x 2^max(0, N/2 - 7) by default); larger requests return
 * cudaErrorInvalidValue.  The work queue is written on the device by a fill
 * kernel, so no host buffer is read after the call returns.  The first call on a
 * device looks up the array's address; calls that overlap on the GPU share the
 * array and race.  Asynchronous on `stream` (a
 * cudaStream_t).  Values equal gbs_haf_host's bit for bit for complex input
 * (same split, same kernel).  Every input here runs the complex power loop: for a
 * real input (every imaginary part zero) gbs_haf_host runs the real one instead,
 * and the two then agree to rounding, not bit for bit.                          */
int gbs_haf_noalloc(const double* d_mats, int N, int batch, double* d_out, void* stream);
const char* gbs_haf_noalloc_last_error(void);

/* ---- measurement ------------------------------------------------------------
 * FP64 tensor-core throughput of this GPU (mma .m16n8k8 .f64 chains on every SM),
 * the denominator of the kernels' roofline fraction.  No reference counterpart.  */
int gbs_probe_fp64_peak(double* tflops, float* ms);
/* the same probe for one mma shape: k = 8 (m16n8k8, = gbs_probe_fp64_peak) or
 * k = 4 (m16n8k4); flops counted per shape.  No reference counterpart.           */
int gbs_probe_fp64_mma(int k, double* tflops, float* ms);
/* the probe as a sweep: k = 8 or 4, chains_per_warp in {1, 2, 4, 8} independent
 * accumulator chains, warps_per_block (1..16) warps in each of `blocks` blocks;
 * *cycles = cycles per mma of warp 0 (clock64), its latency when chains = 1.
 * No reference counterpart.                                                      */
int gbs_probe_fp64_mma_chains(int k, int chains_per_warp, int warps_per_block, int blocks, double* tflops,
                              double* cycles);

#ifdef __cplusplus
}
#endif

#endif /* GBS_B200_H */
