/*
 * kinet-b200: B200-native (sm_100a) polynomial-commitment path -- C ABI.
 *
 * Drop-in GPU bodies for the reference's C entry points on this path, plus
 * the Fr-NTT, synthetic-SRS commit, batched-commit and serving entry points
 * the reference does not have, named in its <alg>_<op> style.
 *
 * All entry points are synchronous unless their name ends in _device, take
 * caller-owned buffers, allocate nothing the caller must free, and are safe
 * to call from several host threads (calls on one device are serialised).
 * There is no CPU fallback: without a usable CUDA device every entry point
 * returns its backend error code and kb200_last_error() says why.
 *
 * Encodings at this boundary (all canonical, never Montgomery):
 *   scalar / Fr element : 32 bytes little-endian
 *   G1 affine point     : x || y big-endian; 96 B (BLS12-381), 64 B (BN254);
 *                         all-zero bytes = point at infinity
 *   compressed G1       : 48 bytes, ZCash/IETF flags (BLS12-381)
 */
#ifndef KINET_B200_CRYPTO_B200_H
#define KINET_B200_CRYPTO_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
/* gpukit codes: gpukit/include/kinet/gpukit/gpukit.h:38-46 */
#define KB200_GPUKIT_OK 0
#define KB200_GPUKIT_ERR_NULL_ARG -1
#define KB200_GPUKIT_ERR_BAD_SIZE -2
#define KB200_GPUKIT_ERR_BACKEND -3
#define KB200_GPUKIT_ERR_DISPATCH -4
#define KB200_GPUKIT_ERR_NOTIMPL -5
/* crypto.h codes: c-abi/crypto.h:60-66 */
#define KB200_CRYPTO_OK 0
#define KB200_CRYPTO_ERR_INPUT -1
#define KB200_CRYPTO_ERR_LENGTH -2
#define KB200_CRYPTO_ERR_VERIFY -3
#define KB200_CRYPTO_ERR_BACKEND -4
#define KB200_CRYPTO_ERR_NOTIMPL -5
#define KB200_CRYPTO_ERR_INTERNAL -6

/* Curve ids: gpukit_curve, gpukit/include/kinet/gpukit/multi_pippenger.h:51-56 */
#define KB200_CURVE_BN254_G1 1
#define KB200_CURVE_BLS12_381_G1 2

/* ---- MSM: drop-in for gpukit ------------------------------------------- */

/* result = sum_i scalars[i] * points[i].
 * Replaces gpukit_multi_pippenger (gpukit/c-abi/c_multi_pippenger.cpp:9-41,
 * declared at gpukit/include/kinet/gpukit/multi_pippenger.h:69-91) with a
 * GPU-only body: same argument order and meaning, same wire formats, same
 * null checks first, n == 0 gives the all-zero identity, and output bytes
 * equal gpukit_multi_pippenger_cpu's (multi_pippenger.cpp:356-405) for every
 * input, including its dropped top-window carry for scalars >= 2^255 when
 * its window size is 4 or 8.  Curves: BN254 G1 (1) and BLS12-381 G1 (2);
 * secp256k1 (0) and banderwagon (3) return GPUKIT_ERR_NOTIMPL so the
 * reference dispatcher's CPU fallback still covers them; unknown ids return
 * GPUKIT_ERR_BACKEND as the CPU body does.  Points must be on the curve
 * (neither implementation checks; off-curve input is undefined).  Like the
 * reference's reader (gpukit/curve_traits/bls12_381_g1_first_party_traits.h:
 * 58-69), no subgroup check is made and none is needed: a BLS12-381 point
 * outside G1 gets the same bytes as from the reference.  (BN254 sums use
 * the GLV endomorphism, which acts as [lambda] on every BN254 point:
 * cofactor 1.) */
int gpukit_multi_pippenger(uint32_t curve, const uint8_t* scalars, const uint8_t* points,
                           size_t n, uint8_t* result);

/* The CUDA body the reference declares at multi_pippenger.h:81-85 (and stubs
 * to NOTIMPL at gpukit/gpu/cuda/multi_pippenger.cu:38-44).  Same contract. */
int gpukit_multi_pippenger_cuda(uint32_t curve, const uint8_t* scalars,
                                const uint8_t* points, size_t n, uint8_t* result);

/* New (no reference counterpart): gpukit_multi_pippenger for callers that
 * know every point lies in the prime-order subgroup G1 -- points they
 * validated, an SRS, multiples of the generator.  The BLS12-381 sum then
 * uses the GLV endomorphism phi(x, y) = (beta x, y) = [lambda](x, y), which
 * holds on G1 only: half the windows over twice the points, half the
 * buckets.  For G1 points the bytes equal gpukit_multi_pippenger's; for a
 * curve point outside G1 the result is unspecified (use
 * gpukit_multi_pippenger).  BN254: identical to gpukit_multi_pippenger. */
int gpukit_multi_pippenger_subgroup(uint32_t curve, const uint8_t* scalars,
                                    const uint8_t* points, size_t n, uint8_t* result);

/* ---- EIP-4844 blobs (replaces kzg_blob_to_commit / kzg_commit_to_proof,
 * crypto.h:238-239, bodies kzg/c-abi/c_kzg_blob.cpp:26-43) ------------------ */

/* The reference embeds the mainnet trusted setup and evaluates through
 * c-kzg-4844.  Here the setup is loaded once per device: the setup's 4096
 * G1 Lagrange points, 48-byte compressed, in the trusted-setup file's order
 * (natural order of the roots of unity; they are kept bit-reversed, as
 * c-kzg does).  Each point is checked (encoding, curve, G1).  Returns
 * CRYPTO_OK, CRYPTO_ERR_LENGTH (n != 4096), CRYPTO_ERR_INPUT (a bad point;
 * the setup is then unusable until a good load). */
int kzg_blob_setup_load_g1_lagrange(const uint8_t* points48, size_t n);
/* Test setup [L_i(tau)]G1 for a 32-byte little-endian tau. */
int kzg_blob_setup_generate(const uint8_t tau32le[32]);
/* EIP-4844 blob_to_kzg_commitment: blob = 4096 big-endian field elements,
 * element i the polynomial's value at w^brp(i) (w = 7^((r-1)/4096)); commit
 * = 48-byte compressed [p(tau)]G1.  CRYPTO_ERR_INPUT for null pointers, an
 * element not below r, or no loaded setup. */
int kzg_blob_to_commit(const uint8_t blob[131072], uint8_t commit[48]);
/* EIP-4844 compute_kzg_proof(blob, z): y = p(z) (32 B big-endian) and the
 * 48-byte compressed proof [(p(X) - y)/(X - z) at tau]G1; z is 32 B
 * big-endian below r (a domain point is allowed).  Same errors. */
int kzg_commit_to_proof(const uint8_t blob[131072], const uint8_t z[32], uint8_t proof[48],
                        uint8_t y[32]);

/* ---- EIP-2537 G1 MSM (replaces bls12_381_g1_msm, bls/c-abi/c_bls_pairing.h:
 * 153-156, body bls/cpp/bls.cpp:194-254) ----------------------------------- */

/* BLS12_G1MSM: xycs holds N entries of x[64] || y[64] || c[32], all big
 * endian, size = 160 N.  Each coordinate must be below p (so its top 16
 * bytes are zero), each point on the curve and in G1; (0,0) is the point at
 * infinity and is skipped.  The scalar is any 256-bit value.  Writes the sum
 * as rx, ry (16 zero bytes then the 48-byte big-endian coordinate; (0,0) for
 * infinity) and returns 1; returns 0 for invalid input (also for size not a
 * multiple of 160, which the reference only asserts, and for null
 * pointers), and CRYPTO_ERR_BACKEND (< 0) when no GPU is usable -- a value
 * the reference's CPU body never returns. */
int bls12_381_g1_msm(uint8_t rx[64], uint8_t ry[64], const uint8_t* xycs, size_t size);

/* ---- Word-prime NTT (replaces ntt_forward/ntt_inverse, crypto.h:368-369,
 * bodies ntt/c-abi/c_ntt.cpp:81-179) --------------------------------------- */

/* In-place transform of n 64-bit words mod `modulus`, with the reference's
 * dispatch and results:
 *   n <= 2^16   : natural order in and out.  modulus 998244353 with root
 *                 629671588 (its 2^16-th root; for the inverse also its
 *                 inverse) selects the reference's Montgomery path with
 *                 w = root^(2^16/n); any other pair the generic path with
 *                 `root` as the n-th root (`root_inv` used as given).
 *   2^16 < n <= 2^20 : six-step; `root` is a 2n-th root, the transform root
 *                 is root^2, and the forward output (= inverse input) is in
 *                 the transposed N2 x N1 layout: word k1*N2 + k2 holds
 *                 X[k1 + N1*k2], N1 = 2^floor(log2(n)/2), N2 = n/N1.
 * The inverse includes the 1/n scaling.  Results match the reference for
 * every input word, reduced or not (so, like the reference, the n <= 2^16
 * generic path does not round-trip for moduli above 2^63: its addition has
 * no overflow check).  Returns CRYPTO_OK, or CRYPTO_ERR_INPUT for a null
 * pointer, n not a power of two, n > 2^20 or modulus 0 (the reference's
 * 2^64 sentinel, which it rejects for every n > 1); CRYPTO_ERR_BACKEND
 * without a usable GPU. */
int ntt_forward(uint64_t* coeffs, size_t n, uint64_t modulus, uint64_t root);
int ntt_inverse(uint64_t* coeffs, size_t n, uint64_t modulus, uint64_t root_inv);

/* ---- Fr NTT (new; same style as ntt_forward/ntt_inverse, crypto.h:368-369) */

/* In-place transform of n canonical Fr elements (32 B LE each), natural
 * order in and out.  forward: X_k = sum_j x_j w^(jk); inverse: x_j = n^-1
 * sum_k X_k w^(-jk); w = g^((r-1)/n), g = 7 (BLS12-381) or 5 (BN254).
 * coset != 0 evaluates on g*H: forward pre-multiplies x_j by g^j, inverse
 * post-multiplies by g^-j.  Inputs are reduced mod r.  n must be a power of
 * two up to 2^28.  Returns CRYPTO_OK, CRYPTO_ERR_INPUT (null / bad curve),
 * CRYPTO_ERR_LENGTH (bad n) or CRYPTO_ERR_BACKEND. */
int ntt_fr_forward(int curve, uint8_t* coeffs32le, size_t n, int coset);
int ntt_fr_inverse(int curve, uint8_t* coeffs32le, size_t n, int coset);

/* ---- KZG over BLS12-381 with a resident SRS (new) ---------------------- */

/* Load n monomial-basis SRS points [tau^i]G1 (96 B BE each) into device
 * memory, replacing any resident SRS.  The reference loads its setup once
 * per process (kzg/cpp/kzg_blob.cpp:23-65); this is the resident analogue.
 * Both SRS calls also build the shifted tables commits select and size the
 * per-call commit buffers (one commit of zeros per power of two up to n), so
 * later kzg_commit_fr calls allocate nothing. */
int kzg_srs_load_g1(const uint8_t* points96be, size_t n);
/* Build the synthetic SRS [tau^i]G1, i < n, on the device from a 32-byte LE
 * tau (reduced mod r).  For tests and benchmarks. */
int kzg_srs_generate_g1(const uint8_t tau32le[32], size_t n);
/* Copy `count` resident SRS points starting at `offset` back to the host. */
int kzg_srs_read_g1(uint8_t* points96be, size_t offset, size_t count);
/* Number of resident SRS points (0 if none). */
size_t kzg_srs_size(void);

/* commit = [p(tau)]G1 for the polynomial p given by n evaluations
 * (32 B LE Fr) at the n-th roots of unity, natural order: an inverse NTT to
 * monomial coefficients, an MSM against the resident SRS, then the 48-byte
 * compressed encoding.  n must be a power of two <= kzg_srs_size().  Returns
 * CRYPTO_ERR_LENGTH if the SRS is too short or n is not a power of two. */
int kzg_commit_fr(const uint8_t* evals32le, size_t n, uint8_t commit48[48]);

/* `count` independent commits in one batched pass.  Polynomial c has
 * sizes[c] evaluations, stored back to back in evals32le (in order);
 * commits48 receives 48 * count bytes.  Byte-equal to count kzg_commit_fr
 * calls. */
int kzg_commit_batch(const uint8_t* evals32le, const size_t* sizes, size_t count,
                     uint8_t* commits48);

/* ---- Served commits (continuous batching, new) -------------------------- */
/* A request server over the resident SRS (which must stay loaded while the
 * server lives).  Requests are admitted into batches as execution slots and
 * device memory free up; batches on different slots overlap on the device.
 * max_batch: requests per batch (0 = 64); slots: concurrent batches
 * (0 = 2); mem_budget_bytes: cap on a batch's computed device footprint
 * (0 = free device memory).  Creation builds, once per SRS, the shifted SRS
 * tables the commit sizes use (up to three window sizes; about 5 GB and
 * well under a second for a 2^20 SRS) and runs one warm-up batch per slot,
 * so no request waits for a table build or a buffer to grow.
 * Returns NULL on failure (kb200_last_error). */
void* kzg_server_create(size_t max_batch, int slots, size_t mem_budget_bytes);
/* Queue one polynomial (n evaluations, 32 B LE); *ticket identifies it. */
int kzg_server_submit(void* server, const uint8_t* evals32le, size_t n, uint64_t* ticket);
/* Wait for a ticket (timeout_ms < 0: no limit).  0 = done (commit48 and
 * latency filled, ticket released), 1 = timed out, < 0 = error. */
int kzg_server_wait(void* server, uint64_t ticket, uint8_t commit48[48], double* latency_ms,
                    double timeout_ms);
/* p50 / p99 submit-to-completion latency and sustained commits/s. */
int kzg_server_stats(void* server, double* p50_ms, double* p99_ms, double* commits_per_s,
                     uint64_t* completed, int reset);
int kzg_server_destroy(void* server);

/* ---- Allocation-free Fr NTT -------------------------------------------- */
/* No counterpart in the reference.  ntt_fr_forward / ntt_fr_inverse grow
 * their device scratch with cudaMalloc the first time they meet a size.
 * Some callers cannot allow that: a process whose device memory is reserved
 * up front by another allocator (a framework's caching pool, a fixed
 * arena), where cudaMalloc fails or fragments that reservation, or a
 * latency-bound service that cannot afford the device-wide waits of
 * cudaMalloc and cudaFree.  This entry point computes the same transform
 * (inverse != 0: ntt_fr_inverse's) for n <= 2^16 with all its scratch in
 * one fixed 6.8 MB file-scope device array, which every GPU that loads this
 * library holds until the process exits, and calls no cudaMalloc, cudaFree
 * or allocating library routine.  n > 2^16 returns CRYPTO_ERR_LENGTH.  The
 * first call on a device looks up the array's device address for that
 * device (cudaGetSymbolAddress) and should come before any stream capture.
 * The call is synchronous: it copies the host buffer in and out and runs
 * its kernels on the legacy default stream.  All calls share the one
 * array, so calls that overlap on the GPU (from several host threads) race;
 * callers must serialise them. */
int ntt_fr_transform_noalloc(int curve, uint8_t* coeffs32le, size_t n, int inverse, int coset);

/* ---- Device-pointer entry points (inputs already resident in HBM) ------ */
/* Pointers are device pointers (16-byte aligned), `stream` is a
 * cudaStream_t (NULL = legacy default stream); work is queued, not
 * synchronised.  Calls sharing a device must not overlap across streams. */
int kb200_msm_device(uint32_t curve, const void* d_scalars, const void* d_points, size_t n,
                     void* d_result, void* stream);
/* kb200_msm_device with the G1 promise of gpukit_multi_pippenger_subgroup. */
int kb200_msm_device_subgroup(uint32_t curve, const void* d_scalars, const void* d_points,
                              size_t n, void* d_result, void* stream);
/* bls12_381_g1_msm on device memory: d_out_wire96 receives x || y (48 B BE
 * each, zeros for infinity), d_status one 32-bit word: 0 valid, 1 invalid. */
int kb200_bls12_381_g1_msm_device(const void* d_xycs, size_t size, void* d_out_wire96,
                                  void* d_status, void* stream);
/* ntt_forward (inverse = 0) / ntt_inverse (inverse = 1) on device words;
 * d_scratch (n words) is needed for 2^11 < n <= 2^16. */
int kb200_word_ntt_device(void* d_coeffs, void* d_scratch, size_t n, uint64_t modulus,
                          uint64_t root, int inverse, void* stream);
int kb200_ntt_device(int curve, void* d_data, size_t n, int inverse, int coset, size_t batch,
                     void* stream);
/* d_out_points[i] = d_scalars[i] * G1 (wire encoding), fixed-base windows. */
int kb200_g1_fixed_base_device(uint32_t curve, const void* d_scalars, size_t n,
                               void* d_out_points, void* stream);
/* d_out[i] = tau^i (32 B LE Fr). */
int kb200_fr_powers_device(int curve, const void* d_tau, size_t n, void* d_out, void* stream);
/* KZG commit on device buffers against the resident SRS (evals are consumed:
 * the buffer is transformed in place). */
int kb200_kzg_commit_device(void* d_evals, size_t n, void* d_commit48, void* stream);

/* ---- Seeded synthetic inputs (host only, no GPU needed) ---------------- */
/* xorshift64* streams; uniform Fr by rejection sampling of 255-bit (BLS12-381)
 * or 254-bit (BN254) draws.  kind: 0 = uniform in [0, r); 1 = skewed
 * (25% zero, 25% one, 20% uniform below 2^64, 30% uniform in [0, r)). */
int kb200_gen_scalars(int curve, uint64_t seed, size_t n, int kind, uint8_t* out32le);

/* ---- Autotuner (new) --------------------------------------------------- */
/* Time, for log2 sizes in [log_lo, log_hi] on this GPU: MSM window widths
 * around the cost model's choice (256-bit windows, and the windows of GLV
 * halves), NTT first-pass radix splits, and -- for BLS12-381 with a
 * resident SRS -- the shifted-table window (13, 16 or 19) of single KZG
 * commits, which batched and served commits use per commit.  Keeps the
 * fastest, appends them to cache_path (keyed by GPU name and driver
 * version).  Returns size classes tuned or < 0. */
int kb200_autotune(uint32_t curve, int log_lo, int log_hi, const char* cache_path);
/* Apply the cached entries that match this GPU; returns entries applied. */
int kb200_autotune_load(const char* cache_path);
/* kind 0 = MSM window bits (256-bit windows), 1 = NTT first-pass log radix,
 * 2 = MSM window bits of GLV halves, 3 = commit window (BLS12-381 only);
 * 0 = untuned. */
int kb200_tune_get(int kind, uint32_t curve, int log_n);
void kb200_tune_set(int kind, uint32_t curve, int log_n, int value);

/* ---- Introspection ------------------------------------------------------ */
const char* kb200_last_error(void);
/* 1 if a CUDA device is usable, else 0. */
int kb200_device_available(void);
/* Window size the MSM planner picks for n on gpukit_multi_pippenger's path
 * (for tests of the planner; on BN254 the window of the GLV halves), and on
 * the G1-promise path of gpukit_multi_pippenger_subgroup (GLV halves on both
 * curves). */
int kb200_msm_window(uint32_t curve, size_t n);
int kb200_msm_window_subgroup(uint32_t curve, size_t n);
/* Expected bucket additions of one n-point MSM on those two paths (entries
 * of non-zero digits: points x populated windows x (1 - 2^-c)). */
double kb200_msm_entries(uint32_t curve, size_t n);
double kb200_msm_entries_subgroup(uint32_t curve, size_t n);
/* Device self-check of the field inversion used throughout (binary GCD)
 * against the Fermat chain a^(p-2), plus x * x^-1 = 1, over `count` elements
 * (edge values, then seeded pseudo-random ones) of field 0 = BLS12-381 Fp,
 * 1 = BLS12-381 Fr, 2 = BN254 Fp, 3 = BN254 Fr.  *mismatches receives the
 * number of failing elements.  Diagnostic: no reference counterpart. */
int kb200_field_inverse_check(int field, uint64_t seed, size_t count, unsigned long long* mismatches);
/* Device products of n canonical little-endian elements of the same fields
 * (48 B for BLS12-381 Fp, 32 B otherwise): out_mul[i] = a[i] * b[i] and
 * out_sqr[i] = a[i]^2, computed in Montgomery form by the Karatsuba product
 * and squaring every kernel uses; *form_mismatches counts elements where the
 * interleaved (CIOS) product disagrees.  Diagnostic: no reference
 * counterpart. */
int kb200_field_mul_check(int field, const uint8_t* a_le, const uint8_t* b_le, size_t n,
                          uint8_t* out_mul_le, uint8_t* out_sqr_le,
                          unsigned long long* form_mismatches);
/* Number of this library's kernel launches since load. */
unsigned long long kb200_launch_count(void);
/* Per-stage CUDA-event timing of MSMs (off by default). */
void kb200_profile_enable(int on);
/* Stage times (ms) of the last MSM on this device for the curve, in order:
 * wire->table, recode (with the ranking of the sort), sort (scan and
 * scatter), pairing levels, accumulation, fold, reduction (both stages),
 * combine.  Returns the number written (0 if none recorded), or -1. */
int kb200_msm_stage_ms(uint32_t curve, float* out, int max);

#ifdef __cplusplus
}
#endif
#endif
