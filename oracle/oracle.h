/*
 * CPU oracle for the polynomial-commitment path (TEST INFRASTRUCTURE ONLY).
 *
 * This library is a plain-C restatement of the reference's CPU algorithms for
 * the Fr NTT, the G1 Pippenger MSM, the compressed-G1 encoder and the KZG
 * commit composition, over BLS12-381 and BN254.  It is the checker: only the
 * test suite, the smoke check and the CPU-baseline leg of the benchmark load
 * it.  The product library never links or calls it.
 *
 * Pinning: the MSM restatement is checked byte-for-byte against the
 * reference's own gpukit_multi_pippenger_cpu, compiled unmodified from the
 * reference sources into oracle/_ref/ (see oracle/Makefile), and against the
 * committed fixtures under tests/golden/ that the same build produced.  The
 * compressed encoder is pinned by the reference's own vectors
 * (kzg/test/kzg_test.cpp:38-42 for infinity, :64-81 for the generator).  The
 * Fr NTT has no reference implementation (the reference's NTTs are
 * word-prime only); it is pinned by an O(n^2) DFT, round trips and Horner
 * evaluation, which is "parity unpinned" with respect to reference vectors.
 *
 * Encodings (all canonical, never Montgomery, at this boundary):
 *   Fr element   : 32 bytes little-endian.
 *   G1 affine    : x || y, each big-endian (48 B for BLS12-381, 32 B for
 *                  BN254); the all-zero encoding is the point at infinity.
 *   compressed G1: 48 bytes, ZCash/IETF flags (BLS12-381 only).
 */
#ifndef KINET_B200_ORACLE_H
#define KINET_B200_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Curve ids follow gpukit_curve (gpukit/include/kinet/gpukit/multi_pippenger.h:51-56). */
#define ORC_CURVE_BN254 1
#define ORC_CURVE_BLS12_381 2

/* Field-level helpers, exposed so tests can cross-check device arithmetic.
 * which: 0 = BLS12-381 Fp, 1 = BLS12-381 Fr, 2 = BN254 Fp, 3 = BN254 Fr.
 * Operands are canonical little-endian byte strings of the field width
 * (48 B for BLS12-381 Fp, 32 B otherwise). */
int orc_field_mul(int which, const uint8_t* a, const uint8_t* b, uint8_t* out);
int orc_field_inv(int which, const uint8_t* a, uint8_t* out);

/* Pippenger MSM restated from gpukit/cpp/cpu_reference/multi_pippenger.cpp:67-181
 * and :356-405: scalars n x 32 B LE, points n x (64|96) B BE affine,
 * result (64|96) B BE affine.  Returns 0 or a gpukit status code. */
int orc_msm(uint32_t curve, const uint8_t* scalars, const uint8_t* points,
            size_t n, uint8_t* result);

/* Naive sum of scalar multiplications (double-and-add per point), the
 * reference harness's oracle shape (gpukit/test/multi_pippenger_test.cpp:375-405). */
int orc_msm_naive(uint32_t curve, const uint8_t* scalars, const uint8_t* points,
                  size_t n, uint8_t* result);

/* k * G for the curve generator, k 32 B LE; result BE affine. */
int orc_g1_mul_gen(uint32_t curve, const uint8_t* k_le, uint8_t* result);
/* k * P for an arbitrary affine point P (BE), k 32 B LE. */
int orc_g1_mul(uint32_t curve, const uint8_t* point, const uint8_t* k_le,
               uint8_t* result);
/* P + Q in affine BE form. */
int orc_g1_add(uint32_t curve, const uint8_t* p, const uint8_t* q, uint8_t* result);
/* 1 if the (BE affine) point is on the curve or is the all-zero infinity. */
int orc_g1_on_curve(uint32_t curve, const uint8_t* p);

/* Fr NTT in place on n canonical 32 B LE elements.  Natural order in and out.
 *   inverse = 0 : X_k = sum_j x_j * w^(jk)                 (coset: x_j * g^j first)
 *   inverse = 1 : x_j = n^-1 sum_k X_k * w^(-jk)            (coset: result * g^-j)
 * w = g^((r-1)/n) with g = 7 (BLS12-381 Fr) or g = 5 (BN254 Fr); the coset
 * shift is g itself.  Inputs are reduced mod r first.  Radix-2 DIT in the
 * order of ntt/cpp/ntt.cpp:128-172.  Returns 0, or -2 if n is not a power of
 * two within the field's 2-adicity. */
int orc_ntt(uint32_t curve, uint8_t* data, size_t n, int inverse, int coset);
/* O(n^2) DFT with the same contract, used to pin orc_ntt at small sizes. */
int orc_dft(uint32_t curve, uint8_t* data, size_t n, int inverse, int coset);
/* w_n (canonical 32 B LE) for the given size. */
int orc_root_of_unity(uint32_t curve, size_t n, uint8_t* out);

/* ZCash/IETF compressed encoding of a BLS12-381 G1 affine point (96 B BE in,
 * all-zero = infinity) into 48 bytes. */
int orc_g1_compress(const uint8_t* point96, uint8_t* out48);

/* KZG commit of n evaluations (32 B LE each, at the n-th roots of unity in
 * natural order) against the monomial SRS [tau^i]G1 (n x 96 B BE):
 * iNTT -> MSM -> compress.  BLS12-381 only. */
int orc_kzg_commit(const uint8_t* evals, size_t n, const uint8_t* srs,
                   uint8_t* commit48);

/* Fr helpers: powers tau^0..tau^(n-1) (canonical 32 B LE), and a*b mod r. */
int orc_fr_powers(uint32_t curve, const uint8_t* tau, size_t n, uint8_t* out);

/* EIP-2537 BLS12_G1MSM with the contract of the reference's
 * bls12_381_g1_msm (bls/c-abi/c_bls_pairing.h:155, bls/cpp/bls.cpp:194-254):
 * xycs = N x (x[64] || y[64] || c[32]) big-endian, size = 160 N; returns 1
 * with rx, ry (64 B each, 16 zero bytes then 48 B BE) or 0 if any point is
 * out of range, off the curve or outside G1.  (0,0) is infinity and is
 * skipped. */
int orc_bls12_381_g1_msm(uint8_t rx[64], uint8_t ry[64], const uint8_t* xycs, size_t size);

/* EIP-4844 blob commitment / opening proof (kzg/c-abi/c_kzg_blob.cpp:26-43)
 * against a monomial setup srs = [tau^i]G1, i < 4096 (96 B BE each): blob =
 * 4096 x 32 B big-endian elements in bit-reversed evaluation order; z and y
 * 32 B big-endian; commitment and proof 48 B compressed.  Returns 0, or -1
 * if an element or z is not below r. */
int orc_kzg_blob_commit(const uint8_t* blob_be, const uint8_t* srs, uint8_t commit48[48]);
int orc_kzg_blob_proof(const uint8_t* blob_be, const uint8_t z_be[32], const uint8_t* srs,
                       uint8_t proof48[48], uint8_t y_be[32]);

/* Word-prime NTT with the contract of the reference's ntt_forward /
 * ntt_inverse (ntt/c-abi/c_ntt.cpp:81-179): in place on n uint64 words;
 * n <= 2^16 natural order (Cyclone prime 998244353 with its pinned root on
 * the Montgomery path, anything else on the generic path, root = n-th root);
 * 2^16 < n <= 2^20 six-step with output in the transposed N2 x N1 layout,
 * root = 2n-th root.  Returns 0 or -1 (CRYPTO_ERR_INPUT).  word_ntt.c. */
int orc_word_ntt_forward(uint64_t* a, size_t n, uint64_t q, uint64_t root);
int orc_word_ntt_inverse(uint64_t* a, size_t n, uint64_t q, uint64_t root_inv);

/* Seeded scalars with the contract of the library's kb200_gen_scalars
 * (xorshift64*; kind 0 uniform in [0, r), 1 skewed), restated so CPU-only
 * code builds the same workload.  32 B LE each. */
int orc_gen_scalars(uint32_t curve, uint64_t seed, size_t n, int kind, uint8_t* out);
/* out[i] = k_i * G (BE affine, all-zero for infinity) for n scalars k_i
 * (32 B LE), fixed-base 8-bit windows, `threads` POSIX threads. */
int orc_g1_fixed_base_batch(uint32_t curve, const uint8_t* scalars_le, size_t n,
                            uint8_t* out, int threads);

#ifdef __cplusplus
}
#endif
#endif
