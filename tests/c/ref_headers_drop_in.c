/* Compiles against the reference's own C headers and links the B200 library:
 * a caller written for the reference (c-abi/crypto.h,
 * gpukit/include/kinet/gpukit/multi_pippenger.h, bls/c-abi/c_bls_pairing.h)
 * builds and runs unchanged.  The reference's headers declare some symbols
 * differently from one another (bls_aggregate_verify in crypto.h and
 * c_bls_pairing.h), so each is used in its own translation unit: this file
 * is compiled once per header (PART_CRYPTO, PART_GPUKIT, PART_BLS) and once
 * more for main (PART_MAIN).  With KB200_BOTH_HEADERS each part also
 * includes the library's header, so every declaration they share must be
 * type-compatible.  Only argument checks run (no device needed): each call
 * returns the reference's documented error code for its bad argument. */
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#if defined(PART_CRYPTO)
#include "crypto.h"
#elif defined(PART_GPUKIT)
#include "kinet/gpukit/multi_pippenger.h"
#elif defined(PART_BLS)
#include "c_bls_pairing.h"
#endif
#if defined(KB200_BOTH_HEADERS) && !defined(PART_MAIN)
#include "kinet_b200/crypto_b200.h"
#endif

#define EXPECT(expr, want)                                                         \
    do {                                                                           \
        int got_ = (expr);                                                         \
        if (got_ != (want)) {                                                      \
            printf("FAIL %s = %d, want %d\n", #expr, got_, (int)(want));           \
            ++fails;                                                               \
        }                                                                          \
    } while (0)

#if defined(PART_CRYPTO)
int check_crypto(void) {
    int fails = 0;
    uint8_t out[48], proof[48], y[32], z[32];
    uint64_t words[4] = {1, 2, 3, 4};
    memset(z, 0, sizeof z);
    EXPECT(ntt_forward(NULL, 4, 998244353ull, 3ull), CRYPTO_ERR_INPUT);
    EXPECT(ntt_inverse(words, 3, 998244353ull, 3ull), CRYPTO_ERR_INPUT);
    EXPECT(kzg_blob_to_commit(NULL, out), CRYPTO_ERR_INPUT);
    EXPECT(kzg_commit_to_proof(NULL, z, proof, y), CRYPTO_ERR_INPUT);
    return fails;
}
#elif defined(PART_GPUKIT)
/* The dispatcher's definition (gpukit/c-abi/c_multi_pippenger.cpp:9), which
 * no reference header declares. */
int gpukit_multi_pippenger(uint32_t curve, const uint8_t* scalars, const uint8_t* points,
                           size_t n, uint8_t* result);
int check_gpukit(void) {
    int fails = 0;
    uint8_t out[96];
    /* null checks first (c_multi_pippenger.cpp:14-15): GPUKIT_ERR_NULL_ARG */
    EXPECT(gpukit_multi_pippenger(GPUKIT_CURVE_BLS12_381_G1, NULL, NULL, 4, out), -1);
    EXPECT(gpukit_multi_pippenger_cuda(GPUKIT_CURVE_BN254_G1, NULL, NULL, 4, out), -1);
    EXPECT(gpukit_multi_pippenger(GPUKIT_CURVE_BLS12_381_G1, out, out, 1, NULL), -1);
    return fails;
}
#elif defined(PART_BLS)
int check_bls(void) {
    int fails = 0;
    uint8_t rx[64], ry[64], buf[7];
    memset(buf, 0, sizeof buf);
    /* EIP-2537: 0 = invalid input */
    EXPECT(bls12_381_g1_msm(rx, ry, NULL, 160), 0);
    EXPECT(bls12_381_g1_msm(rx, ry, buf, 7), 0);
    return fails;
}
#elif defined(PART_MAIN)
int check_crypto(void);
int check_gpukit(void);
int check_bls(void);
int main(void) {
    const int fails = check_crypto() + check_gpukit() + check_bls();
    if (fails) return 1;
    printf("ok\n");
    return 0;
}
#endif
