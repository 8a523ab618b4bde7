// Seeded synthetic inputs (host only).  xorshift64* streams, the generator
// family the reference's determinism harnesses use
// (kzg/test/kzg_gpu_determinism_test.cpp:29-36); uniform Fr by rejection
// sampling so that every value is canonical and below r.
#include "../../include/kinet_b200/crypto_b200.h"

#include <cstdint>
#include <cstring>

namespace {

struct XorShift64Star {
    uint64_t x;
    explicit XorShift64Star(uint64_t seed) : x(seed ^ 0x9E3779B97F4A7C15ull) {
        if (x == 0) x = 0x2545F4914F6CDD1Dull;
    }
    uint64_t next() {
        x ^= x >> 12;
        x ^= x << 25;
        x ^= x >> 27;
        return x * 0x2545F4914F6CDD1Dull;
    }
};

// r for each scalar field, 4 little-endian 64-bit words.
// BLS12-381: kzg/cpp/kzg_oracle.hpp:66-71; BN254: bn254/cpp/bn254_fp.hpp:79-81.
const uint64_t R_BLS[4] = {0xFFFFFFFF00000001ull, 0x53BDA402FFFE5BFEull, 0x3339D80809A1D805ull,
                           0x73EDA753299D7D48ull};
const uint64_t R_BN[4] = {0x43E1F593F0000001ull, 0x2833E84879B97091ull, 0xB85045B68181585Dull,
                          0x30644E72E131A029ull};

bool less_than(const uint64_t a[4], const uint64_t b[4]) {
    for (int i = 3; i >= 0; --i) {
        if (a[i] < b[i]) return true;
        if (a[i] > b[i]) return false;
    }
    return false;
}

void put_le(uint8_t* out, const uint64_t w[4]) {
    for (int i = 0; i < 4; ++i)
        for (int b = 0; b < 8; ++b) out[8 * i + b] = (uint8_t)(w[i] >> (8 * b));
}

void uniform_fr(XorShift64Star& g, int curve, uint64_t w[4]) {
    const uint64_t* r = curve == 2 ? R_BLS : R_BN;
    const uint64_t top_mask = curve == 2 ? 0x7FFFFFFFFFFFFFFFull : 0x3FFFFFFFFFFFFFFFull;
    for (;;) {
        for (int i = 0; i < 4; ++i) w[i] = g.next();
        w[3] &= top_mask;
        if (less_than(w, r)) return;
    }
}

}  // namespace

extern "C" int kb200_gen_scalars(int curve, uint64_t seed, size_t n, int kind, uint8_t* out32le) {
    if (!out32le && n) return KB200_CRYPTO_ERR_INPUT;
    if (curve != 1 && curve != 2) return KB200_CRYPTO_ERR_INPUT;
    if (kind != 0 && kind != 1) return KB200_CRYPTO_ERR_INPUT;
    XorShift64Star g(seed);
    for (size_t i = 0; i < n; ++i) {
        uint64_t w[4] = {0, 0, 0, 0};
        if (kind == 0) {
            uniform_fr(g, curve, w);
        } else {
            const uint64_t u = g.next() % 100;
            if (u < 25) {
                // zero
            } else if (u < 50) {
                w[0] = 1;
            } else if (u < 70) {
                w[0] = g.next();
            } else {
                uniform_fr(g, curve, w);
            }
        }
        put_le(out32le + 32 * i, w);
    }
    return KB200_CRYPTO_OK;
}
