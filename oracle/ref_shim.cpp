// Thin C wrapper over the reference's own CPU code (TEST INFRASTRUCTURE ONLY).
//
// Compiled by oracle/Makefile together with the reference's unmodified
// sources (gpukit/cpp/cpu_reference/multi_pippenger.cpp, gpukit.cpp and the
// banderwagon files that translation unit links against) into
// oracle/_ref/libref_msm.so.  Nothing here re-implements reference
// arithmetic: every group operation below calls the reference headers.
//
//   ref_msm          -> gpukit_multi_pippenger_cpu, as shipped (1 thread).
//   ref_msm_parallel -> the same function on T contiguous slices in T threads,
//                       the slice results summed with the reference g1_add.
//                       By the group law this is byte-identical to ref_msm;
//                       it is "the reference parallelised by composition",
//                       not threading the reference itself has.
//   ref_g1_mul_gen   -> the reference Montgomery ladder on the generator
//                       (bls/cpp/bls12_381_g1.hpp:171-193,
//                        bn254/cpp/bn254_g1.hpp:184-206).
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "kinet/gpukit/gpukit.h"
#include "kinet/gpukit/multi_pippenger.h"
#include "bls/cpp/bls12_381_g1.hpp"
#include "bn254/cpp/bn254_g1.hpp"

namespace {

namespace bls = kinet::crypto::bls12_381;
namespace bn = kinet::crypto::bn254;

bls::G1Jac bls_read(const uint8_t* xy) {
    bool any = false;
    for (int i = 0; i < 96; ++i) any |= xy[i] != 0;
    if (!any) return bls::g1_jac_zero();
    bls::G1Affine a;
    a.x = bls::to_mont_fp(bls::U384::from_be48(xy));
    a.y = bls::to_mont_fp(bls::U384::from_be48(xy + 48));
    a.infinity = false;
    return bls::g1_to_jac(a);
}
void bls_write(const bls::G1Jac& p, uint8_t* xy) {
    bls::G1Affine a = bls::g1_to_affine(p);
    if (a.infinity) { std::memset(xy, 0, 96); return; }
    bls::from_mont_fp(a.x).to_be48(xy);
    bls::from_mont_fp(a.y).to_be48(xy + 48);
}
bn::G1Jac bn_read(const uint8_t* xy) {
    bool any = false;
    for (int i = 0; i < 64; ++i) any |= xy[i] != 0;
    if (!any) return bn::g1_jac_zero();
    bn::G1Affine a;
    a.x = bn::to_mont_fp(bn::U256::from_be32(xy));
    a.y = bn::to_mont_fp(bn::U256::from_be32(xy + 32));
    a.infinity = false;
    return bn::g1_to_jac(a);
}
void bn_write(const bn::G1Jac& p, uint8_t* xy) {
    bn::G1Affine a = bn::g1_to_affine(p);
    if (a.infinity) { std::memset(xy, 0, 64); return; }
    bn::from_mont_fp(a.x).to_be32(xy);
    bn::from_mont_fp(a.y).to_be32(xy + 32);
}

}  // namespace

extern "C" {

int ref_msm(uint32_t curve, const uint8_t* scalars, const uint8_t* points,
            size_t n, uint8_t* result) {
    return gpukit_multi_pippenger_cpu(curve, scalars, points, n, result);
}

int ref_msm_parallel(uint32_t curve, const uint8_t* scalars, const uint8_t* points,
                     size_t n, uint8_t* result, int threads) {
    if (curve != GPUKIT_CURVE_BLS12_381_G1 && curve != GPUKIT_CURVE_BN254_G1)
        return GPUKIT_ERR_BACKEND;
    const size_t pb = curve == GPUKIT_CURVE_BLS12_381_G1 ? 96 : 64;
    if (threads < 1) threads = 1;
    if ((size_t)threads > n) threads = n ? (int)n : 1;
    std::vector<std::vector<uint8_t>> parts(threads, std::vector<uint8_t>(pb));
    std::vector<int> rcs(threads, 0);
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) {
        const size_t lo = n * t / threads, hi = n * (t + 1) / threads;
        pool.emplace_back([&, t, lo, hi] {
            rcs[t] = gpukit_multi_pippenger_cpu(curve, scalars + 32 * lo,
                                                points + pb * lo, hi - lo,
                                                parts[t].data());
        });
    }
    for (auto& th : pool) th.join();
    for (int rc : rcs) if (rc) return rc;
    if (curve == GPUKIT_CURVE_BLS12_381_G1) {
        bls::G1Jac acc = bls::g1_jac_zero();
        for (auto& p : parts) acc = bls::g1_add(acc, bls_read(p.data()));
        bls_write(acc, result);
    } else {
        bn::G1Jac acc = bn::g1_jac_zero();
        for (auto& p : parts) acc = bn::g1_add(acc, bn_read(p.data()));
        bn_write(acc, result);
    }
    return GPUKIT_OK;
}

int ref_g1_mul_gen(uint32_t curve, const uint8_t* k_le, uint8_t* result) {
    if (curve == GPUKIT_CURVE_BLS12_381_G1) {
        uint64_t k[4];
        for (int l = 0; l < 4; ++l) {
            uint64_t v = 0;
            for (int b = 0; b < 8; ++b) v |= (uint64_t)k_le[8 * l + b] << (8 * b);
            k[l] = v;
        }
        bls_write(bls::g1_scalar_mul_256(bls::g1_generator(), k), result);
        return 0;
    }
    if (curve == GPUKIT_CURVE_BN254_G1) {
        bn::U256 k;
        for (int l = 0; l < 4; ++l) {
            uint64_t v = 0;
            for (int b = 0; b < 8; ++b) v |= (uint64_t)k_le[8 * l + b] << (8 * b);
            k.limbs[l] = v;
        }
        bn::G1Affine g;
        g.x = bn::to_mont_fp(bn::U256{1, 0, 0, 0});
        g.y = bn::to_mont_fp(bn::U256{2, 0, 0, 0});
        g.infinity = false;
        bn_write(bn::g1_scalar_mul(g, k), result);
        return 0;
    }
    return GPUKIT_ERR_BACKEND;
}

}  // extern "C"
