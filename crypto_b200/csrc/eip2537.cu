// EIP-2537 BLS12_G1MSM on the GPU, behind the reference's bls12_381_g1_msm
// (bls/c-abi/c_bls_pairing.cpp:106-110; body bls/cpp/bls.cpp:194-254, which
// hands the work to blst).  One thread per entry checks, as the reference
// does before its Pippenger call:
//   * each coordinate, a 64-byte big-endian integer, is below p
//     (bls.cpp:33-41; so its top 16 bytes are zero);
//   * the point is on y^2 = x^3 + 4, or is (0,0), the EIP-2537 infinity
//     (bls.cpp:44-58);
//   * the point is in G1 (bls.cpp:217-218), by the endomorphism test:
//     P in G1 iff sigma(P) = -[u^2]P, with sigma(x, y) = (beta x, y), beta a
//     cube root of unity in Fp and u = -0xd201000000010000 the curve
//     parameter (M. Scott, "A note on group membership tests for G1, G2 and
//     GT on BLS pairing-friendly curves", 2021);
// then drops infinity entries (bls.cpp:220-222), reduces the big-endian
// scalar mod r (the sum over points of order r is unchanged), and runs the
// G1 MSM of msm.cu on the resulting table.
#include "curve.cuh"
#include "eip2537.cuh"
#include "g1check.cuh"
#include "runtime.cuh"

namespace kb200 {
namespace {

using F = FpBLS;
using FR = FrBLS;

// A 64-byte big-endian coordinate below p (its top 16 bytes zero).
__device__ bool coord_ok(const uint8_t* c, Fe<F>& v) {
    uint32_t hi = 0;
    for (int i = 0; i < 16; ++i) hi |= c[i];
    fe_from_be_bytes(v, c + 16);
    return hi == 0 && below_modulus(v);
}

__global__ void __launch_bounds__(128) k_g1msm_unpack(const uint8_t* __restrict__ xycs, uint32_t n,
                                                      uint32_t* __restrict__ table,
                                                      uint8_t* __restrict__ scalars,
                                                      uint32_t* __restrict__ flag) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint8_t* e = xycs + (size_t)160 * i;
    uint32_t* row = table + (size_t)i * 2 * F::N;
    uint32_t* sc = reinterpret_cast<uint32_t*>(scalars + (size_t)32 * i);
    Fe<F> x, y;
    bool ok = coord_ok(e, x);
    ok = coord_ok(e + 64, y) && ok;
    bool inf = false;
    if (ok) {
        inf = fe_is_zero(x) && fe_is_zero(y);
        if (!inf) {
            Affine<F> a;
            fe_to_mont(a.x, x);
            fe_to_mont(a.y, y);
            ok = g1_on_curve(a) && g1_in_subgroup(a);
            fe_store(row, a.x);
            fe_store(row + F::N, a.y);
        }
    }
    // GLV row n + i: phi(P) = (beta2 x, y) = [lambda]P, valid because every
    // accepted point is in G1 (the subgroup check above)
    uint32_t* grow = row + (size_t)n * 2 * F::N;
    if (!ok) atomicOr(flag, 1u);
    if (!ok || inf) {
        for (int k = 0; k < 2 * F::N; ++k) row[k] = grow[k] = 0;
        row[F::N - 1] = grow[F::N - 1] = INF_FLAG;
        for (int k = 0; k < 8; ++k) sc[k] = 0;
        return;
    }
    {
        Fe<F> bx, b, yy;
        fe_load(bx, row);
        fe_load(yy, row + F::N);
        for (int k = 0; k < F::N; ++k) b.v[k] = kGlvBeta2Mont[k];
        fe_mul(bx, bx, b);
        fe_store(grow, bx);
        fe_store(grow + F::N, yy);
    }
    Fe<FR> s;
    fe_from_be_bytes(s, e + 128);
    while (!below_modulus(s)) {  // at most twice: 2^256 < 3r
        uint32_t b = 0;
        for (int k = 0; k < FR::N; ++k) {
            const uint64_t d = (uint64_t)s.v[k] - FR::P(k) - b;
            s.v[k] = (uint32_t)d;
            b = (uint32_t)(d >> 63);
        }
    }
    for (int k = 0; k < 8; ++k) sc[k] = s.v[k];
}

}  // namespace

void g1_msm_eip2537_device(MsmEngine* eng, const uint8_t* d_xycs, size_t n, uint32_t* d_table,
                           uint8_t* d_scalars, uint32_t* d_flag, uint8_t* d_out_wire,
                           cudaStream_t st) {
    KB_CUDA(cudaMemsetAsync(d_flag, 0, sizeof(uint32_t), st));
    if (n) {
        k_g1msm_unpack<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(d_xycs, (uint32_t)n, d_table,
                                                                     d_scalars, d_flag);
        KB_LAUNCH_CHECK();
    }
    MsmOptions opt;
    opt.glv = true;  // d_table holds the phi rows from row n on
    opt.glv_rows = n;
    msm_run_table(eng, d_scalars, d_table, n, d_out_wire, nullptr, st, opt);
}

}  // namespace kb200
