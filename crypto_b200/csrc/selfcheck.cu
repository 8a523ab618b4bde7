// Device self-checks of the field arithmetic: the binary-GCD inversion used
// everywhere (fe_inv) against the Fermat chain a^(p-2), and x * x^-1 = 1, on
// edge values and seeded pseudo-random elements of each field; and the
// products (Karatsuba product and squaring, interleaved product) on caller
// operands, returned for comparison with a CPU product.
#include "../../include/kinet_b200/crypto_b200.h"
#include "field.cuh"
#include "runtime.cuh"

namespace kb200 {
namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t x) {  // splitmix64 finaliser
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

template <class F>
__global__ void k_inverse_check(uint64_t seed, size_t count, unsigned long long* bad) {
    constexpr int N = F::N;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    Fe<F> x;
    // i < 6: 0, 1, 2, p - 1, p - 2, (p - 1) / 2; then random words below 2^(len p - 1)
    if (i < 6) {
        uint32_t p[N];
#pragma unroll
        for (int k = 0; k < N; ++k) p[k] = F::P(k);
        fe_zero(x);
        if (i == 1 || i == 2) x.v[0] = (uint32_t)i;
        if (i == 3 || i == 4) {
            int64_t br = -(int64_t)(i - 2);
            for (int k = 0; k < N; ++k) {
                const int64_t s = (int64_t)p[k] + br;
                x.v[k] = (uint32_t)s;
                br = s >> 32;
            }
        }
        if (i == 5)
            for (int k = 0; k < N; ++k) x.v[k] = (p[k] >> 1) | (k + 1 < N ? p[k + 1] << 31 : 0u);
    } else {
        uint64_t st = mix64(seed ^ (i * 0x632be59bd9b4e019ull));
#pragma unroll
        for (int k = 0; k < N; ++k) {
            st = mix64(st);
            x.v[k] = (uint32_t)st;
        }
        constexpr int L = gcd_detail::bit_length_p<F>();
        constexpr int top_bits = (L - 1) - 32 * (N - 1);  // bits kept in the top word
        x.v[N - 1] &= top_bits >= 32 ? 0xffffffffu : ((1u << top_bits) - 1u);
    }
    Fe<F> r1, r2, t, one;
    fe_inv_gcd<F>(r1, x);
    fe_inv_fermat<F>(r2, x);
    bool ok = fe_eq(r1, r2);
    if (!fe_is_zero(x)) {
        fe_mul(t, x, r1);
        fe_one(one);
        ok = ok && fe_eq(t, one);
    }
    if (!ok) atomicAdd(bad, 1ull);
}

// out_mul[i] = a[i] b[i], out_sqr[i] = a[i]^2 (canonical, through the
// Montgomery forms) with fe_mul and fe_sqr; *bad counts elements where the
// interleaved product fe_mul_inl disagrees with either.
template <class F>
__global__ void k_mul_check(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b, size_t n,
                            uint32_t* __restrict__ out_mul, uint32_t* __restrict__ out_sqr,
                            unsigned long long* bad) {
    constexpr int N = F::N;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Fe<F> x, y, m1, m2, s1, s2;
#pragma unroll
    for (int k = 0; k < N; ++k) {
        x.v[k] = a[i * N + k];
        y.v[k] = b[i * N + k];
    }
    fe_to_mont(x, x);
    fe_to_mont(y, y);
    fe_mul(m1, x, y);
    fe_mul_inl(m2, x, y);
    fe_sqr(s1, x);
    fe_mul_inl(s2, x, x);
    if (!fe_eq(m1, m2) || !fe_eq(s1, s2)) atomicAdd(bad, 1ull);
    fe_from_mont(m1, m1);
    fe_from_mont(s1, s1);
#pragma unroll
    for (int k = 0; k < N; ++k) {
        out_mul[i * N + k] = m1.v[k];
        out_sqr[i * N + k] = s1.v[k];
    }
}

template <class F>
void run_check(uint64_t seed, size_t count, unsigned long long* d_bad) {
    k_inverse_check<F><<<ceil_div_u(count, 128), 128>>>(seed, count, d_bad);
    KB_LAUNCH_CHECK();
}

}  // namespace
}  // namespace kb200

using namespace kb200;

extern "C" int kb200_field_inverse_check(int field, uint64_t seed, size_t count,
                                         unsigned long long* mismatches) {
    if (!mismatches || field < 0 || field > 3) return KB200_CRYPTO_ERR_INPUT;
    unsigned long long* d_bad = nullptr;
    try {
        KB_CUDA(cudaMalloc(&d_bad, sizeof(unsigned long long)));
        KB_CUDA(cudaMemset(d_bad, 0, sizeof(unsigned long long)));
        if (count) {
            switch (field) {
                case 0: run_check<FpBLS>(seed, count, d_bad); break;
                case 1: run_check<FrBLS>(seed, count, d_bad); break;
                case 2: run_check<FpBN>(seed, count, d_bad); break;
                default: run_check<FrBN>(seed, count, d_bad); break;
            }
        }
        KB_CUDA(cudaMemcpy(mismatches, d_bad, sizeof(unsigned long long), cudaMemcpyDeviceToHost));
        cudaFree(d_bad);
        return KB200_CRYPTO_OK;
    } catch (const std::exception& e) {
        if (d_bad) cudaFree(d_bad);
        set_last_error(e.what());
        return KB200_CRYPTO_ERR_BACKEND;
    }
}

extern "C" int kb200_field_mul_check(int field, const uint8_t* a_le, const uint8_t* b_le, size_t n,
                                     uint8_t* out_mul_le, uint8_t* out_sqr_le,
                                     unsigned long long* form_mismatches) {
    if (field < 0 || field > 3 || !form_mismatches || (n && (!a_le || !b_le || !out_mul_le || !out_sqr_le)))
        return KB200_CRYPTO_ERR_INPUT;
    const size_t bytes = n * (field == 0 ? 48 : 32);
    unsigned long long* d_bad = nullptr;
    uint32_t* d = nullptr;
    try {
        KB_CUDA(cudaMalloc(&d_bad, sizeof(unsigned long long)));
        KB_CUDA(cudaMemset(d_bad, 0, sizeof(unsigned long long)));
        if (n) {
            KB_CUDA(cudaMalloc(&d, 4 * bytes));
            uint32_t* da = d;
            uint32_t* db = d + bytes / 4;
            uint32_t* dm = d + 2 * (bytes / 4);
            uint32_t* ds = d + 3 * (bytes / 4);
            KB_CUDA(cudaMemcpy(da, a_le, bytes, cudaMemcpyHostToDevice));
            KB_CUDA(cudaMemcpy(db, b_le, bytes, cudaMemcpyHostToDevice));
            const unsigned g = ceil_div_u(n, 128);
            switch (field) {
                case 0: k_mul_check<FpBLS><<<g, 128>>>(da, db, n, dm, ds, d_bad); break;
                case 1: k_mul_check<FrBLS><<<g, 128>>>(da, db, n, dm, ds, d_bad); break;
                case 2: k_mul_check<FpBN><<<g, 128>>>(da, db, n, dm, ds, d_bad); break;
                default: k_mul_check<FrBN><<<g, 128>>>(da, db, n, dm, ds, d_bad); break;
            }
            KB_LAUNCH_CHECK();
            KB_CUDA(cudaMemcpy(out_mul_le, dm, bytes, cudaMemcpyDeviceToHost));
            KB_CUDA(cudaMemcpy(out_sqr_le, ds, bytes, cudaMemcpyDeviceToHost));
        }
        KB_CUDA(cudaMemcpy(form_mismatches, d_bad, sizeof(unsigned long long), cudaMemcpyDeviceToHost));
        if (d) cudaFree(d);
        cudaFree(d_bad);
        return KB200_CRYPTO_OK;
    } catch (const std::exception& e) {
        if (d) cudaFree(d);
        if (d_bad) cudaFree(d_bad);
        set_last_error(e.what());
        return KB200_CRYPTO_ERR_BACKEND;
    }
}
