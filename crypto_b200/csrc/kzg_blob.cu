// EIP-4844 blob operations on the GPU, behind the reference's
// kzg_blob_to_commit and kzg_commit_to_proof (kzg/c-abi/c_kzg_blob.cpp:26-43;
// bodies kzg/cpp/kzg_blob.cpp:69-81 and :106-125, which call c-kzg-4844
// v2.1.7 over the mainnet trusted setup).  The published EIP-4844 algorithm:
//
//   A blob is 4096 field elements, 32 bytes big-endian each, every one below
//   r; element i is p(w^brp(i)) for the polynomial p, w the 4096-th root of
//   unity 7^((r-1)/4096) and brp the 12-bit bit reversal.
//   commitment = sum_i blob[i] * L_brp(i)(tau) G1, an MSM against the setup's
//   Lagrange points in bit-reversed order, compressed to 48 bytes.
//   compute_kzg_proof(blob, z): y = p(z) by the barycentric formula (or the
//   blob element itself when z is a domain point); the quotient
//   q = (p - y) / (X - z) in evaluation form, q_i = (p_i - y) / (w_i - z),
//   and at a domain point z = w_m
//   q_m = sum_{i != m} (p_i - y) w_i / (z (z - w_i)); proof = MSM(q, setup).
//
// Every step runs on the device: one thread per blob element for the
// parsing, inversions and quotient; one block for the two sums; the MSM of
// msm.cu.  The setup is resident (loaded from the trusted setup's 4096
// compressed Lagrange points, or generated from a test tau).
#include "g1check.cuh"
#include "kzg.cuh"
#include "kzg_blob.cuh"
#include "runtime.cuh"

namespace kb200 {
namespace {

using F = FpBLS;
using FR = FrBLS;
constexpr int RED_T = 1024;

// (p + 1) / 4 (square roots, p = 3 mod 4) and (p - 1) / 2, little-endian words.
__constant__ uint32_t kSqrtExp[12] = {0xffffeaab, 0xee7fbfff, 0xac54ffff, 0x07aaffff,
                                      0x3dac3d89, 0xd9cc34a8, 0x3ce144af, 0xd91dd2e1,
                                      0x90d2eb35, 0x92c6e9ed, 0x8e5ff9a6, 0x0680447a};
__constant__ uint32_t kHalfP[12] = {0xffffd555, 0xdcff7fff, 0x58a9ffff, 0x0f55ffff,
                                    0x7b587b12, 0xb3986950, 0x79c2895f, 0xb23ba5c2,
                                    0x21a5d66b, 0x258dd3db, 0x1cbff34d, 0x0d0088f5};

__device__ __forceinline__ uint32_t brp12(uint32_t i) { return __brev(i) >> (32 - BLOB_LOG); }

// a^e for a little-endian exponent of nw words (left-to-right binary).
template <class Fx>
__device__ void fe_pow_words(Fe<Fx>& r, const Fe<Fx>& a, const uint32_t* e, int nw) {
    Fe<Fx> acc;
    fe_one(acc);
    bool started = false;
    for (int w = nw - 1; w >= 0; --w) {
        const uint32_t word = e[w];
        for (int b = 31; b >= 0; --b) {
            if (started) fe_sqr(acc, acc);
            if ((word >> b) & 1u) {
                if (started) {
                    fe_mul(acc, acc, a);
                } else {
                    acc = a;
                    started = true;
                }
            }
        }
    }
    r = acc;
}

// (r - 1) / 4096 as 8 little-endian words.
__device__ void order_cofactor(uint32_t e[8]) {
    uint32_t t[8];
    for (int k = 0; k < 8; ++k) t[k] = FR::P(k);
    t[0] -= 1;  // r's low word is 1
    for (int k = 0; k < 8; ++k) e[k] = (t[k] >> BLOB_LOG) | (k + 1 < 8 ? t[k + 1] << (32 - BLOB_LOG) : 0u);
}

// w^k (Montgomery), w = 7^((r-1)/4096).
__device__ void root_pow(Fe<FR>& r, uint32_t k) {
    uint32_t e[8];
    order_cofactor(e);
    Fe<FR> g, w;
    fe_zero(g);
    g.v[0] = 7;
    fe_to_mont(g, g);
    fe_pow_words(w, g, e, 8);
    const uint32_t kk[1] = {k};
    fe_pow_words(r, w, kk, 1);
}

// 1/4096 mod r = r - (r - 1)/4096 (Montgomery).
__device__ void inv_blob_n(Fe<FR>& r) {
    uint32_t e[8];
    order_cofactor(e);
    uint32_t b = 0;
    for (int k = 0; k < 8; ++k) {
        const uint64_t d = (uint64_t)FR::P(k) - e[k] - b;
        r.v[k] = (uint32_t)d;
        b = (uint32_t)(d >> 63);
    }
    fe_to_mont(r, r);
}

__device__ __forceinline__ void store_le(uint8_t* dst, const Fe<FR>& canon) {
    uint32_t* o = reinterpret_cast<uint32_t*>(dst);
    for (int k = 0; k < FR::N; ++k) o[k] = canon.v[k];
}

// roots[i] = w^brp(i) (Montgomery, 8 words).
__global__ void k_roots_brp(uint32_t* roots) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= BLOB_N) return;
    Fe<FR> r;
    root_pow(r, brp12(i));
    fe_store(roots + 8 * i, r);
}

// Slot i of the synthetic setup: L_brp(i)(tau) as a canonical LE scalar,
// L_j(tau) = w^j (tau^n - 1) / (n (tau - w^j)).
__global__ void k_lagrange_scalars(const uint8_t* __restrict__ tau_le, const uint32_t* __restrict__ roots,
                                   uint8_t* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= BLOB_N) return;
    Fe<FR> tau, wj, d, t, num;
    fe_load(tau, reinterpret_cast<const uint32_t*>(tau_le));
    fe_to_mont(tau, tau);
    fe_load(wj, roots + 8 * i);
    fe_sub(d, tau, wj);
    if (fe_is_zero(d)) {
        fe_one(t);
    } else {
        num = tau;
        for (int k = 0; k < BLOB_LOG; ++k) fe_sqr(num, num);  // tau^4096
        Fe<FR> one;
        fe_one(one);
        fe_sub(num, num, one);
        fe_mul(num, num, wj);
        Fe<FR> ninv;
        inv_blob_n(ninv);
        fe_mul(num, num, ninv);
        fe_inv(d, d);
        fe_mul(t, num, d);
    }
    fe_from_mont(t, t);
    store_le(out + 32 * (size_t)i, t);
}

// Trusted-setup point i (48-byte compressed, natural order) -> table slot
// brp(i).  Checks the encoding flags, x < p, that x^3 + 4 is a square, and
// G1 membership.
__global__ void k_setup_decompress(const uint8_t* __restrict__ pts, uint32_t* __restrict__ table,
                                   uint32_t* __restrict__ flag) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= BLOB_N) return;
    const uint8_t* b = pts + 48 * (size_t)i;
    uint32_t* row = table + (size_t)brp12(i) * 2 * F::N;
    const uint32_t c_bit = b[0] >> 7, inf_bit = (b[0] >> 6) & 1, sign = (b[0] >> 5) & 1;
    bool ok = c_bit == 1;
    if (inf_bit) {
        uint32_t rest = b[0] & 0x3f;
        for (int k = 1; k < 48; ++k) rest |= b[k];
        ok = ok && rest == 0 && sign == 0;
        for (int k = 0; k < 2 * F::N; ++k) row[k] = 0;
        row[F::N - 1] = INF_FLAG;
        if (!ok) atomicOr(flag, 1u);
        return;
    }
    uint8_t xb[48];
    for (int k = 0; k < 48; ++k) xb[k] = b[k];
    xb[0] &= 0x1f;
    Fe<F> x;
    fe_from_be_bytes(x, xb);
    ok = ok && below_modulus(x);
    Affine<F> a;
    fe_to_mont(a.x, x);
    Fe<F> rhs, y, b4;
    fe_sqr(rhs, a.x);
    fe_mul(rhs, rhs, a.x);
    fe_one(b4);
    fe_add(b4, b4, b4);
    fe_add(b4, b4, b4);
    fe_add(rhs, rhs, b4);
    Fe<F> e;
    fe_load(e, kSqrtExp);
    fe_pow_words(y, rhs, e.v, F::N);
    Fe<F> y2;
    fe_sqr(y2, y);
    ok = ok && fe_eq(y2, rhs);
    // choose the root whose canonical value is above (p-1)/2 iff sign is set
    Fe<F> yc;
    fe_from_mont(yc, y);
    bool big = false;
    for (int k = F::N - 1; k >= 0; --k) {
        if (yc.v[k] != kHalfP[k]) {
            big = yc.v[k] > kHalfP[k];
            break;
        }
    }
    if (big != (sign != 0)) fe_neg(y, y);
    a.y = y;
    ok = ok && g1_in_subgroup(a);
    if (!ok) {
        atomicOr(flag, 1u);
        for (int k = 0; k < 2 * F::N; ++k) row[k] = 0;
        row[F::N - 1] = INF_FLAG;
        return;
    }
    fe_store(row, a.x);
    fe_store(row + F::N, a.y);
}

// Blob element i: big-endian 32 bytes, must be below r.
__global__ void k_blob_load(const uint8_t* __restrict__ blob, uint32_t* __restrict__ p_mont,
                            uint8_t* __restrict__ p_le, uint32_t* __restrict__ flag) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= BLOB_N) return;
    Fe<FR> v;
    fe_from_be_bytes(v, blob + 32 * (size_t)i);
    if (!below_modulus(v)) {
        atomicOr(flag, 1u);
        fe_zero(v);
    }
    store_le(p_le + 32 * (size_t)i, v);
    fe_to_mont(v, v);
    fe_store(p_mont + 8 * i, v);
}

// d_i = z - w_i: inv_i = 1/d_i and term_i = p_i w_i / d_i, or (z a domain
// point) the index m of that point.
__global__ void k_blob_terms(const uint32_t* __restrict__ p_mont, const uint32_t* __restrict__ roots,
                             const uint8_t* __restrict__ z_be, uint32_t* __restrict__ inv,
                             uint32_t* __restrict__ term, uint32_t* __restrict__ flag,
                             uint32_t* __restrict__ misc) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= BLOB_N) return;
    Fe<FR> z, w, d, t;
    fe_from_be_bytes(z, z_be);
    if (!below_modulus(z)) {
        if (i == 0) atomicOr(flag, 1u);
        fe_zero(z);
    }
    fe_to_mont(z, z);
    fe_load(w, roots + 8 * i);
    fe_sub(d, z, w);
    if (fe_is_zero(d)) {
        atomicMin(misc, i);  // misc[0]: domain index of z (initialised to ~0)
        fe_zero(t);
        fe_store(inv + 8 * i, t);
        fe_store(term + 8 * i, t);
        return;
    }
    fe_inv(d, d);
    fe_store(inv + 8 * i, d);
    Fe<FR> p;
    fe_load(p, p_mont + 8 * i);
    fe_mul(t, p, w);
    fe_mul(t, t, d);
    fe_store(term + 8 * i, t);
}

// out = sum of the 4096 terms (one block of RED_T threads).
__global__ void __launch_bounds__(RED_T) k_blob_sum(const uint32_t* __restrict__ term,
                                                    uint32_t* __restrict__ out) {
    __shared__ uint32_t sm[RED_T * 8];
    const uint32_t t = threadIdx.x;
    Fe<FR> acc, x;
    fe_zero(acc);
    for (uint32_t i = t; i < BLOB_N; i += RED_T) {
        fe_load(x, term + 8 * i);
        fe_add(acc, acc, x);
    }
    fe_store(sm + 8 * t, acc);
    __syncthreads();
    for (uint32_t s = RED_T / 2; s > 0; s >>= 1) {
        if (t < s) {
            fe_load(acc, sm + 8 * t);
            fe_load(x, sm + 8 * (t + s));
            fe_add(acc, acc, x);
            fe_store(sm + 8 * t, acc);
        }
        __syncthreads();
    }
    if (t == 0)
        for (int k = 0; k < 8; ++k) out[k] = sm[k];
}

// y = p_m (z = w_m), else y = (z^n - 1)/n * sum_i p_i w_i / (z - w_i).
__global__ void k_blob_y(const uint32_t* __restrict__ p_mont, const uint8_t* __restrict__ z_be,
                         const uint32_t* __restrict__ sum, const uint32_t* __restrict__ misc,
                         uint32_t* __restrict__ y_mont, uint8_t* __restrict__ y_be) {
    Fe<FR> y;
    const uint32_t m = misc[0];
    if (m < BLOB_N) {
        fe_load(y, p_mont + 8 * m);
    } else {
        Fe<FR> z, zn, one, ninv, s;
        fe_from_be_bytes(z, z_be);
        if (!below_modulus(z)) fe_zero(z);
        fe_to_mont(z, z);
        zn = z;
        for (int k = 0; k < BLOB_LOG; ++k) fe_sqr(zn, zn);
        fe_one(one);
        fe_sub(zn, zn, one);
        inv_blob_n(ninv);
        fe_load(s, sum);
        fe_mul(y, s, zn);
        fe_mul(y, y, ninv);
    }
    fe_store(y_mont, y);
    Fe<FR> yc;
    fe_from_mont(yc, y);
    fe_to_be_bytes(y_be, yc);
}

// q_i = (y - p_i) / (z - w_i) for i != m; term_i = (p_i - y) w_i / (z - w_i)
// (0 at m) for the domain-point quotient.
__global__ void k_blob_quotient(const uint32_t* __restrict__ p_mont, const uint32_t* __restrict__ roots,
                                const uint32_t* __restrict__ inv, const uint32_t* __restrict__ y_mont,
                                const uint32_t* __restrict__ misc, uint8_t* __restrict__ q_le,
                                uint32_t* __restrict__ term) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= BLOB_N) return;
    Fe<FR> p, y, d, q, w, t;
    if (i == misc[0]) {
        fe_zero(q);
        store_le(q_le + 32 * (size_t)i, q);
        fe_store(term + 8 * i, q);
        return;
    }
    fe_load(p, p_mont + 8 * i);
    fe_load(y, y_mont);
    fe_load(d, inv + 8 * i);
    fe_sub(q, y, p);
    fe_mul(q, q, d);
    Fe<FR> qc;
    fe_from_mont(qc, q);
    store_le(q_le + 32 * (size_t)i, qc);
    fe_load(w, roots + 8 * i);
    fe_neg(t, q);   // (p_i - y) / (z - w_i)
    fe_mul(t, t, w);
    fe_store(term + 8 * i, t);
}

// q_m = z^-1 sum_{i != m} (p_i - y) w_i / (z - w_i), with z^-1 = w^(n - brp(m)).
__global__ void k_blob_qm(const uint32_t* __restrict__ sum, const uint32_t* __restrict__ misc,
                          uint8_t* __restrict__ q_le) {
    const uint32_t m = misc[0];
    if (m >= BLOB_N) return;
    Fe<FR> zi, s;
    root_pow(zi, (BLOB_N - brp12(m)) & (BLOB_N - 1));
    fe_load(s, sum);
    fe_mul(s, s, zi);
    fe_from_mont(s, s);
    store_le(q_le + 32 * (size_t)m, s);
}

}  // namespace

struct BlobSetup {
    DevBuf table;  // 4096 rows (Montgomery affine), bit-reversed order
    DevBuf roots;  // w^brp(i), Montgomery
    DevBuf p_mont, p_le, inv, term, q_le, misc, sum, y_mont, wire;
    bool ready = false;
    bool roots_ready = false;
    ShiftTables* shifts = shift_tables_create();  // shifted levels of `table`
    ~BlobSetup() { shift_tables_destroy(shifts); }
};

BlobSetup* blob_setup_create() { return new BlobSetup(); }
void blob_setup_destroy(BlobSetup* s) { delete s; }

// The MSM against the setup: through its shifted levels (one shared bucket
// window per blob, no doubling chain), or the plain table if unavailable.
static void blob_msm(BlobSetup* s, MsmEngine* eng, const uint8_t* d_scalars, uint8_t* d_out48,
                     cudaStream_t st) {
    MsmOptions opt;
    const uint32_t* table = s->table.as<uint32_t>();
    const size_t n = BLOB_N;
    const int c = shift_c_for(&n, 1);
    if (const uint32_t* t = shift_tables_get(s->shifts, c, st)) {
        opt.shift_c = c;
        opt.shift_stride = BLOB_N;
        table = t;
    }
    msm_run_table(eng, d_scalars, table, BLOB_N, s->wire.as<uint8_t>(), d_out48, st, opt);
}
bool blob_setup_ready(const BlobSetup* s) { return s && s->ready; }

static void ensure_buffers(BlobSetup* s, cudaStream_t st) {
    s->table.reserve((size_t)BLOB_N * 2 * F::N * 4, st);
    s->roots.reserve((size_t)BLOB_N * 32, st);
    s->p_mont.reserve((size_t)BLOB_N * 32, st);
    s->p_le.reserve((size_t)BLOB_N * 32, st);
    s->inv.reserve((size_t)BLOB_N * 32, st);
    s->term.reserve((size_t)BLOB_N * 32, st);
    s->q_le.reserve((size_t)BLOB_N * 32, st);
    s->misc.reserve(64, st);
    s->sum.reserve(64, st);
    s->y_mont.reserve(64, st);
    s->wire.reserve(128, st);
    if (!s->roots_ready) {
        k_roots_brp<<<BLOB_N / 128, 128, 0, st>>>(s->roots.as<uint32_t>());
        KB_LAUNCH_CHECK();
        s->roots_ready = true;
    }
}

void blob_setup_load_lagrange(BlobSetup* s, const uint8_t* d_pts48, uint32_t* d_flag, cudaStream_t st) {
    ensure_buffers(s, st);
    KB_CUDA(cudaMemsetAsync(d_flag, 0, 4, st));
    k_setup_decompress<<<BLOB_N / 128, 128, 0, st>>>(d_pts48, s->table.as<uint32_t>(), d_flag);
    KB_LAUNCH_CHECK();
    shift_tables_reset(s->shifts, s->table.as<uint32_t>(), BLOB_N);
    s->ready = true;  // the caller clears it if the flag comes back set
}

void blob_setup_mark(BlobSetup* s, bool ready) { s->ready = ready; }

void blob_setup_generate(BlobSetup* s, FixedBase* fb, const uint8_t* d_tau_le, cudaStream_t st) {
    ensure_buffers(s, st);
    k_lagrange_scalars<<<BLOB_N / 128, 128, 0, st>>>(d_tau_le, s->roots.as<uint32_t>(),
                                                     s->q_le.as<uint8_t>());
    KB_LAUNCH_CHECK();
    fixed_base_mul(fb, s->q_le.as<uint8_t>(), BLOB_N, s->table.as<uint32_t>(), nullptr, st);
    shift_tables_reset(s->shifts, s->table.as<uint32_t>(), BLOB_N);
    s->ready = true;
}

void blob_commit_device(BlobSetup* s, MsmEngine* eng, const uint8_t* d_blob, uint8_t* d_commit48,
                        uint32_t* d_flag, cudaStream_t st) {
    ensure_buffers(s, st);
    KB_CUDA(cudaMemsetAsync(d_flag, 0, 4, st));
    k_blob_load<<<BLOB_N / 128, 128, 0, st>>>(d_blob, s->p_mont.as<uint32_t>(), s->p_le.as<uint8_t>(),
                                              d_flag);
    KB_LAUNCH_CHECK();
    blob_msm(s, eng, s->p_le.as<uint8_t>(), d_commit48, st);
}

void blob_proof_device(BlobSetup* s, MsmEngine* eng, const uint8_t* d_blob, const uint8_t* d_z_be,
                       uint8_t* d_proof48, uint8_t* d_y_be, uint32_t* d_flag, cudaStream_t st) {
    ensure_buffers(s, st);
    uint32_t* misc = s->misc.as<uint32_t>();
    KB_CUDA(cudaMemsetAsync(d_flag, 0, 4, st));
    KB_CUDA(cudaMemsetAsync(misc, 0xff, 4, st));
    k_blob_load<<<BLOB_N / 128, 128, 0, st>>>(d_blob, s->p_mont.as<uint32_t>(), s->p_le.as<uint8_t>(),
                                              d_flag);
    k_blob_terms<<<BLOB_N / 128, 128, 0, st>>>(s->p_mont.as<uint32_t>(), s->roots.as<uint32_t>(), d_z_be,
                                               s->inv.as<uint32_t>(), s->term.as<uint32_t>(), d_flag,
                                               misc);
    k_blob_sum<<<1, RED_T, 0, st>>>(s->term.as<uint32_t>(), s->sum.as<uint32_t>());
    k_blob_y<<<1, 1, 0, st>>>(s->p_mont.as<uint32_t>(), d_z_be, s->sum.as<uint32_t>(), misc,
                              s->y_mont.as<uint32_t>(), d_y_be);
    k_blob_quotient<<<BLOB_N / 128, 128, 0, st>>>(s->p_mont.as<uint32_t>(), s->roots.as<uint32_t>(),
                                                  s->inv.as<uint32_t>(), s->y_mont.as<uint32_t>(), misc,
                                                  s->q_le.as<uint8_t>(), s->term.as<uint32_t>());
    k_blob_sum<<<1, RED_T, 0, st>>>(s->term.as<uint32_t>(), s->sum.as<uint32_t>());
    k_blob_qm<<<1, 1, 0, st>>>(s->sum.as<uint32_t>(), misc, s->q_le.as<uint8_t>());
    KB_LAUNCH_CHECK();
    blob_msm(s, eng, s->q_le.as<uint8_t>(), d_proof48, st);
}

}  // namespace kb200
