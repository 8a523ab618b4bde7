// Scalar-field (Fr) NTT on one GPU, BLS12-381 and BN254.
//
// Contract (natural order in and out, canonical 32-byte little-endian
// elements, inputs reduced mod r first):
//   forward : X_k = sum_j x_j w^(jk)               coset: x_j * g^j first
//   inverse : x_j = n^-1 sum_k X_k w^(-jk)         coset: result * g^-j
// with w = g^((r-1)/n), g = 7 (BLS12-381 Fr) or 5 (BN254 Fr).
//
// n = R_1 * ... * R_P (P <= 3, R_p <= 2^10).  Pass p performs radix-R_p DFTs
// in shared memory (radix-2 decimation-in-frequency stages) on columns of
// stride m_p = n / (R_1 ... R_p) inside blocks of m_{p-1} elements and
// multiplies by the four-step twiddle w_{m_{p-1}}^(i_lo * j); every pass
// reads and writes coalesced runs of adjacent columns.  The last pass
// writes the mixed-radix digit-reversed (= natural) order directly, out of
// place, with the inverse scaling and coset factors fused into its store.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace kb200 {

class NttEngine;
NttEngine* ntt_engine_create(int curve);
void ntt_engine_destroy(NttEngine* e);

// In-place transform of `batch` consecutive vectors of n elements each
// (d_data: batch * n * 32 bytes on device).  Uses engine scratch of the same
// size.  Queued on `stream`.
void ntt_run(NttEngine* e, uint32_t* d_data, size_t n, int inverse, int coset, size_t batch,
             cudaStream_t stream);

// Transform `count` vectors of n elements whose element offsets (into d)
// are listed on the device in d_vec_off; d_scratch mirrors d's layout
// (needed when n > 2^12).  Queues kernels only once ntt_prepare(n, coset)
// has run, so it can be captured in a CUDA graph.
void ntt_run_list(NttEngine* e, uint32_t* d, size_t n, int inverse, int coset, size_t count,
                  const unsigned long long* d_vec_off, uint32_t* d_scratch, cudaStream_t stream);

// Build (or grow) the resident twiddle table so that sizes up to n need no
// further set-up work.  Synchronises the stream when it builds.
void ntt_prepare(NttEngine* e, size_t n, int coset, cudaStream_t stream);

// Autotuner table: log2 of the first-pass radix for a size class (0 = the
// default balanced split).
void ntt_tune_set(int curve, int log_n, int log_r1);
int ntt_tune_get(int curve, int log_n);

// Largest supported log2 size for a curve (2-adicity, capped).
int ntt_max_log(int curve);

}  // namespace kb200
