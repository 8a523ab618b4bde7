// Word-prime NTT (one 64-bit word per coefficient) behind the reference's
// ntt_forward / ntt_inverse (ntt/c-abi/c_ntt.cpp:81-179).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace kb200 {

// Per-device cache of twiddle tables keyed by (n, modulus, root, direction).
struct WordNttCache;
WordNttCache* word_ntt_cache_create();
void word_ntt_cache_destroy(WordNttCache* c);

// Transforms the n words at d_data in place on `st` (d_scratch: n words,
// needed for 2^11 < n <= 2^16).  Dispatch, arguments and results follow the
// reference C ABI:
//   n <= 2^16: natural order; modulus 998244353 with the pinned root
//              629671588 takes the reference's Montgomery (R = 2^32) path,
//              any other (modulus, root) its generic path, root = n-th root.
//   2^16 < n <= 2^20: six-step, forward output (and inverse input) in the
//              transposed N2 x N1 layout, root = 2n-th root.
// Returns 0 or -1 (CRYPTO_ERR_INPUT) for arguments the reference rejects;
// throws CudaError on device failures.  Inputs need not be reduced: every
// path reproduces the reference's arithmetic on unreduced words.
int word_ntt_device(WordNttCache* cache, uint64_t* d_data, uint64_t* d_scratch, size_t n,
                    uint64_t modulus, uint64_t root, bool inverse, cudaStream_t st);

}  // namespace kb200
