// EIP-2537 BLS12_G1MSM input path on the GPU, behind the reference's
// bls12_381_g1_msm (bls/c-abi/c_bls_pairing.cpp:106-110, bls/cpp/bls.cpp:194-254).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "msm.cuh"

namespace kb200 {

// Validates and unpacks n entries of 160 bytes (x[64] || y[64] || c[32], big
// endian) into the affine table and reduced little-endian scalars, then runs
// the MSM with the GLV split.  d_table: 2n * 24 words (rows n.. hold
// phi(P) = (beta2 x, y)), d_scalars: n * 32 bytes, d_flag: one word,
// set to 1 if any entry is invalid (coordinate >= p or top 16 bytes non-zero,
// off the curve, or outside G1); d_out_wire: 96 bytes (x || y, 48 B BE each,
// zeros for infinity).  Queued on `st`, nothing synchronised.
void g1_msm_eip2537_device(MsmEngine* eng, const uint8_t* d_xycs, size_t n, uint32_t* d_table,
                           uint8_t* d_scalars, uint32_t* d_flag, uint8_t* d_out_wire,
                           cudaStream_t st);

}  // namespace kb200
