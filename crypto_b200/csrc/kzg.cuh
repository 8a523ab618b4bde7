// KZG commit building blocks on device: fixed-base G1 multiplication (used
// to build synthetic SRS tables [tau^i]G1 and seeded input points s_i*G1),
// powers of tau in Fr, and the commit composition iNTT -> MSM -> compress.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace kb200 {

class FixedBase;
FixedBase* fixed_base_create(int curve, cudaStream_t stream);  // builds the G table
void fixed_base_destroy(FixedBase* fb);
// out (table layout, 2N words per point, Montgomery affine) = s_i * G for
// n scalars (32-byte little-endian).  If out_wire is non-null the canonical
// big-endian wire encoding is written there as well.
void fixed_base_mul(FixedBase* fb, const uint8_t* d_scalars, size_t n, uint32_t* d_table_out,
                    uint8_t* d_wire_out, cudaStream_t stream);

// out[i] = tau^i (canonical 32-byte little-endian Fr), i < n.
void fr_powers(int curve, const uint8_t* d_tau, size_t n, uint8_t* d_out, cudaStream_t stream);

}  // namespace kb200
