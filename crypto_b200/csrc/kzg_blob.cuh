// EIP-4844 blob commitment and opening proof on the device (see kzg_blob.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "kzg.cuh"
#include "msm.cuh"

namespace kb200 {

constexpr uint32_t BLOB_N = 4096;   // field elements per blob
constexpr uint32_t BLOB_LOG = 12;
constexpr size_t BLOB_BYTES = (size_t)BLOB_N * 32;

// Resident setup (Lagrange-form G1 points in bit-reversed order) and work
// buffers, one per device.
struct BlobSetup;
BlobSetup* blob_setup_create();
void blob_setup_destroy(BlobSetup* s);
bool blob_setup_ready(const BlobSetup* s);
void blob_setup_mark(BlobSetup* s, bool ready);

// 4096 compressed points (the trusted setup's Lagrange points, natural order)
// -> resident table.  *d_flag (one word) is set if a point is invalid.
void blob_setup_load_lagrange(BlobSetup* s, const uint8_t* d_pts48, uint32_t* d_flag, cudaStream_t st);
// Synthetic setup [L_i(tau)]G1 from a 32-byte little-endian tau.
void blob_setup_generate(BlobSetup* s, FixedBase* fb, const uint8_t* d_tau_le, cudaStream_t st);

// commitment of a 131072-byte blob (48 bytes compressed); *d_flag set if an
// element is not below r.
void blob_commit_device(BlobSetup* s, MsmEngine* eng, const uint8_t* d_blob, uint8_t* d_commit48,
                        uint32_t* d_flag, cudaStream_t st);
// proof (48 bytes compressed) and y = p(z) (32 bytes big-endian) for a
// 32-byte big-endian z; *d_flag set if an element or z is not below r.
void blob_proof_device(BlobSetup* s, MsmEngine* eng, const uint8_t* d_blob, const uint8_t* d_z_be,
                       uint8_t* d_proof48, uint8_t* d_y_be, uint32_t* d_flag, cudaStream_t st);

}  // namespace kb200
