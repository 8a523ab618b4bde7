// G1 multi-scalar multiplication (signed-digit Pippenger) on one GPU.
//
// Pipeline, all on device, all launched on the caller's stream:
//   1. wire -> table   : big-endian affine points -> Montgomery affine words
//   2. recode          : each scalar -> W signed c-bit digits, one
//                        (bucket, point|sign) entry per non-zero digit
//   3. histogram/scan  : per-bucket counts -> bucket offsets
//   4. scatter         : counting sort of the entries by bucket
//   5. accumulate      : buckets split into segments of <= K entries; one
//                        thread sums one segment with mixed XYZZ additions
//   6. segment levels  : partial sums of buckets that span several segments
//                        are folded K2 at a time until one sum per bucket
//   7. reduce          : per window, sum_k (k+1) * B_k via grouped running
//                        sums (groups of S buckets), then a tree per window
//   8. combine         : Horner over windows (c doublings each), affine
//                        normalisation and big-endian (and compressed) encode
// The digit recoding follows gpukit/cpp/cpu_reference/multi_pippenger.cpp:90-134
// (digits in (-2^(c-1), 2^(c-1)], carry into the next window), with enough
// windows (ceil(257 / c)) that no carry leaves the top window.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace kb200 {

struct MsmPlan {
    int c = 0;          // window bits
    int W = 0;          // windows
    uint32_t M = 0;     // buckets per window (2^(c-1))
    uint32_t B = 0;     // W * M
    int K = 32;         // entries per level-1 segment
    int K2 = 8;         // fan-in of later segment levels
    int levels = 0;     // segment levels after level 1
    int S = 8;          // buckets per reduction group
    uint32_t G = 0;     // reduction groups per window
    size_t seg_cap = 0; // upper bound on level-1 segments
};

struct MsmOptions {
    // Reproduce the reference's signed-digit behaviour for n (its window size
    // best_c(n) in [4,12]; for c = 4 and c = 8 it drops the carry out of the
    // top window, multi_pippenger.cpp:161-180).  Set by the drop-in entry
    // point so results stay byte-equal to gpukit_multi_pippenger_cpu even
    // for scalars >= 2^255.
    bool ref_carry_quirk = false;
    int force_c = 0;  // 0 = autotuned / cost model
    int force_K = 0;
};

// Reference window size for n: multi_pippenger.cpp:69-88.
int reference_best_c(size_t n);

MsmPlan make_msm_plan(int curve, size_t n, const MsmOptions& opt);

// Device-side MSM.  scalars: n x 32 B little-endian; points: n x WIRE bytes
// big-endian affine (all-zero = infinity); out_wire: WIRE bytes; out_comp:
// 48-byte compressed encoding (BLS12-381 only, may be null).  All pointers
// are device pointers; work is queued on `stream` and not synchronised.
class MsmEngine;
MsmEngine* msm_engine_create(int curve);
void msm_engine_destroy(MsmEngine* e);
void msm_run_wire(MsmEngine* e, const uint8_t* d_scalars, const uint8_t* d_points, size_t n,
                  uint8_t* d_out_wire, uint8_t* d_out_comp, cudaStream_t stream,
                  const MsmOptions& opt);
// Same with points already in the internal Montgomery table layout
// (2N words per point) -- used for resident SRS tables.
void msm_run_table(MsmEngine* e, const uint8_t* d_scalars, const uint32_t* d_table, size_t n,
                   uint8_t* d_out_wire, uint8_t* d_out_comp, cudaStream_t stream,
                   const MsmOptions& opt);
// Convert wire points to the internal table layout (device to device).
void points_wire_to_table(int curve, const uint8_t* d_wire, uint32_t* d_table, size_t n,
                          cudaStream_t stream);
// Inverse of points_wire_to_table (canonical big-endian, zeros = infinity).
void points_table_to_wire(int curve, const uint32_t* d_table, uint8_t* d_wire, size_t n,
                          cudaStream_t stream);
// Stage times of the engine's last run when profiling is enabled.
int msm_stage_ms(MsmEngine* e, float* out, int max);
// Words per table entry for a curve.
int table_words(int curve);
// Scratch bytes the engine needs for an MSM of size n (admission control).
size_t msm_scratch_bytes(int curve, size_t n);

}  // namespace kb200
