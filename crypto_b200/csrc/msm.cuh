// G1 multi-scalar multiplication (signed-digit Pippenger) on one GPU, for a
// batch of independent MSMs in one pass (a single MSM is a batch of one).
//
// Pipeline, all on device, all queued on the caller's stream:
//   1. recode          : each scalar -> W signed c-bit digits (c per item);
//                        one (global bucket, point|sign) entry per non-zero
//                        digit; buckets of all items share one key space
//   2. histogram/scan  : per-bucket counts -> bucket offsets
//   3. scatter         : counting sort of the entries by bucket
//   4. accumulate      : buckets split into near-equal segments of <= K
//                        entries, one thread per segment, mixed XYZZ adds;
//                        a persistent grid pulls segments from a device
//                        work counter
//   5. fold            : buckets with more than K2 segments are folded K2
//                        partial sums at a time (skewed inputs); smaller
//                        splits are summed inside stage 6
//   6. reduce          : per window, sum_k (k+1) B_k: running sums per
//                        thread, shared-memory suffix scan and trees per
//                        block, then one block per window over its blocks
//   7. combine         : per item, Horner over windows (c doublings each),
//                        affine normalisation, big-endian / compressed out
// The digit recoding follows gpukit/cpp/cpu_reference/multi_pippenger.cpp:90-134
// (digits in (-2^(c-1), 2^(c-1)], carry into the next window), with enough
// windows (ceil(257 / c)) that no carry leaves the top window.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <climits>
#include <vector>

namespace kb200 {

// Planner cost of one bucket of the reduction, in units of one accumulated
// entry (mixed addition): its two full additions.  (The reduction also has
// a fixed per-block part, the scan and tree phases, that the per-bucket
// model does not see; window choices were checked against measured times.)
constexpr double RED_COST = 2.8;
// The same weight once the batch-affine pairing levels run (from about 2^22
// sorted entries: a level needs 2M pair sums): entries cost less than a
// mixed addition, so a bucket weighs more.  Fitted on B200: BLS12-381 at
// 2^22 over 256-bit windows (the exact drop-in) takes 28.57 / 30.03 / 29.34
// ms at windows 16 / 17 / 15 (reduction 3.9 ms at 524 K buckets, 5.5 ms at
// 983 K), which needs a weight between 9.1 and 17; the GLV halves at 2^22
// keep window 16 (27.2 ms) for any weight above 5.3, BN254 GLV at 2^24
// window 18.
constexpr double RED_COST_PAIRED = 12.0;
constexpr double PAIRED_ENTRIES = (double)(1u << 22);

struct MsmPlan {
    int c = 0;          // window bits
    int W = 0;          // windows
    uint32_t M = 0;     // buckets per window (2^(c-1))
    uint32_t M_top = 0; // live buckets in the top window (its digits are small)
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
    // Shifted fixed-base table: the table passed to the launch holds
    // msm_windows_for(shift_c) levels of shift_stride rows, level w row i =
    // [2^(shift_c * w)] (row i of level 0).  Every item then uses window
    // size shift_c and one bucket range shared by all its windows: no
    // per-window reduction and no doubling chain in the combine.
    // 0 = plain table.
    int shift_c = 0;
    size_t shift_stride = 0;
    // GLV split (plain tables): rows glv_rows + i of the table hold
    // phi(row i) = (beta x, y); scalars split into two halves of at most
    // 128 bits (half the windows over twice the points).  phi acts as
    // [lambda] on the prime-order subgroup: on every BN254 point (cofactor
    // 1), but on BLS12-381 only on G1, not on the whole curve.
    bool glv = false;
    size_t glv_rows = 0;
    // msm_run_wire / msm_run_host_wire: the caller vouches that every point
    // lies in the prime-order subgroup, which lets BLS12-381 use the GLV
    // split.  Without it BLS12-381 keeps 256-bit windows, whose sum equals
    // the reference's for every curve point.  (BN254 always splits.)
    bool points_in_g1 = false;
    int pair_levels = -1; // batch-affine pairing levels (-1: planner's choice or KB200_MSM_PAIR_LEVELS)
    // Host-input pipeline: the first pairing level runs per chunk of point
    // rows as the chunks arrive (sort keys chunk-major).  Single items only;
    // ignored when the planner runs no pairing level.
    int point_chunks = 1;
};

// Average entries per live bucket from which a batch-affine pairing level
// runs before the accumulation, and the most levels the planner runs.
constexpr double PAIR_MIN_RUN = 8.0;
constexpr int PAIR_MAX_LEVELS = 4;
constexpr unsigned long long PAIR_MIN_SLOTS = 1ull << 21;  // additions per level

// Windows of a c-bit signed-digit decomposition of 256-bit scalars.
int msm_windows_for(int c);

// Reference window size for n: multi_pippenger.cpp:69-88.
int reference_best_c(size_t n);
// Window plan for one MSM of size n (autotuner cache, else cost model).
MsmPlan make_msm_plan(int curve, size_t n, const MsmOptions& opt);
// Window plan for a GLV-split MSM of n scalars (2n points; halves below
// 2^128 on BLS12-381, 2^126 on BN254).
MsmPlan make_msm_plan_glv(int curve, size_t n, const MsmOptions& opt);
// Whether a single MSM through msm_run_wire / msm_run_host_wire splits its
// scalars (BN254 always; BLS12-381 when the caller vouches for G1).
bool msm_wire_uses_glv(int curve, const MsmOptions& opt);

// One MSM of a batch: n scalars starting at scalar index `scalar_off` of the
// batch's scalar array, against table rows point_off .. point_off + n - 1.
struct MsmItem {
    size_t scalar_off;
    size_t n;
    size_t point_off;
    size_t out_index = SIZE_MAX;  // result slot (default: the item's position)
};

class MsmBatchPlan;
// Builds the launch plan (descriptors uploaded to the device; synchronous).
MsmBatchPlan* msm_batch_plan_create(int curve, const MsmItem* items, size_t count,
                                    const MsmOptions& opt, cudaStream_t stream);
void msm_batch_plan_destroy(MsmBatchPlan* p);
// Rebuilds an existing plan for new items in place, reusing its device
// descriptor buffers (grow-only) and without synchronising: the upload is
// ordered on `stream` after earlier launches that used the plan, which must
// have been on the same stream.
void msm_batch_plan_update(MsmBatchPlan* p, const MsmItem* items, size_t count,
                           const MsmOptions& opt, cudaStream_t stream);
size_t msm_batch_plan_count(const MsmBatchPlan* p);

class MsmEngine;
MsmEngine* msm_engine_create(int curve);
void msm_engine_destroy(MsmEngine* e);
// Allocates the engine scratch a plan needs (may synchronise the stream).
void msm_engine_reserve(MsmEngine* e, const MsmBatchPlan* p, cudaStream_t stream);
// Queues the whole pipeline for a plan; no allocation and no host
// synchronisation after msm_engine_reserve, so it can be captured in a
// CUDA graph.  out_wire: count * WIRE bytes; out_comp: count * 48 bytes
// (BLS12-381 only, may be null).
// table_ready: null, or n_ready events recorded in order on one stream, the
// last when d_table is complete (event c: the rows of point chunk c, when
// the plan sorts by chunk).  The recode and sort then run without reading
// the table; the stream waits for chunk c before its first pairing level,
// or for the last event before the first stage that reads points.
// scalars_ready: null, or n_ready events, event c when scalar rows
// [c S, (c + 1) S) (S = ceil(n / n_ready)) are resident; for a one-MSM plan
// each chunk's recode and ranking wait only for their own rows.
void msm_engine_launch(MsmEngine* e, const MsmBatchPlan* p, const uint8_t* d_scalars,
                       const uint32_t* d_table, uint8_t* d_out_wire, uint8_t* d_out_comp,
                       cudaStream_t stream, const cudaEvent_t* table_ready = nullptr,
                       int n_ready = 0, const cudaEvent_t* scalars_ready = nullptr);

// Convenience single-MSM entry points (plan cached per (n, options)).
void msm_run_wire(MsmEngine* e, const uint8_t* d_scalars, const uint8_t* d_points, size_t n,
                  uint8_t* d_out_wire, uint8_t* d_out_comp, cudaStream_t stream,
                  const MsmOptions& opt);
// From host buffers: one copy stream brings the scalars and the points in
// row chunks, each point chunk converted to table rows on a third stream.
// When the plan pairs per chunk, chunk by chunk: each chunk is sorted and
// paired (first level) on `stream` once its own scalars and points are
// resident; otherwise all scalars first, each chunk recoded and ranked as it
// lands.  d_scalars (n * 32 bytes) and d_points (n * WIRE bytes) are the
// staging.
void msm_run_host_wire(MsmEngine* e, const uint8_t* h_scalars, const uint8_t* h_points, size_t n,
                       uint8_t* d_scalars, uint8_t* d_points, uint8_t* d_out_wire,
                       cudaStream_t stream, const MsmOptions& opt);
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
// Device scratch bytes an MSM batch of these sizes needs (admission control).
size_t msm_scratch_bytes(int curve, const size_t* ns, size_t count);
// The same bound split into per-item and per-batch parts (additive).
size_t msm_item_scratch_bytes(int curve, size_t n);
size_t msm_batch_fixed_bytes(int curve);

// Autotuner: record the best window for a size class (log2 n) and curve,
// for 256-bit windows or for the windows of GLV halves.
void msm_tune_set(int curve, int log_n, int c, bool glv);
int msm_tune_get(int curve, int log_n, bool glv);  // 0 if untuned

}  // namespace kb200
