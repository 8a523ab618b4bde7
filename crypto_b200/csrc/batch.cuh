// Batched KZG commits over BLS12-381 against a resident SRS table.
//
// A batch of polynomials of uneven sizes (evaluations stored back to back)
// is committed in one pass: the inverse NTTs run grouped by size class (one
// launch sequence per class, over a device list of vector offsets), then a
// single batched MSM covers every commit against the shared SRS (per-commit
// window sizes, one bucket key space, persistent accumulation kernel with a
// device work counter, one combine thread per commit).  The whole device
// sequence is captured once per size signature into a CUDA graph and
// replayed.  Results are byte-identical to one kzg_commit_fr per polynomial.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

namespace kb200 {

class CommitBatcher;
struct ShiftTables;
CommitBatcher* commit_batcher_create();
void commit_batcher_destroy(CommitBatcher* b);
// Shifted tables over the SRS the batcher is given (null = plain MSMs).
void commit_batcher_set_shift(CommitBatcher* b, ShiftTables* shifts);
// Transient mode: no per-signature cache or graphs; one plan set rebuilt in
// place per batch without synchronising (for streams of unrepeated batches).
void commit_batcher_set_transient(CommitBatcher* b, bool transient);

// Commits `count` polynomials.  h_evals: host evaluations (32 B LE each,
// back to back in the order of sizes); h_out: 48 * count bytes.  srs_table:
// device SRS in table layout with srs_n points.  `use_graph` selects graph
// capture/replay (on by default at the C ABI).  Synchronous.
void commit_batch_host(CommitBatcher* b, const uint8_t* h_evals, const size_t* sizes,
                       size_t count, const uint32_t* srs_table, size_t srs_n, uint8_t* h_out,
                       cudaStream_t stream, bool use_graph);

// Same, with the evaluations already in the batcher's device buffer
// (commit_batch_device_input returns it, sized for the signature) and the
// compressed results left on the device (commit_batch_device_output).
uint8_t* commit_batch_device_input(CommitBatcher* b, const size_t* sizes, size_t count,
                                   const uint32_t* srs_table, size_t srs_n, cudaStream_t stream);
void commit_batch_device(CommitBatcher* b, const size_t* sizes, size_t count,
                         const uint32_t* srs_table, size_t srs_n, cudaStream_t stream,
                         bool use_graph);
const uint8_t* commit_batch_device_output(CommitBatcher* b);

// Device bytes a batch of these sizes needs (evaluations, NTT scratch, MSM).
size_t commit_batch_scratch_bytes(const size_t* sizes, size_t count);
// Its additive parts: per commit and per batch.
size_t commit_item_scratch_bytes(size_t n);
size_t commit_batch_fixed_bytes();

// Number of graph replays / captures so far (for tests).
unsigned long long commit_batcher_graph_launches(CommitBatcher* b);
unsigned long long commit_batcher_graph_captures(CommitBatcher* b);

}  // namespace kb200
