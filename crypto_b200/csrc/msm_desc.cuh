// Device-side descriptors and launcher table shared by the MSM host driver
// (msm.cu) and the per-curve kernel units (msm_bls.cu, msm_bn.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace kb200 {

constexpr uint32_t KEY_SENTINEL = 0xffffffffu;
constexpr int RED_THREADS = 256;
constexpr int RED_QSLOTS = RED_THREADS / 4;       // slots of a quad-lane reduction block
constexpr size_t RED_QUAD_MAX_LIVE = 16384;      // live buckets up to which the quads run

// One MSM of a batch.
struct ItemDesc {
    unsigned long long scalar_off;  // first scalar (element index) of the item
    unsigned long long entry_base;  // first entry slot (W * n slots per item)
    uint32_t n;
    uint32_t point_off;             // first table row
    uint32_t c, W, M;               // window bits, windows, buckets per window
    uint32_t bucket_base;           // first global bucket of the item
    uint32_t win_base;              // first WinDesc of the item
    int32_t quirk_c;                // reference carry emulation (0, 4 or 8)
    uint32_t row_stride;            // shifted table: rows per level (0 = plain table)
    uint32_t Wr;                    // windows reduced and combined (W, or 1 when shifted)
    uint32_t out_index;             // result slot in the output arrays
    uint32_t glv;                   // 1: GLV split (BLS12-381), 2 W n entries
    uint32_t glv_off;               // row offset of the phi(P) rows in the table
    uint32_t chunk_rows;            // >0: sort key (chunk of the point) * chunk_stride + bucket,
    uint32_t chunk_stride;          //     chunk = point index / chunk_rows (per-chunk level 0)
};

// One window of one item.
struct WinDesc {
    uint32_t bucket_base;  // global id of the window's bucket 0
    uint32_t Mw;           // live buckets of the window
    uint32_t S;            // buckets per thread in reduction stage 1
    uint32_t blk_base;     // first stage-1 block of the window
    uint32_t nb;           // stage-1 blocks (<= RED_THREADS)
    uint32_t blk;          // buckets per stage-1 block (RED_THREADS * S)
    uint32_t shift;        // c * w: the window's weight is 2^shift
};

struct BlkDesc {
    uint32_t win;  // WinDesc index
    uint32_t b;    // block index within the window
};

// Level-1 accumulation over fixed chunks of K sorted entries.  Chunk t
// writes the sum of its first bucket's run to rec_first[t], of its last
// bucket's run (when different) to rec_last[t], and of every bucket lying
// strictly inside the chunk directly to buckets[].
struct AccArgs {
    const uint32_t* sorted;   // entry -> table row | sign << 31 (null: entry e is row e)
    const uint32_t* offsets;  // B + 1 bucket offsets into sorted; offsets[B] = entries
    uint32_t B;
    uint32_t K;               // entries per chunk
    const uint32_t* table;
    uint32_t* rec_first;
    uint32_t* rec_last;
    uint32_t* buckets;
    uint32_t* queue;
};

// Buckets spanning more than K2 + 1 chunks ("big": the top window's carry
// bucket for uniform scalars, the small-digit buckets of skewed inputs) have
// their records rec_first[t0+1 .. t1] folded FK at a time per level; the
// total lands in rec_first[t0 + 1].  big_list = {count, bucket ids...}.
struct FoldArgs {
    const uint32_t* offsets;
    uint32_t B;
    uint32_t K;
    int K2;
    int FK;
    const uint32_t* big_list;
    uint32_t big_cap;
    const uint32_t* prefix;  // the level's slice (big_cap + 1) of the exclusive prefix of
                             // all levels' group counts; relative to prefix[0]
    uint32_t* rec_first;
};

// Batch-affine pairing level: the bucket-sorted list (runs in_off[b] ..
// in_off[b+1]) -> each run's consecutive pairs added in affine coordinates
// (an odd run's last point passes through), output runs at out_off.
struct PairArgs {
    const uint32_t* in_off;   // B + 1
    const uint32_t* out_off;  // B + 1
    uint32_t B;
    const uint32_t* sorted;   // level 0: table rows | sign << 31; later levels: null
    const uint32_t* src;      // level 0: the point table; later: previous level's rows
    uint32_t* dst;            // output rows (affine, 2N words, infinity flagged)
    const uint32_t* dst_off;  // null: slot k writes row k; else run r's slots go to rows
                              // dst_off[r] + (k - out_off[r]) (per-chunk level 0)
};

// Pairing-level geometry: slots per thread of the pair passes; the
// batch inversion of the level's per-thread totals runs as one grid of
// INV_T-thread blocks, each thread chaining up to INV_G elements and each
// block inverting its own product.  G is the smallest chain length that keeps
// the grid at about INV_FILL threads (two 256-thread blocks on each of 148
// SMs), so large levels stay throughput-bound and small ones short; up to 32
// keeps a 2^22 MSM's first level in one wave (16 left it 549 blocks, about
// two waves, each paying a block's inversion latency).
constexpr int PAIR_J = 16;
constexpr int INV_G = 32;
constexpr int INV_T = 256;
constexpr size_t INV_FILL = (size_t)2 * 148 * INV_T;

struct InvGeom {
    uint32_t G;   // elements per thread
    uint32_t nb;  // blocks
};
inline InvGeom inv_geom(size_t M) {
    size_t G = (M + INV_FILL - 1) / INV_FILL;
    G = G < 1 ? 1 : (G > (size_t)INV_G ? (size_t)INV_G : G);
    const size_t per_block = (size_t)INV_T * G;
    return {(uint32_t)G, (uint32_t)((M + per_block - 1) / per_block)};
}

// Scratch words of one pairing level with T0 pair threads and N-word field
// elements: the pair prefixes and totals, then the inversion's running
// products (the layout pair_level carves).
inline size_t pair_scratch_words(size_t T0, int N) {
    const InvGeom g = inv_geom(T0);
    return (size_t)PAIR_J * N * T0 + (size_t)(g.G - 1) * N * g.nb * INV_T;
}

struct RedArgs {
    const uint32_t* offsets;
    uint32_t B;
    const uint32_t* buckets;
    const uint32_t* rec_first;
    const uint32_t* rec_last;
    uint32_t K;
    int K2;
    const WinDesc* wins;
    const BlkDesc* blks;
    uint32_t* blk_out;   // 2 XYZZ points per stage-1 block
    uint32_t* win_out;   // 1 XYZZ point per window
    uint32_t* win_done;  // stage-1 blocks finished per window (zeroed before the launch)
};

struct MsmLaunchers {
    void (*wire_to_table)(const uint8_t*, uint32_t*, size_t, size_t, cudaStream_t);
    void (*table_to_wire)(const uint32_t*, uint8_t*, size_t, cudaStream_t);
    void (*recode)(const ItemDesc*, uint32_t, unsigned long long, unsigned long long,
                   const uint32_t*, const uint32_t*, uint32_t*, uint32_t*, cudaStream_t);
    void (*accumulate)(const AccArgs&, unsigned, cudaStream_t);
    void (*pair_level)(const PairArgs&, uint32_t, uint32_t*, cudaStream_t);
    void (*fold)(const FoldArgs&, int, const uint32_t*, uint32_t*, unsigned, cudaStream_t);
    void (*reduce_blocks)(const RedArgs&, unsigned, cudaStream_t);
    void (*reduce_blocks_quad)(const RedArgs&, unsigned, cudaStream_t);
    void (*combine)(const ItemDesc*, uint32_t, const uint32_t*, uint8_t*, uint8_t*, cudaStream_t);
    int (*accumulate_occupancy)();
    int point_words;  // XYZZ point
    int table_words;  // affine table row
    int wire_bytes;
};

// Items of fold level l for big bucket g: n_1 = t1 - t0 records, n_l =
// ceil(n_{l-1} / FK); a level has n_l groups when n_{l-1} > 1, else none.
__device__ __forceinline__ void fold_sizes(uint32_t o, uint32_t c, uint32_t K, int FK, int level,
                                           uint32_t& t0, uint32_t& n_prev, uint32_t& n_cur) {
    t0 = o / K;
    const uint32_t t1 = (o + c - 1) / K;
    n_prev = t1 - t0;
    for (int l = 2; l < level; ++l) n_prev = (n_prev + FK - 1) / FK;
    n_cur = n_prev <= 1 ? 0u : (n_prev + FK - 1) / FK;
}

const MsmLaunchers& msm_launchers(int curve);

// Raises a kernel's dynamic shared-memory limit once per device.
void set_smem_attr(const void* kernel, size_t bytes);

}  // namespace kb200
