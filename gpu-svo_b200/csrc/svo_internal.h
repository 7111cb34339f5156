// svo_internal.h -- launch wrappers shared between the kernel files and the C ABI.
#pragma once
#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>

#include "svo_b200.h"
#include "svo_device.cuh"

namespace svo {

// Counts kernel launches (svo_kernel_launches).
void count_launches(int n);

constexpr int kMaxLevels = 24;
constexpr int kMaxRes = 2048;

// Voxelizer work split.
struct VoxTuning {
    uint32_t serial_max = 64;    // grid-bbox voxels tested by one thread, row by row
    uint32_t warp_max = 256;     // 4x4x4 bricks per queue entry (one warp walks one entry)
    uint32_t split = 0;          // cull 2x2x2 sub-bricks of surviving bricks too
    uint32_t inplace_max = 32;   // bricks of a triangle walked by the warp that set it up
    uint32_t serial_packed = 0;  // serial tier: rows packed across the warp's lanes (else one triangle per lane)
};

// Occupancy bitmap pyramid: level 0 is the voxel grid (one bit per Morton
// code), level l+1 bit j = OR of level-l bits 8j..8j+7.  Every level is stored
// as u64 words padded to whole 512-bit blocks; cnt holds one popcount per
// 512-bit block of every level, pre its exclusive prefix sum.
struct Pyramid {
    int levels = 0;                      // stored levels (>= 5)
    int grid_levels = 0;                 // log2(R) + 1 levels of the real grid
    uint64_t woff[kMaxLevels] = {};      // u64 word offset of level l
    uint64_t words[kMaxLevels] = {};     // u64 words of level l
    uint64_t coff[kMaxLevels + 1] = {};  // block-count offset of level l
    uint64_t total_words = 0;
    uint64_t total_blocks = 0;
    uint32_t ctas = 0;                   // pyramid CTAs (level-0 chunks of 2048 words)
};

Pyramid make_pyramid(int rx, int ry, int rz);

// One mesh of a batch, as the kernels see it (an array in device memory).
// A single build is a batch of one.
struct MeshDev {
    const float *pts;        // device
    const int32_t *tris;     // device; null = soup (3 points per triangle)
    int64_t n_pts;
    int64_t n_tris;
    int res[3];
    int regions;             // 1: level 0 is zeroed and read only in the regions triangles reach
    GridParams *gp;
    uint32_t *mm;            // bbox scratch (6 u32)
    uint64_t *bits;          // this mesh's pyramid (level l at bits + py.woff[l])
    uint32_t *cnt;           // this mesh's block counts (level l at cnt + py.coff[l])
    uint32_t *pre;           // exclusive prefix at this mesh's first block
    uint32_t *totals;        // set bits per level (kMaxLevels)
    uint32_t *done;          // pyramid CTAs finished
    Pyramid py;
};

// Prefix tables over the meshes of a batch (device memory, n + 1 entries).
struct BatchDev {
    const MeshDev *mesh;
    int n;
    const uint64_t *tri_off;   // global index of each mesh's first triangle
    const uint32_t *cta_off;   // first pyramid CTA of each mesh
    const uint32_t *bbox_off;  // first bbox-reduction block of each mesh
    uint8_t *rflag = nullptr;  // per pyramid CTA (a 2048-word region of level 0): a triangle reaches it
};

// Level-0 regions (2048 words: 64 x 64 x 32 voxels) are tracked from this
// level-0 size on (resolution >= 1024).
constexpr uint64_t kRegionWords = 1ull << 24;

// Per-level inputs of the node emission kernel.
struct EmitLevel {
    uint32_t off;          // first node index of the level
    uint32_t n;            // nodes in the level
    const uint64_t *K1;    // sorted codes of level l+1 (the level's groups); level T: its own code
    const uint64_t *bits;  // bitmap of level l
    const uint32_t *wpre;  // rank at each non-empty word of level l (l >= 1)
    uint64_t coff;         // block-count offset of level l
    uint32_t side;         // grid side at this level (R >> l)
    float width;           // node width
};

// One mesh of an emission pass (an array in device memory).
struct EmitParams {
    int T;                  // top level index (depth - 1)
    uint32_t N;             // total nodes
    uint32_t flags;
    EmitLevel lv[kMaxLevels];
    const uint32_t *pre;    // exclusive prefix of the block counts (this mesh's base)
    const GridParams *gp;
    svo_node *nodes;
    svo_vertex *verts;      // may be null (SVO_FLAG_NO_VERT_EDGE)
    svo_edge *edges;
    unsigned long long *dups;  // [0] vertex, [1] edge consecutive duplicates
};

// The meshes of one emission pass: mesh i owns global node slots
// [node_off[i], node_off[i] + N_i), node_off[i] a multiple of 32 (a warp never
// straddles two meshes).
struct EmitBatch {
    const EmitParams *p;
    int n;
    const uint64_t *node_off;  // n + 1 entries
};

// One compaction job: the set bits of levels [l0, l1) of one mesh, level l
// written to out + koff[l]; jobs own consecutive ranges of a global word
// index (word_off, n + 1 entries).
struct CompactJob {
    const uint64_t *bits;
    const uint32_t *pre;
    Pyramid py;
    int l0, l1;
    uint64_t *out;
    uint32_t *wpre;  // optional: rank at each non-empty word of levels >= 1 (indexed from woff[1])
    uint64_t koff[kMaxLevels];
    const uint8_t *rflag;  // region-mode mesh: its level-0 region flags (unflagged regions read as empty)
};
struct CompactBatch {
    const CompactJob *job;
    int n;
    const uint64_t *word_off;
};
// The surface-voxel keys of one mesh, from its non-empty level-0 blocks
// (= its level-3 code list).
struct KeyJob {
    const uint64_t *bits;    // level-0 bitmap
    const uint32_t *pre;     // the mesh's scanned block counts (level 0 first)
    const uint64_t *blocks;  // sorted non-empty block indices
    uint64_t *out;
};
struct KeyBatch {
    const KeyJob *job;
    int n;
    const uint64_t *blk_off;  // prefix of the jobs' block counts
};

// Binary search: the i with off[i] <= x < off[i + 1] (off has n + 1 entries).
template <class T>
__host__ __device__ __forceinline__ int find_segment(const T *off, int n, T x) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= x) lo = mid; else hi = mid - 1;
    }
    return lo;
}

cudaError_t launch_bbox(const BatchDev &b, uint32_t total_blocks, cudaStream_t st);
// mm[0] = min, mm[1] = max of n int32 indices.
cudaError_t launch_index_range(const int32_t *idx, int64_t n, int32_t *mm, cudaStream_t st);
// The same for a table of n index arrays in one launch: job k gets
// index_blocks(jobs[k].n) blocks, block_off their prefix (n + 1 entries);
// mm[2k], mm[2k+1] = min, max of job k.
struct IndexJob {
    const int32_t *idx;
    int64_t n;
};
uint32_t index_blocks(int64_t n);
cudaError_t launch_index_ranges(const IndexJob *jobs, int n, const uint32_t *block_off, uint32_t total_blocks,
                                int32_t *mm, cudaStream_t st);
// counters: 4 u32 (queue entries, queue cursor, -, small-list length); small:
// room for one u64 per triangle, or null (then no in-warp tier unless big is
// null too, which walks every large triangle in the warp that set it up).
cudaError_t launch_voxelize(const BatchDev &b, int64_t total_tris, bool strict, const VoxTuning &tune,
                            uint4 *big, uint32_t big_cap, uint32_t *counters, int num_sms, cudaStream_t st,
                            uint64_t *small = nullptr);
// Builds levels 1.. of every mesh's pyramid and the per-block counts.
cudaError_t launch_pyramid(const BatchDev &b, uint32_t total_ctas, int num_sms, cudaStream_t st);
// Flags the level-0 regions that triangles of region-mode meshes reach, then
// zeroes level 0 where needed (every region of other meshes, the flagged ones
// of region-mode meshes) and each mesh's levels >= 3.  Replaces a memset of
// the whole pyramid; rflag must be zeroed (total_ctas bytes).
cudaError_t launch_regions(const BatchDev &b, int64_t total_tris, uint32_t total_ctas, int num_sms, cudaStream_t st);
// Exclusive scan of n u32 values; out has n + 1 entries (out[n] = total).
// scratch: >= scan_scratch_words(n) u64 words, zeroed by the call.
size_t scan_scratch_words(uint64_t n);
cudaError_t launch_scan(const uint32_t *in, uint32_t *out, uint64_t n, unsigned long long *scratch,
                        uint32_t *status, cudaStream_t st);
// Self-test of the scan's bounded look-back wait: the single-pass scan with
// its tile counter started at 1, so tile 0 never publishes and every
// look-back that reaches it gives up after spin_limit polls and records
// kStatusScanTimeout in *status.  n must span at least 2 tiles; scratch holds
// scan_stalled_scratch_words(n) words (the CTA that draws index `tiles` has no
// tile and publishes one slot past the last).  out (n + 1 entries) receives
// partial sums.  Synchronises st before the launch.
size_t scan_stalled_scratch_words(uint64_t n);
cudaError_t launch_scan_stalled(const uint32_t *in, uint32_t *out, uint64_t n, unsigned long long *scratch,
                                uint32_t *status, int spin_limit, cudaStream_t st);
// Stream-ordered allocation from one of a context's pools: the one place a
// build allocates device memory (svo_debug_fail_alloc injects failures here).
cudaError_t pool_malloc(void **p, size_t bytes, cudaMemPool_t pool, cudaStream_t st);
// totals of every (mesh, level).
cudaError_t launch_level_totals(const BatchDev &b, cudaStream_t st);
cudaError_t launch_compact(const CompactBatch &c, uint64_t total_words, cudaStream_t st);
cudaError_t launch_compact_keys(const KeyBatch &k, uint64_t total_blocks, cudaStream_t st);
// Levels 1 and 2 of a region-mode job (job.rflag set), one block per level-0 region.
cudaError_t launch_compact_regions(const CompactJob &job, uint32_t regions, int num_sms, cudaStream_t st);
// one: the EmitParams of a one-mesh batch (host copy, passed by value to the
// kernel), or null for a batch of several meshes.
cudaError_t launch_emit(const EmitBatch &b, const EmitParams *one, uint64_t total_nodes, uint32_t flags,
                        int num_sms, cudaStream_t st);
// Stable removal of consecutive duplicates (thrust::unique semantics).
cudaError_t launch_unique_vertices(const svo_vertex *in, uint64_t n, svo_vertex *out,
                                   uint32_t *tile_counts, uint32_t *tile_pre,
                                   unsigned long long *scan_scratch, uint32_t *status,
                                   cudaStream_t st);
cudaError_t launch_unique_edges(const svo_edge *in, uint64_t n, svo_edge *out, uint32_t *tile_counts,
                                uint32_t *tile_pre, unsigned long long *scan_scratch,
                                uint32_t *status, cudaStream_t st);
constexpr uint32_t kUniqueTile = 4096;

// Morton-keyed unique vertex/edge/face keys of all nodes (SVO_FLAG_DEDUP), in
// two steps on one stream.  dedup_begin needs only the level bitmaps (bits[l],
// side sides[l], l = 0..T): it takes the scratch and builds the level-1 part
// of the candidate bitmap, so it can run before the code lists exist.
// dedup_finish (after the code lists, ep) writes the keys and frees the run;
// dedup_abort frees a run that will not be finished.
struct DedupRun;
int dedup_begin(cudaMemPool_t scratch_pool, cudaStream_t st, int T, const uint64_t *const *bits,
                const uint32_t *sides, int num_sms, DedupRun **run);
int dedup_finish(DedupRun *run, cudaMemPool_t out_pool, const EmitParams &ep, uint64_t n_out[3], uint64_t *out[3]);
void dedup_abort(DedupRun *run);

// Blocks of the bbox reduction for a mesh of n points.
inline uint32_t bbox_blocks(int64_t n) {
    return (uint32_t)std::max<int64_t>(1, std::min<int64_t>((n / 4 + 255) / 256, 148 * 4));
}

}  // namespace svo
