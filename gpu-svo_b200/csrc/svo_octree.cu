// svo_octree.cu -- octree levels, node records, vertex/edge arrays.
//
// The reference builds the octree bottom-up one level per host iteration
// (src/SVO.cu:383-495): compact a dense flag array, group codes by parent,
// place each group's 8 siblings, fill missing siblings, link parents and
// children.  Here every level comes out of one occupancy-bitmap pyramid:
//   * level l+1 bit j is the OR of level-l bits 8j..8j+7 (a byte test), so
//     one streaming pass builds all levels (k_pyramid);
//   * one popcount per 512-bit block and a single exclusive scan give O(1)
//     rank queries on every level (k_scan);
//   * the node at local index 8g+k of level l has code 8*K[l+1][g] + k, where
//     K[l+1] is the sorted list of set bits of level l+1 (k_compact); its
//     children start at 8*rank_l(code) in level l-1, its parent sits at
//     8*rank_{l+2}(code >> 6) + ((code >> 3) & 7) in level l+1 -- exactly the
//     indices the reference's scans produce (src/SVO.cu:221-339);
//   * k_emit writes node records, vertex and edge arrays in one pass, staged
//     per warp in shared memory so every global store is a full 512-byte
//     coalesced streaming write.
#include <cuda/atomic>

#include "svo_internal.h"

namespace svo {

Pyramid make_pyramid(int rx, int ry, int rz) {
    Pyramid py;
    int rmax = std::max(rx, std::max(ry, rz));
    int k = 0;
    while ((1 << k) < rmax) ++k;
    py.grid_levels = k + 1;
    py.levels = std::max(py.grid_levels, 5);
    const uint64_t bits0 = 1ull << (3 * k);
    uint64_t w0 = (bits0 + 63) / 64;
    w0 = std::max<uint64_t>(w0, 2048);
    w0 = (w0 + 2047) / 2048 * 2048;
    auto up8 = [](uint64_t v) { return (v + 7) / 8 * 8; };
    py.words[0] = w0;
    py.words[1] = w0 / 8;
    py.words[2] = w0 / 64;
    py.words[3] = up8(w0 / 512);
    py.words[4] = up8((w0 / 2048 + 1) / 2);
    for (int l = 5; l < py.levels; ++l) py.words[l] = up8((py.words[l - 1] + 7) / 8);
    uint64_t wo = 0, co = 0;
    for (int l = 0; l < py.levels; ++l) {
        py.woff[l] = wo;
        py.coff[l] = co;
        wo += py.words[l];
        co += py.words[l] / 8;
    }
    py.coff[py.levels] = co;
    py.total_words = wo;
    py.total_blocks = co;
    py.ctas = (uint32_t)(w0 / 2048);
    return py;
}

namespace {

// 8-bit mask of the non-zero bytes of v.
__device__ __forceinline__ uint32_t nz_bytes(uint64_t v) {
    uint64_t m = v | (v >> 4);
    m |= m >> 2;
    m |= m >> 1;
    m &= 0x0101010101010101ull;
    return (uint32_t)((m * 0x0102040810204080ull) >> 56);
}

// Levels 1..4 of 2048-word chunks of level 0 (regions), a persistent grid
// taking them in turn (one 512-bit block of level 0 per thread, 16-byte
// streaming loads); the levels above 4 come from k_pyramid_top.  A
// region-mode mesh's region that no triangle reaches is empty and is not read
// (its level-0 words are not zeroed in memory): its words of levels 1..4 are
// written as zeros and its counts stay at their memset zero.
__global__ void __launch_bounds__(256, 8) k_pyramid(BatchDev bd, uint32_t total) {
    __shared__ uint64_t s1[256];
    __shared__ uint64_t s2[32];
    __shared__ uint64_t s3[4];
    const uint32_t t = threadIdx.x;
    for (uint32_t g = blockIdx.x; g < total; g += gridDim.x) {
        const int m = find_segment(bd.cta_off, bd.n, g);
        const MeshDev &md = bd.mesh[m];
        const Pyramid &py = md.py;
        uint64_t *__restrict__ bits = md.bits;
        uint32_t *__restrict__ cnt = md.cnt;
        const uint32_t b = g - bd.cta_off[m];
        if (md.regions && !bd.rflag[g]) {  // the same for the whole CTA
            bits[py.woff[1] + (uint64_t)b * 256 + t] = 0;
            if (t < 32) bits[py.woff[2] + (uint64_t)b * 32 + t] = 0;
            if (t < 4) bits[py.woff[3] + (uint64_t)b * 4 + t] = 0;
            if (t == 0) reinterpret_cast<uint32_t *>(bits + py.woff[4])[b] = 0;
            continue;
        }
        {
            const uint4 *src = reinterpret_cast<const uint4 *>(bits + py.woff[0] + (uint64_t)b * 2048 + t * 8);
            uint64_t w1 = 0;
            uint32_t c0 = 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint4 v = __ldcs(src + q);
                const uint64_t a = ((uint64_t)v.y << 32) | v.x, c = ((uint64_t)v.w << 32) | v.z;
                c0 += __popcll(a) + __popcll(c);
                w1 |= (uint64_t)nz_bytes(a) << (16 * q);
                w1 |= (uint64_t)nz_bytes(c) << (16 * q + 8);
            }
            cnt[py.coff[0] + (uint64_t)b * 256 + t] = c0;
            bits[py.woff[1] + (uint64_t)b * 256 + t] = w1;
            s1[t] = w1;
        }
        __syncthreads();
        if (t < 32) {
            uint64_t w = 0;
            uint32_t c = 0;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const uint64_t v = s1[8 * t + k];
                c += __popcll(v);
                w |= (uint64_t)nz_bytes(v) << (8 * k);
            }
            cnt[py.coff[1] + (uint64_t)b * 32 + t] = c;
            bits[py.woff[2] + (uint64_t)b * 32 + t] = w;
            s2[t] = w;
        }
        __syncthreads();
        if (t < 4) {
            uint64_t w = 0;
            uint32_t c = 0;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const uint64_t v = s2[8 * t + k];
                c += __popcll(v);
                w |= (uint64_t)nz_bytes(v) << (8 * k);
            }
            cnt[py.coff[2] + (uint64_t)b * 4 + t] = c;
            bits[py.woff[3] + (uint64_t)b * 4 + t] = w;
            s3[t] = w;
        }
        __syncthreads();
        if (t == 0) {
            uint32_t w = 0, c = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                c += __popcll(s3[k]);
                w |= nz_bytes(s3[k]) << (8 * k);
            }
            if (c) atomicAdd(cnt + py.coff[3] + b / 2, c);
            reinterpret_cast<uint32_t *>(bits + py.woff[4])[b] = w;
        }
        __syncthreads();  // s1..s3 are rewritten by the next region
    }
}

// Levels 5.. and the counts of levels 4.. of every mesh: one CTA per mesh.
__global__ void __launch_bounds__(256) k_pyramid_top(BatchDev bd) {
    const MeshDev &md = bd.mesh[blockIdx.x];
    const Pyramid &py = md.py;
    uint64_t *__restrict__ bits = md.bits;
    uint32_t *__restrict__ cnt = md.cnt;
    const uint32_t t = threadIdx.x;
    for (int l = 4; l < py.levels; ++l) {
        const uint64_t *in = bits + py.woff[l];
        const uint64_t nblk = py.words[l] / 8;
        const bool has_next = l + 1 < py.levels;
        uint64_t *out = has_next ? bits + py.woff[l + 1] : nullptr;
        for (uint64_t j = t; j < nblk; j += blockDim.x) {
            uint64_t w = 0;
            uint32_t c = 0;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const uint64_t v = in[8 * j + k];
                c += __popcll(v);
                w |= (uint64_t)nz_bytes(v) << (8 * k);
            }
            cnt[py.coff[l] + j] = c;
            if (has_next) out[j] = w;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Single-pass exclusive scan (decoupled look-back).  Tile status words hold
// (flag << 32 | value): flag 1 = tile aggregate, 2 = inclusive prefix.  The
// look-back wait is bounded; on timeout the kernel records
// kStatusScanTimeout and the host fails the build.
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr uint64_t kScanTile = kScanThreads * kScanItems;
constexpr int kSpinLimit = 1 << 22;
constexpr uint64_t kScanSplitTiles = 64;  // from this many tiles on (aligned data): reduce-then-scan

__device__ __forceinline__ unsigned long long ld_relaxed(unsigned long long *p) {
    return cuda::atomic_ref<unsigned long long, cuda::thread_scope_device>(*p).load(
        cuda::memory_order_relaxed);
}
__device__ __forceinline__ void st_relaxed(unsigned long long *p, unsigned long long v) {
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device>(*p).store(v, cuda::memory_order_relaxed);
}

__global__ void __launch_bounds__(kScanThreads) k_scan(const uint32_t *__restrict__ in,
                                                       uint32_t *__restrict__ out, uint64_t n,
                                                       unsigned long long *__restrict__ scratch,
                                                       uint32_t *__restrict__ status, int spin_limit) {
    __shared__ uint32_t s_tile, s_prefix;
    __shared__ uint32_t s_warp[kScanThreads / 32];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    if (t == 0) s_tile = atomicAdd(reinterpret_cast<unsigned int *>(scratch), 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    unsigned long long *st = scratch + 1;
    const uint64_t base = tile * kScanTile + (uint64_t)t * kScanItems;
    uint32_t v[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < n ? in[base + k] : 0u;
        sum += v[k];
    }
    uint32_t incl = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, incl, d);
        if (lane >= d) incl += o;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kScanThreads / 32 ? s_warp[lane] : 0u;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, w, d);
            if (lane >= d) w += o;
        }
        if (lane < kScanThreads / 32) s_warp[lane] = w;  // inclusive warp totals
    }
    __syncthreads();
    const uint32_t aggregate = s_warp[kScanThreads / 32 - 1];
    if (warp == 0) {
        uint32_t prefix = 0;
        if (tile == 0) {
            if (lane == 0) st_relaxed(st, (2ull << 32) | aggregate);
        } else {
            if (lane == 0) st_relaxed(st + tile, (1ull << 32) | aggregate);
            int64_t j = (int64_t)tile - 1;
            int spins = 0;
            for (;;) {
                const int64_t q = j - lane;
                const unsigned long long s = q >= 0 ? ld_relaxed(st + q) : (2ull << 32);
                const uint32_t flag = (uint32_t)(s >> 32);
                if (__any_sync(0xFFFFFFFFu, flag == 0)) {
                    if (++spins > spin_limit) {
                        if (lane == 0) atomicOr(status, kStatusScanTimeout);
                        break;
                    }
                    __nanosleep(64);
                    continue;
                }
                const uint32_t m2 = __ballot_sync(0xFFFFFFFFu, flag == 2);
                const int stop = m2 ? __ffs(m2) - 1 : 31;
                uint32_t val = lane <= stop ? (uint32_t)s : 0u;
#pragma unroll
                for (int d = 16; d > 0; d >>= 1) val += __shfl_xor_sync(0xFFFFFFFFu, val, d);
                prefix += val;
                if (m2) break;
                j -= 32;
            }
            if (lane == 0) st_relaxed(st + tile, (2ull << 32) | (prefix + aggregate));
        }
        if (lane == 0) s_prefix = prefix;
    }
    __syncthreads();
    uint32_t run = s_prefix + (warp ? s_warp[warp - 1] : 0u) + (incl - sum);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    const uint64_t last_tile = (n + kScanTile - 1) / kScanTile - 1;
    if (tile == last_tile && t == kScanThreads - 1) out[n] = s_prefix + aggregate;
}

// Reduce-then-scan for long, 16-byte aligned arrays: tile sums, one CTA
// scanning them, then each tile scanned again with its prefix added.  Three
// streaming passes, no inter-CTA waiting; every thread moves its 16 items
// with 16-byte loads and stores.
__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t *s_warp) {
    v = __reduce_add_sync(0xFFFFFFFFu, v);
    if ((threadIdx.x & 31) == 0) s_warp[threadIdx.x >> 5] = v;
    __syncthreads();
    uint32_t t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_warp[w];
    return t;
}

__device__ __forceinline__ void load_items(const uint32_t *in, uint64_t base, uint64_t n, uint32_t v[kScanItems]) {
    if (base + kScanItems <= n) {
        const uint4 *p = reinterpret_cast<const uint4 *>(in + base);
#pragma unroll
        for (int q = 0; q < kScanItems / 4; ++q) {
            const uint4 x = __ldcs(p + q);
            v[4 * q] = x.x;
            v[4 * q + 1] = x.y;
            v[4 * q + 2] = x.z;
            v[4 * q + 3] = x.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) v[k] = base + k < n ? in[base + k] : 0u;
    }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const uint32_t *__restrict__ in, uint64_t n,
                                                              uint32_t *__restrict__ tsum) {
    __shared__ uint32_t s_warp[kScanThreads / 32];
    uint32_t v[kScanItems];
    load_items(in, blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems, n, v);
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) sum += v[k];
    sum = block_sum(sum, s_warp);
    if (threadIdx.x == 0) tsum[blockIdx.x] = sum;
}

// Exclusive prefix of the tile sums (one CTA of 1024 threads) and the grand
// total at *total.
__global__ void __launch_bounds__(1024) k_scan_tiles(const uint32_t *__restrict__ tsum, uint32_t *__restrict__ tpre,
                                                     uint64_t tiles, uint32_t *__restrict__ total) {
    __shared__ uint32_t s_warp[32];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    uint32_t carry = 0;
    for (uint64_t base = 0; base < tiles; base += 1024) {
        const uint64_t i = base + t;
        const uint32_t v = i < tiles ? tsum[i] : 0u;
        uint32_t incl = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, incl, d);
            if (lane >= d) incl += o;
        }
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = s_warp[lane];
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, w, d);
                if (lane >= d) w += o;
            }
            s_warp[lane] = w;  // inclusive warp totals
        }
        __syncthreads();
        if (i < tiles) tpre[i] = carry + (warp ? s_warp[warp - 1] : 0u) + incl - v;
        carry += s_warp[31];
        __syncthreads();  // s_warp is rewritten by the next round
    }
    if (t == 0) *total = carry;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_down(const uint32_t *__restrict__ in, uint32_t *__restrict__ out,
                                                            uint64_t n, const uint32_t *__restrict__ tpre) {
    __shared__ uint32_t s_warp[kScanThreads / 32];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint64_t base = blockIdx.x * kScanTile + (uint64_t)t * kScanItems;
    uint32_t v[kScanItems];
    load_items(in, base, n, v);
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) sum += v[k];
    uint32_t incl = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, incl, d);
        if (lane >= d) incl += o;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    uint32_t run = tpre[blockIdx.x] + incl - sum;
    for (int w = 0; w < warp; ++w) run += s_warp[w];
    uint32_t o[kScanItems];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        o[k] = run;
        run += v[k];
    }
    if (base + kScanItems <= n) {
        uint4 *q = reinterpret_cast<uint4 *>(out + base);
#pragma unroll
        for (int j = 0; j < kScanItems / 4; ++j) q[j] = make_uint4(o[4 * j], o[4 * j + 1], o[4 * j + 2], o[4 * j + 3]);
    } else {
#pragma unroll
        for (int k = 0; k < kScanItems; ++k)
            if (base + k < n) out[base + k] = o[k];
    }
}

__global__ void k_level_totals(BatchDev bd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = i / kMaxLevels, l = i % kMaxLevels;
    if (m >= bd.n) return;
    const MeshDev &md = bd.mesh[m];
    if (l < md.py.levels) md.totals[l] = md.pre[md.py.coff[l + 1]] - md.pre[md.py.coff[l]];
}

// One thread per 64-bit word of every job's levels: its first rank is the
// block prefix plus the popcounts of the preceding words of its block.
// One thread per bitmap word; the 8 lanes of a 512-bit block are 8 aligned
// lanes of a warp (every level and job starts on a block boundary), so a
// word's rank in its level is the block's scanned base plus an 8-lane prefix
// of popcounts.  Writes the sorted set-bit positions and, for levels >= 1
// when wpre is given, the rank at each non-empty word (rank_of's table).
// In a region-mode mesh a word of levels 0-3 lies inside one level-0 region
// (level-l word w covers level-0 words w * 8^l ..): an unflagged one is
// empty and is not read.
// The set-bit codes of the warp's 32 words, whose outputs are one contiguous
// range in lane order (lane i's codes at o, o + 1, ...; lanes without bits
// hold pc = 0): staged in shared memory as (lane, bit) entries, then read in
// order, each turned into its code (the owning lane's b64 + bit) and stored
// coalesced.  All 32 lanes call; lane 0 must hold a word of the range.
__device__ __forceinline__ void warp_codes(uint64_t *out, uint32_t o, uint32_t pc, uint64_t v, uint64_t b64,
                                           uint16_t *stage, int lane) {
    const uint32_t start = __shfl_sync(0xFFFFFFFFu, o, 0);
    const uint32_t tot = __reduce_add_sync(0xFFFFFFFFu, pc);
    uint32_t at = o - start;
    for (uint64_t m = v; m; m &= m - 1) stage[at++] = (uint16_t)((uint32_t)lane << 6 | (uint32_t)(__ffsll((long long)m) - 1));
    __syncwarp();
    const uint32_t blo = (uint32_t)b64, bhi = (uint32_t)(b64 >> 32);
    for (uint32_t i0 = 0; i0 < tot; i0 += 32) {
        const uint32_t i = i0 + lane;
        const uint32_t e = i < tot ? stage[i] : 0u;
        const int src = (int)(e >> 6);
        const uint64_t base = (uint64_t)__shfl_sync(0xFFFFFFFFu, bhi, src) << 32 | __shfl_sync(0xFFFFFFFFu, blo, src);
        if (i < tot) out[start + i] = base + (e & 63u);
    }
    __syncwarp();
}

// Word w of level l holding v (read by the caller; 0 for a lane without a
// word): rank from the block prefix and the 8-lane popcount prefix, then the
// positions.  All 32 lanes of the warp call (8 aligned lanes per block).
__device__ __forceinline__ void compact_word(const CompactJob &job, int l, uint64_t w, uint64_t v) {
    const int sub = threadIdx.x & 7;
    const uint32_t r0 = v ? job.pre[job.py.coff[l] + (w >> 3)] - job.pre[job.py.coff[l]] : 0u;
    const uint32_t pc = __popcll(v);
    uint32_t x = pc;
#pragma unroll
    for (int d = 1; d < 8; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d, 8);
        if (sub >= d) x += y;
    }
    const uint32_t r = r0 + x - pc;
    if (!v) return;
    if (job.wpre && l >= 1) job.wpre[job.py.woff[l] - job.py.woff[1] + w] = r;
    uint64_t *o = job.out + job.koff[l] + r;
    const uint64_t b64 = w * 64;
    while (v) {
        *o++ = b64 + __ffsll((long long)v) - 1;
        v &= v - 1;
    }
}

__global__ void __launch_bounds__(256) k_compact(CompactBatch cb, uint64_t total) {
    const uint64_t gi = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (gi >= ((total + 31) & ~31ull)) return;  // whole warps stay for the shuffles
    uint64_t v = 0, w = 0;
    int l = 0, j = 0;
    if (gi < total) {
        j = find_segment(cb.word_off, cb.n, gi);
        const CompactJob &job = cb.job[j];
        const Pyramid &py = job.py;
        const uint64_t gw = py.woff[job.l0] + (gi - cb.word_off[j]);
        l = job.l0;
        while (l + 1 < job.l1 && gw >= py.woff[l + 1]) ++l;
        w = gw - py.woff[l];
        v = (l <= 3 && job.rflag && !job.rflag[w >> (11 - 3 * l)]) ? 0ull : job.bits[gw];
    }
    compact_word(cb.job[j], l, w, v);
}

// Levels 1 and 2 of a region-mode mesh, region by region (a block takes
// level-0 regions in turn): the 256 level-1 and 32 level-2 words above a
// region lie inside it, so an unflagged region (most of them at res 2048)
// costs one flag read.
__global__ void __launch_bounds__(256) k_compact_regions(const __grid_constant__ CompactJob job, uint32_t regions) {
    for (uint32_t rg = blockIdx.x; rg < regions; rg += gridDim.x) {
        if (!job.rflag[rg]) continue;
        const uint64_t w1 = (uint64_t)rg * 256 + threadIdx.x;
        compact_word(job, 1, w1, job.bits[job.py.woff[1] + w1]);
        if (threadIdx.x < 32) {
            const uint64_t w2 = (uint64_t)rg * 32 + threadIdx.x;
            compact_word(job, 2, w2, job.bits[job.py.woff[2] + w2]);
        }
    }
}

// Level-0 set bits (the surface-voxel keys) from the non-empty 512-bit blocks
// only: a mesh's level-3 code list is exactly its non-empty level-0 blocks,
// in order.  8 lanes per block, one word each.
__global__ void __launch_bounds__(256) k_compact_keys(KeyBatch kb, uint64_t total_blocks) {
    __shared__ uint16_t stage[8][2048];  // a warp's 4 blocks x 512 bits
    const uint64_t gi = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t item = gi >> 3;
    if (((gi >> 5) << 2) >= total_blocks) return;  // whole warps stay for the shuffles
    const int sub = threadIdx.x & 7;
    uint64_t v = 0, blk = 0;
    uint32_t r = 0;
    int j = 0;
    if (item < total_blocks) {
        j = find_segment(kb.blk_off, kb.n, item);
        const KeyJob &job = kb.job[j];
        blk = job.blocks[item - kb.blk_off[j]];
        v = job.bits[blk * 8 + sub];
        r = job.pre[blk] - job.pre[0];
    }
    const uint32_t pc = __popcll(v);
    uint32_t x = pc;
#pragma unroll
    for (int d = 1; d < 8; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d, 8);
        if (sub >= d) x += y;
    }
    // the warp's blocks are consecutive non-empty blocks of one mesh (its
    // outputs one range) unless it straddles two meshes
    const int j0 = __shfl_sync(0xFFFFFFFFu, j, 0);
    if (__all_sync(0xFFFFFFFFu, item >= total_blocks || j == j0)) {
        warp_codes(kb.job[j0].out, item < total_blocks ? r + x - pc : 0xFFFFFFFFu, pc, v, (blk * 8 + sub) * 64,
                   stage[threadIdx.x >> 5], threadIdx.x & 31);
        return;
    }
    if (!v) return;
    uint64_t *o = kb.job[j].out + r + x - pc;
    const uint64_t b64 = (blk * 8 + sub) * 64;
    while (v) {
        *o++ = b64 + __ffsll((long long)v) - 1;
        v &= v - 1;
    }
}

// ---------------------------------------------------------------------------
// Node emission.
// ---------------------------------------------------------------------------
struct NodeInfo {
    uint64_t code;
    uint64_t pc;  // parent code (level l+1)
    int l;
    bool real;
    uint32_t child0;
    uint32_t parent;
    float o[3];
    float w;
};

// Rank of set bit c among level l's set bits (l >= 1): the word's rank from
// k_compact plus the set bits below c in its word.
__device__ __forceinline__ uint32_t rank_of(const EmitParams &P, int l, uint64_t c) {
    const uint64_t w = c >> 6;
    return P.lv[l].wpre[w] + (uint32_t)__popcll(P.lv[l].bits[w] & ((1ull << (c & 63)) - 1ull));
}

template <bool S>
__device__ __forceinline__ void node_info(const EmitParams &P, const float go[3], uint32_t t, NodeInfo &ni) {
    int l = 0;
    while (l < P.T && t >= P.lv[l + 1].off) ++l;
    const uint32_t i = t - P.lv[l].off;
    ni.l = l;
    if (l < P.T) {
        ni.pc = P.lv[l].K1[i >> 3];
        ni.code = (ni.pc << 3) | (i & 7);
    } else {
        ni.code = P.lv[l].K1[0];
        ni.pc = ni.code >> 3;
    }
    ni.real = false;
    ni.child0 = kNone;
    if (l >= 1) {  // one word load serves both the bit test and the rank
        const uint64_t w = ni.code >> 6;
        const uint64_t wd = P.lv[l].bits[w];
        const uint32_t wp = P.lv[l].wpre[w];
        ni.real = (wd >> (ni.code & 63)) & 1ull;
        if (ni.real) ni.child0 = P.lv[l - 1].off + 8u * (wp + (uint32_t)__popcll(wd & ((1ull << (ni.code & 63)) - 1ull)));
    }
    if (l < P.T) {
        const uint32_t pl = (l + 1 < P.T) ? 8u * rank_of(P, l + 2, ni.pc >> 3) + (uint32_t)(ni.pc & 7) : 0u;
        ni.parent = P.lv[l + 1].off + pl;
    } else {
        ni.parent = kNone;
    }
    ni.w = P.lv[l].width;
    const uint32_t x = compact3(ni.code), y = compact3(ni.code >> 1), z = compact3(ni.code >> 2);
    ni.o[0] = Fp<S>::origin(go[0], ni.w, (float)x);
    ni.o[1] = Fp<S>::origin(go[1], ni.w, (float)y);
    ni.o[2] = Fp<S>::origin(go[2], ni.w, (float)z);
}

// Full 27-neighbourhood.  The same-level node at offset d exists iff its
// parent group is a set bit of the next level.  A node with coordinate parity
// s has its neighbours' parents among 8 groups: its own and, per axis, the
// one on the side it borders (-1 where s_i = 0, +1 where s_i = 1).  Those 7
// other groups are ranked once; neighbour d then lies in group b (b_i = 1
// where d crosses into the bordering group) at child (s ^ [d != 0]).
__device__ __forceinline__ void full_neighbors(const EmitParams &P, const NodeInfo &ni, uint32_t self,
                                               uint32_t nb[27]) {
    nb[13] = self;
    if (ni.l >= P.T) return;
    const int l1 = ni.l + 1;
    const uint64_t pc = ni.code >> 3;
    const uint32_t s = (uint32_t)(ni.code & 7);
    const uint64_t sx = spread3(P.lv[l1].side);
    const uint64_t m[3] = {pc & kDilX, pc & kDilY, pc & kDilZ};
    const uint64_t lim[3] = {sx, sx << 1, sx << 2};
    const uint64_t msk[3] = {kDilX, kDilY, kDilZ};
    uint64_t step[3];
    bool ok[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if ((s >> a) & 1) {
            step[a] = dil_inc(m[a], msk[a]);
            ok[a] = step[a] < lim[a] && step[a] != 0;
        } else {
            ok[a] = m[a] != 0;
            step[a] = dil_dec(m[a], msk[a]);
        }
    }
    const uint32_t own = self - (uint32_t)(ni.code & 7);  // child 0 of the node's own group
    // the 7 other groups: codes first, then all word loads (in range even for
    // groups outside the grid, which fall back to the node's own group), then
    // existence and rank from the loaded words
    uint64_t q[8];
    bool in[8];
#pragma unroll
    for (int b = 1; b < 8; ++b) {
        in[b] = !(((b & 1) && !ok[0]) || ((b & 2) && !ok[1]) || ((b & 4) && !ok[2]));
        q[b] = in[b] ? (((b & 1) ? step[0] : m[0]) | ((b & 2) ? step[1] : m[1]) | ((b & 4) ? step[2] : m[2])) : pc;
    }
    uint64_t wd[8];
    uint32_t wp[8];
    const bool top = l1 >= P.T;  // the root level: rank 0
#pragma unroll
    for (int b = 1; b < 8; ++b) {
        wd[b] = P.lv[l1].bits[q[b] >> 6];
        wp[b] = top ? 0u : P.lv[l1].wpre[q[b] >> 6];
    }
    uint32_t base[8];
    base[0] = own;
#pragma unroll
    for (int b = 1; b < 8; ++b) {
        const uint32_t sh = (uint32_t)(q[b] & 63);
        const bool ex = in[b] && ((wd[b] >> sh) & 1ull);
        base[b] = ex ? P.lv[ni.l].off + 8u * (wp[b] + (uint32_t)__popcll(wd[b] & ((1ull << sh) - 1ull))) : kNone;
    }
    // Neighbour d = base[b] | k with, per axis a, (b_a, k_a) = (1, 1), (0, 0),
    // (0, 1) for d_a = -1, 0, +1 when s_a = 0 and (0, 0), (0, 1), (1, 0) when
    // s_a = 1 (every base is a multiple of 8, and kNone | k = kNone): the
    // 3 x 3 x 3 table follows from the 8 bases one axis at a time.
    const uint32_t sxa = s & 1u, sya = (s >> 1) & 1u, sza = (s >> 2) & 1u;
    uint32_t X[3][4];  // [dx + 1][b_y | b_z << 1]
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const uint32_t b0 = base[r << 1], b1 = base[(r << 1) | 1];
        X[0][r] = sxa ? b0 : (b1 | 1u);
        X[1][r] = b0 | sxa;
        X[2][r] = sxa ? b1 : (b0 | 1u);
    }
    uint32_t Y[3][3][2];  // [dx + 1][dy + 1][b_z]
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int z = 0; z < 2; ++z) {
            const uint32_t c0 = X[i][z << 1], c1 = X[i][(z << 1) | 1];
            Y[i][0][z] = sya ? c0 : (c1 | 2u);
            Y[i][1][z] = c0 | (sya << 1);
            Y[i][2][z] = sya ? c1 : (c0 | 2u);
        }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int jy = 0; jy < 3; ++jy) {
            const uint32_t c0 = Y[i][jy][0], c1 = Y[i][jy][1];
            nb[i + 3 * jy] = sza ? c0 : (c1 | 4u);
            nb[i + 3 * jy + 9] = c0 | (sza << 2);
            nb[i + 3 * jy + 18] = sza ? c1 : (c0 | 4u);
        }
}

// Corners (Morton-numbered) joined by edge e, in the reference's edge order
// 02 23 31 10 46 67 75 54 04 26 37 15 (src/SVO.cu:610,638-663).
__host__ __device__ constexpr int edge_corner(int e, int s) {
    return (int)(((s ? 0x576445760132ull : 0x132057641320ull) >> (4 * e)) & 0xFull);
}

// Warp copy of nbytes (multiple of 8) from shared to global memory, in
// 16-byte streaming stores.
__device__ __forceinline__ void warp_copy_out(const uint4 *src, char *dst, uint32_t nbytes, int lane) {
    const uint32_t nv = nbytes / 16;
    uint4 *d4 = reinterpret_cast<uint4 *>(dst);
    for (uint32_t v = lane; v < nv; v += 32) __stcs(d4 + v, src[v]);
    if ((nbytes & 15) && lane == 0) {
        const unsigned long long *s8 = reinterpret_cast<const unsigned long long *>(src);
        __stcs(reinterpret_cast<unsigned long long *>(dst) + nv * 2, s8[nv * 2]);
    }
}

__device__ __forceinline__ bool veq(const float *a, const float *b) {
    return a[0] == b[0] && a[1] == b[1] && a[2] == b[2];
}

constexpr int kEmitWarps = 4;
constexpr int kEmitBufBytes = 32 * 336;  // per warp

// ONE: a single mesh whose parameters travel in the kernel's parameter space
// (`one`, read through the constant cache); otherwise each warp looks up its
// mesh in the batch table (global memory, L1-cached).
template <bool S, bool FULL, bool VE, bool ONE>
// 5 CTAs per SM for the full-neighbour and single-mesh variants (the
// shared-memory staging allows 5; 102 registers hold them without spills);
// the batched parity variant measured faster with the compiler's own choice.
__global__ void __launch_bounds__(kEmitWarps * 32, (FULL || ONE) ? 5 : 1)
    k_emit(EmitBatch eb, const __grid_constant__ EmitParams one, uint64_t total) {
    extern __shared__ uint4 smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint4 *wbuf = smem + warp * (kEmitBufBytes / 16);
    const uint64_t nwarps = (uint64_t)gridDim.x * kEmitWarps;
    for (uint64_t gbase = ((uint64_t)blockIdx.x * kEmitWarps + warp) * 32; gbase < total; gbase += nwarps * 32) {
        const int mj = ONE ? 0 : find_segment(eb.node_off, eb.n, gbase);
        const EmitParams &P = ONE ? one : eb.p[mj];
        const uint64_t base = ONE ? gbase : gbase - eb.node_off[mj];
        if (base >= P.N) continue;  // padding between meshes
        const float go[3] = {P.gp->origin[0], P.gp->origin[1], P.gp->origin[2]};
        unsigned long long vdup = 0, edup = 0;
        const uint32_t t = (uint32_t)(base + lane);
        const bool valid = base + lane < P.N;
        const uint32_t cnt = (uint32_t)(P.N - base < 32 ? P.N - base : 32);
        NodeInfo ni;
        if (valid) node_info<S>(P, go, t, ni);
        uint32_t nb[27];
#pragma unroll
        for (int j = 0; j < 27; ++j) nb[j] = kNone;
        if (valid) {
            if (FULL) {
                full_neighbors(P, ni, t, nb);
            } else if (ni.l == P.T && P.T >= 1) {
                nb[13] = t;  // root self entry, src/SVO.cu:522-529,556-557
            }
        }
        // ---- node records (21 u64 words each) ----
        if (valid) {
            unsigned long long *d = reinterpret_cast<unsigned long long *>(wbuf) + lane * 21;
            const uint32_t leaf = (ni.l == 0 || !ni.real) ? 1u : 0u;
            uint32_t ch[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) ch[k] = ni.real ? ni.child0 + k : kNone;
            auto pk = [](uint32_t lo, uint32_t hi) { return ((unsigned long long)hi << 32) | lo; };
            d[0] = pk((uint32_t)ni.code, leaf);
            d[1] = pk(__float_as_uint(ni.o[0]), __float_as_uint(ni.o[1]));
            d[2] = pk(__float_as_uint(ni.o[2]), __float_as_uint(ni.w));
            d[3] = pk(ni.parent, ch[0]);
            d[4] = pk(ch[1], ch[2]);
            d[5] = pk(ch[3], ch[4]);
            d[6] = pk(ch[5], ch[6]);
            d[7] = pk(ch[7], nb[0]);
#pragma unroll
            for (int k = 0; k < 13; ++k) d[8 + k] = pk(nb[1 + 2 * k], nb[2 + 2 * k]);
        }
        __syncwarp();
        warp_copy_out(wbuf, reinterpret_cast<char *>(P.nodes) + base * 168, cnt * 168, lane);
        __syncwarp();
        if (!VE) continue;
        // ---- vertices: corner i = width * (i&1, i>>1&1, i>>2&1), src/SVO.cu:586-608 ----
        float vp[8][3];
        uint32_t vown[8];
        if (valid) {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                vp[i][0] = __fmul_rn(ni.w, (float)(i & 1));
                vp[i][1] = __fmul_rn(ni.w, (float)((i >> 1) & 1));
                vp[i][2] = __fmul_rn(ni.w, (float)((i >> 2) & 1));
                uint32_t own = t;
                if (FULL) {
                    const int cx = i & 1, cy = (i >> 1) & 1, cz = (i >> 2) & 1;
                    uint32_t best = kNone;
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const int s = (cx - 1 + (q & 1) + 1) + 3 * (cy - 1 + ((q >> 1) & 1) + 1) +
                                      9 * (cz - 1 + ((q >> 2) & 1) + 1);
                        best = min(best, nb[s]);
                    }
                    own = best;
                }
                vown[i] = own;
                wbuf[lane * 8 + (i ^ (lane & 7))] =
                    make_uint4(__float_as_uint(vp[i][0]), __float_as_uint(vp[i][1]),
                               __float_as_uint(vp[i][2]), own);
            }
        }
        __syncwarp();
        {
            const uint32_t nv = cnt * 8;
            uint4 *d4 = reinterpret_cast<uint4 *>(P.verts + base * 8);
            for (uint32_t v = lane; v < nv; v += 32) {
                const uint32_t node = v >> 3, k = v & 7;
                __stcs(d4 + v, wbuf[node * 8 + (k ^ (node & 7))]);
            }
        }
        __syncwarp();
        // ---- edges: 12 per node in the reference's order, src/SVO.cu:629-677 ----
        float cp[8][3];
        float pw = 0.0f;
        float po[3] = {0.0f, 0.0f, 0.0f};
        {
            // previous node's width and origin (for the duplicate checks)
            pw = __shfl_up_sync(0xFFFFFFFFu, valid ? ni.w : 0.0f, 1);
#pragma unroll
            for (int a = 0; a < 3; ++a) po[a] = __shfl_up_sync(0xFFFFFFFFu, valid ? ni.o[a] : 0.0f, 1);
            if (lane == 0 && valid && t > 0) {
                NodeInfo pn;
                node_info<S>(P, go, t - 1, pn);
                pw = pn.w;
                po[0] = pn.o[0];
                po[1] = pn.o[1];
                po[2] = pn.o[2];
            }
        }
        if (valid) {
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                if (c == 0) {
                    cp[0][0] = ni.o[0];
                    cp[0][1] = ni.o[1];
                    cp[0][2] = ni.o[2];
                } else {
                    cp[c][0] = __fadd_rn(ni.o[0], (c & 1) ? ni.w : 0.0f);
                    cp[c][1] = __fadd_rn(ni.o[1], (c & 2) ? ni.w : 0.0f);
                    cp[c][2] = __fadd_rn(ni.o[2], (c & 4) ? ni.w : 0.0f);
                }
            }
            uint32_t eown[12];
#pragma unroll
            for (int e = 0; e < 12; ++e) {
                uint32_t own = t;
                if (FULL) {
                    const int a = edge_corner(e, 0), b = edge_corner(e, 1);
                    uint32_t best = kNone;
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        int d[3], qq = 0;
#pragma unroll
                        for (int ax = 0; ax < 3; ++ax) {
                            const int ca = (a >> ax) & 1, cb = (b >> ax) & 1;
                            if (ca != cb) {
                                d[ax] = 0;
                            } else {
                                d[ax] = ca - 1 + ((q >> qq) & 1);
                                ++qq;
                            }
                        }
                        best = min(best, nb[(d[0] + 1) + 3 * (d[1] + 1) + 9 * (d[2] + 1)]);
                    }
                    own = best;
                }
                eown[e] = own;
            }
            // 84 words per node: edge e = p0 (3), p1 (3), owner
            uint4 *d = wbuf + lane * 21;
#pragma unroll
            for (int j = 0; j < 21; ++j) {
                uint32_t wv[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int wi = 4 * j + q, e = wi / 7, f = wi % 7;
                    wv[q] = f < 3   ? __float_as_uint(cp[edge_corner(e, 0)][f])
                            : f < 6 ? __float_as_uint(cp[edge_corner(e, 1)][f - 3])
                                    : eown[e];
                }
                d[j] = make_uint4(wv[0], wv[1], wv[2], wv[3]);
            }
            // consecutive duplicates (thrust::unique, src/SVO.cu:679-725)
#pragma unroll
            for (int i = 1; i < 8; ++i) vdup += veq(vp[i], vp[i - 1]);
            if (t > 0) {
                const float pv7[3] = {__fmul_rn(pw, 1.0f), __fmul_rn(pw, 1.0f), __fmul_rn(pw, 1.0f)};
                vdup += veq(vp[0], pv7);
            }
#pragma unroll
            for (int e = 1; e < 12; ++e) {
                const float *a0 = cp[edge_corner(e - 1, 0)], *a1 = cp[edge_corner(e - 1, 1)];
                const float *b0 = cp[edge_corner(e, 0)], *b1 = cp[edge_corner(e, 1)];
                edup += (veq(a0, b0) && veq(a1, b1)) || (veq(a0, b1) && veq(a1, b0));
            }
            if (t > 0) {
                // previous node's edge 11 = (corner 1, corner 5)
                const float q1[3] = {__fadd_rn(po[0], pw), __fadd_rn(po[1], 0.0f), __fadd_rn(po[2], 0.0f)};
                const float q5[3] = {__fadd_rn(po[0], pw), __fadd_rn(po[1], 0.0f), __fadd_rn(po[2], pw)};
                const float *b0 = cp[0], *b1 = cp[2];
                edup += (veq(q1, b0) && veq(q5, b1)) || (veq(q1, b1) && veq(q5, b0));
            }
        }
        __syncwarp();
        warp_copy_out(wbuf, reinterpret_cast<char *>(P.edges) + base * 336, cnt * 336, lane);
        __syncwarp();
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
            vdup += __shfl_xor_sync(0xFFFFFFFFu, vdup, d);
            edup += __shfl_xor_sync(0xFFFFFFFFu, edup, d);
        }
        if (lane == 0 && vdup) atomicAdd(P.dups, vdup);
        if (lane == 0 && edup) atomicAdd(P.dups + 1, edup);
    }
}

// ---------------------------------------------------------------------------
// Stable removal of consecutive duplicates (rare path).
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool same(const svo_vertex &a, const svo_vertex &b) { return veq(a.pos, b.pos); }
__device__ __forceinline__ bool same(const svo_edge &a, const svo_edge &b) {
    return (veq(a.p0, b.p0) && veq(a.p1, b.p1)) || (veq(a.p0, b.p1) && veq(a.p1, b.p0));
}

template <class T>
__global__ void __launch_bounds__(256) k_unique_count(const T *__restrict__ in, uint64_t n,
                                                      uint32_t *__restrict__ tile_counts) {
    __shared__ uint32_t s[8];
    const uint64_t t0 = (uint64_t)blockIdx.x * kUniqueTile;
    uint32_t c = 0;
    for (uint32_t k = threadIdx.x; k < kUniqueTile; k += blockDim.x) {
        const uint64_t i = t0 + k;
        if (i < n) c += (i == 0 || !same(in[i - 1], in[i]));
    }
    c = __reduce_add_sync(0xFFFFFFFFu, c);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t tot = 0;
        for (int w = 0; w < 8; ++w) tot += s[w];
        tile_counts[blockIdx.x] = tot;
    }
}

template <class T>
__global__ void __launch_bounds__(256) k_unique_scatter(const T *__restrict__ in, uint64_t n,
                                                        const uint32_t *__restrict__ tile_pre,
                                                        T *__restrict__ out) {
    __shared__ uint32_t s_w[8];
    const uint64_t t0 = (uint64_t)blockIdx.x * kUniqueTile;
    uint32_t run = tile_pre[blockIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t k0 = 0; k0 < kUniqueTile; k0 += blockDim.x) {
        const uint64_t i = t0 + k0 + threadIdx.x;
        const bool keep = i < n && (i == 0 || !same(in[i - 1], in[i]));
        const uint32_t m = __ballot_sync(0xFFFFFFFFu, keep);
        if (lane == 0) s_w[warp] = __popc(m);
        __syncthreads();
        uint32_t before = 0, tot = 0;
        for (int w = 0; w < 8; ++w) {
            if (w < warp) before += s_w[w];
            tot += s_w[w];
        }
        if (keep) out[run + before + __popc(m & ((1u << lane) - 1u))] = in[i];
        run += tot;
        __syncthreads();
    }
}

template <class T>
cudaError_t unique_impl(const T *in, uint64_t n, T *out, uint32_t *tile_counts, uint32_t *tile_pre,
                        unsigned long long *scan_scratch, uint32_t *status, cudaStream_t st) {
    const uint64_t tiles = (n + kUniqueTile - 1) / kUniqueTile;
    if (tiles == 0) return cudaSuccess;
    k_unique_count<T><<<(unsigned)tiles, 256, 0, st>>>(in, n, tile_counts);
    count_launches(1);
    cudaError_t e = launch_scan(tile_counts, tile_pre, tiles, scan_scratch, status, st);
    if (e != cudaSuccess) return e;
    k_unique_scatter<T><<<(unsigned)tiles, 256, 0, st>>>(in, n, tile_pre, out);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_pyramid(const BatchDev &b, uint32_t total_ctas, int num_sms, cudaStream_t st) {
    if (total_ctas == 0) return cudaSuccess;
    k_pyramid<<<std::min<uint32_t>(total_ctas, (uint32_t)num_sms * 8), 256, 0, st>>>(b, total_ctas);
    k_pyramid_top<<<b.n, 256, 0, st>>>(b);
    count_launches(2);
    return cudaGetLastError();
}

size_t scan_scratch_words(uint64_t n) { return 1 + (n + kScanTile - 1) / kScanTile; }

cudaError_t launch_scan(const uint32_t *in, uint32_t *out, uint64_t n, unsigned long long *scratch,
                        uint32_t *status, cudaStream_t st) {
    const uint64_t tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles >= kScanSplitTiles && tiles <= 0x7FFFFFFFull &&
        ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15) == 0) {
        // tile sums and their prefixes live in the look-back scratch (tiles + 1 u64 words)
        uint32_t *tsum = reinterpret_cast<uint32_t *>(scratch), *tpre = tsum + tiles;
        k_scan_reduce<<<(unsigned)tiles, kScanThreads, 0, st>>>(in, n, tsum);
        k_scan_tiles<<<1, 1024, 0, st>>>(tsum, tpre, tiles, out + n);
        k_scan_down<<<(unsigned)tiles, kScanThreads, 0, st>>>(in, out, n, tpre);
        count_launches(3);
        return cudaGetLastError();
    }
    cudaError_t e = cudaMemsetAsync(scratch, 0, scan_scratch_words(n) * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    if (tiles == 0) return cudaMemsetAsync(out, 0, sizeof(uint32_t), st);
    k_scan<<<(unsigned)tiles, kScanThreads, 0, st>>>(in, out, n, scratch, status, kSpinLimit);
    count_launches(1);
    return cudaGetLastError();
}

size_t scan_stalled_scratch_words(uint64_t n) { return scan_scratch_words(n) + 1; }

cudaError_t launch_scan_stalled(const uint32_t *in, uint32_t *out, uint64_t n, unsigned long long *scratch,
                                uint32_t *status, int spin_limit, cudaStream_t st) {
    const uint64_t tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles < 2 || tiles > 0x7FFFFFFFull || spin_limit < 1) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(scratch, 0, scan_stalled_scratch_words(n) * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    // the tile counter starts at 1: tile 0 is never run and never publishes
    const unsigned long long one = 1;
    if ((e = cudaMemcpyAsync(scratch, &one, sizeof(one), cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    k_scan<<<(unsigned)tiles, kScanThreads, 0, st>>>(in, out, n, scratch, status, spin_limit);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_level_totals(const BatchDev &b, cudaStream_t st) {
    const int n = b.n * kMaxLevels;
    k_level_totals<<<(n + 127) / 128, 128, 0, st>>>(b);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_compact(const CompactBatch &c, uint64_t total_words, cudaStream_t st) {
    if (total_words == 0) return cudaSuccess;
    k_compact<<<(unsigned)((total_words + 255) / 256), 256, 0, st>>>(c, total_words);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_compact_regions(const CompactJob &job, uint32_t regions, int num_sms, cudaStream_t st) {
    if (regions == 0) return cudaSuccess;
    k_compact_regions<<<std::min<uint32_t>(regions, (uint32_t)num_sms * 8), 256, 0, st>>>(job, regions);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_compact_keys(const KeyBatch &k, uint64_t total_blocks, cudaStream_t st) {
    if (total_blocks == 0) return cudaSuccess;
    k_compact_keys<<<(unsigned)((total_blocks * 8 + 255) / 256), 256, 0, st>>>(k, total_blocks);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_emit(const EmitBatch &b, const EmitParams *one, uint64_t total, uint32_t flags, int num_sms,
                        cudaStream_t st) {
    if (total == 0) return cudaSuccess;
    const uint64_t warps = (total + 31) / 32;
    const unsigned blocks = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>((warps + kEmitWarps - 1) / kEmitWarps, 0x7FFFFFFFull));
    const size_t shmem = (size_t)kEmitWarps * kEmitBufBytes;
    const bool s = (flags & SVO_FLAG_STRICT_FP) != 0, f = (flags & SVO_FLAG_FULL_NEIGHBORS) != 0,
               ve = (flags & SVO_FLAG_NO_VERT_EDGE) == 0;
    const EmitParams p1 = one ? *one : EmitParams{};
#define SVO_EMIT1(S_, F_, V_)                                                                       \
    do {                                                                                             \
        if (one) k_emit<S_, F_, V_, true><<<blocks, kEmitWarps * 32, shmem, st>>>(b, p1, total);      \
        else k_emit<S_, F_, V_, false><<<blocks, kEmitWarps * 32, shmem, st>>>(b, p1, total);        \
    } while (0)
#define SVO_EMIT(S_, F_, V_) SVO_EMIT1(S_, F_, V_)
    if (s) {
        if (f) { if (ve) SVO_EMIT(true, true, true); else SVO_EMIT(true, true, false); }
        else { if (ve) SVO_EMIT(true, false, true); else SVO_EMIT(true, false, false); }
    } else {
        if (f) { if (ve) SVO_EMIT(false, true, true); else SVO_EMIT(false, true, false); }
        else { if (ve) SVO_EMIT(false, false, true); else SVO_EMIT(false, false, false); }
    }
#undef SVO_EMIT1
#undef SVO_EMIT
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_unique_vertices(const svo_vertex *in, uint64_t n, svo_vertex *out, uint32_t *tile_counts,
                                   uint32_t *tile_pre, unsigned long long *scan_scratch, uint32_t *status,
                                   cudaStream_t st) {
    return unique_impl(in, n, out, tile_counts, tile_pre, scan_scratch, status, st);
}

cudaError_t launch_unique_edges(const svo_edge *in, uint64_t n, svo_edge *out, uint32_t *tile_counts,
                                uint32_t *tile_pre, unsigned long long *scan_scratch, uint32_t *status,
                                cudaStream_t st) {
    return unique_impl(in, n, out, tile_counts, tile_pre, scan_scratch, status, st);
}

}  // namespace svo
