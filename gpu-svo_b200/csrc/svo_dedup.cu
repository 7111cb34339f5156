// svo_dedup.cu -- Morton-keyed unique vertices, edges and faces of the octree.
//
// Keys live on the finest lattice (voxel corners, coordinates 0..R):
//   vertex key = morton(P)
//   edge key   = morton(P) << 6 | level << 2 | axis     (P = the edge's low end)
//   face key   = morton(P) << 6 | level << 2 | normal   (P = the face's low corner)
// over every node of every level (sibling-filled nodes included), each list
// sorted and unique.  The reference has no such lists (its README promises
// them); the semantics are this library's and the oracle restates them.
//
// No sort is needed.  Every key names a lattice point P that is a node
// corner, and a key of P exists iff some node touching P exists at that
// level: at level l (P a multiple of 2^l, u = P >> l) the cells u - d,
// d in {0,1}^3, and a cell exists iff its parent is set in the level l+1
// occupancy bitmap (at the top level: iff it is the root).  So:
//   1. build a candidate bitmap D over Q = P >> 1 (each bit stands for the 8
//      lattice points 2Q + r): the corners of the nodes of levels >= 1 --
//      every level-0 corner is also a corner of a level-1 node.  The
//      level-1 corners come word by word from the level-2 bitmap
//      (k_dedup_build), the coarser levels' by marking their node groups;
//   2. walk D's words in order and derive, per Q, what its 8 points need
//      from the parent bitmaps (coarser levels only for r = 0), for the 64 Q
//      of a word at once by shifts of whole bitmap words; pack it into one
//      64-bit state per Q (layout at kQcMask) and count keys per tile of 32
//      states;
//   3. scan the counts and expand the states into keys: the keys come out in
//      Morton order because D is in Morton order and each point's keys are
//      produced in (level, axis) order.  Each warp stages 16-bit key
//      entries in shared memory and stores the keys coalesced.
// D has R^3 bits (1 GiB at R = 2048); a 1-bit-per-chunk summary lets the walk
// skip untouched chunks without reading them.
#include <cstdio>
#include <cstring>

#include "svo_host.h"
#include "svo_internal.h"

namespace svo {
namespace {

constexpr int kDedupWarps = 8;
constexpr uint64_t kChunkWords = 32;  // u64 words of D per chunk (2048 bits)
constexpr uint32_t kStageKeys = 2048;  // key entries of one kind a warp stages in shared memory

struct DedupLevel {
    const uint64_t *bits;  // occupancy bitmap of this level
    const uint64_t *K1;    // sorted codes of level l+1 (this level's sibling groups)
    uint32_t groups;       // number of those codes
    uint32_t side;         // grid side at this level
};

struct DedupParams {
    int T;                      // top level
    const uint64_t *root;       // device: the root's code
    DedupLevel lv[kMaxLevels];
    uint32_t gstart[kMaxLevels + 1];  // marking threads of levels 1..T-1 (prefix of groups)
    uint32_t *D;                // candidate bitmap over Q (u32 view)
    uint32_t *G;                // one bit per chunk of D
    uint64_t chunks;
    const uint32_t *list;       // the touched chunks (a set bit in G), in order
    uint64_t ntouched;
    unsigned long long *nq;     // set bits of D (counted while marking)
    uint32_t *qn;               // [ntouched] set bits per touched chunk
    const uint32_t *qpre;       // [ntouched + 1] their prefix: the first state of each chunk
    uint64_t *qs;               // one state per set bit of D, in order
    uint64_t ntiles;            // tiles of 32 consecutive states
    uint32_t *tcnt;             // [3][ntiles] keys per tile and kind
    const uint32_t *tpre;       // [3][ntiles + 1] their prefixes
    uint64_t *out[3];
    const struct DedupTables *tables;  // built once per dedup by k_dedup_tables
};

// Adds the block's sum of v (each thread's share) to *dst with one atomic.
// All threads of the block call.
__device__ __forceinline__ void block_add(unsigned long long *dst, uint32_t v) {
    __shared__ uint32_t part[32];
    v = __reduce_add_sync(0xFFFFFFFFu, v);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint32_t s = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0u;
        s = __reduce_add_sync(0xFFFFFFFFu, s);
        if (threadIdx.x == 0 && s) atomicAdd(dst, (unsigned long long)s);
    }
}

__device__ __forceinline__ void mark_chunk(const DedupParams &p, uint64_t bit) {
    const uint64_t ch = bit >> 11;
    uint32_t *g = p.G + (ch >> 5);
    const uint32_t m = 1u << (ch & 31);
    if (!(*(volatile uint32_t *)g & m)) atomicOr(g, m);
}

// Returns 1 when the bit was not set before.
__device__ __forceinline__ uint32_t mark_bit(const DedupParams &p, uint64_t bit) {
    const uint32_t m = 1u << (bit & 31);
    const uint32_t old = atomicOr(p.D + (bit >> 5), m);
    mark_chunk(p, bit);
    return (old & m) ? 0u : 1u;
}

// Marks the Q of every corner of every node at levels >= 1.
//   level 1, group g (a level-2 code): nodes 2g + {0,1}^3, corners
//     Q = 2g + {0,1,2}^3, i.e. for each e in {0,1}^3 the byte morton(g + e)
//     of D gets the sub-points k' with k'_i = 0 wherever e_i = 1;
//   level l >= 2: Q = (2g + {0,1,2}^3) << (l - 1), one bit each;
//   the root (level T): Q = (root + {0,1}^3) << (T - 1).
//   Also counts the bits it sets first (*p.nq: the set bits of D).  Threads
//   from `first` on (first = gstart[2] when k_dedup_build did level 1).
__global__ void k_dedup_mark(const __grid_constant__ DedupParams p, uint32_t first, uint32_t total) {
    uint32_t fresh = 0;
    for (uint32_t t = first + blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        if (t == total - 1) {
            const uint64_t rc = *p.root;
            const uint32_t r[3] = {compact3(rc), compact3(rc >> 1), compact3(rc >> 2)};
            const int sh = p.T - 1;
            for (int d = 0; d < 8; ++d)
                fresh += mark_bit(p, morton3((r[0] + (d & 1)) << sh, (r[1] + ((d >> 1) & 1)) << sh,
                                             (r[2] + ((d >> 2) & 1)) << sh));
            continue;
        }
        int l = 1;
        while (l + 1 < p.T && t >= p.gstart[l + 1]) ++l;
        const uint64_t gc = p.lv[l].K1[t - p.gstart[l]];
        const uint32_t g[3] = {compact3(gc), compact3(gc >> 1), compact3(gc >> 2)};
        if (l == 1) {
            for (int e = 0; e < 8; ++e) {
                const uint64_t byte = morton3(g[0] + (e & 1), g[1] + ((e >> 1) & 1), g[2] + ((e >> 2) & 1));
                uint32_t m = 0xFFu;
                if (e & 1) m &= 0x55u;
                if (e & 2) m &= 0x33u;
                if (e & 4) m &= 0x0Fu;
                m <<= 8 * (byte & 3);
                fresh += __popc(m & ~atomicOr(p.D + (byte >> 2), m));
                mark_chunk(p, byte << 3);
            }
        } else {
            const int sh = l - 1;
            for (int k = 0; k < 27; ++k) {
                const uint32_t kx = k % 3, ky = (k / 3) % 3, kz = k / 9;
                fresh += mark_bit(p, morton3((2 * g[0] + kx) << sh, (2 * g[1] + ky) << sh, (2 * g[2] + kz) << sh));
            }
        }
    }
    block_add(p.nq, fresh);
}

// Bit e of the result: cell v - e exists at the level whose occupancy bitmap
// is `bits` and whose side, dilated, is sx (x position).  v is given by its
// Morton code vc (dilated coordinates, stepped in place); its coordinates are
// at most the level's side.
__device__ __forceinline__ uint32_t cell_mask(const uint64_t *bits, uint64_t vc, uint64_t sx) {
    const uint64_t xm = vc & kDilX, ym = vc & kDilY, zm = vc & kDilZ;
    const uint64_t xd = dil_dec(xm, kDilX), yd = dil_dec(ym, kDilY), zd = dil_dec(zm, kDilZ);
    const bool vx0 = xm < sx, vy0 = ym < (sx << 1), vz0 = zm < (sx << 2);
    const bool vx1 = xm != 0, vy1 = ym != 0, vz1 = zm != 0;
    uint32_t m = 0;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const bool ok = ((e & 1) ? vx1 : vx0) && ((e & 2) ? vy1 : vy0) && ((e & 4) ? vz1 : vz0);
        if (!ok) continue;
        const uint64_t c = ((e & 1) ? xd : xm) | ((e & 2) ? yd : ym) | ((e & 4) ? zd : zm);
        m |= (uint32_t)((bits[c >> 6] >> (c & 63)) & 1ull) << e;
    }
    return m;
}

// Bit e of cell_mask(bits, vc, sx) alone.
__device__ __forceinline__ uint32_t cell_bit(const uint64_t *bits, uint64_t vc, uint64_t sx, int e) {
    const uint64_t xm = vc & kDilX, ym = vc & kDilY, zm = vc & kDilZ;
    const bool ok = ((e & 1) ? xm != 0 : xm < sx) && ((e & 2) ? ym != 0 : ym < (sx << 1)) &&
                    ((e & 4) ? zm != 0 : zm < (sx << 2));
    if (!ok) return 0;
    const uint64_t c = ((e & 1) ? dil_dec(xm, kDilX) : xm) | ((e & 2) ? dil_dec(ym, kDilY) : ym) |
                       ((e & 4) ? dil_dec(zm, kDilZ) : zm);
    return (uint32_t)(bits[c >> 6] >> (c & 63)) & 1u;
}

// Shared tables.
//   around[E * 8 + s]: existence of the 8 cells u - d around a point of
//     parity s (bit d), given the parent mask E: cell u - d has parent
//     v - (d & ~s)
//   kinds[ex]: bit 0 vertex, bits 1-3 edges along x/y/z, bits 4-6 faces
//     with normal x/y/z, from the cell existence mask ex
//   cnt0[E]: keys of the 8 points 2Q + r at level 0 given E, packed
//     (vertices | edges << 8 | faces << 16)
//   v0/e0/f0[E]: the level-0 slots of those keys as the write pass orders
//     them (QMasks below): v0 bit r; e0/f0 bits axis (r = 0) and
//     9 + 3(r - 1) + axis (r = 1..7)
struct alignas(16) DedupTables {
    uint8_t around[2048];
    uint8_t kinds[256];
    uint32_t cnt0[256];
    uint8_t v0[256];
    uint32_t e0[256], f0[256];
};

__device__ void init_tables(DedupTables &t) {
    for (int i = threadIdx.x; i < 2048; i += blockDim.x) {
        const uint32_t E = i >> 3, s = i & 7;
        uint32_t ex = 0;
        for (int d = 0; d < 8; ++d) ex |= ((E >> (d & ~s & 7)) & 1u) << d;
        t.around[i] = (uint8_t)ex;
    }
    for (int ex = threadIdx.x; ex < 256; ex += blockDim.x) {
        uint32_t k = ex != 0;
        k |= (uint32_t)((ex & 0x55) != 0) << 1 | (uint32_t)((ex & 0x33) != 0) << 2 | (uint32_t)((ex & 0x0F) != 0) << 3;
        k |= (uint32_t)((ex & 0x03) != 0) << 4 | (uint32_t)((ex & 0x05) != 0) << 5 | (uint32_t)((ex & 0x11) != 0) << 6;
        t.kinds[ex] = (uint8_t)k;
    }
    __syncthreads();
    for (int E = threadIdx.x; E < 256; E += blockDim.x) {
        uint32_t v = 0, e = 0, f = 0;
        for (int r = 0; r < 8; ++r) {
            const uint32_t k = t.kinds[t.around[E * 8 + r]];
            v += k & 1;
            e += __popc((k >> 1) & 7);
            f += __popc((k >> 4) & 7);
        }
        t.cnt0[E] = v | e << 8 | f << 16;
        uint32_t vm = 0, em = 0, fm = 0;
        for (int r = 0; r < 8; ++r) {
            const uint32_t k = t.kinds[t.around[E * 8 + r]];
            const int at = r == 0 ? 0 : 9 + 3 * (r - 1);
            vm |= (k & 1u) << r;
            em |= ((k >> 1) & 7u) << at;
            fm |= ((k >> 4) & 7u) << at;
        }
        t.v0[E] = (uint8_t)vm;
        t.e0[E] = em;
        t.f0[E] = fm;
    }
    __syncthreads();
}

// The tables of one dedup, built by one block into global memory; the state
// and write passes copy them into shared memory.
__global__ void __launch_bounds__(256) k_dedup_tables(DedupTables *t) { init_tables(*t); }

__device__ __forceinline__ void load_tables(DedupTables &sh, const DedupTables *g) {
    const uint4 *src = reinterpret_cast<const uint4 *>(g);
    uint4 *dst = reinterpret_cast<uint4 *>(&sh);
    for (int i = threadIdx.x; i < (int)(sizeof(DedupTables) / 16); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
}

// Cell existence around P = 2Q at level l >= 1 (u = P >> l has Morton code
// uc): from the level l+1 bitmap, or at the top level, which holds the root
// alone, cell u - d exists iff d = u - root.
__device__ __forceinline__ uint32_t coarse_ex(const DedupParams &p, const DedupTables &tb, const uint64_t *sx,
                                              uint64_t root, int l, uint64_t uc) {
    if (l < p.T) return tb.around[cell_mask(p.lv[l + 1].bits, uc >> 3, sx[l + 1]) * 8 + (uint32_t)(uc & 7)];
    const int dx = (int)compact3(uc) - (int)compact3(root);
    const int dy = (int)compact3(uc >> 1) - (int)compact3(root >> 1);
    const int dz = (int)compact3(uc >> 2) - (int)compact3(root >> 2);
    return (dx >= 0 && dx <= 1 && dy >= 0 && dy <= 1 && dz >= 0 && dz <= 1) ? 1u << (dx | dy << 1 | dz << 2) : 0u;
}

// What one Q needs for all its keys, packed into 64 bits:
//   bits 0-35  qc, the Morton code of Q
//   bits 36-43 E0, the level-1 parent mask around Q (the 8 points 2Q + r at
//              level 0 follow from it through the tables)
//   bits 44-50 key kinds of the point 2Q at level 1
//   bits 51-57 key kinds of the point 2Q at level 2 (Q a multiple of 8 in
//              Morton code, i.e. even in every coordinate)
//   bit  58    levels >= 3 apply as well (Q a multiple of 64); they are
//              derived where needed, from the coarser bitmaps
constexpr uint64_t kQcMask = (1ull << 36) - 1;

// Key kinds of the point 2Q at levels >= 3 (state bit 58): vertex flag into
// v, edges/faces of level l at bits 3(l - 3)..3(l - 3) + 2 of eh/fh.
__device__ __forceinline__ void q_deep(const DedupParams &p, const DedupTables &tb, const uint64_t *sx,
                                       uint64_t root, uint64_t qc, uint32_t &v, uint32_t &eh, uint32_t &fh) {
    uint64_t uc = qc >> 6;
    for (int l = 3; l <= p.T; ++l) {
        if (l > 3) {
            if (uc & 7) break;
            uc >>= 3;
        }
        const uint32_t k = tb.kinds[coarse_ex(p, tb, sx, root, l, uc)];
        v |= k & 1;
        eh |= ((k >> 1) & 7) << (3 * (l - 3));
        fh |= ((k >> 4) & 7) << (3 * (l - 3));
    }
}

// The keys of one Q as slot masks, each kind in output order:
//   v: bit r = vertex of the point 2Q + r (r = 0 at any level);
//   el/fl: bits 3l + axis for the point 2Q at levels 0..2, then bits
//          9 + 3(r - 1) + axis for the points r = 1..7 at level 0;
//   eh/fh: the point 2Q at levels 3..T (bit 3(l - 3) + axis), which come
//          between bits 8 and 9 of el/fl in the output.
struct QMasks {
    uint32_t v, el, fl, eh, fh;
};

__device__ __forceinline__ QMasks q_masks(const DedupParams &p, const DedupTables &tb, const uint64_t *sx,
                                          uint64_t root, uint64_t s) {
    const uint32_t E0 = (uint32_t)(s >> 36) & 0xFFu, k1 = (uint32_t)(s >> 44) & 0x7Fu, k2 = (uint32_t)(s >> 51) & 0x7Fu;
    QMasks m;
    m.v = tb.v0[E0] | ((k1 | k2) & 1u);
    m.el = tb.e0[E0] | ((k1 >> 1) & 7) << 3 | ((k2 >> 1) & 7) << 6;
    m.fl = tb.f0[E0] | ((k1 >> 4) & 7) << 3 | ((k2 >> 4) & 7) << 6;
    m.eh = m.fh = 0;
    if ((s >> 58) & 1) q_deep(p, tb, sx, root, s & kQcMask, m.v, m.eh, m.fh);
    return m;
}

// ---------------------------------------------------------------------------
// The state pass works on whole words of D.  A word holds the 64 Q of an
// aligned 4 x 4 x 4 block b (its index is b's Morton code), and the bitmaps'
// words are such blocks too, so what the Qs of a word need comes from a few
// bitmap words by shifts, for all 64 at once:
//   M_e (e in {0,1}^3): bit i = the level-1 cell Q_i - e is occupied
//       (the level-0 parents around the points 2Q + r: E0 of every Q);
//   X_d: bit i = the level-1 cell Q_i - d exists, i.e. its level-2 parent
//       (Q_i - d) >> 1 is occupied (the cells around the point Q at level 1).
// Bit i of a block is its cell with x = i & 1 | (i >> 2) & 2, y = (i >> 1) &
// 1 | (i >> 3) & 2, z = (i >> 2) & 1 | (i >> 4) & 2.
// ---------------------------------------------------------------------------

// The bits of a block whose coordinate along axis a equals v.
__host__ __device__ constexpr uint64_t block_plane(int a, int v) {
    uint64_t m = 0;
    for (int i = 0; i < 64; ++i)
        if ((((i >> a) & 1) | (((i >> (a + 3)) & 1) << 1)) == v) m |= 1ull << i;
    return m;
}

// A block's field moved one cell up along axis A: bit i of the result is the
// field at cell(i) - e_A, taken from `cur` (the block) or, for coordinate 0,
// from `low` (the block below along A).
template <int A>
__device__ __forceinline__ uint64_t shift_up(uint64_t cur, uint64_t low) {
    constexpr int s0 = 1 << A, s1 = 8 << A;
    constexpr uint64_t P0 = block_plane(A, 0), P13 = block_plane(A, 1) | block_plane(A, 3), P2 = block_plane(A, 2);
    return ((cur << s0) & P13) | ((cur << (s1 - s0)) & P2) | ((low >> (s0 + s1)) & P0);
}

// A 2 x 2 x 2 block of level-2 cells (bit m = Morton code m) seen from the
// 4 x 4 x 4 level-1 cells below it: bit i of the result is bit i >> 3.
__device__ __forceinline__ uint64_t upsample8(uint64_t b) {
    b = (b | (b << 28)) & 0x0000000F0000000Full;
    b = (b | (b << 14)) & 0x0003000300030003ull;
    b = (b | (b << 7)) & 0x0101010101010101ull;
    return b * 0xFFull;
}

// Valid cells of a block at a level of side s (only s < 4 leaves some out).
__device__ __forceinline__ uint64_t block_valid(uint32_t s) {
    return s >= 4 ? ~0ull : s == 2 ? 0xFFull : 0x1ull;
}

// The 8 fields M_e = "cell Q - e" of a block from the blocks b - d
// (A[d], d in {0,1}^3): 12 shifts, separable per axis.  dst[e] gets M_e.
__device__ __forceinline__ void block_offsets(const uint64_t (&A)[8], uint64_t *dst, int stride) {
    const uint64_t Fx[4] = {shift_up<0>(A[0], A[1]), shift_up<0>(A[2], A[3]), shift_up<0>(A[4], A[5]),
                            shift_up<0>(A[6], A[7])};
#pragma unroll
    for (int ex = 0; ex < 2; ++ex) {
        const uint64_t B0 = ex ? Fx[0] : A[0], B2 = ex ? Fx[1] : A[2], B4 = ex ? Fx[2] : A[4], B6 = ex ? Fx[3] : A[6];
        const uint64_t Fy0 = shift_up<1>(B0, B2), Fy4 = shift_up<1>(B4, B6);
#pragma unroll
        for (int ey = 0; ey < 2; ++ey) {
            const uint64_t C0 = ey ? Fy0 : B0, C4 = ey ? Fy4 : B4;
            dst[(ex | ey << 1) * stride] = C0;
            dst[(ex | ey << 1 | 4) * stride] = shift_up<2>(C0, C4);
        }
    }
}

// One warp per touched chunk of D (32 words), in two phases.
//  1. Lane w takes word w (the 64 Q of block b): it fetches the level-1
//     words of the blocks b - d and the level-2 bytes above them (upsampled
//     to level-1 cells), shifts them into M_e = "level-1 cell Q - e occupied"
//     (E0's bits) and X_d = "level-1 cell Q - d exists" (its level-2 parent
//     is occupied: the cells around the point Q at level 1), and stores the
//     16 masks in shared memory; with them the level-3 cell mask of b (the
//     cells around the level-2 points of its even Q) and the deeper levels of
//     its Q_0 (q_deep).
//  2. The chunk's set bits are listed in order and taken 32 at a time: lane
//     j reads its Q's 16 mask bits, stores the Q's state at its rank (the
//     chunk's first state + j) and counts its keys, summed per tile of 32
//     states (a round of 32 ranks spans at most two tiles).
constexpr int kStateWarps = 4;

__global__ void __launch_bounds__(kStateWarps * 32) k_dedup_state(const __grid_constant__ DedupParams p) {
    __shared__ DedupTables tb;
    __shared__ uint64_t masks[kStateWarps][16][kChunkWords];  // [mask][word]: M_0..7, X_0..7
    __shared__ uint16_t list[kStateWarps][2048];
    __shared__ uint32_t wdeep[kStateWarps][kChunkWords];  // E2 | deep key counts of Q_0 (packed as below)
    __shared__ uint64_t sx[kMaxLevels];  // dilated side of each level
    if (threadIdx.x < kMaxLevels) sx[threadIdx.x] = (int)threadIdx.x <= p.T ? spread3(p.lv[threadIdx.x].side) : 0;
    load_tables(tb, p.tables);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t nwarps = (uint64_t)gridDim.x * kStateWarps;
    const uint64_t root = *p.root;
    const uint64_t *D64 = reinterpret_cast<const uint64_t *>(p.D);
    const int T = p.T;
    const uint32_t s1 = p.lv[1].side, s2 = T >= 2 ? p.lv[2].side : 1u;
    const uint64_t nb1 = spread3((s1 + 3) / 4), nb2 = spread3((s2 + 1) / 2);  // blocks per axis, dilated
    const uint64_t valid1 = block_valid(s1), valid2 = s2 >= 2 ? 0xFFull : 0x1ull;
    uint64_t(*mk)[kChunkWords] = masks[warp];
    const uint32_t *mk32 = reinterpret_cast<const uint32_t *>(masks[warp]);
    uint16_t *lst = list[warp];
    uint32_t *wd = wdeep[warp];
    for (uint64_t ci = (uint64_t)blockIdx.x * kStateWarps + warp; ci < p.ntouched; ci += nwarps) {
        const uint64_t ch = p.list[ci];
        const uint64_t bc = ch * kChunkWords + lane;  // this lane's block
        const uint64_t W = D64[bc];
        if (W) {
            const uint64_t xm = bc & kDilX, ym = bc & kDilY, zm = bc & kDilZ;
            const uint64_t xd = dil_dec(xm, kDilX), yd = dil_dec(ym, kDilY), zd = dil_dec(zm, kDilZ);
            uint64_t A[8], U[8];
#pragma unroll
            for (int d = 0; d < 8; ++d) {
                const bool low = (!(d & 1) || xm != 0) && (!(d & 2) || ym != 0) && (!(d & 4) || zm != 0);
                const uint64_t nc = ((d & 1) ? xd : xm) | ((d & 2) ? yd : ym) | ((d & 4) ? zd : zm);
                const uint64_t ncx = nc & kDilX, ncy = nc & kDilY, ncz = nc & kDilZ;
                const bool in1 = low && ncx < nb1 && ncy < (nb1 << 1) && ncz < (nb1 << 2);
                const bool in2 = low && T >= 2 && ncx < nb2 && ncy < (nb2 << 1) && ncz < (nb2 << 2);
                A[d] = in1 ? p.lv[1].bits[nc] & valid1 : 0ull;
                U[d] = in2 ? upsample8((p.lv[2].bits[nc >> 3] >> (8 * (nc & 7))) & valid2) : 0ull;
            }
            block_offsets(A, &mk[0][lane], kChunkWords);
            block_offsets(U, &mk[8][lane], kChunkWords);
            uint32_t info = T > 2 ? cell_mask(p.lv[3].bits, bc, sx[3]) : 0u;
            if (T >= 3 && (W & 1ull)) {
                uint32_t v = 0, eh = 0, fh = 0;
                q_deep(p, tb, sx, root, bc << 6, v, eh, fh);
                info |= (uint32_t)__popc(eh) << 9 | (uint32_t)__popc(fh) << 20 | (v & 1u) << 8;
            }
            wd[lane] = info;
        }
        // list the chunk's set bits in order
        const uint32_t n = __popcll(W);
        uint32_t incl = n;
#pragma unroll
        for (int k = 1; k < 32; k <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, k);
            if (lane >= k) incl += y;
        }
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        uint64_t word = W;
        for (uint32_t k = incl - n; word; word &= word - 1, ++k)
            lst[k] = (uint16_t)(lane * 64 + __ffsll((long long)word) - 1);
        __syncwarp();
        const uint32_t q0 = p.qpre[ci];
        for (uint32_t j0 = 0; j0 < total; j0 += 32) {
            const uint32_t j = j0 + lane;
            uint32_t c = 0;
            if (j < total) {
                const uint32_t ent = lst[j], w = ent >> 6, i = ent & 63u;
                const uint32_t *m = mk32 + 2 * w + (i >> 5);  // bits of Q_i in mask e: m[e * 64]
                const uint32_t sh = i & 31u;
                uint32_t E0 = 0, X = 0;
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    E0 |= ((m[e * 2 * kChunkWords] >> sh) & 1u) << e;
                    X |= ((m[(8 + e) * 2 * kChunkWords] >> sh) & 1u) << e;
                }
                const uint64_t qc = ((ch * kChunkWords + w) << 6) | i;
                const uint32_t k1 = T >= 2 ? tb.kinds[X] : tb.kinds[coarse_ex(p, tb, sx, root, 1, qc)];
                uint64_t st = qc | (uint64_t)E0 << 36 | (uint64_t)k1 << 44;
                uint32_t k2 = 0, deep = 0;
                if (T >= 2 && (i & 7u) == 0) {
                    const uint32_t info = wd[w];
                    k2 = T > 2 ? tb.kinds[tb.around[(info & 0xFFu) * 8 + (i >> 3)]]
                               : tb.kinds[coarse_ex(p, tb, sx, root, 2, qc >> 3)];
                    st |= (uint64_t)k2 << 51;
                    if (T >= 3 && i == 0) {
                        st |= 1ull << 58;
                        deep = info;
                    }
                }
                p.qs[q0 + j] = st;
                // keys: cnt0 covers level 0; levels 1, 2 and the deep ones
                // add edges and faces, and the vertex of 2Q when level 0 has none
                const uint32_t k0 = tb.cnt0[E0];
                const uint32_t vtx = (k1 | k2 | (deep >> 8)) & 1u;
                c = (k0 & 0xFFu) + ((E0 == 0 && vtx) ? 1u : 0u) +
                    (((k0 >> 8) & 0xFFu) + __popc((k1 >> 1) & 7u) + __popc((k2 >> 1) & 7u)) * (1u << 9) +
                    ((k0 >> 16) + __popc((k1 >> 4) & 7u) + __popc((k2 >> 4) & 7u)) * (1u << 20) +
                    (deep & 0xFFFFFE00u);
            }
            // the round's ranks q0 + j0 + lane cross a tile boundary at lane `split`
            const uint32_t r0 = q0 + j0, split = 32u - (r0 & 31u);
            const uint32_t c0 = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)lane < split ? c : 0u);
            const uint32_t c1 = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)lane < split ? 0u : c);
            if (lane < 6) {
                const uint32_t t = lane < 3 ? c0 : c1, k = lane % 3;
                const uint32_t val = k == 0 ? (t & 0x1FFu) : k == 1 ? ((t >> 9) & 0x7FFu) : (t >> 20);
                if (val) atomicAdd(p.tcnt + k * p.ntiles + (r0 >> 5) + (lane < 3 ? 0 : 1), val);
            }
        }
        __syncwarp();
    }
}

// Key offsets of the edge/face slots: lo bit sl of el/fl is (r << 6) |
// (l << 2) | axis; hi bit t of eh/fh is level 3 + t / 3, axis t % 3.
__host__ __device__ constexpr uint32_t lo_offset(int sl) {
    return sl < 9 ? (uint32_t)((sl / 3) << 2 | (sl % 3)) : (uint32_t)((1 + (sl - 9) / 3) << 6 | ((sl - 9) % 3));
}
__device__ __forceinline__ uint32_t hi_offset(int t) { return (uint32_t)((3 + t / 3) << 2 | (t % 3)); }

// One kind's keys of the warp's 32 Qs (lane j: Q j, slot masks lo/hi).  Slot
// by slot, in output order (vertices: r = 0..7; edges/faces: lo bits 0-8,
// hi bits, lo bits 9-29), every lane appends a 16-bit entry (lane << 9 |
// the slot's key offset) for each key its Q has to the warp's stage at its
// scanned offset: the same short sequence for every lane, no per-lane
// loops.  The stage is then read in order, each entry expanded to its key
// (the owning lane's key base, Q's code shifted, fetched by shuffles, OR the
// offset) and stored coalesced.  A tile has at most 32 x 60 keys of a kind,
// so the stage always suffices.
// `pos` is the lane's first stage position, `tot` the warp's keys of this kind.
template <int KIND>
__device__ __forceinline__ void emit_kind(uint64_t *out, uint64_t base, uint32_t lo, uint32_t hi, uint64_t qc,
                                          uint16_t *stage, int lane, uint32_t pos, uint32_t tot) {
    if (tot == 0) return;
    const uint32_t tag = (uint32_t)lane << 9;
    if (KIND == 0) {
#pragma unroll
        for (int r = 0; r < 8; ++r)
            if ((lo >> r) & 1u) stage[pos++] = (uint16_t)(tag | r);
    } else {
#pragma unroll
        for (int sl = 0; sl < 9; ++sl)
            if ((lo >> sl) & 1u) stage[pos++] = (uint16_t)(tag | lo_offset(sl));
        const uint32_t anyhi = __reduce_or_sync(0xFFFFFFFFu, hi);
        for (int t = 0; (anyhi >> t) != 0; ++t)
            if ((hi >> t) & 1u) stage[pos++] = (uint16_t)(tag | hi_offset(t));
#pragma unroll
        for (int sl = 9; sl < 30; ++sl)
            if ((lo >> sl) & 1u) stage[pos++] = (uint16_t)(tag | lo_offset(sl));
    }
    __syncwarp();
    const uint64_t kb = qc << (KIND == 0 ? 3 : 9);
    const uint32_t kblo = (uint32_t)kb, kbhi = (uint32_t)(kb >> 32);
    // two keys per lane, as 16-byte stores: an odd base first stores key 0 alone
    const uint32_t peel = (uint32_t)(base & 1);
    if (peel) {
        const uint32_t e = stage[0];
        const uint32_t klo = __shfl_sync(0xFFFFFFFFu, kblo, (int)(e >> 9)) | (e & 511u);
        const uint32_t khi = __shfl_sync(0xFFFFFFFFu, kbhi, (int)(e >> 9));
        if (lane == 0) out[base] = (uint64_t)khi << 32 | klo;
    }
    for (uint32_t i0 = peel; i0 < tot; i0 += 64) {
        const uint32_t i = i0 + 2 * lane;
        const uint32_t ea = i < tot ? stage[i] : 0u, eb = i + 1 < tot ? stage[i + 1] : 0u;
        const uint32_t alo = __shfl_sync(0xFFFFFFFFu, kblo, (int)(ea >> 9)) | (ea & 511u);
        const uint32_t ahi = __shfl_sync(0xFFFFFFFFu, kbhi, (int)(ea >> 9));
        const uint32_t blo = __shfl_sync(0xFFFFFFFFu, kblo, (int)(eb >> 9)) | (eb & 511u);
        const uint32_t bhi = __shfl_sync(0xFFFFFFFFu, kbhi, (int)(eb >> 9));
        if (i + 1 < tot)
            *reinterpret_cast<ulonglong2 *>(out + base + i) =
                make_ulonglong2((unsigned long long)ahi << 32 | alo, (unsigned long long)bhi << 32 | blo);
        else if (i < tot)
            out[base + i] = (uint64_t)ahi << 32 | alo;
    }
    __syncwarp();
}

// One warp per tile of 32 consecutive states, expanded into keys at the
// tile's scanned offsets.
__global__ void __launch_bounds__(kDedupWarps * 32) k_dedup_write(const __grid_constant__ DedupParams p,
                                                                 uint64_t nq) {
    __shared__ DedupTables tb;
    __shared__ uint16_t stage[kDedupWarps][kStageKeys];
    __shared__ uint64_t sx[kMaxLevels];
    if (threadIdx.x < kMaxLevels) sx[threadIdx.x] = (int)threadIdx.x <= p.T ? spread3(p.lv[threadIdx.x].side) : 0;
    load_tables(tb, p.tables);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t nwarps = (uint64_t)gridDim.x * kDedupWarps;
    const uint64_t root = *p.root;
    uint16_t *stg = stage[warp];
    for (uint64_t t = (uint64_t)blockIdx.x * kDedupWarps + warp; t < p.ntiles; t += nwarps) {
        const uint64_t r = t * 32 + lane;
        const bool act = r < nq;
        const uint64_t s = act ? p.qs[r] : 0;
        const QMasks m = act ? q_masks(p, tb, sx, root, s) : QMasks{0, 0, 0, 0, 0};
        const uint64_t qc = s & kQcMask;
        // one scan for the three kinds: counts packed v | e << 9 | f << 20
        // (at most 32 x 8 and 32 x 60 per tile)
        const uint32_t c = (uint32_t)__popc(m.v) | (uint32_t)(__popc(m.el) + __popc(m.eh)) << 9 |
                           (uint32_t)(__popc(m.fl) + __popc(m.fh)) << 20;
        uint32_t x = c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
            if (lane >= d) x += y;
        }
        const uint32_t tot = __shfl_sync(0xFFFFFFFFu, x, 31), ex = x - c;
        emit_kind<0>(p.out[0], p.tpre[t], m.v, 0u, qc, stg, lane, ex & 0x1FFu, tot & 0x1FFu);
        emit_kind<1>(p.out[1], p.tpre[(p.ntiles + 1) + t], m.el, m.eh, qc, stg, lane, (ex >> 9) & 0x7FFu,
                     (tot >> 9) & 0x7FFu);
        emit_kind<2>(p.out[2], p.tpre[2 * (p.ntiles + 1) + t], m.fl, m.fh, qc, stg, lane, ex >> 20, tot >> 20);
    }
}

// Set bits per touched chunk (one warp per chunk).
__global__ void k_chunk_bits(const __grid_constant__ DedupParams p) {
    const uint64_t w = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= p.ntouched) return;
    const uint64_t *D64 = reinterpret_cast<const uint64_t *>(p.D);
    const uint32_t n = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)__popcll(D64[(uint64_t)p.list[w] * kChunkWords + lane]));
    if (lane == 0) p.qn[w] = n;
}

// Zeroes the 2048-word regions of D that can hold a candidate: every lattice
// cell Q has coordinates <= side / 2 (corners of the grid's cells), and a
// region -- an aligned box of 64 x 64 x 32 Q -- holds one iff its lowest
// corner does.  At side 2048 that is 9,537 of 65,536 regions; only the
// touched chunks of D are read later, all inside these.
__global__ void __launch_bounds__(256) k_dedup_zero(uint64_t *__restrict__ D, uint64_t regions, uint32_t half) {
    for (uint64_t b = blockIdx.x; b < regions; b += gridDim.x) {
        const uint64_t c = b << 17;
        if (compact3(c) > half || compact3(c >> 1) > half || compact3(c >> 2) > half) continue;
        uint4 *w = reinterpret_cast<uint4 *>(D + b * 2048);
#pragma unroll
        for (int q = 0; q < 4; ++q) w[threadIdx.x + 256 * q] = make_uint4(0, 0, 0, 0);
    }
}

// The level-1 part of D, word by word over the same regions: bit Q is set
// iff some level-1 node has corner Q, i.e. a level-1 cell Q - d (d in
// {0,1}^3) exists -- its level-2 parent is occupied.  The level-2 bytes
// above the blocks b - d, upsampled to level-1 cells, dilated by one cell
// along each axis (separable: 7 shifts).  Every word of a region is
// written, zeros included, so D needs no zeroing; G gets every chunk with a
// set bit and *p.nq the set bits.  Needs T >= 2 (the level-2 bitmap).
// Most words lie far from every node: a region (64 x 64 x 32 Q) whose
// level-7 cells c - e (c = its origin >> 6, e in {0,1}^3: they hold every
// level-2 parent of the cells Q - d it needs) are all empty is only
// zeroed, and so is a warp's chunk (16 x 16 x 8 Q) whose level-5 cells
// c - e (c = its origin >> 4) are empty.
__global__ void __launch_bounds__(256) k_dedup_build(const __grid_constant__ DedupParams p, uint64_t regions,
                                                     uint32_t half) {
    const int lane = threadIdx.x & 31;
    const uint32_t s2 = p.lv[2].side;
    const uint64_t nb2 = spread3((s2 + 1) / 2), valid2 = s2 >= 2 ? 0xFFull : 0x1ull;
    const uint64_t *bits2 = p.lv[2].bits;
    const int T = p.T;
    const uint64_t sx5 = T >= 5 ? spread3(p.lv[5].side) : 0, sx7 = T >= 7 ? spread3(p.lv[7].side) : 0;
    uint64_t *D64 = reinterpret_cast<uint64_t *>(p.D);
    uint32_t cnt = 0;
    for (uint64_t r = blockIdx.x; r < regions; r += gridDim.x) {
        const uint64_t c = r << 17;  // the region's first Q
        if (compact3(c) > half || compact3(c >> 1) > half || compact3(c >> 2) > half) continue;
        const uint32_t near7 = T >= 7 && threadIdx.x < 8 ? cell_bit(p.lv[7].bits, c >> 18, sx7, threadIdx.x) : 0u;
        if (!__syncthreads_or(T < 7 || near7)) {
            uint4 *w = reinterpret_cast<uint4 *>(D64 + r * 2048);
#pragma unroll
            for (int q = 0; q < 4; ++q) w[threadIdx.x + 256 * q] = make_uint4(0, 0, 0, 0);
            continue;
        }
        for (int k = 0; k < 8; ++k) {
            const uint64_t bc = r * 2048 + k * 256 + threadIdx.x;  // word = block code
            if (T >= 5) {
                const uint64_t c5 = ((bc & ~31ull) << 6) >> 12;  // the chunk's origin at level 5
                const uint32_t near5 = lane < 8 ? cell_bit(p.lv[5].bits, c5, sx5, lane) : 0u;
                if (!__ballot_sync(0xFFFFFFFFu, near5)) {
                    D64[bc] = 0;
                    continue;
                }
            }
            const uint64_t xm = bc & kDilX, ym = bc & kDilY, zm = bc & kDilZ;
            const uint64_t xd = dil_dec(xm, kDilX), yd = dil_dec(ym, kDilY), zd = dil_dec(zm, kDilZ);
            uint64_t U[8];
#pragma unroll
            for (int d = 0; d < 8; ++d) {
                const bool low = (!(d & 1) || xm != 0) && (!(d & 2) || ym != 0) && (!(d & 4) || zm != 0);
                const uint64_t nc = ((d & 1) ? xd : xm) | ((d & 2) ? yd : ym) | ((d & 4) ? zd : zm);
                const bool in2 = low && (nc & kDilX) < nb2 && (nc & kDilY) < (nb2 << 1) && (nc & kDilZ) < (nb2 << 2);
                U[d] = in2 ? (bits2[nc >> 3] >> (8 * (nc & 7))) & valid2 : 0ull;
            }
            uint64_t w = 0;
            if (U[0] | U[1] | U[2] | U[3] | U[4] | U[5] | U[6] | U[7]) {
#pragma unroll
                for (int d = 0; d < 8; ++d) U[d] = upsample8(U[d]);
                const uint64_t G0 = U[0] | shift_up<0>(U[0], U[1]), G2 = U[2] | shift_up<0>(U[2], U[3]);
                const uint64_t G4 = U[4] | shift_up<0>(U[4], U[5]), G6 = U[6] | shift_up<0>(U[6], U[7]);
                const uint64_t H0 = G0 | shift_up<1>(G0, G2), H4 = G4 | shift_up<1>(G4, G6);
                w = H0 | shift_up<2>(H0, H4);
            }
            D64[bc] = w;
            const uint32_t any = __ballot_sync(0xFFFFFFFFu, w != 0);  // the warp's 32 words: one chunk
            if (lane == 0 && any) atomicOr(p.G + (bc >> 10), 1u << ((bc >> 5) & 31));
            cnt += __popcll(w);
        }
    }
    block_add(p.nq, cnt);
}

// The touched chunks in order: per-word popcounts of G, then (after a scan)
// the chunk index of every set bit.
__global__ void k_touched_count(const uint32_t *__restrict__ G, uint64_t n, uint32_t *__restrict__ cnt) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n) cnt[i] = __popc(G[i]);
}

__global__ void k_touched_list(const uint32_t *__restrict__ G, uint64_t n, const uint32_t *__restrict__ pre,
                               uint32_t *__restrict__ list) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t g = G[i];
    uint32_t at = pre[i];
    while (g) {
        list[at++] = (uint32_t)(i * 32 + __ffs(g) - 1);
        g &= g - 1;
    }
}

int dedup_fail(int code, const char *msg) {
    svo::host::set_error(msg);
    return code;
}

}  // namespace

// A dedup between dedup_begin (scratch, tables, the candidate bitmap's
// level-1 part: bitmaps only) and dedup_finish (coarse marks, states, keys:
// they need the code lists).  Its scratch is freed on its stream.
struct DedupRun {
    cudaMemPool_t pool;
    cudaStream_t st;
    int num_sms;
    DedupParams p;
    void *base;    // one pool block holding blk[0..7]
    void *blk[8];
    size_t sz[8];
    uint64_t side, d_words, g_words;
    bool build1;
};

void dedup_abort(DedupRun *run) {
    if (!run) return;
    if (run->base) cudaFreeAsync(run->base, run->st);
    delete run;
}

int dedup_begin(cudaMemPool_t pool, cudaStream_t st, int T, const uint64_t *const *bits, const uint32_t *sides,
                int num_sms, DedupRun **out) {
    svo::host::TraceRange trace("svo: dedup candidates");
    *out = nullptr;
    if (T < 1) return dedup_fail(SVO_ERR_DEGENERATE, "dedup needs at least two levels");
    if (T > 12) return dedup_fail(SVO_ERR_UNSUPPORTED, "dedup of more than 13 levels");
    DedupRun *run = new DedupRun{};
    run->pool = pool;
    run->st = st;
    run->num_sms = num_sms;
    DedupParams &p = run->p;
    p.T = T;
    for (int l = 0; l <= T; ++l) p.lv[l] = DedupLevel{bits[l], nullptr, 0, sides[l]};
    const uint64_t side = sides[0];
    const uint64_t d_bits = side * side * side;
    const uint64_t d_words = std::max<uint64_t>((d_bits + 63) / 64 + kChunkWords - 1, kChunkWords) / kChunkWords * kChunkWords;
    p.chunks = d_words / kChunkWords;
    const uint64_t g_words = (p.chunks + 31) / 32;
    run->side = side;
    run->d_words = d_words;
    run->g_words = g_words;
    if (p.chunks > 0xFFFFFFFFull) {
        delete run;
        return dedup_fail(SVO_ERR_UNSUPPORTED, "dedup grid too large");
    }
    // scratch: D, G, G popcounts + prefix, touched list, scan scratch, status, tables
    const size_t sz[8] = {d_words * 8, g_words * 4, g_words * 4, (g_words + 1) * 4, p.chunks * 4,
                          scan_scratch_words(std::max<uint64_t>(p.chunks, g_words)) * 8, 256, sizeof(DedupTables)};
    std::memcpy(run->sz, sz, sizeof sz);
    size_t at[8], total = 0;
    for (int i = 0; i < 8; ++i) {
        at[i] = total;
        total += (sz[i] + 255) / 256 * 256;
    }
    cudaError_t e = pool_malloc(&run->base, total, pool, st);
    if (e == cudaSuccess)
        for (int i = 0; i < 8; ++i) run->blk[i] = static_cast<char *>(run->base) + at[i];
    auto fail = [&](cudaError_t err, const char *what) {
        dedup_abort(run);
        char msg[256];
        snprintf(msg, sizeof msg, "dedup %s: %s", what, cudaGetErrorString(err));
        return dedup_fail(err == cudaErrorMemoryAllocation ? SVO_ERR_OUT_OF_MEMORY : SVO_ERR_CUDA, msg);
    };
    if (e != cudaSuccess) return fail(e, "scratch");
    void **blk = run->blk;
    p.D = static_cast<uint32_t *>(blk[0]);
    p.G = static_cast<uint32_t *>(blk[1]);
    p.list = static_cast<uint32_t *>(blk[4]);
    p.nq = reinterpret_cast<unsigned long long *>(static_cast<char *>(blk[6]) + 8);
    p.tables = static_cast<const DedupTables *>(blk[7]);
    k_dedup_tables<<<1, 256, 0, st>>>(static_cast<DedupTables *>(blk[7]));
    count_launches(1);
    // D: in 2048-word regions, level 1 by k_dedup_build (T >= 2), the
    // coarser levels marked after it; else zeroed and marked at all levels
    const bool build1 = d_words % 2048 == 0 && T >= 2;
    run->build1 = build1;
    if ((e = cudaMemsetAsync(p.G, 0, sz[1], st)) || (e = cudaMemsetAsync(blk[6], 0, 16, st)))
        return fail(e, "memset");
    if (d_words % 2048 == 0) {
        const uint64_t regions = d_words / 2048;
        const unsigned rb = (unsigned)std::min<uint64_t>(regions, (uint64_t)num_sms * 8);
        if (build1)
            k_dedup_build<<<rb, 256, 0, st>>>(p, regions, (uint32_t)(side / 2));
        else
            k_dedup_zero<<<rb, 256, 0, st>>>(reinterpret_cast<uint64_t *>(p.D), regions, (uint32_t)(side / 2));
        count_launches(1);
        e = cudaGetLastError();
    } else {
        e = cudaMemsetAsync(p.D, 0, sz[0], st);
    }
    if (e != cudaSuccess) return fail(e, "clear");
    *out = run;
    return SVO_OK;
}

int dedup_finish(DedupRun *run, cudaMemPool_t out_pool, const EmitParams &ep, uint64_t n_out[3], uint64_t *out[3]) {
    svo::host::TraceRange trace("svo: dedup keys");
    for (int k = 0; k < 3; ++k) {
        n_out[k] = 0;
        out[k] = nullptr;
    }
    const cudaMemPool_t pool = run->pool;
    const cudaStream_t st = run->st;
    const int num_sms = run->num_sms;
    DedupParams &p = run->p;
    const int T = p.T;
    if (ep.T != T || (uint64_t)ep.N * 12 > 0xFFFFFFFFull) {
        dedup_abort(run);
        return dedup_fail(SVO_ERR_UNSUPPORTED, "dedup of more than 357M nodes");
    }
    p.root = ep.lv[T].K1;
    for (int l = 0; l <= T; ++l) {
        p.lv[l].K1 = ep.lv[l].K1;
        p.lv[l].groups = ep.lv[l].n / 8;
    }
    uint32_t g = 0;
    for (int l = 1; l < T; ++l) {
        p.gstart[l] = g;
        g += p.lv[l].groups;
    }
    p.gstart[T] = g;
    const uint32_t mark_total = g + 1;
    const uint64_t g_words = run->g_words;
    void **blk = run->blk;
    void *blk2[6] = {};  // sized once the counts are known: states per chunk, the states, keys per tile
    void *base2 = nullptr;  // one pool block holding blk2
    uint32_t *gcnt = static_cast<uint32_t *>(blk[2]);
    uint32_t *gpre = static_cast<uint32_t *>(blk[3]);
    uint32_t *list = static_cast<uint32_t *>(blk[4]);
    auto *scan = static_cast<unsigned long long *>(blk[5]);
    uint32_t *status = static_cast<uint32_t *>(blk[6]);
    cudaError_t e = cudaSuccess;
    auto release = [&]() {
        if (base2) cudaFreeAsync(base2, st);
        dedup_abort(run);
    };
    auto fail = [&](cudaError_t err, const char *what) {
        release();
        char msg[256];
        snprintf(msg, sizeof msg, "dedup %s: %s", what, cudaGetErrorString(err));
        return dedup_fail(err == cudaErrorMemoryAllocation ? SVO_ERR_OUT_OF_MEMORY : SVO_ERR_CUDA, msg);
    };
    const bool build1 = run->build1;
    const uint32_t mark_first = build1 ? p.gstart[2] : 0u;
    k_dedup_mark<<<(mark_total - mark_first + 255) / 256, 256, 0, st>>>(p, mark_first, mark_total);
    k_touched_count<<<(unsigned)((g_words + 255) / 256), 256, 0, st>>>(p.G, g_words, gcnt);
    count_launches(2);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "mark");
    if ((e = launch_scan(gcnt, gpre, g_words, scan, status, st)) != cudaSuccess) return fail(e, "scan");
    k_touched_list<<<(unsigned)((g_words + 255) / 256), 256, 0, st>>>(p.G, g_words, gpre, list);
    count_launches(1);
    uint32_t h[4] = {0, 0, 0, 0};
    unsigned long long h_nq = 0;
    if ((e = cudaMemcpyAsync(h, gpre + g_words, 4, cudaMemcpyDeviceToHost, st)) ||
        (e = cudaMemcpyAsync(&h_nq, p.nq, 8, cudaMemcpyDeviceToHost, st)) || (e = cudaStreamSynchronize(st)))
        return fail(e, "touched chunks");
    p.ntouched = h[0];
    const uint64_t nt = p.ntouched;
    if (h_nq > 0xFFFFFFFFull) {
        release();
        return dedup_fail(SVO_ERR_UNSUPPORTED, "dedup of more than 2^32 lattice cells");
    }
    const uint64_t ntiles = (h_nq + 31) / 32;
    p.ntiles = ntiles;
    const size_t sz2[6] = {std::max<uint64_t>(nt, 1) * 4, (nt + 1) * 4, std::max<uint64_t>(h_nq, 1) * 8,
                           3 * std::max<uint64_t>(ntiles, 1) * 4, 3 * (ntiles + 1) * 4,
                           scan_scratch_words(std::max<uint64_t>(std::max<uint64_t>(nt, ntiles), 1)) * 8};
    size_t at2[6], total2 = 0;
    for (int i = 0; i < 6; ++i) {
        at2[i] = total2;
        total2 += (sz2[i] + 255) / 256 * 256;
    }
    if ((e = pool_malloc(&base2, total2, pool, st)) != cudaSuccess) return fail(e, "scratch");
    for (int i = 0; i < 6; ++i) blk2[i] = static_cast<char *>(base2) + at2[i];
    p.qn = static_cast<uint32_t *>(blk2[0]);
    uint32_t *qpre = static_cast<uint32_t *>(blk2[1]);
    p.qpre = qpre;
    p.qs = static_cast<uint64_t *>(blk2[2]);
    p.tcnt = static_cast<uint32_t *>(blk2[3]);
    uint32_t *tpre = static_cast<uint32_t *>(blk2[4]);
    p.tpre = tpre;
    auto *scan2 = static_cast<unsigned long long *>(blk2[5]);
    if ((e = cudaMemsetAsync(p.tcnt, 0, sz2[3], st)) != cudaSuccess) return fail(e, "memset");
    if (nt > 0) {
        k_chunk_bits<<<(unsigned)((nt + 7) / 8), 256, 0, st>>>(p);
        count_launches(1);
        if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "chunk bits");
        if ((e = launch_scan(p.qn, qpre, nt, scan2, status, st)) != cudaSuccess) return fail(e, "scan");
        const unsigned sblocks =
            (unsigned)std::min<uint64_t>((nt + kStateWarps - 1) / kStateWarps, (uint64_t)num_sms * 32);
        k_dedup_state<<<sblocks, kStateWarps * 32, 0, st>>>(p);
        count_launches(1);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "count");
    for (int k = 0; k < 3; ++k)
        if ((e = launch_scan(p.tcnt + k * ntiles, tpre + k * (ntiles + 1), ntiles, scan2, status, st)) != cudaSuccess)
            return fail(e, "scan");
    for (int k = 0; k < 3; ++k)
        if ((e = cudaMemcpyAsync(h + k, tpre + k * (ntiles + 1) + ntiles, 4, cudaMemcpyDeviceToHost, st)))
            return fail(e, "read totals");
    if ((e = cudaMemcpyAsync(h + 3, status, 4, cudaMemcpyDeviceToHost, st)) || (e = cudaStreamSynchronize(st)))
        return fail(e, "read totals");
    if (h[3] & kStatusScanTimeout) {
        release();
        return dedup_fail(SVO_ERR_DEVICE_TIMEOUT, "dedup scan look-back timed out");
    }
    for (int k = 0; k < 3; ++k) {
        if (h[k] == 0) continue;
        void *o = nullptr;
        if ((e = pool_malloc(&o, (size_t)h[k] * 8, out_pool, st)) != cudaSuccess) {
            for (int j = 0; j < k; ++j)
                if (out[j]) cudaFreeAsync(out[j], st);
            for (int j = 0; j < 3; ++j) out[j] = nullptr;
            return fail(e, "output");
        }
        out[k] = p.out[k] = static_cast<uint64_t *>(o);
        n_out[k] = h[k];
    }
    if (ntiles > 0) {
        const unsigned wblocks =
            (unsigned)std::min<uint64_t>((ntiles + kDedupWarps - 1) / kDedupWarps, (uint64_t)num_sms * 16);
        k_dedup_write<<<wblocks, kDedupWarps * 32, 0, st>>>(p, h_nq);
        count_launches(1);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) {
        for (int j = 0; j < 3; ++j) {
            if (out[j]) cudaFreeAsync(out[j], st);
            out[j] = nullptr;
            n_out[j] = 0;
        }
        return fail(e, "emit");
    }
    release();
    return SVO_OK;
}

}  // namespace svo
