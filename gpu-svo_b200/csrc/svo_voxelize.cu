// svo_voxelize.cu -- bounding cube and conservative surface voxelization.
//
// Restates the reference's BaseModel bounding cube (src/BaseModel.h:24-49,
// 64-73) and surfaceVoxelize (src/SVO.cu:37-188) for sm_100a.  Instead of one
// thread per triangle writing a dense u32 array of res^3 entries, each overlap
// sets one bit of a Morton-ordered occupancy bitmap (res^3 bits); the test
// arithmetic is the reference's, operation for operation (svo_device.cuh Fp).
//
// Work split: a triangle whose grid bbox has at most `serial_max` voxels is
// tested by its own thread, row by row.  Larger ones go to a queue of entries
// (triangle, at most `warp_max` 4x4x4 bricks aligned to the grid) that
// warps take one at a time; a brick is 64 consecutive Morton codes, two
// bitmap words.  Without a queue (the allocation-free entry point) the
// triangle's own warp walks its bricks in place.
//
// Brick culling is exact.  Every predicate of the voxel test is monotone in
// each grid coordinate separately (each is built from rounded products,
// sums and fmas of p = coordinate * unit, and IEEE rounding is monotone), so
// over a brick an edge test is largest at the corner picked by the signs of
// its two coefficients, and n.p is smallest/largest at the corners picked by
// the signs of n.  A brick is skipped only when one predicate, evaluated at
// its best corner with the voxel test's own arithmetic, already fails; every
// other brick is split and tested again, and the voxels of surviving
// sub-bricks are tested one per lane.  Triangles with any non-finite setup
// value are never culled.
#include "svo_internal.h"

namespace svo {

namespace {


__device__ __forceinline__ uint32_t f2ord(float f) {
    uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o);
}

// ---------------------------------------------------------------------------
// Bounding box of all vertices (exact min/max through an order-preserving
// integer map), then the bounding cube on one thread.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void bbox_take(float v, int a, uint32_t lo[3], uint32_t hi[3], bool &bad) {
    bad |= !isfinite(v);
    const uint32_t o = f2ord(v);
    lo[a] = min(lo[a], o);
    hi[a] = max(hi[a], o);
}

// Block b belongs to mesh m = the segment of bbox_off holding b.  When the
// mesh's points are 16-byte aligned, 4 points (12 floats, 3 float4) per step;
// the component of float k is k % 3, the same in every 12-float group.
__global__ void k_bbox_reduce(BatchDev bd) {
    const int m = find_segment(bd.bbox_off, bd.n, (uint32_t)blockIdx.x);
    const MeshDev &md = bd.mesh[m];
    const float *__restrict__ pts = md.pts;
    const int64_t n = md.n_pts;
    uint32_t lo[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, hi[3] = {0u, 0u, 0u};
    bool bad = false;
    const uint32_t nb = bd.bbox_off[m + 1] - bd.bbox_off[m];
    const int64_t tid = (blockIdx.x - bd.bbox_off[m]) * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nth = (int64_t)nb * blockDim.x;
    int64_t done = 0;
    if ((reinterpret_cast<uintptr_t>(pts) & 15) == 0) {
        const float4 *p4 = reinterpret_cast<const float4 *>(pts);
        const int64_t groups = n / 4;
        for (int64_t gi = tid; gi < groups; gi += nth) {
            const float4 a = __ldcs(p4 + 3 * gi), b = __ldcs(p4 + 3 * gi + 1), c = __ldcs(p4 + 3 * gi + 2);
            bbox_take(a.x, 0, lo, hi, bad); bbox_take(a.y, 1, lo, hi, bad); bbox_take(a.z, 2, lo, hi, bad);
            bbox_take(a.w, 0, lo, hi, bad); bbox_take(b.x, 1, lo, hi, bad); bbox_take(b.y, 2, lo, hi, bad);
            bbox_take(b.z, 0, lo, hi, bad); bbox_take(b.w, 1, lo, hi, bad); bbox_take(c.x, 2, lo, hi, bad);
            bbox_take(c.y, 0, lo, hi, bad); bbox_take(c.z, 1, lo, hi, bad); bbox_take(c.w, 2, lo, hi, bad);
        }
        done = groups * 4;
    }
    for (int64_t i = done + tid; i < n; i += nth)
#pragma unroll
        for (int a = 0; a < 3; ++a) bbox_take(__ldg(pts + 3 * i + a), a, lo, hi, bad);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        lo[a] = __reduce_min_sync(0xFFFFFFFFu, lo[a]);
        hi[a] = __reduce_max_sync(0xFFFFFFFFu, hi[a]);
    }
    if (__any_sync(0xFFFFFFFFu, bad) && (threadIdx.x & 31) == 0) atomicOr(&md.gp->status, kStatusNonFinite);
    // the block's extremes, then one atomic per value and block (the 6 words
    // are shared by every block of the mesh)
    __shared__ uint32_t wmm[32][6];
    const int warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            wmm[warp][a] = lo[a];
            wmm[warp][3 + a] = hi[a];
        }
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        uint32_t v = wmm[0][threadIdx.x];
        for (int w = 1; w < nwarp; ++w) v = threadIdx.x < 3 ? min(v, wmm[w][threadIdx.x]) : max(v, wmm[w][threadIdx.x]);
        if (threadIdx.x < 3) atomicMin(md.mm + threadIdx.x, v);
        else atomicMax(md.mm + threadIdx.x, v);
    }
}

// createMeshBBCube (src/BaseModel.h:24-49) and unitVoxelSize
// (src/SVO.cu:348-350).  Host code in the reference: no contraction there, so
// every operation is an explicitly rounded intrinsic.
__global__ void k_grid_setup(BatchDev bd) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= bd.n) return;
    const MeshDev &md = bd.mesh[m];
    const uint32_t *mm = md.mm;
    GridParams *gp = md.gp;
    const int rx = md.res[0], ry = md.res[1], rz = md.res[2];
    float mn[3], mx[3], len[3], amin[3], amax[3];
    for (int a = 0; a < 3; ++a) {
        mn[a] = ord2f(mm[a]);
        mx[a] = ord2f(mm[3 + a]);
        len[a] = __fsub_rn(mx[a], mn[a]);
        amin[a] = mn[a];
        amax[a] = mx[a];
    }
    const float maxlen = cmaxf(len[0], cmaxf(len[1], len[2]));
    for (int a = 0; a < 3; ++a) {
        if (maxlen == len[a]) continue;
        const float half = __fdiv_rn(__fsub_rn(maxlen, len[a]), 2.0f);
        amin[a] = __fsub_rn(mn[a], half);
        amax[a] = __fadd_rn(mx[a], half);
    }
    const int res[3] = {rx, ry, rz};
    for (int a = 0; a < 3; ++a) {
        const float eps = __fdiv_rn(__fsub_rn(amax[a], amin[a]), 10001.0f);
        amin[a] = __fsub_rn(amin[a], eps);
        amax[a] = __fadd_rn(amax[a], eps);
        const float w = __fsub_rn(amax[a], amin[a]);
        gp->bbox[a] = amin[a];
        gp->bbox[3 + a] = amax[a];
        gp->bbox[6 + a] = w;
        gp->origin[a] = amin[a];
        gp->unit[a] = __fdiv_rn(w, (float)res[a]);
    }
}

// ---------------------------------------------------------------------------
// Triangle setup (src/SVO.cu:53-149).
// ---------------------------------------------------------------------------
struct Tri {
    float n[3];
    float d1, d2;
    float ea[9], eb[9], ed[9];  // edge test k of plane p at 3p+k: XY, YZ, ZX
    int lo[3], hi[3];
    int cull;                   // all setup values finite: brick culling allowed
};

__device__ __forceinline__ int f2i_rz(float f) { return __float2int_rz(f); }
__device__ __forceinline__ int clampi(int f, int a, int b) { return max(a, min(f, b)); }

// Voxel bbox of a triangle (vertices relative to the grid origin), clamped
// to the grid: src/SVO.cu:58-66.  The region marker and the voxel test use
// this one function, so the regions cover every voxel the test can set.
__device__ __forceinline__ void tri_box(const GridParams &g, const int res[3], const float v[3][3], int lo[3],
                                        int hi[3]) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float mn = cminf(v[0][a], cminf(v[1][a], v[2][a]));
        const float mx = cmaxf(v[0][a], cmaxf(v[1][a], v[2][a]));
        lo[a] = clampi(f2i_rz(__fdiv_rn(mn, g.unit[a])), 0, res[a] - 1);
        hi[a] = clampi(f2i_rz(__fdiv_rn(mx, g.unit[a])), 0, res[a] - 1);
    }
}

template <bool S>
__device__ __forceinline__ void tri_setup(const GridParams &g, const int res[3], const float *p0,
                                          const float *p1, const float *p2, Tri &t) {
    float v[3][3], e[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        v[0][a] = __fsub_rn(p0[a], g.origin[a]);
        v[1][a] = __fsub_rn(p1[a], g.origin[a]);
        v[2][a] = __fsub_rn(p2[a], g.origin[a]);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        e[0][a] = __fsub_rn(v[1][a], v[0][a]);
        e[1][a] = __fsub_rn(v[2][a], v[1][a]);
        e[2][a] = __fsub_rn(v[0][a], v[2][a]);
    }
    // n = e0.cross(e1).normalized()
    float c0 = Fp<S>::diffprod(e[0][1], e[1][2], e[0][2], e[1][1]);
    float c1 = Fp<S>::diffprod(e[0][2], e[1][0], e[0][0], e[1][2]);
    float c2 = Fp<S>::diffprod(e[0][0], e[1][1], e[0][1], e[1][0]);
    // squared norm: c0*c0 + (c1*c1 + c2*c2), the inner sum fusing c2*c2
    const float sq = Fp<S>::dot3_head(c0, c0, Fp<S>::dot2_late(c1, c2, c1, c2));
    if (sq > 0.0f) {
        const float r = __fsqrt_rn(sq);
        c0 = __fdiv_rn(c0, r);
        c1 = __fdiv_rn(c1, r);
        c2 = __fdiv_rn(c2, r);
    }
    t.n[0] = c0;
    t.n[1] = c1;
    t.n[2] = c2;
    const float *u = g.unit;
    tri_box(g, res, v, t.lo, t.hi);
    float ca[3], cb[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float c = t.n[a] > 0.0f ? u[a] : 0.0f;
        ca[a] = __fsub_rn(c, v[0][a]);
        cb[a] = __fsub_rn(__fsub_rn(u[a], c), v[0][a]);
    }
    t.d1 = Fp<S>::dot3(t.n[0], t.n[1], t.n[2], ca[0], ca[1], ca[2]);
    t.d2 = Fp<S>::dot3(t.n[0], t.n[1], t.n[2], cb[0], cb[1], cb[2]);
    // projections: plane (i, j) with flip axis f: XY (0,1,2), YZ (1,2,0), ZX (2,0,1)
#pragma unroll
    for (int p = 0; p < 3; ++p) {
        const int i = p == 0 ? 0 : (p == 1 ? 1 : 2);
        const int j = p == 0 ? 1 : (p == 1 ? 2 : 0);
        const int f = p == 0 ? 2 : (p == 1 ? 0 : 1);
        const bool flip = t.n[f] < 0.0f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            float a0 = -e[k][j];
            float a1 = e[k][i];
            if (flip) {
                a0 = -a0;
                a1 = -a1;
            }
            const float dt = Fp<S>::dot2(a0, a1, v[k][i], v[k][j]);
            t.ea[3 * p + k] = a0;
            t.eb[3 * p + k] = a1;
            t.ed[3 * p + k] = __fadd_rn(__fadd_rn(-dt, cmaxf(0.0f, __fmul_rn(u[i], a0))),
                                        cmaxf(0.0f, __fmul_rn(u[j], a1)));
        }
    }
    bool fin = isfinite(t.n[0]) && isfinite(t.n[1]) && isfinite(t.n[2]) && isfinite(t.d1) && isfinite(t.d2) &&
               isfinite(u[0]) && isfinite(u[1]) && isfinite(u[2]);
#pragma unroll
    for (int k = 0; k < 9; ++k) fin = fin && isfinite(t.ea[k]) && isfinite(t.eb[k]) && isfinite(t.ed[k]);
    t.cull = fin ? 1 : 0;
}

// Per-row state: everything of the voxel test that depends only on (y, z).
struct Row {
    float inner;      // tail of n.dot(p)
    float xyb[3];     // XY: b * p.y
    float zxp[3];     // ZX: a * p.z
};

template <bool S>
__device__ __forceinline__ bool row_prep(const Tri &t, const GridParams &g, int y, int z, Row &r) {
    const float py = __fmul_rn((float)y, g.unit[1]);
    const float pz = __fmul_rn((float)z, g.unit[2]);
#pragma unroll
    for (int k = 0; k < 3; ++k)  // YZ tests depend on the row only
        if (__fadd_rn(Fp<S>::dot2(t.ea[3 + k], t.eb[3 + k], py, pz), t.ed[3 + k]) < 0.0f) return false;
    r.inner = Fp<S>::dot3_tail(t.n[1], t.n[2], py, pz);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        r.xyb[k] = __fmul_rn(t.eb[k], py);
        r.zxp[k] = __fmul_rn(t.ea[6 + k], pz);
    }
    return true;
}

template <bool S>
__device__ __forceinline__ bool voxel_test(const Tri &t, const GridParams &g, const Row &r, int x) {
    const float px = __fmul_rn((float)x, g.unit[0]);
    const float nd = Fp<S>::dot3_head(t.n[0], px, r.inner);
    bool ok = !(__fmul_rn(__fadd_rn(nd, t.d1), __fadd_rn(nd, t.d2)) > 0.0f);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float f = S ? __fadd_rn(__fmul_rn(t.ea[k], px), r.xyb[k]) : __fmaf_rn(t.ea[k], px, r.xyb[k]);
        ok &= !(__fadd_rn(f, t.ed[k]) < 0.0f);
        // the ZX tests fuse b*p.x (a*p.z is loop-invariant, hoisted out of the x loop)
        const float h = S ? __fadd_rn(r.zxp[k], __fmul_rn(t.eb[6 + k], px)) : __fmaf_rn(t.eb[6 + k], px, r.zxp[k]);
        ok &= !(__fadd_rn(h, t.ed[6 + k]) < 0.0f);
    }
    return ok;
}

// OR-accumulates hits of consecutive voxels that share a bitmap word.
struct HitSink {
    uint32_t *bm;
    uint64_t word = ~0ull;
    uint32_t mask = 0;
    __device__ __forceinline__ void add(uint64_t code) {
        const uint64_t w = code >> 5;
        if (w != word) {
            if (mask) atomicOr(bm + word, mask);
            word = w;
            mask = 0;
        }
        mask |= 1u << (code & 31);
    }
    __device__ __forceinline__ void flush() {
        if (mask) atomicOr(bm + word, mask);
        mask = 0;
        word = ~0ull;
    }
};

// Tests voxels x in [x0, x1] of row (y, z); syz holds the Morton bits of y
// and z, and x's are stepped in place (dil_inc).
template <bool S>
__device__ __forceinline__ void row_segment(const Tri &t, const GridParams &g, int y, int z, uint64_t syz, int x0,
                                            int x1, HitSink &sink) {
    Row r;
    if (!row_prep<S>(t, g, y, z, r)) return;
    uint64_t xm = spread3((uint32_t)x0);
    for (int x = x0; x <= x1; ++x, xm = dil_inc(xm, kDilX))
        if (voxel_test<S>(t, g, r, x)) sink.add(xm | syz);
}

// The full voxel test at one voxel (the same arithmetic as row_prep +
// voxel_test, src/SVO.cu:156-177), without early exits.
template <bool S>
__device__ __forceinline__ bool voxel_pass(const Tri &t, const GridParams &g, int x, int y, int z) {
    const float px = __fmul_rn((float)x, g.unit[0]);
    const float py = __fmul_rn((float)y, g.unit[1]);
    const float pz = __fmul_rn((float)z, g.unit[2]);
    const float nd = Fp<S>::dot3_head(t.n[0], px, Fp<S>::dot3_tail(t.n[1], t.n[2], py, pz));
    bool ok = !(__fmul_rn(__fadd_rn(nd, t.d1), __fadd_rn(nd, t.d2)) > 0.0f);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        ok &= !(__fadd_rn(Fp<S>::dot2(t.ea[k], t.eb[k], px, py), t.ed[k]) < 0.0f);
        ok &= !(__fadd_rn(Fp<S>::dot2(t.ea[3 + k], t.eb[3 + k], py, pz), t.ed[3 + k]) < 0.0f);
        const float zx = Fp<S>::dot2_late(t.ea[6 + k], t.eb[6 + k], pz, px);
        ok &= !(__fadd_rn(zx, t.ed[6 + k]) < 0.0f);
    }
    return ok;
}

// True when no voxel of the box lo..hi (inclusive) can pass: one predicate
// fails at its most favourable corner (see the comment at the top).
template <bool S>
__device__ __forceinline__ bool brick_reject(const Tri &t, const GridParams &g, const int lo[3], const int hi[3]) {
    float pl[3], ph[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        pl[a] = __fmul_rn((float)lo[a], g.unit[a]);
        ph[a] = __fmul_rn((float)hi[a], g.unit[a]);
    }
#pragma unroll
    for (int p = 0; p < 3; ++p) {
        const int i = p == 0 ? 0 : (p == 1 ? 1 : 2);
        const int j = p == 0 ? 1 : (p == 1 ? 2 : 0);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float a = t.ea[3 * p + k], b = t.eb[3 * p + k];
            const float pi = a >= 0.0f ? ph[i] : pl[i];
            const float pj = b >= 0.0f ? ph[j] : pl[j];
            const float f = p == 2 ? Fp<S>::dot2_late(a, b, pi, pj) : Fp<S>::dot2(a, b, pi, pj);
            if (__fadd_rn(f, t.ed[3 * p + k]) < 0.0f) return true;
        }
    }
    // n.p at its smallest and largest corners
    const float x0 = t.n[0] >= 0.0f ? pl[0] : ph[0], x1 = t.n[0] >= 0.0f ? ph[0] : pl[0];
    const float y0 = t.n[1] >= 0.0f ? pl[1] : ph[1], y1 = t.n[1] >= 0.0f ? ph[1] : pl[1];
    const float z0 = t.n[2] >= 0.0f ? pl[2] : ph[2], z1 = t.n[2] >= 0.0f ? ph[2] : pl[2];
    const float nd0 = Fp<S>::dot3_head(t.n[0], x0, Fp<S>::dot3_tail(t.n[1], t.n[2], y0, z0));
    const float nd1 = Fp<S>::dot3_head(t.n[0], x1, Fp<S>::dot3_tail(t.n[1], t.n[2], y1, z1));
    const float dlo = t.d1 <= t.d2 ? t.d1 : t.d2, dhi = t.d1 <= t.d2 ? t.d2 : t.d1;
    {  // everything above the slab: both factors positive from the smallest n.p on
        const float sa = __fadd_rn(nd0, dlo), sb = __fadd_rn(nd0, dhi);
        if (sa > 0.0f && __fmul_rn(sa, sb) > 0.0f) return true;
    }
    {  // everything below: both factors negative up to the largest n.p
        const float sa = __fadd_rn(nd1, dlo), sb = __fadd_rn(nd1, dhi);
        if (sb < 0.0f && __fmul_rn(sa, sb) > 0.0f) return true;
    }
    return false;
}

// Two bricks per round, one per half-warp: lane r = lane & 15 of a half
// tests the 4 voxels of row (y, z) = (r & 3, r >> 2) of its half's brick,
// hoisted like the serial tier (row_prep: the YZ edge tests reject whole
// rows; then voxel_test per x -- the same arithmetic as voxel_pass).  The
// half's 64-bit hit mask (local Morton order) is OR-reduced over its 16 lanes
// and written with two atomicOr.  t, g, bm and the brick may differ between
// the halves; `on` is false for a half without a brick.  All 32 lanes call.
template <bool S>
__device__ __forceinline__ void brick_rows(const Tri &t, const GridParams &g, uint32_t *__restrict__ bm, int sx,
                                           int sy, int sz, bool on, int lane) {
    const int r = lane & 15, ly = r & 3, lz = r >> 2;
    const int y = 4 * sy + ly, z = 4 * sz + lz;
    uint64_t hits = 0;
    if (on && y >= t.lo[1] && y <= t.hi[1] && z >= t.lo[2] && z <= t.hi[2]) {
        Row rw;
        if (row_prep<S>(t, g, y, z, rw)) {
            const int x0 = max(4 * sx, t.lo[0]), x1 = min(4 * sx + 3, t.hi[0]);
            const int yz = ((ly & 1) << 1) | ((lz & 1) << 2) | ((ly >> 1) << 4) | ((lz >> 1) << 5);
            for (int x = x0; x <= x1; ++x) {
                const int lx = x - 4 * sx;
                if (voxel_test<S>(t, g, rw, x)) hits |= 1ull << (yz | (lx & 1) | ((lx >> 1) << 3));
            }
        }
    }
    uint32_t lo = (uint32_t)hits, hi = (uint32_t)(hits >> 32);
#pragma unroll
    for (int d = 8; d > 0; d >>= 1) {
        lo |= __shfl_xor_sync(0xFFFFFFFFu, lo, d);
        hi |= __shfl_xor_sync(0xFFFFFFFFu, hi, d);
    }
    if (on && r == 0) {
        uint32_t *w = bm + (morton3((uint32_t)sx, (uint32_t)sy, (uint32_t)sz) << 1);
        if (lo) atomicOr(w, lo);
        if (hi) atomicOr(w + 1, hi);
    }
}

// Brick j (row-major over the triangle's brick box) of triangle t: its brick
// coordinates, and whether it survives the culling test.
template <bool S>
__device__ __forceinline__ bool brick_live(const Tri &t, const GridParams &g, uint32_t j, int &bx, int &by, int &bz) {
    const int bx0 = t.lo[0] >> 2, by0 = t.lo[1] >> 2, bz0 = t.lo[2] >> 2;
    const uint32_t nbx = (uint32_t)((t.hi[0] >> 2) - bx0 + 1), nby = (uint32_t)((t.hi[1] >> 2) - by0 + 1);
    const uint32_t jy = j / nbx, jz = jy / nby;
    bx = bx0 + (int)(j - jy * nbx);
    by = by0 + (int)(jy - jz * nby);
    bz = bz0 + (int)jz;
    const int lo[3] = {max(4 * bx, t.lo[0]), max(4 * by, t.lo[1]), max(4 * bz, t.lo[2])};
    const int hi[3] = {min(4 * bx + 3, t.hi[0]), min(4 * by + 3, t.hi[1]), min(4 * bz + 3, t.hi[2])};
    return !t.cull || !brick_reject<S>(t, g, lo, hi);
}

// Bricks [b0, b1) of triangle t (the same t in every lane), chunks of 32
// bricks taken with stride `step` starting at b0 + first.  Three rounds, each
// with one item per lane: 32 bricks (4^3); the 8 sub-bricks (2^3) of 4
// surviving bricks; the 8 voxels of 4 surviving sub-bricks.  A 2^3 sub-brick
// is 8 consecutive Morton codes, one byte of a bitmap word.
template <bool S>
__device__ __forceinline__ void warp_bricks(const Tri &t, const GridParams &g, uint32_t *__restrict__ bm,
                                            uint32_t b0, uint32_t b1, uint32_t first, uint32_t step,
                                            bool split) {
    const int lane = threadIdx.x & 31, grp = lane >> 3, sub = lane & 7;
    for (uint32_t c = b0 + first; c < b1; c += step) {
        const uint32_t j = c + lane;
        int bx = 0, by = 0, bz = 0;
        const bool live = j < b1 && brick_live<S>(t, g, j, bx, by, bz);
        uint32_t m = __ballot_sync(0xFFFFFFFFu, live);
        while (m && !split) {
            // two surviving bricks at a time, one per half-warp
            const int sa = __ffs(m) - 1;
            m &= m - 1;
            const int sb = m ? __ffs(m) - 1 : -1;
            if (m) m &= m - 1;
            const bool on = (lane < 16) || sb >= 0;
            const int src = (lane < 16 || sb < 0) ? sa : sb;
            brick_rows<S>(t, g, bm, __shfl_sync(0xFFFFFFFFu, bx, src), __shfl_sync(0xFFFFFFFFu, by, src),
                          __shfl_sync(0xFFFFFFFFu, bz, src), on, lane);
        }
        while (m) {
            // up to 4 surviving bricks: lane = (brick, sub-brick)
            int src = 0;
            const int nsv = min(4, __popc(m));
            for (int i = 0; i < nsv; ++i) {
                const int s_ = __ffs(m) - 1;
                m &= m - 1;
                if (i == grp) src = s_;
            }
            const int sx = __shfl_sync(0xFFFFFFFFu, bx, src), sy = __shfl_sync(0xFFFFFFFFu, by, src),
                      sz = __shfl_sync(0xFFFFFFFFu, bz, src);
            const int x2 = 4 * sx + 2 * (sub & 1), y2 = 4 * sy + ((sub >> 1) & 1) * 2, z2 = 4 * sz + ((sub >> 2) & 1) * 2;
            bool slive = false;
            if (grp < nsv) {
                int lo[3] = {max(x2, t.lo[0]), max(y2, t.lo[1]), max(z2, t.lo[2])};
                int hi[3] = {min(x2 + 1, t.hi[0]), min(y2 + 1, t.hi[1]), min(z2 + 1, t.hi[2])};
                slive = lo[0] <= hi[0] && lo[1] <= hi[1] && lo[2] <= hi[2] && (!t.cull || !brick_reject<S>(t, g, lo, hi));
            }
            uint32_t m2 = __ballot_sync(0xFFFFFFFFu, slive);
            while (m2) {
                // up to 4 surviving sub-bricks: lane = (sub-brick, voxel)
                int src2 = 0;
                const int n2 = min(4, __popc(m2));
                for (int i = 0; i < n2; ++i) {
                    const int s_ = __ffs(m2) - 1;
                    m2 &= m2 - 1;
                    if (i == grp) src2 = s_;
                }
                const int vx = __shfl_sync(0xFFFFFFFFu, x2, src2), vy = __shfl_sync(0xFFFFFFFFu, y2, src2),
                          vz = __shfl_sync(0xFFFFFFFFu, z2, src2);
                const int x = vx + (sub & 1), y = vy + ((sub >> 1) & 1), z = vz + ((sub >> 2) & 1);
                const bool in = grp < n2 && x >= t.lo[0] && x <= t.hi[0] && y >= t.lo[1] && y <= t.hi[1] &&
                                z >= t.lo[2] && z <= t.hi[2];
                const uint32_t w = __ballot_sync(0xFFFFFFFFu, in && voxel_pass<S>(t, g, x, y, z));
                if (sub == 0 && grp < n2) {
                    const uint32_t bits = (w >> (8 * grp)) & 0xFFu;
                    if (bits) {
                        const uint64_t code = morton3((uint32_t)vx, (uint32_t)vy, (uint32_t)vz);
                        atomicOr(bm + (code >> 5), bits << (code & 31));
                    }
                }
            }
        }
    }
}

__device__ __forceinline__ uint32_t brick_count(const Tri &t) {
    return (uint32_t)((t.hi[0] >> 2) - (t.lo[0] >> 2) + 1) * (uint32_t)((t.hi[1] >> 2) - (t.lo[1] >> 2) + 1) *
           (uint32_t)((t.hi[2] >> 2) - (t.lo[2] >> 2) + 1);
}

// The vertices of an indexed triangle after checking its indices against the
// mesh's n_pts vertices; false (nothing read) when one is outside.  Soups are
// always in range.
__device__ __forceinline__ bool load_tri_checked(const float *__restrict__ pts, const int32_t *__restrict__ tris,
                                                 int64_t n_pts, int64_t t, float p[3][3]) {
    if (tris) {
        int64_t vi[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) vi[k] = __ldg(tris + 3 * t + k);
        if ((uint64_t)vi[0] >= (uint64_t)n_pts || (uint64_t)vi[1] >= (uint64_t)n_pts ||
            (uint64_t)vi[2] >= (uint64_t)n_pts)
            return false;
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int a = 0; a < 3; ++a) p[k][a] = __ldg(pts + 3 * vi[k] + a);
        return true;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int a = 0; a < 3; ++a) p[k][a] = __ldg(pts + 9 * t + 3 * k + a);
    return true;
}

// The same for a triangle that k_voxelize has already checked.
__device__ __forceinline__ void load_tri(const float *__restrict__ pts, const int32_t *__restrict__ tris,
                                         int64_t t, float p[3][3]) {
    if (tris) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int64_t vi = __ldg(tris + 3 * t + k);
#pragma unroll
            for (int a = 0; a < 3; ++a) p[k][a] = __ldg(pts + 3 * vi + a);
        }
    } else {
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int a = 0; a < 3; ++a) p[k][a] = __ldg(pts + 9 * t + 3 * k + a);
    }
}

// The bricks of the warp's in-warp triangles (lane i's triangle st[i] when
// it has cnt > 0 bricks), packed across triangles: rounds of 32 (triangle,
// brick) items, each lane culling one brick of its item's triangle (read from
// shared memory: the 39-word stride is odd, so distinct triangles fall in
// distinct banks); the surviving bricks are then tested one at a time by the
// whole warp, the current triangle held in registers.
template <bool S>
__device__ __forceinline__ void warp_packed(const BatchDev &bd, const Tri *st, int m, uint32_t cnt, int lane) {
    uint32_t incl = cnt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
        if (lane >= d) incl += y;
    }
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    const uint32_t excl = incl - cnt;
    int cur = -1;  // lane whose triangle is held in ct
    Tri ct;
    GridParams cg;
    uint32_t *cbm = nullptr;
    for (uint32_t base = 0; base < total; base += 32) {
        const uint32_t item = base + lane;
        // owner lane: the number of lanes whose inclusive count is <= item
        int pos = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
            const uint32_t v = __shfl_sync(0xFFFFFFFFu, incl, pos + step - 1);
            if (v <= item) pos += step;
        }
        const bool valid = item < total;
        const int src = valid ? pos : 0;
        const int wm = __shfl_sync(0xFFFFFFFFu, m, src);
        const uint32_t j = item - __shfl_sync(0xFFFFFFFFu, excl, src);
        int bx = 0, by = 0, bz = 0;
        bool live = false;
        if (valid) {
            const GridParams g = *bd.mesh[wm].gp;
            live = brick_live<S>(st[src], g, j, bx, by, bz);
        }
        uint32_t lm = __ballot_sync(0xFFFFFFFFu, live);
        while (lm) {
            // two surviving bricks at a time, one per half-warp, each with its own triangle
            const int sa = __ffs(lm) - 1;
            lm &= lm - 1;
            const int sb = lm ? __ffs(lm) - 1 : -1;
            if (lm) lm &= lm - 1;
            const bool on = (lane < 16) || sb >= 0;
            const int s = (lane < 16 || sb < 0) ? sa : sb;
            const int own = __shfl_sync(0xFFFFFFFFu, src, s);
            const int mm = __shfl_sync(0xFFFFFFFFu, m, own);
            if (own != cur) {
                cur = own;
                ct = st[own];
                cg = *bd.mesh[mm].gp;
                cbm = reinterpret_cast<uint32_t *>(bd.mesh[mm].bits);
            }
            brick_rows<S>(ct, cg, cbm, __shfl_sync(0xFFFFFFFFu, bx, s), __shfl_sync(0xFFFFFFFFu, by, s),
                          __shfl_sync(0xFFFFFFFFu, bz, s), on, lane);
        }
    }
}

// The rows (y, z) of the warp's serial-tier triangles (lane i's triangle
// st[i], mesh sm[i], with nrows > 0 rows along x), packed 32 per round: each
// lane takes one row, copies its triangle's setup from shared memory and
// tests the row along x with the serial arithmetic (row_prep: YZ tests
// reject the whole row; voxel_test per x), so lanes stay busy whatever the
// triangles' shapes.
template <bool S>
__device__ __forceinline__ void warp_rows(const BatchDev &bd, const Tri *st, const int *sm, uint32_t nrows,
                                          int lane) {
    uint32_t incl = nrows;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
        if (lane >= d) incl += y;
    }
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    const uint32_t excl = incl - nrows;
    for (uint32_t base = 0; base < total; base += 32) {
        const uint32_t item = base + lane;
        int pos = 0;  // owner lane: the number of lanes whose inclusive count is <= item
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
            const uint32_t v = __shfl_sync(0xFFFFFFFFu, incl, pos + step - 1);
            if (v <= item) pos += step;
        }
        const int src = item < total ? pos : 0;
        const uint32_t j = item - __shfl_sync(0xFFFFFFFFu, excl, src);
        if (item < total) {
            const Tri &t = st[src];
            const int mm = sm[src];
            const GridParams g = *bd.mesh[mm].gp;
            const uint32_t ny = (uint32_t)(t.hi[1] - t.lo[1] + 1);
            HitSink sink{reinterpret_cast<uint32_t *>(bd.mesh[mm].bits)};
            const int y = t.lo[1] + (int)(j % ny), z = t.lo[2] + (int)(j / ny);
            row_segment<S>(t, g, y, z, spread3((uint32_t)y) << 1 | spread3((uint32_t)z) << 2, t.lo[0], t.hi[0], sink);
            sink.flush();
        }
    }
}

// One thread per triangle of the batch (global index -> mesh by tri_off):
// setup, then
//   tier 0 (grid bbox <= serial_max voxels): the serial row-by-row test, by
//     this thread (serial_packed 0) or packed one row per lane (ROWS);
//   tier 1 (<= inplace_max 4^3 bricks, or any size when INPLACE): with a
//     small-triangle list, its index is appended there for
//     k_voxelize_small; INPLACE (no list or queue), its bricks are walked by
//     this warp right away (warp_packed);
//   tier 2 (more bricks): queue entries of <= warp_max bricks for
//     k_voxelize_bricks, which balances them across the GPU.
template <bool S, bool INPLACE, bool ROWS>
__global__ void __launch_bounds__(256, INPLACE ? 2 : 3)
    k_voxelize(BatchDev bd, int64_t total, VoxTuning tune, uint4 *__restrict__ big, uint32_t big_cap,
               uint32_t *__restrict__ big_count, uint64_t *__restrict__ small, uint32_t *__restrict__ small_count) {
    __shared__ Tri s_tri[8][32];  // the warp's serial-tier triangles, then (INPLACE) its tier-1 ones
    __shared__ int s_mesh[8][32];  // their meshes
    const int lane = threadIdx.x & 31;
    Tri *st = s_tri[threadIdx.x >> 5];
    int *sm = s_mesh[threadIdx.x >> 5];
    const int64_t warp0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) - lane;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = warp0; base < total; base += stride) {
        const int64_t gid = base + lane;
        Tri t;
        uint32_t nb = 0;
        int tier = -1, m = 0;
        if (gid < total) {
            m = find_segment(bd.tri_off, bd.n, (uint64_t)gid);
            const MeshDev &md = bd.mesh[m];
            const GridParams g = *md.gp;
            float p[3][3];
            if (load_tri_checked(md.pts, md.tris, md.n_pts, gid - (int64_t)bd.tri_off[m], p)) {
                tri_setup<S>(g, md.res, p[0], p[1], p[2], t);
                const uint64_t vol = (uint64_t)(t.hi[0] - t.lo[0] + 1) * (uint64_t)(t.hi[1] - t.lo[1] + 1) *
                                     (uint64_t)(t.hi[2] - t.lo[2] + 1);
                nb = brick_count(t);
                tier = vol <= (uint64_t)tune.serial_max ? 0 : (INPLACE || nb <= tune.inplace_max) ? 1 : 2;
            } else {
                atomicOr(&md.gp->status, kStatusBadIndex);  // tier stays -1: the triangle is skipped
            }
            if (tier == 2) {
                const uint32_t eb = tune.warp_max;
                const uint32_t ne = (nb + eb - 1) / eb;
                const uint32_t at = atomicAdd(big_count, ne);
                if (at + ne <= big_cap) {
                    for (uint32_t e = 0; e < ne; ++e)
                        big[at + e] = make_uint4((uint32_t)gid, e * eb, min(nb, (e + 1) * eb), (uint32_t)(gid >> 32));
                }
            }
        }
        if (ROWS) {  // the warp's serial-tier rows, packed across lanes
            if (__any_sync(0xFFFFFFFFu, tier == 0)) {
                const uint32_t nrows =
                    tier == 0 ? (uint32_t)(t.hi[1] - t.lo[1] + 1) * (uint32_t)(t.hi[2] - t.lo[2] + 1) : 0u;
                if (tier == 0) {
                    st[lane] = t;
                    sm[lane] = m;
                }
                __syncwarp();
                warp_rows<S>(bd, st, sm, nrows, lane);
                __syncwarp();  // st is rewritten below or by the next round
            }
        } else if (tier == 0) {  // each lane walks its own triangle's rows
            const MeshDev &md = bd.mesh[m];
            const GridParams g = *md.gp;
            HitSink sink{reinterpret_cast<uint32_t *>(md.bits)};
            const uint64_t ym0 = spread3((uint32_t)t.lo[1]) << 1;
            uint64_t zm = spread3((uint32_t)t.lo[2]) << 2;
            for (int z = t.lo[2]; z <= t.hi[2]; ++z, zm = dil_inc(zm, kDilZ)) {
                uint64_t ym = ym0;
                for (int y = t.lo[1]; y <= t.hi[1]; ++y, ym = dil_inc(ym, kDilY))
                    row_segment<S>(t, g, y, z, ym | zm, t.lo[0], t.hi[0], sink);
            }
            sink.flush();
        }
        if (INPLACE) {
            if (__any_sync(0xFFFFFFFFu, tier == 1)) {
                if (tier == 1) st[lane] = t;
                __syncwarp();
                warp_packed<S>(bd, st, m, tier == 1 ? nb : 0u, lane);
                __syncwarp();  // st is rewritten by the next round
            }
        } else {
            // warp-aggregated append to the small-triangle list (room for every triangle)
            const uint32_t mask = __ballot_sync(0xFFFFFFFFu, tier == 1);
            if (mask) {
                uint32_t at = 0;
                if (lane == __ffs(mask) - 1) at = atomicAdd(small_count, (uint32_t)__popc(mask));
                at = __shfl_sync(0xFFFFFFFFu, at, __ffs(mask) - 1);
                if (tier == 1) small[at + __popc(mask & ((1u << lane) - 1u))] = (uint64_t)gid;
            }
        }
    }
}

// The small-triangle list: each lane sets up one listed triangle (32
// different triangles per warp), stages it in shared memory, and the warp
// walks their bricks packed 32 per round (warp_packed).
template <bool S>
__global__ void __launch_bounds__(256, 2) k_voxelize_small(BatchDev bd, const uint64_t *__restrict__ small,
                                                           const uint32_t *__restrict__ small_count) {
    __shared__ Tri s_tri[8][32];
    const int lane = threadIdx.x & 31;
    Tri *st = s_tri[threadIdx.x >> 5];
    const uint32_t n = *small_count;
    const uint64_t warp0 = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) - lane;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = warp0; base < n; base += stride) {
        const uint64_t i = base + lane;
        uint32_t nb = 0;
        int m = 0;
        if (i < n) {
            const uint64_t gid = small[i];
            m = find_segment(bd.tri_off, bd.n, gid);
            const MeshDev &md = bd.mesh[m];
            const GridParams g = *md.gp;
            float p[3][3];
            load_tri(md.pts, md.tris, (int64_t)(gid - bd.tri_off[m]), p);
            Tri t;
            tri_setup<S>(g, md.res, p[0], p[1], p[2], t);
            nb = brick_count(t);
            st[lane] = t;
        }
        __syncwarp();
        warp_packed<S>(bd, st, m, nb, lane);
        __syncwarp();
    }
}

// Queued triangles: each warp takes an entry (triangle, brick range) and
// walks its bricks.
template <bool S>
__global__ void __launch_bounds__(256, 3) k_voxelize_bricks(BatchDev bd, const uint4 *__restrict__ big,
                                                            const uint32_t *__restrict__ big_count,
                                                            uint32_t big_cap, uint32_t *__restrict__ cursor,
                                                            bool split) {
    const int lane = threadIdx.x & 31;
    const uint32_t n = *big_count;
    if (n > big_cap) return;  // reported by the host; the build is retried
    for (;;) {
        uint32_t e = 0;
        if (lane == 0) e = atomicAdd(cursor, 1u);
        e = __shfl_sync(0xFFFFFFFFu, e, 0);
        if (e >= n) return;
        const uint4 ent = big[e];
        const int64_t gid = (int64_t)ent.x | ((int64_t)ent.w << 32);
        const int m = find_segment(bd.tri_off, bd.n, (uint64_t)gid);
        const MeshDev &md = bd.mesh[m];
        const GridParams g = *md.gp;
        float p[3][3];
        load_tri(md.pts, md.tris, gid - (int64_t)bd.tri_off[m], p);
        Tri t;
        tri_setup<S>(g, md.res, p[0], p[1], p[2], t);
        warp_bricks<S>(t, g, reinterpret_cast<uint32_t *>(md.bits), ent.y, ent.z, 0, 32, split);
    }
}

__global__ void k_index_init(int32_t *mm) {
    mm[0] = 0x7FFFFFFF;
    mm[1] = (int32_t)0x80000000;
}

__global__ void k_index_range(const int32_t *__restrict__ idx, int64_t n, int32_t *__restrict__ mm) {
    int32_t lo = 0x7FFFFFFF, hi = (int32_t)0x80000000;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = __ldg(idx + i);
        lo = min(lo, v);
        hi = max(hi, v);
    }
    lo = __reduce_min_sync(0xFFFFFFFFu, lo);
    hi = __reduce_max_sync(0xFFFFFFFFu, hi);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(mm, lo);
        atomicMax(mm + 1, hi);
    }
}

// Min/max index of each job of a table (jobs whose blocks follow block_off).
__global__ void k_index_ranges_init(int32_t *mm, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        mm[2 * i] = 0x7FFFFFFF;
        mm[2 * i + 1] = (int32_t)0x80000000;
    }
}

__global__ void k_index_ranges(const IndexJob *__restrict__ jobs, int n, const uint32_t *__restrict__ block_off,
                               int32_t *__restrict__ mm) {
    const int k = find_segment(block_off, n, (uint32_t)blockIdx.x);
    const IndexJob jb = jobs[k];
    const int64_t nb = block_off[k + 1] - block_off[k];
    int32_t lo = 0x7FFFFFFF, hi = (int32_t)0x80000000;
    for (int64_t i = (blockIdx.x - block_off[k]) * (int64_t)blockDim.x + threadIdx.x; i < jb.n;
         i += nb * blockDim.x) {
        const int32_t v = __ldg(jb.idx + i);
        lo = min(lo, v);
        hi = max(hi, v);
    }
    lo = __reduce_min_sync(0xFFFFFFFFu, lo);
    hi = __reduce_max_sync(0xFFFFFFFFu, hi);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(mm + 2 * k, lo);
        atomicMax(mm + 2 * k + 1, hi);
    }
}

}  // namespace

cudaError_t launch_index_range(const int32_t *idx, int64_t n, int32_t *mm, cudaStream_t st) {
    k_index_init<<<1, 1, 0, st>>>(mm);
    count_launches(1);
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8));
    k_index_range<<<blocks, 256, 0, st>>>(idx, n, mm);
    count_launches(1);
    return cudaGetLastError();
}

uint32_t index_blocks(int64_t n) { return (uint32_t)std::max<int64_t>(1, std::min<int64_t>((n + 2047) / 2048, 2048)); }

cudaError_t launch_index_ranges(const IndexJob *jobs, int n, const uint32_t *block_off, uint32_t total_blocks,
                                int32_t *mm, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_index_ranges_init<<<(n + 127) / 128, 128, 0, st>>>(mm, n);
    k_index_ranges<<<total_blocks, 256, 0, st>>>(jobs, n, block_off, mm);
    count_launches(2);
    return cudaGetLastError();
}

cudaError_t launch_bbox(const BatchDev &b, uint32_t total_blocks, cudaStream_t st) {
    k_bbox_reduce<<<total_blocks, 256, 0, st>>>(b);
    k_grid_setup<<<(b.n + 127) / 128, 128, 0, st>>>(b);
    count_launches(2);
    return cudaGetLastError();
}

namespace {

// Flags the level-0 regions (Morton code >> 17: x >> 6, y >> 6, z >> 5) that
// each triangle's voxel bbox overlaps, for region-mode meshes.  The bbox is
// tri_box's widened by one voxel on each side, with a product by the
// reciprocal voxel size in place of the division: the two differ by a few
// ulps at coordinates <= 2048, far less than the margin, so the flagged
// regions cover every voxel the voxel test can set.
// Bits of v (< 2^10) spread to every third bit.
__device__ __forceinline__ uint32_t spread3_small(uint32_t v) {
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    return (v | (v << 2)) & 0x09249249u;
}

// The flags of the level-0 regions (64 x 64 x 32 voxels, region index =
// morton3(x, y, z) >> 17) each triangle's voxel box (with a one-voxel margin)
// reaches.  The kernel waits on gathers (indices, then vertices), so each
// thread takes 3 triangles at a time and issues all their loads before using
// them; the mesh's grid and reciprocal units are kept while the mesh stays
// the same.
constexpr int kMarkBatch = 3;

__global__ void __launch_bounds__(256) k_region_mark(BatchDev bd, int64_t total) {
    int cur = -1;
    float org[3] = {0, 0, 0}, inv[3] = {0, 0, 0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t g0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g0 < total; g0 += stride * kMarkBatch) {
        int mk[kMarkBatch];
        bool live[kMarkBatch];
        int64_t vi[kMarkBatch][3];
#pragma unroll
        for (int k = 0; k < kMarkBatch; ++k) {
            const int64_t gid = g0 + k * stride;
            live[k] = gid < total;
            mk[k] = live[k] ? find_segment(bd.tri_off, bd.n, (uint64_t)gid) : 0;
            const MeshDev &md = bd.mesh[mk[k]];
            live[k] = live[k] && md.regions != 0;
            const int64_t t = gid - (int64_t)bd.tri_off[mk[k]];
#pragma unroll
            for (int j = 0; j < 3; ++j) vi[k][j] = live[k] ? (md.tris ? (int64_t)__ldg(md.tris + 3 * t + j) : 3 * t + j) : 0;
        }
        float p[kMarkBatch][3][3];
#pragma unroll
        for (int k = 0; k < kMarkBatch; ++k) {
            const MeshDev &md = bd.mesh[mk[k]];
            // an index outside the mesh: skipped here, k_voxelize reports it
            live[k] = live[k] && (uint64_t)vi[k][0] < (uint64_t)md.n_pts && (uint64_t)vi[k][1] < (uint64_t)md.n_pts &&
                      (uint64_t)vi[k][2] < (uint64_t)md.n_pts;
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int a = 0; a < 3; ++a) p[k][j][a] = live[k] ? __ldg(md.pts + 3 * vi[k][j] + a) : 0.0f;
        }
#pragma unroll
        for (int k = 0; k < kMarkBatch; ++k) {
            if (!live[k]) continue;
            const MeshDev &md = bd.mesh[mk[k]];
            if (mk[k] != cur) {
                cur = mk[k];
                // the one-voxel margin absorbs an approximate reciprocal (2 ulp)
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    org[a] = md.gp->origin[a];
                    inv[a] = __fdividef(1.0f, md.gp->unit[a]);
                }
            }
            int lo[3], hi[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const float v0 = __fsub_rn(p[k][0][a], org[a]), v1 = __fsub_rn(p[k][1][a], org[a]),
                            v2 = __fsub_rn(p[k][2][a], org[a]);
                // the margin is applied before the conversion, so +-inf and NaN clamp as in tri_box
                lo[a] = clampi(f2i_rz(__fsub_rn(__fmul_rn(cminf(v0, cminf(v1, v2)), inv[a]), 1.0f)), 0, md.res[a] - 1);
                hi[a] = clampi(f2i_rz(__fadd_rn(__fmul_rn(cmaxf(v0, cmaxf(v1, v2)), inv[a]), 1.0f)), 0, md.res[a] - 1);
            }
            uint8_t *flag = bd.rflag + bd.cta_off[mk[k]];
            // region bits: z at 3i, x at 3i + 1, y at 3i + 2 (z in 32-voxel, x and y in 64-voxel steps)
            for (uint32_t rz = (uint32_t)lo[2] >> 5; rz <= (uint32_t)hi[2] >> 5; ++rz)
                for (uint32_t ry = (uint32_t)lo[1] >> 6; ry <= (uint32_t)hi[1] >> 6; ++ry)
                    for (uint32_t rx = (uint32_t)lo[0] >> 6; rx <= (uint32_t)hi[0] >> 6; ++rx) {
                        uint8_t *f = flag + (spread3_small(rz) | spread3_small(rx) << 1 | spread3_small(ry) << 2);
                        if (!*f) *f = 1;
                    }
        }
    }
}

// Level-0 regions, a persistent grid taking them in turn: zeroes each unless
// it is a region-mode mesh's unflagged region.  The pyramid writes every word of levels 1 and 2 and the
// first 4 * ctas of level 3; the words after those (level-3 padding, level 4,
// which the pyramid writes as 32-bit halves, and levels >= 5) are zeroed
// here, spread over the mesh's CTAs.
__global__ void __launch_bounds__(256) k_region_zero(BatchDev bd, uint32_t total) {
    for (uint32_t g = blockIdx.x; g < total; g += gridDim.x) {
        const int m = find_segment(bd.cta_off, bd.n, g);
        const MeshDev &md = bd.mesh[m];
        const uint32_t r = g - bd.cta_off[m];
        if (!md.regions || bd.rflag[g]) {
            uint4 *w = reinterpret_cast<uint4 *>(md.bits + md.py.woff[0] + (uint64_t)r * 2048);
#pragma unroll
            for (int q = 0; q < 4; ++q) w[threadIdx.x + 256 * q] = make_uint4(0, 0, 0, 0);
        }
        const uint64_t z0 = md.py.woff[3] + 4ull * md.py.ctas;
        for (uint64_t i = z0 + (uint64_t)r * 256 + threadIdx.x; i < md.py.total_words; i += (uint64_t)md.py.ctas * 256)
            md.bits[i] = 0;
    }
}

}  // namespace

cudaError_t launch_regions(const BatchDev &b, int64_t total_tris, uint32_t total_ctas, int num_sms,
                           cudaStream_t st) {
    if (total_tris > 0) {
        const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((total_tris + 255) / 256, (int64_t)num_sms * 8));
        k_region_mark<<<blocks, 256, 0, st>>>(b, total_tris);
        count_launches(1);
    }
    if (total_ctas > 0) {
        k_region_zero<<<std::min<uint32_t>(total_ctas, (uint32_t)num_sms * 8), 256, 0, st>>>(b, total_ctas);
        count_launches(1);
    }
    return cudaGetLastError();
}

cudaError_t launch_voxelize(const BatchDev &b, int64_t total, bool strict, const VoxTuning &tune, uint4 *big,
                            uint32_t big_cap, uint32_t *counters, int num_sms, cudaStream_t st, uint64_t *small) {
    // counters[0] = queue entries, counters[1] = queue cursor, counters[3] = small-list length
    cudaError_t e = cudaMemsetAsync(counters, 0, 2 * sizeof(uint32_t), st);
    if (e == cudaSuccess && small) e = cudaMemsetAsync(counters + 3, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    if (total > 0) {
        const int64_t want = (total + 255) / 256;
        const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)num_sms * 16));
        const bool inplace = big == nullptr || big_cap == 0;
        // Few triangles, or no small-triangle list: the queue spreads the bricks over all SMs.
        VoxTuning tn = tune;
        if (!inplace && (total < (int64_t)num_sms * 256 || !small)) tn.inplace_max = 0;
        uint32_t *small_count = counters + 3;
#define SVO_VOX(S_, I_, R_) \
    k_voxelize<S_, I_, R_><<<blocks, 256, 0, st>>>(b, total, tn, big, big_cap, counters, small, small_count)
#define SVO_VOX2(S_, I_) \
    do {                   \
        if (tn.serial_packed) SVO_VOX(S_, I_, true); \
        else SVO_VOX(S_, I_, false);                 \
    } while (0)
        if (strict) {
            if (inplace) SVO_VOX2(true, true); else SVO_VOX2(true, false);
        } else {
            if (inplace) SVO_VOX2(false, true); else SVO_VOX2(false, false);
        }
#undef SVO_VOX2
#undef SVO_VOX
        count_launches(1);
        if (!inplace) {
            if (tn.inplace_max > 0) {
                const int sblocks = num_sms * 2;
                if (strict) k_voxelize_small<true><<<sblocks, 256, 0, st>>>(b, small, small_count);
                else k_voxelize_small<false><<<sblocks, 256, 0, st>>>(b, small, small_count);
                count_launches(1);
            }
            const int bblocks = num_sms * 4;
            if (strict)
                k_voxelize_bricks<true><<<bblocks, 256, 0, st>>>(b, big, counters, big_cap, counters + 1,
                                                                tune.split != 0);
            else
                k_voxelize_bricks<false><<<bblocks, 256, 0, st>>>(b, big, counters, big_cap, counters + 1,
                                                                 tune.split != 0);
            count_launches(1);
        }
    }
    return cudaGetLastError();
}

}  // namespace svo
