// svo_voxelize.cu -- bounding cube and conservative surface voxelization.
//
// Restates the reference's BaseModel bounding cube (src/BaseModel.h:24-49,
// 64-73) and surfaceVoxelize (src/SVO.cu:37-188) for sm_100a.  Instead of one
// thread per triangle writing a dense u32 array of res^3 entries, each overlap
// sets one bit of a Morton-ordered occupancy bitmap (res^3 bits); the test
// arithmetic is the reference's, operation for operation (svo_device.cuh Fp).
//
// Work split: a triangle whose grid bbox has at most `serial_max` voxels is
// tested by its own thread; up to `warp_max` voxels by its warp (row segments
// spread over the lanes); larger ones are cut into entries of at most
// kEntryItems row segments that whole CTAs take from a queue.
#include "svo_internal.h"

namespace svo {

namespace {

constexpr int kSeg = 16;            // voxels per row segment (one work item)
constexpr uint32_t kEntryItems = 2048;  // row segments per big-triangle entry

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
__global__ void k_bbox_reduce(const float *__restrict__ pts, int64_t n, uint32_t *__restrict__ mm,
                              GridParams *__restrict__ gp) {
    uint32_t lo[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, hi[3] = {0u, 0u, 0u};
    bool bad = false;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            float v = __ldg(pts + 3 * i + a);
            bad |= !isfinite(v);
            uint32_t o = f2ord(v);
            lo[a] = min(lo[a], o);
            hi[a] = max(hi[a], o);
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        lo[a] = __reduce_min_sync(0xFFFFFFFFu, lo[a]);
        hi[a] = __reduce_max_sync(0xFFFFFFFFu, hi[a]);
    }
    if (__any_sync(0xFFFFFFFFu, bad) && (threadIdx.x & 31) == 0) atomicOr(&gp->status, kStatusNonFinite);
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            atomicMin(mm + a, lo[a]);
            atomicMax(mm + 3 + a, hi[a]);
        }
    }
}

// createMeshBBCube (src/BaseModel.h:24-49) and unitVoxelSize
// (src/SVO.cu:348-350).  Host code in the reference: no contraction there, so
// every operation is an explicitly rounded intrinsic.
__global__ void k_grid_setup(const uint32_t *__restrict__ mm, int rx, int ry, int rz,
                             GridParams *__restrict__ gp) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
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
};

__device__ __forceinline__ int f2i_rz(float f) { return __float2int_rz(f); }
__device__ __forceinline__ int clampi(int f, int a, int b) { return max(a, min(f, b)); }

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
    const float sq = Fp<S>::dot3(c0, c1, c2, c0, c1, c2);
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
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float mn = cminf(v[0][a], cminf(v[1][a], v[2][a]));
        const float mx = cmaxf(v[0][a], cmaxf(v[1][a], v[2][a]));
        t.lo[a] = clampi(f2i_rz(__fdiv_rn(mn, u[a])), 0, res[a] - 1);
        t.hi[a] = clampi(f2i_rz(__fdiv_rn(mx, u[a])), 0, res[a] - 1);
    }
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
}

// Per-row state: everything of the voxel test that depends only on (y, z).
struct Row {
    float inner;      // tail of n.dot(p)
    float xyb[3];     // XY: b * p.y
    float zxp[3];     // ZX: a * p.z (strict) or p.z (fused)
    uint64_t syz;     // Morton bits of y and z
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
        r.zxp[k] = S ? __fmul_rn(t.ea[6 + k], pz) : pz;
    }
    r.syz = (spread3((uint32_t)y) << 1) | (spread3((uint32_t)z) << 2);
    return true;
}

template <bool S>
__device__ __forceinline__ bool voxel_test(const Tri &t, const GridParams &g, const Row &r, int x) {
    const float px = __fmul_rn((float)x, g.unit[0]);
    const float nd = Fp<S>::dot3_head(t.n[0], px, r.inner);
    if (__fmul_rn(__fadd_rn(nd, t.d1), __fadd_rn(nd, t.d2)) > 0.0f) return false;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float f = S ? __fadd_rn(__fmul_rn(t.ea[k], px), r.xyb[k]) : __fmaf_rn(t.ea[k], px, r.xyb[k]);
        if (__fadd_rn(f, t.ed[k]) < 0.0f) return false;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float q = __fmul_rn(t.eb[6 + k], px);
        const float f = S ? __fadd_rn(r.zxp[k], q) : __fmaf_rn(t.ea[6 + k], r.zxp[k], q);
        if (__fadd_rn(f, t.ed[6 + k]) < 0.0f) return false;
    }
    return true;
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

// Tests voxels x in [x0, x1] of row (y, z).
template <bool S>
__device__ __forceinline__ void row_segment(const Tri &t, const GridParams &g, int y, int z, int x0,
                                            int x1, HitSink &sink) {
    Row r;
    if (!row_prep<S>(t, g, y, z, r)) return;
    for (int x = x0; x <= x1; ++x)
        if (voxel_test<S>(t, g, r, x)) sink.add(spread3((uint32_t)x) | r.syz);
}

// Work item i of a triangle: row segment (y, z, x0..x1).
__device__ __forceinline__ void item_coords(const Tri &t, uint32_t segs, uint32_t ny, uint32_t i, int &y,
                                            int &z, int &x0, int &x1) {
    const uint32_t row = i / segs, s = i - row * segs;
    const uint32_t zr = row / ny;
    y = t.lo[1] + (int)(row - zr * ny);
    z = t.lo[2] + (int)zr;
    x0 = t.lo[0] + (int)s * kSeg;
    x1 = min(x0 + kSeg - 1, t.hi[0]);
}

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

__device__ __forceinline__ void shfl_tri(Tri &dst, const Tri &src, int lane) {
    const float *s = reinterpret_cast<const float *>(&src);
    float *d = reinterpret_cast<float *>(&dst);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(Tri) / 4); ++i) d[i] = __shfl_sync(0xFFFFFFFFu, s[i], lane);
}

template <bool S>
__global__ void __launch_bounds__(256) k_voxelize(const float *__restrict__ pts,
                                                  const int32_t *__restrict__ tris, int64_t nt,
                                                  const GridParams *__restrict__ gpp, int rx, int ry,
                                                  int rz, uint32_t *__restrict__ bm, VoxTuning tune,
                                                  uint4 *__restrict__ big, uint32_t big_cap,
                                                  uint32_t *__restrict__ big_count) {
    const GridParams g = *gpp;
    const int res[3] = {rx, ry, rz};
    const int lane = threadIdx.x & 31;
    const int64_t warp0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) - lane;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    HitSink sink{bm};
    for (int64_t base = warp0; base < nt; base += stride) {
        const int64_t tid = base + lane;
        Tri t;
        uint32_t items = 0;
        uint64_t vol = 0;
        int tier = -1;
        if (tid < nt) {
            float p[3][3];
            load_tri(pts, tris, tid, p);
            tri_setup<S>(g, res, p[0], p[1], p[2], t);
            const uint32_t nx = t.hi[0] - t.lo[0] + 1, ny = t.hi[1] - t.lo[1] + 1, nz = t.hi[2] - t.lo[2] + 1;
            vol = (uint64_t)nx * ny * nz;
            items = ((nx + kSeg - 1) / kSeg) * ny * nz;
            tier = vol <= (uint64_t)tune.serial_max ? 0 : (vol <= (uint64_t)tune.warp_max ? 1 : 2);
        }
        if (tier == 0) {
            for (int z = t.lo[2]; z <= t.hi[2]; ++z)
                for (int y = t.lo[1]; y <= t.hi[1]; ++y) row_segment<S>(t, g, y, z, t.lo[0], t.hi[0], sink);
            sink.flush();
        } else if (tier == 2) {
            const uint32_t ne = (items + kEntryItems - 1) / kEntryItems;
            const uint32_t at = atomicAdd(big_count, ne);
            if (at + ne <= big_cap) {
                for (uint32_t e = 0; e < ne; ++e)
                    big[at + e] = make_uint4((uint32_t)tid, e * kEntryItems, min(items, (e + 1) * kEntryItems), 0);
            }
        }
        // warp-cooperative triangles, one at a time
        uint32_t coop = __ballot_sync(0xFFFFFFFFu, tier == 1);
        while (coop) {
            const int src = __ffs(coop) - 1;
            coop &= coop - 1;
            Tri w;
            shfl_tri(w, t, src);
            const uint32_t witems = __shfl_sync(0xFFFFFFFFu, items, src);
            const uint32_t segs = (w.hi[0] - w.lo[0] + 1 + kSeg - 1) / kSeg;
            const uint32_t wny = w.hi[1] - w.lo[1] + 1;
            for (uint32_t i = lane; i < witems; i += 32) {
                int y, z, x0, x1;
                item_coords(w, segs, wny, i, y, z, x0, x1);
                row_segment<S>(w, g, y, z, x0, x1, sink);
                sink.flush();
            }
        }
    }
}

// Big triangles: CTAs take entries (triangle, range of row segments) from a
// queue and spread the segments over their threads.
template <bool S>
__global__ void __launch_bounds__(256) k_voxelize_big(const float *__restrict__ pts,
                                                      const int32_t *__restrict__ tris,
                                                      const GridParams *__restrict__ gpp, int rx,
                                                      int ry, int rz, uint32_t *__restrict__ bm,
                                                      const uint4 *__restrict__ big,
                                                      const uint32_t *__restrict__ big_count,
                                                      uint32_t big_cap, uint32_t *__restrict__ cursor) {
    __shared__ uint32_t s_e;
    const GridParams g = *gpp;
    const int res[3] = {rx, ry, rz};
    const uint32_t n = min(*big_count, big_cap);
    if (*big_count > big_cap) return;  // reported by the host; the build is retried
    HitSink sink{bm};
    for (;;) {
        if (threadIdx.x == 0) s_e = atomicAdd(cursor, 1u);
        __syncthreads();
        const uint32_t e = s_e;
        __syncthreads();
        if (e >= n) return;
        const uint4 ent = big[e];
        float p[3][3];
        load_tri(pts, tris, ent.x, p);
        Tri t;
        tri_setup<S>(g, res, p[0], p[1], p[2], t);
        const uint32_t segs = (t.hi[0] - t.lo[0] + 1 + kSeg - 1) / kSeg;
        const uint32_t ny = t.hi[1] - t.lo[1] + 1;
        for (uint32_t i = ent.y + threadIdx.x; i < ent.z; i += blockDim.x) {
            int y, z, x0, x1;
            item_coords(t, segs, ny, i, y, z, x0, x1);
            row_segment<S>(t, g, y, z, x0, x1, sink);
            sink.flush();
        }
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

}  // namespace

cudaError_t launch_index_range(const int32_t *idx, int64_t n, int32_t *mm, cudaStream_t st) {
    k_index_init<<<1, 1, 0, st>>>(mm);
    count_launches(1);
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8));
    k_index_range<<<blocks, 256, 0, st>>>(idx, n, mm);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_bbox(const float *pts, int64_t n, int rx, int ry, int rz, uint32_t *mm_scratch,
                        GridParams *gp, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(mm_scratch, 0xFF, 3 * sizeof(uint32_t), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(mm_scratch + 3, 0, 3 * sizeof(uint32_t), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(gp, 0, sizeof(GridParams), st);
    if (e != cudaSuccess) return e;
    int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
    blocks = std::max(blocks, 1);
    k_bbox_reduce<<<blocks, 256, 0, st>>>(pts, n, mm_scratch, gp);
    count_launches(1);
    k_grid_setup<<<1, 32, 0, st>>>(mm_scratch, rx, ry, rz, gp);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_voxelize(const float *pts, const int32_t *tris, int64_t nt, const GridParams *gp,
                            int rx, int ry, int rz, bool strict, uint32_t *bm, const VoxTuning &tune,
                            uint4 *big, uint32_t big_cap, uint32_t *counters, int num_sms,
                            cudaStream_t st) {
    // counters[0] = big entries, counters[1] = big cursor
    cudaError_t e = cudaMemsetAsync(counters, 0, 2 * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    if (nt > 0) {
        const int64_t want = (nt + 255) / 256;
        const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)num_sms * 16));
        const int bblocks = num_sms * 2;
        if (strict) {
            k_voxelize<true><<<blocks, 256, 0, st>>>(pts, tris, nt, gp, rx, ry, rz, bm, tune, big, big_cap,
                                                    counters);
            k_voxelize_big<true><<<bblocks, 256, 0, st>>>(pts, tris, gp, rx, ry, rz, bm, big, counters,
                                                         big_cap, counters + 1);
        } else {
            k_voxelize<false><<<blocks, 256, 0, st>>>(pts, tris, nt, gp, rx, ry, rz, bm, tune, big, big_cap,
                                                     counters);
            k_voxelize_big<false><<<bblocks, 256, 0, st>>>(pts, tris, gp, rx, ry, rz, bm, big, counters,
                                                          big_cap, counters + 1);
        }
        count_launches(2);
    }
    return cudaGetLastError();
}

}  // namespace svo
