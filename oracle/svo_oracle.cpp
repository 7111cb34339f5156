// svo_oracle.cpp -- CPU restatement of GPU-SVO's octree build pipeline.
//
// TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline); the
// product never links it.  See svo_oracle.h for the map from each function to
// the reference source it restates, and for what is pinned and what is not.
//
// Compile with -ffp-contract=off: every float operation below is rounded
// exactly where it is written, and std::fmaf marks the places where nvcc's
// default contraction fuses a multiply into an add in the reference's device
// code (see fp:: below).
#include "svo_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <limits>
#include <new>
#include <string>
#include <thread>
#include <utility>
#include <vector>

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

constexpr uint32_t kNone = 0xFFFFFFFFu;  // UINT_MAX, the reference's "no index"

// Allocator whose resize() leaves trivial elements uninitialised, so that large
// output arrays are first touched by the threads that fill them.
template <class T>
struct NoInit : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = NoInit<U>;
    };
    NoInit() = default;
    template <class U>
    NoInit(const NoInit<U> &) {}
    template <class U>
    void construct(U *p) noexcept {
        ::new ((void *)p) U;
    }
    template <class U, class... A>
    void construct(U *p, A &&...a) {
        ::new ((void *)p) U(std::forward<A>(a)...);
    }
};
template <class T>
using big_vector = std::vector<T, NoInit<T>>;

// body(begin, end) over [0, n) in chunks of `chunk`, handed out dynamically to
// `nth` std::threads.
template <class F>
void parallel_for(int64_t n, int64_t chunk, int nth, F body) {
    if (nth <= 1 || n <= chunk) {
        body((int64_t)0, n);
        return;
    }
    std::atomic<int64_t> next{0};
    auto worker = [&]() {
        for (;;) {
            int64_t b = next.fetch_add(chunk);
            if (b >= n) return;
            body(b, std::min(n, b + chunk));
        }
    };
    std::vector<std::thread> pool;
    for (int i = 1; i < nth; ++i) pool.emplace_back(worker);
    worker();
    for (auto &t : pool) t.join();
}

// ---------------------------------------------------------------------------
// Morton codes.  The reference encodes with byte LUTs into a u32
// (src/MortonLUT.h:482-501): bit i of x/y/z goes to bit 3i/3i+1/3i+2 and the
// result is truncated to 32 bits, so it is exact for coordinates < 1024.  This
// is the same interleave computed by bit spreading and kept in 64 bits, which
// extends it to coordinates < 2^21.
// ---------------------------------------------------------------------------
inline uint64_t spread3(uint64_t v) {
    v &= 0x1FFFFFull;
    v = (v | (v << 32)) & 0x1F00000000FFFFull;
    v = (v | (v << 16)) & 0x1F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

inline uint32_t compact3(uint64_t v) {
    v &= 0x1249249249249249ull;
    v = (v | (v >> 2)) & 0x10C30C30C30C30C3ull;
    v = (v | (v >> 4)) & 0x100F00F00F00F00Full;
    v = (v | (v >> 8)) & 0x1F0000FF0000FFull;
    v = (v | (v >> 16)) & 0x1F00000000FFFFull;
    v = (v | (v >> 32)) & 0x1FFFFFull;
    return (uint32_t)v;
}

inline uint64_t morton(uint32_t x, uint32_t y, uint32_t z) {
    return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}

inline void demorton(uint64_t c, uint32_t &x, uint32_t &y, uint32_t &z) {
    x = compact3(c);
    y = compact3(c >> 1);
    z = compact3(c >> 2);
}

// ---------------------------------------------------------------------------
// Floating-point model.  The reference's device arithmetic is Eigen 3.4
// expression templates compiled by nvcc with its default --fmad=true.
//   * Eigen evaluates a fixed-size dot/sum by halving the range: a 3-term dot
//     is a0*b0 + (a1*b1 + a2*b2), a 2-term dot a0*b0 + a1*b1.
//   * cross(a,b) = (a1*b2 - a2*b1, a2*b0 - a0*b2, a0*b1 - a1*b0).
//   * normalized() = v / sqrt(squaredNorm) when squaredNorm > 0, else v.
// nvcc then fuses each single-use product into the add/sub that consumes it;
// "reference" mode below states which product becomes the FMA: the left
// operand of the add, the minuend of the sub -- except inside the voxel loop,
// where a product that does not depend on the loop's x is hoisted first and
// the other one is fused.  The reference's own build pins the pattern (its
// recorded voxels, nodes and arrays, tests/test_ref_pins.py); a GPU probe test
// checks the same machinery against nvcc on restated expressions.  "strict"
// mode rounds every operation (what a non-contracting compiler would produce).
// ---------------------------------------------------------------------------
namespace fp {
// Contraction sites of the reference's arithmetic.  Choice per site: 0 fuse
// the first product of the sum, 1 fuse the second, 2 no fusion.  Strict mode
// never fuses.  The defaults are the pattern of the reference's own build
// (src/SVO.cu compiled by nvcc 12.9 for sm_100a; its surface voxels are
// recorded in tests/golden/ref_pins.json and ref_voxels.npz): everything
// fuses its first product except the inner sum of the squared norm
// (c1*c1 + c2*c2 fuses c2*c2) and the three ZX edge tests in the voxel loop
// (a*p.z does not vary with x and is hoisted out of the x loop; b*p.x is
// fused).  oracle_set_fp_sites changes them (used to search for the pattern,
// and by the probe test, whose restated loop nvcc fuses differently in the
// third ZX test).
enum Site {
    kCross, kSqInner, kSqOuter, kD12Inner, kD12Outer, kDEdge, kPlaneInner, kPlaneOuter,
    kLoopXY, kLoopYZ = kLoopXY + 3, kLoopZX = kLoopYZ + 3, kNumSites = kLoopZX + 3
};
int g_site[kNumSites] = {0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1};

inline float dot2s(int site, bool strict, float a0, float a1, float b0, float b1) {
    const int c = strict ? 2 : g_site[site];
    if (c == 0) return std::fmaf(a0, b0, a1 * b1);
    if (c == 1) return std::fmaf(a1, b1, a0 * b0);
    return a0 * b0 + a1 * b1;
}
inline float dot3s(int inner, int outer, bool strict, float a0, float a1, float a2, float b0, float b1,
                   float b2) {
    const float t = dot2s(inner, strict, a1, a2, b1, b2);
    const int c = strict ? 2 : g_site[outer];
    return c == 2 ? a0 * b0 + t : std::fmaf(a0, b0, t);
}
// a*b - c*d
inline float diffs(int site, bool strict, float a, float b, float c, float d) {
    const int k = strict ? 2 : g_site[site];
    if (k == 0) return std::fmaf(a, b, -(c * d));
    if (k == 1) return std::fmaf(-c, d, a * b);
    return a * b - c * d;
}
inline float dot2(bool strict, float a0, float a1, float b0, float b1) {
    if (strict) return a0 * b0 + a1 * b1;
    return std::fmaf(a0, b0, a1 * b1);
}
inline float dot3(bool strict, float a0, float a1, float a2, float b0, float b1, float b2) {
    if (strict) return a0 * b0 + (a1 * b1 + a2 * b2);
    return std::fmaf(a0, b0, std::fmaf(a1, b1, a2 * b2));
}
inline float diffprod(bool strict, float a, float b, float c, float d) {
    if (strict) return a * b - c * d;
    return std::fmaf(a, b, -(c * d));
}
// o + w * x (a node origin component, src/SVO.cu:262,296,335)
inline float origin(bool strict, float o, float w, float x) {
    if (strict) return o + w * x;
    return std::fmaf(w, x, o);
}
}  // namespace fp

// The reference's own float min/max (src/CUDAUtil.h:72-80): plain compares.
inline float cmin(float a, float b) { return a < b ? a : b; }
inline float cmax(float a, float b) { return a > b ? a : b; }

// float -> int conversion as the device does it (cvt.rzi.s32.f32: truncate,
// saturate, NaN -> 0), used for the triangle's grid bbox (src/SVO.cu:76-85).
inline int f2i_rz(float f) {
    if (std::isnan(f)) return 0;
    if (f >= 2147483648.0f) return std::numeric_limits<int>::max();
    if (f <= -2147483648.0f) return std::numeric_limits<int>::min();
    return (int)f;
}
inline int clampi(int f, int a, int b) {  // src/CUDAUtil.h:82-110
    int lo = f < b ? f : b;
    return a > lo ? a : lo;
}

struct Grid {
    int res[3];
    float origin[3];  // modelBBox.min
    float unit[3];    // unitVoxelSize (src/SVO.cu:348-350)
    float bbox[9];
};

// ---------------------------------------------------------------------------
// Per-triangle setup and voxel test: src/SVO.cu:53-185, in the same operation
// order.
// ---------------------------------------------------------------------------
struct TriSetup {
    float n[3];
    float d1, d2;
    float nxy[3][2], dxy[3];
    float nyz[3][2], dyz[3];
    float nzx[3][2], dzx[3];
    int lo[3], hi[3];
};

void tri_setup(bool strict, const Grid &g, const float *p0, const float *p1, const float *p2,
               TriSetup &s) {
    const float *u = g.unit;
    float v0[3], v1[3], v2[3], e0[3], e1[3], e2[3];
    for (int i = 0; i < 3; ++i) {
        v0[i] = p0[i] - g.origin[i];
        v1[i] = p1[i] - g.origin[i];
        v2[i] = p2[i] - g.origin[i];
    }
    for (int i = 0; i < 3; ++i) {
        e0[i] = v1[i] - v0[i];
        e1[i] = v2[i] - v1[i];
        e2[i] = v0[i] - v2[i];
    }
    // n = e0.cross(e1).normalized()   (src/SVO.cu:69)
    float c[3];
    c[0] = fp::diffs(fp::kCross, strict, e0[1], e1[2], e0[2], e1[1]);
    c[1] = fp::diffs(fp::kCross, strict, e0[2], e1[0], e0[0], e1[2]);
    c[2] = fp::diffs(fp::kCross, strict, e0[0], e1[1], e0[1], e1[0]);
    float sq = fp::dot3s(fp::kSqInner, fp::kSqOuter, strict, c[0], c[1], c[2], c[0], c[1], c[2]);
    if (sq > 0.0f) {
        float r = std::sqrt(sq);
        for (int i = 0; i < 3; ++i) s.n[i] = c[i] / r;
    } else {
        for (int i = 0; i < 3; ++i) s.n[i] = c[i];
    }
    const float *n = s.n;
    // triangle bbox in grid (src/SVO.cu:73-85)
    for (int i = 0; i < 3; ++i) {
        float mn = cmin(v0[i], cmin(v1[i], v2[i]));
        float mx = cmax(v0[i], cmax(v1[i], v2[i]));
        s.lo[i] = clampi(f2i_rz(mn / u[i]), 0, g.res[i] - 1);
        s.hi[i] = clampi(f2i_rz(mx / u[i]), 0, g.res[i] - 1);
    }
    // plane test constants (src/SVO.cu:88-93)
    float cc[3];
    for (int i = 0; i < 3; ++i) cc[i] = n[i] > 0.0f ? u[i] : 0.0f;
    float a[3], b[3];
    for (int i = 0; i < 3; ++i) {
        a[i] = cc[i] - v0[i];
        b[i] = (u[i] - cc[i]) - v0[i];
    }
    s.d1 = fp::dot3s(fp::kD12Inner, fp::kD12Outer, strict, n[0], n[1], n[2], a[0], a[1], a[2]);
    s.d2 = fp::dot3s(fp::kD12Inner, fp::kD12Outer, strict, n[0], n[1], n[2], b[0], b[1], b[2]);
    // projection tests (src/SVO.cu:96-149).  For the projection onto axes
    // (i, j) the edge normal is (-e[j], e[i]), negated when n on the third
    // axis is negative.
    const float *vs[3] = {v0, v1, v2};
    const float *es[3] = {e0, e1, e2};
    // XY: n_xy_e = (-e.y, e.x), flipped if n.z < 0; d uses (v.x, v.y), (u.x, u.y)
    // YZ: n_yz_e = (-e.z, e.y), flipped if n.x < 0; d uses (v.y, v.z), (u.y, u.z)
    // ZX: n_zx_e = (-e.x, e.z), flipped if n.y < 0; d uses (v.z, v.x), (u.z, u.x)
    struct Plane {
        int i, j;  // the two axes of the 2-D projection, in the reference's order
        int flip_axis;
        float (*nn)[2];
        float *dd;
    } planes[3] = {{0, 1, 2, s.nxy, s.dxy}, {1, 2, 0, s.nyz, s.dyz}, {2, 0, 1, s.nzx, s.dzx}};
    for (const Plane &pl : planes) {
        for (int k = 0; k < 3; ++k) {
            float ne0 = -1.0f * es[k][pl.j];
            float ne1 = es[k][pl.i];
            if (n[pl.flip_axis] < 0.0f) {
                ne0 = -ne0;
                ne1 = -ne1;
            }
            pl.nn[k][0] = ne0;
            pl.nn[k][1] = ne1;
            float dt = fp::dot2s(fp::kDEdge, strict, ne0, ne1, vs[k][pl.i], vs[k][pl.j]);
            pl.dd[k] = ((-1.0f * dt) + cmax(0.0f, u[pl.i] * ne0)) + cmax(0.0f, u[pl.j] * ne1);
        }
    }
}

// src/SVO.cu:156-177 for one voxel
inline bool voxel_hit(bool strict, const Grid &g, const TriSetup &s, int x, int y, int z) {
    const float p[3] = {(float)x * g.unit[0], (float)y * g.unit[1], (float)z * g.unit[2]};
    const float nDOTp =
        fp::dot3s(fp::kPlaneInner, fp::kPlaneOuter, strict, s.n[0], s.n[1], s.n[2], p[0], p[1], p[2]);
    if ((nDOTp + s.d1) * (nDOTp + s.d2) > 0.0f) return false;
    for (int k = 0; k < 3; ++k)
        if (fp::dot2s(fp::kLoopXY + k, strict, s.nxy[k][0], s.nxy[k][1], p[0], p[1]) + s.dxy[k] < 0.0f)
            return false;
    for (int k = 0; k < 3; ++k)
        if (fp::dot2s(fp::kLoopYZ + k, strict, s.nyz[k][0], s.nyz[k][1], p[1], p[2]) + s.dyz[k] < 0.0f)
            return false;
    for (int k = 0; k < 3; ++k)
        if (fp::dot2s(fp::kLoopZX + k, strict, s.nzx[k][0], s.nzx[k][1], p[2], p[0]) + s.dzx[k] < 0.0f)
            return false;
    return true;
}

// ---------------------------------------------------------------------------
// Bounding cube: src/BaseModel.h:24-49 (host code, no FMA possible).
// ---------------------------------------------------------------------------
int bbox_cube(const float *pts, int64_t n, float out[9]) {
    if (n <= 0) return fail(ORACLE_ERR_EMPTY, "mesh has no vertices");
    float mn[3], mx[3];
    for (int i = 0; i < 3; ++i) mn[i] = mx[i] = pts[i];
    for (int64_t k = 0; k < n; ++k) {
        for (int i = 0; i < 3; ++i) {
            float v = pts[3 * k + i];
            if (!std::isfinite(v)) return fail(ORACLE_ERR_INVALID_ARGUMENT, "non-finite vertex");
            mn[i] = std::min(mn[i], v);
            mx[i] = std::max(mx[i], v);
        }
    }
    float amin[3], amax[3], len[3];
    for (int i = 0; i < 3; ++i) {
        amin[i] = mn[i];
        amax[i] = mx[i];
        len[i] = mx[i] - mn[i];
    }
    float maxlen = cmax(len[0], cmax(len[1], len[2]));
    for (int i = 0; i < 3; ++i) {
        if (maxlen == len[i]) continue;
        float delta = maxlen - len[i];
        amin[i] = mn[i] - (delta / 2.0f);
        amax[i] = mx[i] + (delta / 2.0f);
    }
    float eps[3];
    for (int i = 0; i < 3; ++i) eps[i] = (amax[i] - amin[i]) / 10001.0f;
    for (int i = 0; i < 3; ++i) {
        amin[i] -= eps[i];
        amax[i] += eps[i];
    }
    for (int i = 0; i < 3; ++i) {
        out[i] = amin[i];
        out[3 + i] = amax[i];
        out[6 + i] = amax[i] - amin[i];
    }
    return ORACLE_OK;
}

int nthreads_of(int n) {
    if (n > 0) return n;
    unsigned h = std::thread::hardware_concurrency();
    return h ? (int)h : 1;
}

int check_mesh(const float *points, int64_t np, const int32_t *tris, int64_t nt, const int res[3]) {
    if (!points || np <= 0) return fail(ORACLE_ERR_EMPTY, "mesh has no vertices");
    if (nt < 0 || (nt > 0 && !tris)) return fail(ORACLE_ERR_INVALID_ARGUMENT, "bad triangle array");
    for (int i = 0; i < 3; ++i)
        if (res[i] < 1 || res[i] > 4096)
            return fail(ORACLE_ERR_UNSUPPORTED, "resolution must be in [1, 4096]");
    for (int64_t k = 0; k < 3 * nt; ++k)
        if (tris[k] < 0 || tris[k] >= np)
            return fail(ORACLE_ERR_INVALID_ARGUMENT, "triangle index out of range");
    return ORACLE_OK;
}

int make_grid(const float *points, int64_t np, const int res[3], Grid &g) {
    int rc = bbox_cube(points, np, g.bbox);
    if (rc) return rc;
    for (int i = 0; i < 3; ++i) {
        g.res[i] = res[i];
        g.origin[i] = g.bbox[i];
        g.unit[i] = g.bbox[6 + i] / (float)res[i];  // src/SVO.cu:348-350
    }
    return ORACLE_OK;
}

// Voxelize into a dense flag bitmap indexed by Morton code (the reference's
// dense array d_CNodeMortonArray, src/SVO.cu:367, with bit 31 -> one bit),
// then compact it to the sorted unique codes (src/SVO.cu:384-408).
int voxelize(const float *points, const int32_t *tris, int64_t nt, const Grid &g, bool strict,
             int nth, std::vector<uint64_t> &codes) {
    const uint64_t ncodes = morton(g.res[0] - 1, g.res[1] - 1, g.res[2] - 1) + 1;
    const uint64_t nwords = (ncodes + 63) / 64;
    std::vector<uint64_t> bits;
    try {
        bits.assign(nwords, 0);
    } catch (const std::bad_alloc &) {
        return fail(ORACLE_ERR_OUT_OF_MEMORY, "bitmap allocation failed");
    }
    uint64_t *bw = bits.data();
    parallel_for(nt, 256, nth, [&](int64_t tb, int64_t te) {
    for (int64_t t = tb; t < te; ++t) {
        TriSetup s;
        tri_setup(strict, g, points + 3 * (int64_t)tris[3 * t], points + 3 * (int64_t)tris[3 * t + 1],
                  points + 3 * (int64_t)tris[3 * t + 2], s);
        for (int z = s.lo[2]; z <= s.hi[2]; ++z)
            for (int y = s.lo[1]; y <= s.hi[1]; ++y)
                for (int x = s.lo[0]; x <= s.hi[0]; ++x) {
                    if (!voxel_hit(strict, g, s, x, y, z)) continue;
                    uint64_t c = morton(x, y, z);
                    std::atomic_ref<uint64_t>(bw[c >> 6]).fetch_or(1ull << (c & 63),
                                                                   std::memory_order_relaxed);
                }
    }
    });
    codes.clear();
    for (uint64_t w = 0; w < nwords; ++w) {
        uint64_t v = bw[w];
        while (v) {
            int b = __builtin_ctzll(v);
            codes.push_back(w * 64 + b);
            v &= v - 1;
        }
    }
    return ORACLE_OK;
}

}  // namespace

struct oracle_result {
    int depth = 0;
    int res[3] = {0, 0, 0};
    float bbox[9];
    std::vector<int64_t> level_counts;  // depthNumNodes + the top level
    std::vector<oracle_node> nodes;
    big_vector<oracle_vertex> verts;
    big_vector<oracle_edge> edges;
    std::vector<uint64_t> keys;
    std::vector<uint64_t> codes;  // full-width Morton code per node
    big_vector<uint64_t> dedup[3];
};

namespace {

// Neighbour tables of src/MortonLUT.h:531-596, generated: for child octant
// `key` and direction j = (dx+1) + 3(dy+1) + 9(dz+1), the parent-level
// neighbour that holds the target and the target's octant in it.
struct NeighborLUT {
    short parent[8][27];
    short child[8][27];
    NeighborLUT() {
        for (int key = 0; key < 8; ++key)
            for (int j = 0; j < 27; ++j) {
                int d[3] = {j % 3 - 1, (j / 3) % 3 - 1, j / 9 - 1};
                int k[3] = {key & 1, (key >> 1) & 1, (key >> 2) & 1};
                int pj = 0, cj = 0, mul = 1;
                for (int a = 0; a < 3; ++a) {
                    int c = k[a] + d[a];                 // -1..2 in child units
                    int pd = c < 0 ? -1 : (c > 1 ? 1 : 0);  // parent step
                    pj += (pd + 1) * mul;
                    cj |= (c & 1) << a;
                    mul *= 3;
                }
                parent[key][j] = (short)pj;
                child[key][j] = (short)cj;
            }
    }
};

// d_vertSharedLUT (src/SVO.cu:567-584) and d_edgeSharedLUT (src/SVO.cu:611-627),
// generated: the neighbour slots (ascending) of the nodes sharing corner i /
// edge i.  Edge i runs between the corners in kEdgeCorners (src/SVO.cu:610,638-663).
const int kEdgeCorners[12][2] = {{0, 2}, {2, 3}, {3, 1}, {1, 0}, {4, 6}, {6, 7},
                                 {7, 5}, {5, 4}, {0, 4}, {2, 6}, {3, 7}, {1, 5}};
struct SharedLUT {
    short vert[8][8];
    short edge[12][4];
    SharedLUT() {
        for (int i = 0; i < 8; ++i) {
            int c[3] = {i & 1, (i >> 1) & 1, (i >> 2) & 1};
            int n = 0;
            for (int dz = c[2] - 1; dz <= c[2]; ++dz)
                for (int dy = c[1] - 1; dy <= c[1]; ++dy)
                    for (int dx = c[0] - 1; dx <= c[0]; ++dx)
                        vert[i][n++] = (short)((dx + 1) + 3 * (dy + 1) + 9 * (dz + 1));
        }
        for (int e = 0; e < 12; ++e) {
            int a = kEdgeCorners[e][0], b = kEdgeCorners[e][1];
            int ca[3] = {a & 1, (a >> 1) & 1, (a >> 2) & 1};
            int cb[3] = {b & 1, (b >> 1) & 1, (b >> 2) & 1};
            int lo[3], hi[3];
            for (int k = 0; k < 3; ++k) {
                if (ca[k] != cb[k]) {
                    lo[k] = hi[k] = 0;  // along the edge: same node row
                } else {
                    lo[k] = ca[k] - 1;
                    hi[k] = ca[k];
                }
            }
            int n = 0;
            for (int dz = lo[2]; dz <= hi[2]; ++dz)
                for (int dy = lo[1]; dy <= hi[1]; ++dy)
                    for (int dx = lo[0]; dx <= hi[0]; ++dx)
                        edge[e][n++] = (short)((dx + 1) + 3 * (dy + 1) + 9 * (dz + 1));
        }
    }
};

const NeighborLUT kNbr;
const SharedLUT kShared;

// One level of the reference's create() loop (src/SVO.cu:383-495), run on the
// sorted unique coarse codes P of this level.  Returns the parents (sorted
// unique P >> 3) for the next level.
struct LevelState {
    std::vector<oracle_node> all;   // d_SVONodeArray
    std::vector<int64_t> esum{};    // d_esumTreeNodesArray
    std::vector<int64_t> depthNum;  // depthNumNodes
    std::vector<int64_t> lastS;     // d_sumTreeNodesArray (kept across levels)
    std::vector<uint64_t> codes;    // full-width code of every node
};

int build_levels(const std::vector<uint64_t> &leaf, const Grid &g, bool strict, oracle_result &r) {
    LevelState st;
    std::vector<uint64_t> P = leaf;
    float width = g.unit[0];  // unitNodeWidth = unitVoxelSize.x (src/SVO.cu:351)
    int depth = 0;
    if (P.empty()) return fail(ORACLE_ERR_EMPTY, "no surface voxels");
    if (P.size() == 1)
        return fail(ORACLE_ERR_DEGENERATE,
                    "a single surface voxel: the reference's build is undefined for it");
    while (true) {
        const size_t numC = P.size();
        if (numC == 0) break;
        ++depth;
        size_t numNodes = 1;
        std::vector<int64_t> S;
        std::vector<uint64_t> parents;
        if (numC > 1) {
            // cpNumNodes + inclusive_scan (src/SVO.cu:221-235, 423-438)
            S.assign(numC, 0);
            parents.push_back(P[0] >> 3);
            for (size_t i = 1; i < numC; ++i) {
                int64_t add = ((P[i] >> 3) == (P[i - 1] >> 3)) ? 0 : 8;
                if (add) parents.push_back(P[i] >> 3);
                S[i] = S[i - 1] + add;
            }
            numNodes = (size_t)S.back() + 8;
            st.depthNum.push_back((int64_t)numNodes);
            st.lastS = S;
        } else {
            S.assign(1, st.lastS.empty() ? 0 : st.lastS[0]);
            if ((P[0] & 7) != 0)
                return fail(ORACLE_ERR_DEGENERATE,
                            "single top-level node with a non-zero octant: undefined in the reference");
        }
        oracle_node def;
        std::memset(&def, 0, sizeof(def));
        def.is_leaf = 1;
        def.parent = kNone;
        for (int k = 0; k < 8; ++k) def.childs[k] = kNone;
        for (int k = 0; k < 27; ++k) def.neighbors[k] = kNone;
        std::vector<oracle_node> lvl(numNodes, def);
        std::vector<uint64_t> lcode(numNodes, 0);
        const int64_t preDepth = st.esum.empty() ? 0 : st.esum.back();
        const int64_t preChild = st.esum.size() >= 2 ? st.esum[st.esum.size() - 2] : 0;
        if (depth >= 2 && st.esum.empty()) return fail(ORACLE_ERR_INVALID_ARGUMENT, "internal");
        // createNode_1 / createNode_2 (src/SVO.cu:237-309)
        for (size_t i = 0; i < numC; ++i) {
            const uint64_t m = P[i];
            const size_t addr = (size_t)S[i] + (m & 7);
            oracle_node &nd = lvl[addr];
            nd.morton_code = (uint32_t)m;
            uint32_t x, y, z;
            demorton(m, x, y, z);
            nd.origin[0] = fp::origin(strict, g.origin[0], width, (float)x);
            nd.origin[1] = fp::origin(strict, g.origin[1], width, (float)y);
            nd.origin[2] = fp::origin(strict, g.origin[2], width, (float)z);
            nd.width = width;
            lcode[addr] = m;
            if (depth >= 2) {
                nd.is_leaf = 0;
                for (int k = 0; k < 8; ++k) {
                    nd.childs[k] = (uint32_t)(preChild + (int64_t)i * 8 + k);
                    st.all[(size_t)(preChild + (int64_t)i * 8 + k)].parent =
                        (uint32_t)(preDepth + S[i] + (int64_t)(m & 7));
                }
            }
        }
        // unique(begMorton) + createRemainNode (src/SVO.cu:311-339, 461-469):
        // slots still holding morton 0 become the missing siblings.
        std::vector<uint64_t> beg;
        for (size_t i = 0; i < numC; ++i) {
            uint64_t b = (P[i] / 8) * 8;
            if (beg.empty() || beg.back() != b) beg.push_back(b);
        }
        for (size_t t = 0; t < numNodes; ++t) {
            oracle_node &nd = lvl[t];
            if (nd.morton_code != 0) continue;  // src/SVO.cu:324
            const uint64_t m = beg[t / 8] + (t & 7);
            nd.morton_code = (uint32_t)m;
            lcode[t] = m;
            uint32_t x, y, z;
            demorton(m, x, y, z);
            nd.origin[0] = fp::origin(strict, g.origin[0], width, (float)x);
            nd.origin[1] = fp::origin(strict, g.origin[1], width, (float)y);
            nd.origin[2] = fp::origin(strict, g.origin[2], width, (float)z);
            nd.width = width;
        }
        if (st.esum.empty()) st.esum.push_back(0);
        st.all.insert(st.all.end(), lvl.begin(), lvl.end());
        st.codes.insert(st.codes.end(), lcode.begin(), lcode.end());
        st.esum.push_back((int64_t)numNodes + st.esum.back());
        if (st.all.size() >= (size_t)kNone)
            return fail(ORACLE_ERR_UNSUPPORTED, "more than 2^32-2 nodes");
        if (numC == 1) break;  // numNodes/8 == 0 (src/SVO.cu:487-490)
        P.swap(parents);
        width *= 2.0f;  // unitNodeWidth *= 2.0 (exact doubling, src/SVO.cu:483)
    }
    r.depth = depth;
    r.level_counts.clear();
    for (size_t d = 0; d + 1 < st.esum.size(); ++d) r.level_counts.push_back(st.esum[d + 1] - st.esum[d]);
    r.nodes.swap(st.all);
    r.codes.swap(st.codes);
    return ORACLE_OK;
}

// constructNodeNeighbors (src/SVO.cu:522-565).  The reference's per-level
// kernel stores into a local copy (src/SVO.cu:535-542), so its effective
// output is only the root's self entry; `full` runs the intended top-down
// propagation through the neighbour tables instead.
void neighbors(oracle_result &r, bool full) {
    auto &nodes = r.nodes;
    if (r.depth < 2) return;
    const size_t root = nodes.size() - 1;
    nodes[root].neighbors[13] = (uint32_t)root;
    if (!full) return;
    std::vector<int64_t> off(1, 0);
    for (int64_t c : r.level_counts) off.push_back(off.back() + c);
    for (int lvl = r.depth - 2; lvl >= 0; --lvl) {
        for (int64_t t = off[lvl]; t < off[lvl + 1]; ++t) {
            oracle_node &nd = nodes[(size_t)t];
            const oracle_node &p = nodes[nd.parent];
            const int key = nd.morton_code & 7;
            for (int j = 0; j < 27; ++j) {
                uint32_t pn = p.neighbors[kNbr.parent[key][j]];
                nd.neighbors[j] = pn != kNone ? nodes[pn].childs[kNbr.child[key][j]] : kNone;
            }
        }
    }
}

// determineNodeVertex / determineNodeEdge + consecutive unique
// (src/SVO.cu:567-728).  Owner: the reference keeps the last sharing slot that
// holds an index (its running minimum is never updated, src/SVO.cu:600-603);
// with `min_owner` the owner is the smallest index among the sharing nodes.
inline uint32_t owner_of(const oracle_node &nd, const short *slots, int ns, uint32_t self,
                         bool min_owner) {
    uint32_t idx = self;
    if (min_owner) {
        uint32_t best = kNone;
        for (int j = 0; j < ns; ++j) best = std::min(best, nd.neighbors[slots[j]]);
        return best != kNone ? best : self;
    }
    for (int j = 0; j < ns; ++j)
        if (nd.neighbors[slots[j]] < kNone) idx = nd.neighbors[slots[j]];
    return idx;
}

inline bool veq(const float *a, const float *b) { return a[0] == b[0] && a[1] == b[1] && a[2] == b[2]; }

// Vertex i of node t (src/SVO.cu:596-605): the corner offset without the origin.
inline void make_vertex(const oracle_node &nd, uint32_t t, int i, bool min_owner, oracle_vertex &v) {
    const float w = nd.width;
    v.pos[0] = w * (float)(i & 1);
    v.pos[1] = w * (float)((i >> 1) & 1);
    v.pos[2] = w * (float)((i >> 2) & 1);
    v.owner = owner_of(nd, kShared.vert[i], 8, t, min_owner);
}

// Edge e of node t (src/SVO.cu:638-674): origin plus 0 or width per component.
inline void make_edge(const oracle_node &nd, uint32_t t, int e, bool min_owner, oracle_edge &ed) {
    const float *o = nd.origin;
    const float w = nd.width;
    for (int s = 0; s < 2; ++s) {
        const int c = kEdgeCorners[e][s];
        float *dst = s ? ed.p1 : ed.p0;
        if (c == 0) {  // `origin` itself, no add
            dst[0] = o[0];
            dst[1] = o[1];
            dst[2] = o[2];
        } else {
            dst[0] = o[0] + ((c & 1) ? w : 0.0f);
            dst[1] = o[1] + ((c & 2) ? w : 0.0f);
            dst[2] = o[2] + ((c & 4) ? w : 0.0f);
        }
    }
    ed.owner = owner_of(nd, kShared.edge[e], 4, t, min_owner);
}

inline bool same_edge(const oracle_edge &a, const oracle_edge &b) {  // uniqueEdge, src/SVO.cu:686-693
    return (veq(a.p0, b.p0) && veq(a.p1, b.p1)) || (veq(a.p0, b.p1) && veq(a.p1, b.p0));
}

// The 8N vertices and 12N edges in node order, then thrust::unique's
// consecutive-duplicate removal (src/SVO.cu:710-725): element k is kept unless
// it equals element k - 1.  Element k - 1 is recomputed from its node, so the
// work splits into independent node ranges: one pass counts what each range
// keeps, a second writes it at the range's offset.
void vert_edge(oracle_result &r, bool min_owner, int nth) {
    const auto &nodes = r.nodes;
    const int64_t N = (int64_t)nodes.size();
    constexpr int64_t kChunk = 1 << 14;
    const int64_t nchunks = (N + kChunk - 1) / kChunk;
    std::vector<int64_t> vcount(nchunks + 1, 0), ecount(nchunks + 1, 0);
    auto vert_at = [&](int64_t k, oracle_vertex &v) {
        make_vertex(nodes[(size_t)(k >> 3)], (uint32_t)(k >> 3), (int)(k & 7), min_owner, v);
    };
    auto edge_at = [&](int64_t k, oracle_edge &e) {
        make_edge(nodes[(size_t)(k / 12)], (uint32_t)(k / 12), (int)(k % 12), min_owner, e);
    };
    // pass(c, write): walks chunk c's elements, counting (write = false) or
    // storing (write = true) the kept ones.
    auto pass = [&](int64_t c, bool write) {
        const int64_t tb = c * kChunk, te = std::min(N, tb + kChunk);
        int64_t nv = write ? vcount[c] : 0, ne = write ? ecount[c] : 0;
        oracle_vertex pv{}, cv{};
        if (tb > 0) vert_at(8 * tb - 1, pv);
        for (int64_t k = 8 * tb; k < 8 * te; ++k) {
            vert_at(k, cv);
            if (k == 0 || !veq(pv.pos, cv.pos)) {
                if (write) r.verts[(size_t)nv] = cv;
                ++nv;
            }
            pv = cv;
        }
        oracle_edge pe{}, ce{};
        if (tb > 0) edge_at(12 * tb - 1, pe);
        for (int64_t k = 12 * tb; k < 12 * te; ++k) {
            edge_at(k, ce);
            if (k == 0 || !same_edge(pe, ce)) {
                if (write) r.edges[(size_t)ne] = ce;
                ++ne;
            }
            pe = ce;
        }
        if (!write) {
            vcount[c + 1] = nv;
            ecount[c + 1] = ne;
        }
    };
    parallel_for(nchunks, 1, nth, [&](int64_t cb, int64_t ce) {
        for (int64_t c = cb; c < ce; ++c) pass(c, false);
    });
    for (int64_t c = 0; c < nchunks; ++c) {
        vcount[c + 1] += vcount[c];
        ecount[c + 1] += ecount[c];
    }
    r.verts.resize((size_t)vcount[nchunks]);
    r.edges.resize((size_t)ecount[nchunks]);
    parallel_for(nchunks, 1, nth, [&](int64_t cb, int64_t ce) {
        for (int64_t c = cb; c < ce; ++c) pass(c, true);
    });
}

// Sorts v and drops repeats (std::sort + std::unique), with the work split
// over `nth` threads: contiguous slices are sorted and uniqued on their own,
// then merged pairwise (uniqued again after each merge).
void sort_unique(big_vector<uint64_t> &v, int nth) {
    const size_t n = v.size();
    size_t parts = 1;
    while ((int)parts < nth && parts < 64 && n / (parts * 2) >= (1u << 16)) parts *= 2;
    std::vector<size_t> lo(parts), hi(parts);
    for (size_t p = 0; p < parts; ++p) {
        lo[p] = n * p / parts;
        hi[p] = n * (p + 1) / parts;
    }
    auto each = [&](size_t count, auto fn) {
        std::vector<std::thread> pool;
        for (size_t p = 1; p < count; ++p) pool.emplace_back(fn, p);
        fn(0);
        for (auto &t : pool) t.join();
    };
    each(parts, [&](size_t p) {
        std::sort(v.begin() + lo[p], v.begin() + hi[p]);
        hi[p] = (size_t)(std::unique(v.begin() + lo[p], v.begin() + hi[p]) - v.begin());
    });
    big_vector<uint64_t> tmp(n);
    for (size_t width = 1; width < parts; width *= 2) {
        // merge slice p with slice p + width into tmp at lo[p], then back
        const size_t pairs = (parts + 2 * width - 1) / (2 * width);
        each(pairs, [&](size_t q) {
            const size_t p = q * 2 * width, o = p + width;
            size_t end = lo[p];
            if (o < parts) {
                end = (size_t)(std::merge(v.begin() + lo[p], v.begin() + hi[p], v.begin() + lo[o],
                                          v.begin() + hi[o], tmp.begin() + lo[p]) - tmp.begin());
                end = (size_t)(std::unique(tmp.begin() + lo[p], tmp.begin() + end) - tmp.begin());
                std::copy(tmp.begin() + lo[p], tmp.begin() + end, v.begin() + lo[p]);
                hi[p] = end;
            }
        });
    }
    v.resize(hi[0]);
}

// Morton-keyed dedup of the nodes' vertices, edges and faces (no reference
// counterpart).  Lattice = finest-level voxel corners; a level-d node covers
// [c, c + 2^(d-1)) per axis with c its node coordinate << (d-1).
//   vertex key = morton(X, Y, Z)
//   edge key   = morton(min corner) << 6 | (d-1) << 2 | axis
//   face key   = morton(min corner) << 6 | (d-1) << 2 | normal axis
void dedup(oracle_result &r, int nth) {
    std::vector<int64_t> off(1, 0);
    for (int64_t c : r.level_counts) off.push_back(off.back() + c);
    const int64_t N = off.back();
    r.dedup[0].resize((size_t)N * 8);
    r.dedup[1].resize((size_t)N * 12);
    r.dedup[2].resize((size_t)N * 6);
    for (int lvl = 0; lvl < r.depth; ++lvl) {
        const uint32_t s = 1u << lvl;
        parallel_for(off[lvl + 1] - off[lvl], 1 << 14, nth, [&](int64_t tb, int64_t te) {
        for (int64_t t = off[lvl] + tb; t < off[lvl] + te; ++t) {
            uint32_t x, y, z;
            demorton(r.codes[(size_t)t], x, y, z);
            uint32_t c[3] = {x << lvl, y << lvl, z << lvl};
            uint64_t *vk = &r.dedup[0][(size_t)t * 8];
            uint64_t *ek = &r.dedup[1][(size_t)t * 12];
            uint64_t *fk = &r.dedup[2][(size_t)t * 6];
            for (int i = 0; i < 8; ++i)
                vk[i] = morton(c[0] + ((i & 1) ? s : 0), c[1] + ((i & 2) ? s : 0), c[2] + ((i & 4) ? s : 0));
            for (int a = 0; a < 3; ++a) {
                const int b1 = (a + 1) % 3, b2 = (a + 2) % 3;
                for (int k = 0; k < 4; ++k) {
                    uint32_t q[3] = {c[0], c[1], c[2]};
                    if (k & 1) q[b1] += s;
                    if (k & 2) q[b2] += s;
                    ek[4 * a + k] = (morton(q[0], q[1], q[2]) << 6) | ((uint64_t)lvl << 2) | a;
                }
                for (int k = 0; k < 2; ++k) {
                    uint32_t q[3] = {c[0], c[1], c[2]};
                    if (k) q[a] += s;
                    fk[2 * a + k] = (morton(q[0], q[1], q[2]) << 6) | ((uint64_t)lvl << 2) | a;
                }
            }
        }
        });
    }
    for (auto &v : r.dedup) sort_unique(v, nth);
}

}  // namespace

extern "C" {

const char *oracle_last_error(void) { return g_err.c_str(); }

void oracle_free(void *p) { std::free(p); }

// The oracle's floating-point model on batches of operands, for comparing it
// with what nvcc makes of the same expressions.  op (operands -> results):
//   0 dot2 (a0,a1,b0,b1)            1 dot3 (a0,a1,a2,b0,b1,b2)
//   2 a*b-c*d (a,b,c,d)             3 origin o+w*x (o,w,x)
//   4 normalize (c0,c1,c2) -> 3     5 voxel test: tri (9), voxel (x,y,z),
//                                     unit, res -> 1.0 / 0.0 (grid origin 0)
//   6 triangle setup, same operands -> n (3), d1, d2, dxy (3), dyz (3), dzx (3)
int oracle_set_fp_sites(const int *choice, int n) {
    for (int i = 0; i < n && i < fp::kNumSites; ++i) fp::g_site[i] = choice[i];
    return fp::kNumSites;
}

int oracle_fp_eval(int op, int strict, const float *in, int64_t n, float *out) {
    const bool st = strict != 0;
    for (int64_t i = 0; i < n; ++i) {
        switch (op) {
            case 0: {
                const float *a = in + 4 * i;
                out[i] = fp::dot2(st, a[0], a[1], a[2], a[3]);
                break;
            }
            case 1: {
                const float *a = in + 6 * i;
                out[i] = fp::dot3(st, a[0], a[1], a[2], a[3], a[4], a[5]);
                break;
            }
            case 2: {
                const float *a = in + 4 * i;
                out[i] = fp::diffprod(st, a[0], a[1], a[2], a[3]);
                break;
            }
            case 3: {
                const float *a = in + 3 * i;
                out[i] = fp::origin(st, a[0], a[1], a[2]);
                break;
            }
            case 4: {
                const float *c = in + 3 * i;
                const float sq = fp::dot3(st, c[0], c[1], c[2], c[0], c[1], c[2]);
                for (int k = 0; k < 3; ++k) out[3 * i + k] = sq > 0.0f ? c[k] / std::sqrt(sq) : c[k];
                break;
            }
            case 5: {
                const float *a = in + 14 * i;
                Grid g;
                const int res = (int)a[13];
                for (int k = 0; k < 3; ++k) {
                    g.res[k] = res;
                    g.origin[k] = 0.0f;
                    g.unit[k] = a[12];
                }
                TriSetup ts;
                tri_setup(st, g, a, a + 3, a + 6, ts);
                const int x = (int)a[9], y = (int)a[10], z = (int)a[11];
                const bool inside = x >= ts.lo[0] && x <= ts.hi[0] && y >= ts.lo[1] && y <= ts.hi[1] &&
                                    z >= ts.lo[2] && z <= ts.hi[2];
                out[i] = inside && voxel_hit(st, g, ts, x, y, z) ? 1.0f : 0.0f;
                break;
            }
            case 6: {
                const float *a = in + 14 * i;
                Grid g;
                const int res = (int)a[13];
                for (int k = 0; k < 3; ++k) {
                    g.res[k] = res;
                    g.origin[k] = 0.0f;
                    g.unit[k] = a[12];
                }
                TriSetup ts;
                tri_setup(st, g, a, a + 3, a + 6, ts);
                float *o = out + 14 * i;
                for (int k = 0; k < 3; ++k) o[k] = ts.n[k];
                o[3] = ts.d1;
                o[4] = ts.d2;
                for (int k = 0; k < 3; ++k) {
                    o[5 + k] = ts.dxy[k];
                    o[8 + k] = ts.dyz[k];
                    o[11 + k] = ts.dzx[k];
                }
                break;
            }
            default:
                return fail(ORACLE_ERR_INVALID_ARGUMENT, "unknown op");
        }
    }
    return ORACLE_OK;
}

void oracle_tables(int16_t *nbr_parent, int16_t *nbr_child, int16_t *vert_shared,
                   int16_t *edge_shared) {
    std::memcpy(nbr_parent, kNbr.parent, sizeof(kNbr.parent));
    std::memcpy(nbr_child, kNbr.child, sizeof(kNbr.child));
    std::memcpy(vert_shared, kShared.vert, sizeof(kShared.vert));
    std::memcpy(edge_shared, kShared.edge, sizeof(kShared.edge));
}

uint64_t oracle_morton_encode(uint32_t x, uint32_t y, uint32_t z) { return morton(x, y, z); }

void oracle_morton_decode(uint64_t code, uint32_t *x, uint32_t *y, uint32_t *z) {
    demorton(code, *x, *y, *z);
}

// BaseModel::loadOBJ (src/BaseModel.cpp:3-25).  Same line reader and the same
// three sscanf patterns (sscanf_s behaves as sscanf for %f/%d).  Quirks kept:
// only "v " / "f " lines, `a/t/n` faces match no pattern and are dropped, an
// unterminated last line is dropped (the eof test fires first).  Two cases
// where the reference has no defined result become errors: a line of 255+
// characters (the reference loops forever) and a face index outside the
// vertex list (the reference reads out of bounds).
int oracle_load_obj(const char *path, float **points, int64_t *n_points, int32_t **tris,
                    int64_t *n_tris) {
    std::ifstream in(path);
    if (!in) return fail(ORACLE_ERR_IO, std::string("cannot open ") + path);
    std::vector<float> P;
    std::vector<int32_t> T;
    float x, y, z;
    int f0, f0_, f1, f1_, f2, f2_;
    char buffer[256] = {0};
    while (!in.getline(buffer, 255).eof()) {
        if (in.fail()) return fail(ORACLE_ERR_PARSE, "line longer than 254 characters");
        if (buffer[0] == 'v' && buffer[1] == ' ') {
            if (std::sscanf(buffer, "v %f %f %f", &x, &y, &z) == 3) {
                P.push_back(x);
                P.push_back(y);
                P.push_back(z);
            }
        } else if (buffer[0] == 'f' && buffer[1] == ' ') {
            if (std::sscanf(buffer, "f %d//%d %d//%d %d//%d", &f0, &f0_, &f1, &f1_, &f2, &f2_) == 6 ||
                std::sscanf(buffer, "f %d/%d %d/%d %d/%d", &f0, &f0_, &f1, &f1_, &f2, &f2_) == 6 ||
                std::sscanf(buffer, "f %d %d %d", &f0, &f1, &f2) == 3) {
                T.push_back(f0 - 1);
                T.push_back(f1 - 1);
                T.push_back(f2 - 1);
            }
        }
    }
    const int64_t np = (int64_t)P.size() / 3;
    for (int32_t v : T)
        if (v < 0 || v >= np) return fail(ORACLE_ERR_PARSE, "face index out of range");
    *points = (float *)std::malloc(std::max<size_t>(1, P.size()) * sizeof(float));
    *tris = (int32_t *)std::malloc(std::max<size_t>(1, T.size()) * sizeof(int32_t));
    if (!*points || !*tris) return fail(ORACLE_ERR_OUT_OF_MEMORY, "malloc failed");
    std::memcpy(*points, P.data(), P.size() * sizeof(float));
    std::memcpy(*tris, T.data(), T.size() * sizeof(int32_t));
    *n_points = np;
    *n_tris = (int64_t)T.size() / 3;
    return ORACLE_OK;
}

int oracle_bbox_cube(const float *points, int64_t n_points, float out[9]) {
    return bbox_cube(points, n_points, out);
}

int oracle_voxelize(const float *points, int64_t n_points, const int32_t *tris, int64_t n_tris,
                    int res_x, int res_y, int res_z, uint32_t flags, int n_threads,
                    uint64_t **codes, int64_t *n_codes) {
    const int res[3] = {res_x, res_y, res_z};
    int rc = check_mesh(points, n_points, tris, n_tris, res);
    if (rc) return rc;
    Grid g;
    if ((rc = make_grid(points, n_points, res, g))) return rc;
    std::vector<uint64_t> c;
    rc = voxelize(points, tris, n_tris, g, (flags & ORACLE_FLAG_STRICT_FP) != 0, nthreads_of(n_threads), c);
    if (rc) return rc;
    *codes = (uint64_t *)std::malloc(std::max<size_t>(1, c.size()) * sizeof(uint64_t));
    if (!*codes) return fail(ORACLE_ERR_OUT_OF_MEMORY, "malloc failed");
    std::memcpy(*codes, c.data(), c.size() * sizeof(uint64_t));
    *n_codes = (int64_t)c.size();
    return ORACLE_OK;
}

int oracle_build(const float *points, int64_t n_points, const int32_t *tris, int64_t n_tris,
                 int res_x, int res_y, int res_z, uint32_t flags, int n_threads,
                 oracle_result **out) {
    *out = nullptr;
    const int res[3] = {res_x, res_y, res_z};
    int rc = check_mesh(points, n_points, tris, n_tris, res);
    if (rc) return rc;
    const bool strict = (flags & ORACLE_FLAG_STRICT_FP) != 0;
    const bool full = (flags & ORACLE_FLAG_FULL_NEIGHBORS) != 0;
    Grid g;
    if ((rc = make_grid(points, n_points, res, g))) return rc;
    oracle_result *r = new (std::nothrow) oracle_result();
    if (!r) return fail(ORACLE_ERR_OUT_OF_MEMORY, "alloc");
    std::memcpy(r->bbox, g.bbox, sizeof(g.bbox));
    for (int a = 0; a < 3; ++a) r->res[a] = res[a];
    const int nth = nthreads_of(n_threads);
    rc = voxelize(points, tris, n_tris, g, strict, nth, r->keys);
    if (!rc) rc = build_levels(r->keys, g, strict, *r);
    if (rc) {
        delete r;
        return rc;
    }
    neighbors(*r, full);
    if (!(flags & ORACLE_FLAG_NO_VERT_EDGE)) vert_edge(*r, full, nth);
    if (flags & ORACLE_FLAG_DEDUP) dedup(*r, nth);
    *out = r;
    return ORACLE_OK;
}

void oracle_result_free(oracle_result *r) { delete r; }
int oracle_result_depth(const oracle_result *r) { return r->depth; }
int64_t oracle_result_num_nodes(const oracle_result *r) { return (int64_t)r->nodes.size(); }
int64_t oracle_result_num_vertices(const oracle_result *r) { return (int64_t)r->verts.size(); }
int64_t oracle_result_num_edges(const oracle_result *r) { return (int64_t)r->edges.size(); }
int64_t oracle_result_num_keys(const oracle_result *r) { return (int64_t)r->keys.size(); }
int oracle_result_level_counts(const oracle_result *r, int64_t *counts, int cap) {
    int n = (int)r->level_counts.size();
    for (int i = 0; i < n && i < cap; ++i) counts[i] = r->level_counts[i];
    return n;
}
const oracle_node *oracle_result_nodes(const oracle_result *r) { return r->nodes.data(); }
const oracle_vertex *oracle_result_vertices(const oracle_result *r) { return r->verts.data(); }
const oracle_edge *oracle_result_edges(const oracle_result *r) { return r->edges.data(); }
const uint64_t *oracle_result_keys(const oracle_result *r) { return r->keys.data(); }
const float *oracle_result_bbox(const oracle_result *r) { return r->bbox; }
int64_t oracle_result_num_dedup(const oracle_result *r, int kind) {
    return (kind >= 0 && kind < 3) ? (int64_t)r->dedup[kind].size() : -1;
}
const uint64_t *oracle_result_dedup(const oracle_result *r, int kind) {
    return (kind >= 0 && kind < 3) ? r->dedup[kind].data() : nullptr;
}

}  // extern "C"

namespace {

// write_cube (src/IO.h:23-90) over a list of cubes, with the same
// std::ofstream insertions (default float format = "%.6g" of the value
// widened to double; indices through Eigen::Vector2i, i.e. int).
template <class Cube>
int write_cubes(const char *path, size_t n, Cube cube) {
    std::ofstream output(path, std::ios::out);
    if (!output) return fail(ORACLE_ERR_IO, std::string("cannot open ") + path);
    size_t faceBegIdx = 0;
    auto vtx = [&](float a, float b, float c) {
        output << "v " << a << " " << b << " " << c << std::endl;
    };
    auto line = [&](size_t a, size_t b) {
        output << "l " << (int)a << " " << (int)b << std::endl;
    };
    for (size_t i = 0; i < n; ++i) {
        float o[3], w;
        cube(i, o, w);
        vtx(o[0] + 0.0f, o[1] + w, o[2] + w);        // v1
        vtx(o[0] + 0.0f, o[1] + 0.0f, o[2] + w);     // v2
        vtx(o[0] + 0.0f, o[1] + w, o[2] + 0.0f);     // v3
        vtx(o[0], o[1], o[2]);                       // v4
        vtx(o[0] + w, o[1] + 0.0f, o[2] + 0.0f);     // v5
        vtx(o[0] + w, o[1] + w, o[2] + 0.0f);        // v6
        vtx(o[0] + w, o[1] + 0.0f, o[2] + w);        // v7
        vtx(o[0] + w, o[1] + w, o[2] + w);           // v8
        const size_t b = faceBegIdx;
        line(b + 1, b + 2);
        line(b + 2, b + 7);
        line(b + 7, b + 8);
        line(b + 8, b + 1);
        line(b + 3, b + 4);
        line(b + 4, b + 5);
        line(b + 5, b + 6);
        line(b + 6, b + 3);
        line(b + 3, b + 1);
        line(b + 4, b + 2);
        line(b + 5, b + 7);
        line(b + 6, b + 8);
        faceBegIdx += 8;
    }
    output.close();
    return output.fail() ? fail(ORACLE_ERR_IO, "write failed") : ORACLE_OK;
}

}  // namespace

extern "C" {

// writeTree (src/SVO.cu:737-753): one cube per node, at its origin and width.
int oracle_write_tree(const oracle_result *r, const char *path) {
    return write_cubes(path, r->nodes.size(), [&](size_t i, float o[3], float &w) {
        for (int a = 0; a < 3; ++a) o[a] = r->nodes[i].origin[a];
        w = r->nodes[i].width;
    });
}

// writeTree's loop over any node array (the bench times it against the
// product's writer on the same nodes).
int oracle_write_tree_nodes(const oracle_node *nodes, int64_t n, const char *path) {
    return write_cubes(path, (size_t)n, [&](size_t i, float o[3], float &w) {
        for (int a = 0; a < 3; ++a) o[a] = nodes[i].origin[a];
        w = nodes[i].width;
    });
}

// writeVoxel (src/SVO.cu:755-777), as create() calls it on the surface voxels
// (src/SVO.cu:411-419): width = unitNodeWidth = the voxel size along x, and
// cube i at modelBBox.min + width * (x, y, z) of voxel i, host arithmetic
// (each product and sum rounded; x86-64 code without FMA).
int oracle_write_voxels(const oracle_result *r, const char *path) {
    const float width = r->bbox[6] / (float)r->res[0];
    return write_cubes(path, r->keys.size(), [&](size_t i, float o[3], float &w) {
        uint32_t c[3];
        demorton(r->keys[i], c[0], c[1], c[2]);
        for (int a = 0; a < 3; ++a) o[a] = r->bbox[a] + width * (float)c[a];
        w = width;
    });
}

}  // extern "C"
