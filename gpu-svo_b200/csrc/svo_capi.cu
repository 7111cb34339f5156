// svo_capi.cu -- C ABI: context, build orchestration, results.
//
// One build = (host->device copy of the mesh) -> bounding cube -> voxelize
// into the level-0 bitmap -> pyramid + block counts -> one scan -> one small
// device->host read of the level totals (the only mid-build sync, to size the
// outputs) -> per-level code lists -> one emission pass writing nodes,
// vertices and edges -> one small read of the duplicate counters.
// The reference's equivalent (src/SVO.cu:341-735) synchronises with the host
// at least six times per level and reallocates its node array per level.
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "svo_internal.h"
#include "svo_host.h"

using namespace svo;

struct svo_ctx {
    int device = 0;
    int num_sms = 148;
    cudaMemPool_t pool = nullptr;
    VoxTuning tune;
};

struct svo_result {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;
    int depth = 0;
    std::vector<int64_t> level_counts;
    svo_aabb bbox{};
    float unit[3] = {0.0f, 0.0f, 0.0f};
    uint64_t n_nodes = 0, n_verts = 0, n_edges = 0, n_keys = 0;
    svo_node *nodes = nullptr;
    svo_vertex *verts = nullptr;
    svo_edge *edges = nullptr;
    uint64_t *keys = nullptr;
    uint64_t n_dedup[3] = {0, 0, 0};
    uint64_t *dedup[3] = {nullptr, nullptr, nullptr};
    int n_timings = 0;
    float timings[9] = {};
};

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char *what) {
    if (e == cudaErrorMemoryAllocation)
        return fail(SVO_ERR_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
    return fail(SVO_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define SVO_TRY(call, what)                               \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

bool is_device_ptr(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Stream-ordered scratch owned by one build; everything is returned to the
// pool at the end of the build.
struct Scratch {
    cudaMemPool_t pool;
    cudaStream_t st;
    std::vector<void *> ptrs;
    cudaError_t err = cudaSuccess;
    template <class T>
    T *get(size_t count) {
        void *p = nullptr;
        if (err != cudaSuccess) return nullptr;
        err = cudaMallocFromPoolAsync(&p, std::max<size_t>(count * sizeof(T), 256), pool, st);
        if (err != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        return static_cast<T *>(p);
    }
    void release() {
        for (void *p : ptrs) cudaFreeAsync(p, st);
        ptrs.clear();
    }
    ~Scratch() { release(); }
};

template <class T>
T *pool_alloc(cudaMemPool_t pool, cudaStream_t st, size_t count, cudaError_t &err) {
    void *p = nullptr;
    if (err != cudaSuccess) return nullptr;
    err = cudaMallocFromPoolAsync(&p, std::max<size_t>(count * sizeof(T), 256), pool, st);
    return static_cast<T *>(p);
}

// CUDA events at stage boundaries (SVO_FLAG_TIMINGS).
struct StageTimer {
    enum { kStart, kBbox, kVox, kPyr, kScan, kCompact0, kCompact, kEmit, kUnique, kDedup, kN };
    bool on = false;
    cudaEvent_t ev[kN] = {};
    bool rec[kN] = {};
    explicit StageTimer(bool enable) : on(enable) {
        if (!on) return;
        for (auto &e : ev) cudaEventCreate(&e);
    }
    ~StageTimer() {
        if (!on) return;
        for (auto &e : ev) cudaEventDestroy(e);
    }
    void mark(int i, cudaStream_t st) {
        if (!on) return;
        cudaEventRecord(ev[i], st);
        rec[i] = true;
    }
    float span(int a, int b) const {
        float ms = 0.0f;
        if (on && rec[a] && rec[b]) cudaEventElapsedTime(&ms, ev[a], ev[b]);
        return ms;
    }
    void store(svo_result *r) const {
        if (!on) return;
        cudaEventSynchronize(ev[kDedup]);
        r->n_timings = 9;
        r->timings[0] = span(kStart, kDedup);
        r->timings[1] = span(kStart, kBbox);
        r->timings[2] = span(kBbox, kVox);
        r->timings[3] = span(kVox, kPyr);
        r->timings[4] = span(kPyr, kScan);
        r->timings[5] = span(kCompact0, kCompact);
        r->timings[6] = span(kCompact, kEmit);
        r->timings[7] = span(kEmit, kUnique);
        r->timings[8] = span(kUnique, kDedup);
    }
};

// Device-side meta block read back by the host after the count phase.
struct Meta {
    GridParams gp;
    uint32_t totals[kMaxLevels];
    uint32_t counters[2];  // big-triangle entries, queue cursor
    unsigned long long dups[2];
    uint64_t top_code;
};

int build_one(svo_ctx *ctx, const float *points, int64_t n_points, const int32_t *tris, int64_t n_tris,
              int rx, int ry, int rz, uint32_t flags, cudaStream_t st, svo_result **out) {
    *out = nullptr;
    if (!points || n_points <= 0) return fail(SVO_ERR_EMPTY, "mesh has no vertices");
    if (n_tris < 0 || (!tris && n_points % 3 != 0))
        return fail(SVO_ERR_INVALID_ARGUMENT, "triangle soup needs 3 points per triangle");
    const int64_t nt = tris ? n_tris : n_points / 3;
    if (nt > 0x7FFFFFFF) return fail(SVO_ERR_UNSUPPORTED, "more than 2^31-1 triangles");
    const int res[3] = {rx, ry, rz};
    for (int a = 0; a < 3; ++a)
        if (res[a] < 1 || res[a] > kMaxRes)
            return fail(SVO_ERR_UNSUPPORTED, "resolution %d outside [1, %d]", res[a], kMaxRes);
    SVO_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");

    Scratch S{ctx->pool, st};
    // ---- mesh on the device ----
    const float *d_pts = points;
    const int32_t *d_tris = tris;
    if (!is_device_ptr(points)) {
        float *p = S.get<float>((size_t)n_points * 3);
        if (!p) return cuda_fail(S.err, "alloc points");
        SVO_TRY(cudaMemcpyAsync(p, points, (size_t)n_points * 12, cudaMemcpyHostToDevice, st), "copy points");
        d_pts = p;
    }
    if (tris && nt > 0 && !is_device_ptr(tris)) {
        // validate indices on the host while they are here
        for (int64_t i = 0; i < 3 * nt; ++i)
            if (tris[i] < 0 || tris[i] >= n_points)
                return fail(SVO_ERR_INVALID_ARGUMENT, "triangle index %d out of range", tris[i]);
        int32_t *p = S.get<int32_t>((size_t)nt * 3);
        if (!p) return cuda_fail(S.err, "alloc tris");
        SVO_TRY(cudaMemcpyAsync(p, tris, (size_t)nt * 12, cudaMemcpyHostToDevice, st), "copy tris");
        d_tris = p;
    } else if (tris && nt > 0) {
        std::vector<int32_t> mm(2);
        int32_t *d_mm = S.get<int32_t>(2);
        if (!d_mm) return cuda_fail(S.err, "alloc");
        SVO_TRY(launch_index_range(d_tris, nt * 3, d_mm, st), "index range");
        SVO_TRY(cudaMemcpyAsync(mm.data(), d_mm, 8, cudaMemcpyDeviceToHost, st), "copy");
        SVO_TRY(cudaStreamSynchronize(st), "sync");
        if (mm[0] < 0 || mm[1] >= n_points)
            return fail(SVO_ERR_INVALID_ARGUMENT, "triangle index out of range");
    }

    const Pyramid py = make_pyramid(rx, ry, rz);
    Meta *d_meta = S.get<Meta>(1);
    uint32_t *d_mm = S.get<uint32_t>(8);
    uint64_t *d_bits = S.get<uint64_t>(py.total_words);
    uint32_t *d_cnt = S.get<uint32_t>(py.total_blocks);
    uint32_t *d_pre = S.get<uint32_t>(py.total_blocks + 1);
    unsigned long long *d_scan = S.get<unsigned long long>(scan_scratch_words(py.total_blocks));
    uint32_t *d_done = S.get<uint32_t>(1);
    uint32_t big_cap = (uint32_t)std::min<int64_t>(std::max<int64_t>(2 * nt, 1 << 16), 0x7FFFFFFF);
    uint4 *d_big = S.get<uint4>(big_cap);
    if (S.err != cudaSuccess) return cuda_fail(S.err, "scratch allocation");
    SVO_TRY(cudaMemsetAsync(d_meta, 0, sizeof(Meta), st), "memset");
    SVO_TRY(cudaMemsetAsync(d_done, 0, 4, st), "memset");
    GridParams *d_gp = &d_meta->gp;
    StageTimer tm((flags & SVO_FLAG_TIMINGS) != 0);
    tm.mark(StageTimer::kStart, st);
    SVO_TRY(launch_bbox(d_pts, n_points, rx, ry, rz, d_mm, d_gp, st), "bbox");
    tm.mark(StageTimer::kBbox, st);
    const bool strict = (flags & SVO_FLAG_STRICT_FP) != 0;
    Meta meta;
    for (int attempt = 0; attempt < 2; ++attempt) {
        SVO_TRY(cudaMemsetAsync(d_bits, 0, py.total_words * 8, st), "memset bitmap");
        SVO_TRY(cudaMemsetAsync(d_cnt, 0, py.total_blocks * 4, st), "memset counts");
        SVO_TRY(launch_voxelize(d_pts, d_tris, nt, d_gp, rx, ry, rz, strict, reinterpret_cast<uint32_t *>(d_bits),
                                ctx->tune, d_big, big_cap, d_meta->counters, ctx->num_sms, st),
                "voxelize");
        tm.mark(StageTimer::kVox, st);
        SVO_TRY(launch_pyramid(py, d_bits, d_cnt, d_done, st), "pyramid");
        tm.mark(StageTimer::kPyr, st);
        SVO_TRY(launch_scan(d_cnt, d_pre, py.total_blocks, d_scan, &d_meta->gp.status, st), "scan");
        SVO_TRY(launch_level_totals(py, d_pre, d_meta->totals, st), "totals");
        tm.mark(StageTimer::kScan, st);
        SVO_TRY(cudaMemcpyAsync(&meta, d_meta, sizeof(Meta), cudaMemcpyDeviceToHost, st), "read meta");
        SVO_TRY(cudaStreamSynchronize(st), "count phase");
        if (meta.counters[0] <= big_cap) break;
        // more big-triangle entries than the queue holds: grow it and redo
        big_cap = meta.counters[0];
        d_big = S.get<uint4>(big_cap);
        if (!d_big) return cuda_fail(S.err, "big-triangle queue");
    }
    if (meta.gp.status & kStatusNonFinite) return fail(SVO_ERR_INVALID_ARGUMENT, "non-finite vertex coordinate");
    if (meta.gp.status & kStatusScanTimeout) return fail(SVO_ERR_DEVICE_TIMEOUT, "scan look-back timed out");
    if (meta.counters[0] > big_cap) return fail(SVO_ERR_CUDA, "big-triangle queue overflow");

    // ---- level structure (src/SVO.cu:383-495) ----
    const uint32_t C0 = meta.totals[0];
    if (C0 == 0) return fail(SVO_ERR_EMPTY, "no surface voxels");
    if (C0 == 1) return fail(SVO_ERR_DEGENERATE, "a single surface voxel: the reference's build is undefined");
    int T = -1;
    for (int l = 0; l < py.levels; ++l)
        if (meta.totals[l] == 1) {
            T = l;
            break;
        }
    if (T < 0) return fail(SVO_ERR_CUDA, "octree levels did not converge");
    uint64_t off[kMaxLevels + 1] = {};
    uint64_t n_l[kMaxLevels] = {};
    for (int l = 0; l <= T; ++l) {
        n_l[l] = l < T ? 8ull * meta.totals[l + 1] : 1ull;
        off[l + 1] = off[l] + n_l[l];
    }
    const uint64_t N = off[T + 1];
    if (N >= 0xFFFFFFFFull) return fail(SVO_ERR_UNSUPPORTED, "more than 2^32-2 nodes");

    svo_result *r = new svo_result();
    r->device = ctx->device;
    r->stream = st;
    r->pool = ctx->pool;
    r->depth = T + 1;
    for (int l = 0; l <= T; ++l) r->level_counts.push_back((int64_t)n_l[l]);
    for (int a = 0; a < 3; ++a) {
        r->bbox.min[a] = meta.gp.bbox[a];
        r->bbox.max[a] = meta.gp.bbox[3 + a];
        r->bbox.width[a] = meta.gp.bbox[6 + a];
        r->unit[a] = meta.gp.unit[a];
    }
    r->n_nodes = N;
    const bool ve = !(flags & SVO_FLAG_NO_VERT_EDGE);
    const bool want_keys = !(flags & SVO_FLAG_NO_KEYS);
    cudaError_t err = cudaSuccess;
    r->nodes = pool_alloc<svo_node>(ctx->pool, st, N, err);
    if (ve) {
        r->verts = pool_alloc<svo_vertex>(ctx->pool, st, N * 8, err);
        r->edges = pool_alloc<svo_edge>(ctx->pool, st, N * 12, err);
        r->n_verts = N * 8;
        r->n_edges = N * 12;
    }
    if (want_keys) {
        r->keys = pool_alloc<uint64_t>(ctx->pool, st, C0, err);
        r->n_keys = C0;
    }
    uint64_t koff[kMaxLevels] = {};
    uint64_t ktot = 0;
    for (int l = 1; l <= T; ++l) {
        koff[l] = ktot;
        ktot += meta.totals[l];
    }
    uint64_t *d_K = S.get<uint64_t>(ktot + 1);
    if (err != cudaSuccess || S.err != cudaSuccess) {
        svo_result_free(r);
        return cuda_fail(err != cudaSuccess ? err : S.err, "output allocation");
    }
    int rc = SVO_OK;
    auto check = [&](cudaError_t e, const char *what) {
        if (e != cudaSuccess && rc == SVO_OK) rc = cuda_fail(e, what);
    };
    tm.mark(StageTimer::kCompact0, st);
    check(launch_compact(py, d_bits, d_pre, 1, T + 1, d_K, koff, st), "compact levels");
    if (want_keys) {
        uint64_t k0[kMaxLevels] = {};
        check(launch_compact(py, d_bits, d_pre, 0, 1, r->keys, k0, st), "compact keys");
    }
    tm.mark(StageTimer::kCompact, st);
    EmitParams P{};
    P.T = T;
    P.N = (uint32_t)N;
    P.flags = flags;
    const uint32_t R = 1u << (py.grid_levels - 1);
    float w = 0.0f;
    for (int l = 0; l <= T; ++l) {
        P.lv[l].off = (uint32_t)off[l];
        P.lv[l].n = (uint32_t)n_l[l];
        P.lv[l].K1 = d_K + (l < T ? koff[l + 1] : koff[T]);
        P.lv[l].bits = d_bits + py.woff[l];
        P.lv[l].coff = py.coff[l];
        P.lv[l].side = std::max<uint32_t>(1u, R >> l);
    }
    // widths: unitVoxelSize.x doubled per level (src/SVO.cu:351,483)
    w = meta.gp.unit[0];
    for (int l = 0; l <= T; ++l) {
        P.lv[l].width = w;
        w = w * 2.0f;
    }
    P.pre = d_pre;
    P.gp = d_gp;
    P.nodes = r->nodes;
    P.verts = ve ? r->verts : nullptr;
    P.edges = ve ? r->edges : nullptr;
    P.dups = d_meta->dups;
    check(launch_emit(P, ctx->num_sms, st), "emit");
    tm.mark(StageTimer::kEmit, st);
    check(cudaMemcpyAsync(&meta.top_code, d_K + koff[T], 8, cudaMemcpyDeviceToHost, st), "read top");
    check(cudaMemcpyAsync(meta.dups, d_meta->dups, 16, cudaMemcpyDeviceToHost, st), "read dups");
    check(cudaStreamSynchronize(st), "emit phase");
    if (rc == SVO_OK && (T == 0 || (meta.top_code & 7) != 0))
        rc = fail(SVO_ERR_DEGENERATE, "single top-level node with a non-zero octant: undefined in the reference");
    if (rc == SVO_OK && ve && (meta.dups[0] || meta.dups[1])) {
        // consecutive duplicates present (degenerate widths or absorbed
        // coordinates): compact both arrays as thrust::unique does
        const uint64_t nv = N * 8, ne = N * 12;
        const uint64_t tiles = (std::max(nv, ne) + kUniqueTile - 1) / kUniqueTile;
        uint32_t *tc = S.get<uint32_t>(tiles), *tp = S.get<uint32_t>(tiles + 1);
        unsigned long long *ss = S.get<unsigned long long>(scan_scratch_words(tiles));
        svo_vertex *v2 = meta.dups[0] ? pool_alloc<svo_vertex>(ctx->pool, st, nv, err) : nullptr;
        svo_edge *e2 = meta.dups[1] ? pool_alloc<svo_edge>(ctx->pool, st, ne, err) : nullptr;
        if (S.err != cudaSuccess || err != cudaSuccess) {
            rc = cuda_fail(S.err != cudaSuccess ? S.err : err, "unique scratch");
        } else {
            uint32_t cv = 0, ce = 0;
            if (v2) {
                check(launch_unique_vertices(r->verts, nv, v2, tc, tp, ss, &d_meta->gp.status, st), "unique v");
                check(cudaMemcpyAsync(&cv, tp + (nv + kUniqueTile - 1) / kUniqueTile, 4, cudaMemcpyDeviceToHost, st),
                      "read");
                check(cudaStreamSynchronize(st), "unique v");
            }
            if (e2) {
                check(launch_unique_edges(r->edges, ne, e2, tc, tp, ss, &d_meta->gp.status, st), "unique e");
                check(cudaMemcpyAsync(&ce, tp + (ne + kUniqueTile - 1) / kUniqueTile, 4, cudaMemcpyDeviceToHost, st),
                      "read");
                check(cudaStreamSynchronize(st), "unique e");
            }
            if (v2) {
                cudaFreeAsync(r->verts, st);
                r->verts = v2;
                r->n_verts = cv;
            }
            if (e2) {
                cudaFreeAsync(r->edges, st);
                r->edges = e2;
                r->n_edges = ce;
            }
        }
    }
    tm.mark(StageTimer::kUnique, st);
    if (rc == SVO_OK && (flags & SVO_FLAG_DEDUP)) rc = build_dedup(ctx->pool, st, P, r->n_dedup, r->dedup, ctx->num_sms);
    tm.mark(StageTimer::kDedup, st);
    if (rc == SVO_OK) tm.store(r);
    S.release();
    if (rc != SVO_OK) {
        svo_result_free(r);
        return rc;
    }
    *out = r;
    return SVO_OK;
}

}  // namespace

extern "C" {

const char *svo_last_error(void) { return g_err.c_str(); }

int svo_ctx_create(int device, svo_ctx **out) {
    if (!out) return fail(SVO_ERR_INVALID_ARGUMENT, "null output");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) return fail(SVO_ERR_CUDA, "no CUDA device: %s", cudaGetErrorString(e));
    if (device < 0 || device >= n) return fail(SVO_ERR_INVALID_ARGUMENT, "bad device %d", device);
    SVO_TRY(cudaSetDevice(device), "cudaSetDevice");
    cudaDeviceProp prop;
    SVO_TRY(cudaGetDeviceProperties(&prop, device), "properties");
    if (prop.major < 10) return fail(SVO_ERR_UNSUPPORTED, "needs a Blackwell (sm_100) device, got sm_%d%d", prop.major, prop.minor);
    svo_ctx *c = new svo_ctx();
    c->device = device;
    c->num_sms = prop.multiProcessorCount;
    SVO_TRY(cudaDeviceGetDefaultMemPool(&c->pool, device), "mem pool");
    uint64_t keep = UINT64_MAX;  // keep freed blocks cached for the next build
    SVO_TRY(cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep), "pool attr");
    *out = c;
    return SVO_OK;
}

void svo_ctx_destroy(svo_ctx *ctx) { delete ctx; }

int svo_ctx_set_tuning(svo_ctx *ctx, const svo_tuning *t) {
    if (!ctx || !t) return fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    if (t->warp_max == 0) return fail(SVO_ERR_INVALID_ARGUMENT, "warp_max must be positive");
    ctx->tune.serial_max = t->serial_max;
    ctx->tune.warp_max = t->warp_max;
    ctx->tune.split = t->split;
    return SVO_OK;
}

int svo_ctx_get_tuning(const svo_ctx *ctx, svo_tuning *t) {
    if (!ctx || !t) return fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    t->serial_max = ctx->tune.serial_max;
    t->warp_max = ctx->tune.warp_max;
    t->split = ctx->tune.split;
    return SVO_OK;
}

int svo_build(svo_ctx *ctx, const float *points, int64_t n_points, const int32_t *tris, int64_t n_tris,
              int res_x, int res_y, int res_z, uint32_t flags, void *stream, svo_result **out) {
    if (!ctx || !out) return fail(SVO_ERR_INVALID_ARGUMENT, "null context or output");
    return build_one(ctx, points, n_points, tris, n_tris, res_x, res_y, res_z, flags,
                     static_cast<cudaStream_t>(stream), out);
}

int svo_build_batch(svo_ctx *ctx, const svo_mesh_desc *descs, int n, void *stream, svo_result **out,
                    int *status_out) {
    if (!ctx || (!descs && n > 0) || !out) return fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    int first = SVO_OK;
    for (int i = 0; i < n; ++i) {
        const svo_mesh_desc &d = descs[i];
        int rc = build_one(ctx, d.points, d.n_points, d.tris, d.n_tris, d.res[0], d.res[1], d.res[2], d.flags,
                           static_cast<cudaStream_t>(stream), &out[i]);
        if (status_out) status_out[i] = rc;
        if (rc != SVO_OK && first == SVO_OK) first = rc;
    }
    return first;
}

void svo_result_free(svo_result *r) {
    if (!r) return;
    cudaSetDevice(r->device);
    void *ptrs[] = {r->nodes, r->verts, r->edges, r->keys, r->dedup[0], r->dedup[1], r->dedup[2]};
    for (void *p : ptrs)
        if (p) cudaFreeAsync(p, r->stream);
    cudaStreamSynchronize(r->stream);
    delete r;
}

int svo_result_depth(const svo_result *r) { return r ? r->depth : 0; }
int64_t svo_result_num_nodes(const svo_result *r) { return r ? (int64_t)r->n_nodes : 0; }
int64_t svo_result_num_vertices(const svo_result *r) { return r ? (int64_t)r->n_verts : 0; }
int64_t svo_result_num_edges(const svo_result *r) { return r ? (int64_t)r->n_edges : 0; }
int64_t svo_result_num_keys(const svo_result *r) { return r ? (int64_t)r->n_keys : 0; }

int svo_result_level_counts(const svo_result *r, int64_t *counts, int cap) {
    if (!r) return 0;
    const int n = (int)r->level_counts.size();
    for (int i = 0; i < n && i < cap; ++i) counts[i] = r->level_counts[i];
    return n;
}

int svo_result_bbox(const svo_result *r, svo_aabb *out) {
    if (!r || !out) return fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    *out = r->bbox;
    return SVO_OK;
}

const svo_node *svo_result_nodes_device(const svo_result *r) { return r ? r->nodes : nullptr; }
const svo_vertex *svo_result_vertices_device(const svo_result *r) { return r ? r->verts : nullptr; }
const svo_edge *svo_result_edges_device(const svo_result *r) { return r ? r->edges : nullptr; }
const uint64_t *svo_result_keys_device(const svo_result *r) { return r ? r->keys : nullptr; }

static int copy_out(const svo_result *r, void *dst, const void *src, uint64_t n, int64_t cap, size_t esz,
                    const char *what) {
    if (!r || (!dst && n > 0)) return fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    if ((uint64_t)cap < n) return fail(SVO_ERR_INVALID_ARGUMENT, "%s: capacity %lld < %llu", what, (long long)cap,
                                       (unsigned long long)n);
    if (n == 0) return SVO_OK;
    if (!src) return fail(SVO_ERR_INVALID_ARGUMENT, "%s were not built", what);
    SVO_TRY(cudaSetDevice(r->device), "cudaSetDevice");
    SVO_TRY(cudaMemcpyAsync(dst, src, n * esz, cudaMemcpyDeviceToHost, r->stream), what);
    SVO_TRY(cudaStreamSynchronize(r->stream), what);
    return SVO_OK;
}

int svo_result_copy_nodes(const svo_result *r, svo_node *dst, int64_t cap) {
    return copy_out(r, dst, r ? r->nodes : nullptr, r ? r->n_nodes : 0, cap, sizeof(svo_node), "nodes");
}
int svo_result_copy_vertices(const svo_result *r, svo_vertex *dst, int64_t cap) {
    return copy_out(r, dst, r ? r->verts : nullptr, r ? r->n_verts : 0, cap, sizeof(svo_vertex), "vertices");
}
int svo_result_copy_edges(const svo_result *r, svo_edge *dst, int64_t cap) {
    return copy_out(r, dst, r ? r->edges : nullptr, r ? r->n_edges : 0, cap, sizeof(svo_edge), "edges");
}
int svo_result_copy_keys(const svo_result *r, uint64_t *dst, int64_t cap) {
    return copy_out(r, dst, r ? r->keys : nullptr, r ? r->n_keys : 0, cap, sizeof(uint64_t), "keys");
}
int svo_result_timings(const svo_result *r, float *ms, int cap) {
    if (!r) return 0;
    for (int i = 0; i < r->n_timings && i < cap; ++i) ms[i] = r->timings[i];
    return r->n_timings;
}

int64_t svo_result_num_dedup(const svo_result *r, int kind) {
    return (r && kind >= 0 && kind < 3) ? (int64_t)r->n_dedup[kind] : -1;
}
int svo_result_copy_dedup(const svo_result *r, int kind, uint64_t *dst, int64_t cap) {
    if (!r || kind < 0 || kind > 2) return fail(SVO_ERR_INVALID_ARGUMENT, "bad kind");
    return copy_out(r, dst, r->dedup[kind], r->n_dedup[kind], cap, sizeof(uint64_t), "dedup keys");
}

int svo_write_tree(const svo_result *r, const char *path) {
    if (!r || !path) return fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    std::vector<svo_node> h(r->n_nodes);
    int rc = svo_result_copy_nodes(r, h.data(), (int64_t)h.size());
    if (rc) return rc;
    return svo_write_tree_nodes(h.data(), (int64_t)h.size(), path);
}

int svo_write_voxels(const svo_result *r, const char *path) {
    if (!r || !path) return fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    std::vector<uint64_t> k(r->n_keys);
    int rc = svo_result_copy_keys(r, k.data(), (int64_t)k.size());
    if (rc) return rc;
    return svo::host::write_voxels(k.data(), (int64_t)k.size(), r->bbox.min, r->unit[0], path);
}

}  // extern "C"

namespace svo::host {
void set_error(const char *msg) { g_err = msg; }
}  // namespace svo::host

namespace svo {
static std::atomic<int64_t> g_launches{0};
void count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
}  // namespace svo

extern "C" int64_t svo_kernel_launches(void) { return svo::g_launches.load(std::memory_order_relaxed); }
