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
#include <mutex>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "svo_internal.h"
#include "svo_host.h"

using namespace svo;

// Extra streams over which an emission wave spreads its per-mesh launches
// (fork from and join back to the build stream with events).
struct AuxStreams {
    static constexpr int kCount = 3;
    cudaStream_t s[kCount] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[kCount] = {};
};

struct svo_ctx {
    int device = 0;
    int num_sms = 148;
    cudaMemPool_t pool = nullptr;      // per-build scratch
    cudaMemPool_t out_pool = nullptr;  // result arrays, kept apart so scratch never splits their blocks
    VoxTuning tune;                    // read and written under tune_mu
    std::mutex tune_mu;
    std::mutex aux_mu;                 // builds on other threads take sets of their own
    std::vector<AuxStreams *> aux_free, aux_all;
};

// One device block that holds the output arrays of several results (a wave of
// a batch); freed with the last of them.
struct svo_arena {
    void *base = nullptr;
    std::atomic<int> refs{0};
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
    svo_arena *arena = nullptr;  // holds nodes/verts/edges/keys when set
    uint32_t own = 0x7F;         // bit i: array i of {nodes, verts, edges, keys, dedup x3} is freed on its own
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
        err = pool_malloc(&p, std::max<size_t>(count * sizeof(T), 256), pool, st);
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
    err = pool_malloc(&p, std::max<size_t>(count * sizeof(T), 256), pool, st);
    return static_cast<T *>(p);
}

// CUDA events at stage boundaries (SVO_FLAG_TIMINGS).
struct StageTimer {
    enum { kStart, kBbox, kVox, kPyr, kScan, kCompact0, kCompact, kEmit, kUnique, kDedup0, kDedup, kEnd, kN };
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
};

// ---------------------------------------------------------------------------
// Batches.  Phase A (svo_batch_create) runs for every mesh at once: bounding
// cube, voxelization, bitmap pyramid, one scan over all block counts, level
// totals, then one small device->host read.  Phase B (svo_batch_emit) writes
// the octrees of any subset of the meshes in one compaction launch and one
// emission launch.  svo_build is a batch of one.
// ---------------------------------------------------------------------------
struct MeshHost {
    const float *h_pts = nullptr;      // caller's pointers
    const int32_t *h_tris = nullptr;
    int64_t n_pts = 0, n_tris = 0;     // n_tris: triangles (soup: n_pts / 3)
    int res[3] = {0, 0, 0};
    const float *d_pts = nullptr;      // device copies or the caller's device pointers
    const int32_t *d_tris = nullptr;
    bool tris_on_device = false;
    Pyramid py;
    uint64_t bits_off = 0, cnt_off = 0;  // into the batch's bitmap / count buffers
    uint32_t cta0 = 0;                   // first pyramid CTA (level-0 region) in the batch
    int status = SVO_OK;
    std::string error;
    GridParams gp{};
    uint32_t totals[kMaxLevels] = {};
    int T = -1;
    uint64_t n_l[kMaxLevels] = {}, off[kMaxLevels + 1] = {};
    uint64_t N = 0;
    bool emitted = false;
};

// Layout of the small per-batch meta block (device), read back after phase A.
struct MetaLayout {
    size_t counters = 0, gp = 0, totals = 0, mm = 0, done = 0, imm = 0, bytes = 0;
    explicit MetaLayout(int n) {
        auto take = [&](size_t b) {
            const size_t o = (bytes + 255) / 256 * 256;
            bytes = o + b;
            return o;
        };
        counters = take(4 * sizeof(uint32_t));
        gp = take(sizeof(GridParams) * n);
        totals = take(sizeof(uint32_t) * kMaxLevels * n);
        mm = take(sizeof(uint32_t) * 8 * n);
        done = take(sizeof(uint32_t) * n);
        imm = take(sizeof(int32_t) * 2 * n);
    }
};

__global__ void k_meta_init(uint32_t *mm, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int a = 0; a < 3; ++a) {
        mm[8 * i + a] = 0xFFFFFFFFu;
        mm[8 * i + 3 + a] = 0u;
    }
}

// top_codes[i] = *ptrs[i] (the single code of each mesh's top level)
__global__ void k_gather_top(const uint64_t *const *ptrs, int n, uint64_t *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = *ptrs[i];
}

}  // namespace

struct svo_batch {
    svo_ctx *ctx = nullptr;
    cudaStream_t st = nullptr;
    uint32_t flags = 0;
    VoxTuning tune;                         // the voxelizer split this batch runs with
    std::vector<MeshHost> m;
    std::vector<int> live;                  // meshes with device work
    std::vector<void *> allocs;             // phase A buffers (pool)
    uint64_t *bits = nullptr;
    uint32_t *cnt = nullptr, *pre = nullptr;
    uint8_t *rflag = nullptr;               // level-0 regions that triangles reach (one byte per pyramid CTA)
    unsigned char *meta = nullptr;
    MeshDev *d_mesh = nullptr;
    std::vector<MeshDev> h_mesh;
    uint64_t total_blocks = 0;
    float timings_a[5] = {};                // total, bbox, voxelize, pyramid, scan
    bool timed = false;
};

namespace {

template <class T>
T *batch_alloc(svo_batch *b, size_t count, cudaError_t &err) {
    T *p = pool_alloc<T>(b->ctx->pool, b->st, count, err);
    if (p) b->allocs.push_back(p);
    return p;
}

void batch_release(svo_batch *b) {
    for (void *p : b->allocs) cudaFreeAsync(p, b->st);
    b->allocs.clear();
}

int mesh_error(MeshHost &mh, int code, const char *msg) {
    mh.status = code;
    mh.error = msg;
    return code;
}

// Offsets of arrays laid out one after another in one block (256-byte aligned):
// fewer pool allocations per build.
struct Layout {
    size_t bytes = 0;
    template <class T>
    size_t add(size_t count) {
        const size_t at = bytes;
        bytes += (std::max<size_t>(count * sizeof(T), 1) + 255) / 256 * 256;
        return at;
    }
};

// Small host tables packed into one buffer, uploaded with one copy.
struct HostPack {
    std::vector<unsigned char> buf;
    template <class T>
    size_t add(const T *src, size_t count) {
        const size_t at = (buf.size() + 15) / 16 * 16;
        buf.resize(at + count * sizeof(T));
        if (count) std::memcpy(buf.data() + at, src, count * sizeof(T));
        return at;
    }
    template <class T>
    size_t add(const std::vector<T> &v) { return add(v.data(), v.size()); }
};

template <class T>
cudaError_t upload(T *dst, const std::vector<T> &src, cudaStream_t st) {
    if (src.empty()) return cudaSuccess;
    return cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, st);
}

// Phase A.  Returns SVO_OK when the batch itself works (individual meshes
// may still carry an error status).
int batch_phase_a(svo_batch *b) {
    svo::host::TraceRange trace("svo: counting phase (voxelize, pyramid, scan)");
    svo_ctx *ctx = b->ctx;
    cudaStream_t st = b->st;
    SVO_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaError_t err = cudaSuccess;
    // ---- validation and mesh data on the device ----
    for (int i = 0; i < (int)b->m.size(); ++i) {
        MeshHost &mh = b->m[i];
        if (!mh.h_pts || mh.n_pts <= 0) {
            mesh_error(mh, SVO_ERR_EMPTY, "mesh has no vertices");
            continue;
        }
        if (mh.n_tris < 0 || (!mh.h_tris && mh.n_pts % 3 != 0)) {
            mesh_error(mh, SVO_ERR_INVALID_ARGUMENT, "triangle soup needs 3 points per triangle");
            continue;
        }
        if (!mh.h_tris) mh.n_tris = mh.n_pts / 3;
        if (mh.n_tris > 0x7FFFFFFF) {
            mesh_error(mh, SVO_ERR_UNSUPPORTED, "more than 2^31-1 triangles");
            continue;
        }
        bool bad_res = false;
        for (int a = 0; a < 3; ++a) bad_res |= mh.res[a] < 1 || mh.res[a] > kMaxRes;
        if (bad_res) {
            char msg[96];
            snprintf(msg, sizeof(msg), "resolution outside [1, %d]", kMaxRes);
            mesh_error(mh, SVO_ERR_UNSUPPORTED, msg);
            continue;
        }
        // face indices are checked on the device by the kernels that read them
        // (kStatusBadIndex, reported with the level totals)
        if (mh.h_tris && mh.n_tris > 0) mh.tris_on_device = is_device_ptr(mh.h_tris);
        if (is_device_ptr(mh.h_pts)) {
            mh.d_pts = mh.h_pts;
        } else {
            float *p = batch_alloc<float>(b, (size_t)mh.n_pts * 3, err);
            if (!p) return cuda_fail(err, "alloc points");
            SVO_TRY(cudaMemcpyAsync(p, mh.h_pts, (size_t)mh.n_pts * 12, cudaMemcpyHostToDevice, st), "copy points");
            mh.d_pts = p;
        }
        if (mh.h_tris && mh.n_tris > 0) {
            if (mh.tris_on_device) {
                mh.d_tris = mh.h_tris;
            } else {
                int32_t *p = batch_alloc<int32_t>(b, (size_t)mh.n_tris * 3, err);
                if (!p) return cuda_fail(err, "alloc tris");
                SVO_TRY(cudaMemcpyAsync(p, mh.h_tris, (size_t)mh.n_tris * 12, cudaMemcpyHostToDevice, st),
                        "copy tris");
                mh.d_tris = p;
            }
        }
        b->live.push_back(i);
    }
    const int n = (int)b->live.size();
    if (n == 0) return SVO_OK;
    const MetaLayout ml(n);
    b->meta = batch_alloc<unsigned char>(b, ml.bytes, err);
    if (!b->meta) return cuda_fail(err, "alloc meta");
    // ---- layout ----
    uint64_t words = 0, blocks = 0, tris = 0;
    uint32_t ctas = 0, bblocks = 0;
    std::vector<uint64_t> tri_off(n + 1);
    std::vector<uint32_t> cta_off(n + 1), bbox_off(n + 1);
    for (int k = 0; k < n; ++k) {
        MeshHost &mh = b->m[b->live[k]];
        mh.py = make_pyramid(mh.res[0], mh.res[1], mh.res[2]);
        mh.bits_off = words;
        mh.cnt_off = blocks;
        words += (mh.py.total_words + 31) / 32 * 32;
        blocks += mh.py.total_blocks;
        tri_off[k] = tris;
        cta_off[k] = ctas;
        mh.cta0 = ctas;
        bbox_off[k] = bblocks;
        tris += (uint64_t)mh.n_tris;
        ctas += mh.py.ctas;
        bblocks += bbox_blocks(mh.n_pts);
    }
    tri_off[n] = tris;
    cta_off[n] = ctas;
    bbox_off[n] = bblocks;
    b->total_blocks = blocks;
    // the batch's scratch arrays and its mesh tables: one block, one upload
    uint32_t big_cap = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(2 * tris, 1 << 16), 0x7FFFFFFFu);
    HostPack tables;  // mesh table, triangle / CTA / bbox-block offsets (filled below)
    auto a16 = [](size_t x) { return (x + 15) / 16 * 16; };
    const size_t t_bytes = a16(sizeof(MeshDev) * n) + a16(8 * (size_t)(n + 1)) + a16(4 * (size_t)(n + 1)) + 4 * (size_t)(n + 1);
    Layout lay;
    const size_t o_bits = lay.add<uint64_t>(words), o_cnt = lay.add<uint32_t>(blocks),
                 o_pre = lay.add<uint32_t>(blocks + 1), o_scan = lay.add<unsigned long long>(scan_scratch_words(blocks)),
                 o_big = lay.add<uint4>(big_cap), o_small = lay.add<uint64_t>(std::max<uint64_t>(tris, 1)),
                 o_rflag = lay.add<uint8_t>(std::max<uint32_t>(ctas, 1));
    const size_t o_tables = lay.add<unsigned char>(t_bytes);
    unsigned char *blk = batch_alloc<unsigned char>(b, lay.bytes, err);
    if (err != cudaSuccess || !blk) return cuda_fail(err, "batch scratch");
    b->bits = reinterpret_cast<uint64_t *>(blk + o_bits);
    b->cnt = reinterpret_cast<uint32_t *>(blk + o_cnt);
    b->pre = reinterpret_cast<uint32_t *>(blk + o_pre);
    unsigned long long *scan = reinterpret_cast<unsigned long long *>(blk + o_scan);
    uint4 *big = reinterpret_cast<uint4 *>(blk + o_big);
    uint64_t *small = reinterpret_cast<uint64_t *>(blk + o_small);
    uint8_t *rflag = b->rflag = blk + o_rflag;
    GridParams *gp = reinterpret_cast<GridParams *>(b->meta + ml.gp);
    uint32_t *totals = reinterpret_cast<uint32_t *>(b->meta + ml.totals);
    uint32_t *mm = reinterpret_cast<uint32_t *>(b->meta + ml.mm);
    uint32_t *done = reinterpret_cast<uint32_t *>(b->meta + ml.done);
    uint32_t *counters = reinterpret_cast<uint32_t *>(b->meta + ml.counters);
    b->h_mesh.assign(n, MeshDev{});
    for (int k = 0; k < n; ++k) {
        const MeshHost &mh = b->m[b->live[k]];
        MeshDev &d = b->h_mesh[k];
        d.pts = mh.d_pts;
        d.tris = mh.d_tris;
        d.n_pts = mh.n_pts;
        d.n_tris = mh.n_tris;
        for (int a = 0; a < 3; ++a) d.res[a] = mh.res[a];
        d.gp = gp + k;
        d.mm = mm + 8 * k;
        d.bits = b->bits + mh.bits_off;
        d.cnt = b->cnt + mh.cnt_off;
        d.pre = b->pre + mh.cnt_off;
        d.totals = totals + kMaxLevels * k;
        d.done = done + k;
        d.py = mh.py;
        d.regions = mh.py.words[0] >= kRegionWords ? 1 : 0;
    }
    const size_t p_mesh = tables.add(b->h_mesh), p_tri = tables.add(tri_off), p_cta = tables.add(cta_off),
                 p_bbox = tables.add(bbox_off);
    unsigned char *dt = blk + o_tables;
    b->d_mesh = reinterpret_cast<MeshDev *>(dt + p_mesh);
    const uint64_t *d_tri_off = reinterpret_cast<const uint64_t *>(dt + p_tri);
    const uint32_t *d_cta_off = reinterpret_cast<const uint32_t *>(dt + p_cta);
    const uint32_t *d_bbox_off = reinterpret_cast<const uint32_t *>(dt + p_bbox);
    SVO_TRY(cudaMemcpyAsync(dt, tables.buf.data(), tables.buf.size(), cudaMemcpyHostToDevice, st), "upload meshes");
    const BatchDev bd{b->d_mesh, n, d_tri_off, d_cta_off, d_bbox_off, rflag};
    const bool strict = (b->flags & SVO_FLAG_STRICT_FP) != 0;
    StageTimer tm((b->flags & SVO_FLAG_TIMINGS) != 0);
    for (int attempt = 0; attempt < 2; ++attempt) {
        tm.mark(StageTimer::kStart, st);
        SVO_TRY(cudaMemsetAsync(b->meta, 0, ml.imm, st), "memset meta");
        k_meta_init<<<(n + 127) / 128, 128, 0, st>>>(mm, n);
        count_launches(1);
        SVO_TRY(launch_bbox(bd, bblocks, st), "bbox");
        tm.mark(StageTimer::kBbox, st);
        SVO_TRY(cudaMemsetAsync(rflag, 0, std::max<uint32_t>(ctas, 1), st), "memset regions");
        SVO_TRY(cudaMemsetAsync(b->cnt, 0, blocks * 4, st), "memset counts");
        SVO_TRY(launch_regions(bd, (int64_t)tris, ctas, ctx->num_sms, st), "zero bitmaps");
        SVO_TRY(launch_voxelize(bd, (int64_t)tris, strict, b->tune, big, big_cap, counters, ctx->num_sms, st,
                                small),
                "voxelize");
        tm.mark(StageTimer::kVox, st);
        SVO_TRY(launch_pyramid(bd, ctas, ctx->num_sms, st), "pyramid");
        tm.mark(StageTimer::kPyr, st);
        SVO_TRY(launch_scan(b->cnt, b->pre, blocks, scan, counters + 2, st), "scan");
        SVO_TRY(launch_level_totals(bd, st), "totals");
        tm.mark(StageTimer::kScan, st);
        std::vector<unsigned char> h(ml.imm);
        SVO_TRY(cudaMemcpyAsync(h.data(), b->meta, ml.imm, cudaMemcpyDeviceToHost, st), "read meta");
        SVO_TRY(cudaStreamSynchronize(st), "count phase");
        const uint32_t *hc = reinterpret_cast<const uint32_t *>(h.data() + ml.counters);
        if (hc[2] & kStatusScanTimeout) return fail(SVO_ERR_DEVICE_TIMEOUT, "scan look-back timed out");
        if (hc[0] > big_cap) {  // more big-triangle entries than the queue holds: grow it, redo
            big_cap = hc[0];
            big = batch_alloc<uint4>(b, big_cap, err);
            if (!big) return cuda_fail(err, "big-triangle queue");
            continue;
        }
        for (int k = 0; k < n; ++k) {
            MeshHost &mh = b->m[b->live[k]];
            std::memcpy(&mh.gp, h.data() + ml.gp + sizeof(GridParams) * k, sizeof(GridParams));
            std::memcpy(mh.totals, h.data() + ml.totals + sizeof(uint32_t) * kMaxLevels * k, sizeof(mh.totals));
        }
        break;
    }
    if (tm.on) {
        b->timed = true;
        b->timings_a[0] = tm.span(StageTimer::kStart, StageTimer::kScan);
        b->timings_a[1] = tm.span(StageTimer::kStart, StageTimer::kBbox);
        b->timings_a[2] = tm.span(StageTimer::kBbox, StageTimer::kVox);
        b->timings_a[3] = tm.span(StageTimer::kVox, StageTimer::kPyr);
        b->timings_a[4] = tm.span(StageTimer::kPyr, StageTimer::kScan);
    }
    // ---- level structure per mesh (src/SVO.cu:383-495) ----
    for (int k = 0; k < n; ++k) {
        MeshHost &mh = b->m[b->live[k]];
        if (mh.gp.status & kStatusBadIndex) {
            mesh_error(mh, SVO_ERR_INVALID_ARGUMENT, "triangle index out of range");
            continue;
        }
        if (mh.gp.status & kStatusNonFinite) {
            mesh_error(mh, SVO_ERR_INVALID_ARGUMENT, "non-finite vertex coordinate");
            continue;
        }
        const uint32_t C0 = mh.totals[0];
        if (C0 == 0) {
            mesh_error(mh, SVO_ERR_EMPTY, "no surface voxels");
            continue;
        }
        if (C0 == 1) {
            mesh_error(mh, SVO_ERR_DEGENERATE, "a single surface voxel: the reference's build is undefined");
            continue;
        }
        mh.T = -1;
        for (int l = 0; l < mh.py.levels; ++l)
            if (mh.totals[l] == 1) {
                mh.T = l;
                break;
            }
        if (mh.T < 0) {
            mesh_error(mh, SVO_ERR_CUDA, "octree levels did not converge");
            continue;
        }
        for (int l = 0; l <= mh.T; ++l) {
            mh.n_l[l] = l < mh.T ? 8ull * mh.totals[l + 1] : 1ull;
            mh.off[l + 1] = mh.off[l] + mh.n_l[l];
        }
        mh.N = mh.off[mh.T + 1];
        if (mh.N >= 0xFFFFFFFFull) mesh_error(mh, SVO_ERR_UNSUPPORTED, "more than 2^32-2 nodes");
    }
    return SVO_OK;
}

// Bytes of the outputs of one mesh.
uint64_t output_bytes(const MeshHost &mh, uint32_t flags) {
    uint64_t b = mh.N * sizeof(svo_node);
    if (!(flags & SVO_FLAG_NO_VERT_EDGE)) b += mh.N * (8 * sizeof(svo_vertex) + 12 * sizeof(svo_edge));
    if (!(flags & SVO_FLAG_NO_KEYS)) b += (uint64_t)mh.totals[0] * 8;
    return b;
}

AuxStreams *aux_acquire(svo_ctx *ctx) {
    std::lock_guard<std::mutex> lk(ctx->aux_mu);
    if (!ctx->aux_free.empty()) {
        AuxStreams *a = ctx->aux_free.back();
        ctx->aux_free.pop_back();
        return a;
    }
    // The highest stream priority: when a wave's dedup runs beside its
    // emission, the block scheduler places the dedup kernels' CTAs ahead of
    // the emission grid's pending ones instead of after all of them.
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    auto *a = new AuxStreams();
    bool ok = cudaEventCreateWithFlags(&a->fork, cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; i < AuxStreams::kCount && ok; ++i)
        ok = cudaStreamCreateWithPriority(&a->s[i], cudaStreamNonBlocking, greatest) == cudaSuccess &&
             cudaEventCreateWithFlags(&a->join[i], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        for (int i = 0; i < AuxStreams::kCount; ++i) {
            if (a->s[i]) cudaStreamDestroy(a->s[i]);
            if (a->join[i]) cudaEventDestroy(a->join[i]);
        }
        if (a->fork) cudaEventDestroy(a->fork);
        delete a;
        return nullptr;
    }
    ctx->aux_all.push_back(a);
    return a;
}

void aux_release(svo_ctx *ctx, AuxStreams *a) {
    if (!a) return;
    std::lock_guard<std::mutex> lk(ctx->aux_mu);
    ctx->aux_free.push_back(a);
}

size_t arena_round(size_t b) { return (b + 255) / 256 * 256; }

template <class T>
T *arena_take(unsigned char *&at, uint64_t count) {
    T *p = reinterpret_cast<T *>(at);
    at += arena_round(count * sizeof(T));
    return p;
}

// Meshes of at least this many nodes are emitted by a launch of their own.
#ifndef SVO_OWN_EMIT_NODES
#define SVO_OWN_EMIT_NODES (1ull << 17)
#endif
constexpr uint64_t kOwnEmitNodes = SVO_OWN_EMIT_NODES;

// Phase B for meshes [first, first + count).
int batch_phase_b(svo_batch *b, int first, int count, svo_result **out, int *status_out) {
    svo::host::TraceRange trace("svo: emission wave (codes, nodes, vertices, edges, dedup)");
    svo_ctx *ctx = b->ctx;
    cudaStream_t st = b->st;
    const uint32_t flags = b->flags;
    const bool ve = !(flags & SVO_FLAG_NO_VERT_EDGE);
    const bool want_keys = !(flags & SVO_FLAG_NO_KEYS);
    SVO_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    std::vector<int> wave;   // batch mesh indices emitted now
    std::vector<int> dev_k;  // their index in b->live
    for (int i = first; i < first + count; ++i) {
        out[i - first] = nullptr;
        MeshHost &mh = b->m[i];
        if (mh.status == SVO_OK && mh.emitted) mesh_error(mh, SVO_ERR_INVALID_ARGUMENT, "mesh already emitted");
        if (mh.status != SVO_OK) continue;
        wave.push_back(i);
        dev_k.push_back((int)(std::find(b->live.begin(), b->live.end(), i) - b->live.begin()));
    }
    const int n = (int)wave.size();
    std::vector<svo_result *> res(n, nullptr);
    int rc = SVO_OK;
    auto check = [&](cudaError_t e, const char *what) {
        if (e != cudaSuccess && rc == SVO_OK) rc = cuda_fail(e, what);
    };
    Scratch S{ctx->pool, st};
    StageTimer tm((flags & SVO_FLAG_TIMINGS) != 0);
    auto free_results = [&]() {
        for (svo_result *&r : res) {
            svo_result_free(r);
            r = nullptr;
        }
    };
    if (n > 0) {
        // The wave body: an error return from it still reaches the per-mesh
        // status loop below, which marks every mesh of the wave as failed.
        const int wave_rc = [&]() -> int {
            cudaError_t err = cudaSuccess;
            // The dedup keys read only the bitmaps and code lists: they run on
            // a stream of their own, forked here, where their first step (the
            // level-1 candidate bitmap, from the bitmaps alone) runs while the
            // host prepares the wave; the rest follows the code lists and runs
            // beside the emission.  The wave joins it before returning.
            const bool dd = (flags & SVO_FLAG_DEDUP) != 0;
            AuxStreams *dset = dd ? aux_acquire(ctx) : nullptr;
            const cudaStream_t ds = dset ? dset->s[0] : st;
            auto join_dedup = [&]() {
                if (!dset) return;
                check(cudaEventRecord(dset->join[0], ds), "join");
                check(cudaStreamWaitEvent(st, dset->join[0], 0), "join");
                aux_release(ctx, dset);
                dset = nullptr;
            };
            std::vector<DedupRun *> druns(n, nullptr);
            std::vector<int> drc(n, SVO_OK);
            std::vector<std::string> dmsg(n);
            std::vector<char> dstarted(n, 0);
            auto dedup_start = [&](int j) {  // the first step of mesh j's dedup (bitmaps only)
                dstarted[j] = 1;
                const MeshHost &mh = b->m[wave[j]];
                const MeshDev &md = b->h_mesh[dev_k[j]];
                const uint32_t R = 1u << (mh.py.grid_levels - 1);
                const uint64_t *bits[kMaxLevels];
                uint32_t sides[kMaxLevels];
                for (int l = 0; l <= mh.T && l < kMaxLevels; ++l) {
                    bits[l] = md.bits + mh.py.woff[l];
                    sides[l] = std::max<uint32_t>(1u, R >> l);
                }
                drc[j] = dedup_begin(ctx->pool, ds, mh.T, bits, sides, ctx->num_sms, &druns[j]);
                if (drc[j] != SVO_OK) dmsg[j] = svo_last_error();
            };
            struct DedupGuard {  // on every exit: unfinished runs freed, the dedup stream joined
                std::vector<DedupRun *> &runs;
                decltype(join_dedup) &join;
                ~DedupGuard() {
                    for (DedupRun *&r : runs) {
                        dedup_abort(r);
                        r = nullptr;
                    }
                    join();
                }
            } dguard{druns, join_dedup};
            if (dd) {
                if (dset) {
                    check(cudaEventRecord(dset->fork, st), "fork");
                    check(cudaStreamWaitEvent(ds, dset->fork, 0), "fork");
                }
                tm.mark(StageTimer::kDedup0, ds);
                // early starts hold their candidate bitmaps (R^3 / 8 bytes each) until their
                // finish: up to 4 GiB of them; the other meshes start just before they finish
                uint64_t early = 0;
                for (int j = 0; j < n; ++j) {
                    const MeshHost &mh = b->m[wave[j]];
                    const uint64_t R = 1ull << (mh.py.grid_levels - 1);
                    if (j > 0 && early + R * R * R / 8 > (4ull << 30)) break;
                    early += R * R * R / 8;
                    dedup_start(j);
                }
            }
            // outputs, code lists, job tables
            std::vector<CompactJob> jobs;
            std::vector<uint64_t> word_off(1, 0);
            std::vector<CompactJob> region_jobs;  // region-mode meshes' levels 1-2
            std::vector<uint32_t> region_counts;
            std::vector<KeyJob> kjobs;
            std::vector<uint64_t> blk_off(1, 0);
            std::vector<EmitParams> ep(n);
            std::vector<const uint64_t *> top_ptr(n);
            uint64_t ktot = 0;
            std::vector<uint64_t> kbase(n);
            for (int j = 0; j < n; ++j) {
                const MeshHost &mh = b->m[wave[j]];
                kbase[j] = ktot;
                for (int l = 1; l <= mh.T; ++l) ktot += mh.totals[l];
            }
            // per-word ranks of levels >= 1 (k_compact writes them, rank lookups read them)
            uint64_t wtot = 0;
            std::vector<uint64_t> wbase(n);
            for (int j = 0; j < n; ++j) {
                const MeshHost &mh = b->m[wave[j]];
                wbase[j] = wtot;
                wtot += mh.py.woff[mh.T] + mh.py.words[mh.T] - mh.py.woff[1];
            }
            // code lists, word ranks, duplicate counts, top codes: one block
            Layout wl;
            const size_t o_K = wl.add<uint64_t>(ktot + 1), o_WP = wl.add<uint32_t>(wtot + 1),
                         o_dups = wl.add<unsigned long long>(2 * (size_t)n), o_top = wl.add<uint64_t>(n);
            unsigned char *wblk = S.get<unsigned char>(wl.bytes);
            if (!wblk) return cuda_fail(S.err, "wave scratch");
            uint64_t *K = reinterpret_cast<uint64_t *>(wblk + o_K);
            uint32_t *WP = reinterpret_cast<uint32_t *>(wblk + o_WP);
            unsigned long long *dups = reinterpret_cast<unsigned long long *>(wblk + o_dups);
            uint64_t *top = reinterpret_cast<uint64_t *>(wblk + o_top);
            check(cudaMemsetAsync(dups, 0, 16 * (size_t)n, st), "memset");
            // one block for the output arrays of the whole wave
            size_t arena_bytes = 0;
            for (int j = 0; j < n; ++j) {
                const MeshHost &mh = b->m[wave[j]];
                arena_bytes += arena_round(mh.N * sizeof(svo_node));
                if (ve) arena_bytes += arena_round(mh.N * 8 * sizeof(svo_vertex)) + arena_round(mh.N * 12 * sizeof(svo_edge));
                if (want_keys) arena_bytes += arena_round((size_t)mh.totals[0] * 8);
            }
            svo_arena *arena = new svo_arena();
            arena->refs = 1;  // the wave's own reference, dropped below
            if (pool_malloc(&arena->base, std::max<size_t>(arena_bytes, 256), ctx->out_pool, st) != cudaSuccess) {
                delete arena;
                cudaGetLastError();
                return fail(SVO_ERR_OUT_OF_MEMORY, "wave outputs: %zu bytes", arena_bytes);
            }
            unsigned char *arena_at = static_cast<unsigned char *>(arena->base);
            auto drop_arena = [&]() {
                if (arena && arena->refs.fetch_sub(1) == 1) {
                    cudaFreeAsync(arena->base, st);
                    delete arena;
                }
                arena = nullptr;
            };
            for (int j = 0; j < n; ++j) {
                const MeshHost &mh = b->m[wave[j]];
                const MeshDev &md = b->h_mesh[dev_k[j]];
                svo_result *r = new svo_result();
                res[j] = r;
                r->device = ctx->device;
                r->stream = st;
                r->pool = ctx->pool;
                r->depth = mh.T + 1;
                for (int l = 0; l <= mh.T; ++l) r->level_counts.push_back((int64_t)mh.n_l[l]);
                for (int a = 0; a < 3; ++a) {
                    r->bbox.min[a] = mh.gp.bbox[a];
                    r->bbox.max[a] = mh.gp.bbox[3 + a];
                    r->bbox.width[a] = mh.gp.bbox[6 + a];
                    r->unit[a] = mh.gp.unit[a];
                }
                r->n_nodes = mh.N;
                r->nodes = arena_take<svo_node>(arena_at, mh.N);
                if (ve) {
                    r->verts = arena_take<svo_vertex>(arena_at, mh.N * 8);
                    r->edges = arena_take<svo_edge>(arena_at, mh.N * 12);
                    r->n_verts = mh.N * 8;
                    r->n_edges = mh.N * 12;
                }
                if (want_keys) {
                    r->keys = arena_take<uint64_t>(arena_at, mh.totals[0]);
                    r->n_keys = mh.totals[0];
                }
                r->arena = arena;
                r->own = 0x70;
                arena->refs.fetch_add(1);
                // compaction jobs: levels 1..T into K, level 0 into the keys
                CompactJob job{};
                job.bits = md.bits;
                job.pre = md.pre;
                job.py = mh.py;
                job.l0 = 1;
                job.l1 = mh.T + 1;
                job.out = K + kbase[j];
                job.wpre = WP + wbase[j];
                uint64_t ko = 0;
                for (int l = 1; l <= mh.T; ++l) {
                    job.koff[l] = ko;
                    ko += mh.totals[l];
                }
                if (mh.py.words[0] >= kRegionWords) {
                    // region mode: levels 1-2 region by region (k_compact_regions);
                    // level 3 words of unflagged regions are empty, not read
                    job.rflag = b->rflag + mh.cta0;
                    region_jobs.push_back(job);
                    region_counts.push_back(mh.py.ctas);
                    job.l0 = 3;
                }
                jobs.push_back(job);
                word_off.push_back(word_off.back() + mh.py.woff[mh.T] + mh.py.words[mh.T] - mh.py.woff[job.l0]);
                if (want_keys && mh.T >= 3) {
                    // the level-3 code list is the list of non-empty level-0 blocks
                    kjobs.push_back(KeyJob{md.bits, md.pre, job.out + job.koff[3], r->keys});
                    blk_off.push_back(blk_off.back() + mh.totals[3]);
                } else if (want_keys) {
                    CompactJob k0 = job;
                    k0.l0 = 0;
                    k0.l1 = 1;
                    k0.out = r->keys;
                    k0.wpre = nullptr;
                    std::memset(k0.koff, 0, sizeof(k0.koff));
                    jobs.push_back(k0);
                    word_off.push_back(word_off.back() + mh.py.words[0]);
                }
                // emission parameters
                EmitParams &P = ep[j];
                P.T = mh.T;
                P.N = (uint32_t)mh.N;
                P.flags = flags;
                const uint32_t R = 1u << (mh.py.grid_levels - 1);
                float w = mh.gp.unit[0];  // unitVoxelSize.x doubled per level (src/SVO.cu:351,483)
                for (int l = 0; l <= mh.T; ++l) {
                    P.lv[l].off = (uint32_t)mh.off[l];
                    P.lv[l].n = (uint32_t)mh.n_l[l];
                    P.lv[l].K1 = job.out + (l < mh.T ? job.koff[l + 1] : job.koff[mh.T]);
                    P.lv[l].bits = md.bits + mh.py.woff[l];
                    P.lv[l].wpre = l >= 1 ? job.wpre + (mh.py.woff[l] - mh.py.woff[1]) : nullptr;
                    P.lv[l].coff = mh.py.coff[l];
                    P.lv[l].side = std::max<uint32_t>(1u, R >> l);
                    P.lv[l].width = w;
                    w = w * 2.0f;
                }
                P.pre = md.pre;
                P.gp = md.gp;
                P.nodes = r->nodes;
                P.verts = ve ? r->verts : nullptr;
                P.edges = ve ? r->edges : nullptr;
                P.dups = dups + 2 * j;
                top_ptr[j] = job.out + job.koff[mh.T];
            }
            if (err != cudaSuccess) {
                free_results();
                drop_arena();
                return cuda_fail(err, "output allocation");
            }
            // the wave's job tables: one block, one upload
            HostPack wt;
            const size_t p_jobs = wt.add(jobs), p_woff = wt.add(word_off), p_kjobs = wt.add(kjobs),
                         p_boff = wt.add(blk_off), p_top = wt.add(top_ptr);
            unsigned char *dwt = S.get<unsigned char>(wt.buf.size());
            CompactJob *d_jobs = dwt ? reinterpret_cast<CompactJob *>(dwt + p_jobs) : nullptr;
            uint64_t *d_word_off = dwt ? reinterpret_cast<uint64_t *>(dwt + p_woff) : nullptr;
            KeyJob *d_kjobs = (dwt && !kjobs.empty()) ? reinterpret_cast<KeyJob *>(dwt + p_kjobs) : nullptr;
            uint64_t *d_blk_off = (dwt && !kjobs.empty()) ? reinterpret_cast<uint64_t *>(dwt + p_boff) : nullptr;
            const uint64_t **d_top_ptr = dwt ? reinterpret_cast<const uint64_t **>(dwt + p_top) : nullptr;
            if (S.err != cudaSuccess) {
                free_results();
                drop_arena();
                return cuda_fail(S.err, "wave tables");
            }
            check(cudaMemcpyAsync(dwt, wt.buf.data(), wt.buf.size(), cudaMemcpyHostToDevice, st), "upload");
            tm.mark(StageTimer::kCompact0, st);
            check(launch_compact(CompactBatch{d_jobs, (int)jobs.size(), d_word_off}, word_off.back(), st), "compact");
            for (size_t i = 0; i < region_jobs.size(); ++i)
                check(launch_compact_regions(region_jobs[i], region_counts[i], ctx->num_sms, st), "compact");
            if (!kjobs.empty())
                check(launch_compact_keys(KeyBatch{d_kjobs, (int)kjobs.size(), d_blk_off}, blk_off.back(), st), "keys");
            tm.mark(StageTimer::kCompact, st);
            // The dedup keys read only the bitmaps and code lists: they run on
            // a stream of their own, forked here, while the emission writes.
            // the dedup's coarse marks, states and keys need the code lists
            if (dset) {
                check(cudaEventRecord(dset->fork, st), "fork");
                check(cudaStreamWaitEvent(ds, dset->fork, 0), "fork");
            }
            // Large meshes get launches of their own (parameters in the kernel's
            // constant space); the rest share one launch over the mesh table.
            // With two or more of them, they spread round-robin over the build
            // stream and three more, so that one kernel's tail overlaps the next.
            std::vector<EmitParams> ep_small;
            std::vector<uint64_t> off_small(1, 0);
            int n_own = 0;
            for (int j = 0; j < n; ++j) n_own += (n == 1 || ep[j].N >= kOwnEmitNodes) ? 1 : 0;
            AuxStreams *aux = n_own >= 2 ? aux_acquire(ctx) : nullptr;
            if (aux) {
                check(cudaEventRecord(aux->fork, st), "fork");
                for (int i = 0; i < AuxStreams::kCount; ++i) check(cudaStreamWaitEvent(aux->s[i], aux->fork, 0), "fork");
            }
            int k_own = 0;
            for (int j = 0; j < n; ++j) {
                if (n == 1 || ep[j].N >= kOwnEmitNodes) {
                    const int lane = aux ? k_own % (AuxStreams::kCount + 1) : 0;
                    cudaStream_t es = lane == 0 ? st : aux->s[lane - 1];
                    ++k_own;
                    check(launch_emit(EmitBatch{nullptr, 1, nullptr}, &ep[j], ep[j].N, flags, ctx->num_sms, es), "emit");
                } else {
                    ep_small.push_back(ep[j]);
                    off_small.push_back(off_small.back() + (ep[j].N + 31) / 32 * 32);
                }
            }
            if (aux) {
                for (int i = 0; i < AuxStreams::kCount; ++i) {
                    check(cudaEventRecord(aux->join[i], aux->s[i]), "join");
                    check(cudaStreamWaitEvent(st, aux->join[i], 0), "join");
                }
                aux_release(ctx, aux);
            }
            if (!ep_small.empty()) {
                EmitParams *d_eps = S.get<EmitParams>(ep_small.size());
                uint64_t *d_offs = S.get<uint64_t>(off_small.size());
                if (S.err != cudaSuccess) {
                    join_dedup();
                    free_results();
                    drop_arena();
                    return cuda_fail(S.err, "wave tables");
                }
                check(upload(d_eps, ep_small, st), "upload");
                check(upload(d_offs, off_small, st), "upload");
                check(launch_emit(EmitBatch{d_eps, (int)ep_small.size(), d_offs}, nullptr, off_small.back(), flags,
                                  ctx->num_sms, st),
                      "emit");
            }
            tm.mark(StageTimer::kEmit, st);
            // the top codes, gathered after the emission
            k_gather_top<<<(n + 127) / 128, 128, 0, st>>>(d_top_ptr, n, top);
            count_launches(1);
            // Dedup of every mesh on the forked stream (its host-side waits
            // overlap the emission running on the GPU); statuses are applied
            // after the emission's own checks.
            if (dd) {
                for (int j = 0; j < n && rc == SVO_OK; ++j) {
                    if (b->m[wave[j]].status != SVO_OK) continue;
                    if (!dstarted[j]) dedup_start(j);
                    if (!druns[j]) continue;
                    drc[j] = dedup_finish(druns[j], ctx->out_pool, ep[j], res[j]->n_dedup, res[j]->dedup);
                    druns[j] = nullptr;
                    if (drc[j] != SVO_OK) dmsg[j] = svo_last_error();
                }
                tm.mark(StageTimer::kDedup, ds);
            }
            // read back the top codes and duplicate counts (pageable copies:
            // these wait for the emission, so they come after the dedup launches)
            std::vector<uint64_t> h_top(n);
            std::vector<unsigned long long> h_dups(2 * n);
            check(cudaMemcpyAsync(h_top.data(), top, 8 * (size_t)n, cudaMemcpyDeviceToHost, st), "read top");
            check(cudaMemcpyAsync(h_dups.data(), dups, 16 * (size_t)n, cudaMemcpyDeviceToHost, st), "read dups");
            check(cudaStreamSynchronize(st), "emit phase");
            for (int j = 0; j < n && rc == SVO_OK; ++j) {
                MeshHost &mh = b->m[wave[j]];
                svo_result *r = res[j];
                if (mh.T == 0 || (h_top[j] & 7) != 0) {
                    mesh_error(mh, SVO_ERR_DEGENERATE,
                               "single top-level node with a non-zero octant: undefined in the reference");
                    continue;
                }
                if (ve && (h_dups[2 * j] || h_dups[2 * j + 1])) {
                    // consecutive duplicates (degenerate widths or absorbed
                    // coordinates): compact both arrays as thrust::unique does
                    const uint64_t nv = mh.N * 8, ne = mh.N * 12;
                    const uint64_t tiles = (std::max(nv, ne) + kUniqueTile - 1) / kUniqueTile;
                    Scratch U{ctx->pool, st};
                    uint32_t *tc = U.get<uint32_t>(tiles), *tp = U.get<uint32_t>(tiles + 1);
                    unsigned long long *ss = U.get<unsigned long long>(scan_scratch_words(tiles));
                    uint32_t *ustat = U.get<uint32_t>(1);
                    svo_vertex *v2 = h_dups[2 * j] ? pool_alloc<svo_vertex>(ctx->out_pool, st, nv, err) : nullptr;
                    svo_edge *e2 = h_dups[2 * j + 1] ? pool_alloc<svo_edge>(ctx->out_pool, st, ne, err) : nullptr;
                    if (U.err != cudaSuccess || err != cudaSuccess) {
                        rc = cuda_fail(U.err != cudaSuccess ? U.err : err, "unique scratch");
                        break;
                    }
                    check(cudaMemsetAsync(ustat, 0, 4, st), "memset");
                    uint32_t cv = 0, ce = 0;
                    if (v2) {
                        check(launch_unique_vertices(r->verts, nv, v2, tc, tp, ss, ustat, st), "unique v");
                        check(cudaMemcpyAsync(&cv, tp + (nv + kUniqueTile - 1) / kUniqueTile, 4, cudaMemcpyDeviceToHost,
                                              st), "read");
                        check(cudaStreamSynchronize(st), "unique v");
                    }
                    if (e2) {
                        check(launch_unique_edges(r->edges, ne, e2, tc, tp, ss, ustat, st), "unique e");
                        check(cudaMemcpyAsync(&ce, tp + (ne + kUniqueTile - 1) / kUniqueTile, 4, cudaMemcpyDeviceToHost,
                                              st), "read");
                        check(cudaStreamSynchronize(st), "unique e");
                    }
                    if (v2) {
                        if (r->own & 2) cudaFreeAsync(r->verts, st);
                        r->verts = v2;
                        r->own |= 2;
                        r->n_verts = cv;
                    }
                    if (e2) {
                        if (r->own & 4) cudaFreeAsync(r->edges, st);
                        r->edges = e2;
                        r->own |= 4;
                        r->n_edges = ce;
                    }
                }
            }
            tm.mark(StageTimer::kUnique, st);
            join_dedup();
            for (int j = 0; j < n; ++j) {
                MeshHost &mh = b->m[wave[j]];
                if (mh.status == SVO_OK && drc[j] != SVO_OK) mesh_error(mh, drc[j], dmsg[j].c_str());
            }
            tm.mark(StageTimer::kEnd, st);
            if (tm.on) cudaEventSynchronize(tm.ev[StageTimer::kEnd]);
            drop_arena();
            return SVO_OK;
        }();
        if (wave_rc != SVO_OK && rc == SVO_OK) rc = wave_rc;
    }
    int first_err = rc;
    for (int j = 0; j < n; ++j) {
        MeshHost &mh = b->m[wave[j]];
        if (rc != SVO_OK && mh.status == SVO_OK) mesh_error(mh, rc, svo_last_error());
        if (mh.status == SVO_OK) {
            mh.emitted = true;
            svo_result *r = res[j];
            if (tm.on && b->timed) {
                r->n_timings = 9;
                r->timings[1] = b->timings_a[1];
                r->timings[2] = b->timings_a[2];
                r->timings[3] = b->timings_a[3];
                r->timings[4] = b->timings_a[4];
                r->timings[5] = tm.span(StageTimer::kCompact0, StageTimer::kCompact);
                r->timings[6] = tm.span(StageTimer::kCompact, StageTimer::kEmit);
                r->timings[7] = tm.span(StageTimer::kEmit, StageTimer::kUnique);
                r->timings[8] = tm.span(StageTimer::kDedup0, StageTimer::kDedup);
                r->timings[0] = b->timings_a[0] + tm.span(StageTimer::kCompact0, StageTimer::kEnd);
            }
            out[wave[j] - first] = r;
        } else {
            svo_result_free(res[j]);
        }
    }
    for (int i = first; i < first + count; ++i) {
        if (status_out) status_out[i - first] = b->m[i].status;
        if (b->m[i].status != SVO_OK && first_err == SVO_OK) first_err = b->m[i].status;
    }
    if (first_err != SVO_OK) {
        for (int i = first; i < first + count; ++i)
            if (b->m[i].status != SVO_OK) {
                g_err = b->m[i].error;
                break;
            }
    }
    return first_err;
}

// tune: the voxelizer split to use (null: the context's, read once here).
int batch_create(svo_ctx *ctx, const svo_mesh_desc *descs, int n, uint32_t flags, cudaStream_t st,
                 svo_batch **out, const VoxTuning *tune = nullptr) {
    svo_batch *b = new svo_batch();
    b->ctx = ctx;
    b->st = st;
    b->flags = flags;
    if (tune) {
        b->tune = *tune;
    } else {
        std::lock_guard<std::mutex> lk(ctx->tune_mu);
        b->tune = ctx->tune;
    }
    b->m.resize(n);
    for (int i = 0; i < n; ++i) {
        MeshHost &mh = b->m[i];
        mh.h_pts = descs[i].points;
        mh.n_pts = descs[i].n_points;
        mh.h_tris = descs[i].tris;
        mh.n_tris = descs[i].tris ? descs[i].n_tris : 0;
        for (int a = 0; a < 3; ++a) mh.res[a] = descs[i].res[a];
    }
    const int rc = batch_phase_a(b);
    if (rc != SVO_OK) {
        batch_release(b);
        cudaStreamSynchronize(st);
        delete b;
        return rc;
    }
    *out = b;
    return SVO_OK;
}

void batch_destroy(svo_batch *b) {
    if (!b) return;
    cudaSetDevice(b->ctx->device);
    batch_release(b);
    cudaStreamSynchronize(b->st);
    delete b;
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
    // Two pools of its own: per-build scratch, and result arrays (kept apart
    // so scratch never splits their blocks).  Freed blocks stay cached.
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    uint64_t keep = UINT64_MAX;
    for (cudaMemPool_t *pp : {&c->pool, &c->out_pool}) {
        if (cudaMemPoolCreate(pp, &props) != cudaSuccess ||
            cudaMemPoolSetAttribute(*pp, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) {
            svo_ctx_destroy(c);
            cudaGetLastError();
            return fail(SVO_ERR_CUDA, "memory pool");
        }
    }
    *out = c;
    return SVO_OK;
}

int svo_ctx_reserve(svo_ctx *ctx, uint64_t result_bytes, uint64_t scratch_bytes, void *stream) {
    if (!ctx) return fail(SVO_ERR_INVALID_ARGUMENT, "null context");
    SVO_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const std::pair<cudaMemPool_t, uint64_t> want[2] = {{ctx->out_pool, result_bytes}, {ctx->pool, scratch_bytes}};
    for (const auto &w : want) {
        if (w.second == 0) continue;
        void *p = nullptr;
        if (cudaMallocFromPoolAsync(&p, w.second, w.first, st) != cudaSuccess) {
            cudaGetLastError();
            return fail(SVO_ERR_OUT_OF_MEMORY, "cannot reserve %llu bytes", (unsigned long long)w.second);
        }
        SVO_TRY(cudaFreeAsync(p, st), "free");
    }
    SVO_TRY(cudaStreamSynchronize(st), "reserve");
    return SVO_OK;
}

int svo_ctx_device(const svo_ctx *ctx, int *device) {
    if (!ctx || !device) return fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    *device = ctx->device;
    return SVO_OK;
}

// Results may outlive the context: a pool destroyed with allocations
// outstanding is released once they are freed.
void svo_ctx_destroy(svo_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    for (AuxStreams *a : ctx->aux_all) {
        for (int i = 0; i < AuxStreams::kCount; ++i) {
            cudaStreamDestroy(a->s[i]);
            cudaEventDestroy(a->join[i]);
        }
        cudaEventDestroy(a->fork);
        delete a;
    }
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    if (ctx->out_pool) cudaMemPoolDestroy(ctx->out_pool);
    delete ctx;
}

int svo_ctx_set_tuning(svo_ctx *ctx, const svo_tuning *t) {
    if (!ctx || !t) return fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    if (t->warp_max == 0) return fail(SVO_ERR_INVALID_ARGUMENT, "warp_max must be positive");
    if (t->serial_max > (1u << 16)) return fail(SVO_ERR_INVALID_ARGUMENT, "serial_max must be <= 65536");
    if (t->serial_packed > 1) return fail(SVO_ERR_INVALID_ARGUMENT, "serial_packed must be 0 or 1");
    std::lock_guard<std::mutex> lk(ctx->tune_mu);
    ctx->tune.serial_max = t->serial_max;
    ctx->tune.warp_max = t->warp_max;
    ctx->tune.split = t->split;
    ctx->tune.inplace_max = t->inplace_max;
    ctx->tune.serial_packed = t->serial_packed;
    return SVO_OK;
}

int svo_ctx_get_tuning(const svo_ctx *ctx, svo_tuning *t) {
    if (!ctx || !t) return fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(const_cast<svo_ctx *>(ctx)->tune_mu);
    t->serial_max = ctx->tune.serial_max;
    t->warp_max = ctx->tune.warp_max;
    t->split = ctx->tune.split;
    t->inplace_max = ctx->tune.inplace_max;
    t->serial_packed = ctx->tune.serial_packed;
    return SVO_OK;
}

int svo_ctx_memory(const svo_ctx *ctx, uint64_t *scratch_used, uint64_t *result_used) {
    if (!ctx) return fail(SVO_ERR_INVALID_ARGUMENT, "null context");
    uint64_t a = 0, b = 0;  // the attribute is a 64-bit unsigned count
    SVO_TRY(cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrUsedMemCurrent, &a), "pool attribute");
    SVO_TRY(cudaMemPoolGetAttribute(ctx->out_pool, cudaMemPoolAttrUsedMemCurrent, &b), "pool attribute");
    if (scratch_used) *scratch_used = (uint64_t)a;
    if (result_used) *result_used = (uint64_t)b;
    return SVO_OK;
}

int svo_selftest_scan_timeout(svo_ctx *ctx, void *stream) {
    if (!ctx) return fail(SVO_ERR_INVALID_ARGUMENT, "null context");
    SVO_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint64_t n = 3 * 4096 + 17;  // four tiles of the single-pass scan
    Scratch S{ctx->pool, st};
    uint32_t *in = S.get<uint32_t>(n), *out = S.get<uint32_t>(n + 1), *status = S.get<uint32_t>(1);
    unsigned long long *scratch = S.get<unsigned long long>(scan_stalled_scratch_words(n));
    if (S.err != cudaSuccess) return cuda_fail(S.err, "self-test scratch");
    SVO_TRY(cudaMemsetAsync(in, 0, n * sizeof(uint32_t), st), "memset");
    SVO_TRY(cudaMemsetAsync(status, 0, sizeof(uint32_t), st), "memset");
    SVO_TRY(launch_scan_stalled(in, out, n, scratch, status, 1 << 12, st), "stalled scan");
    uint32_t h = 0;
    SVO_TRY(cudaMemcpyAsync(&h, status, sizeof(h), cudaMemcpyDeviceToHost, st), "read status");
    SVO_TRY(cudaStreamSynchronize(st), "stalled scan");
    if (h & kStatusScanTimeout) return fail(SVO_ERR_DEVICE_TIMEOUT, "scan look-back timed out (self-test)");
    return SVO_OK;
}

int svo_build(svo_ctx *ctx, const float *points, int64_t n_points, const int32_t *tris, int64_t n_tris,
              int res_x, int res_y, int res_z, uint32_t flags, void *stream, svo_result **out) {
    if (!ctx || !out) return fail(SVO_ERR_INVALID_ARGUMENT, "null context or output");
    *out = nullptr;
    svo_mesh_desc d{points, n_points, tris, n_tris, {res_x, res_y, res_z}, flags};
    svo_batch *b = nullptr;
    int rc = batch_create(ctx, &d, 1, flags, static_cast<cudaStream_t>(stream), &b);
    if (rc != SVO_OK) return rc;
    int st = SVO_OK;
    rc = batch_phase_b(b, 0, 1, out, &st);
    const std::string msg = g_err;
    batch_destroy(b);
    g_err = msg;
    return rc != SVO_OK ? rc : st;
}

int svo_build_batch(svo_ctx *ctx, const svo_mesh_desc *descs, int n, void *stream, svo_result **out,
                    int *status_out) {
    if (!ctx || (!descs && n > 0) || !out) return fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    // one batch per distinct flags value (the kernels are specialised on them)
    std::vector<uint32_t> kinds;
    for (int i = 0; i < n; ++i)
        if (std::find(kinds.begin(), kinds.end(), descs[i].flags) == kinds.end()) kinds.push_back(descs[i].flags);
    int first = SVO_OK;
    std::string first_msg;
    for (uint32_t f : kinds) {
        std::vector<int> idx;
        std::vector<svo_mesh_desc> sub;
        for (int i = 0; i < n; ++i)
            if (descs[i].flags == f) {
                idx.push_back(i);
                sub.push_back(descs[i]);
            }
        svo_batch *b = nullptr;
        int rc = batch_create(ctx, sub.data(), (int)sub.size(), f, static_cast<cudaStream_t>(stream), &b);
        std::vector<svo_result *> r(sub.size(), nullptr);
        std::vector<int> st(sub.size(), rc);
        if (rc == SVO_OK) {
            rc = batch_phase_b(b, 0, (int)sub.size(), r.data(), st.data());
            const std::string msg = g_err;
            batch_destroy(b);
            g_err = msg;
        }
        for (size_t k = 0; k < sub.size(); ++k) {
            out[idx[k]] = r[k];
            if (status_out) status_out[idx[k]] = st[k];
        }
        if (rc != SVO_OK && first == SVO_OK) {
            first = rc;
            first_msg = g_err;
        }
    }
    if (first != SVO_OK) g_err = first_msg;
    return first;
}

int svo_batch_create(svo_ctx *ctx, const svo_mesh_desc *descs, int n, uint32_t flags, void *stream,
                     svo_batch **out) {
    if (!ctx || (!descs && n > 0) || !out) return fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    return batch_create(ctx, descs, n, flags, static_cast<cudaStream_t>(stream), out);
}

int svo_batch_size(const svo_batch *b) { return b ? (int)b->m.size() : 0; }

int svo_batch_mesh_status(const svo_batch *b, int i) {
    if (!b || i < 0 || i >= (int)b->m.size()) return SVO_ERR_INVALID_ARGUMENT;
    return b->m[i].status;
}

int64_t svo_batch_mesh_nodes(const svo_batch *b, int i) {
    if (!b || i < 0 || i >= (int)b->m.size() || b->m[i].status != SVO_OK) return -1;
    return (int64_t)b->m[i].N;
}

int64_t svo_batch_mesh_output_bytes(const svo_batch *b, int i) {
    if (!b || i < 0 || i >= (int)b->m.size() || b->m[i].status != SVO_OK) return -1;
    return (int64_t)output_bytes(b->m[i], b->flags);
}

int svo_batch_emit(svo_batch *b, int first, int count, svo_result **out, int *status_out) {
    if (!b || !out || first < 0 || count < 0 || first + count > (int)b->m.size())
        return fail(SVO_ERR_INVALID_ARGUMENT, "bad batch range");
    return batch_phase_b(b, first, count, out, status_out);
}

void svo_batch_free(svo_batch *b) { batch_destroy(b); }

int svo_ctx_autotune(svo_ctx *ctx, const svo_mesh_desc *descs, int n, uint32_t flags, void *stream,
                     svo_tuning *best) {
    if (!ctx || !descs || n <= 0) return fail(SVO_ERR_INVALID_ARGUMENT, "null argument or empty sample");
    VoxTuning saved;
    {
        std::lock_guard<std::mutex> lk(ctx->tune_mu);
        saved = ctx->tune;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // device ms of the voxelizer stage of the counting phase, best of 2 (after
    // one untimed run); the candidate goes to the measured batches only, so
    // builds on other threads keep the context's split meanwhile
    auto measure = [&](const VoxTuning &t, float &ms) -> int {
        ms = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {
            svo_batch *b = nullptr;
            const int rc = batch_create(ctx, descs, n, flags | SVO_FLAG_TIMINGS, st, &b, &t);
            if (rc != SVO_OK) {
                batch_destroy(b);
                return rc;
            }
            if (rep > 0 && b->timed) ms = std::min(ms, b->timings_a[2]);
            batch_destroy(b);
        }
        return SVO_OK;
    };
    VoxTuning cur = saved, win = saved;
    cur.split = 0;
    float best_ms = 1e30f;
    int rc = SVO_OK;
    // stage 1: the serial / small-triangle thresholds and the serial tier's
    // layout; stage 2: queue entry size
    for (uint32_t sm : {32u, 64u, 128u, 256u}) {
        for (uint32_t cand = 0; cand < 6; ++cand) {
            VoxTuning t = cur;
            t.serial_max = sm;
            t.inplace_max = cand % 3 == 0 ? 16u : cand % 3 == 1 ? 32u : 64u;
            t.serial_packed = cand / 3;
            t.warp_max = 256;
            float ms = 0.0f;
            if ((rc = measure(t, ms)) != SVO_OK) break;
            if (ms < best_ms) {
                best_ms = ms;
                win = t;
            }
        }
        if (rc != SVO_OK) break;
    }
    for (uint32_t wm : {64u, 128u, 512u, 1024u}) {
        if (rc != SVO_OK) break;
        VoxTuning t = win;
        t.warp_max = wm;
        float ms = 0.0f;
        if ((rc = measure(t, ms)) != SVO_OK) break;
        if (ms < best_ms) {
            best_ms = ms;
            win = t;
        }
    }
    if (rc != SVO_OK) return rc;
    {
        std::lock_guard<std::mutex> lk(ctx->tune_mu);
        ctx->tune = win;
    }
    if (best) {
        best->serial_max = win.serial_max;
        best->warp_max = win.warp_max;
        best->split = win.split;
        best->inplace_max = win.inplace_max;
        best->serial_packed = win.serial_packed;
    }
    return SVO_OK;
}

void svo_result_free(svo_result *r) {
    if (!r) return;
    cudaSetDevice(r->device);
    void *ptrs[] = {r->nodes, r->verts, r->edges, r->keys, r->dedup[0], r->dedup[1], r->dedup[2]};
    for (int i = 0; i < 7; ++i)
        if (ptrs[i] && ((r->own >> i) & 1)) cudaFreeAsync(ptrs[i], r->stream);
    if (r->arena && r->arena->refs.fetch_sub(1) == 1) {
        cudaFreeAsync(r->arena->base, r->stream);
        delete r->arena;
    }
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
    svo::host::TraceRange trace("svo: write tree .obj");
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

// Countdown of svo_debug_fail_alloc: when it reaches the allocation it names,
// that allocation reports cudaErrorMemoryAllocation without asking the pool.
static std::atomic<int64_t> g_fail_alloc{0};

cudaError_t pool_malloc(void **p, size_t bytes, cudaMemPool_t pool, cudaStream_t st) {
    int64_t k = g_fail_alloc.load(std::memory_order_relaxed);
    while (k > 0 && !g_fail_alloc.compare_exchange_weak(k, k - 1, std::memory_order_relaxed)) {
    }
    if (k == 1) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMallocFromPoolAsync(p, bytes, pool, st);
}
}  // namespace svo

extern "C" int64_t svo_kernel_launches(void) { return svo::g_launches.load(std::memory_order_relaxed); }

extern "C" int64_t svo_debug_fail_alloc(int64_t n) {
    return svo::g_fail_alloc.exchange(n > 0 ? n : 0, std::memory_order_relaxed);
}
