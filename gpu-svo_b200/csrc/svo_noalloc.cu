// svo_noalloc.cu -- surface-voxel keys without any device allocation.
//
// Some callers cannot let this library call cudaMalloc: a host application
// that owns all device memory through its own arena, a process that runs
// with allocation locked after start-up, or code that must not trigger an
// allocator's synchronisation in the middle of its own stream work.  This
// entry point produces the sorted surface-voxel keys of a mesh (the first
// stage of the octree build) using only memory the caller passes in plus a
// fixed scratch area that lives in the library itself: a file-scope
// __device__ array of kNoAllocScratchBytes (3 MiB), present on every GPU that
// loads the library, for as long as the process runs.
//
// Host code may not use the array's name as a device address (in host code
// it names a host-side stand-in), so the first call on each device looks up
// the array's real device address with cudaGetSymbolAddress, with that device
// current, and keeps it; that first call should therefore come before any
// stream capture.  All calls share the one array: it holds whatever the last
// call left, the call clears what must start at zero, and two calls whose
// work overlaps on the GPU (different streams, or different host threads)
// race on it -- serialise them.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "svo_host.h"
#include "svo_internal.h"

namespace svo {
namespace {

constexpr size_t kNoAllocScratchBytes = 3u << 20;
constexpr int kNoAllocMaxRes = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

unsigned char *g_scratch_addr[kMaxDevices] = {};
int g_num_sms[kMaxDevices] = {};
std::mutex g_scratch_mu;

int noalloc_fail(int code, const char *msg) {
    svo::host::set_error(msg);
    return code;
}

// Device address of the scratch array on the current device and the device's
// SM count (looked up once per device, with that device current).
cudaError_t scratch_address(int device, unsigned char **out, int *num_sms) {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[device]) {
        int sms = 0;
        cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (e != cudaSuccess) return e;
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_num_sms[device] = sms;
        g_scratch_addr[device] = static_cast<unsigned char *>(p);
    }
    *out = g_scratch_addr[device];
    *num_sms = g_num_sms[device];
    return cudaSuccess;
}

struct Carve {
    unsigned char *base;
    size_t used = 0;
    template <class T>
    T *take(size_t count) {
        used = (used + 255) / 256 * 256;
        T *p = reinterpret_cast<T *>(base + used);
        used += count * sizeof(T);
        return p;
    }
};

bool on_device(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace
}  // namespace svo

using namespace svo;

extern "C" int svo_voxelize_keys_noalloc(const float *points, int64_t n_points, const int32_t *tris,
                                         int64_t n_tris, int res_x, int res_y, int res_z, uint32_t flags,
                                         uint64_t *keys, int64_t keys_cap, int64_t *n_keys, void *stream) {
    if (!points || n_points <= 0 || !keys || !n_keys || n_tris < 0)
        return noalloc_fail(SVO_ERR_INVALID_ARGUMENT, "null argument or empty mesh");
    *n_keys = 0;
    const int res[3] = {res_x, res_y, res_z};
    for (int a = 0; a < 3; ++a)
        if (res[a] < 1 || res[a] > kNoAllocMaxRes)
            return noalloc_fail(SVO_ERR_UNSUPPORTED,
                                "svo_voxelize_keys_noalloc: resolution must be in [1, 256] "
                                "(its fixed 3 MiB scratch holds a 256^3 bitmap); use svo_build above that");
    if (!tris && n_points % 3 != 0)
        return noalloc_fail(SVO_ERR_INVALID_ARGUMENT, "triangle soup needs 3 points per triangle");
    const int64_t nt = tris ? n_tris : n_points / 3;
    if (nt > 0x7FFFFFFF) return noalloc_fail(SVO_ERR_UNSUPPORTED, "more than 2^31-1 triangles");
    if (!on_device(points) || (tris && nt > 0 && !on_device(tris)) || !on_device(keys))
        return noalloc_fail(SVO_ERR_INVALID_ARGUMENT,
                            "svo_voxelize_keys_noalloc takes device pointers only (it copies nothing)");
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess || device < 0 || device >= kMaxDevices)
        return noalloc_fail(SVO_ERR_CUDA, "cudaGetDevice failed");
    unsigned char *base = nullptr;
    int num_sms = 0;
    if ((e = scratch_address(device, &base, &num_sms)) != cudaSuccess)
        return noalloc_fail(SVO_ERR_CUDA, cudaGetErrorString(e));

    const Pyramid py = make_pyramid(res_x, res_y, res_z);
    Carve c{base};
    GridParams *gp = c.take<GridParams>(1);
    uint32_t *mm = c.take<uint32_t>(8);
    int32_t *imm = c.take<int32_t>(2);
    uint32_t *totals = c.take<uint32_t>(kMaxLevels);
    uint32_t *counters = c.take<uint32_t>(4);
    uint32_t *done = c.take<uint32_t>(1);
    MeshDev *d_mesh = c.take<MeshDev>(1);
    uint64_t *d_tri_off = c.take<uint64_t>(2);
    uint32_t *d_cta_off = c.take<uint32_t>(2);
    uint32_t *d_bbox_off = c.take<uint32_t>(2);
    CompactJob *d_job = c.take<CompactJob>(1);
    uint64_t *d_word_off = c.take<uint64_t>(2);
    uint64_t *bits = c.take<uint64_t>(py.total_words);
    uint32_t *cnt = c.take<uint32_t>(py.total_blocks);
    uint32_t *pre = c.take<uint32_t>(py.total_blocks + 1);
    unsigned long long *scan = c.take<unsigned long long>(scan_scratch_words(py.total_blocks));
    if (c.used > kNoAllocScratchBytes) return noalloc_fail(SVO_ERR_UNSUPPORTED, "scratch layout exceeds 3 MiB");

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    auto cuda = [](cudaError_t err) { return err == cudaSuccess ? SVO_OK : noalloc_fail(SVO_ERR_CUDA, cudaGetErrorString(err)); };
    int rc;
    if (tris && nt > 0) {
        int32_t h[2];
        if ((rc = cuda(launch_index_range(tris, nt * 3, imm, st)))) return rc;
        if ((rc = cuda(cudaMemcpyAsync(h, imm, sizeof(h), cudaMemcpyDeviceToHost, st)))) return rc;
        if ((rc = cuda(cudaStreamSynchronize(st)))) return rc;
        if (h[0] < 0 || h[1] >= n_points) return noalloc_fail(SVO_ERR_INVALID_ARGUMENT, "triangle index out of range");
    }
    // the one-mesh tables, copied from the host stack (no device allocation)
    MeshDev md{};
    md.pts = points;
    md.tris = tris;
    md.n_pts = n_points;
    md.n_tris = nt;
    md.res[0] = res_x;
    md.res[1] = res_y;
    md.res[2] = res_z;
    md.gp = gp;
    md.mm = mm;
    md.bits = bits;
    md.cnt = cnt;
    md.pre = pre;
    md.totals = totals;
    md.done = done;
    md.py = py;
    const uint64_t h_tri_off[2] = {0, (uint64_t)nt};
    const uint32_t h_cta_off[2] = {0, py.ctas};
    const uint32_t h_bbox_off[2] = {0, bbox_blocks(n_points)};
    // everything that must start at zero (the array keeps the last call's data)
    if ((rc = cuda(cudaMemsetAsync(base, 0, c.used, st)))) return rc;
    const uint32_t mm_init[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u};
    if ((rc = cuda(cudaMemcpyAsync(mm, mm_init, sizeof(mm_init), cudaMemcpyHostToDevice, st)))) return rc;
    if ((rc = cuda(cudaMemcpyAsync(d_mesh, &md, sizeof(md), cudaMemcpyHostToDevice, st)))) return rc;
    if ((rc = cuda(cudaMemcpyAsync(d_tri_off, h_tri_off, sizeof(h_tri_off), cudaMemcpyHostToDevice, st)))) return rc;
    if ((rc = cuda(cudaMemcpyAsync(d_cta_off, h_cta_off, sizeof(h_cta_off), cudaMemcpyHostToDevice, st)))) return rc;
    if ((rc = cuda(cudaMemcpyAsync(d_bbox_off, h_bbox_off, sizeof(h_bbox_off), cudaMemcpyHostToDevice, st)))) return rc;
    const BatchDev bd{d_mesh, 1, d_tri_off, d_cta_off, d_bbox_off};
    if ((rc = cuda(launch_bbox(bd, h_bbox_off[1], st)))) return rc;
    VoxTuning tune;
    tune.warp_max = 0xFFFFFFFFu;  // no big-triangle queue: warps take every large triangle
    if ((rc = cuda(launch_voxelize(bd, nt, (flags & SVO_FLAG_STRICT_FP) != 0, tune, nullptr, 0, counters,
                                   num_sms, st))))
        return rc;
    if ((rc = cuda(launch_pyramid(bd, py.ctas, num_sms, st)))) return rc;
    if ((rc = cuda(launch_scan(cnt, pre, py.total_blocks, scan, &gp->status, st)))) return rc;
    if ((rc = cuda(launch_level_totals(bd, st)))) return rc;
    uint32_t h_tot = 0, h_status = 0;
    if ((rc = cuda(cudaMemcpyAsync(&h_tot, totals, 4, cudaMemcpyDeviceToHost, st)))) return rc;
    if ((rc = cuda(cudaMemcpyAsync(&h_status, &gp->status, 4, cudaMemcpyDeviceToHost, st)))) return rc;
    if ((rc = cuda(cudaStreamSynchronize(st)))) return rc;
    if (h_status & kStatusNonFinite) return noalloc_fail(SVO_ERR_INVALID_ARGUMENT, "non-finite vertex coordinate");
    if (h_status & kStatusScanTimeout) return noalloc_fail(SVO_ERR_DEVICE_TIMEOUT, "scan look-back timed out");
    *n_keys = h_tot;
    if ((int64_t)h_tot > keys_cap) return noalloc_fail(SVO_ERR_INVALID_ARGUMENT, "keys buffer too small (see *n_keys)");
    CompactJob job{};
    job.bits = bits;
    job.pre = pre;
    job.py = py;
    job.l0 = 0;
    job.l1 = 1;
    job.out = keys;
    const uint64_t h_word_off[2] = {0, py.words[0]};
    if ((rc = cuda(cudaMemcpyAsync(d_job, &job, sizeof(job), cudaMemcpyHostToDevice, st)))) return rc;
    if ((rc = cuda(cudaMemcpyAsync(d_word_off, h_word_off, sizeof(h_word_off), cudaMemcpyHostToDevice, st)))) return rc;
    if ((rc = cuda(launch_compact(CompactBatch{d_job, 1, d_word_off}, py.words[0], st)))) return rc;
    return cuda(cudaStreamSynchronize(st));
}
