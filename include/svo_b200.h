/*
 * svo_b200.h -- C ABI of the B200-native sparse voxel octree builder.
 *
 * This is the drop-in boundary for GPU-SVO's build path.  Each entry point
 * names the reference interface it replaces (paths relative to the GPU-SVO
 * project root).  The reference itself is a C++ static library with no C
 * entry points; these are the calls an FFI binding of its `SparseVoxelOctree`
 * / `BaseModel` classes would make.  All functions return SVO_OK (0) or a
 * status code; none of them exits the process (the reference's CUDA_CHECK /
 * getLastCudaError call exit(), src/CUDAUtil.h:21-48).  svo_last_error()
 * returns the calling thread's last error message.
 *
 * Pointers to mesh data may be host or device memory; the library detects
 * which.  Result arrays live in device memory until copied out.
 */
#ifndef SVO_B200_H
#define SVO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------------- */
#define SVO_OK 0
#define SVO_ERR_INVALID_ARGUMENT 1
#define SVO_ERR_CUDA 2
#define SVO_ERR_OUT_OF_MEMORY 3
#define SVO_ERR_EMPTY 4       /* no surface voxels (the reference aborts) */
#define SVO_ERR_DEGENERATE 5  /* input for which the reference's build is undefined */
#define SVO_ERR_IO 6
#define SVO_ERR_PARSE 7
#define SVO_ERR_UNSUPPORTED 8
#define SVO_ERR_DEVICE_TIMEOUT 9 /* a bounded device-side wait gave up */
#define SVO_ERR_TIMEOUT 10       /* a host-side wait ran out (svo_server_wait) */
#define SVO_ERR_CANCELLED 11     /* the request was cancelled before it was built (svo_server_cancel) */

/* ---- build flags ---------------------------------------------------------- */
/* Default (0): the reference's effective behaviour bit for bit, including its
 * neighbour tables (only the root's self entry is ever stored,
 * src/SVO.cu:535-542) and its vertex/edge arrays (src/SVO.cu:567-728). */
#define SVO_FLAG_FULL_NEIGHBORS 0x1u /* real 27-neighbourhood per node (intended semantics),
                                        vertex/edge owner = smallest sharing node index */
#define SVO_FLAG_DEDUP 0x2u          /* also emit Morton-keyed unique vertex/edge/face keys */
#define SVO_FLAG_STRICT_FP 0x4u      /* round every float op (no FMA contraction) */
#define SVO_FLAG_NO_VERT_EDGE 0x8u   /* skip the per-node vertex/edge arrays */
#define SVO_FLAG_NO_KEYS 0x10u       /* skip the sorted leaf-voxel key list */
#define SVO_FLAG_TIMINGS 0x20u       /* record per-stage device times (svo_result_timings) */

/* ---- records (byte layouts of the reference's types) --------------------- */
/* SVONode, src/SVO.h:20-35 (168 bytes; pad_ is written as zero). */
typedef struct svo_node {
    uint32_t morton_code;
    uint8_t is_leaf;
    uint8_t pad_[3];
    float origin[3];
    float width;
    uint32_t parent;
    uint32_t childs[8];
    uint32_t neighbors[27];
} svo_node;

/* thrust::pair<Eigen::Vector3f, uint32_t>, src/SVO.h:50 (16 bytes). */
typedef struct svo_vertex {
    float pos[3];
    uint32_t owner;
} svo_vertex;

/* thrust::pair<thrust::pair<Vector3f, Vector3f>, uint32_t>, src/SVO.h:37,51 (28 bytes). */
typedef struct svo_edge {
    float p0[3];
    float p1[3];
    uint32_t owner;
} svo_edge;

/* AABox<Eigen::Vector3f>, src/BaseModel.h:10-22. */
typedef struct svo_aabb {
    float min[3];
    float max[3];
    float width[3];
} svo_aabb;

typedef struct svo_ctx svo_ctx;
typedef struct svo_result svo_result;

/* ---- context -------------------------------------------------------------- */
/* Per-device state: stream-ordered memory pool, scratch, tuning.  Replaces the
 * reference's process-global launch state (src/SVO.cu:15-18) and its
 * per-call cudaMalloc/thrust allocations (src/SVO.cu:353-376). */
int svo_ctx_create(int device, svo_ctx **out);
void svo_ctx_destroy(svo_ctx *ctx);
int svo_ctx_device(const svo_ctx *ctx, int *device);
/* Maps device memory into the context's pools up front (result arrays,
 * per-build scratch); builds then carve it without growing the pools.  The
 * memory stays with the context until svo_ctx_destroy. */
int svo_ctx_reserve(svo_ctx *ctx, uint64_t result_bytes, uint64_t scratch_bytes, void *stream);
/* Device bytes currently allocated from the context's two pools: per-build
 * scratch and result arrays (0 and the size of the live results once every
 * build has finished and its stream is idle).  No counterpart in the
 * reference. */
int svo_ctx_memory(const svo_ctx *ctx, uint64_t *scratch_used, uint64_t *result_used);

/* Voxelizer work split: triangles whose grid bbox has at most serial_max
 * (<= 65536) voxels are tested row by row without culling, the rows of a
 * warp's such triangles handed out one row per lane per round
 * (serial_packed = 1) or one triangle per lane (0, the default); triangles of at most inplace_max 4x4x4
 * bricks are walked by the warp that set them up, packed 32 bricks per round
 * across the warp's triangles; larger ones are cut into queue entries of at
 * most warp_max bricks, one warp per entry.  Results do not depend on these
 * values, only the speed.  No counterpart in the reference (one thread per
 * triangle there, src/SVO.cu:37-188). */
typedef struct svo_tuning {
    uint32_t serial_max;
    uint32_t warp_max;
    uint32_t split; /* also cull the 2x2x2 sub-bricks of surviving bricks (queue tier) */
    uint32_t inplace_max;
    uint32_t serial_packed;
} svo_tuning;
int svo_ctx_set_tuning(svo_ctx *ctx, const svo_tuning *t);
int svo_ctx_get_tuning(const svo_ctx *ctx, svo_tuning *t);

/* Thread-local message for the last non-zero status. */
const char *svo_last_error(void);

/* Process-wide number of CUDA kernels this library has launched (for
 * accounting in benchmarks; no counterpart in the reference). */
int64_t svo_kernel_launches(void);

/* ---- mesh input ----------------------------------------------------------- */
/* BaseModel::loadOBJ, src/BaseModel.cpp:3-25.  Same accepted lines and quirks
 * (only "v " / "f " lines; `a/t/n` faces dropped; unterminated last line
 * dropped).  A line of 255+ characters (the reference loops forever) and a
 * face index outside the vertex list are SVO_ERR_PARSE.  *points (3 floats per
 * vertex) and *tris (3 zero-based int32 per triangle) are malloc'd host
 * arrays; release them with svo_free_host. */
int svo_load_obj(const char *path, float **points, int64_t *n_points, int32_t **tris,
                 int64_t *n_tris);
void svo_free_host(void *p);

/* BaseModel(filename) bounding box + createMeshBBCube, src/BaseModel.h:24-49,64-73.
 * Host arrays only. */
int svo_bbox_cube(const float *points, int64_t n_points, svo_aabb *out);

/* ---- build ---------------------------------------------------------------- */
/* SparseVoxelOctree::create(), src/SVO.cu:341-520 (with meshVoxelize,
 * src/SVO.cu:37-206, and constructNodeAtrributes, src/SVO.cu:522-735), for
 * the mesh a SparseVoxelOctree(filename, res_x, res_y, res_z) would hold
 * (src/SVO.h:61-67): `points` are the model's vertices, `tris` its triangles
 * (zero-based).  tris == NULL means a triangle soup: n_points = 3 * triangles.
 * Resolutions up to 1024 reproduce the reference exactly; 1025..2048 use
 * 64-bit Morton codes (the reference's 32-bit codes are wrong above 1024;
 * svo_node.morton_code then holds the low 32 bits, svo_result_copy_keys the
 * full codes).
 * `stream` is a cudaStream_t (NULL = the legacy default stream).  On success
 * *out owns the device arrays of the octree.  The result remembers `stream`:
 * svo_result_free releases its arrays there (stream-ordered) and the copy
 * functions copy there, so the stream must outlive the result. */
int svo_build(svo_ctx *ctx, const float *points, int64_t n_points, const int32_t *tris,
              int64_t n_tris, int res_x, int res_y, int res_z, uint32_t flags, void *stream,
              svo_result **out);

/* Many independent builds in one pass over the device: every kernel of the
 * pipeline runs once for all meshes (meshes with equal flags share a pass);
 * each mesh's result equals its own svo_build bit for bit.  descs[i]
 * describes mesh i; out[i] receives its result (NULL on error).  Returns the
 * status of the first failing mesh; per-mesh status in status_out (may be
 * NULL).  No counterpart in the reference (one mesh per process there). */
typedef struct svo_mesh_desc {
    const float *points;
    int64_t n_points;
    const int32_t *tris;
    int64_t n_tris;
    int res[3];
    uint32_t flags;
} svo_mesh_desc;
int svo_build_batch(svo_ctx *ctx, const svo_mesh_desc *descs, int n, void *stream,
                    svo_result **out, int *status_out);

/* Autotuner for the work split: runs the counting phase of the sample meshes
 * (a batch, as svo_batch_create) for a grid of candidate splits, times the
 * voxelizer stage on the device, installs the fastest split in the context
 * and returns it in *best (may be null).  Results do not depend on the split.
 * Builds that other threads run on the context meanwhile keep its previous
 * split (each build reads the split once, when it starts).  No counterpart in
 * the reference. */
int svo_ctx_autotune(svo_ctx *ctx, const svo_mesh_desc *descs, int n, uint32_t flags, void *stream,
                     svo_tuning *best);

/* The same in two steps, for callers that bound device memory:
 * svo_batch_create runs the counting phase of every mesh (voxelization,
 * octree level sizes; about res^3/7 bytes of scratch per mesh) and knows each
 * mesh's exact node count and output size; svo_batch_emit then writes the
 * octrees of meshes [first, first + count) in one pass -- call it for
 * consecutive ranges that fit the memory at hand and free their results
 * between calls.  The node/vertex/edge/key arrays of the results of one
 * svo_batch_emit call share one device block, released when the last of
 * those results is freed.  All meshes of a batch use `flags` (descs[i].flags
 * is ignored).  The batch holds its scratch until svo_batch_free. */
typedef struct svo_batch svo_batch;
int svo_batch_create(svo_ctx *ctx, const svo_mesh_desc *descs, int n, uint32_t flags, void *stream,
                     svo_batch **out);
int svo_batch_size(const svo_batch *b);
int svo_batch_mesh_status(const svo_batch *b, int i);
int64_t svo_batch_mesh_nodes(const svo_batch *b, int i);        /* -1 on error */
int64_t svo_batch_mesh_output_bytes(const svo_batch *b, int i); /* device bytes of its result */
int svo_batch_emit(svo_batch *b, int first, int count, svo_result **out, int *status_out);
void svo_batch_free(svo_batch *b);

/* ---- served builds (no counterpart in the reference) ------------------------
 * A request loop with continuous batching: worker threads, one CUDA stream
 * each, take the longest FIFO prefix of queued requests that fits mem_budget
 * (at most max_batch) and build it as one batch, while the other workers
 * admit later arrivals and overlap their batches on the device.  Admission
 * reserves svo_estimate_bytes() per request.  When a batch's counting phase
 * has the exact result sizes, the batch builds the longest prefix of its
 * requests that fits the budget beside the other reservations and puts the
 * rest back at the front of the queue with their exact sizes (a request larger
 * than the whole budget is built alone).  A built request holds the exact size
 * of its result until svo_server_release.  Mesh pointers (host or device)
 * must stay valid until the request is finished. */
typedef struct svo_server svo_server;
typedef struct svo_server_config {
    uint64_t mem_budget; /* device bytes for admitted requests and live results */
    int workers;         /* batches on the device at once */
    int max_batch;       /* requests per batch */
    uint32_t flags;      /* build flags of every request */
} svo_server_config;
typedef struct svo_server_stats_t {
    int64_t queued;
    int busy_workers;
    uint64_t reserved_bytes;
    uint64_t batches; /* batches built so far */
    uint64_t built;   /* requests built so far */
    double build_seconds; /* wall time of all batches (summed over workers) */
    double queue_seconds; /* time requests waited for admission (summed) */
    uint64_t peak_reserved_bytes; /* most device bytes reserved at any time */
    uint64_t requeued;            /* requests sent back to the queue once their exact size was known */
    uint64_t admitted_batches;    /* batches taken from the queue so far */
    uint64_t decided_batches;     /* of those, batches that have made their keep/requeue decision */
} svo_server_stats_t;
/* Device bytes admission reserves for a mesh: inputs, scratch of a res^3
 * grid (with SVO_FLAG_DEDUP its res^3-bit candidate bitmap too) and the
 * outputs of 16*res^2 nodes (a closed surface spanning it). */
uint64_t svo_estimate_bytes(int64_t n_points, int64_t n_tris, int res_x, int res_y, int res_z, uint32_t flags);
int svo_server_create(svo_ctx *ctx, const svo_server_config *cfg, svo_server **out);
int svo_server_submit(svo_server *s, const svo_mesh_desc *desc, uint64_t *ticket);
/* Blocks until the request is built (timeout_us < 0: no limit; else
 * SVO_ERR_TIMEOUT when it runs out).  *result stays owned by the server and
 * valid until svo_server_release; latency = build finished - submitted. */
int svo_server_wait(svo_server *s, uint64_t ticket, int64_t timeout_us, svo_result **result, int *status,
                    double *latency_s);
/* The next finished request in completion order (each reported once, unless
 * released first); same outputs as svo_server_wait. */
int svo_server_next(svo_server *s, int64_t timeout_us, uint64_t *ticket, svo_result **result, int *status,
                    double *latency_s);
int svo_server_release(svo_server *s, uint64_t ticket);
/* Withdraws a request that is still queued: it finishes at once with status
 * SVO_ERR_CANCELLED and no result (reported by svo_server_wait/next, then
 * released as usual).  A request already building or finished cannot be
 * cancelled (SVO_ERR_INVALID_ARGUMENT). */
int svo_server_cancel(svo_server *s, uint64_t ticket);
int svo_server_stats(const svo_server *s, svo_server_stats_t *out);
/* Frees the results not yet released, finishes every queued request and frees
 * its result too.  A finished result holds its bytes of the budget until it is
 * released: a client that waits for a request while holding results can keep
 * that request from being admitted. */
void svo_server_destroy(svo_server *s);

/* ---- served builds over several GPUs (no counterpart in the reference) -----
 * One svo_server per context -- one context per GPU, each made by
 * svo_ctx_create on its own device -- behind one ticket space.  Every request
 * is built whole on one member: a submission goes to the member with the
 * fewest estimated bytes (svo_estimate_bytes) submitted and not yet released,
 * ties to the lowest index.  The members share nothing and never exchange
 * data; cfg (mem_budget included) applies to each member.  The calls mirror
 * svo_server_*: results stay owned by their member until svo_fleet_release,
 * svo_fleet_next reports finished requests of all members in completion
 * order.  The contexts must outlive the fleet. */
typedef struct svo_fleet svo_fleet;
int svo_fleet_create(svo_ctx *const *ctxs, int n, const svo_server_config *cfg, svo_fleet **out);
int svo_fleet_submit(svo_fleet *f, const svo_mesh_desc *desc, uint64_t *ticket);
int svo_fleet_wait(svo_fleet *f, uint64_t ticket, int64_t timeout_us, svo_result **result, int *status,
                   double *latency_s);
int svo_fleet_next(svo_fleet *f, int64_t timeout_us, uint64_t *ticket, svo_result **result, int *status,
                   double *latency_s);
int svo_fleet_release(svo_fleet *f, uint64_t ticket);
int svo_fleet_cancel(svo_fleet *f, uint64_t ticket);
/* The member (index into ctxs) that builds a ticket, -1 for a ticket the fleet
 * does not hold (never issued, or released). */
int svo_fleet_member(const svo_fleet *f, uint64_t ticket);
int svo_fleet_stats(const svo_fleet *f, int member, svo_server_stats_t *out);
/* Destroys the members (svo_server_destroy each), then the fleet. */
void svo_fleet_destroy(svo_fleet *f);

/* Sorted surface-voxel Morton keys of a mesh (the first stage of svo_build:
 * same bounding cube, same voxel test, same key list as svo_result_copy_keys)
 * without allocating any device memory.  No counterpart in the reference.
 * It exists for callers that cannot let a library call cudaMalloc or cudaFree
 * -- applications that hand out all device memory from their own arena, or
 * that must not have an allocation synchronise the device in the middle of
 * their stream work.  Inputs (points, tris; tris == NULL means a soup) and the
 * output `keys` (capacity keys_cap, count in *n_keys) are device memory the
 * caller owns; the only other memory used is a fixed 3 MiB scratch array
 * compiled into the library, which every GPU that loads the library holds
 * until the process exits.  Resolutions above 256 on any axis are rejected
 * with SVO_ERR_UNSUPPORTED (the scratch holds a 256^3 bitmap).  The first call
 * on a device looks up the scratch array's device address (make it before any
 * stream capture).  All calls share the one scratch array: calls whose work
 * overlaps on the GPU race, so serialise them.  Synchronises `stream`. */
int svo_voxelize_keys_noalloc(const float *points, int64_t n_points, const int32_t *tris,
                              int64_t n_tris, int res_x, int res_y, int res_z, uint32_t flags,
                              uint64_t *keys, int64_t keys_cap, int64_t *n_keys, void *stream);

/* ---- results (SparseVoxelOctree's private members, src/SVO.h:41-51) ------- */
void svo_result_free(svo_result *r);
int svo_result_depth(const svo_result *r);                 /* treeDepth */
int64_t svo_result_num_nodes(const svo_result *r);         /* numTreeNodes */
int64_t svo_result_num_vertices(const svo_result *r);      /* nodeVertexArray.size() */
int64_t svo_result_num_edges(const svo_result *r);         /* nodeEdgeArray.size() */
int64_t svo_result_num_keys(const svo_result *r);          /* surface voxels */
/* Node count of each level, finest first (depthNumNodes + the root level);
 * returns the number of levels. */
int svo_result_level_counts(const svo_result *r, int64_t *counts, int cap);
int svo_result_bbox(const svo_result *r, svo_aabb *out);   /* modelBBox */
/* Device pointers (valid until svo_result_free). */
const svo_node *svo_result_nodes_device(const svo_result *r);
const svo_vertex *svo_result_vertices_device(const svo_result *r);
const svo_edge *svo_result_edges_device(const svo_result *r);
const uint64_t *svo_result_keys_device(const svo_result *r);
/* Copies to host memory (cap = capacity in elements; returns SVO_ERR_INVALID_ARGUMENT
 * when too small). */
int svo_result_copy_nodes(const svo_result *r, svo_node *dst, int64_t cap);
int svo_result_copy_vertices(const svo_result *r, svo_vertex *dst, int64_t cap);
int svo_result_copy_edges(const svo_result *r, svo_edge *dst, int64_t cap);
int svo_result_copy_keys(const svo_result *r, uint64_t *dst, int64_t cap);
/* Per-stage device times in ms of a build made with SVO_FLAG_TIMINGS, from
 * CUDA events on the build stream: [0] first to last event (includes the
 * host round trip that sizes the outputs), [1] bounding cube, [2] voxelize,
 * [3] bitmap pyramid, [4] block-count scan, [5] level code lists,
 * [6] node/vertex/edge emission, [7] duplicate removal, [8] dedup keys (on a
 * stream of its own, concurrent with [6] and [7], so the stages need not add
 * up to [0]).  Returns the number of entries (9), or 0 without timings.  No
 * counterpart in the reference (it has no instrumentation). */
int svo_result_timings(const svo_result *r, float *ms, int cap);

/* Morton-keyed unique primitives (SVO_FLAG_DEDUP): kind 0 vertices, 1 edges,
 * 2 faces.  Sorted u64 keys. */
int64_t svo_result_num_dedup(const svo_result *r, int kind);
int svo_result_copy_dedup(const svo_result *r, int kind, uint64_t *dst, int64_t cap);

/* ---- output ---------------------------------------------------------------- */
/* SparseVoxelOctree::writeTree, src/SVO.cu:737-753 with write_cube,
 * src/IO.h:23-90: writes `path` byte-identical to the reference's file
 * (the caller forms the name "<stem>_<depth>_tree.obj"). */
int svo_write_tree(const svo_result *r, const char *path);
/* The same writer over host node records (e.g. a copied node array). */
int svo_write_tree_nodes(const svo_node *nodes, int64_t n, const char *path);
/* SparseVoxelOctree::writeVoxel, src/SVO.cu:755-777: one cube per surface
 * voxel, decoded from its key (the reference only calls it in NDEBUG builds). */
int svo_write_voxels(const svo_result *r, const char *path);
/* The same writer over host keys: cube i at origin + width * (x, y, z) of
 * keys[i], computed on the host (src/SVO.cu:766-775). */
int svo_write_voxel_keys(const uint64_t *keys, int64_t n, const float origin[3], float width,
                         const char *path);

/* ---- diagnostics and fault injection (no counterpart in the reference) ------
 * The reference stops the process on any CUDA error (CUDA_CHECK and
 * getLastCudaError call exit(), src/CUDAUtil.h:21-48); this library returns a
 * status instead and keeps the context usable.  These two calls let a test
 * provoke the two failures a build can meet without faulting a GPU. */
/* Runs the single-pass scan that every build uses, over a small array, with
 * its first tile never run: every look-back wait that reaches that tile gives
 * up after its poll limit.  Returns SVO_ERR_DEVICE_TIMEOUT when the bounded
 * wait ended the kernel as designed (any other status is a failure of the
 * self-test); the context stays usable afterwards.  Synchronises `stream`. */
int svo_selftest_scan_timeout(svo_ctx *ctx, void *stream);
/* Process-wide: the n-th device allocation that a build makes from now on
 * (1 = the next one) fails as out of memory; n <= 0 disarms.  Returns the
 * countdown it replaces (> 0: the previous injection has not fired yet).  For
 * tests of the SVO_ERR_OUT_OF_MEMORY paths. */
int64_t svo_debug_fail_alloc(int64_t n);

#ifdef __cplusplus
}
#endif

#endif /* SVO_B200_H */
