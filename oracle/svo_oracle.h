/*
 * svo_oracle.h -- CPU restatement of GPU-SVO's octree build pipeline.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links or calls this
 * library: only tests/, __graft_entry__.smoke() and bench.py's CPU legs use
 * it, and only as the checker (or, in bench.py, as the timed CPU baseline).
 *
 * Every function restates a piece of the reference (paths are relative to the
 * GPU-SVO project root):
 *   oracle_load_obj   BaseModel::loadOBJ            src/BaseModel.cpp:3-25
 *   oracle_bbox_cube  BaseModel(filename) ctor      src/BaseModel.h:64-73
 *                     createMeshBBCube              src/BaseModel.h:24-49
 *   oracle_build      SparseVoxelOctree::create()   src/SVO.cu:341-520
 *                     meshVoxelize/surfaceVoxelize  src/SVO.cu:37-206
 *                     constructNodeAtrributes       src/SVO.cu:522-735
 *   oracle_write_tree SparseVoxelOctree::writeTree  src/SVO.cu:737-753
 *   oracle_write_voxels SparseVoxelOctree::writeVoxel src/SVO.cu:755-777 (as called at :411-419)
 *                     write_cube                    src/IO.h:8-90
 *
 * Parity pinning: the Morton encoder/decoder and the neighbour/shared-corner
 * tables are pinned against the reference's own MortonLUT.h (compiled from the
 * reference sources by oracle/ref/build_ref.sh) and against tables read as
 * text from src/SVO.cu (tests/golden/make_golden.py).  The floating-point
 * voxel test and node origins depend on Eigen 3.4 (absent here, so the
 * reference cannot be built): their operation order follows Eigen's
 * documented evaluation order, and the FMA contraction pattern is pinned
 * against nvcc's own default contraction by a GPU probe test.  For those
 * parts parity with the reference build itself is UNPINNED.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (same values as the product's C-ABI). */
#define ORACLE_OK 0
#define ORACLE_ERR_INVALID_ARGUMENT 1
#define ORACLE_ERR_OUT_OF_MEMORY 3
#define ORACLE_ERR_EMPTY 4
#define ORACLE_ERR_DEGENERATE 5
#define ORACLE_ERR_IO 6
#define ORACLE_ERR_PARSE 7
#define ORACLE_ERR_UNSUPPORTED 8

/* Build flags (same bit values as the product). */
#define ORACLE_FLAG_FULL_NEIGHBORS 0x1u /* real 27-neighbourhood (intended semantics) */
#define ORACLE_FLAG_DEDUP 0x2u          /* Morton-keyed vertex/edge/face dedup keys */
#define ORACLE_FLAG_STRICT_FP 0x4u      /* no FMA contraction anywhere */
#define ORACLE_FLAG_NO_VERT_EDGE 0x8u   /* skip the per-node vertex/edge arrays */

/* SVONode (src/SVO.h:20-35): 168 bytes. */
typedef struct oracle_node {
    uint32_t morton_code;
    uint8_t is_leaf;
    uint8_t pad_[3];
    float origin[3];
    float width;
    uint32_t parent;
    uint32_t childs[8];
    uint32_t neighbors[27];
} oracle_node;

/* thrust::pair<Eigen::Vector3f, uint32_t> (src/SVO.h:50): 16 bytes. */
typedef struct oracle_vertex {
    float pos[3];
    uint32_t owner;
} oracle_vertex;

/* thrust::pair<thrust_edge, uint32_t> (src/SVO.h:37,51): 28 bytes. */
typedef struct oracle_edge {
    float p0[3];
    float p1[3];
    uint32_t owner;
} oracle_edge;

typedef struct oracle_result oracle_result;

/* Reference OBJ loader.  Arrays are malloc'd; free with oracle_free. */
int oracle_load_obj(const char *path, float **points, int64_t *n_points, int32_t **tris,
                    int64_t *n_tris);
void oracle_free(void *p);

/* Bounding cube: out = {min[3], max[3], width[3]}. */
int oracle_bbox_cube(const float *points, int64_t n_points, float out[9]);

/* Morton code of (x,y,z), generalised to 64 bits (equal to the reference's
 * 32-bit code for coordinates < 1024). */
uint64_t oracle_morton_encode(uint32_t x, uint32_t y, uint32_t z);
void oracle_morton_decode(uint64_t code, uint32_t *x, uint32_t *y, uint32_t *z);

/* The oracle's neighbour (8x27, 8x27) and shared-corner/edge (8x8, 12x4)
 * tables, for comparison with the reference's. */
void oracle_tables(int16_t *nbr_parent, int16_t *nbr_child, int16_t *vert_shared,
                   int16_t *edge_shared);

/* The floating-point model on operand batches (see svo_oracle.cpp for ops). */
int oracle_set_fp_sites(const int *choice, int n);
int oracle_fp_eval(int op, int strict, const float *in, int64_t n, float *out);

/* Full create(): voxelize, octree levels, neighbours, vertex/edge arrays.
 * n_threads <= 0 means all hardware threads. */
int oracle_build(const float *points, int64_t n_points, const int32_t *tris, int64_t n_tris,
                 int res_x, int res_y, int res_z, uint32_t flags, int n_threads,
                 oracle_result **out);

/* Only the voxelizer: sorted unique Morton codes of surface voxels. */
int oracle_voxelize(const float *points, int64_t n_points, const int32_t *tris, int64_t n_tris,
                    int res_x, int res_y, int res_z, uint32_t flags, int n_threads,
                    uint64_t **codes, int64_t *n_codes);

void oracle_result_free(oracle_result *r);
int oracle_result_depth(const oracle_result *r);
int64_t oracle_result_num_nodes(const oracle_result *r);
int64_t oracle_result_num_vertices(const oracle_result *r);
int64_t oracle_result_num_edges(const oracle_result *r);
int64_t oracle_result_num_keys(const oracle_result *r);
/* level_counts[d] = node count of level d+1 (bottom-up), d < depth. */
int oracle_result_level_counts(const oracle_result *r, int64_t *counts, int cap);
const oracle_node *oracle_result_nodes(const oracle_result *r);
const oracle_vertex *oracle_result_vertices(const oracle_result *r);
const oracle_edge *oracle_result_edges(const oracle_result *r);
const uint64_t *oracle_result_keys(const oracle_result *r);
const float *oracle_result_bbox(const oracle_result *r); /* min[3], max[3], width[3] */
/* Dedup keys (ORACLE_FLAG_DEDUP): kind 0 = vertices, 1 = edges, 2 = faces. */
int64_t oracle_result_num_dedup(const oracle_result *r, int kind);
const uint64_t *oracle_result_dedup(const oracle_result *r, int kind);

/* writeTree: writes <path> exactly as the reference's std::ofstream writer. */
int oracle_write_tree(const oracle_result *r, const char *path);
int oracle_write_voxels(const oracle_result *r, const char *path);
int oracle_write_tree_nodes(const oracle_node *nodes, int64_t n, const char *path);

const char *oracle_last_error(void);

#ifdef __cplusplus
}
#endif
