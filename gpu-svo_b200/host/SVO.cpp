// SVO.cpp -- the C++ facade (include/svo/SVO.h, include/svo/BaseModel.h):
// the reference's SparseVoxelOctree / BaseModel interface over the C ABI.
#include "svo/SVO.h"

#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <mutex>

namespace {

[[noreturn]] void die(const char *what) {
    std::fprintf(stderr, "SVO error: %s: %s\n", what, svo_last_error());
    std::exit(EXIT_FAILURE);
}

// One context per process, on the current device (the reference uses the
// default device through the runtime API).
svo_ctx *process_ctx() {
    static std::once_flag once;
    static svo_ctx *ctx = nullptr;
    std::call_once(once, [] {
        if (svo_ctx_create(0, &ctx) != SVO_OK) die("svo_ctx_create");
    });
    return ctx;
}

}  // namespace

AABox<Vec3f> createMeshBBCube(AABox<Vec3f> box) {
    // svo_bbox_cube works from points; the two corners span the same box.
    const float pts[6] = {box.min[0], box.min[1], box.min[2], box.max[0], box.max[1], box.max[2]};
    svo_aabb out;
    if (svo_bbox_cube(pts, 2, &out) != SVO_OK) die("createMeshBBCube");
    AABox<Vec3f> r;
    for (int i = 0; i < 3; ++i) {
        r.min[i] = out.min[i];
        r.max[i] = out.max[i];
        r.width[i] = out.width[i];
    }
    return r;
}

BaseModel::BaseModel(const std::string &filename) {
    loadOBJ(filename);
    nModelTris = idx2Points.size();
    nPoints = modelPoints.size();
    svo_aabb box;
    if (svo_bbox_cube(reinterpret_cast<const float *>(modelPoints.data()), (int64_t)nPoints, &box) != SVO_OK)
        die("bounding box");
    for (int i = 0; i < 3; ++i) {
        modelBBox.min[i] = box.min[i];
        modelBBox.max[i] = box.max[i];
        modelBBox.width[i] = box.width[i];
    }
}

void BaseModel::loadOBJ(const std::string &in_file) {
    float *pts = nullptr;
    int32_t *tris = nullptr;
    int64_t np = 0, nt = 0;
    const int rc = svo_load_obj(in_file.c_str(), &pts, &np, &tris, &nt);
    if (rc == SVO_ERR_IO) {
        std::cerr << "ERROR: loading obj:(" << in_file << ") file is not good" << std::endl;
        std::exit(1);
    }
    if (rc != SVO_OK) die("loadOBJ");
    modelPoints.resize((size_t)np);
    idx2Points.resize((size_t)nt);
    for (int64_t i = 0; i < np; ++i) modelPoints[i] = Vec3f(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
    for (int64_t i = 0; i < nt; ++i) idx2Points[i] = Vec3i(tris[3 * i], tris[3 * i + 1], tris[3 * i + 2]);
    svo_free_host(pts);
    svo_free_host(tris);
}

void SparseVoxelOctree::create() {
    svo_result *r = nullptr;
    const int rc = svo_build(process_ctx(), reinterpret_cast<const float *>(modelPoints.data()), (int64_t)nPoints,
                             reinterpret_cast<const int32_t *>(idx2Points.data()), (int64_t)nModelTris,
                             surfaceVoxelGridSize.x(), surfaceVoxelGridSize.y(), surfaceVoxelGridSize.z(),
                             buildFlags, nullptr, &r);
    if (rc != SVO_OK) die("create");
    treeDepth = svo_result_depth(r);
    numTreeNodes = (size_t)svo_result_num_nodes(r);
    int64_t counts[64];
    const int nl = svo_result_level_counts(r, counts, 64);
    depthNumNodes.clear();
    for (int l = 0; l + 1 < nl; ++l) depthNumNodes.push_back((size_t)counts[l]);  // the root level is not listed
    svoNodeArray.resize(numTreeNodes);
    nodeVertexArray.resize((size_t)svo_result_num_vertices(r));
    nodeEdgeArray.resize((size_t)svo_result_num_edges(r));
    voxelKeys.resize((size_t)svo_result_num_keys(r));
    if (svo_result_copy_nodes(r, reinterpret_cast<svo_node *>(svoNodeArray.data()), (int64_t)svoNodeArray.size()) ||
        svo_result_copy_vertices(r, reinterpret_cast<svo_vertex *>(nodeVertexArray.data()),
                                 (int64_t)nodeVertexArray.size()) ||
        svo_result_copy_edges(r, reinterpret_cast<svo_edge *>(nodeEdgeArray.data()), (int64_t)nodeEdgeArray.size()) ||
        svo_result_copy_keys(r, voxelKeys.data(), (int64_t)voxelKeys.size()))
        die("copy results");
    svo_result_free(r);
#ifdef NDEBUG
    // the reference's release build dumps the surface voxels of level 1 under
    // a fixed name (src/SVO.cu:410-419)
    {
        std::vector<uint32_t> codes(voxelKeys.begin(), voxelKeys.end());
        const int depth = treeDepth;
        treeDepth = 1;
        writeVoxel(codes, "bunny", modelBBox.width.x() / (float)surfaceVoxelGridSize.x());
        treeDepth = depth;
    }
#endif
    std::printf("Sparse Voxel Octree depth: %d\n", treeDepth);
}

void SparseVoxelOctree::writeTree(const std::string base_filename) {
    const std::string name = base_filename + "_" + std::to_string(treeDepth) + "_tree.obj";
#ifndef SILENT
    std::fprintf(stdout, "[I/O] Writing octree data in obj format to file %s \n", name.c_str());
#endif
    if (svo_write_tree_nodes(reinterpret_cast<const svo_node *>(svoNodeArray.data()), (int64_t)svoNodeArray.size(),
                             name.c_str()) != SVO_OK)
        die("writeTree");
}

void SparseVoxelOctree::writeVoxel(const std::vector<uint32_t> &voxelArray, const std::string &base_filename,
                                   const float &width) {
    const std::string name = base_filename + "_" + std::to_string(treeDepth) + "_voxel.obj";
#ifndef SILENT
    std::fprintf(stdout, "[I/O] Writing data in obj voxels format to file %s \n", name.c_str());
#endif
    std::vector<uint64_t> keys(voxelArray.size());
    for (size_t i = 0; i < keys.size(); ++i) keys[i] = voxelArray[i] & 0x7FFFFFFFu;
    if (svo_write_voxel_keys(keys.data(), (int64_t)keys.size(), modelBBox.min.v, width, name.c_str()) != SVO_OK)
        die("writeVoxel");
}
