// SVO.h -- drop-in for the reference's src/SVO.h (SVONode,
// SparseVoxelOctree) on top of the C ABI in svo_b200.h.  create() runs the
// sm_100a build and leaves the same host arrays the reference leaves.
#pragma once

#include <climits>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "BaseModel.h"

// SVONode (src/SVO.h:20-35), 168 bytes, same field order and defaults.
struct SVONode {
    uint32_t mortonCode = 0;
    bool isLeaf = true;
    Vec3f origin;
    float width = 0.0f;
    unsigned int parent{UINT_MAX};
    unsigned int childs[8];
    unsigned int neighbors[27];
    SVONode() {
        for (int i = 0; i < 8; ++i) childs[i] = UINT_MAX;
        for (int i = 0; i < 27; ++i) neighbors[i] = UINT_MAX;
    }
};
static_assert(sizeof(SVONode) == sizeof(svo_node), "SVONode layout");

using NodeVertex = std::pair<Vec3f, uint32_t>;                    // src/SVO.h:50
using NodeEdge = std::pair<std::pair<Vec3f, Vec3f>, uint32_t>;   // src/SVO.h:37,51
static_assert(sizeof(NodeVertex) == sizeof(svo_vertex) && sizeof(NodeEdge) == sizeof(svo_edge), "pair layouts");

// SparseVoxelOctree (src/SVO.h:39-89).
struct SparseVoxelOctree : public BaseModel {
private:
    int treeDepth = 0;
    size_t numTreeNodes = 0;
    Vec3i surfaceVoxelGridSize;
    std::vector<size_t> depthNumNodes;
    std::vector<SVONode> svoNodeArray;
    std::vector<NodeVertex> nodeVertexArray;
    std::vector<NodeEdge> nodeEdgeArray;
    std::vector<uint64_t> voxelKeys;
    uint32_t buildFlags = 0;

public:
    SparseVoxelOctree() : treeDepth(0) {}
    SparseVoxelOctree(const std::string &filename, const Vec3i &gridSize)
        : BaseModel(filename), surfaceVoxelGridSize(gridSize) {}
    SparseVoxelOctree(const std::string &filename, const int &grid_x, const int &grid_y, const int &grid_z)
        : BaseModel(filename), surfaceVoxelGridSize(grid_x, grid_y, grid_z) {}

    // Builds the octree on the GPU and copies nodes, vertices and edges to the
    // host members; prints "Sparse Voxel Octree depth: <d>" like the
    // reference.  Errors print a message and exit(EXIT_FAILURE), as the
    // reference's CUDA_CHECK does.
    void create();
    // Writes "<base>_<depth>_tree.obj" (src/SVO.cu:737-753).
    void writeTree(const std::string base_filename);
    // Writes "<base>_<depth>_voxel.obj" from 32-bit codes whose bit 31 may be
    // the reference's surface flag (src/SVO.cu:755-777).
    void writeVoxel(const std::vector<uint32_t> &voxelArray, const std::string &base_filename, const float &width);

    // Build options (svo_b200.h SVO_FLAG_*); default 0 = reference behaviour.
    void setBuildFlags(uint32_t flags) { buildFlags = flags; }

    // Read access to what the reference keeps private.
    int depth() const { return treeDepth; }
    size_t numNodes() const { return numTreeNodes; }
    const std::vector<size_t> &levelNodeCounts() const { return depthNumNodes; }
    const std::vector<SVONode> &nodes() const { return svoNodeArray; }
    const std::vector<NodeVertex> &vertices() const { return nodeVertexArray; }
    const std::vector<NodeEdge> &edges() const { return nodeEdgeArray; }
    const std::vector<uint64_t> &surfaceVoxels() const { return voxelKeys; }
};
