// ref_dump.cu -- runs GPU-SVO's own build (the reference's unmodified
// src/SVO.cu + src/BaseModel.cpp, linked beside this file) on one OBJ mesh and
// dumps what it computed, for pinning the oracle and the product.
//
// TEST INFRASTRUCTURE ONLY: built by oracle/ref/build_ref.sh into oracle/_ref/
// and run by tests/golden/make_ref_fixtures.py.  Nothing in the product links
// or runs it.
//
//   ref_dump <mesh.obj> <res> <outdir> <stem> [tree]
//
// writes <outdir>/meta.json (depth, counts, depthNumNodes, bounding cube,
// timings) and, with `tree`, <outdir>/<stem>_<depth>_tree.obj
// (SparseVoxelOctree::writeTree, src/SVO.cu:737-753); then streams to stdout
// the magic "SVOREF1" + NUL, four u64 counts (nodes, vertices, edges, voxels)
// and the arrays themselves, in that order:
//   nodes      svoNodeArray, 168 B per SVONode (src/SVO.h:20-35); the three
//              padding bytes after isLeaf are zeroed (the reference leaves
//              them indeterminate)
//   vertices   nodeVertexArray, 16 B per pair<Vector3f, uint32_t>
//   edges      nodeEdgeArray, 28 B per pair<pair<Vector3f, Vector3f>, uint32_t>
//   voxels     the surface voxels of surfaceVoxelize (src/SVO.cu:37-188): the
//              Morton codes whose dense-array entry carries the flag bit,
//              ascending, u32
//
// The results are private members of SparseVoxelOctree; they are read through
// pointers to members formed in explicit template instantiations (where
// access checking does not apply), so the reference's headers stay unmodified.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <unistd.h>

#include "SVO.h"

namespace {

template <typename Tag, typename Tag::type M>
struct Expose {
    friend typename Tag::type get(Tag) { return M; }
};

struct NodesTag {
    typedef std::vector<SVONode> SparseVoxelOctree::*type;
    friend type get(NodesTag);
};
struct VertsTag {
    typedef std::vector<thrust::pair<Eigen::Vector3f, uint32_t>> SparseVoxelOctree::*type;
    friend type get(VertsTag);
};
struct EdgesTag {
    typedef std::vector<thrust::pair<thrust_edge, uint32_t>> SparseVoxelOctree::*type;
    friend type get(EdgesTag);
};
struct DepthTag {
    typedef int SparseVoxelOctree::*type;
    friend type get(DepthTag);
};
struct DepthNumTag {
    typedef std::vector<size_t> SparseVoxelOctree::*type;
    friend type get(DepthNumTag);
};
struct BBoxTag {
    typedef AABox<Eigen::Vector3f> BaseModel::*type;
    friend type get(BBoxTag);
};
struct VoxelizeTag {
    typedef void (SparseVoxelOctree::*type)(const Eigen::Vector3i *, const Eigen::Vector3f *,
                                            const Eigen::Vector3f *, thrust::device_vector<uint32_t> &);
    friend type get(VoxelizeTag);
};

template struct Expose<NodesTag, &SparseVoxelOctree::svoNodeArray>;
template struct Expose<VertsTag, &SparseVoxelOctree::nodeVertexArray>;
template struct Expose<EdgesTag, &SparseVoxelOctree::nodeEdgeArray>;
template struct Expose<DepthTag, &SparseVoxelOctree::treeDepth>;
template struct Expose<DepthNumTag, &SparseVoxelOctree::depthNumNodes>;
template struct Expose<BBoxTag, &BaseModel::modelBBox>;
template struct Expose<VoxelizeTag, &SparseVoxelOctree::meshVoxelize>;

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void die(const char *what) {
    std::fprintf(stderr, "ref_dump: %s\n", what);
    std::exit(2);
}

void check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "ref_dump: %s: %s\n", what, cudaGetErrorString(e));
        std::exit(2);
    }
}

FILE *g_bin = nullptr;  // the original stdout; fd 1 itself is pointed at stderr

template <typename T>
void put(const T *data, size_t n) {
    if (n && std::fwrite(data, sizeof(T), n, g_bin) != n) die("short write to stdout");
}

// 3-D interleave of (x, y, z), x in the lowest bit (the reference's order).
uint64_t interleave(uint32_t x, uint32_t y, uint32_t z) {
    uint64_t m = 0;
    for (int b = 0; b < 21; ++b)
        m |= (uint64_t)((x >> b) & 1) << (3 * b) | (uint64_t)((y >> b) & 1) << (3 * b + 1) |
             (uint64_t)((z >> b) & 1) << (3 * b + 2);
    return m;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc != 5 && !(argc == 6 && std::strcmp(argv[5], "tree") == 0))
        die("usage: ref_dump <mesh.obj> <res> <outdir> <stem> [tree]");
    const bool tree = argc == 6;
    // the reference prints progress lines with printf; keep them off the binary stream
    std::fflush(stdout);
    const int bin_fd = dup(STDOUT_FILENO);
    if (bin_fd < 0 || dup2(STDERR_FILENO, STDOUT_FILENO) < 0 || !(g_bin = fdopen(bin_fd, "wb")))
        die("cannot redirect stdout");
    const std::string mesh = argv[1], outdir = argv[3], stem = argv[4];
    const int res = std::atoi(argv[2]);
    if (res < 2 || res > 1024) die("resolution must be in [2, 1024] (32-bit Morton codes)");
    check(cudaFree(nullptr), "context");

    const double t0 = now_ms();
    SparseVoxelOctree svo(mesh, res, res, res);  // BaseModel: loadOBJ + bounding cube
    const double t1 = now_ms();
    svo.create();
    check(cudaDeviceSynchronize(), "create");
    const double t2 = now_ms();
    if (tree) svo.writeTree(outdir + "/" + stem);
    const double t3 = now_ms();

    std::vector<SVONode> &nodes = svo.*get(NodesTag());
    for (SVONode &n : nodes) std::memset(reinterpret_cast<unsigned char *>(&n) + 5, 0, 3);
    static_assert(sizeof(SVONode) == 168, "SVONode layout");
    const auto &verts = svo.*get(VertsTag());
    const auto &edges = svo.*get(EdgesTag());
    static_assert(sizeof(verts[0]) == 16 && sizeof(edges[0]) == 28, "pair layouts");

    // The voxelizer alone, with create()'s own prologue (src/SVO.cu:343-365):
    // a zeroed dense array of morton(res-1)^3 + 1 entries and the per-axis
    // voxel size width / res.
    const AABox<Eigen::Vector3f> bbox = svo.*get(BBoxTag());
    const Eigen::Vector3i grid(res, res, res);
    const Eigen::Vector3f unit(bbox.width.x() / grid.x(), bbox.width.y() / grid.y(), bbox.width.z() / grid.z());
    const size_t dense_n = (size_t)interleave(res - 1, res - 1, res - 1) + 1;
    Eigen::Vector3i *d_grid;
    Eigen::Vector3f *d_unit, *d_origin;
    check(cudaMalloc(&d_grid, sizeof(grid)), "malloc");
    check(cudaMalloc(&d_unit, sizeof(unit)), "malloc");
    check(cudaMalloc(&d_origin, sizeof(bbox.min)), "malloc");
    check(cudaMemcpy(d_grid, &grid, sizeof(grid), cudaMemcpyHostToDevice), "copy");
    check(cudaMemcpy(d_unit, &unit, sizeof(unit), cudaMemcpyHostToDevice), "copy");
    check(cudaMemcpy(d_origin, &bbox.min, sizeof(bbox.min), cudaMemcpyHostToDevice), "copy");
    std::vector<uint32_t> voxels;
    double vox_ms;
    {
        thrust::device_vector<uint32_t> dense(dense_n, 0);
        const double v0 = now_ms();
        (svo.*get(VoxelizeTag()))(d_grid, d_unit, d_origin, dense);
        check(cudaDeviceSynchronize(), "voxelize");
        vox_ms = now_ms() - v0;
        std::vector<uint32_t> h(dense_n);
        check(cudaMemcpy(h.data(), dense.data().get(), dense_n * 4, cudaMemcpyDeviceToHost), "copy back");
        for (size_t i = 0; i < dense_n; ++i)
            if (h[i] >> 31) {
                if ((h[i] & 0x7FFFFFFFu) != (uint32_t)i) die("dense entry does not hold its own code");
                voxels.push_back((uint32_t)i);
            }
    }
    cudaFree(d_grid);
    cudaFree(d_unit);
    cudaFree(d_origin);

    const int depth = svo.*get(DepthTag());
    const auto &dn = svo.*get(DepthNumTag());
    FILE *f = std::fopen((outdir + "/meta.json").c_str(), "w");
    if (!f) die("cannot write meta.json");
    std::fprintf(f, "{\"depth\": %d, \"num_nodes\": %zu, \"num_vertices\": %zu, \"num_edges\": %zu, "
                    "\"num_voxels\": %zu, \"depth_num_nodes\": [",
                 depth, nodes.size(), verts.size(), edges.size(), voxels.size());
    for (size_t i = 0; i < dn.size(); ++i) std::fprintf(f, "%s%zu", i ? ", " : "", dn[i]);
    std::fprintf(f, "], \"bbox\": [");
    const float bb[9] = {bbox.min.x(), bbox.min.y(), bbox.min.z(), bbox.max.x(), bbox.max.y(),
                         bbox.max.z(), bbox.width.x(), bbox.width.y(), bbox.width.z()};
    for (int i = 0; i < 9; ++i) std::fprintf(f, "%s%.9g", i ? ", " : "", bb[i]);
    std::fprintf(f, "], \"load_ms\": %.3f, \"create_ms\": %.3f, \"write_tree_ms\": %.3f, \"voxelize_ms\": %.3f}\n",
                 t1 - t0, t2 - t1, t3 - t2, vox_ms);
    std::fclose(f);

    const char magic[8] = {'S', 'V', 'O', 'R', 'E', 'F', '1', 0};
    const uint64_t counts[4] = {nodes.size(), verts.size(), edges.size(), voxels.size()};
    put(magic, 8);
    put(counts, 4);
    put(nodes.data(), nodes.size());
    put(verts.data(), verts.size());
    put(edges.data(), edges.size());
    put(voxels.data(), voxels.size());
    if (std::fflush(g_bin) != 0) die("flush");
    return 0;
}
