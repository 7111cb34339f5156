// svo_main -- command line of the reference's main.cpp:7-17:
//   svo_main [mesh.obj = bunny.obj] [resolution = 64]
// builds the octree at resolution^3 and writes <stem>_<depth>_tree.obj.
#include <filesystem>
#include <string>

#include "svo/SVO.h"

int main(int argc, char **argv) {
    const std::string mesh = argc > 1 ? argv[1] : "bunny.obj";
    const int res = argc > 2 ? std::stoi(argv[2]) : 64;
    SparseVoxelOctree svo(mesh, res, res, res);
    svo.create();
    svo.writeTree(std::filesystem::path(mesh).stem().string());
    return 0;
}
