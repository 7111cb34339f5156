#!/bin/sh
# Builds GPU-SVO itself, from its unmodified sources where they lie, into
# oracle/_ref/ (git-ignored; the built files travel with the repository to a
# GPU machine).  Test infrastructure only: these binaries pin the oracle and
# the product to the reference's own outputs.
#
#   oracle/_ref/pin_morton  harness over the reference's src/MortonLUT.h
#   oracle/_ref/ref_main    the reference's CLI (main.cpp): main <mesh.obj> <res>
#   oracle/_ref/ref_main_ndebug  the same built with NDEBUG, where create() also
#                           writes bunny_1_voxel.obj with writeVoxel
#   oracle/_ref/ref_dump    oracle/ref/ref_dump.cu over the reference's build:
#                           dumps nodes, vertex/edge arrays, voxels, tree .obj
#
# The reference's CMake step fetches Eigen 3.4 from the network
# (cmake/eigen.cmake:9-14); oracle/ref/eigen_api/Eigen/Dense stands in for the
# part of Eigen it uses.  src/BaseModel.cpp calls the MSVC-only sscanf_s with
# %f/%d conversions only, where it behaves as sscanf (-Dsscanf_s=sscanf).
# Device code is compiled for sm_100a with nvcc's defaults (FMA contraction
# on), as the reference's CMakeLists.txt does (it sets no architecture and no
# optimisation flags); NDEBUG stays undefined, as in its default build type, so
# create() does not write its debug voxel file (ref_main_ndebug does).
#
# The reference tree is GPU_SVO_REF (default /root/reference); without it,
# nothing is built and the script exits 0.
set -e
REF=${GPU_SVO_REF:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
if [ ! -f "$REF/src/SVO.cu" ]; then
    echo "reference sources not found under $REF: nothing built" >&2
    exit 0
fi
exec make -s -C "$HERE" REF="$REF"
