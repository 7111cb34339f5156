// BaseModel.h -- drop-in for the reference's src/BaseModel.h (BaseModel,
// AABox, createMeshBBCube) on top of the C ABI in svo_b200.h.  Eigen is not
// required: Vec3f / Vec3i are 12-byte value types with the accessors the
// reference's code uses (x(), y(), z(), operator[]).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "svo_b200.h"

struct Vec3f {
    float v[3] = {0.0f, 0.0f, 0.0f};
    Vec3f() = default;
    Vec3f(float x, float y, float z) : v{x, y, z} {}
    float &operator[](int i) { return v[i]; }
    const float &operator[](int i) const { return v[i]; }
    float &x() { return v[0]; }
    float &y() { return v[1]; }
    float &z() { return v[2]; }
    const float &x() const { return v[0]; }
    const float &y() const { return v[1]; }
    const float &z() const { return v[2]; }
};

struct Vec3i {
    int v[3] = {0, 0, 0};
    Vec3i() = default;
    Vec3i(int x, int y, int z) : v{x, y, z} {}
    int &operator[](int i) { return v[i]; }
    const int &operator[](int i) const { return v[i]; }
    int &x() { return v[0]; }
    int &y() { return v[1]; }
    int &z() { return v[2]; }
    const int &x() const { return v[0]; }
    const int &y() const { return v[1]; }
    const int &z() const { return v[2]; }
};
static_assert(sizeof(Vec3f) == 12 && sizeof(Vec3i) == 12, "12-byte vectors");

// AABox<Real> (src/BaseModel.h:10-22).
template <typename Real>
struct AABox {
    Real min;
    Real max;
    Real width;
    AABox() = default;
    AABox(Real mn, Real mx) : min(mn), max(mx) {
        for (int i = 0; i < 3; ++i) width[i] = mx[i] - mn[i];
    }
};

// createMeshBBCube (src/BaseModel.h:24-49), for float boxes.
AABox<Vec3f> createMeshBBCube(AABox<Vec3f> box);

// BaseModel (src/BaseModel.h:51-76): the loaded mesh and its bounding cube.
class BaseModel {
protected:
    size_t nModelTris = 0;
    size_t nPoints = 0;
    std::vector<Vec3i> idx2Points;
    std::vector<Vec3f> modelPoints;
    AABox<Vec3f> modelBBox;

public:
    BaseModel() {}
    // loadOBJ, then the bounding cube of all vertices.  As in the reference,
    // an unreadable file prints "ERROR: loading obj:(<file>) file is not good"
    // and exits with status 1.
    explicit BaseModel(const std::string &filename);
    void loadOBJ(const std::string &in_file);

    const std::vector<Vec3f> &points() const { return modelPoints; }
    const std::vector<Vec3i> &triangles() const { return idx2Points; }
    const AABox<Vec3f> &bbox() const { return modelBBox; }
};
