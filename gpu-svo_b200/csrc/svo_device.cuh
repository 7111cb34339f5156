// svo_device.cuh -- device helpers shared by the octree build kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace svo {

constexpr uint32_t kNone = 0xFFFFFFFFu;  // UINT_MAX, "no index" in the node records

// ---------------------------------------------------------------------------
// Morton codes: bit i of x/y/z -> bit 3i/3i+1/3i+2, 21 bits per axis in a
// u64.  For coordinates < 1024 the low 32 bits equal the reference's LUT
// encoder (src/MortonLUT.h:482-501) exactly.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint64_t spread3(uint64_t v) {
    v &= 0x1FFFFFull;
    v = (v | (v << 32)) & 0x1F00000000FFFFull;
    v = (v | (v << 16)) & 0x1F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}
__host__ __device__ __forceinline__ uint32_t compact3(uint64_t v) {
    v &= 0x1249249249249249ull;
    v = (v | (v >> 2)) & 0x10C30C30C30C30C3ull;
    v = (v | (v >> 4)) & 0x100F00F00F00F00Full;
    v = (v | (v >> 8)) & 0x1F0000FF0000FFull;
    v = (v | (v >> 16)) & 0x1F00000000FFFFull;
    v = (v | (v >> 32)) & 0x1FFFFFull;
    return (uint32_t)v;
}
__host__ __device__ __forceinline__ uint64_t morton3(uint32_t x, uint32_t y, uint32_t z) {
    return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}

// Dilated (Morton-interleaved) coordinates: x at bits 0,3,6,..., y at
// 1,4,7,..., z at 2,5,8,....  A coordinate can be stepped without decoding:
// for xm = code & kDilX, (xm - 1) & kDilX is x - 1 (x >= 1) and
// ((xm | ~kDilX) + 1) & kDilX is x + 1; comparisons of dilated values follow
// the coordinates.
constexpr uint64_t kDilX = 0x1249249249249249ull, kDilY = kDilX << 1, kDilZ = kDilX << 2;
__host__ __device__ __forceinline__ uint64_t dil_dec(uint64_t m, uint64_t mask) {
    return (m - (mask & (~mask + 1))) & mask;  // mask & -mask: the axis's lowest bit
}
__host__ __device__ __forceinline__ uint64_t dil_inc(uint64_t m, uint64_t mask) {
    return ((m | ~mask) + (mask & (~mask + 1))) & mask;
}

#if defined(__CUDACC__)
// ---------------------------------------------------------------------------
// Floating-point model.  The reference's voxel test and node origins are
// Eigen 3.4 expressions compiled by nvcc with --fmad=true.  Eigen evaluates a
// 3-term dot as a0*b0 + (a1*b1 + a2*b2) and a 2-term dot as a0*b0 + a1*b1;
// nvcc fuses products into the adds consuming them.  Which product it fuses
// was measured on nvcc 12.9 with the reference's loop structure: the first
// one, except in the squared norm's inner sum and in the first two ZX edge
// tests of the voxel loop (see tri_setup / voxel_test).  Every operation here
// is an explicit round-to-nearest intrinsic, so the compiler cannot re-fuse
// or reorder anything: STRICT=false reproduces the fused pattern,
// STRICT=true rounds every operation.
// ---------------------------------------------------------------------------
template <bool STRICT>
struct Fp {
    static __device__ __forceinline__ float dot2(float a0, float a1, float b0, float b1) {
        return STRICT ? __fadd_rn(__fmul_rn(a0, b0), __fmul_rn(a1, b1))
                      : __fmaf_rn(a0, b0, __fmul_rn(a1, b1));
    }
    // a0*b0 + a1*b1 inside the voxel loop when only the second product varies
    // with x: nvcc hoists the first product out of the loop, then fuses the
    // second (the ZX projection test).
    static __device__ __forceinline__ float dot2_late(float a0, float a1, float b0, float b1) {
        return STRICT ? __fadd_rn(__fmul_rn(a0, b0), __fmul_rn(a1, b1))
                      : __fmaf_rn(a1, b1, __fmul_rn(a0, b0));
    }
    // a1*b1 + a2*b2 (inner part of a 3-term dot)
    static __device__ __forceinline__ float dot3_tail(float a1, float a2, float b1, float b2) {
        return STRICT ? __fadd_rn(__fmul_rn(a1, b1), __fmul_rn(a2, b2))
                      : __fmaf_rn(a1, b1, __fmul_rn(a2, b2));
    }
    // a0*b0 + tail
    static __device__ __forceinline__ float dot3_head(float a0, float b0, float tail) {
        return STRICT ? __fadd_rn(__fmul_rn(a0, b0), tail) : __fmaf_rn(a0, b0, tail);
    }
    static __device__ __forceinline__ float dot3(float a0, float a1, float a2, float b0, float b1,
                                                 float b2) {
        return dot3_head(a0, b0, dot3_tail(a1, a2, b1, b2));
    }
    // a*b - c*d (one cross-product component)
    static __device__ __forceinline__ float diffprod(float a, float b, float c, float d) {
        return STRICT ? __fsub_rn(__fmul_rn(a, b), __fmul_rn(c, d))
                      : __fmaf_rn(a, b, -__fmul_rn(c, d));
    }
    // o + w * x (node origin component)
    static __device__ __forceinline__ float origin(float o, float w, float x) {
        return STRICT ? __fadd_rn(o, __fmul_rn(w, x)) : __fmaf_rn(w, x, o);
    }
};

// The reference's float min/max (src/CUDAUtil.h:72-80): plain compares.
__device__ __forceinline__ float cminf(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float cmaxf(float a, float b) { return a > b ? a : b; }
#endif  // __CUDACC__

// ---------------------------------------------------------------------------
// Grid parameters, computed on the device from the mesh's vertices.
// ---------------------------------------------------------------------------
struct GridParams {
    float origin[3];  // modelBBox.min
    float unit[3];    // unitVoxelSize
    float bbox[9];    // min, max, width
    uint32_t status;  // kStatus* bits of this mesh
    uint32_t pad_;
};

// Status word bits reported back to the host.
enum : uint32_t {
    kStatusNonFinite = 1u,
    kStatusBigOverflow = 2u,
    kStatusScanTimeout = 4u,
    kStatusBadIndex = 8u,  // a triangle names a vertex outside the mesh (that triangle is skipped)
};

}  // namespace svo
