// Floating-point contraction probe (test infrastructure, built by
// tests/test_gpu_fp_contraction.py with nvcc's default --fmad=true and with
// --fmad=false).  The expressions are written in plain float arithmetic in
// the evaluation order Eigen 3.4 gives the reference's vector code (fixed-size
// dot = a0*b0 + (a1*b1 + a2*b2), 2-term dot = a0*b0 + a1*b1, cross,
// normalized = v / sqrt(squaredNorm)), so nvcc decides the contractions
// exactly as it does when it compiles the reference; the test compares the
// results with the oracle's model of those decisions.
#include <cuda_runtime.h>

namespace {

struct V3 {
    float x, y, z;
};
struct V2 {
    float x, y;
};
__device__ __forceinline__ V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + (a.y * b.y + a.z * b.z); }
__device__ __forceinline__ float dot(V2 a, V2 b) { return a.x * b.x + a.y * b.y; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ V3 normalized(V3 v) {
    const float s = dot(v, v);
    if (s > 0.0f) {
        const float r = sqrtf(s);
        return {v.x / r, v.y / r, v.z / r};
    }
    return v;
}
__device__ __forceinline__ float mn(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float mx(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ int clampi(int f, int a, int b) {
    const int lo = f < b ? f : b;
    return a > lo ? a : lo;
}

__global__ void k_small(int op, const float *in, int n, float *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (op == 0) {
        const float *a = in + 4 * i;
        out[i] = dot(V2{a[0], a[1]}, V2{a[2], a[3]});
    } else if (op == 1) {
        const float *a = in + 6 * i;
        out[i] = dot(V3{a[0], a[1], a[2]}, V3{a[3], a[4], a[5]});
    } else if (op == 2) {
        const float *a = in + 4 * i;
        out[i] = a[0] * a[1] - a[2] * a[3];
    } else if (op == 3) {
        const float *a = in + 3 * i;
        out[i] = a[0] + a[1] * a[2];
    } else if (op == 4) {
        const float *a = in + 3 * i;
        const V3 r = normalized(V3{a[0], a[1], a[2]});
        out[3 * i] = r.x;
        out[3 * i + 1] = r.y;
        out[3 * i + 2] = r.z;
    }
}

// Triangle setup in the reference's statement order (grid origin and
// per-axis voxel size are runtime values).  Inputs per sample: triangle (9),
// target voxel (3), voxel size, resolution.
struct Setup {
    V3 nrm;
    float d1, d2;
    V2 nxy[3], nyz[3], nzx[3];
    float dxy[3], dyz[3], dzx[3];
    int lo[3], hi[3];
};

__device__ __forceinline__ void setup(const float *a, const float *org_p, Setup &s) {
    const int res = (int)a[13];
    const V3 org{org_p[0], org_p[1], org_p[2]};
    const V3 unit{a[12], a[12], a[12]};
    const int gmax[3] = {res - 1, res - 1, res - 1};
    const V3 v0 = sub(V3{a[0], a[1], a[2]}, org), v1 = sub(V3{a[3], a[4], a[5]}, org),
             v2 = sub(V3{a[6], a[7], a[8]}, org);
    const V3 e0 = sub(v1, v0), e1 = sub(v2, v1), e2 = sub(v0, v2);
    s.nrm = normalized(cross(e0, e1));
    const V3 bmin{mn(v0.x, mn(v1.x, v2.x)), mn(v0.y, mn(v1.y, v2.y)), mn(v0.z, mn(v1.z, v2.z))};
    const V3 bmax{mx(v0.x, mx(v1.x, v2.x)), mx(v0.y, mx(v1.y, v2.y)), mx(v0.z, mx(v1.z, v2.z))};
    s.lo[0] = clampi((int)(bmin.x / unit.x), 0, gmax[0]);
    s.lo[1] = clampi((int)(bmin.y / unit.y), 0, gmax[1]);
    s.lo[2] = clampi((int)(bmin.z / unit.z), 0, gmax[2]);
    s.hi[0] = clampi((int)(bmax.x / unit.x), 0, gmax[0]);
    s.hi[1] = clampi((int)(bmax.y / unit.y), 0, gmax[1]);
    s.hi[2] = clampi((int)(bmax.z / unit.z), 0, gmax[2]);
    V3 c{0.0f, 0.0f, 0.0f};
    if (s.nrm.x > 0.0f) c.x = unit.x;
    if (s.nrm.y > 0.0f) c.y = unit.y;
    if (s.nrm.z > 0.0f) c.z = unit.z;
    s.d1 = dot(s.nrm, sub(c, v0));
    s.d2 = dot(s.nrm, sub(sub(unit, c), v0));
    const V3 ev[3] = {e0, e1, e2}, vv[3] = {v0, v1, v2};
    for (int k = 0; k < 3; ++k) s.nxy[k] = V2{-1.0f * ev[k].y, ev[k].x};
    if (s.nrm.z < 0.0f)
        for (int k = 0; k < 3; ++k) s.nxy[k] = V2{-s.nxy[k].x, -s.nxy[k].y};
    for (int k = 0; k < 3; ++k)
        s.dxy[k] = (-1.0f * dot(s.nxy[k], V2{vv[k].x, vv[k].y})) + mx(0.0f, unit.x * s.nxy[k].x) +
                   mx(0.0f, unit.y * s.nxy[k].y);
    for (int k = 0; k < 3; ++k) s.nyz[k] = V2{-1.0f * ev[k].z, ev[k].y};
    if (s.nrm.x < 0.0f)
        for (int k = 0; k < 3; ++k) s.nyz[k] = V2{-s.nyz[k].x, -s.nyz[k].y};
    for (int k = 0; k < 3; ++k)
        s.dyz[k] = (-1.0f * dot(s.nyz[k], V2{vv[k].y, vv[k].z})) + mx(0.0f, unit.y * s.nyz[k].x) +
                   mx(0.0f, unit.z * s.nyz[k].y);
    for (int k = 0; k < 3; ++k) s.nzx[k] = V2{-1.0f * ev[k].x, ev[k].z};
    if (s.nrm.y < 0.0f)
        for (int k = 0; k < 3; ++k) s.nzx[k] = V2{-s.nzx[k].x, -s.nzx[k].y};
    for (int k = 0; k < 3; ++k)
        s.dzx[k] = (-1.0f * dot(s.nzx[k], V2{vv[k].z, vv[k].x})) + mx(0.0f, unit.z * s.nzx[k].x) +
                   mx(0.0f, unit.x * s.nzx[k].y);
}

// Setup values only: n, d1, d2, dxy, dyz, dzx (14 per sample).
__global__ void k_setup(const float *in, const float *org, int n, float *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Setup s;
    setup(in + 14 * i, org, s);
    float *o = out + 14 * i;
    o[0] = s.nrm.x; o[1] = s.nrm.y; o[2] = s.nrm.z; o[3] = s.d1; o[4] = s.d2;
    for (int k = 0; k < 3; ++k) {
        o[5 + k] = s.dxy[k];
        o[8 + k] = s.dyz[k];
        o[11 + k] = s.dzx[k];
    }
}

// The whole voxel test inside the reference's bbox triple loop (uint16
// counters); 1.0 when the target voxel passes.
__global__ void k_voxel(const float *in, const float *org, int n, float *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *a = in + 14 * i;
    const int tx = (int)a[9], ty = (int)a[10], tz = (int)a[11];
    const V3 unit{a[12], a[12], a[12]};
    Setup s;
    setup(a, org, s);
    float hit = 0.0f;
    for (unsigned short z = s.lo[2]; z <= s.hi[2]; z++) {
        for (unsigned short y = s.lo[1]; y <= s.hi[1]; y++) {
            for (unsigned short x = s.lo[0]; x <= s.hi[0]; x++) {
                const V3 p{x * unit.x, y * unit.y, z * unit.z};
                const float np = dot(s.nrm, p);
                if ((np + s.d1) * (np + s.d2) > 0.0f) continue;
                const V2 pxy{p.x, p.y};
                if ((dot(s.nxy[0], pxy) + s.dxy[0]) < 0.0f) continue;
                if ((dot(s.nxy[1], pxy) + s.dxy[1]) < 0.0f) continue;
                if ((dot(s.nxy[2], pxy) + s.dxy[2]) < 0.0f) continue;
                const V2 pyz{p.y, p.z};
                if ((dot(s.nyz[0], pyz) + s.dyz[0]) < 0.0f) continue;
                if ((dot(s.nyz[1], pyz) + s.dyz[1]) < 0.0f) continue;
                if ((dot(s.nyz[2], pyz) + s.dyz[2]) < 0.0f) continue;
                const V2 pzx{p.z, p.x};
                if ((dot(s.nzx[0], pzx) + s.dzx[0]) < 0.0f) continue;
                if ((dot(s.nzx[1], pzx) + s.dzx[1]) < 0.0f) continue;
                if ((dot(s.nzx[2], pzx) + s.dzx[2]) < 0.0f) continue;
                if (x == tx && y == ty && z == tz) hit = 1.0f;
            }
        }
    }
    out[i] = hit;
}

}  // namespace

extern "C" int fp_probe_run(int op, const float *h_in, int n, int k_in, int k_out, float *h_out) {
    float *d_in = nullptr, *d_out = nullptr, *d_org = nullptr;
    if (cudaMalloc(&d_in, sizeof(float) * (size_t)n * k_in) != cudaSuccess) return 1;
    if (cudaMalloc(&d_out, sizeof(float) * (size_t)n * k_out) != cudaSuccess) return 1;
    if (cudaMalloc(&d_org, sizeof(float) * 3) != cudaSuccess) return 1;
    cudaMemcpy(d_in, h_in, sizeof(float) * (size_t)n * k_in, cudaMemcpyHostToDevice);
    cudaMemset(d_org, 0, sizeof(float) * 3);
    const int blocks = (n + 127) / 128;
    if (op == 5)
        k_voxel<<<blocks, 128>>>(d_in, d_org, n, d_out);
    else if (op == 6)
        k_setup<<<blocks, 128>>>(d_in, d_org, n, d_out);
    else
        k_small<<<blocks, 128>>>(op, d_in, n, d_out);
    cudaError_t e = cudaMemcpy(h_out, d_out, sizeof(float) * (size_t)n * k_out, cudaMemcpyDeviceToHost);
    cudaFree(d_in);
    cudaFree(d_out);
    cudaFree(d_org);
    return e == cudaSuccess ? 0 : 2;
}
