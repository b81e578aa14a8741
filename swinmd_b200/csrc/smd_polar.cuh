// Small vector/tensor helpers for the multipole and induction kernels.
// Quadrupoles are symmetric 3x3 tensors stored as (xx, xy, xz, yy, yz, zz).
#pragma once
#include "smd_common.cuh"

namespace smd {

struct V3 {
    double x, y, z;
};
__device__ __forceinline__ V3 v3(double x, double y, double z) { return {x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 crs(V3 a, V3 b) {
    return {a.y * b.z - b.y * a.z, b.x * a.z - a.x * b.z, a.x * b.y - b.x * a.y};
}
__device__ __forceinline__ double len(V3 a) { return sqrt(dot(a, a)); }

struct Q6 {
    double xx, xy, xz, yy, yz, zz;
};
__device__ __forceinline__ V3 qv(const Q6 &q, V3 r) {
    return {q.xx * r.x + q.xy * r.y + q.xz * r.z, q.xy * r.x + q.yy * r.y + q.yz * r.z,
            q.xz * r.x + q.yz * r.y + q.zz * r.z};
}
__device__ __forceinline__ double qtr(const Q6 &q) { return q.xx + q.yy + q.zz; }
__device__ __forceinline__ double qdd(const Q6 &a, const Q6 &b) {
    return a.xx * b.xx + a.yy * b.yy + a.zz * b.zz + 2.0 * (a.xy * b.xy + a.xz * b.xz + a.yz * b.yz);
}
// sum over columns c of col_c(A) x col_c(B) (the reference's matrix "cross")
__device__ __forceinline__ V3 qcross(const Q6 &a, const Q6 &b) {
    V3 a0 = v3(a.xx, a.xy, a.xz), a1 = v3(a.xy, a.yy, a.yz), a2 = v3(a.xz, a.yz, a.zz);
    V3 b0 = v3(b.xx, b.xy, b.xz), b1 = v3(b.xy, b.yy, b.yz), b2 = v3(b.xz, b.yz, b.zz);
    return crs(a0, b0) + crs(a1, b1) + crs(a2, b2);
}

// FP32 counterparts for the mixed-precision pair algebra
struct F3 {
    float x, y, z;
};
__device__ __forceinline__ F3 f3(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ F3 operator+(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ F3 operator-(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ F3 operator-(F3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ F3 operator*(float s, F3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ float dot(F3 a, F3 b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }
__device__ __forceinline__ F3 crs(F3 a, F3 b) {
    return {a.y * b.z - b.y * a.z, b.x * a.z - a.x * b.z, a.x * b.y - b.x * a.y};
}
struct Q6F {
    float xx, xy, xz, yy, yz, zz;
};
__device__ __forceinline__ F3 qv(const Q6F &q, F3 r) {
    return {fmaf(q.xx, r.x, fmaf(q.xy, r.y, q.xz * r.z)), fmaf(q.xy, r.x, fmaf(q.yy, r.y, q.yz * r.z)),
            fmaf(q.xz, r.x, fmaf(q.yz, r.y, q.zz * r.z))};
}
__device__ __forceinline__ float qtr(const Q6F &q) { return q.xx + q.yy + q.zz; }
__device__ __forceinline__ float qdd(const Q6F &a, const Q6F &b) {
    return a.xx * b.xx + a.yy * b.yy + a.zz * b.zz + 2.f * (a.xy * b.xy + a.xz * b.xz + a.yz * b.yz);
}
__device__ __forceinline__ F3 qcross(const Q6F &a, const Q6F &b) {
    F3 a0 = f3(a.xx, a.xy, a.xz), a1 = f3(a.xy, a.yy, a.yz), a2 = f3(a.xz, a.yz, a.zz);
    F3 b0 = f3(b.xx, b.xy, b.xz), b1 = f3(b.xy, b.yy, b.yz), b2 = f3(b.xz, b.yz, b.zz);
    return crs(a0, b0) + crs(a1, b1) + crs(a2, b2);
}
__device__ __forceinline__ V3 to_v3(F3 a) { return v3(a.x, a.y, a.z); }

__device__ __forceinline__ void add_fix3(long long *arr, int n, int i, V3 v, double s) {
    arr[i] += to_fix(s * v.x, FRC_SCALE);
    arr[n + i] += to_fix(s * v.y, FRC_SCALE);
    arr[2 * n + i] += to_fix(s * v.z, FRC_SCALE);
}

}  // namespace smd
