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

__device__ __forceinline__ void add_fix3(long long *arr, int n, int i, V3 v, double s) {
    arr[i] += to_fix(s * v.x, FRC_SCALE);
    arr[n + i] += to_fix(s * v.y, FRC_SCALE);
    arr[2 * n + i] += to_fix(s * v.z, FRC_SCALE);
}

}  // namespace smd
