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

// Extrapolation over the dipole history ring ph ([4][6][N]: p x y z, E0 x y
// z per stored step, slot (count - k) & 3 for step t - k): with k = min(order,
// cnt) steps and the alternating binomial weights w_j (1; 2, -1; 3, -3, 1),
// the guess is sum_j w_j p(t-j) + M^-1 (E0(t) - sum_j w_j E0(t-j)), the mutual
// part p - M^-1 E0 of the stored steps extrapolated to t (weights sum to 1).
// idx = axis * n + site.
__device__ __forceinline__ double hist_w(int k, int j) {
    return k == 1 ? 1.0 : (k == 2 ? (j == 1 ? 2.0 : -1.0) : (j == 2 ? -3.0 : (j == 1 ? 3.0 : 1.0)));
}
__device__ __forceinline__ double hist_base_p(const double *ph, int n, int cnt, int order, size_t idx) {
    const int k = min(order, cnt);
    double s = 0.0;
    for (int j = 1; j <= k; j++) s += hist_w(k, j) * ph[(size_t)((cnt - j) & 3) * 6 * n + idx];
    return s;
}
__device__ __forceinline__ double hist_diff_e(const double *ph, int n, int cnt, int order, size_t idx, double e0) {
    const int k = min(order, cnt);
    double s = e0;
    for (int j = 1; j <= k; j++) s -= hist_w(k, j) * ph[(size_t)((cnt - j) & 3) * 6 * n + 3 * (size_t)n + idx];
    return s;
}

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
// the same through integer atomics, for sites that several threads or
// kernels add to: the sum does not depend on the order
__device__ __forceinline__ void add_fix3_at(long long *arr, int n, int i, V3 v, double s) {
    atomicAdd((unsigned long long *)&arr[i], (unsigned long long)to_fix(s * v.x, FRC_SCALE));
    atomicAdd((unsigned long long *)&arr[n + i], (unsigned long long)to_fix(s * v.y, FRC_SCALE));
    atomicAdd((unsigned long long *)&arr[2 * n + i], (unsigned long long)to_fix(s * v.z, FRC_SCALE));
}

constexpr double SQRT_PI_POLAR = 1.7724538509055160273;

// ---------------------------------------------------------------------------
// pair invariants of the multipole-multipole interaction (r = r_i - r_j)
// ---------------------------------------------------------------------------
template <class R, class V>
struct MPPair {
    R G[5];
    V gG[5];   // gradients of G1..G4 (gG[0] unused)
};

// The invariants and torque coefficients are written once for the FP64 path
// (V3, Q6, double) and the mixed path's FP32 algebra (F3, Q6F, float).
template <class R, class V, class Q>
__device__ __forceinline__ void mp_invariants(R qi, V mi, const Q &Qi, R qj, V mj, const Q &Qj, V r,
                                              MPPair<R, V> &P) {
    const R QiI = qtr(Qi), QjI = qtr(Qj);
    const V Qir = qv(Qi, r), Qjr = qv(Qj, r);
    const R QiRij = dot(r, Qir), QjRij = dot(r, Qjr);
    const R mir = dot(mi, r), mjr = dot(mj, r);
    P.G[0] = qi * qj;
    P.G[1] = qj * mir - qi * mjr - dot(mi, mj) + qj * QiI + qi * QjI;
    P.G[2] = qj * QiRij + qi * QjRij - mir * mjr - mjr * QiI + mir * QjI - R(2) * dot(mj, Qir) +
             R(2) * dot(mi, Qjr) + QiI * QjI + R(2) * qdd(Qi, Qj);
    P.G[3] = mir * QjRij - mjr * QiRij + QiI * QjRij + QjI * QiRij + R(4) * dot(Qir, Qjr);
    P.G[4] = QiRij * QjRij;
    P.gG[1] = qj * mi - qi * mj;
    P.gG[2] = (R(2) * qj) * Qir - mjr * mi - mir * mj - R(2) * qv(Qi, mj) - QiI * mj + (R(2) * qi) * Qjr +
              R(2) * qv(Qj, mi) + QjI * mi;
    P.gG[3] = (-QiRij) * mj - (R(2) * mjr) * Qir + QjRij * mi + (R(2) * mir) * Qjr + (R(2) * QiI) * Qjr +
              (R(2) * QjI) * Qir + R(4) * qv(Qi, Qjr) + R(4) * qv(Qj, Qir);
    P.gG[4] = (R(2) * QjRij) * Qir + (R(2) * QiRij) * Qjr;
}

// torque coefficients on site i (Multipole.cpp real_term, Gt1i..Gt4i)
template <class R, class V, class Q>
__device__ __forceinline__ void mp_torque_i(R qj, V mi, const Q &Qi, V mj, const Q &Qj, V r, V Gt[5]) {
    const V Qir = qv(Qi, r), Qjr = qv(Qj, r);
    const R QjI = qtr(Qj), QjRij = dot(r, Qjr), mjr = dot(mj, r);
    const V rxmi = crs(r, mi);
    const V RxQi = crs(r, Qir);
    Gt[1] = qj * rxmi - crs(mj, mi);
    Gt[2] = (-mjr) * rxmi + R(2) * crs(Qjr, mi) + QjI * rxmi + (R(2) * qj) * RxQi -
            R(2) * crs(mj, Qir) - R(2) * crs(r, qv(Qi, mj)) + R(4) * qcross(Qj, Qi);
    Gt[3] = QjRij * rxmi - (R(2) * mjr) * RxQi + (R(2) * QjI) * RxQi + R(4) * crs(r, qv(Qi, Qjr)) +
            R(4) * crs(Qjr, Qir);
    Gt[4] = (R(2) * QjRij) * RxQi;
}

// B_n of erfc(a r)/r (Multipole.cpp:632-637); D_n of erf(a r)/r (:1495-1500)
__device__ __forceinline__ void bn_erfc(double r2, double alpha, double B[6]) {
    const double a2 = alpha * alpha, a2pi = 2.0 * alpha / SQRT_PI_POLAR;
    const double r = sqrt(r2), ex = exp(-a2 * r2), ir2 = 1.0 / r2;
    B[0] = erfc(alpha * r) / r;
    B[1] = (-B[0] - a2pi * ex) * ir2;
    B[2] = (-3 * B[1] + 2 * a2pi * a2 * ex) * ir2;
    B[3] = (-5 * B[2] - 4 * a2pi * a2 * a2 * ex) * ir2;
    B[4] = (-7 * B[3] + 8 * a2pi * a2 * a2 * a2 * ex) * ir2;
    B[5] = (-9 * B[4] - 16 * a2pi * a2 * a2 * a2 * a2 * ex) * ir2;
}
// the same B_n for a pass that also needs r and 1/r^2, from one reciprocal
// square root
__device__ __forceinline__ void bn_erfc_r(double r2, double alpha, double B[6], double &r, double &ir2) {
    const double a2 = alpha * alpha, a2pi = 2.0 * alpha / SQRT_PI_POLAR;
    const double ir = rsqrt(r2);
    r = r2 * ir;
    ir2 = ir * ir;
    const double ex = exp(-a2 * r2);
    B[0] = erfc(alpha * r) * ir;
    B[1] = (-B[0] - a2pi * ex) * ir2;
    B[2] = (-3 * B[1] + 2 * a2pi * a2 * ex) * ir2;
    B[3] = (-5 * B[2] - 4 * a2pi * a2 * a2 * ex) * ir2;
    B[4] = (-7 * B[3] + 8 * a2pi * a2 * a2 * a2 * ex) * ir2;
    B[5] = (-9 * B[4] - 16 * a2pi * a2 * a2 * a2 * a2 * ex) * ir2;
}
__device__ __forceinline__ void dn_erf(double r2, double alpha, double D[6]) {
    const double a2 = alpha * alpha, a2pi = 2.0 * alpha / SQRT_PI_POLAR;
    const double r = sqrt(r2), ex = exp(-a2 * r2);
    D[0] = erf(alpha * r) / r;
    D[1] = (-D[0] + a2pi * ex) / r2;
    D[2] = (-3 * D[1] - 2 * a2pi * a2 * ex) / r2;
    D[3] = (-5 * D[2] + 4 * a2pi * a2 * a2 * ex) / r2;
    D[4] = (-7 * D[3] - 8 * a2pi * a2 * a2 * a2 * ex) / r2;
    D[5] = (-9 * D[4] + 16 * a2pi * a2 * a2 * a2 * a2 * ex) / r2;
}

}  // namespace smd
