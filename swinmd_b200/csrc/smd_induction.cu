// Induced dipoles of the polarisable water model (Induction::compute /
// compute_long, src/forces/Induction.cpp).
//
//   k_ind_field   permanent field E0 at every site from the charges, dipoles
//                 and quadrupoles of all non-excluded sites within cutoffInd,
//                 Thole-damped (lambda3/5/7 with u = r^3/sqrt(a_i a_j))
//                 (Induction::InducedDipoles, :181-455)
//   k_ind_cg      the dipoles p solving A p = E0, A = diag(1/a_i) - T_ij
//                 (damped dipole tensor for every site pair within cutoffInd,
//                 intramolecular pairs included), matrix-free: the reference
//                 stores A densely (3N x 3N) and runs unpreconditioned CG
//                 (:2401-2467); here one persistent kernel runs Jacobi-
//                 preconditioned CG with the matrix applied on the fly from
//                 the Verlet list and the molecule's own sites, FP64 dot
//                 products in a fixed order, and stops on the RMS change of
//                 p (the dipole tolerance) or its iteration cap
//   k_ind_real    induced-permanent and induced-induced real-space energy,
//                 force and torque (:762-1355; Thole branch with the
//                 induced-induced force of the minimised dipoles)
//   k_ind_mol     self energy and torque (:688-759) and the intramolecular
//                 correction energy (:1760-2150; energy only under
//                 constraints)
// The reciprocal term is mp_recip<6> in smd_multipole.cu.
#include "smd_ctx.cuh"
#include "smd_polar.cuh"

namespace smd {

constexpr double COU = 138.93548501;
constexpr double SQC = 11.78708976;
constexpr double SQRT_PI_I = 1.7724538509055160273;

__device__ __forceinline__ V3 ld3i(const double *a, int n, int i) { return v3(a[i], a[n + i], a[2 * n + i]); }
__device__ __forceinline__ Q6 ldqi(const double *a, int n, int i) {
    return {a[i], a[n + i], a[2 * n + i], a[3 * n + i], a[4 * n + i], a[5 * n + i]};
}
__device__ __forceinline__ V3 mind(double4 pi, double4 pj, const Box &b) {
    return v3(pbc1(pi.x - pj.x, b.L[0], b.half[0]), pbc1(pi.y - pj.y, b.L[1], b.half[1]),
              pbc1(pi.z - pj.z, b.L[2], b.half[2]));
}
__device__ __forceinline__ bool is_excluded(int i, int j, const int *off, const int *ex) {
    for (int k = off[i]; k < off[i + 1]; k++)
        if (ex[k] == j) return true;
    return false;
}

struct IndArgs {
    int n, nmol;
    const int *nbr, *nnbr, *mol, *mol_off, *mol_atoms, *excl_off, *excl;
    const double4 *pos4;
    const double *tq, *polar, *mu, *qd;
    Box box;
    double cut2, a, alpha, rc2;
    double *e0, *p;
};

// ---------------------------------------------------------------------------
// permanent field
// ---------------------------------------------------------------------------
// field at i from site j, r = r_i - r_j (Induction.cpp:293-425)
__device__ __forceinline__ V3 perm_field(V3 r, double r2, double qj, V3 mj, const Q6 &Qj, double pi_,
                                         double pj_, double a) {
    const double rr = sqrt(r2);
    const double r_1 = 1.0 / rr, r_3 = r_1 * r_1 * r_1, r_5 = r_3 * r_1 * r_1, r_7 = r_5 * r_1 * r_1;
    const double u3 = r2 * rr / sqrt(pi_ * pj_);
    const double e = exp(-a * u3);
    const double l3 = 1.0 - e, l5 = 1.0 - (1.0 + a * u3) * e;
    const double l7 = 1.0 - (1.0 + a * u3 + 3.0 * a * a * u3 * u3 / 5.0) * e;
    const V3 Qjr = qv(Qj, r);
    const double QjRij = dot(r, Qjr), QjI = qtr(Qj);
    return (qj * l3 * r_3) * r + (3.0 * l5 * r_5 * dot(r, mj)) * r - (l3 * r_3) * mj +
           (15.0 * l7 * r_7 * QjRij) * r - (6.0 * l5 * r_5) * Qjr - (3.0 * l5 * r_5 * QjI) * r;
}

__global__ void k_ind_field(IndArgs a) {
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    constexpr int TPP = 8;
    const int i = gt / TPP, t = gt % TPP;
    V3 E = v3(0, 0, 0);
    if (i < a.n) {
        const double4 pi = a.pos4[i];
        const double poli = fmax(1e-8, a.polar[(int)pi.w]);
        const int cnt = a.nnbr[i];
        for (int k = t; k < cnt; k += TPP) {
            const int j = a.nbr[(size_t)k * a.n + i] & 0x7fffffff;
            const double4 pj = a.pos4[j];
            const V3 r = mind(pi, pj, a.box);
            const double rr = sqrt(dot(r, r)), r2 = rr * rr;
            if (!(r2 <= a.cut2)) continue;
            E = E + perm_field(r, r2, a.tq[(int)pj.w] / SQC, ld3i(a.mu, a.n, j), ldqi(a.qd, a.n, j), poli,
                               fmax(1e-8, a.polar[(int)pj.w]), a.a);
        }
    }
    E.x = group_sum<TPP>(E.x); E.y = group_sum<TPP>(E.y); E.z = group_sum<TPP>(E.z);
    if (i < a.n && t == 0) {
        a.e0[i] = E.x; a.e0[a.n + i] = E.y; a.e0[2 * a.n + i] = E.z;
    }
}

// ---------------------------------------------------------------------------
// matrix-free A v and the PCG solve
// ---------------------------------------------------------------------------
// (A v)_i = v_i / a_i - sum_j T_ij v_j, T_ij = l5 3 r r^T / r^5 - l3 / r^3
// over Verlet-list neighbours and the molecule's other sites within cutoffInd
__device__ __forceinline__ V3 tmul(V3 r, double r2, V3 v, double pi_, double pj_, double a) {
    const double rr = sqrt(r2);
    const double r_1 = 1.0 / rr, r_3 = r_1 * r_1 * r_1, r_5 = r_3 * r_1 * r_1;
    const double u3 = r2 * rr / sqrt(pi_ * pj_);
    const double e = exp(-a * u3);
    const double l3 = 1.0 - e, l5 = 1.0 - (1.0 + a * u3) * e;
    return (l5 * 3.0 * r_5 * dot(r, v)) * r - (l3 * r_3) * v;
}

// vectors written by other blocks of the persistent solver are read past L1
__device__ __forceinline__ V3 ld3cg(const double *a, int n, int i) {
    return v3(__ldcg(&a[i]), __ldcg(&a[n + i]), __ldcg(&a[2 * n + i]));
}

__device__ V3 apply_A(const IndArgs &a, int i, const double *v, int t, int tpp) {
    const double4 pi = a.pos4[i];
    const double poli = fmax(1e-8, a.polar[(int)pi.w]);
    V3 acc = v3(0, 0, 0);
    const int cnt = a.nnbr[i];
    for (int k = t; k < cnt; k += tpp) {
        const int j = a.nbr[(size_t)k * a.n + i] & 0x7fffffff;
        const double4 pj = a.pos4[j];
        const V3 r = mind(pi, pj, a.box);
        const double rr = sqrt(dot(r, r)), r2 = rr * rr;
        if (!(r2 <= a.cut2)) continue;
        acc = acc - tmul(r, r2, ld3cg(v, a.n, j), poli, fmax(1e-8, a.polar[(int)pj.w]), a.a);
    }
    if (t == 0) {
        // the molecule's excluded sites (not in the Verlet list, but in A)
        const int m = a.mol[i];
        for (int q = a.mol_off[m]; q < a.mol_off[m + 1]; q++) {
            const int j = a.mol_atoms[q];
            if (j == i || !is_excluded(i, j, a.excl_off, a.excl)) continue;
            const double4 pj = a.pos4[j];
            const V3 r = mind(pi, pj, a.box);
            const double rr = sqrt(dot(r, r)), r2 = rr * rr;
            if (!(r2 <= a.cut2)) continue;
            acc = acc - tmul(r, r2, ld3cg(v, a.n, j), poli, fmax(1e-8, a.polar[(int)pj.w]), a.a);
        }
        acc = acc + (1.0 / poli) * ld3cg(v, a.n, i);
    }
    return acc;
}

// Grid barrier with a bounded spin: every block of the (co-resident)
// cooperative launch arrives once per phase; a block that waits longer than
// the cap raises ST_CG_ITER and returns false, and the caller stops.
__device__ bool grid_barrier(unsigned int *bar, unsigned int target, unsigned int *status) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(bar, 1u);
        unsigned int spins = 0;
        while (atomicAdd(bar, 0u) < target) {
            __nanosleep(64);
            if (++spins > (1u << 24)) {  // ~1 s
                atomicOr(status, ST_CG_ITER);
                break;
            }
        }
        __threadfence();
    }
    __syncthreads();
    return (*(volatile unsigned int *)status & ST_CG_ITER) == 0;
}

struct CGArgs {
    IndArgs ia;
    double *r, *z, *v, *s;   // [3][N] each
    double *part;            // per block partials [nblocks][4]
    double *scal;            // [0] iterations, [1] final rms change, [2] initial guess mode
    unsigned int *bar, *status;
    int nblocks, max_iter, guess;
    double tol;
};

// fixed-order block sums, every block computes the same totals
__device__ void grid_sum(const double *part, int nblocks, int nq, double *out, double *s_tmp) {
    if (threadIdx.x < nq) {
        double t = 0;
        for (int b = 0; b < nblocks; b++) t += __ldcg(&part[b * 4 + threadIdx.x]);
        s_tmp[threadIdx.x] = t;
    }
    __syncthreads();
    for (int q = 0; q < nq; q++) out[q] = s_tmp[q];
    __syncthreads();
}

__device__ void block_partials(double *vals, int nq, double *part, double (*s_w)[4]) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int q = 0; q < nq; q++) {
        double t = warp_sum(vals[q]);
        if (lane == 0) s_w[w][q] = t;
    }
    __syncthreads();
    if (threadIdx.x < nq) {
        double t = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) t += s_w[q][threadIdx.x];
        part[blockIdx.x * 4 + threadIdx.x] = t;
    }
}

constexpr int CG_THREADS = 256;
constexpr int CG_TPP = 8;

__global__ void __launch_bounds__(CG_THREADS) k_ind_cg(CGArgs c) {
    __shared__ double s_w[CG_THREADS / 32][4];
    __shared__ double s_tmp[4];
    const IndArgs &a = c.ia;
    const int n = a.n;
    const int sites_per_pass = (c.nblocks * CG_THREADS) / CG_TPP;
    const int gslot = (blockIdx.x * CG_THREADS + threadIdx.x) / CG_TPP, t = threadIdx.x % CG_TPP;
    // every lane runs the same number of passes, so the group shuffles in
    // the matrix-vector products always see full warps
    const int passes = (n + sites_per_pass - 1) / sites_per_pass;
    unsigned int phase = 0;
    double tot[4];
    // p0: alpha E0 (guess 0) or the dipoles already in p (previous step / learned)
    double vals[4] = {0, 0, 0, 0};
    for (int i = gslot; i < n; i += sites_per_pass) {
        if (c.guess == 0 && t == 0) {
            const double pol = fmax(1e-8, a.polar[(int)a.pos4[i].w]);
            for (int d = 0; d < 3; d++) a.p[d * n + i] = pol * a.e0[d * n + i];
        }
    }
    if (!grid_barrier(c.bar, (++phase) * c.nblocks, c.status)) return;
    // r = E0 - A p ; s = M^-1 r ; v = s ; rs = r.s
    for (int ps = 0; ps < passes; ps++) {
        const int i = gslot + ps * sites_per_pass;
        V3 Ap = i < n ? apply_A(a, i, a.p, t, CG_TPP) : v3(0, 0, 0);
        Ap.x = group_sum<CG_TPP>(Ap.x); Ap.y = group_sum<CG_TPP>(Ap.y); Ap.z = group_sum<CG_TPP>(Ap.z);
        if (i < n && t == 0) {
            const double pol = fmax(1e-8, a.polar[(int)a.pos4[i].w]);
            const double rr[3] = {a.e0[i] - Ap.x, a.e0[n + i] - Ap.y, a.e0[2 * n + i] - Ap.z};
            for (int d = 0; d < 3; d++) {
                c.r[d * n + i] = rr[d];
                c.s[d * n + i] = pol * rr[d];
                c.v[d * n + i] = pol * rr[d];
                vals[0] += rr[d] * pol * rr[d];
            }
        }
    }
    block_partials(vals, 1, c.part, s_w);
    if (!grid_barrier(c.bar, (++phase) * c.nblocks, c.status)) return;
    grid_sum(c.part, c.nblocks, 1, tot, s_tmp);
    double rs = tot[0];
    int it = 0;
    double rms = 0;
    for (; it < c.max_iter; it++) {
        if (!(rs > 0)) break;
        // z = A v ; vz = v.z
        vals[0] = 0;
        for (int ps = 0; ps < passes; ps++) {
            const int i = gslot + ps * sites_per_pass;
            V3 Av = i < n ? apply_A(a, i, c.v, t, CG_TPP) : v3(0, 0, 0);
            Av.x = group_sum<CG_TPP>(Av.x); Av.y = group_sum<CG_TPP>(Av.y); Av.z = group_sum<CG_TPP>(Av.z);
            if (i < n && t == 0) {
                c.z[i] = Av.x; c.z[n + i] = Av.y; c.z[2 * n + i] = Av.z;
                vals[0] += c.v[i] * Av.x + c.v[n + i] * Av.y + c.v[2 * n + i] * Av.z;
            }
        }
        // the previous barrier reused the partials: wait before overwriting
        if (!grid_barrier(c.bar, (++phase) * c.nblocks, c.status)) return;
        block_partials(vals, 1, c.part, s_w);
        if (!grid_barrier(c.bar, (++phase) * c.nblocks, c.status)) return;
        grid_sum(c.part, c.nblocks, 1, tot, s_tmp);
        const double alpha_cg = rs / tot[0];
        // p += alpha v ; r -= alpha z ; s = M^-1 r ; rs' = r.s ; dp2 = |alpha v|^2
        vals[0] = 0; vals[1] = 0;
        for (int i = gslot; i < n; i += sites_per_pass) {
            if (t == 0) {
                const double pol = fmax(1e-8, a.polar[(int)a.pos4[i].w]);
                for (int d = 0; d < 3; d++) {
                    const int idx = d * n + i;
                    const double dp = alpha_cg * c.v[idx];
                    a.p[idx] += dp;
                    c.r[idx] -= alpha_cg * c.z[idx];
                    c.s[idx] = pol * c.r[idx];
                    vals[0] += c.r[idx] * c.s[idx];
                    vals[1] += dp * dp;
                }
            }
        }
        if (!grid_barrier(c.bar, (++phase) * c.nblocks, c.status)) return;
        block_partials(vals, 2, c.part, s_w);
        if (!grid_barrier(c.bar, (++phase) * c.nblocks, c.status)) return;
        grid_sum(c.part, c.nblocks, 2, tot, s_tmp);
        const double rs_new = tot[0];
        rms = sqrt(tot[1] / (3.0 * n));
        if (rms < c.tol) { it++; break; }
        const double beta = rs_new / rs;
        rs = rs_new;
        for (int i = gslot; i < n; i += sites_per_pass)
            if (t == 0)
                for (int d = 0; d < 3; d++) c.v[d * n + i] = c.s[d * n + i] + beta * c.v[d * n + i];
        if (!grid_barrier(c.bar, (++phase) * c.nblocks, c.status)) return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        c.scal[0] = it;
        c.scal[1] = rms;
        if (it >= c.max_iter) atomicOr(c.status, ST_CG_ITER);
    }
}

// ---------------------------------------------------------------------------
// induced-dipole real space (Thole-damped B_n, r = r_i - r_j)
// ---------------------------------------------------------------------------
struct IndPairOut {
    double e;   // Uen without COU and without the 1/2 of the pair double count
    V3 fij;     // force on i (without COU)
    V3 tau;     // torque on i (without COU)
};

__device__ __forceinline__ void ind_pair(double qi, V3 mi, const Q6 &Qi, V3 pi_, double qj, V3 mj,
                                         const Q6 &Qj, V3 pj_, V3 r, double r2, double poli,
                                         double polj, double a, double alpha, double scale,
                                         IndPairOut &o) {
    const V3 rji = -r;
    const double QiI = qtr(Qi), QjI = qtr(Qj);
    const V3 Qir = qv(Qi, r), Qjrji = qv(Qj, rji);
    const double QiRij = dot(r, Qir), QjRji = dot(r, qv(Qj, r));
    const double pjr = dot(pj_, r), pirji = dot(pi_, rji);
    const double G1i = -qi * pjr - dot(mi, pj_);
    const double G2i = -dot(mi, r) * pjr - 2.0 * dot(pj_, Qir) - pjr * QiI;
    const double G3i = -pjr * QiRij;
    const double G1j = -qj * pirji - dot(mj, pi_);
    const double G2j = -dot(mj, rji) * pirji - 2.0 * dot(pi_, Qjrji) - pirji * QjI;
    const double G3j = -pirji * QjRji;
    const V3 gG1i = -qi * pj_;
    const V3 gG2i = (-pjr) * mi - dot(mi, r) * pj_ - 2.0 * qv(Qi, pj_) - QiI * pj_;
    const V3 gG3i = (-QiRij) * pj_ - (2 * pjr) * Qir;
    const V3 gG1j = -qj * pi_;
    const V3 gG2j = (-pirji) * mj - dot(mj, rji) * pi_ - 2.0 * qv(Qj, pi_) - QjI * pi_;
    const V3 gG3j = (-QjRji) * pi_ - (2 * pirji) * Qjrji;
    const double rr = sqrt(r2);
    const double u3 = rr * rr * rr / sqrt(poli * polj);
    const double a2 = alpha * alpha, a2pi = 2.0 * alpha / SQRT_PI_I, ex = exp(-a2 * r2);
    double B[6];
    B[0] = erfc(alpha * rr) / rr;
    B[1] = (-B[0] - a2pi * ex) / r2;
    B[2] = (-3 * B[1] + 2 * a2pi * a2 * ex) / r2;
    B[3] = (-5 * B[2] - 4 * a2pi * a2 * a2 * ex) / r2;
    B[4] = (-7 * B[3] + 8 * a2pi * a2 * a2 * a2 * ex) / r2;
    const double e = exp(-a * u3), au3 = a * u3, a2u6 = au3 * au3, a3u9 = a2u6 * au3;
    const double l3 = 1.0 - e;
    const double gl3 = 3.0 * au3 * e / r2;
    const double gl5 = 3.0 * a2u6 * e / r2;
    const double gl7 = (-3.0 * a2u6 + 9.0 * a3u9) * e / (5.0 * r2);
    const double B1d = B[1] * l3;
    const double B2d = B[2] * l3 + B[1] * gl3;
    const double B3d = B[3] * l3 + B[2] * 2.0 * gl3 + B[1] * (gl3 - 3.0 * gl5) / r2;
    const double B4d = B[4] * l3 + B[3] * 3.0 * gl3 + B[2] * (3.0 * gl3 - 9.0 * gl5) / r2 +
                       B[1] * (-gl3 - 6.0 * gl5 + 15.0 * gl7) / (r2 * r2);
    o.e = 0.5 * ((G1i + G1j) * B1d + (G2i + G2j) * B2d + (G3i + G3j) * B3d) * scale;
    const double G1ip = -dot(pi_, pj_), G2ip = -dot(pi_, r) * pjr;
    const V3 gG2ip = (-pjr) * pi_, gG2jp = (-pirji) * pj_;
    const V3 fi = -(scale * (B1d * gG1i + B2d * gG2i + B3d * gG3i) + B2d * gG2ip) -
                  (scale * (G1i * B2d + G2i * B3d + G3i * B4d) + G1ip * B2d + G2ip * B3d) * r;
    const V3 fj = -(scale * (B1d * gG1j + B2d * gG2j + B3d * gG3j) + B2d * gG2jp) -
                  (scale * (G1j * B2d + G2j * B3d + G3j * B4d)) * rji;
    o.fij = fi - fj;
    // torque on i (Gt1i..Gt3i, Induction.cpp:1213-1230)
    const V3 Gt1 = crs(mi, pj_);
    const V3 Gt2 = pjr * crs(mi, r) + 2.0 * crs(Qir, pj_) + 2.0 * crs(qv(Qi, pj_), r);
    const V3 Gt3 = (2.0 * pjr) * crs(Qir, r);
    o.tau = scale * (B1d * Gt1 + B2d * Gt2 + B3d * Gt3);
}

struct IndRealArgs {
    IndArgs ia;
    long long *frc, *trq, *acc;
};

__global__ void __launch_bounds__(256) k_ind_real(IndRealArgs A) {
    const IndArgs &a = A.ia;
    constexpr int TPP = 8;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gt / TPP, t = gt % TPP;
    V3 f = v3(0, 0, 0), tau = v3(0, 0, 0);
    double en = 0, w[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (i < a.n) {
        const double4 pi = a.pos4[i];
        const double qi = a.tq[(int)pi.w] / SQC, poli = a.polar[(int)pi.w];
        const V3 mi = ld3i(a.mu, a.n, i), pii = ld3i(a.p, a.n, i);
        const Q6 Qi = ldqi(a.qd, a.n, i);
        auto pair = [&](int j, double scale) {
            const double4 pj = a.pos4[j];
            const V3 r = mind(pi, pj, a.box);
            const double r2 = dot(r, r);
            if (!(r2 < a.rc2)) return;
            IndPairOut o;
            ind_pair(qi, mi, Qi, pii, a.tq[(int)pj.w] / SQC, ld3i(a.mu, a.n, j), ldqi(a.qd, a.n, j),
                     ld3i(a.p, a.n, j), r, r2, poli, a.polar[(int)pj.w], a.a, a.alpha, scale, o);
            en += o.e;
            f = f + o.fij;
            tau = tau + o.tau;
            const double fr[3] = {o.fij.x, o.fij.y, o.fij.z}, rr[3] = {r.x, r.y, r.z};
            for (int p = 0; p < 3; p++)
                for (int q = 0; q < 3; q++) w[3 * p + q] -= 0.5 * fr[q] * rr[p];
        };
        // Verlet-list neighbours (never excluded) ...
        const int cnt = a.nnbr[i];
        for (int k = t; k < cnt; k += TPP) pair(a.nbr[(size_t)k * a.n + i] & 0x7fffffff, 1.0);
        // ... and the molecule's excluded sites, which the reference's all-pairs
        // loop also visits with the permanent-induced part scaled by 0
        if (t == 0) {
            const int m = a.mol[i];
            for (int q = a.mol_off[m]; q < a.mol_off[m + 1]; q++) {
                const int j = a.mol_atoms[q];
                if (j != i && is_excluded(i, j, a.excl_off, a.excl)) pair(j, 0.0);
            }
        }
    }
    f.x = group_sum<TPP>(f.x); f.y = group_sum<TPP>(f.y); f.z = group_sum<TPP>(f.z);
    tau.x = group_sum<TPP>(tau.x); tau.y = group_sum<TPP>(tau.y); tau.z = group_sum<TPP>(tau.z);
    if (i < a.n && t == 0) {
        add_fix3(A.frc, a.n, i, f, COU);
        add_fix3(A.trq, a.n, i, tau, COU);
    }
    __shared__ double s_r[8][10];
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    double vals[10] = {0.5 * en * COU, w[0], w[1], w[2], w[3], w[4], w[5], w[6], w[7], w[8]};
    for (int q = 0; q < 10; q++) {
        double s = warp_sum(vals[q]);
        if (lane == 0) s_r[wp][q] = s;
    }
    __syncthreads();
    if (threadIdx.x < 10) {
        double s = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) s += s_r[q][threadIdx.x];
        const int slot = threadIdx.x == 0 ? ACC_E_POL_REAL : ACC_VIR + threadIdx.x - 1;
        if (s != 0.0) atomicAdd((unsigned long long *)&A.acc[slot], (unsigned long long)to_fix(s, ACC_SCALE));
    }
}

// self energy + torque, intramolecular correction energy
__global__ void k_ind_mol(IndArgs a, long long *trq, long long *acc) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    double eself = 0, eintra = 0;
    if (m < a.nmol) {
        const double a2 = a.alpha * a.alpha, a2pi = 2.0 * a.alpha / SQRT_PI_I;
        const int s = a.mol_off[m], e = a.mol_off[m + 1];
        for (int p = s; p < e; p++) {
            const int i = a.mol_atoms[p];
            const double4 pi = a.pos4[i];
            const V3 mi = ld3i(a.mu, a.n, i), pii = ld3i(a.p, a.n, i);
            eself += -dot(mi, pii) * a2pi * a2 / 3 * COU;
            add_fix3(trq, a.n, i, crs(mi, pii), COU * (2.0 / 3.0) * a2pi * a2);
            const double qi = a.tq[(int)pi.w] / SQC;
            const Q6 Qi = ldqi(a.qd, a.n, i);
            for (int q = p + 1; q < e; q++) {
                const int j = a.mol_atoms[q];
                if (!is_excluded(i, j, a.excl_off, a.excl)) continue;
                const double4 pj = a.pos4[j];
                const V3 r = mind(pi, pj, a.box);
                const double r2 = dot(r, r), rr = sqrt(r2), ex = exp(-a2 * r2);
                const V3 rji = -r;
                const V3 mj = ld3i(a.mu, a.n, j), pjj = ld3i(a.p, a.n, j);
                const Q6 Qj = ldqi(a.qd, a.n, j);
                const double qj = a.tq[(int)pj.w] / SQC;
                const double pjr = dot(pjj, r), pirji = dot(pii, rji);
                const double G1i = -qi * pjr - dot(mi, pjj);
                const double G2i = -dot(mi, r) * pjr - 2.0 * dot(pjj, qv(Qi, r)) - pjr * qtr(Qi);
                const double G3i = -pjr * dot(r, qv(Qi, r));
                const double G1j = -qj * pirji - dot(mj, pii);
                const double G2j = -dot(mj, rji) * pirji - 2.0 * dot(pii, qv(Qj, rji)) - pirji * qtr(Qj);
                const double G3j = -pirji * dot(r, qv(Qj, r));
                const double D0 = erf(a.alpha * rr) / rr;
                const double D1 = (-D0 + a2pi * ex) / r2;
                const double D2 = (-3 * D1 - 2 * a2pi * a2 * ex) / r2;
                const double D3 = (-5 * D2 + 4 * a2pi * a2 * a2 * ex) / r2;
                eintra += (G1i + G1j) * D1 + (G2i + G2j) * D2 + (G3i + G3j) * D3;
            }
        }
    }
    __shared__ double s_r[2][4];
    double v0 = warp_sum(eself), v1 = warp_sum(-0.5 * eintra * COU);
    if ((threadIdx.x & 31) == 0) { s_r[0][threadIdx.x >> 5] = v0; s_r[1][threadIdx.x >> 5] = v1; }
    __syncthreads();
    if (threadIdx.x < 2) {
        double t = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) t += s_r[threadIdx.x][q];
        atomicAdd((unsigned long long *)&acc[threadIdx.x == 0 ? ACC_E_POL_SELF : ACC_E_POL_INTRA],
                  (unsigned long long)to_fix(t, ACC_SCALE));
    }
}

static IndArgs ind_args(Ctx &c) {
    IndArgs a;
    a.n = c.n; a.nmol = c.nmol; a.nbr = c.pl.nbr; a.nnbr = c.pl.nnbr; a.mol = c.mol;
    a.mol_off = c.mol_off; a.mol_atoms = c.mol_atoms; a.excl_off = c.excl_off; a.excl = c.excl;
    a.pos4 = c.pos4; a.tq = c.type_q; a.polar = c.type_polar; a.mu = c.mu; a.qd = c.qd;
    a.box = c.box; a.cut2 = c.ind_cut2; a.a = c.thole_a; a.alpha = c.ew_alpha; a.rc2 = c.mp_rc2;
    a.e0 = c.e0; a.p = c.pind;
    return a;
}

int setup_cg(Ctx &c) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ind_cg, CG_THREADS, 0) != cudaSuccess)
        return SMD_ERR_CUDA;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, c.device) != cudaSuccess) return SMD_ERR_CUDA;
    int want = (c.n * CG_TPP + CG_THREADS - 1) / CG_THREADS;
    int maxb = per_sm * prop.multiProcessorCount;
    c.cg_blocks = want < maxb ? want : maxb;
    if (c.cg_blocks < 1) c.cg_blocks = 1;
    return 0;
}

void launch_ind_solve(Ctx &c) {
    IndArgs a = ind_args(c);
    const int nb = (int)(((long long)c.n * 8 + 255) / 256);
    k_ind_field<<<nb, 256, 0, c.stream>>>(a);
    const bool learned = c.cg_guess == SMD_GUESS_LEARNED && c.mlp_ready;
    if (learned) launch_mlp_guess(c);  // writes the start dipoles into p
    CGArgs g;
    g.ia = a;
    g.r = c.cgw; g.z = c.cgw + 3 * (size_t)c.n; g.v = c.cgw + 6 * (size_t)c.n; g.s = c.cgw + 9 * (size_t)c.n;
    g.part = c.cgs + 8; g.scal = c.cgs; g.bar = c.cg_bar; g.status = c.status;
    g.nblocks = c.cg_blocks; g.max_iter = c.cg_max_iter; g.tol = c.cg_tol;
    // 0: start from alpha E0; 1: start from the dipoles in p (previous solve or network)
    g.guess = (c.cg_guess == SMD_GUESS_PREVIOUS || learned) ? 1 : 0;
    cudaMemsetAsync(c.cg_bar, 0, sizeof(unsigned int), c.stream);
    // cooperative launch: the runtime refuses it unless every block can be
    // resident at once, which the grid barrier relies on
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c.cg_blocks);
    cfg.blockDim = dim3(CG_THREADS);
    cfg.stream = c.stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_ind_cg, g);
}

void launch_ind_short(Ctx &c) {
    IndRealArgs A;
    A.ia = ind_args(c);
    A.frc = c.frc; A.trq = c.trq; A.acc = c.acc;
    const int nb = (int)(((long long)c.n * 8 + 255) / 256);
    k_ind_real<<<nb, 256, 0, c.stream>>>(A);
    k_ind_mol<<<(c.nmol + 127) / 128, 128, 0, c.stream>>>(A.ia, c.trq, c.acc);
}

}  // namespace smd
