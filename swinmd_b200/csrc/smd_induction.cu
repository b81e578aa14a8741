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
#include <algorithm>
#include <type_traits>
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
    int amoeba;   // induced real space damped as Tinker's AMOEBA (dampAMOEBA)
};

// ---------------------------------------------------------------------------
// permanent field
// ---------------------------------------------------------------------------
// field at i from site j, r = r_i - r_j (Induction.cpp:293-425); also
// returns the damped dipole-tensor coefficients of the pair,
// T = c5 r r^T - c3 I with c3 = l3/r^3, c5 = 3 l5/r^5
__device__ __forceinline__ V3 perm_field(V3 r, double r2, double qj, V3 mj, const Q6 &Qj, double pi_,
                                         double pj_, double a, double &c3, double &c5) {
    const double rr = sqrt(r2);
    const double r_1 = 1.0 / rr, r_3 = r_1 * r_1 * r_1, r_5 = r_3 * r_1 * r_1, r_7 = r_5 * r_1 * r_1;
    const double u3 = r2 * rr / sqrt(pi_ * pj_);
    const double e = exp(-a * u3);
    const double l3 = 1.0 - e, l5 = 1.0 - (1.0 + a * u3) * e;
    const double l7 = 1.0 - (1.0 + a * u3 + 3.0 * a * a * u3 * u3 / 5.0) * e;
    const V3 Qjr = qv(Qj, r);
    const double QjRij = dot(r, Qjr), QjI = qtr(Qj);
    c3 = l3 * r_3;
    c5 = 3.0 * l5 * r_5;
    return (qj * l3 * r_3) * r + (3.0 * l5 * r_5 * dot(r, mj)) * r - (l3 * r_3) * mj +
           (15.0 * l7 * r_7 * QjRij) * r - (6.0 * l5 * r_5) * Qjr - (3.0 * l5 * r_5 * QjI) * r;
}

// Rows of the damped tensor the dipole solve applies: for site i, slot s
// (s < cnt[i]) holds the partner j and (sqrt(c5) r, c3), so that
// T_ij v = (r'.v) r' - c3 v.  TS is the storage type: double in the FP64
// path, float in the mixed path.  Rows are site-major, so the lanes of one
// site read consecutive slots.
struct TRows {
    int *j;       // [N][cap]
    void *c;      // [N][cap] of TS4
    int *cnt;     // [N]
    int *lcnt;    // [N] slots taken by Verlet-list partners (the molecule's sites follow)
    int cap;
};

template <typename TS>
__device__ __forceinline__ void put_row(const TRows &R, int i, int s, int j, V3 r, double c3, double c5,
                                        unsigned int *status) {
    if (s >= R.cap) {
        atomicOr(status, ST_LIST_OVERFLOW);
        return;
    }
    const double sc = sqrt(c5);
    const size_t at = (size_t)i * R.cap + s;
    R.j[at] = j;
    using TS4 = typename std::conditional<sizeof(TS) == 4, float4, double4>::type;
    ((TS4 *)R.c)[at] = TS4{(TS)(sc * r.x), (TS)(sc * r.y), (TS)(sc * r.z), (TS)c3};
}

// Permanent field and tensor rows.  The pairs are those of the reference's
// A matrix within cutoffInd: Verlet-list neighbours (compacted in list order
// with a ballot per pass of the site's lanes) and then the molecule's
// excluded sites, which enter A but not the field.
template <typename TS>
__global__ void __launch_bounds__(256) k_ind_field(IndArgs a, TRows R, unsigned int *status) {
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    constexpr int TPP = 8;
    const int i = gt / TPP, t = gt % TPP;
    const int lane = threadIdx.x & 31, gbase = lane & ~(TPP - 1);
    V3 E = v3(0, 0, 0);
    const bool own = i < a.n;
    double4 pi = make_double4(0, 0, 0, 0);
    double poli = 1;
    int cnt = 0;
    if (own) {
        pi = a.pos4[i];
        poli = fmax(1e-8, a.polar[(int)pi.w]);
        cnt = a.nnbr[i];
    }
    const int wmax = __reduce_max_sync(0xffffffffu, cnt);
    int base = 0;
    for (int k0 = 0; k0 < wmax; k0 += TPP) {
        const int k = k0 + t;
        bool valid = false;
        int j = 0;
        V3 r = v3(0, 0, 0);
        double c3 = 0, c5 = 0;
        if (k < cnt) {
            j = a.nbr[(size_t)k * a.n + i] & 0x7fffffff;
            const double4 pj = a.pos4[j];
            r = mind(pi, pj, a.box);
            const double rr = sqrt(dot(r, r)), r2 = rr * rr;
            if (r2 <= a.cut2) {
                valid = true;
                E = E + perm_field(r, r2, a.tq[(int)pj.w] / SQC, ld3i(a.mu, a.n, j), ldqi(a.qd, a.n, j), poli,
                                   fmax(1e-8, a.polar[(int)pj.w]), a.a, c3, c5);
            }
        }
        const unsigned grp = (__ballot_sync(0xffffffffu, valid) >> gbase) & ((1u << TPP) - 1);
        if (valid) put_row<TS>(R, i, base + __popc(grp & ((1u << t) - 1)), j, r, c3, c5, status);
        base += __popc(grp);
    }
    E.x = group_sum<TPP>(E.x); E.y = group_sum<TPP>(E.y); E.z = group_sum<TPP>(E.z);
    if (own && t == 0) {
        a.e0[i] = E.x; a.e0[a.n + i] = E.y; a.e0[2 * a.n + i] = E.z;
        R.lcnt[i] = base < R.cap ? base : R.cap;
        const int m = a.mol[i];
        for (int q = a.mol_off[m]; q < a.mol_off[m + 1]; q++) {
            const int j = a.mol_atoms[q];
            if (j == i || !is_excluded(i, j, a.excl_off, a.excl)) continue;
            const double4 pj = a.pos4[j];
            const V3 r = mind(pi, pj, a.box);
            const double rr = sqrt(dot(r, r)), r2 = rr * rr;
            if (!(r2 <= a.cut2)) continue;
            const double ipp = 1.0 / sqrt(poli * fmax(1e-8, a.polar[(int)pj.w]));
            const double u3 = r2 * rr * ipp, e = exp(-a.a * u3);
            const double r_3 = 1.0 / (r2 * rr);
            put_row<TS>(R, i, base++, j, r, (1.0 - e) * r_3, 3.0 * (1.0 - (1.0 + a.a * u3) * e) * r_3 / r2, status);
        }
        R.cnt[i] = base < R.cap ? base : R.cap;
    }
}

// Mixed path: displacements from the box fractions (exact integer
// difference, r^2 from the 64-bit integer sum), the partner's multipoles
// from its FP32 site record.  The Thole-damped radial factors c3 = l3/r^3,
// c5 = 3 l5/r^5, c7 = 15 l7/r^7 and the charge term q_j c3 r are FP64; the
// dipole and quadrupole field
//   c5 (r.mu_j) r - c3 mu_j + c7 (r.Q_j.r) r - 2 c5 Q_j r - c5 tr(Q_j) r
// is FP32 algebra on FP32 copies of the factors, summed in FP64.  The rows
// and the molecule's excluded sites are as in k_ind_field<float>.
struct FieldMixArgs {
    const int4 *fixq;
    const float4 *srec;
    double dscale[3];
    int ntypes;
};

__global__ void __launch_bounds__(256) k_ind_field_f(IndArgs a, FieldMixArgs m, TRows R, unsigned int *status) {
    __shared__ double s_ipp[64];   // 1 / sqrt(a_i a_j) per type pair (ntypes <= 8)
    for (int q = threadIdx.x; q < m.ntypes * m.ntypes; q += blockDim.x)
        s_ipp[q] = 1.0 / sqrt(fmax(1e-8, a.polar[q / m.ntypes]) * fmax(1e-8, a.polar[q % m.ntypes]));
    __syncthreads();
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    constexpr int TPP = 8;
    const int i = gt / TPP, t = gt % TPP;
    const int lane = threadIdx.x & 31, gbase = lane & ~(TPP - 1);
    V3 E = v3(0, 0, 0);
    const bool own = i < a.n;
    int4 fi = make_int4(0, 0, 0, 0);
    int cnt = 0;
    if (own) {
        fi = m.fixq[i];
        cnt = a.nnbr[i];
    }
    const double s2u = m.dscale[0] * m.dscale[0];
    const int wmax = __reduce_max_sync(0xffffffffu, cnt);
    int base = 0;
    for (int k0 = 0; k0 < wmax; k0 += TPP) {
        const int k = k0 + t;
        bool valid = false;
        int j = 0;
        F3 rf = f3(0.f, 0.f, 0.f);
        float c3f = 0.f, c5f = 0.f;
        if (k < cnt) {
            j = a.nbr[(size_t)k * a.n + i] & 0x7fffffff;
            const int4 fj = m.fixq[j];
            const int ix = fi.x - fj.x, iy = fi.y - fj.y, iz = fi.z - fj.z;   // r = r_i - r_j
            const unsigned long long s2 = (unsigned long long)((long long)ix * ix) +
                                          (unsigned long long)((long long)iy * iy) +
                                          (unsigned long long)((long long)iz * iz);
            const double r2 = (double)s2 * s2u;
            if (r2 <= a.cut2) {
                valid = true;
                const V3 r = v3(ix * m.dscale[0], iy * m.dscale[1], iz * m.dscale[2]);
                rf = f3((float)r.x, (float)r.y, (float)r.z);
                const double r_1 = rsqrt(r2), rr = r2 * r_1, r_2 = r_1 * r_1, r_3 = r_1 * r_2;
                const double au3 = a.a * r2 * rr * s_ipp[fi.w * m.ntypes + fj.w];
                const double e = exp(-au3);
                const double l3 = 1.0 - e, l5 = 1.0 - (1.0 + au3) * e;
                const double l7 = 1.0 - (1.0 + au3 + 0.6 * au3 * au3) * e;
                const double c3 = l3 * r_3, c5 = 3.0 * l5 * r_3 * r_2, c7 = 15.0 * l7 * r_3 * r_2 * r_2;
                c3f = (float)c3;
                c5f = (float)c5;
                const float4 *rj = m.srec + 4 * (size_t)j;
                const float4 j0 = __ldg(rj), j1 = __ldg(rj + 1), j2 = __ldg(rj + 2);
                const F3 mj = f3(j0.y, j0.z, j0.w);
                const Q6F Qj = {j1.x, j1.y, j1.z, j1.w, j2.x, j2.y};
                const F3 Qjr = qv(Qj, rf);
                const float sc = c5f * (dot(rf, mj) - qtr(Qj)) + (float)c7 * dot(rf, Qjr);
                const F3 em = sc * rf - c3f * mj - (2.f * c5f) * Qjr;
                E = E + (a.tq[fj.w] / SQC * c3) * r + to_v3(em);
            }
        }
        const unsigned grp = (__ballot_sync(0xffffffffu, valid) >> gbase) & ((1u << TPP) - 1);
        if (valid && base + __popc(grp & ((1u << t) - 1)) < R.cap) {
            const size_t at = (size_t)i * R.cap + base + __popc(grp & ((1u << t) - 1));
            const float sc = sqrtf(c5f);
            R.j[at] = j;
            ((float4 *)R.c)[at] = make_float4(sc * rf.x, sc * rf.y, sc * rf.z, c3f);
        } else if (valid) {
            atomicOr(status, ST_LIST_OVERFLOW);
        }
        base += __popc(grp);
    }
    E.x = group_sum<TPP>(E.x); E.y = group_sum<TPP>(E.y); E.z = group_sum<TPP>(E.z);
    if (own && t == 0) {
        a.e0[i] = E.x; a.e0[a.n + i] = E.y; a.e0[2 * a.n + i] = E.z;
        R.lcnt[i] = base < R.cap ? base : R.cap;
        const double4 pi = a.pos4[i];
        const double poli = fmax(1e-8, a.polar[(int)pi.w]);
        const int mo = a.mol[i];
        for (int q = a.mol_off[mo]; q < a.mol_off[mo + 1]; q++) {
            const int j = a.mol_atoms[q];
            if (j == i || !is_excluded(i, j, a.excl_off, a.excl)) continue;
            const double4 pj = a.pos4[j];
            const V3 r = mind(pi, pj, a.box);
            const double rr = sqrt(dot(r, r)), r2 = rr * rr;
            if (!(r2 <= a.cut2)) continue;
            const double ipp = 1.0 / sqrt(poli * fmax(1e-8, a.polar[(int)pj.w]));
            const double u3 = r2 * rr * ipp, e = exp(-a.a * u3);
            const double r_3 = 1.0 / (r2 * rr);
            put_row<float>(R, i, base++, j, r, (1.0 - e) * r_3, 3.0 * (1.0 - (1.0 + a.a * u3) * e) * r_3 / r2, status);
        }
        R.cnt[i] = base < R.cap ? base : R.cap;
    }
}

// ---------------------------------------------------------------------------
// matrix-free A v and the PCG solve
// ---------------------------------------------------------------------------
// (A v)_i = v_i / a_i - sum_j T_ij v_j over the site's tensor row (the
// Verlet-list neighbours and the molecule's other sites within cutoffInd)

// Grid barrier with a bounded wait: every block of the (co-resident)
// cooperative launch arrives once per phase (release add on bar[0]), then
// polls the counter with acquire loads.  A block that has waited longer than
// limit_ns (device global timer) raises ST_WAIT_TIMEOUT, sets this launch's
// abort word bar[1] and returns false; blocks still waiting see the abort
// word and return false too, and every caller then leaves the kernel.  Both
// words are cleared before each launch, so an earlier launch's failure (or a
// solve that ran out of iterations) never cuts a later solve short.
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned int *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ bool grid_barrier(unsigned int *bar, unsigned int target, unsigned int *status,
                             unsigned long long limit_ns) {
    __shared__ int s_ok;   // thread 0's outcome: every thread of the block takes the same branch
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;" : : "l"(bar) : "memory");
        const unsigned long long t0 = global_ns();
        int ok = 1;
        while (ld_acquire_u32(bar) < target) {
            if (ld_acquire_u32(bar + 1) != 0) {   // another block gave up
                ok = 0;
                break;
            }
            __nanosleep(64);
            if (global_ns() - t0 > limit_ns) {
                atomicExch(bar + 1, 1u);
                atomicOr(status, ST_WAIT_TIMEOUT);
                ok = 0;
                break;
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

struct CGArgs {
    IndArgs ia;
    TRows rows;
    double *r, *z, *v, *al;  // [3][N] residual, w = A u, direction p; [N] polarisabilities
    double *s, *u;           // [3][N] s = A p, u = M^-1 r
    void *g0, *g1;           // per-site packed copies (float4 / double4) of the start dipoles and of v
    double *part;            // partials [4][nblocks][4]
    double *scal;            // [0] iterations, [1] final rms change
    unsigned *bar, *status;          // bar[0] barrier counter, bar[1] abort word
    unsigned long long wait_ns;      // limit of one barrier wait
    int skip_block;                  // failure-path test: this block never arrives (-1: none)
    int nblocks, max_iter, guess;
    double tol;
    const double *blk;       // [nmol][81] inverse molecule blocks of A (molecule preconditioner)
    float *srec;             // mixed path: site records (16 floats per site, p at 10..12), kept current
    double *w, *m, *q;       // [3][N] the pipelined form's w = A u, m = M^-1 w, q = M^-1 s
};

// fixed-order block sums, every block computes the same totals: each thread
// loads a strided share of the block partials (all loads in flight at once),
// then a fixed shuffle tree and a fixed pass over the warps
__device__ void grid_sum(const double *part, int nblocks, int nq, double *out, double (*s_w)[4]) {
    double v[4] = {0, 0, 0, 0};
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
        for (int q = 0; q < nq; q++) v[q] += __ldcg(&part[b * 4 + q]);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int q = 0; q < nq; q++) {
        const double t = warp_sum(v[q]);
        if (lane == 0) s_w[w][q] = t;
    }
    __syncthreads();
    for (int q = 0; q < nq; q++) {
        double t = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += s_w[k][q];
        out[q] = t;
    }
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

__device__ __forceinline__ double4 ldcg4(const double4 *p) {
    const double2 a = __ldcg((const double2 *)p), b = __ldcg((const double2 *)p + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float4 ldcg4(const float4 *p) { return __ldcg(p); }

// (A v)_i from the site's row: CG_TPP lanes take consecutive slots; the
// row entries are read in batches of CG_UNROLL per lane before the gathers
// of v, so each lane keeps several loads in flight.  In FP32 the next
// batch's row loads are issued before the current batch's products, so the
// row reads of one batch overlap the gathers of the previous one (in FP64
// the extra registers spill).  GR is the arithmetic type of the products
// (the row's storage type), summed per lane in GR.  The packed vector is
// rewritten every iteration, so it is gathered past L1 (tried through L1,
// relying on the barrier's acquire: slower).
template <typename G4, typename GR>
__device__ V3 amul(const CGArgs &c, int i, int t, const G4 *g) {
    constexpr int CG_UNROLL = sizeof(GR) == 4 ? 3 : 2;
    const TRows &R = c.rows;
    const int cnt = R.cnt[i];
    const int *rj = R.j + (size_t)i * R.cap;
    const G4 *rc = (const G4 *)R.c + (size_t)i * R.cap;
    GR ax = 0, ay = 0, az = 0;
    auto products = [&](const int (&jj)[CG_UNROLL], const G4 (&cc)[CG_UNROLL], const G4 (&vj)[CG_UNROLL]) {
#pragma unroll
        for (int u = 0; u < CG_UNROLL; u++)
            if (jj[u] >= 0) {
                const GR rv = cc[u].x * vj[u].x + cc[u].y * vj[u].y + cc[u].z * vj[u].z;
                ax += cc[u].w * vj[u].x - rv * cc[u].x;
                ay += cc[u].w * vj[u].y - rv * cc[u].y;
                az += cc[u].w * vj[u].z - rv * cc[u].z;
            }
    };
    auto rows = [&](int s0, int (&jj)[CG_UNROLL], G4 (&cc)[CG_UNROLL]) {
#pragma unroll
        for (int u = 0; u < CG_UNROLL; u++) {
            const int s = s0 + u * CG_TPP;
            jj[u] = s < cnt ? rj[s] : -1;
            if (s < cnt) cc[u] = rc[s];
        }
    };
    auto gathers = [&](const int (&jj)[CG_UNROLL], G4 (&vj)[CG_UNROLL]) {
#pragma unroll
        for (int u = 0; u < CG_UNROLL; u++)
            if (jj[u] >= 0) vj[u] = ldcg4(&g[jj[u]]);
    };
    if constexpr (sizeof(GR) == 4) {
        int jj[CG_UNROLL];
        G4 cc[CG_UNROLL];
        rows(t, jj, cc);
        for (int s0 = t; s0 < cnt; s0 += CG_UNROLL * CG_TPP) {
            G4 vj[CG_UNROLL];
            gathers(jj, vj);
            int jn[CG_UNROLL];
            G4 cn[CG_UNROLL];
            rows(s0 + CG_UNROLL * CG_TPP, jn, cn);
            products(jj, cc, vj);
#pragma unroll
            for (int u = 0; u < CG_UNROLL; u++) {
                jj[u] = jn[u];
                cc[u] = cn[u];
            }
        }
    } else {
        for (int s0 = t; s0 < cnt; s0 += CG_UNROLL * CG_TPP) {
            int jj[CG_UNROLL];
            G4 cc[CG_UNROLL], vj[CG_UNROLL];
            rows(s0, jj, cc);
            gathers(jj, vj);
            products(jj, cc, vj);
        }
    }
    V3 acc = v3(ax, ay, az);
    if (t == 0) {
        const G4 vi = ldcg4(&g[i]);
        acc = acc + (1.0 / __ldcg(&c.al[i])) * v3(vi.x, vi.y, vi.z);
    }
    return acc;
}

// Molecule-block preconditioner: for every molecule (at most 3 sites) the
// block of A = diag(1/a_i) - T over its own sites, with T_ij from the
// excluded-site entries of the tensor rows (T v = (r'.v) r' - c3 v), is
// inverted in FP64.  It captures the strong Thole-damped coupling inside a
// water molecule that the diagonal preconditioner leaves out.  Nine threads
// per molecule, each holding one row of its 9 x 9 block in registers
// (unused sites padded with the identity), MB_MOLS molecules per block, and
// an in-place Gauss-Jordan sweep over the nine pivots (no pivoting: the
// block is positive definite): the pivot row, scaled by the reciprocal of
// the pivot, goes through shared memory to the other eight rows.  A block
// with a non-positive pivot falls back to diag(a_i).  The inverses are
// stored entry-major over molecules (entry e of molecule m at e * nmol + m),
// so that the solve's loads of one entry coalesce.
constexpr int MB_MOLS = 32;
// With dl given, the same threads also form the blocks' response to the
// permanent field's difference of the extrapolated guess of the given order,
// dl = M_m^-1 (E0(t) - sum_j w_j E0(t-j)) (M_m^-1 E0 when no step is stored;
// as k_blk_response does from the stored blocks).
template <typename TS>
__global__ void __launch_bounds__(9 * MB_MOLS) k_mol_blocks(int n, int nmol, const int *mol_off, const int *mol_atoms,
                                                            TRows R, const double *polar, const double4 *pos4,
                                                            double *blk, const double *e0, const double *ph,
                                                            const int *flags, double *dl, int order,
                                                            double *dlp) {
    using TS4 = typename std::conditional<sizeof(TS) == 4, float4, double4>::type;
    __shared__ double s_piv[MB_MOLS][9];
    __shared__ int s_bad[MB_MOLS];
    const int lm = threadIdx.x / 9, r = threadIdx.x - 9 * lm, q = r / 3, x = r - 3 * q;
    const int m = blockIdx.x * MB_MOLS + lm;
    const bool act = m < nmol;
    if (r == 0) s_bad[lm] = 0;
    // row r = 3 q + x: site q, axis x; columns 3 qq + y
    // (all indices into row[] are compile-time, so that it stays in registers)
    double row[9];
    int ns = 0;
    double al = 1.0, diag = 1.0;
    int js[3] = {-1, -1, -1};
    int i = -1;
    if (act) {
        const int s0 = mol_off[m];
        ns = min(3, mol_off[m + 1] - s0);
#pragma unroll
        for (int qq = 0; qq < 3; qq++)
            if (qq < ns) js[qq] = mol_atoms[s0 + qq];
        if (q < ns) {
            i = q == 0 ? js[0] : (q == 1 ? js[1] : js[2]);
            al = fmax(1e-8, polar[(int)pos4[i].w]);
            diag = 1.0 / al;
        }
    }
#pragma unroll
    for (int c = 0; c < 9; c++) row[c] = c == r ? diag : 0.0;
    if (i >= 0) {
        const int c1 = min(R.cnt[i], R.cap);
        for (int k = R.lcnt[i]; k < c1; k++) {
            const int j = R.j[(size_t)i * R.cap + k];
#pragma unroll
            for (int qq = 0; qq < 3; qq++)
                if (qq != q && j == js[qq]) {
                    const TS4 t = ((const TS4 *)R.c)[(size_t)i * R.cap + k];
                    const double v0 = (double)t.x, v1 = (double)t.y, v2 = (double)t.z, w = (double)t.w;
                    const double vx = x == 0 ? v0 : (x == 1 ? v1 : v2);
                    row[3 * qq] = -(vx * v0 - (x == 0 ? w : 0.0));
                    row[3 * qq + 1] = -(vx * v1 - (x == 1 ? w : 0.0));
                    row[3 * qq + 2] = -(vx * v2 - (x == 2 ? w : 0.0));
                }
        }
    }
#pragma unroll
    for (int k = 0; k < 9; k++) {
        __syncthreads();   // the previous pivot row has been read by every row
        if (r == k) {
            const double p = row[k];
            if (!(p > 0.0)) {
                s_bad[lm] = 1;
            } else {
                const double ip = 1.0 / p;
#pragma unroll
                for (int c = 0; c < 9; c++) row[c] = c == k ? ip : row[c] * ip;
            }
#pragma unroll
            for (int c = 0; c < 9; c++) s_piv[lm][c] = row[c];
        }
        __syncthreads();
        if (r != k) {
            const double f = row[k];
            const double ip = s_piv[lm][k];
#pragma unroll
            for (int c = 0; c < 9; c++) row[c] = c == k ? -f * ip : fma(-f, s_piv[lm][c], row[c]);
        }
    }
    __syncthreads();
    const int nd = 3 * ns;
    const bool bad = act && s_bad[lm] != 0;
#pragma unroll
    for (int c = 0; c < 9; c++) {
        if (bad) row[c] = (r == c && r < nd) ? al : 0.0;
        if (r >= nd || c >= nd) row[c] = 0.0;
    }
    if (act) {
#pragma unroll
        for (int c = 0; c < 9; c++) blk[(size_t)(r * 9 + c) * nmol + m] = row[c];
    }
    if (dl) {
        __shared__ double s_de[MB_MOLS][9];
        const int cnt = flags[2];
        double de = 0.0;
        if (i >= 0) {
            const size_t idx = (size_t)x * n + i;
            de = hist_diff_e(ph, n, cnt, order, idx, e0[idx]);
        }
        s_de[lm][r] = de;
        __syncthreads();
        if (i >= 0) {
            double u = 0.0;
#pragma unroll
            for (int c = 0; c < 9; c++) u += row[c] * s_de[lm][c];
            dl[(size_t)x * n + i] = u;
        }
        if (dlp) {   // the last step's response, M_m^-1 (E0(t-1) - E0(t-2))
            __syncthreads();
            double dp = 0.0;
            if (i >= 0 && cnt >= 2) {
                const size_t idx = (size_t)x * n + i;
                dp = ph[(size_t)((cnt - 1) & 3) * 6 * n + 3 * (size_t)n + idx] -
                     ph[(size_t)((cnt - 2) & 3) * 6 * n + 3 * (size_t)n + idx];
            }
            s_de[lm][r] = dp;
            __syncthreads();
            if (i >= 0) {
                double u = 0.0;
#pragma unroll
                for (int c = 0; c < 9; c++) u += row[c] * s_de[lm][c];
                dlp[(size_t)x * n + i] = u;
            }
        }
    }
}

// u = B_m^-1 v for every molecule, nine threads per molecule (thread e of a
// molecule owns component e = 3 q + d, site q, axis d) in tiles of
// at most CG_THREADS / 9 molecules, spread over the whole grid; the
// components meet in shared memory.
// in(m, e, i, idx) gives (and may update) component e of v, out(...) takes
// u's component; the packed copy pk of u (one G4 per site) is written here.
// Block-uniform loop: every thread of the block reaches each barrier.
template <typename G4, typename GR, class FIn, class FOut>
__device__ __forceinline__ void mol_tiles(const IndArgs &a, const double *blk, G4 *pk, double *s_v, double *s_u,
                                          FIn &&in, FOut &&out) {
    const int n = a.n, nmol = a.nmol;
    // molecules per tile: spread over every block of the grid
    const int TM = max(1, min(CG_THREADS / 9, (nmol + (int)gridDim.x - 1) / (int)gridDim.x));
    const int ml = threadIdx.x / 9, e = threadIdx.x - 9 * ml, q = e / 3, d = e - 3 * q;
    for (int m0 = blockIdx.x * TM; m0 < nmol; m0 += gridDim.x * TM) {
        const int m = m0 + ml;
        int ns = 0, i = -1;
        if (ml < TM && m < nmol) {
            const int s0 = a.mol_off[m];
            ns = min(3, a.mol_off[m + 1] - s0);
            if (q < ns) i = a.mol_atoms[s0 + q];
        }
        double v = 0.0;
        if (i >= 0) v = in(m, e, i, d * n + i);
        if (ml < TM) s_v[threadIdx.x] = v;
        __syncthreads();
        double u = 0.0;
        if (i >= 0) {
            for (int col = 0; col < 3 * ns; col++) u += __ldcg(&blk[(size_t)(e * 9 + col) * nmol + m]) * s_v[9 * ml + col];
            out(m, e, i, d * n + i, v, u);
        }
        if (ml < TM) s_u[threadIdx.x] = u;
        __syncthreads();
        if (i >= 0 && d == 0)
            pk[i] = G4{(GR)s_u[threadIdx.x], (GR)s_u[threadIdx.x + 1], (GR)s_u[threadIdx.x + 2], (GR)0};
        __syncthreads();
    }
}

// Preconditioned CG as one persistent cooperative kernel, M^-1 = diag(a_i)
// (BJ false) or the inverse molecule blocks of k_mol_blocks (BJ true: the
// start x0 = M^-1 E0 and u = M^-1 r are formed per molecule, which costs one
// more grid barrier before the first product), in the single-reduction form
// of Chronopoulos and Gear (1989): with
// u = M^-1 r and w = A u kept alongside, the direction p = u + beta p and
// s = A p = w + beta s follow by recurrence, and both inner products of an
// iteration, gamma = r.u and delta = w.u, come from one pass each side of
// the matrix-vector product.  Two grid barriers per iteration:
//   U  p = u + beta p, s = w + beta s, x += alpha p, r -= alpha s,
//      u = M^-1 r (and its packed copy); r.u, |alpha p|^2   | barrier, stop
//                                                           |  on the RMS
//                                                           |  change of x
//   W  w = A u (TPP lanes per site); w.u                    | barrier
//   beta = gamma'/gamma, alpha = gamma' / (delta' - beta gamma'/alpha)
// (alpha and beta are those of standard PCG in exact arithmetic).  The
// partial sums of U and W alternate between two buffers each by iteration
// parity, so no barrier is needed to guard their reuse.  Vectors written in
// one phase and read by other blocks in the next are read past L1.
template <bool F32, bool BJ>
__global__ void __launch_bounds__(CG_THREADS, 3) k_ind_cg(CGArgs c) {
    using G4 = typename std::conditional<F32, float4, double4>::type;
    using GR = typename std::conditional<F32, float, double>::type;
    __shared__ double s_w[CG_THREADS / 32][4];
    __shared__ double s_bv[BJ ? CG_THREADS : 1], s_bu[BJ ? CG_THREADS : 1];
    const IndArgs &a = c.ia;
    const int n = a.n;
    G4 *g0 = (G4 *)c.g0, *g1 = (G4 *)c.g1;
    double *const pu0 = c.part, *const pu1 = c.part + 4 * c.nblocks;
    double *const pw0 = c.part + 8 * c.nblocks, *const pw1 = c.part + 12 * c.nblocks;
    const int nthreads = c.nblocks * CG_THREADS;
    const int gtid = blockIdx.x * CG_THREADS + threadIdx.x;
    const int sites_per_pass = nthreads / CG_TPP;
    const int gslot = gtid / CG_TPP, t = threadIdx.x % CG_TPP;
    // every lane runs the same number of passes, so the group shuffles in
    // the matrix-vector products always see full warps
    const int passes = (n + sites_per_pass - 1) / sites_per_pass;
    unsigned int phase = 0;
    double tot[4];
    // failure-path test hook: this block leaves before its first arrival, so
    // the other blocks' first barrier wait runs out (nothing else is skipped:
    // it has written nothing yet)
    if ((int)blockIdx.x == c.skip_block) return;
    // every write of a dipole component also goes to the site records, so
    // that they hold the solution when the solve ends
    auto put_p = [&](int i, int d, double v) {
        a.p[d * n + i] = v;
        if (c.srec) c.srec[16 * (size_t)i + 10 + d] = (float)v;
    };
    // x0: M^-1 E0 (guess 0) or the dipoles already in p (previous step / learned)
    if (BJ) {
        for (int i = gtid; i < n; i += nthreads) c.al[i] = fmax(1e-8, a.polar[(int)a.pos4[i].w]);
        if (c.guess == 0) {
            mol_tiles<G4, GR>(a, c.blk, g0, s_bv, s_bu, [&](int, int, int, int idx) { return a.e0[idx]; },
                              [&](int, int e, int i, int, double, double u) { put_p(i, e % 3, u); });
        } else {
            for (int i = gtid; i < n; i += nthreads) {
                const double p0 = a.p[i], p1 = a.p[n + i], p2 = a.p[2 * n + i];
                g0[i] = G4{(GR)p0, (GR)p1, (GR)p2, (GR)0};
                put_p(i, 0, p0); put_p(i, 1, p1); put_p(i, 2, p2);
            }
        }
    } else {
        for (int i = gtid; i < n; i += nthreads) {
            const double al = fmax(1e-8, a.polar[(int)a.pos4[i].w]);
            c.al[i] = al;
            double p3[3];
            for (int d = 0; d < 3; d++) {
                p3[d] = c.guess == 0 ? al * a.e0[d * n + i] : a.p[d * n + i];
                put_p(i, d, p3[d]);
            }
            g0[i] = G4{(GR)p3[0], (GR)p3[1], (GR)p3[2], (GR)0};
        }
    }
    if (!grid_barrier(c.bar, (++phase) * c.nblocks, c.status, c.wait_ns)) return;
    // r = E0 - A x ; u = M^-1 r ; gamma = r.u
    double vals[4] = {0, 0, 0, 0};
    for (int ps = 0; ps < passes; ps++) {
        const int i = gslot + ps * sites_per_pass;
        V3 Ap = i < n ? amul<G4, GR>(c, i, t, g0) : v3(0, 0, 0);
        Ap.x = group_sum<CG_TPP>(Ap.x); Ap.y = group_sum<CG_TPP>(Ap.y); Ap.z = group_sum<CG_TPP>(Ap.z);
        if (i < n && t == 0) {
            const double al = __ldcg(&c.al[i]);
            const double rr[3] = {a.e0[i] - Ap.x, a.e0[n + i] - Ap.y, a.e0[2 * n + i] - Ap.z};
            for (int d = 0; d < 3; d++) c.r[d * n + i] = rr[d];
            if (!BJ) {
                for (int d = 0; d < 3; d++) {
                    c.u[d * n + i] = al * rr[d];
                    vals[0] += rr[d] * al * rr[d];
                }
                g1[i] = G4{(GR)(al * rr[0]), (GR)(al * rr[1]), (GR)(al * rr[2]), (GR)0};
            }
        }
    }
    if (BJ) {
        // u = B^-1 r per molecule, once every site's residual is in place
        if (!grid_barrier(c.bar, (++phase) * c.nblocks, c.status, c.wait_ns)) return;
        mol_tiles<G4, GR>(a, c.blk, g1, s_bv, s_bu, [&](int, int, int, int idx) { return __ldcg(&c.r[idx]); },
                          [&](int, int, int, int idx, double r, double u) {
                              c.u[idx] = u;
                              vals[0] += r * u;
                          });
    }
    block_partials(vals, 1, pu1, s_w);
    if (!grid_barrier(c.bar, (++phase) * c.nblocks, c.status, c.wait_ns)) return;
    // w = A u ; delta = w.u
    vals[0] = 0;
    for (int ps = 0; ps < passes; ps++) {
        const int i = gslot + ps * sites_per_pass;
        V3 Au = i < n ? amul<G4, GR>(c, i, t, g1) : v3(0, 0, 0);
        Au.x = group_sum<CG_TPP>(Au.x); Au.y = group_sum<CG_TPP>(Au.y); Au.z = group_sum<CG_TPP>(Au.z);
        if (i < n && t == 0) {
            c.z[i] = Au.x; c.z[n + i] = Au.y; c.z[2 * n + i] = Au.z;
            vals[0] += __ldcg(&c.u[i]) * Au.x + __ldcg(&c.u[n + i]) * Au.y + __ldcg(&c.u[2 * n + i]) * Au.z;
        }
    }
    block_partials(vals, 1, pw1, s_w);
    if (!grid_barrier(c.bar, (++phase) * c.nblocks, c.status, c.wait_ns)) return;
    grid_sum(pu1, c.nblocks, 1, tot, s_w);
    double gamma = tot[0];
    grid_sum(pw1, c.nblocks, 1, tot, s_w);
    double alpha_cg = gamma / tot[0], beta = 0.0;
    int it = 0;
    double rms = 0;
    bool conv = false;   // the RMS change fell below the tolerance (or r = 0 exactly)
    for (; it < c.max_iter; it++) {
        if (!(gamma > 0)) {   // r.u = 0: the start already solves A p = E0
            conv = gamma == 0.0;
            break;
        }
        if (!(alpha_cg > 0)) break;   // breakdown (A not positive definite or non-finite)
        // U: p = u + beta p ; s = w + beta s ; x += alpha p ; r -= alpha s ;
        //    u = M^-1 r ; gamma' = r.u ; |alpha p|^2
        vals[0] = 0; vals[1] = 0;
        if (BJ) {
            mol_tiles<G4, GR>(a, c.blk, g1, s_bv, s_bu,
                              [&](int, int e, int i, int idx) {
                                  const double pd = __ldcg(&c.u[idx]) + (it ? beta * __ldcg(&c.v[idx]) : 0.0);
                                  const double sd = __ldcg(&c.z[idx]) + (it ? beta * __ldcg(&c.s[idx]) : 0.0);
                                  c.v[idx] = pd;
                                  c.s[idx] = sd;
                                  const double dp = alpha_cg * pd;
                                  put_p(i, e % 3, __ldcg(&a.p[idx]) + dp);
                                  const double r = __ldcg(&c.r[idx]) - alpha_cg * sd;
                                  c.r[idx] = r;
                                  vals[1] += dp * dp;
                                  return r;
                              },
                              [&](int, int, int, int idx, double r, double u) {
                                  c.u[idx] = u;
                                  vals[0] += r * u;
                              });
        } else {
            for (int i = gtid; i < n; i += nthreads) {
                const double al = __ldcg(&c.al[i]);
                double w3[3];
                for (int d = 0; d < 3; d++) {
                    const int idx = d * n + i;
                    const double pd = __ldcg(&c.u[idx]) + (it ? beta * __ldcg(&c.v[idx]) : 0.0);
                    const double sd = __ldcg(&c.z[idx]) + (it ? beta * __ldcg(&c.s[idx]) : 0.0);
                    c.v[idx] = pd;
                    c.s[idx] = sd;
                    const double dp = alpha_cg * pd;
                    put_p(i, d, __ldcg(&a.p[idx]) + dp);
                    const double r = __ldcg(&c.r[idx]) - alpha_cg * sd;
                    c.r[idx] = r;
                    w3[d] = al * r;
                    c.u[idx] = w3[d];
                    vals[0] += r * w3[d];
                    vals[1] += dp * dp;
                }
                g1[i] = G4{(GR)w3[0], (GR)w3[1], (GR)w3[2], (GR)0};
            }
        }
        double *const pu = (it & 1) ? pu1 : pu0;
        block_partials(vals, 2, pu, s_w);
        if (!grid_barrier(c.bar, (++phase) * c.nblocks, c.status, c.wait_ns)) return;
        grid_sum(pu, c.nblocks, 2, tot, s_w);
        const double gamma_new = tot[0];
        rms = sqrt(tot[1] / (3.0 * n));
        if (blockIdx.x == 0 && threadIdx.x == 0 && it < CG_TRACE) c.scal[CG_SCAL + it] = rms;
        if (rms < c.tol) {
            conv = true;
            it++;
            break;
        }
        // W: w = A u ; delta' = w.u
        vals[0] = 0;
        for (int ps = 0; ps < passes; ps++) {
            const int i = gslot + ps * sites_per_pass;
            V3 Au = i < n ? amul<G4, GR>(c, i, t, g1) : v3(0, 0, 0);
            Au.x = group_sum<CG_TPP>(Au.x); Au.y = group_sum<CG_TPP>(Au.y); Au.z = group_sum<CG_TPP>(Au.z);
            if (i < n && t == 0) {
                c.z[i] = Au.x; c.z[n + i] = Au.y; c.z[2 * n + i] = Au.z;
                vals[0] += __ldcg(&c.u[i]) * Au.x + __ldcg(&c.u[n + i]) * Au.y + __ldcg(&c.u[2 * n + i]) * Au.z;
            }
        }
        double *const pw = (it & 1) ? pw1 : pw0;
        block_partials(vals, 1, pw, s_w);
        if (!grid_barrier(c.bar, (++phase) * c.nblocks, c.status, c.wait_ns)) return;
        grid_sum(pw, c.nblocks, 1, tot, s_w);
        const double delta = tot[0];
        beta = gamma_new / gamma;
        alpha_cg = gamma_new / (delta - beta * gamma_new / alpha_cg);
        gamma = gamma_new;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        c.scal[0] = it;
        c.scal[1] = rms;
        if (!conv) atomicOr(c.status, ST_CG_ITER);
    }
}

// ---------------------------------------------------------------------------
// Pipelined preconditioned CG: one grid barrier per iteration
// ---------------------------------------------------------------------------
// The solve with the molecule blocks (either precision), in the pipelined form of
// Ghysels and Vanroose (2014, Parallel Computing 40: 224-238): with
// m = M^-1 w and n = A m carried along, the recurrences
//   z = n + beta z, q = m + beta q, s = w + beta s, p = u + beta p,
//   x += alpha p,  r -= alpha s,  u -= alpha q,  w -= alpha z
// keep u = M^-1 r and w = A u without a second product.  Both inner
// products of the next iteration (gamma = r.u, delta = w.u) and the RMS
// change come out of the pass that also forms the next m = M^-1 w, so one
// grid barrier per iteration remains instead of two; alpha and beta are
// those of standard PCG in exact arithmetic, and the solve stops on the
// same RMS change.  Each block owns whole molecules (PP_MOLS per pass; the
// sites of molecule k are 3k .. 3k + 2), so applying the molecule blocks
// needs only its own sites and a block barrier.  Start: x0 (M^-1 E0 or the
// dipoles given), r0 = E0 - A x0, u0 = M^-1 r0, w0 = A u0, m0 = M^-1 w0,
// with three grid barriers.  The packed FP32 copies the products gather
// alternate between g0 and g1, and the partial sums between two buffers, by
// iteration parity.
constexpr int PP_MOLS = 8, PP_SITES = 3 * PP_MOLS, PP_THREADS = PP_SITES * CG_TPP;   // 192 threads
constexpr double PP_MIN_TOL = 1e-9;   // e nm: below it the single-reduction form runs

template <bool F32>
__global__ void __launch_bounds__(PP_THREADS, 4) k_ind_pcg_pipe(CGArgs c) {
    using G4 = typename std::conditional<F32, float4, double4>::type;
    using GR = typename std::conditional<F32, float, double>::type;
    __shared__ double s_w[PP_THREADS / 32][4];
    __shared__ double s_in[3 * PP_SITES], s_out[3 * PP_SITES];
    const IndArgs &a = c.ia;
    const int n = a.n, nmol = a.nmol;
    G4 *const gb[2] = {(G4 *)c.g0, (G4 *)c.g1};
    double *const pa[2] = {c.part, c.part + 4 * c.nblocks};
    // lane group sl of CG_TPP lanes per site; lanes d < 3 of a group own the
    // site's component d in the vector updates
    const int sl = threadIdx.x / CG_TPP, t = threadIdx.x - CG_TPP * sl, d = t;
    const int groups = (nmol + PP_MOLS - 1) / PP_MOLS;
    const int passes = (groups + (int)gridDim.x - 1) / (int)gridDim.x;
    unsigned int phase = 0;
    // failure-path test hook, as in k_ind_cg
    if ((int)blockIdx.x == c.skip_block) return;
    auto put_p = [&](int i, int dd, double v) {
        a.p[dd * n + i] = v;
        if (c.srec) c.srec[16 * (size_t)i + 10 + dd] = (float)v;
    };
    // this lane group's site in pass ps, or -1
    auto site_of = [&](int ps) {
        const int gi = blockIdx.x + ps * (int)gridDim.x;
        const int i = gi * PP_SITES + sl;
        return (gi < groups && i < n) ? i : -1;
    };
    // s_out = M^-1 s_in for the pass's molecules (s_in[3 sl + d] written by
    // the component lanes; the inverse blocks are stored entry-major); then
    // the site's packed copy for the products' gathers
    auto precond = [&](int ps, int i, G4 *pk) {
        __syncthreads();
        if (threadIdx.x < 9 * PP_MOLS) {
            const int ml = threadIdx.x / 9, e = threadIdx.x - 9 * ml;
            const int mo = (blockIdx.x + ps * (int)gridDim.x) * PP_MOLS + ml;
            double u = 0.0;
            if (mo < nmol)
                for (int col = 0; col < 9; col++) u += __ldcg(&c.blk[(size_t)(e * 9 + col) * nmol + mo]) * s_in[9 * ml + col];
            s_out[threadIdx.x] = u;
        }
        __syncthreads();
        if (t == 0 && i >= 0)
            pk[i] = G4{(GR)s_out[3 * sl], (GR)s_out[3 * sl + 1], (GR)s_out[3 * sl + 2], (GR)0};
    };
    auto matvec = [&](int i, const G4 *g) {
        V3 v = i >= 0 ? amul<G4, GR>(c, i, t, g) : v3(0, 0, 0);
        v.x = group_sum<CG_TPP>(v.x); v.y = group_sum<CG_TPP>(v.y); v.z = group_sum<CG_TPP>(v.z);
        return d == 0 ? v.x : (d == 1 ? v.y : v.z);   // the lane's component (every lane holds the sum)
    };
    // x0
    for (int ps = 0; ps < passes; ps++) {
        const int i = site_of(ps);
        if (t == 0 && i >= 0) c.al[i] = fmax(1e-8, a.polar[(int)a.pos4[i].w]);
        if (c.guess == 0) {
            if (d < 3) s_in[3 * sl + d] = i >= 0 ? a.e0[d * n + i] : 0.0;
            precond(ps, i, gb[0]);
            if (d < 3 && i >= 0) put_p(i, d, s_out[3 * sl + d]);
        } else {
            if (d < 3 && i >= 0) put_p(i, d, a.p[d * n + i]);
            if (t == 0 && i >= 0)
                gb[0][i] = G4{(GR)a.p[i], (GR)a.p[n + i], (GR)a.p[2 * n + i], (GR)0};
        }
    }
    if (!grid_barrier(c.bar, (++phase) * c.nblocks, c.status, c.wait_ns)) return;
    // r0 = E0 - A x0 ; u0 = M^-1 r0
    for (int ps = 0; ps < passes; ps++) {
        const int i = site_of(ps);
        const double ax = matvec(i, gb[0]);
        if (d < 3) {
            const double r = i >= 0 ? a.e0[d * n + i] - ax : 0.0;
            if (i >= 0) c.r[d * n + i] = r;
            s_in[3 * sl + d] = r;
        }
        precond(ps, i, gb[1]);
        if (d < 3 && i >= 0) c.u[d * n + i] = s_out[3 * sl + d];
    }
    if (!grid_barrier(c.bar, (++phase) * c.nblocks, c.status, c.wait_ns)) return;
    // w0 = A u0 ; m0 = M^-1 w0 ; gamma = r0.u0, delta = w0.u0
    double vals[4] = {0, 0, 0, 0};
    for (int ps = 0; ps < passes; ps++) {
        const int i = site_of(ps);
        const double au = matvec(i, gb[1]);
        if (d < 3) {
            if (i >= 0) {
                const int idx = d * n + i;
                c.w[idx] = au;
                const double u = c.u[idx];
                vals[0] += c.r[idx] * u;
                vals[1] += au * u;
            }
            s_in[3 * sl + d] = i >= 0 ? au : 0.0;
        }
        precond(ps, i, gb[0]);
        if (d < 3 && i >= 0) c.m[d * n + i] = s_out[3 * sl + d];
    }
    block_partials(vals, 2, pa[0], s_w);
    if (!grid_barrier(c.bar, (++phase) * c.nblocks, c.status, c.wait_ns)) return;
    double tot[4];
    grid_sum(pa[0], c.nblocks, 2, tot, s_w);
    double gamma = tot[0], alpha_cg = tot[0] / tot[1], beta = 0.0;
    int it = 0, cur = 0;   // gb[cur] holds the m the next product gathers
    double rms = 0;
    bool conv = false;
    for (; it < c.max_iter; it++) {
        if (!(gamma > 0)) {   // r.u = 0: the start already solves A p = E0
            conv = gamma == 0.0;
            break;
        }
        if (!(alpha_cg > 0)) break;   // breakdown (A not positive definite or non-finite)
        vals[0] = 0; vals[1] = 0; vals[2] = 0;
        for (int ps = 0; ps < passes; ps++) {
            const int i = site_of(ps);
            const double nv = matvec(i, gb[cur]);
            if (d < 3) {
                double wn = 0.0;
                if (i >= 0) {
                    const int idx = d * n + i;
                    const double zv = nv + (it ? beta * c.z[idx] : 0.0);
                    const double qv = c.m[idx] + (it ? beta * c.q[idx] : 0.0);
                    const double sv = c.w[idx] + (it ? beta * c.s[idx] : 0.0);
                    const double pv = c.u[idx] + (it ? beta * c.v[idx] : 0.0);
                    c.z[idx] = zv; c.q[idx] = qv; c.s[idx] = sv; c.v[idx] = pv;
                    const double dp = alpha_cg * pv;
                    put_p(i, d, a.p[idx] + dp);
                    const double rn = c.r[idx] - alpha_cg * sv;
                    const double un = c.u[idx] - alpha_cg * qv;
                    wn = c.w[idx] - alpha_cg * zv;
                    c.r[idx] = rn; c.u[idx] = un; c.w[idx] = wn;
                    vals[0] += rn * un;
                    vals[1] += wn * un;
                    vals[2] += dp * dp;
                }
                s_in[3 * sl + d] = wn;
            }
            precond(ps, i, gb[cur ^ 1]);
            if (d < 3 && i >= 0) c.m[d * n + i] = s_out[3 * sl + d];
        }
        double *const pp = pa[(it + 1) & 1];
        block_partials(vals, 3, pp, s_w);
        if (!grid_barrier(c.bar, (++phase) * c.nblocks, c.status, c.wait_ns)) return;
        grid_sum(pp, c.nblocks, 3, tot, s_w);
        rms = sqrt(tot[2] / (3.0 * n));
        if (blockIdx.x == 0 && threadIdx.x == 0 && it < CG_TRACE) c.scal[CG_SCAL + it] = rms;
        if (rms < c.tol) {
            conv = true;
            it++;
            break;
        }
        const double gamma_new = tot[0], delta = tot[1];
        beta = gamma_new / gamma;
        alpha_cg = gamma_new / (delta - beta * gamma_new / alpha_cg);
        gamma = gamma_new;
        cur ^= 1;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        c.scal[0] = it;
        c.scal[1] = rms;
        if (!conv) atomicOr(c.status, ST_CG_ITER);
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
    const double ir2 = 1.0 / r2;
    B[1] = (-B[0] - a2pi * ex) * ir2;
    B[2] = (-3 * B[1] + 2 * a2pi * a2 * ex) * ir2;
    B[3] = (-5 * B[2] - 4 * a2pi * a2 * a2 * ex) * ir2;
    B[4] = (-7 * B[3] + 8 * a2pi * a2 * a2 * a2 * ex) * ir2;
    const double e = exp(-a * u3), au3 = a * u3, a2u6 = au3 * au3, a3u9 = a2u6 * au3;
    const double l3 = 1.0 - e;
    const double gl3 = 3.0 * au3 * e * ir2;
    const double gl5 = 3.0 * a2u6 * e * ir2;
    const double gl7 = (-3.0 * a2u6 + 9.0 * a3u9) * e * (0.2 * ir2);
    const double B1d = B[1] * l3;
    const double B2d = B[2] * l3 + B[1] * gl3;
    const double B3d = B[3] * l3 + B[2] * 2.0 * gl3 + B[1] * (gl3 - 3.0 * gl5) * ir2;
    const double B4d = B[4] * l3 + B[3] * 3.0 * gl3 + B[2] * (3.0 * gl3 - 9.0 * gl5) * ir2 +
                       B[1] * (-gl3 - 6.0 * gl5 + 15.0 * gl7) * (ir2 * ir2);
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

// The dampAMOEBA branch (Induction.cpp:1051-1079, Tinker's form; the
// minimisation terms G1ip, G2ip with the undamped-by-exclusion factors):
//   B1d = B1 + (1 - s l3)/r^3, B2d = B2 - 3 (1 - s l5)/r^5, B3d = B3 + 15 (1 - s l7)/r^7
// and their radial gradients gB1..gB3 in place of B2d..B4d.  The exclusion
// scale s sits inside the factors, so excluded pairs contribute.
struct IndRadA {
    double c1, c2, c3;    // B1d, B2d, B3d
    double g1, g2, g3;    // gradB1, gradB2, gradB3
    double cp, gp1, gp2;  // B2du, gradB1u, gradB2u (s = 1)
};

__device__ __forceinline__ void ind_radial_amoeba(double rr, double ir2, const double *B, double ipp, double a,
                                                  double s, IndRadA &R) {
    const double au3 = a * rr * rr * rr * ipp, e = exp(-au3), a2u6 = au3 * au3, a3u9 = a2u6 * au3;
    const double l3 = 1.0 - e, l5 = 1.0 - (1.0 + au3) * e, l7 = 1.0 - (1.0 + au3 + 0.6 * a2u6) * e;
    const double gl3 = 3.0 * au3 * e * ir2, gl5 = 3.0 * a2u6 * e * ir2;
    const double gl7 = (-3.0 * a2u6 + 9.0 * a3u9) * e * (0.2 * ir2);
    const double ir3 = ir2 / rr, ir5 = 3.0 * ir3 * ir2, ir7 = 5.0 * ir5 * ir2, ir9 = 7.0 * ir7 * ir2;
    R.c1 = B[1] + (1.0 - s * l3) * ir3;
    R.c2 = B[2] - (1.0 - s * l5) * ir5;
    R.c3 = B[3] + (1.0 - s * l7) * ir7;
    R.g1 = B[2] - s * gl3 * ir3 - (1.0 - s * l3) * ir5;
    R.g2 = B[3] + s * gl5 * ir5 + (1.0 - s * l5) * ir7;
    R.g3 = B[4] - s * gl7 * ir7 - (1.0 - s * l7) * ir9;
    R.cp = B[2] - (1.0 - l5) * ir5;
    R.gp1 = B[2] - gl3 * ir3 - (1.0 - l3) * ir5;
    R.gp2 = B[3] + gl5 * ir5 + (1.0 - l5) * ir7;
}

__device__ __forceinline__ V3 as_v3(V3 v) { return v; }
__device__ __forceinline__ V3 as_v3(F3 v) { return to_v3(v); }

// energy, force and torque of the pair from its angular algebra (FP64 or
// FP32 members) and the AMOEBA radial factors
template <class AL>
__device__ __forceinline__ void ind_pair_amoeba(const AL &A, V3 r, const IndRadA &R, IndPairOut &o) {
    o.e = 0.5 * (((double)A.G1i + A.G1j) * R.c1 + ((double)A.G2i + A.G2j) * R.c2 + ((double)A.G3i + A.G3j) * R.c3);
    const V3 fi = -(R.c1 * as_v3(A.gG1i) + R.c2 * as_v3(A.gG2i) + R.c3 * as_v3(A.gG3i) + R.cp * as_v3(A.gG2ip)) -
                  (A.G1i * R.g1 + A.G2i * R.g2 + A.G3i * R.g3 + A.G1ip * R.gp1 + A.G2ip * R.gp2) * r;
    const V3 fj = -(R.c1 * as_v3(A.gG1j) + R.c2 * as_v3(A.gG2j) + R.c3 * as_v3(A.gG3j) + R.cp * as_v3(A.gG2jp)) -
                  (A.G1j * R.g1 + A.G2j * R.g2 + A.G3j * R.g3) * (-r);
    o.fij = fi - fj;
    o.tau = R.c1 * as_v3(A.Gt1) + R.c2 * as_v3(A.Gt2) + R.c3 * as_v3(A.Gt3);
}

// the angular algebra of the pair in FP64 (members as IndAlgF's)
struct IndAlgD {
    double G1i, G2i, G3i, G1j, G2j, G3j, G1ip, G2ip;
    V3 gG1i, gG2i, gG3i, gG1j, gG2j, gG3j, gG2ip, gG2jp, Gt1, Gt2, Gt3;
};

__device__ __forceinline__ void ind_algebra_d(double qi, V3 mi, const Q6 &Qi, V3 pi_, double qj, V3 mj,
                                              const Q6 &Qj, V3 pj_, V3 r, IndAlgD &A) {
    const V3 rji = -r;
    const double QiI = qtr(Qi), QjI = qtr(Qj);
    const V3 Qir = qv(Qi, r), Qjrji = qv(Qj, rji);
    const double QiRij = dot(r, Qir), QjRji = dot(r, qv(Qj, r));
    const double pjr = dot(pj_, r), pirji = dot(pi_, rji);
    A.G1i = -qi * pjr - dot(mi, pj_);
    A.G2i = -dot(mi, r) * pjr - 2.0 * dot(pj_, Qir) - pjr * QiI;
    A.G3i = -pjr * QiRij;
    A.G1j = -qj * pirji - dot(mj, pi_);
    A.G2j = -dot(mj, rji) * pirji - 2.0 * dot(pi_, Qjrji) - pirji * QjI;
    A.G3j = -pirji * QjRji;
    A.gG1i = (-qi) * pj_;
    A.gG2i = (-pjr) * mi - dot(mi, r) * pj_ - 2.0 * qv(Qi, pj_) - QiI * pj_;
    A.gG3i = (-QiRij) * pj_ - (2.0 * pjr) * Qir;
    A.gG1j = (-qj) * pi_;
    A.gG2j = (-pirji) * mj - dot(mj, rji) * pi_ - 2.0 * qv(Qj, pi_) - QjI * pi_;
    A.gG3j = (-QjRji) * pi_ - (2.0 * pirji) * Qjrji;
    A.G1ip = -dot(pi_, pj_);
    A.G2ip = -dot(pi_, r) * pjr;
    A.gG2ip = (-pjr) * pi_;
    A.gG2jp = (-pirji) * pj_;
    A.Gt1 = crs(mi, pj_);
    A.Gt2 = pjr * crs(mi, r) + 2.0 * crs(Qir, pj_) + 2.0 * crs(qv(Qi, pj_), r);
    A.Gt3 = (2.0 * pjr) * crs(Qir, r);
}

// Mixed path: the same terms with the angular algebra (G, their gradients
// and the torque coefficients) in FP32 and the radial Ewald / Thole factors,
// the energy and the force assembly in FP64.
struct IndAlgF {
    float G1i, G2i, G3i, G1j, G2j, G3j, G1ip, G2ip;
    F3 gG1i, gG2i, gG3i, gG1j, gG2j, gG3j, gG2ip, gG2jp, Gt1, Gt2, Gt3;
};

__device__ __forceinline__ void ind_algebra_f(float qi, F3 mi, const Q6F &Qi, F3 pi_, float qj, F3 mj,
                                              const Q6F &Qj, F3 pj_, F3 r, IndAlgF &A) {
    const F3 rji = -r;
    const float QiI = qtr(Qi), QjI = qtr(Qj);
    const F3 Qir = qv(Qi, r), Qjrji = qv(Qj, rji);
    const float QiRij = dot(r, Qir), QjRji = dot(r, qv(Qj, r));
    const float pjr = dot(pj_, r), pirji = dot(pi_, rji);
    A.G1i = -qi * pjr - dot(mi, pj_);
    A.G2i = -dot(mi, r) * pjr - 2.f * dot(pj_, Qir) - pjr * QiI;
    A.G3i = -pjr * QiRij;
    A.G1j = -qj * pirji - dot(mj, pi_);
    A.G2j = -dot(mj, rji) * pirji - 2.f * dot(pi_, Qjrji) - pirji * QjI;
    A.G3j = -pirji * QjRji;
    A.gG1i = (-qi) * pj_;
    A.gG2i = (-pjr) * mi - dot(mi, r) * pj_ - 2.f * qv(Qi, pj_) - QiI * pj_;
    A.gG3i = (-QiRij) * pj_ - (2.f * pjr) * Qir;
    A.gG1j = (-qj) * pi_;
    A.gG2j = (-pirji) * mj - dot(mj, rji) * pi_ - 2.f * qv(Qj, pi_) - QjI * pi_;
    A.gG3j = (-QjRji) * pi_ - (2.f * pirji) * Qjrji;
    A.G1ip = -dot(pi_, pj_);
    A.G2ip = -dot(pi_, r) * pjr;
    A.gG2ip = (-pjr) * pi_;
    A.gG2jp = (-pirji) * pj_;
    A.Gt1 = crs(mi, pj_);
    A.Gt2 = pjr * crs(mi, r) + 2.f * crs(Qir, pj_) + 2.f * crs(qv(Qi, pj_), r);
    A.Gt3 = (2.f * pjr) * crs(Qir, r);
}

// the radial part given the Ewald B_0..B_4 of the pair (bn_erfc), |r|,
// 1/r^2 and ipp = 1/sqrt(a_i a_j)
__device__ __forceinline__ void ind_pair_mixed_b(const IndAlgF &A, V3 r, double rr, double ir2, const double *B,
                                                 double ipp, double a, double scale, IndPairOut &o) {
    const double u3 = rr * rr * rr * ipp;
    const double e = exp(-a * u3), au3 = a * u3, a2u6 = au3 * au3, a3u9 = a2u6 * au3;
    const double l3 = 1.0 - e;
    const double gl3 = 3.0 * au3 * e * ir2;
    const double gl5 = 3.0 * a2u6 * e * ir2;
    const double gl7 = (-3.0 * a2u6 + 9.0 * a3u9) * e * (0.2 * ir2);
    const double B1d = B[1] * l3;
    const double B2d = B[2] * l3 + B[1] * gl3;
    const double B3d = B[3] * l3 + B[2] * 2.0 * gl3 + B[1] * (gl3 - 3.0 * gl5) * ir2;
    const double B4d = B[4] * l3 + B[3] * 3.0 * gl3 + B[2] * (3.0 * gl3 - 9.0 * gl5) * ir2 +
                       B[1] * (-gl3 - 6.0 * gl5 + 15.0 * gl7) * (ir2 * ir2);
    o.e = 0.5 * (((double)A.G1i + A.G1j) * B1d + ((double)A.G2i + A.G2j) * B2d + ((double)A.G3i + A.G3j) * B3d) *
          scale;
    const V3 fi = -(scale * (B1d * to_v3(A.gG1i) + B2d * to_v3(A.gG2i) + B3d * to_v3(A.gG3i)) +
                    B2d * to_v3(A.gG2ip)) -
                  (scale * (A.G1i * B2d + A.G2i * B3d + A.G3i * B4d) + A.G1ip * B2d + A.G2ip * B3d) * r;
    const V3 fj = -(scale * (B1d * to_v3(A.gG1j) + B2d * to_v3(A.gG2j) + B3d * to_v3(A.gG3j)) +
                    B2d * to_v3(A.gG2jp)) -
                  (scale * (A.G1j * B2d + A.G2j * B3d + A.G3j * B4d)) * (-r);
    o.fij = fi - fj;
    o.tau = scale * (B1d * to_v3(A.Gt1) + B2d * to_v3(A.Gt2) + B3d * to_v3(A.Gt3));
}

__device__ __forceinline__ void ind_pair_mixed(const IndAlgF &A, V3 r, double r2, double poli, double polj,
                                               double a, double alpha, double scale, IndPairOut &o) {
    double B[6];
    bn_erfc(r2, alpha, B);
    ind_pair_mixed_b(A, r, sqrt(r2), 1.0 / r2, B, 1.0 / sqrt(poli * polj), a, scale, o);
}

struct IndRealArgs {
    IndArgs ia;
    long long *frc, *trq, *acc;
    const int4 *fixq;      // mixed path: box fractions
    const float4 *srec;    // mixed path: FP32 site records (q, mu, Q, p)
    double dscale[3];      // L / 2^32 per axis
    const int *rj, *rcnt, *rlcnt;   // the solve's tensor rows (partners within cutoffInd)
    int rcap;
    int ntypes;
};

__global__ void __launch_bounds__(64) k_ind_real(IndRealArgs A) {
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
            if (a.amoeba) {
                IndAlgD al;
                ind_algebra_d(qi, mi, Qi, pii, a.tq[(int)pj.w] / SQC, ld3i(a.mu, a.n, j), ldqi(a.qd, a.n, j),
                              ld3i(a.p, a.n, j), r, al);
                double B[6];
                bn_erfc(r2, a.alpha, B);
                IndRadA R;
                ind_radial_amoeba(sqrt(r2), 1.0 / r2, B, 1.0 / sqrt(poli * a.polar[(int)pj.w]), a.a, scale, R);
                ind_pair_amoeba(al, r, R, o);
            } else {
                ind_pair(qi, mi, Qi, pii, a.tq[(int)pj.w] / SQC, ld3i(a.mu, a.n, j), ldqi(a.qd, a.n, j),
                         ld3i(a.p, a.n, j), r, r2, poli, a.polar[(int)pj.w], a.a, a.alpha, scale, o);
            }
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

// Mixed-path induced real space: displacements from the box fractions (the
// exact integer difference, r^2 from the 64-bit integer sum), FP32 algebra,
// FP64 radial factors and accumulation (cubic boxes)
__global__ void __launch_bounds__(64) k_ind_real_f(IndRealArgs A) {
    const IndArgs &a = A.ia;
    constexpr int TPP = 8;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gt / TPP, t = gt % TPP;
    V3 f = v3(0, 0, 0), tau = v3(0, 0, 0);
    double en = 0, w[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (i < a.n) {
        const int4 fi = A.fixq[i];
        const double poli = a.polar[fi.w];
        const float4 *ri = A.srec + 4 * (size_t)i;
        const float4 i0 = ri[0], i1 = ri[1], i2 = ri[2], i3 = ri[3];
        const float qi = i0.x;
        const F3 mi = f3(i0.y, i0.z, i0.w);
        const F3 pii = f3(i2.z, i2.w, i3.x);
        const Q6F Qi = {i1.x, i1.y, i1.z, i1.w, i2.x, i2.y};
        const double s2u = A.dscale[0] * A.dscale[0];
        auto pair = [&](int j, double scale) {
            const int4 fj = A.fixq[j];
            const int ix = fi.x - fj.x, iy = fi.y - fj.y, iz = fi.z - fj.z;   // r = r_i - r_j
            const unsigned long long s2 = (unsigned long long)((long long)ix * ix) +
                                          (unsigned long long)((long long)iy * iy) +
                                          (unsigned long long)((long long)iz * iz);
            const double r2 = (double)s2 * s2u;
            if (!(r2 < a.rc2)) return;
            const V3 r = v3(ix * A.dscale[0], iy * A.dscale[1], iz * A.dscale[2]);
            const F3 rf = f3((float)r.x, (float)r.y, (float)r.z);
            const float4 *rj = A.srec + 4 * (size_t)j;
            const float4 j0 = __ldg(rj), j1 = __ldg(rj + 1), j2 = __ldg(rj + 2), j3 = __ldg(rj + 3);
            const Q6F Qj = {j1.x, j1.y, j1.z, j1.w, j2.x, j2.y};
            IndAlgF al;
            ind_algebra_f(qi, mi, Qi, pii, j0.x, f3(j0.y, j0.z, j0.w), Qj, f3(j2.z, j2.w, j3.x), rf, al);
            IndPairOut o;
            if (a.amoeba) {
                double B[6];
                bn_erfc(r2, a.alpha, B);
                IndRadA R;
                ind_radial_amoeba(sqrt(r2), 1.0 / r2, B, 1.0 / sqrt(poli * a.polar[fj.w]), a.a, scale, R);
                ind_pair_amoeba(al, r, R, o);
            } else {
                ind_pair_mixed(al, r, r2, poli, a.polar[fj.w], a.a, a.alpha, scale, o);
            }
            en += o.e;
            f = f + o.fij;
            tau = tau + o.tau;
            const double fr[3] = {o.fij.x, o.fij.y, o.fij.z}, rr[3] = {r.x, r.y, r.z};
            for (int p = 0; p < 3; p++)
                for (int q = 0; q < 3; q++) w[3 * p + q] -= 0.5 * fr[q] * rr[p];
        };
        const int cnt = a.nnbr[i];
        for (int k = t; k < cnt; k += TPP) pair(a.nbr[(size_t)k * a.n + i] & 0x7fffffff, 1.0);
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
        double sv = warp_sum(vals[q]);
        if (lane == 0) s_r[wp][q] = sv;
    }
    __syncthreads();
    if (threadIdx.x < 10) {
        double sv = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) sv += s_r[q][threadIdx.x];
        const int slot = threadIdx.x == 0 ? ACC_E_POL_REAL : ACC_VIR + threadIdx.x - 1;
        if (sv != 0.0) atomicAdd((unsigned long long *)&A.acc[slot], (unsigned long long)to_fix(sv, ACC_SCALE));
    }
}

// Mixed path, one pass for both real-space polarisable terms after the
// dipole solve: the multipole real-space term of k_mp_real_f and the induced
// term of k_ind_real_f share the pair loop, the partner's site record and
// the Ewald B_n of the pair.  Energies go to their own slots; forces,
// torques and virial are summed.  ROWS: the partners come from the solve's
// tensor rows (the Verlet-list partners within cutoffInd, compacted, then the
// molecule's excluded sites), which hold every pair inside the real-space
// cutoff when cutoffInd is at least that cutoff, so that no lane idles on a
// list entry beyond it.
template <bool ROWS>
__global__ void __launch_bounds__(128) k_polar_real_f(IndRealArgs A) {
    const IndArgs &a = A.ia;
    __shared__ double s_ipp[64];   // 1 / sqrt(a_i a_j) per type pair (at most 8 types)
    for (int q = threadIdx.x; q < A.ntypes * A.ntypes; q += blockDim.x)
        s_ipp[q] = 1.0 / sqrt(a.polar[q / A.ntypes] * a.polar[q % A.ntypes]);
    __syncthreads();
    constexpr int TPP = 8;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gt / TPP, t = gt % TPP;
    V3 f = v3(0, 0, 0), tau = v3(0, 0, 0);
    double emp = 0, eind = 0, w[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (i < a.n) {
        const int4 fi = A.fixq[i];
        const double qi_d = a.tq[fi.w] / SQC;
        const float4 *ri = A.srec + 4 * (size_t)i;
        const float4 i0 = ri[0], i1 = ri[1], i2 = ri[2], i3 = ri[3];
        const float qi = i0.x;
        const F3 mi = f3(i0.y, i0.z, i0.w);
        const F3 pii = f3(i2.z, i2.w, i3.x);
        const Q6F Qi = {i1.x, i1.y, i1.z, i1.w, i2.x, i2.y};
        const double s2u = A.dscale[0] * A.dscale[0];
        // listed: a Verlet-list neighbour (both terms); otherwise one of the
        // molecule's excluded sites (induced term with its permanent part
        // scaled by 0)
        auto pair = [&](int j, bool listed) {
            const int4 fj = A.fixq[j];
            const int ix = fi.x - fj.x, iy = fi.y - fj.y, iz = fi.z - fj.z;   // r = r_i - r_j
            const unsigned long long s2 = (unsigned long long)((long long)ix * ix) +
                                          (unsigned long long)((long long)iy * iy) +
                                          (unsigned long long)((long long)iz * iz);
            const double r2 = (double)s2 * s2u;
            if (!(r2 < a.rc2)) return;
            const V3 r = v3(ix * A.dscale[0], iy * A.dscale[1], iz * A.dscale[2]);
            const F3 rf = f3((float)r.x, (float)r.y, (float)r.z);
            const float4 *rj = A.srec + 4 * (size_t)j;
            const float4 j0 = __ldg(rj), j1 = __ldg(rj + 1), j2 = __ldg(rj + 2), j3 = __ldg(rj + 3);
            const F3 mj = f3(j0.y, j0.z, j0.w);
            const Q6F Qj = {j1.x, j1.y, j1.z, j1.w, j2.x, j2.y};
            double B[6], rr, ir2;
            bn_erfc_r(r2, a.alpha, B, rr, ir2);
            V3 fij = v3(0, 0, 0), ti = v3(0, 0, 0);
            if (listed) {
                MPPair<float, F3> P;
                mp_invariants(qi, mi, Qi, j0.x, mj, Qj, rf, P);
                const double G0 = qi_d * (a.tq[fj.w] / SQC);
                emp += G0 * B[0] + P.G[1] * B[1] + P.G[2] * B[2] + P.G[3] * B[3] + P.G[4] * B[4];
                const double radial = G0 * B[1] + P.G[1] * B[2] + P.G[2] * B[3] + P.G[3] * B[4] + P.G[4] * B[5];
                fij = -(B[1] * to_v3(P.gG[1]) + B[2] * to_v3(P.gG[2]) + B[3] * to_v3(P.gG[3]) +
                        B[4] * to_v3(P.gG[4])) -
                      radial * r;
                F3 Gt[5];
                mp_torque_i(j0.x, mi, Qi, mj, Qj, rf, Gt);
                ti = B[1] * to_v3(Gt[1]) + B[2] * to_v3(Gt[2]) + B[3] * to_v3(Gt[3]) + B[4] * to_v3(Gt[4]);
            }
            IndAlgF al;
            ind_algebra_f(qi, mi, Qi, pii, j0.x, mj, Qj, f3(j2.z, j2.w, j3.x), rf, al);
            IndPairOut o;
            ind_pair_mixed_b(al, r, rr, ir2, B, s_ipp[fi.w * A.ntypes + fj.w], a.a, listed ? 1.0 : 0.0, o);
            eind += o.e;
            fij = fij + o.fij;
            f = f + fij;
            tau = tau + ti + o.tau;
            const double fr[3] = {fij.x, fij.y, fij.z}, rv[3] = {r.x, r.y, r.z};
            for (int p = 0; p < 3; p++)
                for (int q = 0; q < 3; q++) w[3 * p + q] -= 0.5 * fr[q] * rv[p];
        };
        if (ROWS) {
            const int *rj = A.rj + (size_t)i * A.rcap;
            const int lc = A.rlcnt[i], cnt = A.rcnt[i];
            for (int k = t; k < lc; k += TPP) pair(rj[k], true);
            for (int k = lc + t; k < cnt; k += TPP) pair(rj[k], false);
        } else {
            const int cnt = a.nnbr[i];
            for (int k = t; k < cnt; k += TPP) pair(a.nbr[(size_t)k * a.n + i] & 0x7fffffff, true);
            if (t == 0) {
                const int m = a.mol[i];
                for (int q = a.mol_off[m]; q < a.mol_off[m + 1]; q++) {
                    const int j = a.mol_atoms[q];
                    if (j != i && is_excluded(i, j, a.excl_off, a.excl)) pair(j, false);
                }
            }
        }
    }
    f.x = group_sum<TPP>(f.x); f.y = group_sum<TPP>(f.y); f.z = group_sum<TPP>(f.z);
    tau.x = group_sum<TPP>(tau.x); tau.y = group_sum<TPP>(tau.y); tau.z = group_sum<TPP>(tau.z);
    if (i < a.n && t == 0) {
        add_fix3_at(A.frc, a.n, i, f, COU);
        add_fix3_at(A.trq, a.n, i, tau, COU);
    }
    __shared__ double s_r[4][11];
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    double vals[11] = {0.5 * emp * COU, 0.5 * eind * COU, w[0], w[1], w[2], w[3], w[4], w[5], w[6], w[7], w[8]};
    for (int q = 0; q < 11; q++) {
        double sv = warp_sum(vals[q]);
        if (lane == 0) s_r[wp][q] = sv;
    }
    __syncthreads();
    if (threadIdx.x < 11) {
        double sv = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) sv += s_r[q][threadIdx.x];
        const int slot = threadIdx.x == 0 ? ACC_E_REAL : (threadIdx.x == 1 ? ACC_E_POL_REAL : ACC_VIR + threadIdx.x - 2);
        if (sv != 0.0) atomicAdd((unsigned long long *)&A.acc[slot], (unsigned long long)to_fix(sv, ACC_SCALE));
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
            add_fix3_at(trq, a.n, i, crs(mi, pii), COU * (2.0 / 3.0) * a2pi * a2);
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

// Self and intramolecular corrections of both the multipole and the induced
// terms after the fused real-space pass, three threads per molecule: thread
// t takes the self terms of the molecule's sites t, t + 3, ... and its
// site pairs (p < q, in row order) t, t + 3, ...  The terms are those of
// k_mp_mol (Multipole self and intramolecular energies) and k_ind_mol
// (induced self energy and torque, induced intramolecular energy); spread
// over three threads, one molecule's chain of FP64 work is a third as long.
constexpr int PM_TPM = 3;
__global__ void __launch_bounds__(96) k_polar_mol(IndArgs a, long long *trq, long long *acc) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = g / PM_TPM, t = g - PM_TPM * m;
    double e_mps = 0, e_mpi = 0, e_ps = 0, e_pi = 0;
    if (m < a.nmol) {
        const double a2 = a.alpha * a.alpha, a2pi = 2.0 * a.alpha / SQRT_PI_I;
        const int s = a.mol_off[m], ns = a.mol_off[m + 1] - s;
        for (int p = t; p < ns; p += PM_TPM) {
            const int i = a.mol_atoms[s + p];
            const double4 pi = a.pos4[i];
            const double qi = a.tq[(int)pi.w] / SQC;
            const V3 mi = ld3i(a.mu, a.n, i), pii = ld3i(a.p, a.n, i);
            const Q6 Qi = ldqi(a.qd, a.n, i);
            const double QiI = qtr(Qi), QiQi = qdd(Qi, Qi);
            const double selfterm = qi * qi * a2pi + (dot(mi, mi) - 2 * qi * QiI) * 2 * a2pi * a2 / 3 +
                                    (QiI * QiI + 2 * QiQi) * 4 * a2pi * a2 * a2 / 5;
            e_mps += -0.5 * selfterm * COU;
            e_ps += -dot(mi, pii) * a2pi * a2 / 3 * COU;
            add_fix3_at(trq, a.n, i, crs(mi, pii), COU * (2.0 / 3.0) * a2pi * a2);
        }
        const int npair = ns * (ns - 1) / 2;
        for (int k = t; k < npair; k += PM_TPM) {
            int p = 0, rem = k;
            while (rem >= ns - 1 - p) { rem -= ns - 1 - p; p++; }
            const int q = p + 1 + rem;
            const int i = a.mol_atoms[s + p], j = a.mol_atoms[s + q];
            if (!is_excluded(i, j, a.excl_off, a.excl)) continue;
            const double4 pi = a.pos4[i], pj = a.pos4[j];
            const V3 r = mind(pi, pj, a.box);
            const double r2 = dot(r, r);
            const double qi = a.tq[(int)pi.w] / SQC, qj = a.tq[(int)pj.w] / SQC;
            const V3 mi = ld3i(a.mu, a.n, i), mj = ld3i(a.mu, a.n, j);
            const V3 pii = ld3i(a.p, a.n, i), pjj = ld3i(a.p, a.n, j);
            const Q6 Qi = ldqi(a.qd, a.n, i), Qj = ldqi(a.qd, a.n, j);
            double D[6];
            dn_erf(r2, a.alpha, D);
            // multipole: G . D of the permanent pair
            MPPair<double, V3> P;
            mp_invariants(qi, mi, Qi, qj, mj, Qj, r, P);
            e_mpi += -(P.G[0] * D[0] + P.G[1] * D[1] + P.G[2] * D[2] + P.G[3] * D[3] + P.G[4] * D[4]) * COU;
            // induced: the induced-permanent invariants of the pair
            const V3 rji = -r;
            const double pjr = dot(pjj, r), pirji = dot(pii, rji);
            const double G1i = -qi * pjr - dot(mi, pjj);
            const double G2i = -dot(mi, r) * pjr - 2.0 * dot(pjj, qv(Qi, r)) - pjr * qtr(Qi);
            const double G3i = -pjr * dot(r, qv(Qi, r));
            const double G1j = -qj * pirji - dot(mj, pii);
            const double G2j = -dot(mj, rji) * pirji - 2.0 * dot(pii, qv(Qj, rji)) - pirji * qtr(Qj);
            const double G3j = -pirji * dot(r, qv(Qj, r));
            e_pi += -0.5 * ((G1i + G1j) * D[1] + (G2i + G2j) * D[2] + (G3i + G3j) * D[3]) * COU;
        }
    }
    __shared__ double s_r[4][3];
    const double v[4] = {warp_sum(e_mps), warp_sum(e_mpi), warp_sum(e_ps), warp_sum(e_pi)};
    if ((threadIdx.x & 31) == 0)
        for (int q = 0; q < 4; q++) s_r[q][threadIdx.x >> 5] = v[q];
    __syncthreads();
    if (threadIdx.x < 4) {
        double tot = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) tot += s_r[threadIdx.x][w];
        const int slot[4] = {ACC_E_SELF, ACC_E_INTRA, ACC_E_POL_SELF, ACC_E_POL_INTRA};
        atomicAdd((unsigned long long *)&acc[slot[threadIdx.x]], (unsigned long long)to_fix(tot, ACC_SCALE));
    }
}

// ---------------------------------------------------------------------------
// forces and torques of the intramolecular corrections (flexible molecules)
// ---------------------------------------------------------------------------
// Without constraints the reference also applies the forces and torques of
// its intramolecular corrections (Multipole::intraMolCorrect,
// src/forces/Multipole.cpp:1398-1700; Induction::intraMolCorrect,
// src/forces/Induction.cpp:1900-2140): for every excluded pair of a
// molecule, the real-space expressions with the erf radial functions D_n in
// place of the erfc B_n and the opposite sign, undamped.  Their energies
// are formed by k_mp_mol / k_ind_mol / k_polar_mol with or without
// constraints; this kernel adds the forces and torques, one thread per
// molecule, FP64.  No virial: the reference adds none for these terms.
// fr_mol (may be null): per molecule, sum f_ij . r_ij over its pairs (the
// volume derivative's share, Multipole.cpp:1514, Induction.cpp:2013)
__global__ void k_intra_flex(IndArgs a, long long *frc, long long *trq, int mp, int ind, double *fr_mol) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= a.nmol) return;
    const int s0 = a.mol_off[m], ns = a.mol_off[m + 1] - s0;
    double fr = 0;
    for (int p = 0; p < ns; p++)
        for (int q = p + 1; q < ns; q++) {
            const int i = a.mol_atoms[s0 + p], j = a.mol_atoms[s0 + q];
            if (!is_excluded(i, j, a.excl_off, a.excl)) continue;
            const double4 pi = a.pos4[i], pj = a.pos4[j];
            const V3 r = mind(pi, pj, a.box);   // r_i - r_j
            const double r2 = dot(r, r);
            const double qi = a.tq[(int)pi.w] / SQC, qj = a.tq[(int)pj.w] / SQC;
            const V3 mi = ld3i(a.mu, a.n, i), mj = ld3i(a.mu, a.n, j);
            const Q6 Qi = ldqi(a.qd, a.n, i), Qj = ldqi(a.qd, a.n, j);
            double D[6];
            dn_erf(r2, a.alpha, D);
            V3 fij = v3(0, 0, 0), ti = v3(0, 0, 0), tj = v3(0, 0, 0);
            if (mp) {
                MPPair<double, V3> P;
                mp_invariants(qi, mi, Qi, qj, mj, Qj, r, P);
                const double radial = P.G[0] * D[1] + P.G[1] * D[2] + P.G[2] * D[3] + P.G[3] * D[4] + P.G[4] * D[5];
                fij = fij + (D[1] * P.gG[1] + D[2] * P.gG[2] + D[3] * P.gG[3] + D[4] * P.gG[4] + radial * r);
                V3 Gi[5], Gj[5];
                mp_torque_i(qj, mi, Qi, mj, Qj, r, Gi);
                mp_torque_i(qi, mj, Qj, mi, Qi, -r, Gj);
                ti = ti - (D[1] * Gi[1] + D[2] * Gi[2] + D[3] * Gi[3] + D[4] * Gi[4]);
                tj = tj - (D[1] * Gj[1] + D[2] * Gj[2] + D[3] * Gj[3] + D[4] * Gj[4]);
            }
            if (ind) {
                const V3 pii = ld3i(a.p, a.n, i), pjj = ld3i(a.p, a.n, j);
                const V3 rji = -r;
                const double QiI = qtr(Qi), QjI = qtr(Qj);
                const V3 Qir = qv(Qi, r), Qjrji = qv(Qj, rji);
                const double QiRij = dot(r, Qir), QjRji = dot(r, qv(Qj, r));
                const double pjr = dot(pjj, r), pirji = dot(pii, rji);
                const double G1i = -qi * pjr - dot(mi, pjj);
                const double G2i = -dot(mi, r) * pjr - 2.0 * dot(pjj, Qir) - pjr * QiI;
                const double G3i = -pjr * QiRij;
                const double G1j = -qj * pirji - dot(mj, pii);
                const double G2j = -dot(mj, rji) * pirji - 2.0 * dot(pii, Qjrji) - pirji * QjI;
                const double G3j = -pirji * QjRji;
                const V3 gG1i = -qi * pjj;
                const V3 gG2i = (-pjr) * mi - dot(mi, r) * pjj - 2.0 * qv(Qi, pjj) - QiI * pjj;
                const V3 gG3i = (-QiRij) * pjj - (2 * pjr) * Qir;
                const V3 gG1j = -qj * pii;
                const V3 gG2j = (-pirji) * mj - dot(mj, rji) * pii - 2.0 * qv(Qj, pii) - QjI * pii;
                const V3 gG3j = (-QjRji) * pii - (2 * pirji) * Qjrji;
                const V3 fi = D[1] * gG1i + D[2] * gG2i + D[3] * gG3i + (G1i * D[2] + G2i * D[3] + G3i * D[4]) * r;
                const V3 fj = D[1] * gG1j + D[2] * gG2j + D[3] * gG3j + (G1j * D[2] + G2j * D[3] + G3j * D[4]) * rji;
                fij = fij + (fi - fj);
                // torque coefficients as the real-space term's, for i and with i, j swapped
                const V3 Gt1i = crs(mi, pjj);
                const V3 Gt2i = pjr * crs(mi, r) + 2.0 * crs(Qir, pjj) + 2.0 * crs(qv(Qi, pjj), r);
                const V3 Gt3i = (2.0 * pjr) * crs(Qir, r);
                const V3 Gt1j = crs(mj, pii);
                const V3 Gt2j = pirji * crs(mj, rji) + 2.0 * crs(Qjrji, pii) + 2.0 * crs(qv(Qj, pii), rji);
                const V3 Gt3j = (2.0 * pirji) * crs(Qjrji, rji);
                ti = ti - (D[1] * Gt1i + D[2] * Gt2i + D[3] * Gt3i);
                tj = tj - (D[1] * Gt1j + D[2] * Gt2j + D[3] * Gt3j);
            }
            add_fix3_at(frc, a.n, i, fij, COU);
            add_fix3_at(frc, a.n, j, -fij, COU);
            add_fix3_at(trq, a.n, i, ti, COU);
            add_fix3_at(trq, a.n, j, tj, COU);
            fr += dot(fij, r);
        }
    if (fr_mol) fr_mol[m] = fr;
}


// ring of the last 4 steps' converged dipoles and permanent fields;
// flags[2] counts the stored steps
// Stores the step's dipoles and permanent field in ring slot flags[2] & 3.
// The last block to finish (ticket flags[3]) advances the step count
// flags[2] and clears the ticket: every block has read the count before it
// takes its ticket.
__global__ void k_hist_push(int n, const double *p, const double *e0, double *ph, int *flags) {
    __shared__ bool s_last;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        double *h = ph + (size_t)(flags[2] & 3) * 6 * n;
        h[i] = p[i]; h[n + i] = p[n + i]; h[2 * n + i] = p[2 * n + i];
        h[3 * n + i] = e0[i]; h[4 * n + i] = e0[n + i]; h[5 * n + i] = e0[2 * n + i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(&flags[3], 1) == (int)gridDim.x - 1;
    }
    __syncthreads();
    if (s_last && threadIdx.x == 0) {
        flags[2] += 1;
        flags[3] = 0;
    }
}

static IndArgs ind_args(Ctx &c) {
    IndArgs a;
    a.n = c.n; a.nmol = c.nmol; a.nbr = c.pl.nbr; a.nnbr = c.pl.nnbr; a.mol = c.mol;
    a.mol_off = c.mol_off; a.mol_atoms = c.mol_atoms; a.excl_off = c.excl_off; a.excl = c.excl;
    a.pos4 = c.pos4; a.tq = c.type_q; a.polar = c.type_polar; a.mu = c.mu; a.qd = c.qd;
    a.box = c.box; a.cut2 = c.ind_cut2; a.a = c.thole_a; a.alpha = c.ew_alpha; a.rc2 = c.mp_rc2;
    a.e0 = c.e0; a.p = c.pind;
    a.amoeba = c.ind_amoeba;
    return a;
}

void launch_intra_flex(Ctx &c, bool mp, bool ind) {
    // rigid molecules (constraint lengths set): the reference applies these
    // corrections as energies only
    if (c.clen2 || !(mp || ind)) return;
    k_intra_flex<<<(c.nmol + 127) / 128, 128, 0, c.stream>>>(ind_args(c), c.frc, c.trq, mp ? 1 : 0,
                                                            ind && c.ind_on ? 1 : 0, nullptr);
}

// the same pass with each molecule's sum f_ij . r_ij in fr_mol[nmol]
// (flexible molecules; the volume derivatives' intramolecular share)
void launch_intra_flex_lus(Ctx &c, bool mp, bool ind, double *fr_mol) {
    if (c.clen2 || !(mp || ind)) return;
    k_intra_flex<<<(c.nmol + 127) / 128, 128, 0, c.stream>>>(ind_args(c), c.frc, c.trq, mp ? 1 : 0,
                                                            ind && c.ind_on ? 1 : 0, fr_mol);
}

// FP64 induced real space alone, and the induced self term alone (the
// volume derivatives take each one's virial and torques on their own)
void launch_ind_real_only(Ctx &c) {
    IndRealArgs A;
    A.ia = ind_args(c);
    A.frc = c.frc; A.trq = c.trq; A.acc = c.acc;
    k_ind_real<<<(int)(((long long)c.n * 8 + 63) / 64), 64, 0, c.stream>>>(A);
}

void launch_ind_self_only(Ctx &c) {
    k_ind_mol<<<(c.nmol + 127) / 128, 128, 0, c.stream>>>(ind_args(c), c.trq, c.acc);
}

int setup_cg(Ctx &c) {
    // the grid must be co-resident for every variant of the solve kernel
    const void *kernels[4] = {(const void *)k_ind_cg<false, false>, (const void *)k_ind_cg<true, false>,
                              (const void *)k_ind_cg<false, true>, (const void *)k_ind_cg<true, true>};
    int per_sm = 1 << 30;
    for (const void *k : kernels) {
        int v = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k, CG_THREADS, 0) != cudaSuccess) return SMD_ERR_CUDA;
        per_sm = v < per_sm ? v : per_sm;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, c.device) != cudaSuccess) return SMD_ERR_CUDA;
    int want = (c.n * CG_TPP + CG_THREADS - 1) / CG_THREADS;
    int maxb = per_sm * prop.multiProcessorCount;
    c.cg_blocks = want < maxb ? want : maxb;
    if (c.cg_blocks < 1) c.cg_blocks = 1;
    // the pipelined form: every molecule three sites, molecule k's at 3k .. 3k + 2
    bool ok = c.nmol > 0 && c.n == 3 * c.nmol;
    for (int m = 0; ok && m <= c.nmol; m++) ok = c.h_mol_off[m] == 3 * m;
    for (int k = 0; ok && k < c.n; k++) ok = c.h_mol_atoms[k] == k;
    c.pp_blocks = 0;
    if (ok) {
        int v = 0;
        int v2 = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, (const void *)k_ind_pcg_pipe<true>, PP_THREADS, 0) !=
                cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v2, (const void *)k_ind_pcg_pipe<false>, PP_THREADS, 0) !=
                cudaSuccess)
            return SMD_ERR_CUDA;
        v = v2 < v ? v2 : v;
        const int groups = (c.nmol + PP_MOLS - 1) / PP_MOLS;
        const int mb = v * prop.multiProcessorCount;
        c.pp_blocks = groups < mb ? groups : mb;
    }
    return 0;
}

// tensor rows: one slot per Verlet-list entry plus the molecule's sites
int ensure_ind_rows(Ctx &c) {
    if (!c.mp_on || !c.ind_on || c.n == 0) return 0;
    int maxmol = 1;
    for (size_t m = 0; m + 1 < c.h_mol_off.size(); m++)
        maxmol = std::max(maxmol, c.h_mol_off[m + 1] - c.h_mol_off[m]);
    const int cap = ((c.pl.max_nbr + maxmol + 3) / 4) * 4;
    if (cap == c.ind_cap && c.ind_rj) return 0;
    cudaFree(c.ind_rj); cudaFree(c.ind_rc); cudaFree(c.ind_cnt);
    c.ind_rj = nullptr; c.ind_rc = nullptr; c.ind_cnt = nullptr;
    c.ind_cap = 0;
    const size_t slots = (size_t)c.n * cap;
    if (cudaMalloc(&c.ind_rj, slots * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&c.ind_rc, slots * sizeof(double4)) != cudaSuccess ||
        cudaMalloc(&c.ind_cnt, 2 * (size_t)c.n * sizeof(int)) != cudaSuccess)
        return SMD_ERR_CUDA;
    c.ind_cap = cap;
    c.graph_dirty = 1;
    return 0;
}

// permanent field and tensor rows, then the learned start dipoles
void launch_ind_field(Ctx &c) {
    IndArgs a = ind_args(c);
    const bool f32 = c.precision == SMD_PREC_MIXED;
    TRows R;
    R.j = c.ind_rj; R.c = c.ind_rc; R.cnt = c.ind_cnt; R.lcnt = c.ind_cnt + c.n; R.cap = c.ind_cap;
    const int nb = (int)(((long long)c.n * 8 + 255) / 256);
    const bool cubic = c.box.L[0] == c.box.L[1] && c.box.L[1] == c.box.L[2];
    if (f32 && cubic && c.srec && c.ntypes <= 8) {
        if (!c.fixq_from_integrate) launch_fixq(c);
        FieldMixArgs m;
        m.fixq = c.fixq; m.srec = c.srec; m.ntypes = c.ntypes;
        for (int d = 0; d < 3; d++) m.dscale[d] = c.box.L[d] / 4294967296.0;
        k_ind_field_f<<<nb, 256, 0, c.stream>>>(a, m, R, c.status);
    } else if (f32)
        k_ind_field<float><<<nb, 256, 0, c.stream>>>(a, R, c.status);
    else
        k_ind_field<double><<<nb, 256, 0, c.stream>>>(a, R, c.status);
    // the preconditioner's inverse molecule blocks (they need this step's tensor rows)
    const bool learned = c.cg_guess == SMD_GUESS_LEARNED && c.mlp_ready;
    const bool first_order = guess_order(c) > 0 && !learned;
    const int order = learned ? c.mlp_base : guess_order(c);
    if (c.cg_precond == SMD_PRECOND_MOLECULE && c.cg_blk) {
        // with the learned or extrapolated guess, also the blocks' responses
        double *dl = (learned || first_order) ? guess_response(c) : nullptr;
        double *dlp = learned ? guess_response_prev(c) : nullptr;
        const int nbm = (c.nmol + MB_MOLS - 1) / MB_MOLS;
        if (f32)
            k_mol_blocks<float><<<nbm, 9 * MB_MOLS, 0, c.stream>>>(c.n, c.nmol, c.mol_off, c.mol_atoms, R,
                                                                   c.type_polar, c.pos4, c.cg_blk, c.e0, c.phist,
                                                                   c.flags, dl, order, dlp);
        else
            k_mol_blocks<double><<<nbm, 9 * MB_MOLS, 0, c.stream>>>(c.n, c.nmol, c.mol_off, c.mol_atoms, R,
                                                                    c.type_polar, c.pos4, c.cg_blk, c.e0, c.phist,
                                                                    c.flags, dl, order, dlp);
    }
    if (learned) launch_mlp_guess(c);  // writes the start dipoles into p
    else if (first_order) launch_first_order_guess(c);
}

// Response of each molecule's own block to the permanent field's difference
// of the extrapolated guess of the given order, out = M_m^-1 (E0(t) -
// sum_j w_j E0(t-j)) (M_m^-1 E0(t) when no step is stored), nine threads per
// molecule; with the site preconditioner the block is diag(alpha).
constexpr int RESP_MOLS = 32;
__global__ void __launch_bounds__(9 * RESP_MOLS) k_blk_response(int n, int nmol, const int *mol_off,
                                                               const int *mol_atoms, const double *blk,
                                                               const double *polar, const double4 *pos4,
                                                               const double *e0, const double *ph,
                                                               const int *flags, double *out, int order,
                                                               double *out_prev) {
    __shared__ double s_v[9 * RESP_MOLS];
    const int ml = threadIdx.x / 9, e = threadIdx.x - 9 * ml, q = e / 3, d = e - 3 * q;
    const int m = blockIdx.x * RESP_MOLS + ml;
    const int cnt = flags[2];
    int ns = 0, i = -1;
    if (m < nmol) {
        const int s0 = mol_off[m];
        ns = min(3, mol_off[m + 1] - s0);
        if (q < ns) i = mol_atoms[s0 + q];
    }
    const size_t idx = (size_t)d * n + i;
    s_v[threadIdx.x] = i >= 0 ? hist_diff_e(ph, n, cnt, order, idx, e0[idx]) : 0.0;
    __syncthreads();
    auto apply = [&]() {
        double u = 0.0;
        if (blk) {
            for (int col = 0; col < 3 * ns; col++) u += blk[(size_t)(e * 9 + col) * nmol + m] * s_v[9 * ml + col];
        } else {
            u = fmax(1e-8, polar[(int)pos4[i].w]) * s_v[threadIdx.x];
        }
        return u;
    };
    if (i >= 0) out[idx] = apply();
    if (!out_prev) return;   // block-uniform
    __syncthreads();
    s_v[threadIdx.x] = i >= 0 && cnt >= 2 ? ph[(size_t)((cnt - 1) & 3) * 6 * n + 3 * (size_t)n + idx] -
                                                ph[(size_t)((cnt - 2) & 3) * 6 * n + 3 * (size_t)n + idx]
                                          : 0.0;
    __syncthreads();
    if (i >= 0) out_prev[idx] = apply();
}

void launch_blk_response(Ctx &c, double *out, int order, double *out_prev) {
    const double *blk = c.cg_precond == SMD_PRECOND_MOLECULE ? c.cg_blk : nullptr;
    k_blk_response<<<(c.nmol + RESP_MOLS - 1) / RESP_MOLS, 9 * RESP_MOLS, 0, c.stream>>>(
        c.n, c.nmol, c.mol_off, c.mol_atoms, blk, c.type_polar, c.pos4, c.e0, c.phist, c.flags, out, order,
        out_prev);
}

// the PCG solve from the start dipoles, then the site records' new dipoles
// and the step's dipole history
void launch_ind_cg(Ctx &c) {
    IndArgs a = ind_args(c);
    const bool f32 = c.precision == SMD_PREC_MIXED;
    TRows R;
    R.j = c.ind_rj; R.c = c.ind_rc; R.cnt = c.ind_cnt; R.lcnt = c.ind_cnt + c.n; R.cap = c.ind_cap;
    const bool learned = c.cg_guess == SMD_GUESS_LEARNED && c.mlp_ready;
    CGArgs g;
    g.ia = a;
    g.rows = R;
    const size_t n = c.n;
    g.r = c.cgw; g.z = c.cgw + 3 * n; g.v = c.cgw + 6 * n; g.al = c.cgw + 9 * n;
    g.g0 = c.cgw + 12 * n; g.g1 = c.cgw + 16 * n;
    g.s = c.cgw + 20 * n; g.u = c.cgw + 23 * n;
    g.part = c.cgs + CG_SCAL + CG_TRACE; g.scal = c.cgs; g.bar = c.cg_bar; g.status = c.status;
    g.wait_ns = c.wait_ns;
    g.skip_block = c.test_skip_block;
    g.nblocks = c.cg_blocks; g.max_iter = c.cg_max_iter; g.tol = c.cg_tol;
    // 0: start from alpha E0; 1: start from the dipoles in p (previous solve or network)
    g.guess = (c.cg_guess == SMD_GUESS_PREVIOUS || guess_order(c) > 0 || learned) ? 1 : 0;
    const bool bj = c.cg_precond == SMD_PRECOND_MOLECULE && c.cg_blk;   // blocks built by launch_ind_field
    g.blk = c.cg_blk;
    // the mixed path's site records take the dipoles inside the solve
    g.srec = f32 && c.srec ? (float *)c.srec : nullptr;
    cudaMemsetAsync(c.cg_bar, 0, 2 * sizeof(unsigned int), c.stream);   // counter and abort word
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
    g.w = c.cgw + 26 * n; g.m = c.cgw + 29 * n; g.q = c.cgw + 32 * n;
    // the pipelined recurrences drift by rounding, which limits the change
    // they can resolve: tight tolerances (the checkers' 1e-13) keep the
    // single-reduction form
    // mode 1 (the default): the mixed path only; in FP64 the single-reduction
    // form is the faster one (double4 gathers; 0.450 against 0.480 ms on
    // polwater4096); mode 2: both precisions
    if (bj && c.pp_blocks > 0 && c.cg_pipelined >= (f32 ? 1 : 2) && c.cg_tol >= PP_MIN_TOL) {
        g.nblocks = c.pp_blocks;
        cfg.gridDim = dim3(c.pp_blocks);
        cfg.blockDim = dim3(PP_THREADS);
        if (f32)
            cudaLaunchKernelEx(&cfg, k_ind_pcg_pipe<true>, g);
        else
            cudaLaunchKernelEx(&cfg, k_ind_pcg_pipe<false>, g);
    } else if (f32 && bj)
        cudaLaunchKernelEx(&cfg, k_ind_cg<true, true>, g);
    else if (f32)
        cudaLaunchKernelEx(&cfg, k_ind_cg<true, false>, g);
    else if (bj)
        cudaLaunchKernelEx(&cfg, k_ind_cg<false, true>, g);
    else
        cudaLaunchKernelEx(&cfg, k_ind_cg<false, false>, g);
    // a time step stores its converged dipoles for the next steps' guess
    if (c.in_step && c.phist) {
        k_hist_push<<<(c.n + 255) / 256, 256, 0, c.stream>>>(c.n, c.pind, c.e0, c.phist, c.flags);
    }
}

void launch_ind_solve(Ctx &c) {
    launch_ind_field(c);
    launch_ind_cg(c);
}

void launch_ind_short(Ctx &c) {
    IndRealArgs A;
    A.ia = ind_args(c);
    A.frc = c.frc; A.trq = c.trq; A.acc = c.acc;
    // 64-thread blocks: at this kernel's register count the SM holds more
    // warps in small blocks than in one 256-thread block
    const int nb = (int)(((long long)c.n * 8 + 63) / 64);
    const bool cubic = c.box.L[0] == c.box.L[1] && c.box.L[1] == c.box.L[2];
    if (c.precision == SMD_PREC_MIXED && cubic) {
        if (!c.fixq_from_integrate) launch_fixq(c);
        A.fixq = c.fixq;
        A.srec = c.srec;
        for (int d = 0; d < 3; d++) A.dscale[d] = c.box.L[d] / 4294967296.0;
        k_ind_real_f<<<nb, 64, 0, c.stream>>>(A);
    } else {
        k_ind_real<<<nb, 64, 0, c.stream>>>(A);
    }
    k_ind_mol<<<(c.nmol + 127) / 128, 128, 0, c.stream>>>(A.ia, c.trq, c.acc);
    launch_intra_flex(c, false, true);
}

bool polar_short_fused(const Ctx &c) {
    const bool cubic = c.box.L[0] == c.box.L[1] && c.box.L[1] == c.box.L[2];
    return c.precision == SMD_PREC_MIXED && cubic && c.srec && c.ind_on && !c.ind_amoeba;
}

// Both real-space polarisable terms after the dipole solve: one fused pass
// in the mixed path, the two separate passes otherwise
void launch_polar_short(Ctx &c) {
    if (!polar_short_fused(c)) {
        launch_mp_short(c);
        launch_ind_short(c);
        return;
    }
    IndRealArgs A;
    A.ia = ind_args(c);
    A.frc = c.frc; A.trq = c.trq; A.acc = c.acc;
    if (!c.fixq_from_integrate) launch_fixq(c);
    A.fixq = c.fixq;
    A.srec = c.srec;
    for (int d = 0; d < 3; d++) A.dscale[d] = c.box.L[d] / 4294967296.0;
    A.rj = c.ind_rj; A.rcnt = c.ind_cnt; A.rlcnt = c.ind_cnt + c.n; A.rcap = c.ind_cap;
    A.ntypes = c.ntypes;
    const int nb = (int)(((long long)c.n * 8 + 127) / 128);
    // the rows hold every pair inside the real-space cutoff when cutoffInd
    // reaches it; the pair test r^2 < rc^2 stays in the kernel
    if (c.ind_cut2 >= c.mp_rc2)
        k_polar_real_f<true><<<nb, 128, 0, c.stream>>>(A);
    else
        k_polar_real_f<false><<<nb, 128, 0, c.stream>>>(A);
    k_polar_mol<<<(c.nmol * PM_TPM + 95) / 96, 96, 0, c.stream>>>(A.ia, c.trq, c.acc);
    launch_intra_flex(c, true, true);
}

}  // namespace smd
