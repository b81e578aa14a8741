// Permanent multipole electrostatics of the polarisable water model
// (Multipole::compute / compute_long, src/forces/Multipole.cpp) and the
// torque-to-force mapping shared with the induction terms.
//
// Sites carry a charge, a dipole and a traceless quadrupole given in a
// molecular local frame.  Per step:
//   k_frames      local -> lab frame rotation (Local2Global::FrameofReference,
//                 src/utils/Local2Global.cpp:90-225); quadrupoles are /3
//   k_mp_real     Ewald real space over the full Verlet list with the B_n
//                 erfc recursion and the G_n multipole invariants
//                 (Multipole::real_term, Multipole.cpp:398-913): energy,
//                 force and torque on the owning site
//   k_mp_mol      self energy (:338-396) and the intramolecular erf
//                 correction energy (:1290-1713; under constraints the
//                 reference applies no intramolecular force or torque)
//   k_mp_sk_* / k_mp_recip_force  reciprocal sum with the charge-quadrupole
//                 and dipole structure factors (:951-1245)
//   k_torque2force  torques mapped onto the H-O-H sites
//                 (Multipole::torques2forces, :1946-2134)
// The FP64 path computes in FP64; the mixed path (k_mp_real_f) keeps the
// radial factors and the charge-charge term in FP64 and the multipole
// algebra in FP32.  Forces and torques accumulate in 64-bit fixed point.
#include "smd_ctx.cuh"
#include "smd_polar.cuh"

namespace smd {

constexpr double COULOMBS = 138.93548501;            // src/NEMD_defs.h:98
constexpr double SQRTCOULOMB = 11.78708976;          // src/NEMD_defs.h:97
constexpr double SQRT_PI_D = 1.7724538509055160273;

__device__ __forceinline__ V3 ld3(const double *a, int n, int i) { return v3(a[i], a[n + i], a[2 * n + i]); }
__device__ __forceinline__ Q6 ldq(const double *a, int n, int i) {
    return {a[i], a[n + i], a[2 * n + i], a[3 * n + i], a[4 * n + i], a[5 * n + i]};
}

// ---------------------------------------------------------------------------
// frames
// ---------------------------------------------------------------------------
// Local axes per site of an H O H molecule: H sites take z along O - H and x
// from the lab x axis (lab y when |z.x| > 0.866); O takes z along the sum of
// the unit O->H vectors and x from the unit O->H2 vector; then
// u = x - (x.z) z normalised, v = z x u (Local2Global.cpp:100-150).
// One thread per site (thread q of a molecule takes site q), which then
// writes the site's FP32 record of the mixed path (srec, when given) and
// clears its torque accumulators.  A record is one
// 64-byte row per site, so that a pair kernel gathers a partner's charge and
// multipoles with four vector loads: (q, mu), (Qxx, Qxy, Qxz, Qyy),
// (Qyz, Qzz, px, py), (pz, 0, 0, 0); the dipole solve rewrites p.
__global__ void k_frames(int nmol, int n, const int *mol_off, const int *mol_atoms,
                         const double4 *pos4, const double *type_mp, double *mu, double *qd,
                         double *frame, const double *tq, const double *pind, float4 *srec, long long *trq) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = g / 3, q = g - 3 * m;
    if (m >= nmol) return;
    const int s = mol_off[m];
    if (mol_off[m + 1] - s != 3) return;
    const int ih1 = mol_atoms[s], io = mol_atoms[s + 1], ih2 = mol_atoms[s + 2];
    const double4 a = pos4[ih1], b = pos4[io], c = pos4[ih2];
    const V3 rh1 = v3(a.x, a.y, a.z), ro = v3(b.x, b.y, b.z), rh2 = v3(c.x, c.y, c.z);
    V3 p1, p2;
    if (q == 0) {
        p1 = ro - rh1;
        p2 = fabs(p1.x / len(p1)) > 0.8660 ? v3(0, 1, 0) : v3(1, 0, 0);
    } else if (q == 1) {
        V3 t1 = rh1 - ro, t2 = rh2 - ro;
        t1 = (1.0 / len(t1)) * t1;
        t2 = (1.0 / len(t2)) * t2;
        p1 = t1 + t2;
        p2 = t2;
    } else {
        p1 = ro - rh2;
        p2 = fabs(p1.x / len(p1)) > 0.8660 ? v3(0, 1, 0) : v3(1, 0, 0);
    }
    {
        const V3 w = (1.0 / len(p1)) * p1;
        const V3 ss = p2 - dot(p2, w) * w;
        const V3 u = (1.0 / len(ss)) * ss;
        const V3 v = crs(w, u);
        const int id = q == 0 ? ih1 : (q == 1 ? io : ih2);
        if (frame) {  // axes u, v, w per site, for the dipole-guess network
            const double ax[9] = {u.x, u.y, u.z, v.x, v.y, v.z, w.x, w.y, w.z};
            for (int d = 0; d < 9; d++) frame[(size_t)d * n + id] = ax[d];
        }
        const double *tp = type_mp + 9 * (int)pos4[id].w;
        const double dx = tp[0], dy = tp[1], dz = tp[2];
        mu[id] = u.x * dx + v.x * dy + w.x * dz;
        mu[n + id] = u.y * dx + v.y * dy + w.y * dz;
        mu[2 * n + id] = u.z * dx + v.z * dy + w.z * dz;
        // Q' = R Q R^T / 3 with R = [u v w] (columns)
        const double L[3][3] = {{tp[3], tp[4], tp[5]}, {tp[4], tp[6], tp[7]}, {tp[5], tp[7], tp[8]}};
        const double R[3][3] = {{u.x, v.x, w.x}, {u.y, v.y, w.y}, {u.z, v.z, w.z}};
        double G[3][3];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                double t = 0;
                for (int k = 0; k < 3; k++) {
                    double inner = 0;
                    for (int l = 0; l < 3; l++) inner += R[j][l] * L[k][l];
                    t += R[i][k] * inner;
                }
                G[i][j] = t / 3.0;
            }
        qd[id] = G[0][0];
        qd[n + id] = G[0][1];
        qd[2 * n + id] = G[0][2];
        qd[3 * n + id] = G[1][1];
        qd[4 * n + id] = G[1][2];
        qd[5 * n + id] = G[2][2];
        if (srec) {
            float4 *o = srec + 4 * (size_t)id;
            o[0] = make_float4((float)(tq[(int)pos4[id].w] / SQRTCOULOMB), (float)mu[id], (float)mu[n + id],
                               (float)mu[2 * n + id]);
            o[1] = make_float4((float)G[0][0], (float)G[0][1], (float)G[0][2], (float)G[1][1]);
            o[2] = make_float4((float)G[1][2], (float)G[2][2], (float)pind[id], (float)pind[n + id]);
            o[3] = make_float4((float)pind[2 * n + id], 0.f, 0.f, 0.f);
        }
        trq[id] = 0;
        trq[n + id] = 0;
        trq[2 * n + id] = 0;
    }
}

// local frames, lab-frame multipoles, the mixed path's site records and
// cleared torques in one launch (every multipole molecule is an H O H triple)
void launch_frames(Ctx &c) {
    float4 *srec = c.precision == SMD_PREC_MIXED ? c.srec : nullptr;
    k_frames<<<(3 * c.nmol + 95) / 96, 96, 0, c.stream>>>(c.nmol, c.n, c.mol_off, c.mol_atoms, c.pos4,
                                                         c.type_mp, c.mu, c.qd, c.frame, c.type_q, c.pind, srec,
                                                         c.trq);
}

// ---------------------------------------------------------------------------
// real space
// ---------------------------------------------------------------------------
struct MPArgs {
    int n;
    const int *nbr, *nnbr;
    const double4 *pos4;
    const double *mu, *qd, *tq;
    Box box;
    double alpha, rc2;
    long long *frc, *trq, *acc;
    const int4 *fixq;      // mixed path: box fractions
    const float4 *srec;    // mixed path: FP32 site records (q, mu, Q, p)
    double dscale[3];      // L / 2^32 per axis
};

template <int TPP>
__global__ void __launch_bounds__(128, 3) k_mp_real(MPArgs a) {
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gt / TPP, t = gt % TPP;
    V3 f = v3(0, 0, 0), tau = v3(0, 0, 0);
    double en = 0, w[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (i < a.n) {
        const double4 pi = a.pos4[i];
        const double qi = a.tq[(int)pi.w] / SQRTCOULOMB;
        const V3 mi = ld3(a.mu, a.n, i);
        const Q6 Qi = ldq(a.qd, a.n, i);
        const int cnt = a.nnbr[i];
        for (int k = t; k < cnt; k += TPP) {
            const int j = a.nbr[(size_t)k * a.n + i] & 0x7fffffff;
            const double4 pj = a.pos4[j];
            V3 r = v3(pbc1(pi.x - pj.x, a.box.L[0], a.box.half[0]),
                      pbc1(pi.y - pj.y, a.box.L[1], a.box.half[1]),
                      pbc1(pi.z - pj.z, a.box.L[2], a.box.half[2]));
            const double r2 = dot(r, r);
            if (!(r2 < a.rc2)) continue;
            const double qj = a.tq[(int)pj.w] / SQRTCOULOMB;
            const V3 mj = ld3(a.mu, a.n, j);
            const Q6 Qj = ldq(a.qd, a.n, j);
            MPPair<double, V3> P;
            mp_invariants(qi, mi, Qi, qj, mj, Qj, r, P);
            double B[6];
            bn_erfc(r2, a.alpha, B);
            en += P.G[0] * B[0] + P.G[1] * B[1] + P.G[2] * B[2] + P.G[3] * B[3] + P.G[4] * B[4];
            const double radial = P.G[0] * B[1] + P.G[1] * B[2] + P.G[2] * B[3] + P.G[3] * B[4] + P.G[4] * B[5];
            const V3 fij = -(B[1] * P.gG[1] + B[2] * P.gG[2] + B[3] * P.gG[3] + B[4] * P.gG[4]) - radial * r;
            f = f + fij;
            // Ensemble virial gets -sum fij_b r_a (reference omits COULOMBS here)
            const double fr[3] = {fij.x, fij.y, fij.z}, rr[3] = {r.x, r.y, r.z};
            for (int p = 0; p < 3; p++)
                for (int q = 0; q < 3; q++) w[3 * p + q] -= 0.5 * fr[q] * rr[p];
            V3 Gt[5];
            mp_torque_i(qj, mi, Qi, mj, Qj, r, Gt);
            tau = tau + (B[1] * Gt[1] + B[2] * Gt[2] + B[3] * Gt[3] + B[4] * Gt[4]);
        }
    }
    f.x = group_sum<TPP>(f.x); f.y = group_sum<TPP>(f.y); f.z = group_sum<TPP>(f.z);
    tau.x = group_sum<TPP>(tau.x); tau.y = group_sum<TPP>(tau.y); tau.z = group_sum<TPP>(tau.z);
    if (i < a.n && t == 0) {
        add_fix3(a.frc, a.n, i, f, COULOMBS);
        add_fix3(a.trq, a.n, i, tau, COULOMBS);
    }
    __shared__ double s_r[8][10];
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    double vals[10] = {0.5 * en * COULOMBS, w[0], w[1], w[2], w[3], w[4], w[5], w[6], w[7], w[8]};
    for (int q = 0; q < 10; q++) {
        double s = warp_sum(vals[q]);
        if (lane == 0) s_r[wp][q] = s;
    }
    __syncthreads();
    if (threadIdx.x < 10) {
        double s = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) s += s_r[q][threadIdx.x];
        const int slot = threadIdx.x == 0 ? ACC_E_REAL : ACC_VIR + threadIdx.x - 1;
        if (s != 0.0) atomicAdd((unsigned long long *)&a.acc[slot], (unsigned long long)to_fix(s, ACC_SCALE));
    }
}

// Mixed path: displacement from the box fractions (exact integer difference,
// r^2 from the 64-bit integer sum), the multipole invariants, their
// gradients and the torque coefficients in FP32; the B_n, the charge-charge
// term q_i q_j B_n, the energy and the force assembly in FP64 (cubic boxes).
template <int TPP>
__global__ void __launch_bounds__(128, 3) k_mp_real_f(MPArgs a) {
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gt / TPP, t = gt % TPP;
    V3 f = v3(0, 0, 0), tau = v3(0, 0, 0);
    double en = 0, w[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (i < a.n) {
        const int4 fi = a.fixq[i];
        const double qi_d = a.tq[fi.w] / SQRTCOULOMB;
        const float4 i0 = a.srec[4 * (size_t)i], i1 = a.srec[4 * (size_t)i + 1], i2 = a.srec[4 * (size_t)i + 2];
        const float qi = i0.x;
        const F3 mi = f3(i0.y, i0.z, i0.w);
        const Q6F Qi = {i1.x, i1.y, i1.z, i1.w, i2.x, i2.y};
        const double s2u = a.dscale[0] * a.dscale[0];
        const int cnt = a.nnbr[i];
        for (int k = t; k < cnt; k += TPP) {
            const int j = a.nbr[(size_t)k * a.n + i] & 0x7fffffff;
            const int4 fj = a.fixq[j];
            const int ix = fi.x - fj.x, iy = fi.y - fj.y, iz = fi.z - fj.z;   // r = r_i - r_j
            const unsigned long long s2 = (unsigned long long)((long long)ix * ix) +
                                          (unsigned long long)((long long)iy * iy) +
                                          (unsigned long long)((long long)iz * iz);
            const double r2 = (double)s2 * s2u;
            if (!(r2 < a.rc2)) continue;
            const V3 r = v3(ix * a.dscale[0], iy * a.dscale[1], iz * a.dscale[2]);
            const F3 rf = f3((float)r.x, (float)r.y, (float)r.z);
            const double qj_d = a.tq[fj.w] / SQRTCOULOMB;
            const float4 j0 = __ldg(&a.srec[4 * (size_t)j]), j1 = __ldg(&a.srec[4 * (size_t)j + 1]);
            const float4 j2 = __ldg(&a.srec[4 * (size_t)j + 2]);
            const float qj = j0.x;
            const F3 mj = f3(j0.y, j0.z, j0.w);
            const Q6F Qj = {j1.x, j1.y, j1.z, j1.w, j2.x, j2.y};
            MPPair<float, F3> P;
            mp_invariants(qi, mi, Qi, qj, mj, Qj, rf, P);
            double B[6];
            bn_erfc(r2, a.alpha, B);
            const double G0 = qi_d * qj_d;
            en += G0 * B[0] + P.G[1] * B[1] + P.G[2] * B[2] + P.G[3] * B[3] + P.G[4] * B[4];
            const double radial = G0 * B[1] + P.G[1] * B[2] + P.G[2] * B[3] + P.G[3] * B[4] + P.G[4] * B[5];
            const V3 fij = -(B[1] * to_v3(P.gG[1]) + B[2] * to_v3(P.gG[2]) + B[3] * to_v3(P.gG[3]) +
                             B[4] * to_v3(P.gG[4])) -
                           radial * r;
            f = f + fij;
            const double fr[3] = {fij.x, fij.y, fij.z}, rr[3] = {r.x, r.y, r.z};
            for (int p = 0; p < 3; p++)
                for (int q = 0; q < 3; q++) w[3 * p + q] -= 0.5 * fr[q] * rr[p];
            F3 Gt[5];
            mp_torque_i(qj, mi, Qi, mj, Qj, rf, Gt);
            tau = tau + (B[1] * to_v3(Gt[1]) + B[2] * to_v3(Gt[2]) + B[3] * to_v3(Gt[3]) + B[4] * to_v3(Gt[4]));
        }
    }
    f.x = group_sum<TPP>(f.x); f.y = group_sum<TPP>(f.y); f.z = group_sum<TPP>(f.z);
    tau.x = group_sum<TPP>(tau.x); tau.y = group_sum<TPP>(tau.y); tau.z = group_sum<TPP>(tau.z);
    if (i < a.n && t == 0) {
        add_fix3(a.frc, a.n, i, f, COULOMBS);
        add_fix3(a.trq, a.n, i, tau, COULOMBS);
    }
    __shared__ double s_r[8][10];
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    double vals[10] = {0.5 * en * COULOMBS, w[0], w[1], w[2], w[3], w[4], w[5], w[6], w[7], w[8]};
    for (int q = 0; q < 10; q++) {
        double sv = warp_sum(vals[q]);
        if (lane == 0) s_r[wp][q] = sv;
    }
    __syncthreads();
    if (threadIdx.x < 10) {
        double sv = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) sv += s_r[q][threadIdx.x];
        const int slot = threadIdx.x == 0 ? ACC_E_REAL : ACC_VIR + threadIdx.x - 1;
        if (sv != 0.0) atomicAdd((unsigned long long *)&a.acc[slot], (unsigned long long)to_fix(sv, ACC_SCALE));
    }
}

// ---------------------------------------------------------------------------
// self energy and intramolecular correction (energy only: rigid molecules)
// ---------------------------------------------------------------------------
__global__ void k_mp_mol(int nmol, int n, const int *mol_off, const int *mol_atoms,
                         const int *excl_off, const int *excl, const double4 *pos4, const double *tq,
                         const double *mu, const double *qd, Box box, double alpha, long long *acc) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    double eself = 0, eintra = 0;
    if (m < nmol) {
        const double a2 = alpha * alpha, a2pi = 2.0 * alpha / SQRT_PI_D;
        const int s = mol_off[m], e = mol_off[m + 1];
        for (int p = s; p < e; p++) {
            const int i = mol_atoms[p];
            const double4 pi = pos4[i];
            const double qi = tq[(int)pi.w] / SQRTCOULOMB;
            const V3 mi = ld3(mu, n, i);
            const Q6 Qi = ldq(qd, n, i);
            const double QiI = qtr(Qi), QiQi = qdd(Qi, Qi);
            const double selfterm = qi * qi * a2pi + (dot(mi, mi) - 2 * qi * QiI) * 2 * a2pi * a2 / 3 +
                                    (QiI * QiI + 2 * QiQi) * 4 * a2pi * a2 * a2 / 5;
            eself += -0.5 * selfterm * COULOMBS;
            for (int q = p + 1; q < e; q++) {
                const int j = mol_atoms[q];
                bool ex = false;
                for (int k = excl_off[i]; k < excl_off[i + 1]; k++)
                    if (excl[k] == j) { ex = true; break; }
                if (!ex) continue;
                const double4 pj = pos4[j];
                V3 r = v3(pbc1(pi.x - pj.x, box.L[0], box.half[0]), pbc1(pi.y - pj.y, box.L[1], box.half[1]),
                          pbc1(pi.z - pj.z, box.L[2], box.half[2]));
                const double r2 = dot(r, r);
                MPPair<double, V3> P;
                mp_invariants(qi, mi, Qi, tq[(int)pj.w] / SQRTCOULOMB, ld3(mu, n, j), ldq(qd, n, j), r, P);
                double D[6];
                dn_erf(r2, alpha, D);
                eintra += P.G[0] * D[0] + P.G[1] * D[1] + P.G[2] * D[2] + P.G[3] * D[3] + P.G[4] * D[4];
            }
        }
    }
    __shared__ double s_r[2][4];
    double v0 = warp_sum(eself), v1 = warp_sum(-eintra * COULOMBS);
    if ((threadIdx.x & 31) == 0) { s_r[0][threadIdx.x >> 5] = v0; s_r[1][threadIdx.x >> 5] = v1; }
    __syncthreads();
    if (threadIdx.x < 2) {
        double t = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) t += s_r[threadIdx.x][q];
        atomicAdd((unsigned long long *)&acc[threadIdx.x == 0 ? ACC_E_SELF : ACC_E_INTRA],
                  (unsigned long long)to_fix(t, ACC_SCALE));
    }
}

// ---------------------------------------------------------------------------
// torques -> forces on the H O H sites (Multipole::torques2forces)
// ---------------------------------------------------------------------------
// One thread per site: thread q of a molecule maps site q's torque and adds
// the forces on the molecule's sites atomically (integer adds, so the sum
// does not depend on their order).
__global__ void k_torque2force(int nmol, int n, const int *mol_off, const int *mol_atoms,
                               const double4 *pos4, const long long *trq, long long *frc) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = g / 3, q = g - 3 * m;
    if (m >= nmol) return;
    const int s = mol_off[m];
    if (mol_off[m + 1] - s != 3) return;
    const int h1 = mol_atoms[s], o = mol_atoms[s + 1], h2 = mol_atoms[s + 2];
    const double4 a = pos4[h1], b = pos4[o], c = pos4[h2];
    const V3 rh1 = v3(a.x, a.y, a.z), ro = v3(b.x, b.y, b.z), rh2 = v3(c.x, c.y, c.z);
    auto tq = [&](int id) {
        return v3((double)trq[id] * FRC_INV, (double)trq[n + id] * FRC_INV, (double)trq[2 * n + id] * FRC_INV);
    };
    V3 fh1 = v3(0, 0, 0), fo = v3(0, 0, 0), fh2 = v3(0, 0, 0);
    // H sites: u along H - O, v the lab x (or y) axis
    auto hsite = [&](V3 rh, V3 tau, V3 &fh) {
        V3 u = rh - ro;
        const double ul = len(u);
        V3 v = fabs(u.x / ul) > 0.8666 ? v3(0, 1, 0) : v3(1, 0, 0);
        V3 w = crs(u, v);
        const double wl = len(w);
        u = (1.0 / ul) * u;
        w = (1.0 / wl) * w;
        const V3 vxu = crs(v, u), wxu = crs(w, u);
        const double vxuL = len(vxu), wxuL = len(wxu);
        const V3 dUdu = (-dot(v, tau) / (vxuL * vxuL * ul)) * vxu + (-dot(w, tau) / (wxuL * wxuL * ul)) * wxu;
        fh = fh - dUdu;
        fo = fo + dUdu;
    };
    if (q == 0) hsite(rh1, tq(h1), fh1);
    if (q == 1) {   // O site: u = O - H1, v = O - H2, half weight on the w rotation
        const V3 tau = tq(o);
        V3 u = ro - rh1, v = ro - rh2;
        V3 w = crs(u, v);
        const double ul = len(u), vl = len(v), wl = len(w);
        u = (1.0 / ul) * u;
        v = (1.0 / vl) * v;
        w = (1.0 / wl) * w;
        const V3 vxu = crs(v, u), wxu = crs(w, u), wxv = crs(w, v);
        const double vxuL = len(vxu), wxuL = len(wxu), wxvL = len(wxv);
        const V3 dUdu = (-dot(v, tau) / (vxuL * vxuL * ul)) * vxu + (0.5 * -dot(w, tau) / (wxuL * wxuL * ul)) * wxu;
        const V3 dUdv = (-dot(u, tau) / (vxuL * vxuL * vl)) * (-vxu) + (0.5 * -dot(w, tau) / (wxvL * wxvL * vl)) * wxv;
        fo = fo - dUdu - dUdv;
        fh1 = fh1 + dUdu;
        fh2 = fh2 + dUdv;
    }
    if (q == 2) hsite(rh2, tq(h2), fh2);
    if (q != 2) add_fix3_at(frc, n, h1, fh1, 1.0);
    add_fix3_at(frc, n, o, fo, 1.0);
    if (q != 0) add_fix3_at(frc, n, h2, fh2, 1.0);
}

void launch_torques_end(Ctx &c) {
    k_torque2force<<<(3 * c.nmol + 95) / 96, 96, 0, c.stream>>>(c.nmol, c.n, c.mol_off, c.mol_atoms,
                                                                c.pos4, c.trq, c.frc);
}

// real space + self + intramolecular (Multipole::compute)
void launch_mp_short(Ctx &c) {
    MPArgs a;
    a.n = c.n; a.nbr = c.pl.nbr; a.nnbr = c.pl.nnbr; a.pos4 = c.pos4; a.mu = c.mu; a.qd = c.qd;
    a.tq = c.type_q; a.box = c.box; a.alpha = c.ew_alpha; a.rc2 = c.mp_rc2;
    a.frc = c.frc; a.trq = c.trq; a.acc = c.acc;
    const int tpp = 8;
    // 128-thread blocks: at this kernel's register count the SM holds more
    // warps in small blocks than in one 256-thread block
    const int nb = (int)(((long long)c.n * tpp + 127) / 128);
    const bool cubic = c.box.L[0] == c.box.L[1] && c.box.L[1] == c.box.L[2];
    if (c.precision == SMD_PREC_MIXED && cubic) {
        if (!c.fixq_from_integrate) launch_fixq(c);
        a.fixq = c.fixq;
        a.srec = c.srec;
        for (int d = 0; d < 3; d++) a.dscale[d] = c.box.L[d] / 4294967296.0;
        k_mp_real_f<tpp><<<nb, 128, 0, c.stream>>>(a);
    } else {
        k_mp_real<tpp><<<nb, 128, 0, c.stream>>>(a);
    }
    launch_mp_mol(c);
    launch_intra_flex(c, true, false);   // flexible molecules: the correction's forces and torques
}

// the FP64 real-space pair pass alone (the volume derivative of
// Multipole::real_term takes its virial and torques on their own)
void launch_mp_real_only(Ctx &c) {
    MPArgs a;
    a.n = c.n; a.nbr = c.pl.nbr; a.nnbr = c.pl.nnbr; a.pos4 = c.pos4; a.mu = c.mu; a.qd = c.qd;
    a.tq = c.type_q; a.box = c.box; a.alpha = c.ew_alpha; a.rc2 = c.mp_rc2;
    a.frc = c.frc; a.trq = c.trq; a.acc = c.acc;
    k_mp_real<8><<<(int)(((long long)c.n * 8 + 127) / 128), 128, 0, c.stream>>>(a);
}

// self energy and intramolecular correction of the multipoles
void launch_mp_mol(Ctx &c) {
    k_mp_mol<<<(c.nmol + 127) / 128, 128, 0, c.stream>>>(c.nmol, c.n, c.mol_off, c.mol_atoms, c.excl_off,
                                                         c.excl, c.pos4, c.type_q, c.mu, c.qd, c.box,
                                                         c.ew_alpha, c.acc);
}

}  // namespace smd
