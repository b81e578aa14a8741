// Short-range pair kernel: LJ / Mie n-m / Born-Mayer-Huggins fused with the
// Ewald real-space term, over the full Verlet list.
//
// Reference terms (per pair inside the cutoff, r_ij = r_j - r_i, f_i += f_ij):
//   LJ   LJForce::compute (src/forces/LJForce.cpp:92-229): skips same-molecule
//        pairs, U = 4eps (sr12 - sr6) minus U(rc) when switchOn, force unshifted,
//        cutoff test on r*r <= rc^2 with r = |r_ij|.
//   MIE  MieForce::compute (src/forces/MieForce.cpp:89-196): Cn eps (s^n - s^m),
//        5th-order switch between switchDist and the cutoff.
//   BMH  A exp(-r/rho) - C r^-6 - D r^-8 with the same switch (no reference
//        code for this form; structure of BuckinghamForce.cpp:150-182).
//   real EwaldForce::real_term (src/forces/EwaldForce.cpp:296-527):
//        q_i q_j erfc(a r)/r for r^2 < realCut^2, all listed pairs.
//
// Layout: TPP consecutive threads own one site i and split its list row;
// their partial forces are combined with shuffles in a fixed tree, so the
// result does not depend on scheduling.  The list holds each pair twice, so
// the energy and virial sums are halved.  Energies and the virial go to
// 64-bit fixed-point accumulators (one atomic per block and slot); forces
// are written as fixed point by the owner threads.
//
// Two arithmetic paths:
//   double: positions from pos4 (FP64), minimum image as Ensemble::apply_pbc.
//   float : positions from fixq (32-bit box fractions); the minimum-image
//           displacement is an exact integer difference and r^2 an exact
//           64-bit integer sum (cubic box), so the only roundings are the
//           FP32 pair arithmetic itself.
#include "smd_ctx.cuh"

namespace smd {

struct PairArgs {
    int n, max_nbr, ntypes;
    const int *nbr, *nnbr;
    const double4 *pos4;
    const int4 *fixq;
    Box box;
    int cubic;
    double r2scale;     // (L/2^32)^2, cubic boxes
    float dscale[3];    // L/2^32 per axis
    const double *par;  // [ntypes^2][4]
    const double *type_q;
    double vdw_rc2;
    int switch_on;
    double sw_rs2, sw_c1, sw_c2, sw_c3;
    double alpha, alpha2, alpha2pi, ew_rc2;
    // buffered 14-7 (BuffvdWForce): exponents, buffers, taper
    double bn, bm, bdelta, bgamma, bc[6], bsw2;
    float bswf, bwinv;  // taper start and 1/(cutoff - start), FP32 path
    int buff_int;       // n - m and m are small positive integers
    const double *le;   // Lees-Edwards offset on the device (planar shear), or null
    const Box *dbox;    // the box on the device (barostat, FP64 path), or null: box
    // Wolf summation (WolfForce::real_term): the charge term's energy and
    // force shifts at the cutoff (0 for Ewald)
    double wolf_e, wolf_f;
    int second;         // a pass after another pair pass: add forces, count no pairs
    const double *saap; // SAAP a0..a5 per type pair
    long long *frc;
    long long *acc;
};

constexpr int PAIR_BLOCK = 256;
constexpr int MAX_TYPES = 8;

template <typename R, int VDW>
__device__ __forceinline__ void vdw_pair(R r2, R &e, R &fs, const R *p, const PairArgs &a,
                                         bool same) {
    // fs: scalar with f_ij = -fs * r_ij
    e = R(0);
    fs = R(0);
    if (VDW == VDW_NONE || same) return;
    if (VDW == VDW_BUFF) {
        // BuffvdWForce::compute (src/forces/BuffvdWForce.cpp:186-240):
        // U = eps ((1+d)/(rho+d))^(n-m) ((1+g)/(rho^m+g) - 2), rho = r/sigma,
        // 5th-order taper in r beyond the switch distance
        const R r = sqrt(r2);
        const R rr = r * r;
        if (!(rr <= R(a.vdw_rc2)) || p[1] == R(0)) return;
        const R inv_s = R(1) / p[0];
        const R rho = r * inv_s;
        const R rho_m = pow(rho, R(a.bm)), rho_m1 = pow(rho, R(a.bm) - R(1));
        const R nm = R(a.bn) - R(a.bm);
        const R par1 = (R(1) + R(a.bdelta)) / (rho + R(a.bdelta));
        const R par2 = (R(1) + R(a.bgamma)) / (rho_m + R(a.bgamma));
        const R par1_nm = pow(par1, nm);
        R tmpE = p[1] * par1_nm * (par2 - R(2));
        R tmpf = -p[1] * nm * par1_nm * (par2 - R(2)) * inv_s / (rho + R(a.bdelta)) -
                 p[1] * par1_nm * par2 * R(a.bm) * rho_m1 * inv_s / (rho_m + R(a.bgamma));
        if (a.switch_on && rr > R(a.bsw2)) {
            const R r3 = rr * r, r4 = rr * rr, r5 = rr * r3;
            const R sv = R(a.bc[5]) * r5 + R(a.bc[4]) * r4 + R(a.bc[3]) * r3 + R(a.bc[2]) * rr +
                         R(a.bc[1]) * r + R(a.bc[0]);
            const R dsv = R(5) * R(a.bc[5]) * r4 + R(4) * R(a.bc[4]) * r3 + R(3) * R(a.bc[3]) * rr +
                          R(2) * R(a.bc[2]) * r + R(a.bc[1]);
            tmpf = tmpf * sv + tmpE * dsv;
            tmpE *= sv;
        }
        // the reference's f_ij = -tmpf (r_i - r_j)/r = -fs (r_j - r_i)
        e = tmpE;
        fs = -tmpf / r;
        return;
    }
    if (VDW == VDW_LJ) {
        R r = sqrt(r2);
        R rr = r * r;
        if (rr <= R(a.vdw_rc2)) {
            R r_1 = R(1) / r;
            R rij_2 = r_1 * r_1;
            R sr2 = p[0] * rij_2;
            R sr6 = sr2 * sr2 * sr2;
            R sr12 = sr6 * sr6;
            e = p[1] * (sr12 - sr6);
            fs = (sr12 + sr12 - sr6) * R(6) * p[1] * rij_2;
            if (a.switch_on) e -= p[2];
        }
    } else {
        R r = sqrt(r2);
        R rr = r * r;
        if (rr <= R(a.vdw_rc2)) {
            R r_1 = R(1) / r;
            R rij_2 = r_1 * r_1;
            if (VDW == VDW_MIE) {
                R s = p[0] * r_1;
                R srn = pow(s, p[2]);
                R srm = pow(s, p[3]);
                e = p[1] * (srn - srm);
                fs = p[1] * (p[2] * srn - p[3] * srm) * rij_2;
            } else {  // BMH
                R ex = p[0] * exp(-r * p[1]);
                R r6 = rij_2 * rij_2 * rij_2;
                R r8 = r6 * rij_2;
                e = ex - p[2] * r6 - p[3] * r8;
                fs = ex * p[1] * r_1 - R(6) * p[2] * r8 - R(8) * p[3] * r8 * rij_2;
            }
            if (a.switch_on && rr > R(a.sw_rs2)) {
                R c = R(a.vdw_rc2) - rr;
                R c4 = c * (R(2) * rr + R(a.sw_c2));
                R sv = c * c4 * R(a.sw_c1);
                R dsv = R(a.sw_c3) * (c * c - c4);
                fs = fs * sv - e * dsv;
                e *= sv;
            }
        }
    }
}

// SAAPForce::compute (src/forces/SAAPForce.cpp:140-200): with N = a0 e^(a1 r)/r
// + a2 e^(a3 r) + a4 and D = 1 + a5 r^6, U = N/D and the reference's tmpf =
// U'/r; it takes r_ij = r_i - r_j, so in this kernel's convention (f_ij =
// -fs (r_j - r_i)) fs = -tmpf, and its switch, tmpf s - U ds, becomes
// fs s + U ds.
template <typename R>
__device__ __forceinline__ void saap_pair(R r2, R &e, R &fs, const double *q, const PairArgs &a, bool same) {
    e = R(0);
    fs = R(0);
    if (same || !(r2 <= R(a.vdw_rc2))) return;
    const R a0 = R(q[0]), a1 = R(q[1]), a2 = R(q[2]), a3 = R(q[3]), a4 = R(q[4]), a5 = R(q[5]);
    const R r = sqrt(r2), r_1 = R(1) / r, rij_2 = r_1 * r_1;
    const R ex1 = exp(a1 * r), ex3 = exp(a3 * r);
    const R num = a0 * r_1 * ex1 + a2 * ex3 + a4;
    const R den = R(1) + a5 * r2 * r2 * r2;
    e = num / den;
    const R tmpf = (-a0 * rij_2 * ex1 + a0 * a1 * r_1 * ex1 + a2 * a3 * ex3) * r_1 / den -
                   R(6) * a5 * r2 * r2 * num / (den * den);
    fs = -tmpf;
    if (a.switch_on && r2 > R(a.sw_rs2)) {
        const R c = R(a.vdw_rc2) - r2;
        const R c4 = c * (R(2) * r2 + R(a.sw_c2));
        const R sv = c * c4 * R(a.sw_c1);
        const R dsv = R(a.sw_c3) * (c * c - c4);
        fs = fs * sv + e * dsv;
        e *= sv;
    }
}

// FP32 LJ with the rounding of r^2 and of 1/r^2 corrected to first order:
// r2f is r^2 rounded to float, dr2 = (r^2 - r2f)/r2f from the exact integer
// r^2.  With ir2 = 1/r2f (rounded) the true 1/r^2 = ir2 (1 + eps) with
// eps = (1 - r2f ir2) - dr2 (the first term exact by FMA); the r^-14 and
// r^-8 force terms and the r^-12 / r^-6 energy terms then take the factors
// (1 + 7 eps), (1 + 4 eps), (1 + 6 eps), (1 + 3 eps).  Without it the
// seven-fold amplification of the two roundings dominates the FP32 error.
__device__ __forceinline__ void lj_pair_f(float r2f, float dr2, float &e, float &fs,
                                          const float *p, const PairArgs &a, bool same) {
    e = 0.f;
    fs = 0.f;
    if (same || !(r2f <= (float)a.vdw_rc2)) return;
    const float ir2 = __frcp_rn(r2f);
    const float eps = fmaf(-r2f, ir2, 1.0f) - dr2;
    const float sr2 = p[0] * ir2;
    const float sr6 = sr2 * sr2 * sr2;
    const float sr12 = sr6 * sr6;
    const float t1 = 12.f * p[1] * sr12 * ir2;
    const float t2 = 6.f * p[1] * sr6 * ir2;
    fs = (t1 - t2) + eps * (7.f * t1 - 4.f * t2);
    e = p[1] * (sr12 - sr6) + eps * (p[1] * (6.f * sr12 - 3.f * sr6));
    if (a.switch_on) e -= p[2];
}

// FP32 Mie n-m and Born-Mayer-Huggins with the same first-order correction
// of the rounding of r^2, 1/r^2 and the power/exponent bases (eps as in
// lj_pair_f): s^n = b^(n/2) with b = sigma^2/r^2, and exp(-r/rho) whose
// argument error is amplified by r/rho (about 10 for NaCl).
template <int VDW>
__device__ __forceinline__ void vdw_pair_f(float r2f, float dr2, float &e, float &fs,
                                           const float *p, const PairArgs &a, bool same) {
    e = 0.f;
    fs = 0.f;
    if (same || !(r2f <= (float)a.vdw_rc2)) return;
    const float ir2 = __frcp_rn(r2f);
    const float eps = fmaf(-r2f, ir2, 1.0f) - dr2;   // 1/r^2 = ir2 (1 + eps)
    if (VDW == VDW_MIE) {
        const float s2 = p[0] * p[0];
        const float b = s2 * ir2;
        const float db = fmaf(s2, ir2, -b) / b + eps;  // b_exact = b (1 + db)
        const float hn = 0.5f * p[2], hm = 0.5f * p[3];
        const float srn = powf(b, hn), srm = powf(b, hm);
        const float cn = 1.f + hn * db, cm = 1.f + hm * db;
        e = p[1] * (srn * cn - srm * cm);
        fs = p[1] * (p[2] * srn * cn - p[3] * srm * cm) * ir2 * (1.f + eps);
    } else {
        // r = sqrt(r^2) with the rounding of the root and of r^2 corrected
        const float r = sqrtf(r2f);
        const float dr = 0.5f * (fmaf(-r, r, r2f) / r2f + dr2);   // r_exact = r (1 + dr)
        const float x = r * p[1];
        const float dx = fmaf(r, p[1], -x) + x * dr;              // x_exact = x + dx
        const float ex = p[0] * expf(-x) * (1.f - dx);
        const float r6 = ir2 * ir2 * ir2, r8 = r6 * ir2;
        const float c6 = 1.f + 3.f * eps, c8 = 1.f + 4.f * eps, c10 = 1.f + 5.f * eps;
        e = ex - p[2] * r6 * c6 - p[3] * r8 * c8;
        fs = ex * p[1] * (1.f - dr) / r - 6.f * p[2] * r8 * c8 - 8.f * p[3] * r8 * ir2 * c10;
    }
    const float rr = r2f;
    if (a.switch_on && rr > (float)a.sw_rs2) {
        const float c = (float)a.vdw_rc2 - rr;
        const float c4 = c * (2.f * rr + (float)a.sw_c2);
        const float sv = c * c4 * (float)a.sw_c1;
        const float dsv = (float)a.sw_c3 * (c * c - c4);
        fs = fs * sv - e * dsv;
        e *= sv;
    }
}

// FP32 value with its first-order relative error: true value ~ v (1 + d).
// Every rounding of the buffered 14-7 chain is recovered exactly (FMA
// product/division remainders, two-sum) and carried in d, so the n-m and m
// fold powers do not amplify the roundings of r, rho + delta and the two
// quotients; what is left is a few final roundings per pair.
struct FE {
    float v, d;
};
__device__ __forceinline__ float fe_rel(float err, float v) { return v != 0.f ? __fdividef(err, v) : 0.f; }
__device__ __forceinline__ FE fe_mul(FE a, FE b) {
    const float v = a.v * b.v;
    return {v, a.d + b.d + fe_rel(fmaf(a.v, b.v, -v), v)};
}
__device__ __forceinline__ FE fe_div(FE a, FE b) {
    const float v = __fdiv_rn(a.v, b.v);
    const float rem = fmaf(-v, b.v, a.v);   // exact: a - v b
    return {v, a.d - b.d + fe_rel(rem, a.v)};
}
__device__ __forceinline__ FE fe_add(FE a, FE b) {
    const float s = a.v + b.v;
    const float bb = s - a.v;
    const float err = (a.v - (s - bb)) + (b.v - bb);
    return {s, fe_rel(err + a.v * a.d + b.v * b.d, s)};
}
__device__ __forceinline__ FE fe_pow(FE x, int k) {
    FE r = {1.f, 0.f};
    bool first = true;
    while (k > 0) {
        if (k & 1) {
            r = first ? x : fe_mul(r, x);
            first = false;
        }
        k >>= 1;
        if (k) x = fe_mul(x, x);
    }
    return r;
}
__device__ __forceinline__ FE fe_of(double x) {
    const float v = (float)x;
    return {v, v != 0.f ? (float)((x - (double)v) / (double)v) : 0.f};
}
__device__ __forceinline__ float fe_val(FE a) { return fmaf(a.v, a.d, a.v); }

struct BuffF {
    FE delta, gamma, c1, c2;
    int nm, m;
};

// FP32 buffered 14-7 between virtual sites for integer exponents (the same
// formula as vdw_pair<VDW_BUFF>).  tp = (1/sigma, its relative rounding,
// eps, its relative rounding).  The taper is evaluated in its equivalent
// well-conditioned form S = (1-t)^3 (1 + 3t + 6t^2), t = (r - rs)/(rc - rs),
// which the reference's monomial coefficients c0..c5 expand.
__device__ __forceinline__ void buff_pair_f(float r2f, float dr2, float &e, float &fs, float4 tp,
                                            const BuffF &b, const PairArgs &a, bool same) {
    e = 0.f;
    fs = 0.f;
    if (same || !(r2f <= (float)a.vdw_rc2) || tp.z == 0.f) return;
    const float r = sqrtf(r2f);
    const float dr = 0.5f * (fmaf(-r, r, r2f) / r2f + dr2);   // r_exact = r (1 + dr)
    const FE IS = {tp.x, tp.y}, EPS = {tp.z, tp.w};
    const FE rho = fe_mul(FE{r, dr}, IS);
    const FE sd = fe_add(rho, b.delta);
    const FE P1n = fe_pow(fe_div(b.c1, sd), b.nm);
    const FE rm1 = fe_pow(rho, b.m - 1);
    const FE dm = fe_add(fe_mul(rm1, rho), b.gamma);
    const FE P2 = fe_div(b.c2, dm);
    const FE EP = fe_mul(EPS, P1n);
    const FE E = fe_mul(EP, fe_add(P2, FE{-2.f, 0.f}));
    const FE t1 = fe_div(fe_mul(fe_mul(E, FE{(float)b.nm, 0.f}), IS), sd);
    const FE t2 = fe_div(fe_mul(fe_mul(fe_mul(EP, P2), FE{(float)b.m, 0.f}), fe_mul(rm1, IS)), dm);
    float en = fe_val(E);
    float tmpf = -(fe_val(t1) + fe_val(t2));
    if (a.switch_on && r2f > (float)a.bsw2) {
        const float t = fminf(1.f, fmaxf(0.f, (r - a.bswf) * a.bwinv));
        const float o = 1.f - t;
        const float sv = o * o * o * fmaf(6.f * t, t, fmaf(3.f, t, 1.f));
        const float dsv = -30.f * t * t * o * o * a.bwinv;
        tmpf = tmpf * sv + en * dsv;
        en *= sv;
    }
    e = en;
    fs = -tmpf / r * (1.f - dr);
}

template <typename R, int VDW, bool EWALD, int TPP>
__global__ void __launch_bounds__(PAIR_BLOCK) k_pair(PairArgs a) {
    __shared__ R s_par[MAX_TYPES * MAX_TYPES * 4];
    __shared__ R s_q[MAX_TYPES];
    __shared__ double s_red[PAIR_BLOCK / 32][11];
    constexpr bool BUFF_F = sizeof(R) == 4 && VDW == VDW_BUFF;
    __shared__ float4 s_bf[BUFF_F ? MAX_TYPES * MAX_TYPES : 1];
    const int nt2 = a.ntypes * a.ntypes;
    for (int k = threadIdx.x; k < nt2 * 4; k += blockDim.x) s_par[k] = R(a.par[k]);
    for (int k = threadIdx.x; k < a.ntypes; k += blockDim.x) s_q[k] = R(a.type_q[k]);
    BuffF bf{};
    if (BUFF_F) {
        for (int k = threadIdx.x; k < nt2; k += blockDim.x) {
            const FE is = fe_of(1.0 / a.par[k * 4 + 0]), ep = fe_of(a.par[k * 4 + 1]);
            s_bf[k] = make_float4(is.v, is.d, ep.v, ep.d);
        }
        bf.delta = fe_of(a.bdelta);
        bf.gamma = fe_of(a.bgamma);
        bf.c1 = fe_of(1.0 + a.bdelta);
        bf.c2 = fe_of(1.0 + a.bgamma);
        bf.nm = (int)(a.bn - a.bm);
        bf.m = (int)a.bm;
    }
    __syncthreads();

    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gt / TPP;
    const int t = gt % TPP;
    const Box box = a.dbox ? *a.dbox : a.box;
    const double le_d = a.le ? *a.le : 0.0;
    const unsigned le_f = a.le ? le_frac(le_d, box.inv[0]) : 0u;
    double fx = 0, fy = 0, fz = 0;
    R evdw = 0, ereal = 0;
    int npair = 0;
    R vxx = 0, vxy = 0, vxz = 0, vyy = 0, vyz = 0, vzz = 0;
    if (i < a.n) {
        const int cnt = a.nnbr[i];
        double4 pi64;
        int4 pif;
        int ti;
        if (sizeof(R) == 8) {
            pi64 = a.pos4[i];
            ti = (int)pi64.w;
        } else {
            pif = a.fixq[i];
            ti = pif.w;
        }
        const R qi = s_q[ti];
        for (int k = t; k < cnt; k += TPP) {
            const int raw = a.nbr[(size_t)k * a.n + i];
            const int j = raw & 0x7fffffff;
            const bool same = raw < 0;
            R dx, dy, dz, r2;
            float r2c = 0.f;
            int tj;
            if (sizeof(R) == 8) {
                const double4 pj = a.pos4[j];
                if (a.le) {
                    double ex = pj.x - pi64.x, ey = pj.y - pi64.y, ez = pj.z - pi64.z;
                    min_image_le(ex, ey, ez, box, le_d);
                    dx = ex; dy = ey; dz = ez;
                } else {
                    dx = pbc1(pj.x - pi64.x, box.L[0], box.half[0]);
                    dy = pbc1(pj.y - pi64.y, box.L[1], box.half[1]);
                    dz = pbc1(pj.z - pi64.z, box.L[2], box.half[2]);
                }
                r2 = dx * dx + dy * dy + dz * dz;
                tj = (int)pj.w;
            } else {
                const int4 pj = a.fixq[j];
                const int ix = a.le ? le_dx_frac(pif.x, pif.y, pj.x, pj.y, le_f) : pj.x - pif.x;
                const int iy = pj.y - pif.y, iz = pj.z - pif.z;
                dx = R(ix) * R(a.dscale[0]);
                dy = R(iy) * R(a.dscale[1]);
                dz = R(iz) * R(a.dscale[2]);
                float dr2 = 0.f;
                if (a.cubic) {
                    unsigned long long s2 = (unsigned long long)((long long)ix * ix) +
                                            (unsigned long long)((long long)iy * iy) +
                                            (unsigned long long)((long long)iz * iz);
                    const double r2d = (double)s2 * a.r2scale;
                    r2 = R(r2d);
                    dr2 = (float)((r2d - (double)r2) / r2d);
                } else {
                    r2 = dx * dx + dy * dy + dz * dz;
                }
                tj = pj.w;
                r2c = dr2;
            }
            R e, fs;
            if (sizeof(R) == 4 && VDW == VDW_LJ)
                lj_pair_f((float)r2, r2c, *(float *)&e, *(float *)&fs,
                          (const float *)&s_par[(ti * a.ntypes + tj) * 4], a, same);
            else if (BUFF_F && a.buff_int)
                buff_pair_f((float)r2, r2c, *(float *)&e, *(float *)&fs, s_bf[ti * a.ntypes + tj], bf, a, same);
            else if (sizeof(R) == 4 && (VDW == VDW_MIE || VDW == VDW_BMH))
                vdw_pair_f<VDW>((float)r2, r2c, *(float *)&e, *(float *)&fs,
                                (const float *)&s_par[(ti * a.ntypes + tj) * 4], a, same);
            else if (VDW == VDW_SAAP)
                saap_pair<R>(r2, e, fs, a.saap + (size_t)(ti * a.ntypes + tj) * 6, a, same);
            else
                vdw_pair<R, VDW>(r2, e, fs, &s_par[(ti * a.ntypes + tj) * 4], a, same);
            evdw += e;
            npair += (!a.second && (r2 <= R(a.vdw_rc2) || (EWALD && r2 < R(a.ew_rc2)))) ? 1 : 0;
            if (EWALD) {
                if (r2 < R(a.ew_rc2)) {
                    const R qij = qi * s_q[tj];
                    const R r = sqrt(r2);
                    const R ee = erfc(R(a.alpha) * r) / r;
                    const R ff = (ee + R(a.alpha2pi) * exp(-R(a.alpha2) * r2)) / r2;
                    ereal += qij * (ee - R(a.wolf_e));
                    fs += qij * (ff - R(a.wolf_f));
                }
            }
            const R fijx = -fs * dx, fijy = -fs * dy, fijz = -fs * dz;
            fx += (double)fijx;
            fy += (double)fijy;
            fz += (double)fijz;
            vxx += fijx * dx; vxy += fijy * dx; vxz += fijz * dx;
            vyy += fijy * dy; vyz += fijz * dy; vzz += fijz * dz;
        }
    }
    fx = group_sum<TPP>(fx);
    fy = group_sum<TPP>(fy);
    fz = group_sum<TPP>(fz);
    if (i < a.n && t == 0) {
        if (a.second) {   // this thread owns site i's entries: a plain add
            a.frc[i] += to_fix(fx, FRC_SCALE);
            a.frc[a.n + i] += to_fix(fy, FRC_SCALE);
            a.frc[2 * a.n + i] += to_fix(fz, FRC_SCALE);
        } else {
            a.frc[i] = to_fix(fx, FRC_SCALE);
            a.frc[a.n + i] = to_fix(fy, FRC_SCALE);
            a.frc[2 * a.n + i] = to_fix(fz, FRC_SCALE);
        }
    }
    // energies and virial: warp, then block, then one fixed-point atomic each
    double v[8] = {(double)evdw, (double)ereal, (double)vxx, (double)vxy,
                   (double)vxz,  (double)vyy,   (double)vyz, (double)vzz};
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    {
        int np = warp_sum(npair);
        if (lane == 0 && np) atomicAdd((unsigned long long *)&a.acc[ACC_NPAIR], (unsigned long long)np);
    }
#pragma unroll
    for (int q = 0; q < 8; q++) {
        double s = warp_sum(v[q]);
        if (lane == 0) s_red[w][q] = s;
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        double s = 0;
        for (int q = 0; q < PAIR_BLOCK / 32; q++) s += s_red[q][threadIdx.x];
        s *= 0.5;  // each pair appears twice in the full list
        // local virial convention of the reference (sum f_ij r_ij) has the
        // opposite sign of Ensemble::virial; store the Ensemble sign.
        int slot;
        switch (threadIdx.x) {
            case 0: slot = ACC_E_VDW; break;
            case 1: slot = ACC_E_REAL; break;
            case 2: slot = ACC_VIR + 0; break;
            case 3: slot = ACC_VIR + 1; break;
            case 4: slot = ACC_VIR + 2; break;
            case 5: slot = ACC_VIR + 4; break;
            case 6: slot = ACC_VIR + 5; break;
            default: slot = ACC_VIR + 8; break;
        }
        if (threadIdx.x >= 2) s = -s;
        if (s != 0.0) atomicAdd((unsigned long long *)&a.acc[slot],
                                (unsigned long long)to_fix(s, ACC_SCALE));
        // the virial of central pair forces is symmetric
        if (threadIdx.x == 3) atomicAdd((unsigned long long *)&a.acc[ACC_VIR + 3], (unsigned long long)to_fix(s, ACC_SCALE));
        if (threadIdx.x == 4) atomicAdd((unsigned long long *)&a.acc[ACC_VIR + 6], (unsigned long long)to_fix(s, ACC_SCALE));
        if (threadIdx.x == 6) atomicAdd((unsigned long long *)&a.acc[ACC_VIR + 7], (unsigned long long)to_fix(s, ACC_SCALE));
    }
}

// x^k for a small positive integer k: a fixed product chain when K is a
// compile-time constant, binary powering otherwise
template <int K>
__device__ __forceinline__ double ipow_d(double x, int k) {
    if (K == 7) {
        const double x2 = x * x, x4 = x2 * x2;
        return x4 * x2 * x;
    }
    if (K == 6) {
        const double x2 = x * x;
        return x2 * x2 * x2;
    }
    double r = 1.0;
    for (int q = 0; q < 7 && k > 0; q++) {
        if (k & 1) r *= x;
        k >>= 1;
        if (k) x *= x;
    }
    return r;
}

// Buffered 14-7 with small integer exponents (NM = n - m and M, 0 = taken
// at run time), the pair arithmetic in FP64 with the powers as products and
// the taper in its well-conditioned form S = (1-t)^3 (1 + 3t + 6t^2).
// FIXQ (mixed path): r^2 exact from the box fractions; every pair quantity
// carries FP64 rounding only, at a lower cost on B200 than the FP32 path's
// error-tracking arithmetic (buff_pair_f).  !FIXQ (FP64 path): r from the
// FP64 positions, minimum image as the reference's apply_pbc; the same
// arithmetic as the reference's pow() form to FP64 rounding.  Same list
// walk, accumulation and outputs as k_pair.
template <int TPP, int NM, int M, bool FIXQ = true>
__global__ void __launch_bounds__(PAIR_BLOCK) k_buff_d(PairArgs a) {
    __shared__ double s_is[MAX_TYPES * MAX_TYPES], s_ep[MAX_TYPES * MAX_TYPES];
    __shared__ double s_red[PAIR_BLOCK / 32][11];
    const int nt2 = a.ntypes * a.ntypes;
    for (int k = threadIdx.x; k < nt2; k += blockDim.x) {
        s_is[k] = 1.0 / a.par[k * 4 + 0];
        s_ep[k] = a.par[k * 4 + 1];
    }
    __syncthreads();
    const int nm = NM ? NM : (int)(a.bn - a.bm), mm = M ? M : (int)a.bm;
    const double c1 = 1.0 + a.bdelta, c2 = 1.0 + a.bgamma;
    const double rs = sqrt(a.bsw2), winv = 1.0 / (sqrt(a.vdw_rc2) - rs);
    const double ds0 = (double)a.box.L[0] / 4294967296.0, ds1 = (double)a.box.L[1] / 4294967296.0,
                 ds2 = (double)a.box.L[2] / 4294967296.0;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gt / TPP;
    const int t = gt % TPP;
    double fx = 0, fy = 0, fz = 0, evdw = 0;
    double vxx = 0, vxy = 0, vxz = 0, vyy = 0, vyz = 0, vzz = 0;
    int npair = 0;
    if (i < a.n) {
        const int cnt = a.nnbr[i];
        const int4 pif = FIXQ ? a.fixq[i] : make_int4(0, 0, 0, 0);
        const double4 pid = FIXQ ? make_double4(0, 0, 0, 0) : a.pos4[i];
        const int ti = FIXQ ? pif.w : (int)pid.w;
        for (int k = t; k < cnt; k += TPP) {
            const int raw = a.nbr[(size_t)k * a.n + i];
            const int j = raw & 0x7fffffff;
            double dx, dy, dz, r2;   // r_j - r_i
            int tj;
            if (FIXQ) {
                const int4 pj = a.fixq[j];
                const int ix = pj.x - pif.x, iy = pj.y - pif.y, iz = pj.z - pif.z;
                const unsigned long long s2 = (unsigned long long)((long long)ix * ix) +
                                              (unsigned long long)((long long)iy * iy) +
                                              (unsigned long long)((long long)iz * iz);
                r2 = (double)s2 * a.r2scale;
                dx = ix * ds0; dy = iy * ds1; dz = iz * ds2;
                tj = pj.w;
            } else {
                const double4 pj = a.pos4[j];
                dx = pbc1(pj.x - pid.x, a.box.L[0], a.box.half[0]);
                dy = pbc1(pj.y - pid.y, a.box.L[1], a.box.half[1]);
                dz = pbc1(pj.z - pid.z, a.box.L[2], a.box.half[2]);
                r2 = dx * dx + dy * dy + dz * dz;
                tj = (int)pj.w;
            }
            if (!(r2 <= a.vdw_rc2)) continue;
            npair++;
            const double ep = s_ep[ti * a.ntypes + tj];
            if (raw < 0 || ep == 0.0) continue;   // same molecule, or no well
            const double is = s_is[ti * a.ntypes + tj];
            const double ir = rsqrt(r2), r = r2 * ir;
            const double rho = r * is;
            const double rm1 = ipow_d<(M > 1 ? M - 1 : 0)>(rho, mm - 1);
            // both quotients from one division
            const double sd = rho + a.bdelta, dm = rm1 * rho + a.bgamma, inv = 1.0 / (sd * dm);
            const double t1 = dm * inv, t2 = sd * inv;
            const double p1n = ipow_d<NM>(c1 * t1, nm);
            const double p2 = c2 * t2;
            double en = ep * p1n * (p2 - 2.0);
            double tmpf = -(en * nm * is * t1 + ep * p1n * p2 * mm * rm1 * is * t2);
            if (a.switch_on && r2 > a.bsw2) {
                const double tt = fmin(1.0, fmax(0.0, (r - rs) * winv));
                const double o = 1.0 - tt;
                const double sv = o * o * o * (1.0 + tt * (3.0 + 6.0 * tt));
                const double dsv = -30.0 * tt * tt * o * o * winv;
                tmpf = tmpf * sv + en * dsv;
                en *= sv;
            }
            const double fs = -tmpf * ir;
            const double fijx = -fs * dx, fijy = -fs * dy, fijz = -fs * dz;
            fx += fijx; fy += fijy; fz += fijz;
            evdw += en;
            vxx += fijx * dx; vxy += fijy * dx; vxz += fijz * dx;
            vyy += fijy * dy; vyz += fijz * dy; vzz += fijz * dz;
        }
    }
    fx = group_sum<TPP>(fx);
    fy = group_sum<TPP>(fy);
    fz = group_sum<TPP>(fz);
    if (i < a.n && t == 0) {
        a.frc[i] = to_fix(fx, FRC_SCALE);
        a.frc[a.n + i] = to_fix(fy, FRC_SCALE);
        a.frc[2 * a.n + i] = to_fix(fz, FRC_SCALE);
    }
    double v[8] = {evdw, 0.0, vxx, vxy, vxz, vyy, vyz, vzz};
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    {
        int np = warp_sum(npair);
        if (lane == 0 && np) atomicAdd((unsigned long long *)&a.acc[ACC_NPAIR], (unsigned long long)np);
    }
#pragma unroll
    for (int q = 0; q < 8; q++) {
        double sv = warp_sum(v[q]);
        if (lane == 0) s_red[w][q] = sv;
    }
    __syncthreads();
    if (threadIdx.x < 8 && threadIdx.x != 1) {
        double sv = 0;
        for (int q = 0; q < PAIR_BLOCK / 32; q++) sv += s_red[q][threadIdx.x];
        sv *= 0.5;  // each pair appears twice in the full list
        const int slots[8] = {ACC_E_VDW, 0, ACC_VIR + 0, ACC_VIR + 1, ACC_VIR + 2, ACC_VIR + 4, ACC_VIR + 5, ACC_VIR + 8};
        if (threadIdx.x >= 2) sv = -sv;   // Ensemble::virial sign
        const long long fxv = to_fix(sv, ACC_SCALE);
        if (sv != 0.0) atomicAdd((unsigned long long *)&a.acc[slots[threadIdx.x]], (unsigned long long)fxv);
        // the virial of central pair forces is symmetric
        if (threadIdx.x == 3) atomicAdd((unsigned long long *)&a.acc[ACC_VIR + 3], (unsigned long long)fxv);
        if (threadIdx.x == 4) atomicAdd((unsigned long long *)&a.acc[ACC_VIR + 6], (unsigned long long)fxv);
        if (threadIdx.x == 6) atomicAdd((unsigned long long *)&a.acc[ACC_VIR + 7], (unsigned long long)fxv);
    }
}

template <typename R, int VDW, bool EWALD>
static void dispatch_tpp(Ctx &c, const PairArgs &a) {
    int tpp = c.tpp;
    long long threads = (long long)c.n * tpp;
    int nb = (int)((threads + PAIR_BLOCK - 1) / PAIR_BLOCK);
    switch (tpp) {
        case 1: k_pair<R, VDW, EWALD, 1><<<nb, PAIR_BLOCK, 0, c.stream>>>(a); break;
        case 2: k_pair<R, VDW, EWALD, 2><<<nb, PAIR_BLOCK, 0, c.stream>>>(a); break;
        case 4: k_pair<R, VDW, EWALD, 4><<<nb, PAIR_BLOCK, 0, c.stream>>>(a); break;
        case 8: k_pair<R, VDW, EWALD, 8><<<nb, PAIR_BLOCK, 0, c.stream>>>(a); break;
        case 16: k_pair<R, VDW, EWALD, 16><<<nb, PAIR_BLOCK, 0, c.stream>>>(a); break;
        default: k_pair<R, VDW, EWALD, 32><<<nb, PAIR_BLOCK, 0, c.stream>>>(a); break;
    }
}

template <typename R, bool EWALD>
static void dispatch_vdw(Ctx &c, const PairArgs &a) {
    switch (c.vdw) {
        case VDW_LJ: dispatch_tpp<R, VDW_LJ, EWALD>(c, a); break;
        case VDW_MIE: dispatch_tpp<R, VDW_MIE, EWALD>(c, a); break;
        case VDW_BMH: dispatch_tpp<R, VDW_BMH, EWALD>(c, a); break;
        case VDW_BUFF: dispatch_tpp<R, VDW_BUFF, EWALD>(c, a); break;
        case VDW_SAAP: dispatch_tpp<R, VDW_SAAP, EWALD>(c, a); break;
        default: dispatch_tpp<R, VDW_NONE, EWALD>(c, a); break;
    }
}

// Converts FP64 master positions to box fractions for the FP32 path (le:
// the Lees-Edwards offset on the device under shear, else null).
__global__ void k_fixq(int n, const double4 *pos4, int4 *fixq, Box b, const double *le) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    fixq[i] = site_frac(pos4[i], b, le != nullptr, le ? *le : 0.0);
}

// Charge sites of the Wolf summation (WolfForce::DummyPosition,
// src/forces/WolfForce.cpp:60-80): a flagged site (the O of a "WAT"
// molecule) carries its charge at r_2 + d (r_mid - r_2)/|r_mid - r_2|, with
// r_2 the molecule's second site, r_mid the midpoint of its first and third
// and d the reference's R_OP in nm; other sites stay.  The displacement is
// taken without minimum image, as the reference takes it.
__global__ void k_wolf_sites(int n, const int *mol, const int *mol_off, const int *mol_atoms, const int *msite,
                             const double4 *pos4, double d, double4 *vpos4) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 p = pos4[i];
    if (msite[i]) {
        const int s0 = mol_off[mol[i]];
        const double4 a = pos4[mol_atoms[s0]], o = pos4[mol_atoms[s0 + 1]], b = pos4[mol_atoms[s0 + 2]];
        const double rx = 0.5 * (b.x + a.x) - o.x, ry = 0.5 * (b.y + a.y) - o.y, rz = 0.5 * (b.z + a.z) - o.z;
        const double f = d / sqrt(rx * rx + ry * ry + rz * rz);
        p.x = o.x + f * rx; p.y = o.y + f * ry; p.z = o.z + f * rz;
    }
    vpos4[i] = p;
}

// the charge-site positions of the Wolf sum into c.wpos4 (every site; the
// displaced ones moved as above)
void launch_wolf_sites(Ctx &c) {
    k_wolf_sites<<<(c.n + 127) / 128, 128, 0, c.stream>>>(c.n, c.mol, c.mol_off, c.mol_atoms, c.wolf_msite,
                                                           c.pos4, c.wolf_d, c.wpos4);
}

// Virtual sites of the buffered 14-7 term (BuffvdWForce::VirtualPositions,
// src/forces/BuffvdWForce.cpp:358-385): a type-0 (H) site moves to
// f r_H + (1 - f) r_O, with O the molecule's second site; others stay.
__global__ void k_virtual(int n, const int *mol, const int *mol_off, const int *mol_atoms, const double4 *pos4,
                          double f, Box b, double4 *vpos4, int4 *vfixq) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int m = mol[i];
    const int s = mol_off[m], e = mol_off[m + 1];
    double4 p = pos4[i];
    if ((int)p.w == 0 && e - s > 1) {
        const double4 po = pos4[mol_atoms[s + 1]];
        p.x = f * p.x + (1.0 - f) * po.x;
        p.y = f * p.y + (1.0 - f) * po.y;
        p.z = f * p.z + (1.0 - f) * po.z;
    }
    vpos4[i] = p;
    vfixq[i] = make_int4(frac32(p.x, b.inv[0]), frac32(p.y, b.inv[1]), frac32(p.z, b.inv[2]), (int)p.w);
}

// Force on a virtual H site: f on H, (1 - f) on the molecule's O
// (BuffvdWForce.cpp:257-274).  Writes the sites' forces (first term), one
// thread per site: the O site also gathers the (1 - f) shares of its
// molecule's H sites, in site order.
__global__ void k_buff_distribute(int n, const int *mol, const int *mol_off, const int *mol_atoms,
                                  const double4 *pos4, double f, const long long *fv, long long *frc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int m = mol[i];
    const int s = mol_off[m], e = mol_off[m + 1];
    const bool multi = e - s > 1;
    const int o = mol_atoms[s + (multi ? 1 : 0)];
    long long out[3];
    if ((int)pos4[i].w == 0 && multi) {
        for (int d = 0; d < 3; d++) out[d] = to_fix(f * ((double)fv[d * n + i] * FRC_INV), FRC_SCALE);
    } else {
        for (int d = 0; d < 3; d++) out[d] = fv[d * n + i];
    }
    if (i == o) {
        double acc[3] = {0, 0, 0};
        if (multi)
            for (int k = s; k < e; k++) {
                const int j = mol_atoms[k];
                if ((int)pos4[j].w == 0)
                    for (int d = 0; d < 3; d++) acc[d] += (1.0 - f) * ((double)fv[d * n + j] * FRC_INV);
            }
        for (int d = 0; d < 3; d++) out[d] += to_fix(acc[d], FRC_SCALE);
    }
    for (int d = 0; d < 3; d++) frc[d * n + i] = out[d];
}

void launch_fixq(Ctx &c) {
    const double *le = c.ip.strain_rate != 0.0 && c.integrator_ready ? c.scal + SC_LE : nullptr;
    k_fixq<<<(c.n + 255) / 256, 256, 0, c.stream>>>(c.n, c.pos4, c.fixq, c.box, le);
}

// WolfForce::real_term's shifts: e(rc) = erfc(a rc)/rc and the force term
// (e(rc)/rc + 2a/sqrt(pi) exp(-a^2 rc^2)/rc)/rc, subtracted from every pair's
// energy and force factor
static void wolf_shifts(const Ctx &c, double &we, double &wf) {
    const double rc = c.wolf_rc, al = c.wolf_alpha;
    const double eR = erfc(al * rc) / rc;
    const double Rc = eR / rc + 2.0 * al / 1.7724538509055160273 * exp(-al * al * rc * rc) / rc;
    we = eR;
    wf = Rc / rc;
}

void launch_pair(Ctx &c) {
    PairArgs a;
    a.n = c.n; a.max_nbr = c.pl.max_nbr; a.ntypes = c.ntypes;
    a.nbr = c.pl.nbr; a.nnbr = c.pl.nnbr; a.pos4 = c.pos4; a.fixq = c.fixq;
    a.box = c.box;
    a.cubic = (c.box.L[0] == c.box.L[1] && c.box.L[1] == c.box.L[2]);
    double s = c.box.L[0] / 4294967296.0;
    a.r2scale = s * s;
    for (int d = 0; d < 3; d++) a.dscale[d] = (float)(c.box.L[d] / 4294967296.0);
    a.par = c.pair_par; a.type_q = c.type_q;
    a.vdw_rc2 = c.vdw_rc2; a.switch_on = c.switch_on;
    a.sw_rs2 = c.sw_rs2; a.sw_c1 = c.sw_c1; a.sw_c2 = c.sw_c2; a.sw_c3 = c.sw_c3;
    a.alpha = c.ew_alpha; a.alpha2 = c.ew_alpha * c.ew_alpha;
    a.alpha2pi = 2.0 * c.ew_alpha / 1.7724538509055160273;
    a.ew_rc2 = c.ew_rc2;
    a.frc = c.frc; a.acc = c.acc;
    a.le = c.ip.strain_rate != 0.0 && c.integrator_ready ? c.scal + SC_LE : nullptr;
    a.dbox = c.npt ? c.dbox : nullptr;
    a.wolf_e = a.wolf_f = 0.0;
    a.second = 0;
    a.saap = c.saap;
    // Wolf in the pair pass itself when every charge sits on its atom
    const bool wolf_here = c.wolf_on && !c.wolf_msites;
    if (wolf_here) {
        a.alpha = c.wolf_alpha; a.alpha2 = c.wolf_alpha * c.wolf_alpha;
        a.alpha2pi = 2.0 * c.wolf_alpha / 1.7724538509055160273;
        a.ew_rc2 = c.wolf_rc * c.wolf_rc;
        wolf_shifts(c, a.wolf_e, a.wolf_f);
    }
    const bool elec = c.ewald_on || wolf_here;
    a.bn = c.buff_n; a.bm = c.buff_m; a.bdelta = c.buff_delta; a.bgamma = c.buff_gamma;
    for (int q = 0; q < 6; q++) a.bc[q] = c.buff_c[q];
    a.bsw2 = c.buff_sw * c.buff_sw;
    a.bswf = (float)c.buff_sw;
    a.bwinv = (float)(1.0 / (sqrt(c.vdw_rc2) - c.buff_sw));
    {
        const double nm = c.buff_n - c.buff_m;
        a.buff_int = nm == floor(nm) && c.buff_m == floor(c.buff_m) && nm >= 1 && nm <= 64 && c.buff_m >= 1 &&
                     c.buff_m <= 64;
    }
    const bool buff = c.vdw == VDW_BUFF;
    if (buff) {
        // the pair term acts between the virtual sites; their forces are
        // handed to the real sites afterwards
        k_virtual<<<(c.n + 127) / 128, 128, 0, c.stream>>>(c.n, c.mol, c.mol_off, c.mol_atoms, c.pos4, c.buff_h,
                                                            c.box, c.vpos4, c.vfixq);
        a.pos4 = c.vpos4;
        a.fixq = c.vfixq;
        a.frc = c.fv;
    }
    if (c.precision == SMD_PREC_MIXED && buff && a.buff_int && a.cubic && !c.ewald_on && !a.le) {
        if (!c.fixq_from_integrate) launch_fixq(c);
        const int nb = (int)(((long long)c.n * 8 + PAIR_BLOCK - 1) / PAIR_BLOCK);
        if (c.buff_n - c.buff_m == 7 && c.buff_m == 7)
            k_buff_d<8, 7, 7><<<nb, PAIR_BLOCK, 0, c.stream>>>(a);
        else
            k_buff_d<8, 0, 0><<<nb, PAIR_BLOCK, 0, c.stream>>>(a);
    } else if (c.precision == SMD_PREC_MIXED) {
        if (!c.fixq_from_integrate) launch_fixq(c);
        if (elec) dispatch_vdw<float, true>(c, a);
        else dispatch_vdw<float, false>(c, a);
    } else if (buff && a.buff_int && !c.ewald_on && !a.le && !c.reference_forms) {
        // FP64 path, integer exponents: the same product-form pass on the
        // FP64 positions
        const int nb = (int)(((long long)c.n * 8 + PAIR_BLOCK - 1) / PAIR_BLOCK);
        if (c.buff_n - c.buff_m == 7 && c.buff_m == 7)
            k_buff_d<8, 7, 7, false><<<nb, PAIR_BLOCK, 0, c.stream>>>(a);
        else
            k_buff_d<8, 0, 0, false><<<nb, PAIR_BLOCK, 0, c.stream>>>(a);
    } else {
        if (elec) dispatch_vdw<double, true>(c, a);
        else dispatch_vdw<double, false>(c, a);
    }
    if (c.wolf_on && c.wolf_msites) {
        // charges on displaced sites: a second FP64 pass of the charge term
        // alone over the same list, on the charge sites' positions, adding
        // its forces to the atoms that own them (the reference applies a
        // displaced site's force to its atom unchanged)
        k_wolf_sites<<<(c.n + 127) / 128, 128, 0, c.stream>>>(c.n, c.mol, c.mol_off, c.mol_atoms, c.wolf_msite,
                                                               c.pos4, c.wolf_d, c.wpos4);
        PairArgs w = a;
        w.pos4 = c.wpos4;
        w.frc = c.frc;
        w.alpha = c.wolf_alpha; w.alpha2 = c.wolf_alpha * c.wolf_alpha;
        w.alpha2pi = 2.0 * c.wolf_alpha / 1.7724538509055160273;
        w.ew_rc2 = c.wolf_rc * c.wolf_rc;
        wolf_shifts(c, w.wolf_e, w.wolf_f);
        w.second = 1;
        dispatch_tpp<double, VDW_NONE, true>(c, w);
    }
    if (buff)
        k_buff_distribute<<<(c.n + 127) / 128, 128, 0, c.stream>>>(c.n, c.mol, c.mol_off, c.mol_atoms, c.pos4,
                                                                    c.buff_h, c.fv, c.frc);
}

}  // namespace smd
