// Reciprocal-space sums of the polarisable model (Multipole::reciprocal_term,
// src/forces/Multipole.cpp:951-1245; Induction::reciprocal_term,
// src/forces/Induction.cpp:1395-1710).
//
// Per k (half space, k^2 < kCut^2) and site i, with a = k.r_i:
//   structure factors  C_qQ + i S_qQ = sum (q_i - k.Q_i.k) e^{ia}
//                      C_m  + i S_m  = sum (mu_i.k) e^{ia}
//                      C_p  + i S_p  = sum (p_i.k) e^{ia}      (induced)
//   permanent energy   c [ |S_qQ|^2 + 2 (S_qQ C_m - C_qQ S_m) + |S_m|^2 ] * ke
//   induced energy     c [ S_qQ C_p - C_qQ S_p + C_p C_m + S_p S_m ] * ke
// with c = 4 pi/V exp(-k^2/4a^2)/k^2; forces and torques per site follow
// from the same sums (terms named after the reference's FqQ, FmiqQ, ...).
//
// The reference's permanent and induced force terms together are the force
// of the site's full multipole set (q, mu + p, Q) in the field of the full
// structure factor.  With U = C_qQ - S_m - S_p, W = S_qQ + C_m + C_p,
// A = sin(a) U - cos(a) W and B = cos(a) U + sin(a) W, one k contributes
//   force   2c k [ (q_i - k.Q_i.k) A + ((mu_i + p_i).k) B ]
//   torque  2c [ A (mu_i x k) - 2 B (k x Q_i k) ]
// (permanent terms alone: drop the p terms).
//
// Kernels: partial structure factors over (k tile x site chunk) blocks with
// each chunk's site data staged in shared memory; a fixed-order reduction
// over chunks giving S(k), the energies and the long virial; one per-site
// pass for forces and torques with the k data staged in shared memory.  In
// a time step all six sums come from one pass after the dipole solve and
// one force pass serves the permanent and induced terms.
//   FP64 path: a = k.r in FP64 as the reference computes it, FP64 arithmetic.
//   FP32 path: a is the exact 32-bit integer phase n.(box fractions), sine and
//   cosine from sincospif; the per-(site, k) arithmetic is FP32 with the
//   running sums moved into FP64 after every tile of 64-128 terms.
#include <vector>
#include "smd_ctx.cuh"
#include "smd_polar.cuh"

namespace smd {

constexpr double KE = 138.93548501;
constexpr double SQC_R = 11.78708976;
constexpr int MK_THREADS = 128;
constexpr int MK_CHUNKS = 16;
constexpr int FK_TILE = 256;
constexpr int F_TPS = 4;

// several blocks (k ranges) add into one site: integer atomics keep the sum
// independent of their order
__device__ __forceinline__ void add_fix3_atomic(long long *arr, int n, int i, V3 v, double s) {
    atomicAdd((unsigned long long *)&arr[i], (unsigned long long)to_fix(s * v.x, FRC_SCALE));
    atomicAdd((unsigned long long *)&arr[n + i], (unsigned long long)to_fix(s * v.y, FRC_SCALE));
    atomicAdd((unsigned long long *)&arr[2 * n + i], (unsigned long long)to_fix(s * v.z, FRC_SCALE));
}

// sin and cos of 2 pi ph / 2^32: the top 24 bits go through sincospif
// exactly, the low 8 bits as a first-order rotation
__device__ __forceinline__ void sincos_phase32(int ph, float &s, float &c) {
    const int hi = ph & ~0xff;
    const float b = (float)(ph & 0xff) * 1.4629180792671596e-09f;  // pi / 2^31
    float sh, ch;
    sincospif((float)hi * 4.656612873077393e-10f, &sh, &ch);
    s = fmaf(b, ch, sh);
    c = fmaf(-b, sh, ch);
}

// ---------------------------------------------------------------------------
// FP64 partial structure factors
// ---------------------------------------------------------------------------
struct SiteTile {
    double x[MK_THREADS], y[MK_THREADS], z[MK_THREADS];
    int ix[MK_THREADS], iy[MK_THREADS], iz[MK_THREADS];
    double v[13][MK_THREADS];
};

// MODE 0: permanent sums (slots 0-3); 1: induced sums (4-5); 2: all six.
// R = float takes the phase from the integer box fractions (used for the
// induced-only evaluation of the mixed path).
template <typename R, int MODE>
__global__ void __launch_bounds__(MK_THREADS) k_rsk_partial(int n, int nk, const double4 *pos4, const int4 *fixq,
                                                            const int *kn, const double *kvec, const double *tq,
                                                            const double *mu, const double *qd, const double *pind,
                                                            double *partial) {
    __shared__ SiteTile T;
    const int k = blockIdx.x * MK_THREADS + threadIdx.x;
    const int ch = blockIdx.y;
    const int per = (n + gridDim.y - 1) / gridDim.y;
    const int s0 = ch * per, s1 = min(n, s0 + per);
    double kx = 0, ky = 0, kz = 0;
    int nx = 0, ny = 0, nz = 0;
    if (k < nk) {
        kx = kvec[k]; ky = kvec[nk + k]; kz = kvec[2 * nk + k];
        nx = kn[k]; ny = kn[nk + k]; nz = kn[2 * nk + k];
    }
    // k.Q.k = Qxx kx^2 + Qyy ky^2 + Qzz kz^2 + 2 (Qxy kx ky + Qxz kx kz + Qyz ky kz)
    const double kk[6] = {kx * kx, 2 * kx * ky, 2 * kx * kz, ky * ky, 2 * ky * kz, kz * kz};
    constexpr bool PERM = MODE != 1, IND = MODE != 0;
    constexpr int PV = MODE == 1 ? 0 : 10;   // induced dipole slots in the tile
    double a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0;
    for (int base = s0; base < s1; base += MK_THREADS) {
        const int i = base + threadIdx.x;
        __syncthreads();
        if (i < s1) {
            if (sizeof(R) == 8) {
                const double4 p = pos4[i];
                T.x[threadIdx.x] = p.x; T.y[threadIdx.x] = p.y; T.z[threadIdx.x] = p.z;
            } else {
                const int4 f = fixq[i];
                T.ix[threadIdx.x] = f.x; T.iy[threadIdx.x] = f.y; T.iz[threadIdx.x] = f.z;
            }
            if (PERM) {
                T.v[0][threadIdx.x] = tq[(int)pos4[i].w] / SQC_R;
                for (int d = 0; d < 3; d++) T.v[1 + d][threadIdx.x] = mu[(size_t)d * n + i];
                for (int d = 0; d < 6; d++) T.v[4 + d][threadIdx.x] = qd[(size_t)d * n + i];
            }
            if (IND)
                for (int d = 0; d < 3; d++) T.v[PV + d][threadIdx.x] = pind[(size_t)d * n + i];
        }
        __syncthreads();
        const int cnt = min(MK_THREADS, s1 - base);
        if (k < nk) {
            for (int q = 0; q < cnt; q++) {
                double sn, cs;
                if (sizeof(R) == 8) {
                    sincos(T.x[q] * kx + T.y[q] * ky + T.z[q] * kz, &sn, &cs);
                } else {
                    const int ph = (int)((unsigned)nx * (unsigned)T.ix[q] + (unsigned)ny * (unsigned)T.iy[q] +
                                         (unsigned)nz * (unsigned)T.iz[q]);
                    float sf, cf;
                    sincos_phase32(ph, sf, cf);
                    sn = sf; cs = cf;
                }
                if (PERM) {
                    const double qk = T.v[0][q] - (T.v[4][q] * kk[0] + T.v[5][q] * kk[1] + T.v[6][q] * kk[2] +
                                                   T.v[7][q] * kk[3] + T.v[8][q] * kk[4] + T.v[9][q] * kk[5]);
                    const double mk = T.v[1][q] * kx + T.v[2][q] * ky + T.v[3][q] * kz;
                    a0 += qk * cs; a1 += qk * sn; a2 += mk * cs; a3 += mk * sn;
                }
                if (IND) {
                    const double pk = T.v[PV][q] * kx + T.v[PV + 1][q] * ky + T.v[PV + 2][q] * kz;
                    a4 += pk * cs; a5 += pk * sn;
                }
            }
        }
    }
    if (k < nk) {
        double *base = partial + (size_t)ch * 6 * nk;
        if (PERM) {
            base[k] = a0; base[nk + k] = a1; base[2 * (size_t)nk + k] = a2; base[3 * (size_t)nk + k] = a3;
        }
        if (IND) {
            base[4 * (size_t)nk + k] = a4; base[5 * (size_t)nk + k] = a5;
        }
    }
}

// ---------------------------------------------------------------------------
// FP32 partial structure factors (mixed path)
// ---------------------------------------------------------------------------
template <int MODE>
__global__ void __launch_bounds__(MK_THREADS) k_rsk_partial_f(int n, int nk, const double4 *pos4, const int4 *fixq,
                                                              const int *kn, const double *kvec, const double *tq,
                                                              const double *mu, const double *qd,
                                                              const double *pind, double *partial) {
    constexpr bool PERM = MODE != 1, IND = MODE != 0;
    constexpr int PV = MODE == 1 ? 0 : 10;
    constexpr int NV = MODE == 0 ? 10 : (MODE == 1 ? 3 : 13);
    __shared__ int s_i[3][MK_THREADS];
    __shared__ float s_v[NV][MK_THREADS];
    const int k = blockIdx.x * MK_THREADS + threadIdx.x;
    const int ch = blockIdx.y;
    const int per = (n + gridDim.y - 1) / gridDim.y;
    const int s0 = ch * per, s1 = min(n, s0 + per);
    float kx = 0.f, ky = 0.f, kz = 0.f;
    unsigned nx = 0, ny = 0, nz = 0;
    if (k < nk) {
        kx = (float)kvec[k]; ky = (float)kvec[nk + k]; kz = (float)kvec[2 * nk + k];
        nx = (unsigned)kn[k]; ny = (unsigned)kn[nk + k]; nz = (unsigned)kn[2 * nk + k];
    }
    const float kk[6] = {kx * kx, 2.f * kx * ky, 2.f * kx * kz, ky * ky, 2.f * ky * kz, kz * kz};
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int base = s0; base < s1; base += MK_THREADS) {
        const int i = base + threadIdx.x;
        __syncthreads();
        if (i < s1) {
            const int4 f = fixq[i];
            s_i[0][threadIdx.x] = f.x; s_i[1][threadIdx.x] = f.y; s_i[2][threadIdx.x] = f.z;
            if (PERM) {
                s_v[0][threadIdx.x] = (float)(tq[(int)pos4[i].w] / SQC_R);
                for (int d = 0; d < 3; d++) s_v[1 + d][threadIdx.x] = (float)mu[(size_t)d * n + i];
                for (int d = 0; d < 6; d++) s_v[4 + d][threadIdx.x] = (float)qd[(size_t)d * n + i];
            }
            if (IND)
                for (int d = 0; d < 3; d++) s_v[PV + d][threadIdx.x] = (float)pind[(size_t)d * n + i];
        }
        __syncthreads();
        const int cnt = min(MK_THREADS, s1 - base);
        if (k < nk) {
            float t0 = 0.f, t1 = 0.f, t2 = 0.f, t3 = 0.f, t4 = 0.f, t5 = 0.f;
#pragma unroll 4
            for (int q = 0; q < cnt; q++) {
                const int ph = (int)(nx * (unsigned)s_i[0][q] + ny * (unsigned)s_i[1][q] + nz * (unsigned)s_i[2][q]);
                float sn, cs;
                sincos_phase32(ph, sn, cs);
                if (PERM) {
                    float kqk = s_v[4][q] * kk[0];
                    kqk = fmaf(s_v[5][q], kk[1], kqk);
                    kqk = fmaf(s_v[6][q], kk[2], kqk);
                    kqk = fmaf(s_v[7][q], kk[3], kqk);
                    kqk = fmaf(s_v[8][q], kk[4], kqk);
                    kqk = fmaf(s_v[9][q], kk[5], kqk);
                    const float qk = s_v[0][q] - kqk;
                    const float mk = fmaf(s_v[1][q], kx, fmaf(s_v[2][q], ky, s_v[3][q] * kz));
                    t0 = fmaf(qk, cs, t0); t1 = fmaf(qk, sn, t1);
                    t2 = fmaf(mk, cs, t2); t3 = fmaf(mk, sn, t3);
                }
                if (IND) {
                    const float pk = fmaf(s_v[PV][q], kx, fmaf(s_v[PV + 1][q], ky, s_v[PV + 2][q] * kz));
                    t4 = fmaf(pk, cs, t4); t5 = fmaf(pk, sn, t5);
                }
            }
            acc[0] += t0; acc[1] += t1; acc[2] += t2; acc[3] += t3; acc[4] += t4; acc[5] += t5;
        }
    }
    if (k < nk) {
        double *base = partial + (size_t)ch * 6 * nk;
        if (PERM)
            for (int q = 0; q < 4; q++) base[(size_t)q * nk + k] = acc[q];
        if (IND)
            for (int q = 4; q < 6; q++) base[(size_t)q * nk + k] = acc[q];
    }
}

// ---------------------------------------------------------------------------
// fixed-order chunk sums; energies and long virial
// ---------------------------------------------------------------------------
// MODE 0 permanent, 1 induced, 2 both (permanent energy to slot_e, induced
// to slot_e2); slot_e < 0: sums only.  A block takes RR_K k with one thread
// per (structure factor, k); its first warp forms the energies and virial.
constexpr int RR_K = 32;
template <int MODE>
__global__ void __launch_bounds__(6 * RR_K) k_rsk_reduce(int nk, int nch, const double *partial,
                                                         const double *kcoef, const double *kvec, double alphaR4,
                                                         double *sk, long long *acc, int slot_e, int slot_e2) {
    __shared__ double s_s[6][RR_K];
    const int q0 = MODE == 1 ? 4 : 0, q1 = MODE == 0 ? 4 : 6;
    const int kl = threadIdx.x % RR_K, q = threadIdx.x / RR_K;
    const int k = blockIdx.x * RR_K + kl;
    // one thread per (structure factor, k): the chunk partials in a fixed order
    if (k < nk && q >= q0 && q < q1) {
        double t = 0;
        for (int ch = 0; ch < nch; ch++) t += partial[((size_t)ch * 6 + q) * nk + k];
        sk[(size_t)q * nk + k] = t;
        s_s[q][kl] = t;
    }
    if (slot_e < 0) return;  // sums only (no energy or virial from this call)
    __syncthreads();
    if (threadIdx.x >= RR_K) return;
    // the first warp: energy and virial of its k, then the block totals
    double ep = 0, ei = 0, vxx = 0, vxy = 0, vxz = 0, vyy = 0, vyz = 0, vzz = 0;
    if (k < nk) {
        const double CqQ = MODE != 1 ? s_s[0][kl] : 0.0, SqQ = MODE != 1 ? s_s[1][kl] : 0.0;
        const double Cm = MODE != 1 ? s_s[2][kl] : 0.0, Sm = MODE != 1 ? s_s[3][kl] : 0.0;
        const double c = kcoef[k];
        if (MODE != 1) ep = c * ((CqQ * CqQ + SqQ * SqQ) + 2 * (SqQ * Cm - CqQ * Sm) + (Cm * Cm + Sm * Sm)) * KE;
        if (MODE != 0) {
            // the induced energy needs the permanent sums too: read them back
            const double Cq = MODE == 1 ? sk[k] : CqQ, Sq = MODE == 1 ? sk[nk + k] : SqQ;
            const double C2 = MODE == 1 ? sk[2 * (size_t)nk + k] : Cm, S2 = MODE == 1 ? sk[3 * (size_t)nk + k] : Sm;
            const double Cp = s_s[4][kl], Sp = s_s[5][kl];
            ei = c * ((Sq * Cp - Cq * Sp) + (Cp * C2 + Sp * S2)) * KE;
        }
        const double e = ep + ei;
        const double kx = kvec[k], ky = kvec[nk + k], kz = kvec[2 * nk + k];
        const double k2 = kx * kx + ky * ky + kz * kz;
        const double coeff = 2.0 * (alphaR4 + 1.0 / k2);
        vxx = e - e * coeff * kx * kx; vyy = e - e * coeff * ky * ky; vzz = e - e * coeff * kz * kz;
        vxy = -e * coeff * kx * ky; vxz = -e * coeff * kx * kz; vyz = -e * coeff * ky * kz;
    }
    double v[8] = {ep + (MODE == 1 ? ei : 0.0), ei, vxx, vxy, vxz, vyy, vyz, vzz};
#pragma unroll
    for (int r = 0; r < 8; r++) v[r] = warp_sum(v[r]);
    const int lane = threadIdx.x;
    if (lane < 8) {
        if (lane == 1 && MODE != 2) return;
        double t = v[0];
#pragma unroll
        for (int r = 1; r < 8; r++)
            if (lane == r) t = v[r];
        const int slots[8][2] = {{slot_e, -1}, {slot_e2, -1}, {ACC_LVIR + 0, -1},
                                 {ACC_LVIR + 1, ACC_LVIR + 3}, {ACC_LVIR + 2, ACC_LVIR + 6},
                                 {ACC_LVIR + 4, -1}, {ACC_LVIR + 5, ACC_LVIR + 7}, {ACC_LVIR + 8, -1}};
        const long long fx = to_fix(t, ACC_SCALE);
        atomicAdd((unsigned long long *)&acc[slots[lane][0]], (unsigned long long)fx);
        if (slots[lane][1] >= 0) atomicAdd((unsigned long long *)&acc[slots[lane][1]], (unsigned long long)fx);
    }
}

// ---------------------------------------------------------------------------
// FP64 per-site forces and torques
// ---------------------------------------------------------------------------
// F_TPS threads split the k set, k data staged in shared memory.  PERM / IND
// select the permanent and induced terms.
template <typename R, bool PERM, bool IND>
__global__ void __launch_bounds__(256) k_rforce(int n, int nk, const double4 *pos4, const int4 *fixq,
                                                const int *kn, const double *kvec, const double *kcoef,
                                                const double *sk, const double *tq, const double *mu,
                                                const double *qd, const double *pind, long long *frc,
                                                long long *trq) {
    __shared__ double s_k[3][FK_TILE], s_b[FK_TILE], s_S[6][FK_TILE];
    __shared__ int s_n[3][FK_TILE];
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gt / F_TPS, t = gt % F_TPS;
    V3 f = v3(0, 0, 0), tau = v3(0, 0, 0);
    double4 p64 = make_double4(0, 0, 0, 0);
    int4 pf = make_int4(0, 0, 0, 0);
    double qi = 0;
    V3 mi = v3(0, 0, 0), pi_ = v3(0, 0, 0);
    Q6 Qi = {0, 0, 0, 0, 0, 0};
    if (i < n) {
        p64 = pos4[i];
        if (sizeof(R) == 4) pf = fixq[i];
        qi = tq[(int)p64.w] / SQC_R;
        mi = v3(mu[i], mu[n + i], mu[2 * n + i]);
        Qi = {qd[i], qd[n + i], qd[2 * n + i], qd[3 * n + i], qd[4 * n + i], qd[5 * n + i]};
        if (IND) pi_ = v3(pind[i], pind[n + i], pind[2 * n + i]);
    }
    const int kper = (((nk + gridDim.y - 1) / gridDim.y + FK_TILE - 1) / FK_TILE) * FK_TILE;
    const int kb0 = blockIdx.y * kper, kb1 = min(nk, kb0 + kper);
    for (int base = kb0; base < kb1; base += FK_TILE) {
        __syncthreads();
        const int kk = base + threadIdx.x;
        if (kk < kb1) {
            for (int d = 0; d < 3; d++) {
                s_k[d][threadIdx.x] = kvec[(size_t)d * nk + kk];
                s_n[d][threadIdx.x] = kn[(size_t)d * nk + kk];
            }
            s_b[threadIdx.x] = 2.0 * kcoef[kk];
            for (int d = 0; d < 6; d++)
                s_S[d][threadIdx.x] = (d < 4 || IND) ? sk[(size_t)d * nk + kk] : 0.0;
        }
        __syncthreads();
        const int cnt = min(FK_TILE, kb1 - base);
        if (i < n) {
            for (int q = t; q < cnt; q += F_TPS) {
                const V3 k = v3(s_k[0][q], s_k[1][q], s_k[2][q]);
                double sn, cs;
                if (sizeof(R) == 8) {
                    sincos(p64.x * k.x + p64.y * k.y + p64.z * k.z, &sn, &cs);
                } else {
                    const int ph = (int)((unsigned)s_n[0][q] * (unsigned)pf.x + (unsigned)s_n[1][q] * (unsigned)pf.y +
                                         (unsigned)s_n[2][q] * (unsigned)pf.z);
                    float sf, cf;
                    sincos_phase32(ph, sf, cf);
                    sn = sf; cs = cf;
                }
                const V3 Qk = qv(Qi, k);
                const double qk = qi - dot(k, Qk);
                const double c1 = qk * cs, s1 = qk * sn;
                const double mk = dot(mi, k), mkc = mk * cs, mks = mk * sn;
                const double b = s_b[q];
                const double CqQ = s_S[0][q], SqQ = s_S[1][q], Cm = s_S[2][q], Sm = s_S[3][q];
                const V3 kxm = crs(k, mi), KQ = crs(k, Qk);
                double val = 0;
                V3 tq_ = v3(0, 0, 0);
                if (PERM) {
                    val += (s1 * CqQ - c1 * SqQ) + (mkc * CqQ + mks * SqQ) - (c1 * Cm + s1 * Sm) + (mks * Cm - mkc * Sm);
                    tq_ = tq_ + ((SqQ * cs - CqQ * sn) + (Cm * cs + Sm * sn)) * kxm +
                          (-2.0 * (CqQ * cs + SqQ * sn) + 2.0 * (Sm * cs - Cm * sn)) * KQ;
                }
                if (IND) {
                    const double Cp = s_S[4][q], Sp = s_S[5][q];
                    const double pk = dot(pi_, k), pkc = pk * cs, pks = pk * sn;
                    val += (pkc * CqQ + pks * SqQ) - (c1 * Cp + s1 * Sp) + (pks * (Cm + Cp) - pkc * (Sm + Sp)) +
                           (mks * Cp - mkc * Sp);
                    tq_ = tq_ + (cs * Cp + sn * Sp) * kxm + (2.0 * (cs * Sp - sn * Cp)) * KQ;
                }
                f = f + (b * val) * k;
                tau = tau + b * tq_;
            }
        }
    }
    f.x = group_sum<F_TPS>(f.x); f.y = group_sum<F_TPS>(f.y); f.z = group_sum<F_TPS>(f.z);
    tau.x = group_sum<F_TPS>(tau.x); tau.y = group_sum<F_TPS>(tau.y); tau.z = group_sum<F_TPS>(tau.z);
    if (i < n && t == 0) {
        add_fix3_atomic(frc, n, i, f, KE);
        add_fix3_atomic(trq, n, i, tau, KE);
    }
}

// ---------------------------------------------------------------------------
// FP32 per-site forces and torques (mixed path): permanent terms, with the
// induced ones when IND (the combined form in the header)
// ---------------------------------------------------------------------------
template <bool IND>
__global__ void __launch_bounds__(256) k_rforce_f(int n, int nk, const double4 *pos4, const int4 *fixq,
                                                  const int *kn, const double *kvec, const double *kcoef,
                                                  const double *sk, const double *tq, const double *mu,
                                                  const double *qd, const double *pind, long long *frc,
                                                  long long *trq) {
    __shared__ float4 s_kb[FK_TILE];   // kx, ky, kz, 2c
    __shared__ float2 s_uw[FK_TILE];   // U, W
    __shared__ int4 s_n[FK_TILE];      // integer k
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gt / F_TPS, t = gt % F_TPS;
    int4 pf = make_int4(0, 0, 0, 0);
    float qi = 0.f, dx = 0.f, dy = 0.f, dz = 0.f;
    float Qxx = 0.f, Qxy = 0.f, Qxz = 0.f, Qyy = 0.f, Qyz = 0.f, Qzz = 0.f;
    if (i < n) {
        pf = fixq[i];
        qi = (float)(tq[(int)pos4[i].w] / SQC_R);
        double d3[3] = {mu[i], mu[n + i], mu[2 * n + i]};
        if (IND)
            for (int d = 0; d < 3; d++) d3[d] += pind[(size_t)d * n + i];
        dx = (float)d3[0]; dy = (float)d3[1]; dz = (float)d3[2];
        Qxx = (float)qd[i]; Qxy = (float)qd[n + i]; Qxz = (float)qd[2 * n + i];
        Qyy = (float)qd[3 * n + i]; Qyz = (float)qd[4 * n + i]; Qzz = (float)qd[5 * n + i];
    }
    double F[3] = {0, 0, 0}, EA[3] = {0, 0, 0}, GX[3] = {0, 0, 0};
    const int kper = (((nk + gridDim.y - 1) / gridDim.y + FK_TILE - 1) / FK_TILE) * FK_TILE;
    const int kb0 = blockIdx.y * kper, kb1 = min(nk, kb0 + kper);
    for (int base = kb0; base < kb1; base += FK_TILE) {
        __syncthreads();
        const int kk = base + threadIdx.x;
        if (kk < kb1) {
            const double CqQ = sk[kk], SqQ = sk[nk + kk], Cm = sk[2 * (size_t)nk + kk], Sm = sk[3 * (size_t)nk + kk];
            double U = CqQ - Sm, W = SqQ + Cm;
            if (IND) {
                U -= sk[5 * (size_t)nk + kk];
                W += sk[4 * (size_t)nk + kk];
            }
            s_kb[threadIdx.x] = make_float4((float)kvec[kk], (float)kvec[nk + kk], (float)kvec[2 * (size_t)nk + kk],
                                            (float)(2.0 * kcoef[kk]));
            s_uw[threadIdx.x] = make_float2((float)U, (float)W);
            s_n[threadIdx.x] = make_int4(kn[kk], kn[nk + kk], kn[2 * (size_t)nk + kk], 0);
        }
        __syncthreads();
        const int cnt = min(FK_TILE, kb1 - base);
        if (i < n) {
            float f0 = 0.f, f1 = 0.f, f2 = 0.f, e0 = 0.f, e1 = 0.f, e2 = 0.f, g0 = 0.f, g1 = 0.f, g2 = 0.f;
#pragma unroll 2
            for (int q = t; q < cnt; q += F_TPS) {
                const float4 kb = s_kb[q];
                const float2 uw = s_uw[q];
                const int4 nn = s_n[q];
                const int ph = (int)((unsigned)nn.x * (unsigned)pf.x + (unsigned)nn.y * (unsigned)pf.y +
                                     (unsigned)nn.z * (unsigned)pf.z);
                float sn, cs;
                sincos_phase32(ph, sn, cs);
                const float A = fmaf(sn, uw.x, -cs * uw.y);
                const float B = fmaf(cs, uw.x, sn * uw.y);
                const float qkx = fmaf(Qxx, kb.x, fmaf(Qxy, kb.y, Qxz * kb.z));
                const float qky = fmaf(Qxy, kb.x, fmaf(Qyy, kb.y, Qyz * kb.z));
                const float qkz = fmaf(Qxz, kb.x, fmaf(Qyz, kb.y, Qzz * kb.z));
                const float qk = qi - fmaf(kb.x, qkx, fmaf(kb.y, qky, kb.z * qkz));
                const float mk = fmaf(dx, kb.x, fmaf(dy, kb.y, dz * kb.z));
                const float bA = kb.w * A, bB = kb.w * B;
                const float al = fmaf(qk, bA, mk * bB);
                f0 = fmaf(al, kb.x, f0); f1 = fmaf(al, kb.y, f1); f2 = fmaf(al, kb.z, f2);
                e0 = fmaf(bA, kb.x, e0); e1 = fmaf(bA, kb.y, e1); e2 = fmaf(bA, kb.z, e2);
                // k x (Q k)
                g0 = fmaf(bB, fmaf(kb.y, qkz, -kb.z * qky), g0);
                g1 = fmaf(bB, fmaf(kb.z, qkx, -kb.x * qkz), g1);
                g2 = fmaf(bB, fmaf(kb.x, qky, -kb.y * qkx), g2);
            }
            F[0] += f0; F[1] += f1; F[2] += f2;
            EA[0] += e0; EA[1] += e1; EA[2] += e2;
            GX[0] += g0; GX[1] += g1; GX[2] += g2;
        }
    }
    for (int d = 0; d < 3; d++) {
        F[d] = group_sum<F_TPS>(F[d]);
        EA[d] = group_sum<F_TPS>(EA[d]);
        GX[d] = group_sum<F_TPS>(GX[d]);
    }
    if (i < n && t == 0) {
        // torque on the permanent multipoles: mu x EA - 2 GX
        const V3 m = v3(mu[i], mu[n + i], mu[2 * n + i]);
        const V3 ea = v3(EA[0], EA[1], EA[2]);
        const V3 tau = crs(m, ea) - 2.0 * v3(GX[0], GX[1], GX[2]);
        add_fix3_atomic(frc, n, i, v3(F[0], F[1], F[2]), KE);
        add_fix3_atomic(trq, n, i, tau, KE);
    }
}

// ---------------------------------------------------------------------------
// FP32 passes of the mixed path
// ---------------------------------------------------------------------------
// The k list is stored column by column: nx, then ny, then nz ascending by
// one within a column.  The box is orthorhombic, so kx and ky are fixed
// within a column and every k-dependent weight is a polynomial in kz:
//   q - k.Q.k = a + kz (b + c kz),  a = q - Qxx kx^2 - 2 Qxy kx ky - Qyy ky^2,
//                                  b = -2 (Qxz kx + Qyz ky),  c = -Qzz
//   mu.k      = d + e kz,           d = mux kx + muy ky,  e = muz
// Every phase factor comes from exact integer phases (sincos_phase32) with
// at most two complex products after them.
//
// Site tables (one pass per evaluation): per site and axis the factors
// e^{2 pi i m f / 2^32}, m = 0 .. nmax; the site's q, mu, Q, p in FP32 come
// from the mixed path's site records.
//
// Sums pass: one thread per run of up to TS_SEG k of one column, sites
// staged in shared memory tile by tile.  Per site a run shares X[nx] Y[|ny|]
// and the column parts a, b, d of the weights; per k it takes Z[|nz|]
// (conjugated for negative components) and two FMAs per weight.
//
// Force pass: one thread per site walking whole columns.  The factor of a
// column's first k comes from its exact phase, the others are that times the
// site's e^{2 pi i m fz / 2^32}, m the offset in the column.  With U', W' the
// combined structure factors times 2c, A = sin U' - cos W' and
// B = cos U' + sin W', a column accumulates only sum A kz^j (j = 0..3) and
// sum B kz^j (j = 0..2); at its end these fold into the moments
//   M1_a = sum A k_a,  M2_ab = sum B k_a k_b,  M3_abc = sum A k_a k_b k_c
// (FP64 across column groups), which give at the end
//   force   F_a = q M1_a - Q_bc M3_abc + (mu + p)_b M2_ab
//   torque  mu x M1 - 2 g,  g_a = eps_abc (Q M2)_cb.
constexpr int TAB_MAX = 32;     // |n| < TAB_MAX
constexpr int TS_SEG = 4;       // k per run, sums pass
constexpr int CF_KGROUP = 128;  // k per column group at most, force pass
constexpr int CF_CGROUP = 64;   // columns per group at most

// The column passes in FP32 (mixed path) and FP64 (FP64 path).  FP32: the
// phases are exact 32-bit integer phases n.(box fractions) from fixq and go
// through sincos_phase32; running sums in FP32 within a tile or column group,
// FP64 across them.  FP64: the phases are exact 64-bit integer phases of the
// FP64 positions' 64-bit box fractions, sine and cosine from FP64 sincospi of
// the phase's top 53 bits (an angle error below 1e-15 rad, where the
// reference's k.r carries about 1e-14), all arithmetic FP64.  The FP64
// passes hold half as many sites per tile and per block, so that their
// tables fit shared memory with the same occupancy.
template <typename T> struct ColT;
template <> struct ColT<float> {
    using T2 = float2;
    using T4 = float4;
    static constexpr int SUM_THREADS = 128, SUM_SITES = 128, F_THREADS = 256;
};
template <> struct ColT<double> {
    using T2 = double2;
    using T4 = double4;
    static constexpr int SUM_THREADS = 128, SUM_SITES = 64, F_THREADS = 128;
};
__device__ __forceinline__ float tfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double tfma(double a, double b, double c) { return fma(a, b, c); }

// 64-bit box fraction of a coordinate: (x / L mod 1) 2^64
__device__ __forceinline__ unsigned long long frac64(double x, double invL) {
    double f = x * invL;
    f -= floor(f);
    return __double2ull_rn(f * 18446744073709551616.0);
}
// sin and cos of 2 pi ph / 2^64
__device__ __forceinline__ void sincos_phase64(unsigned long long ph, double &s, double &c) {
    sincospi((double)(long long)ph * 1.0842021724855044e-19, &s, &c);   // 2^-63
}

// a site's phase source: three 32-bit (FP32) or 64-bit (FP64) box fractions
template <typename T> struct SitePhase;
template <> struct SitePhase<float> {
    unsigned x, y, z;
    __device__ __forceinline__ SitePhase(const int4 *fixq, const double4 *, const Box &, int i) {
        const int4 f = fixq[i];
        x = (unsigned)f.x; y = (unsigned)f.y; z = (unsigned)f.z;
    }
    __device__ __forceinline__ SitePhase() : x(0), y(0), z(0) {}
    __device__ __forceinline__ unsigned ax(int a) const { return a == 0 ? x : (a == 1 ? y : z); }
    // e^{2 pi i (nx fx + ny fy + nz fz)}
    __device__ __forceinline__ void rot(int nx, int ny, int nz, float &sn, float &cs) const {
        sincos_phase32((int)((unsigned)nx * x + (unsigned)ny * y + (unsigned)nz * z), sn, cs);
    }
    __device__ __forceinline__ static float2 entry(int m, unsigned f) {
        float sn, cs;
        sincos_phase32((int)((unsigned)m * f), sn, cs);
        return make_float2(cs, sn);
    }
};
template <> struct SitePhase<double> {
    unsigned long long x, y, z;
    __device__ __forceinline__ SitePhase(const int4 *, const double4 *pos4, const Box &b, int i) {
        const double4 p = pos4[i];
        x = frac64(p.x, b.inv[0]); y = frac64(p.y, b.inv[1]); z = frac64(p.z, b.inv[2]);
    }
    __device__ __forceinline__ SitePhase() : x(0), y(0), z(0) {}
    __device__ __forceinline__ unsigned long long ax(int a) const { return a == 0 ? x : (a == 1 ? y : z); }
    __device__ __forceinline__ void rot(int nx, int ny, int nz, double &sn, double &cs) const {
        sincos_phase64((unsigned long long)(long long)nx * x + (unsigned long long)(long long)ny * y +
                           (unsigned long long)(long long)nz * z, sn, cs);
    }
    __device__ __forceinline__ static double2 entry(int m, unsigned long long f) {
        double sn, cs;
        sincos_phase64((unsigned long long)m * f, sn, cs);
        return make_double2(cs, sn);
    }
};

// site tables [n][row]: X[0..nt), Y[0..nt), Z[0..nt), zero padding to an
// even row
template <typename T>
__global__ void k_site_tab(int n, int nt, int row, const int4 *fixq, const double4 *pos4, Box box,
                           typename ColT<T>::T2 *stab) {
    using T2 = typename ColT<T>::T2;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)n * row) return;
    const int i = (int)(e / row), r = (int)(e - (long long)i * row);
    const int ax = r / nt, m = r - ax * nt;
    T2 v;
    v.x = 0; v.y = 0;
    if (ax < 3) {
        const SitePhase<T> f(fixq, pos4, box, i);
        v = SitePhase<T>::entry(m, f.ax(ax));
    }
    stab[e] = v;
}

// FP64 site records of the FP64 column passes, in the layout of the mixed
// path's FP32 records: (q, mu), (Qxx, Qxy, Qxz, Qyy), (Qyz, Qzz, px, py),
// (pz, 0, 0, 0)
__global__ void k_pack_srec_d(int n, const double4 *pos4, const double *tq, const double *mu, const double *qd,
                              const double *pind, double4 *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t N = (size_t)n;
    double4 *o = out + 4 * (size_t)i;
    o[0] = make_double4(tq[(int)pos4[i].w] / SQC_R, mu[i], mu[N + i], mu[2 * N + i]);
    o[1] = make_double4(qd[i], qd[N + i], qd[2 * N + i], qd[3 * N + i]);
    o[2] = make_double4(qd[4 * N + i], qd[5 * N + i], pind ? pind[i] : 0.0, pind ? pind[N + i] : 0.0);
    o[3] = make_double4(pind ? pind[2 * N + i] : 0.0, 0.0, 0.0, 0.0);
}

// MODE 0: permanent sums (slots 0-3); 1: induced sums (4-5); 2: all six.
// kseg[s] = (first k, count, nx | ny << 16, first nz)
template <typename T, int MODE, int SEG>
__global__ void __launch_bounds__(ColT<T>::SUM_THREADS) k_rsk_seg(int n, int nk, int nseg, int nt, int row,
                                                                  const int4 *kseg, const double *kvec,
                                                                  const typename ColT<T>::T2 *stab,
                                                                  const typename ColT<T>::T4 *ssv,
                                                                  double *partial) {
    using T2 = typename ColT<T>::T2;
    using T4 = typename ColT<T>::T4;
    constexpr int THREADS = ColT<T>::SUM_THREADS, SITES = ColT<T>::SUM_SITES;
    constexpr bool PERM = MODE != 1, IND = MODE != 0;
    extern __shared__ float4 s_dyn4[];
    T4 *s_v = (T4 *)s_dyn4;                          // [SITES][4]
    T2 *s_tab = (T2 *)(s_v + 4 * SITES);             // [SITES][row]
    const int sid = blockIdx.x * THREADS + threadIdx.x;
    const bool own = sid < nseg;
    const int ch = blockIdx.y;
    const int per = (n + gridDim.y - 1) / gridDim.y;
    const int s0 = ch * per, s1 = min(n, s0 + per);
    const int4 sg = own ? kseg[sid] : make_int4(0, 0, 0, 0);
    const int nx = (short)(sg.z & 0xffff), ny = sg.z >> 16;
    T kx = 0, ky = 0;
    if (own) {
        kx = (T)kvec[sg.x];
        ky = (T)kvec[nk + sg.x];
    }
    T kz[SEG], zsg[SEG];
    int oz[SEG];
#pragma unroll
    for (int j = 0; j < SEG; j++) {
        const bool v = j < sg.y;
        const int nz = sg.w + j;
        kz[j] = v ? (T)kvec[2 * (size_t)nk + sg.x + j] : (T)0;
        oz[j] = 2 * nt + (v ? (nz < 0 ? -nz : nz) : 0);
        zsg[j] = nz < 0 ? (T)-1 : (T)1;
    }
    const int ox = nx, oy = nt + (ny < 0 ? -ny : ny);
    const T ysg = ny < 0 ? (T)-1 : (T)1;
    const T kxx = kx * kx, kxy2 = (T)2 * kx * ky, kyy = ky * ky, kx2 = (T)2 * kx, ky2 = (T)2 * ky;
    double acc[SEG][6];
#pragma unroll
    for (int j = 0; j < SEG; j++)
#pragma unroll
        for (int q = 0; q < 6; q++) acc[j][q] = 0.0;
    for (int base = s0; base < s1; base += SITES) {
        const int cnt = min(SITES, s1 - base);
        __syncthreads();
        {
            // row is even, so every site's row starts on a 16-byte boundary
            // and a tile is a whole number of 16-byte units
            const float4 *src = (const float4 *)(stab + (size_t)base * row);
            float4 *dst = (float4 *)s_tab;
            const int nv = (int)((size_t)cnt * row * sizeof(T2) / sizeof(float4));
            for (int e = threadIdx.x; e < nv; e += THREADS) dst[e] = src[e];
            const T4 *sv = ssv + (size_t)base * 4;
            for (int e = threadIdx.x; e < cnt * 4; e += THREADS) s_v[e] = sv[e];
        }
        __syncthreads();
        T t[SEG][6];
#pragma unroll
        for (int j = 0; j < SEG; j++)
#pragma unroll
            for (int q = 0; q < 6; q++) t[j][q] = 0;
        const T2 *tp = s_tab;
        for (int q = 0; q < cnt; q++, tp += row) {
            const T2 X = tp[ox], Y = tp[oy];
            const T yi = Y.y * ysg;
            const T xr = tfma(X.x, Y.x, -X.y * yi), xi = tfma(X.x, yi, X.y * Y.x);
            T a = 0, b = 0, c = 0, d = 0, e = 0, pd = 0, pe = 0;
            if (PERM) {
                const T4 v0 = s_v[q * 4], v1 = s_v[q * 4 + 1], v2 = s_v[q * 4 + 2];
                a = v0.x - tfma(v1.x, kxx, tfma(v1.y, kxy2, v1.w * kyy));
                b = -tfma(v1.z, kx2, v2.x * ky2);
                c = -v2.y;
                d = tfma(v0.y, kx, v0.z * ky);
                e = v0.w;
            }
            if (IND) {
                const T4 v2 = s_v[q * 4 + 2], v3 = s_v[q * 4 + 3];
                pd = tfma(v2.z, kx, v2.w * ky);
                pe = v3.x;
            }
#pragma unroll
            for (int j = 0; j < SEG; j++) {
                const T2 Z = tp[oz[j]];
                const T zi = Z.y * zsg[j];
                const T cs = tfma(xr, Z.x, -xi * zi), sn = tfma(xr, zi, xi * Z.x);
                if (PERM) {
                    const T w = tfma(kz[j], tfma(c, kz[j], b), a);
                    const T m = tfma(e, kz[j], d);
                    t[j][0] = tfma(w, cs, t[j][0]); t[j][1] = tfma(w, sn, t[j][1]);
                    t[j][2] = tfma(m, cs, t[j][2]); t[j][3] = tfma(m, sn, t[j][3]);
                }
                if (IND) {
                    const T p = tfma(pe, kz[j], pd);
                    t[j][4] = tfma(p, cs, t[j][4]); t[j][5] = tfma(p, sn, t[j][5]);
                }
            }
        }
#pragma unroll
        for (int j = 0; j < SEG; j++)
#pragma unroll
            for (int q = 0; q < 6; q++) acc[j][q] += t[j][q];
    }
    if (own) {
        double *pb = partial + (size_t)ch * 6 * nk;
#pragma unroll
        for (int j = 0; j < SEG; j++) {
            if (j >= sg.y) break;
            const size_t k = (size_t)sg.x + j;
            if (PERM)
                for (int q = 0; q < 4; q++) pb[(size_t)q * nk + k] = acc[j][q];
            if (IND)
                for (int q = 4; q < 6; q++) pb[(size_t)q * nk + k] = acc[j][q];
        }
    }
}

// index of the symmetric pair (a, b) in xx xy xz yy yz zz and of the
// symmetric triple (a, b, c) in xxx xxy xxz xyy xyz xzz yyy yyz yzz zzz
__device__ __forceinline__ int sym2(int a, int b) {
    const int lo = a < b ? a : b, hi = a < b ? b : a;
    return lo == 0 ? hi : (lo == 1 ? 2 + hi : 5);
}
__device__ __forceinline__ int sym3(int a, int b, int c) {
    int x = a, y = b, z = c, t;
    if (x > y) { t = x; x = y; y = t; }
    if (y > z) { t = y; y = z; z = t; }
    if (x > y) { t = x; x = y; y = t; }
    return x == 0 ? sym2(y, z) : (x == 1 ? 5 + sym2(y, z) - 2 : 9);
}

// kgrp[g] = (first column, columns, first k, k count); kcol[c] = (first k,
// length, nx | ny << 16, first nz); kzr[k] = (kz, kz^2, 2c, 0)
template <typename T, bool IND>
__global__ void __launch_bounds__(ColT<T>::F_THREADS) k_rforce_grp(int n, int nk, int zs, int ngrp, Box box,
                                                                  const double4 *pos4, const int4 *fixq,
                                                                  const int4 *kgrp, const int4 *kcol,
                                                                  const typename ColT<T>::T2 *kcxy,
                                                                  const typename ColT<T>::T4 *kzr,
                                                                  const double *sk, const double *tq,
                                                                  const double *mu, const double *qd,
                                                                  const double *pind, long long *frc,
                                                                  long long *trq) {
    using T2 = typename ColT<T>::T2;
    using T4 = typename ColT<T>::T4;
    constexpr int THREADS = ColT<T>::F_THREADS;
    extern __shared__ float4 s_dyn4[];
    T4 *s_k = (T4 *)s_dyn4;                        // [CF_KGROUP] (U', W', kz, kz^2)
    int4 *s_col = (int4 *)(s_k + CF_KGROUP);       // [CF_CGROUP]
    T2 *s_cxy = (T2 *)(s_col + CF_CGROUP);         // [CF_CGROUP]
    T2 *s_z = s_cxy + CF_CGROUP;                   // [THREADS][zs]
    const int i = blockIdx.x * THREADS + threadIdx.x;
    const bool own = i < n;
    const SitePhase<T> pf = own ? SitePhase<T>(fixq, pos4, box, i) : SitePhase<T>();
    T2 *zt = s_z + threadIdx.x * zs;
    for (int m = 0; m < zs; m++) zt[m] = SitePhase<T>::entry(m, pf.z);
    double D1[3] = {0, 0, 0}, D2[6] = {0, 0, 0, 0, 0, 0}, D3[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int gper = (ngrp + gridDim.y - 1) / gridDim.y;
    const int g0 = blockIdx.y * gper, g1 = min(ngrp, g0 + gper);
    for (int g = g0; g < g1; g++) {
        const int4 gr = kgrp[g];
        __syncthreads();
        for (int e = threadIdx.x; e < gr.w; e += THREADS) {
            const size_t k = (size_t)gr.z + e;
            const T4 r = kzr[k];
            double U = sk[k] - sk[3 * (size_t)nk + k], W = sk[nk + k] + sk[2 * (size_t)nk + k];
            if (IND) {
                U -= sk[5 * (size_t)nk + k];
                W += sk[4 * (size_t)nk + k];
            }
            T4 v;
            v.x = (T)(r.z * U); v.y = (T)(r.z * W); v.z = r.x; v.w = r.y;
            s_k[e] = v;
        }
        for (int e = threadIdx.x; e < gr.y; e += THREADS) {
            int4 cc = kcol[gr.x + e];
            cc.x -= gr.z;
            s_col[e] = cc;
            s_cxy[e] = kcxy[gr.x + e];
        }
        __syncthreads();
        T M1[3] = {0, 0, 0}, M2[6] = {0, 0, 0, 0, 0, 0};
        T M3[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int cix = 0; cix < gr.y; cix++) {
            const int4 cc = s_col[cix];
            const int nx = (short)(cc.z & 0xffff), ny = cc.z >> 16;
            T s0, c0;
            pf.rot(nx, ny, cc.w, s0, c0);
            T P0 = 0, P1 = 0, P2 = 0, P3 = 0, R0 = 0, R1 = 0, R2 = 0;
            const T4 *kr = s_k + cc.x;
            for (int m = 0; m < cc.y; m++) {
                const T4 r = kr[m];
                const T2 z = zt[m];
                const T cs = tfma(c0, z.x, -s0 * z.y), sn = tfma(c0, z.y, s0 * z.x);
                const T A = tfma(sn, r.x, -cs * r.y), B = tfma(cs, r.x, sn * r.y);
                const T Akz = A * r.z;
                P0 += A; P1 += Akz; P2 = tfma(A, r.w, P2); P3 = tfma(Akz, r.w, P3);
                R0 += B; R1 = tfma(B, r.z, R1); R2 = tfma(B, r.w, R2);
            }
            const T2 kk = s_cxy[cix];
            const T kx = kk.x, ky = kk.y, kxx = kx * kx, kxy = kx * ky, kyy = ky * ky;
            M1[0] = tfma(kx, P0, M1[0]); M1[1] = tfma(ky, P0, M1[1]); M1[2] += P1;
            M2[0] = tfma(kxx, R0, M2[0]); M2[1] = tfma(kxy, R0, M2[1]); M2[2] = tfma(kx, R1, M2[2]);
            M2[3] = tfma(kyy, R0, M2[3]); M2[4] = tfma(ky, R1, M2[4]); M2[5] += R2;
            M3[0] = tfma(kxx * kx, P0, M3[0]); M3[1] = tfma(kxx * ky, P0, M3[1]); M3[2] = tfma(kxx, P1, M3[2]);
            M3[3] = tfma(kx * kyy, P0, M3[3]); M3[4] = tfma(kxy, P1, M3[4]); M3[5] = tfma(kx, P2, M3[5]);
            M3[6] = tfma(kyy * ky, P0, M3[6]); M3[7] = tfma(kyy, P1, M3[7]); M3[8] = tfma(ky, P2, M3[8]);
            M3[9] += P3;
        }
#pragma unroll
        for (int q = 0; q < 3; q++) D1[q] += M1[q];
#pragma unroll
        for (int q = 0; q < 6; q++) D2[q] += M2[q];
#pragma unroll
        for (int q = 0; q < 10; q++) D3[q] += M3[q];
    }
    if (own) {
        const size_t N = (size_t)n;
        const double q = tq[(int)pos4[i].w] / SQC_R;
        double m[3], d[3], Q[3][3];
        for (int a = 0; a < 3; a++) {
            m[a] = mu[a * N + i];
            d[a] = m[a] + (IND ? pind[a * N + i] : 0.0);
        }
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) Q[a][b] = qd[sym2(a, b) * N + i];
        double F[3], G[3], QM[3][3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            double f = q * D1[a];
#pragma unroll
            for (int b = 0; b < 3; b++) {
                f += d[b] * D2[sym2(a, b)];
#pragma unroll
                for (int c = 0; c < 3; c++) f -= Q[b][c] * D3[sym3(a, b, c)];
            }
            F[a] = f;
        }
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++) {
                double t = 0;
#pragma unroll
                for (int c = 0; c < 3; c++) t += Q[a][c] * D2[sym2(c, b)];
                QM[a][b] = t;
            }
        G[0] = QM[2][1] - QM[1][2];
        G[1] = QM[0][2] - QM[2][0];
        G[2] = QM[1][0] - QM[0][1];
        const V3 tau = crs(v3(m[0], m[1], m[2]), v3(D1[0], D1[1], D1[2])) - 2.0 * v3(G[0], G[1], G[2]);
        add_fix3_atomic(frc, n, i, v3(F[0], F[1], F[2]), KE);
        add_fix3_atomic(trq, n, i, tau, KE);
    }
}

int tab_row(int nt) { return (3 * nt + 1) & ~1; }
template <typename T>
size_t tsum_smem(int row) {
    return (size_t)ColT<T>::SUM_SITES * (4 * sizeof(typename ColT<T>::T4) + row * sizeof(typename ColT<T>::T2));
}
int zrow(int nmax) { return (2 * nmax + 1) | 1; }
template <typename T>
size_t tforce_smem(int zs) {
    return (size_t)CF_KGROUP * sizeof(typename ColT<T>::T4) +
           (size_t)CF_CGROUP * (sizeof(int4) + sizeof(typename ColT<T>::T2)) +
           (size_t)ColT<T>::F_THREADS * zs * sizeof(typename ColT<T>::T2);
}

// column, run and group records of the column passes, the site-table and
// site-record buffers of both precisions and the kernels' dynamic shared
// memory (once per k set, outside any capture).  Leaves the column passes
// off (rc.kseg null) when the k list is not column ordered with fixed
// (kx, ky) per column or |n| is too large for the tables.
int mp_recip_prepare(Ctx &c) {
    const int nk = c.rc.nk;
    void *old[] = {c.rc.kseg, c.rc.kcol, c.rc.kgrp, c.rc.kzr, c.rc.kcxy, c.rc.stab,
                   c.rc.kzr_d, c.rc.kcxy_d, c.rc.stab_d, c.rc.srec_d};
    for (void *p : old)
        if (p) cudaFree(p);
    c.rc.kseg = nullptr; c.rc.kcol = nullptr; c.rc.kgrp = nullptr; c.rc.kzr = nullptr;
    c.rc.kcxy = nullptr; c.rc.stab = nullptr;
    c.rc.kzr_d = nullptr; c.rc.kcxy_d = nullptr; c.rc.stab_d = nullptr; c.rc.srec_d = nullptr;
    c.rc.nseg = c.rc.ncol = c.rc.ngrp = c.rc.row = 0;
    if (nk == 0 || c.n == 0 || c.rc.nmax + 1 > TAB_MAX || !c.srec) return 0;
    std::vector<int> kn(3 * (size_t)nk);
    std::vector<double> kv(3 * (size_t)nk), kc(nk);
    if (cudaMemcpy(kn.data(), c.rc.kn, kn.size() * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(kv.data(), c.rc.kvec, kv.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(kc.data(), c.rc.kcoef, kc.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        return SMD_ERR_CUDA;
    std::vector<int4> col, seg, grp;
    std::vector<float2> cxy;
    std::vector<float4> kzr(nk);
    std::vector<double2> cxy_d;
    std::vector<double4> kzr_d(nk);
    for (int k = 0; k < nk; k++) {
        const int nx = kn[k], ny = kn[nk + k], nz = kn[2 * nk + k];
        const bool start = k == 0 || nx != kn[k - 1] || ny != kn[nk + k - 1] || nz != kn[2 * nk + k - 1] + 1;
        if (start) {
            col.push_back(make_int4(k, 0, (int)(((unsigned)nx & 0xffffu) | ((unsigned)ny << 16)), nz));
            cxy.push_back(make_float2((float)kv[k], (float)kv[nk + k]));
            cxy_d.push_back(make_double2(kv[k], kv[nk + k]));
        } else if (kv[k] != kv[k - 1] || kv[nk + k] != kv[nk + k - 1]) {
            return 0;  // (kx, ky) varies within a column: not an orthorhombic k set
        }
        col.back().y++;
        const double kz = kv[2 * (size_t)nk + k];
        kzr[k] = make_float4((float)kz, (float)(kz * kz), (float)(2.0 * kc[k]), 0.f);
        kzr_d[k] = make_double4(kz, kz * kz, 2.0 * kc[k], 0.0);
    }
    for (const int4 &cl : col)
        for (int j = 0; j < cl.y; j += TS_SEG)
            seg.push_back(make_int4(cl.x + j, std::min(TS_SEG, cl.y - j), cl.z, cl.w + j));
    for (int q = 0; q < (int)col.size(); q++) {
        const int len = col[q].y;
        if (grp.empty() || grp.back().w + len > CF_KGROUP || grp.back().y >= CF_CGROUP)
            grp.push_back(make_int4(q, 0, col[q].x, 0));
        grp.back().y++;
        grp.back().w += len;
    }
    const int nt = c.rc.nmax + 1, row = tab_row(nt), zs = zrow(c.rc.nmax);
    auto put = [](auto **p, const auto &v) -> bool {
        using T = typename std::remove_reference<decltype(v)>::type::value_type;
        if (cudaMalloc((void **)p, v.size() * sizeof(T)) != cudaSuccess) return false;
        return cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess;
    };
    if (!put(&c.rc.kseg, seg) || !put(&c.rc.kcol, col) || !put(&c.rc.kgrp, grp) || !put(&c.rc.kzr, kzr) ||
        !put(&c.rc.kcxy, cxy) || !put(&c.rc.kzr_d, kzr_d) || !put(&c.rc.kcxy_d, cxy_d) ||
        cudaMalloc((void **)&c.rc.stab, (size_t)c.n * row * sizeof(float2)) != cudaSuccess ||
        cudaMalloc((void **)&c.rc.stab_d, (size_t)c.n * row * sizeof(double2)) != cudaSuccess ||
        cudaMalloc((void **)&c.rc.srec_d, (size_t)c.n * 4 * sizeof(double4)) != cudaSuccess)
        return SMD_ERR_CUDA;
    c.rc.nseg = (int)seg.size();
    c.rc.ncol = (int)col.size();
    c.rc.ngrp = (int)grp.size();
    c.rc.row = row;
    c.rc.tab_n = c.n;
    cudaError_t e = cudaSuccess;
    const cudaFuncAttribute dyn = cudaFuncAttributeMaxDynamicSharedMemorySize;
    if (!e) e = cudaFuncSetAttribute(k_rsk_seg<float, 0, TS_SEG>, dyn, (int)tsum_smem<float>(row));
    if (!e) e = cudaFuncSetAttribute(k_rsk_seg<float, 1, TS_SEG>, dyn, (int)tsum_smem<float>(row));
    if (!e) e = cudaFuncSetAttribute(k_rsk_seg<float, 2, TS_SEG>, dyn, (int)tsum_smem<float>(row));
    if (!e) e = cudaFuncSetAttribute(k_rsk_seg<double, 0, TS_SEG>, dyn, (int)tsum_smem<double>(row));
    if (!e) e = cudaFuncSetAttribute(k_rsk_seg<double, 1, TS_SEG>, dyn, (int)tsum_smem<double>(row));
    if (!e) e = cudaFuncSetAttribute(k_rsk_seg<double, 2, TS_SEG>, dyn, (int)tsum_smem<double>(row));
    if (!e) e = cudaFuncSetAttribute(k_rforce_grp<float, false>, dyn, (int)tforce_smem<float>(zs));
    if (!e) e = cudaFuncSetAttribute(k_rforce_grp<float, true>, dyn, (int)tforce_smem<float>(zs));
    if (!e) e = cudaFuncSetAttribute(k_rforce_grp<double, false>, dyn, (int)tforce_smem<double>(zs));
    if (!e) e = cudaFuncSetAttribute(k_rforce_grp<double, true>, dyn, (int)tforce_smem<double>(zs));
    return e == cudaSuccess ? 0 : SMD_ERR_CUDA;
}

namespace {
struct RecipBufs {
    double *partial, *sk;
};
RecipBufs bufs(Ctx &c) {
    double *partial = (double *)c.rc.sk;
    return {partial, partial + (size_t)6 * c.rc.nk * MK_CHUNKS};
}

// resident blocks per SM of each kernel, looked up once per kernel
int blocks_per_sm(const void *kernel, int threads, size_t smem = 0) {
    static const void *keys[32];
    static size_t smems[32];
    static int vals[32], count = 0;
    for (int q = 0; q < count; q++)
        if (keys[q] == kernel && smems[q] == smem) return vals[q];
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    if (count < 32) {
        keys[count] = kernel;
        smems[count] = smem;
        vals[count++] = per_sm;
    }
    return per_sm;
}
int sm_count() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 1;
    }
    return sms;
}

// site chunks of the partial sums: enough blocks for one full wave of the
// device (at most MK_CHUNKS, the partial buffer's size)
int chunks_for(const void *kernel, int kblocks) {
    const int ch = sm_count() * blocks_per_sm(kernel, MK_THREADS) / (kblocks > 0 ? kblocks : 1);
    return ch < 1 ? 1 : (ch > MK_CHUNKS ? MK_CHUNKS : ch);
}

// the column passes apply: an orthorhombic k set in column order, tables
// for the current site count
bool column_passes(const Ctx &c) { return c.rc.kseg && c.rc.tab_n == c.n; }

template <typename T, int MODE>
int column_sums(Ctx &c, double *partial) {
    const int nk = c.rc.nk, nt = c.rc.nmax + 1, row = c.rc.row;
    const long long ntab = (long long)c.n * row;
    typename ColT<T>::T2 *stab;
    const typename ColT<T>::T4 *ssv;
    if (sizeof(T) == 4) {
        stab = (typename ColT<T>::T2 *)c.rc.stab;
        ssv = (const typename ColT<T>::T4 *)c.srec;   // the frames kernel and the solve keep them current
    } else {
        stab = (typename ColT<T>::T2 *)c.rc.stab_d;
        ssv = (const typename ColT<T>::T4 *)c.rc.srec_d;
        k_pack_srec_d<<<(c.n + 255) / 256, 256, 0, c.stream>>>(c.n, c.pos4, c.type_q, c.mu, c.qd,
                                                              c.ind_on ? c.pind : nullptr, c.rc.srec_d);
    }
    k_site_tab<T><<<(unsigned)((ntab + 255) / 256), 256, 0, c.stream>>>(c.n, nt, row, c.fixq, c.pos4, c.box, stab);
    constexpr int TH = ColT<T>::SUM_THREADS;
    const int kbt = (c.rc.nseg + TH - 1) / TH;
    const size_t sm = tsum_smem<T>(row);
    const int ch = sm_count() * blocks_per_sm((const void *)k_rsk_seg<T, MODE, TS_SEG>, TH, sm) / kbt;
    const int nch = ch < 1 ? 1 : (ch > MK_CHUNKS ? MK_CHUNKS : ch);
    k_rsk_seg<T, MODE, TS_SEG><<<dim3(kbt, nch), TH, sm, c.stream>>>(c.n, nk, c.rc.nseg, nt, row, c.rc.kseg,
                                                                     c.rc.kvec, stab, ssv, partial);
    return nch;
}

template <int MODE>
void sums(Ctx &c, int slot_e, int slot_e2 = -1) {
    const int nk = c.rc.nk;
    RecipBufs B = bufs(c);
    const int kb = (nk + MK_THREADS - 1) / MK_THREADS;
    int nch;
    if (c.precision == SMD_PREC_MIXED && column_passes(c)) {
        nch = column_sums<float, MODE>(c, B.partial);
    } else if (c.precision == SMD_PREC_MIXED) {
        nch = chunks_for((const void *)k_rsk_partial_f<MODE>, kb);
        k_rsk_partial_f<MODE><<<dim3(kb, nch), MK_THREADS, 0, c.stream>>>(c.n, nk, c.pos4, c.fixq, c.rc.kn,
                                                                          c.rc.kvec, c.type_q, c.mu, c.qd, c.pind,
                                                                          B.partial);
    } else if (column_passes(c) && !c.reference_forms) {
        nch = column_sums<double, MODE>(c, B.partial);
    } else {
        nch = chunks_for((const void *)k_rsk_partial<double, MODE>, kb);
        k_rsk_partial<double, MODE><<<dim3(kb, nch), MK_THREADS, 0, c.stream>>>(c.n, nk, c.pos4, c.fixq, c.rc.kn,
                                                                               c.rc.kvec, c.type_q, c.mu, c.qd,
                                                                               c.pind, B.partial);
    }
    k_rsk_reduce<MODE><<<(nk + RR_K - 1) / RR_K, 6 * RR_K, 0, c.stream>>>(nk, nch, B.partial, c.rc.kcoef, c.rc.kvec,
                                                              1.0 / (4.0 * c.ew_alpha * c.ew_alpha), B.sk,
                                                              c.acc, slot_e, slot_e2);
}

// k ranges of the force pass: site blocks x k ranges fill about one wave
int ksplit_for(const void *kernel, int sblocks, int nk) {
    const int ks = sm_count() * blocks_per_sm(kernel, 256) / (sblocks > 0 ? sblocks : 1);
    const int tiles = (nk + FK_TILE - 1) / FK_TILE;
    return ks < 1 ? 1 : (ks > tiles ? tiles : ks);
}

template <typename T, bool IND>
void column_forces(Ctx &c, const double *sk) {
    constexpr int TH = ColT<T>::F_THREADS;
    const int nbs = (c.n + TH - 1) / TH;
    const int ng = c.rc.ngrp;
    const int zs = zrow(c.rc.nmax);
    const size_t sm = tforce_smem<T>(zs);
    int ks = sm_count() * blocks_per_sm((const void *)k_rforce_grp<T, IND>, TH, sm) / nbs;
    ks = ks < 1 ? 1 : (ks > ng ? ng : ks);
    const typename ColT<T>::T2 *kcxy = (const typename ColT<T>::T2 *)(sizeof(T) == 4 ? (void *)c.rc.kcxy
                                                                                     : (void *)c.rc.kcxy_d);
    const typename ColT<T>::T4 *kzr = (const typename ColT<T>::T4 *)(sizeof(T) == 4 ? (void *)c.rc.kzr
                                                                                    : (void *)c.rc.kzr_d);
    k_rforce_grp<T, IND><<<dim3(nbs, ks), TH, sm, c.stream>>>(c.n, c.rc.nk, zs, ng, c.box, c.pos4, c.fixq, c.rc.kgrp,
                                                              c.rc.kcol, kcxy, kzr, sk, c.type_q, c.mu, c.qd,
                                                              c.pind, c.frc, c.trq);
}

template <bool PERM, bool IND>
void forces(Ctx &c) {
    const int nk = c.rc.nk;
    RecipBufs B = bufs(c);
    const int nb = (int)(((long long)c.n * F_TPS + 255) / 256);
    if (c.precision == SMD_PREC_MIXED && PERM && column_passes(c)) {
        column_forces<float, IND>(c, B.sk);
    } else if (c.precision == SMD_PREC_MIXED) {
        if (PERM) {
            const int ks = ksplit_for((const void *)k_rforce_f<IND>, nb, nk);
            k_rforce_f<IND><<<dim3(nb, ks), 256, 0, c.stream>>>(c.n, nk, c.pos4, c.fixq, c.rc.kn, c.rc.kvec,
                                                                c.rc.kcoef, B.sk, c.type_q, c.mu, c.qd, c.pind,
                                                                c.frc, c.trq);
        } else {
            const int ks = ksplit_for((const void *)k_rforce<float, PERM, IND>, nb, nk);
            k_rforce<float, PERM, IND><<<dim3(nb, ks), 256, 0, c.stream>>>(c.n, nk, c.pos4, c.fixq, c.rc.kn,
                                                                          c.rc.kvec, c.rc.kcoef, B.sk, c.type_q,
                                                                          c.mu, c.qd, c.pind, c.frc, c.trq);
        }
    } else if (PERM && column_passes(c) && !c.reference_forms) {
        column_forces<double, IND>(c, B.sk);
    } else {
        const int ks = ksplit_for((const void *)k_rforce<double, PERM, IND>, nb, nk);
        k_rforce<double, PERM, IND><<<dim3(nb, ks), 256, 0, c.stream>>>(c.n, nk, c.pos4, c.fixq, c.rc.kn,
                                                                       c.rc.kvec, c.rc.kcoef, B.sk, c.type_q, c.mu,
                                                                       c.qd, c.pind, c.frc, c.trq);
    }
}
}  // namespace

// Multipole::compute_long on its own
void launch_mp_long(Ctx &c) {
    if (c.rc.nk == 0) return;
    sums<0>(c, ACC_E_LONG);
    forces<true, false>(c);
}

// Induction::compute_long on its own (permanent sums recomputed for it)
void launch_ind_long(Ctx &c) {
    if (c.rc.nk == 0) return;
    sums<0>(c, -1);
    sums<1>(c, ACC_E_POL_LONG);
    forces<false, true>(c);
}

// Both reciprocal terms of a time step, after the dipole solve: one pass for
// all six structure factors, one force pass
void launch_polar_long(Ctx &c) {
    if (c.rc.nk == 0) return;
    sums<2>(c, ACC_E_LONG, ACC_E_POL_LONG);
    forces<true, true>(c);
}

}  // namespace smd
