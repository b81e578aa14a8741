// Surface-dipole corrections (the reference's surfCorrect option) of the
// point-charge Ewald sum, the permanent multipoles and the induced dipoles:
//
//   Ewald      EwaldForce::surfDipoleCorrect (src/forces/EwaldForce.cpp:816-937)
//              S = sum Q_i r_i (scaled charges), c = 2 pi / 3V
//              E = c |S|^2,  F_i = -2 c Q_i S
//   multipole  Multipole::surfDipoleCorrect (src/forces/Multipole.cpp:1753-1920)
//              M = sum (q_i r_i + mu_i),  s = sum (2 q_i tr Q_i - mu_i.mu_i)
//              E = c (|M|^2 + s) ke,  F_i = -2 c q_i M ke,  tau_i = 2 c ke M x mu_i
//   induced    Induction::surfDipoleCorrect (src/forces/Induction.cpp:2188-2380)
//              P = sum p_i,  E = c (sum q_i r_i . P + sum mu_i . P - sum mu_i . p_i) ke
//              F_i = -2 c q_i P ke,  tau_i = 2 c ke (P x mu_i - p_i x mu_i)
// with the positions as stored (Atom::position).  The torques join the
// other torques before their mapping onto the sites.  Virial: the
// reference's multipole and induced terms add -Q_i (sum q_j r_j) r_i per
// site, and the Ewald term -Q_i c S r_i; summed over sites these are the
// outer products below, reproduced as the reference has them.
//
// Three launches: per-block partial sums over sites, a one-block fixed-order
// total that also writes the energies and virials, and a per-site force and
// torque pass.
#include <algorithm>
#include "smd_ctx.cuh"

namespace smd {

constexpr double KE_S = 138.93548501;
constexpr double SQC_S = 11.78708976;
constexpr int SF_THREADS = 256;
constexpr int SF_N = SURF_SUMS;   // qr (3), mu (3), p (3), sum (2 q trQ - mu.mu), sum mu.p

struct SurfArgs {
    int n;
    const double4 *pos4;
    const double *tq, *mu, *qd, *p;   // mu/qd/p null when the model has none
    double *part, *tot;
    long long *frc, *trq, *acc;
    double coeff;                     // 2 pi / 3V
    int ewald, mp, ind;
};

__global__ void __launch_bounds__(SF_THREADS) k_surf_partial(SurfArgs a) {
    double v[SF_N];
    for (int q = 0; q < SF_N; q++) v[q] = 0.0;
    for (int i = blockIdx.x * SF_THREADS + threadIdx.x; i < a.n; i += gridDim.x * SF_THREADS) {
        const double4 r = a.pos4[i];
        const double qi = a.tq[(int)r.w] / SQC_S;
        v[0] += qi * r.x; v[1] += qi * r.y; v[2] += qi * r.z;
        if (a.mu) {
            const double mx = a.mu[i], my = a.mu[a.n + i], mz = a.mu[2 * a.n + i];
            v[3] += mx; v[4] += my; v[5] += mz;
            const double trq = a.qd[i] + a.qd[3 * a.n + i] + a.qd[5 * a.n + i];
            v[9] += 2.0 * qi * trq - (mx * mx + my * my + mz * mz);
            if (a.p) {
                const double px = a.p[i], py = a.p[a.n + i], pz = a.p[2 * a.n + i];
                v[6] += px; v[7] += py; v[8] += pz;
                v[10] += mx * px + my * py + mz * pz;
            }
        }
    }
    __shared__ double s_r[SF_THREADS / 32][SF_N];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int q = 0; q < SF_N; q++) {
        const double t = warp_sum(v[q]);
        if (lane == 0) s_r[w][q] = t;
    }
    __syncthreads();
    if (threadIdx.x < SF_N) {
        double t = 0;
        for (int k = 0; k < SF_THREADS / 32; k++) t += s_r[k][threadIdx.x];
        a.part[blockIdx.x * SF_N + threadIdx.x] = t;
    }
}

// one block: totals in a fixed order, energies and virials
__global__ void k_surf_total(SurfArgs a, int nblocks) {
    __shared__ double s_t[SF_N];
    if (threadIdx.x < SF_N) {
        double t = 0;
        for (int b = 0; b < nblocks; b++) t += a.part[b * SF_N + threadIdx.x];
        s_t[threadIdx.x] = t;
        a.tot[threadIdx.x] = t;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const double qr[3] = {s_t[0], s_t[1], s_t[2]}, mu[3] = {s_t[3], s_t[4], s_t[5]}, P[3] = {s_t[6], s_t[7], s_t[8]};
    const double c = a.coeff;
    auto add = [&](int slot, double v) {
        if (v != 0.0) atomicAdd((unsigned long long *)&a.acc[slot], (unsigned long long)to_fix(v, ACC_SCALE));
    };
    double vir[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};   // Ensemble::virial contribution
    if (a.ewald) {
        // S = sum Q_i r_i = SQC qr
        double S[3];
        for (int d = 0; d < 3; d++) S[d] = SQC_S * qr[d];
        add(ACC_E_SURF, c * (S[0] * S[0] + S[1] * S[1] + S[2] * S[2]));
        for (int x = 0; x < 3; x++)
            for (int y = 0; y < 3; y++) vir[3 * x + y] += c * S[x] * S[y];
    }
    if (a.mp) {
        double M[3];
        for (int d = 0; d < 3; d++) M[d] = qr[d] + mu[d];
        add(ACC_E_SURF, c * (M[0] * M[0] + M[1] * M[1] + M[2] * M[2] + s_t[9]) * KE_S);
        for (int x = 0; x < 3; x++)
            for (int y = 0; y < 3; y++) vir[3 * x + y] += SQC_S * qr[x] * qr[y];
    }
    if (a.ind) {
        const double e = (qr[0] * P[0] + qr[1] * P[1] + qr[2] * P[2]) + (mu[0] * P[0] + mu[1] * P[1] + mu[2] * P[2]) -
                         s_t[10];
        add(ACC_E_POL_SURF, c * e * KE_S);
        for (int x = 0; x < 3; x++)
            for (int y = 0; y < 3; y++) vir[3 * x + y] += SQC_S * qr[x] * qr[y];
    }
    for (int q = 0; q < 9; q++) add(ACC_VIR + q, vir[q]);
}

__global__ void __launch_bounds__(SF_THREADS) k_surf_apply(SurfArgs a) {
    const int i = blockIdx.x * SF_THREADS + threadIdx.x;
    if (i >= a.n) return;
    const double4 r = a.pos4[i];
    const double Q = a.tq[(int)r.w], qi = Q / SQC_S, c = a.coeff;
    const double qr[3] = {a.tot[0], a.tot[1], a.tot[2]}, mus[3] = {a.tot[3], a.tot[4], a.tot[5]};
    const double P[3] = {a.tot[6], a.tot[7], a.tot[8]};
    double f[3] = {0, 0, 0}, t[3] = {0, 0, 0};
    if (a.ewald)
        for (int d = 0; d < 3; d++) f[d] -= 2.0 * c * Q * SQC_S * qr[d];
    double mi[3] = {0, 0, 0};
    if (a.mu) {
        mi[0] = a.mu[i]; mi[1] = a.mu[a.n + i]; mi[2] = a.mu[2 * a.n + i];
    }
    if (a.mp) {
        const double M[3] = {qr[0] + mus[0], qr[1] + mus[1], qr[2] + mus[2]};
        for (int d = 0; d < 3; d++) f[d] -= 2.0 * c * qi * M[d] * KE_S;
        const double k = 2.0 * c * KE_S;
        t[0] += k * (M[1] * mi[2] - M[2] * mi[1]);
        t[1] += k * (M[2] * mi[0] - M[0] * mi[2]);
        t[2] += k * (M[0] * mi[1] - M[1] * mi[0]);
    }
    if (a.ind) {
        for (int d = 0; d < 3; d++) f[d] -= 2.0 * c * qi * P[d] * KE_S;
        const double pi[3] = {a.p[i], a.p[a.n + i], a.p[2 * a.n + i]};
        const double D[3] = {P[0] - pi[0], P[1] - pi[1], P[2] - pi[2]};
        const double k = 2.0 * c * KE_S;
        t[0] += k * (D[1] * mi[2] - D[2] * mi[1]);
        t[1] += k * (D[2] * mi[0] - D[0] * mi[2]);
        t[2] += k * (D[0] * mi[1] - D[1] * mi[0]);
    }
    for (int d = 0; d < 3; d++)
        atomicAdd((unsigned long long *)&a.frc[(size_t)d * a.n + i], (unsigned long long)to_fix(f[d], FRC_SCALE));
    if (a.mp || a.ind)
        for (int d = 0; d < 3; d++)
            atomicAdd((unsigned long long *)&a.trq[(size_t)d * a.n + i], (unsigned long long)to_fix(t[d], FRC_SCALE));
}

void launch_surface(Ctx &c, bool ewald, bool mp, bool ind) {
    if (!c.surface_on || !(ewald || mp || ind) || !c.surf_part) return;
    SurfArgs a;
    a.n = c.n; a.pos4 = c.pos4; a.tq = c.type_q;
    a.mu = c.mp_on ? c.mu : nullptr;
    a.qd = c.mp_on ? c.qd : nullptr;
    a.p = c.mp_on && c.ind_on ? c.pind : nullptr;
    a.part = c.surf_part; a.tot = c.surf_tot;
    a.frc = c.frc; a.trq = c.trq; a.acc = c.acc;
    a.coeff = 2.0 * 3.14159265358979323846 / (3.0 * c.box.L[0] * c.box.L[1] * c.box.L[2]);
    a.ewald = ewald ? 1 : 0;
    a.mp = mp && c.mp_on ? 1 : 0;
    a.ind = ind && c.mp_on && c.ind_on ? 1 : 0;
    const int nb = std::min(SURF_BLOCKS, (c.n + SF_THREADS - 1) / SF_THREADS);
    k_surf_partial<<<nb, SF_THREADS, 0, c.stream>>>(a);
    k_surf_total<<<1, 32, 0, c.stream>>>(a, nb);
    k_surf_apply<<<(c.n + SF_THREADS - 1) / SF_THREADS, SF_THREADS, 0, c.stream>>>(a);
}

}  // namespace smd
