// Lustig's volume derivatives of the LJ energy (LJForce::compute with
// computeLustig, src/forces/LJForce.cpp:136-150, 230-247): per pair of sites
// of different molecules within the cutoff,
//   du  = tmpf (r_ij . R_ij)                       (Lustig 2011 eq. 15b)
//   d2u = 4 eps (156 (s/r)^12 - 42 (s/r)^6) (r_ij . R_ij)^2 / r^4 + 2 du
// with tmpf = 24 eps (2 (s/r)^12 - (s/r)^6) / r^2, and R_ij the minimum-image
// difference of the molecules' centres of mass under constraints (r_ij
// itself otherwise); then
//   U = sum u + E_lrc,  dU/dV = -sum du / 3V + dE_lrc/dV,
//   d2U/dV2 = sum d2u / 9V^2 + d2E_lrc/dV2
// with the tail correction E_lrc = -K / V of LJForce::long_range_correct.
// One thread per site over its full-list row (each pair twice, halved at
// the end); the three sums in 64-bit fixed point, so in a fixed total.
#include <algorithm>
#include <vector>
#include "smd_ctx.cuh"
#include "smd_polar.cuh"

namespace smd {

__global__ void k_mol_com(int nmol, const int *mol_off, const int *mol_atoms, const double4 *pos4,
                          const double *mass, double4 *com) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nmol) return;
    double cx = 0, cy = 0, cz = 0, M = 0;
    for (int k = mol_off[m]; k < mol_off[m + 1]; k++) {
        const int i = mol_atoms[k];
        const double4 p = pos4[i];
        const double w = mass[i];
        cx += w * p.x; cy += w * p.y; cz += w * p.z;
        M += w;
    }
    com[m] = make_double4(cx / M, cy / M, cz / M, M);
}

constexpr double LUS_SCALE = 268435456.0;   // 2^28

__global__ void k_lustig_lj(int n, const int *nbr, const int *nnbr, const double4 *pos4, const int *mol,
                            const double4 *com, const double *par, int nt, Box box, double rc2, int switch_on,
                            int constrained, long long *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double su = 0, s1 = 0, s2 = 0;
    if (i < n) {
        const double4 pi = pos4[i];
        const int ti = (int)pi.w, mi = mol[i];
        const double4 ci = com[mi];
        for (int k = 0; k < nnbr[i]; k++) {
            const int raw = nbr[(size_t)k * n + i];
            if (raw < 0) continue;   // same molecule
            const int j = raw;
            const double4 pj = pos4[j];
            const double dx = pbc1(pj.x - pi.x, box.L[0], box.half[0]);
            const double dy = pbc1(pj.y - pi.y, box.L[1], box.half[1]);
            const double dz = pbc1(pj.z - pi.z, box.L[2], box.half[2]);
            const double r = sqrt(dx * dx + dy * dy + dz * dz), r2 = r * r;
            if (!(r2 <= rc2)) continue;
            const double *p = par + (size_t)(ti * nt + (int)pj.w) * 4;
            const double r_1 = 1.0 / r, rij_2 = r_1 * r_1;
            const double sr2 = p[0] * rij_2, sr6 = sr2 * sr2 * sr2, sr12 = sr6 * sr6;
            double e = p[1] * (sr12 - sr6);
            const double tmpf = (sr12 + sr12 - sr6) * 6.0 * p[1] * rij_2;
            double rr = r2;
            if (constrained) {
                const double4 cj = com[mol[j]];
                const double mx = pbc1(cj.x - ci.x, box.L[0], box.half[0]);
                const double my = pbc1(cj.y - ci.y, box.L[1], box.half[1]);
                const double mz = pbc1(cj.z - ci.z, box.L[2], box.half[2]);
                rr = dx * mx + dy * my + dz * mz;
            }
            const double du = tmpf * rr;
            const double d2u = p[1] * (156.0 * sr12 - 42.0 * sr6) * rr * rr * rij_2 * rij_2 + 2.0 * du;
            if (switch_on) e -= p[2];
            su += e; s1 += du; s2 += d2u;
        }
    }
    su = warp_sum(su); s1 = warp_sum(s1); s2 = warp_sum(s2);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd((unsigned long long *)&out[0], (unsigned long long)to_fix(su, LUS_SCALE));
        atomicAdd((unsigned long long *)&out[1], (unsigned long long)to_fix(s1, LUS_SCALE));
        atomicAdd((unsigned long long *)&out[2], (unsigned long long)to_fix(s2, LUS_SCALE));
    }
}

// grows the evaluation's scratch (the context owns it; freed with the context)
static int lus_reserve(Ctx &c, size_t doubles) {
    if (!c.lus_com) {
        if (cudaMalloc(&c.lus_com, (size_t)c.nmol * sizeof(double4)) != cudaSuccess) return SMD_ERR_CUDA;
    }
    if (doubles > c.lus_cap) {
        if (c.lus_buf) cudaFree(c.lus_buf);
        c.lus_buf = nullptr;
        c.lus_cap = 0;
        if (cudaMalloc(&c.lus_buf, doubles * sizeof(double)) != cudaSuccess) return SMD_ERR_CUDA;
        c.lus_cap = doubles;
    }
    return SMD_OK;
}

int lustig_lj(Ctx &c, double *out) {
    if (c.vdw != VDW_LJ) return SMD_ERR_ARG;
    // the three fixed-point sums in the context's scratch (no allocation
    // after the first call)
    int r = lus_reserve(c, 3);
    if (r) return r;
    long long *acc = reinterpret_cast<long long *>(c.lus_buf);
    cudaMemsetAsync(acc, 0, 3 * sizeof(long long), c.stream);
    launch_nlist(c, !c.list_built);
    k_mol_com<<<(c.nmol + 127) / 128, 128, 0, c.stream>>>(c.nmol, c.mol_off, c.mol_atoms, c.pos4, c.mass,
                                                         c.lus_com);
    k_lustig_lj<<<(c.n + 127) / 128, 128, 0, c.stream>>>(c.n, c.pl.nbr, c.pl.nnbr, c.pos4, c.mol, c.lus_com,
                                                         c.pair_par, c.ntypes, c.box, c.vdw_rc2, c.switch_on,
                                                         c.clen2 != nullptr, acc);
    long long h[3];
    if (cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
        cudaStreamSynchronize(c.stream) != cudaSuccess)
        return SMD_ERR_CUDA;
    const double V = c.box.L[0] * c.box.L[1] * c.box.L[2];
    const double su = 0.5 * (double)h[0] / LUS_SCALE, s1 = 0.5 * (double)h[1] / LUS_SCALE,
                 s2 = 0.5 * (double)h[2] / LUS_SCALE;
    out[0] = su + c.e_lrc;
    out[1] = -s1 / (3.0 * V) - 2.0 * c.e_lrc / V;
    out[2] = s2 / (9.0 * V * V) + 6.0 * c.e_lrc / (V * V);
    return SMD_OK;
}

// ===========================================================================
// Every field of Ensemble::myLustig (src/Ensemble.h:77-108) at the current
// configuration, as the reference's force terms write them during a step.
// On demand and in FP64: one pass per term group, each term's own sums in
// per-block (or per-k) partials that the host adds in a fixed order.
//
//   point charges (EwaldForce)       realDeriv/realSecDeriv (real_term,
//       EwaldForce.cpp:405-411), intravirCorrect/molDeriv/molSecDeriv
//       (intraMolCorrect :770-790), surfDeriv/surfSecDeriv (surfDipoleCorrect
//       :850-863), longDeriv/longSecDeriv (reciprocal_term :596-675)
//   multipoles (Multipole)           realDeriv: -ke sum f_ij.r_ij over the
//       real-space pairs (:661) plus the torque mapping's dU/dV (:943-946);
//       molDeriv (:1514, :1744-1747); surfDeriv/surfSecDeriv (:1827-1836,
//       :1933-1936); longDeriv/longSecDeriv with dUdV3rd (:1133-1138,
//       :1214-1217, :1273-1276)
//   induced dipoles (Induction)      selfPolDeriv (:754-757), realPolDeriv
//       (:1133, :1386-1389), molPolDeriv (:2013), surfPolDeriv/
//       surfSecPolDeriv (:2270-2290), longPolDeriv/longSecPolDeriv
//       (:1597-1613, :1686-1690, :1742-1745)
//   Wolf sum (WolfForce)             realDeriv/realSecDeriv (:200-244)
//   buffered 14-7 (BuffvdWForce)     ljUlus, ljdUlus (:244, :326-330)
//   bonds, Urey-Bradley              BondDeriv/BondSecDeriv (BondForce.cpp:86-87),
//                                    ubDeriv/ubSecDeriv (UreyBradleyForce.cpp:76-77)
// virialcorrect is left at zero: LFIntegrator forms it after the position
// update, from this step's forces and the next step's positions and
// centres (LFIntegrator.cpp:819-836), so no one configuration defines it.
// The torque part of a term's dU/dV is its torques mapped as
// Multipole::torques2forces does (:1946-2134), summing dU/du.u + dU/dv.v.
// ===========================================================================
constexpr double LU_COU = 138.93548501;    // COUlOMBS (src/NEMD_defs.h:98)
constexpr double LU_SQC = 11.78708976;     // SQRTCOULOMBCONSTANT
constexpr double LU_SQRTPI = 1.7724538509055160273;
constexpr int LU_THREADS = 256;

// block totals of NV values into out[blockIdx.x * NV + q]
template <int NV>
__device__ __forceinline__ void lu_block_out(double (&v)[NV], double *out) {
    __shared__ double s[LU_THREADS / 32][NV];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int q = 0; q < NV; q++) {
        const double t = warp_sum(v[q]);
        if (lane == 0) s[w][q] = t;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double t = 0;
        for (int k = 0; k < LU_THREADS / 32; k++) t += s[k][threadIdx.x];
        out[(size_t)blockIdx.x * NV + threadIdx.x] = t;
    }
    __syncthreads();
}

// block totals of NV values handed back to every thread
template <int NV>
__device__ __forceinline__ void lu_block_all(double (&v)[NV]) {
    __shared__ double s[LU_THREADS / 32][NV];
    __shared__ double tot[NV];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int q = 0; q < NV; q++) {
        const double t = warp_sum(v[q]);
        if (lane == 0) s[w][q] = t;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double t = 0;
        for (int k = 0; k < LU_THREADS / 32; k++) t += s[k][threadIdx.x];
        tot[threadIdx.x] = t;
    }
    __syncthreads();
    for (int q = 0; q < NV; q++) v[q] = tot[q];
    __syncthreads();
}

__device__ __forceinline__ void lu_min(double &x, double &y, double &z, const Box &b) {
    x = pbc1(x, b.L[0], b.half[0]);
    y = pbc1(y, b.L[1], b.half[1]);
    z = pbc1(z, b.L[2], b.half[2]);
}

// EwaldForce::real_term's derivatives over the full list (each pair twice):
//   realDeriv    += -q_ij f (r_ij . R_ij)
//   realSecDeriv += q_ij (2f + 2 a2pi a^2 e^{-a^2 r^2}) (r_ij . R_ij)^2 / r^2 + 2 q_ij f (r_ij . R_ij)
// f = (erfc(a r)/r + a2pi e^{-a^2 r^2}) / r^2; r_ij . R_ij is r^2 without
// constraints and uses the molecules' centres with them.
__global__ void __launch_bounds__(LU_THREADS) k_lus_ewald_real(int n, const int *nbr, const int *nnbr,
                                                               const double4 *pos4, const int *mol,
                                                               const double4 *com, const double *tq, Box box,
                                                               double rc2, double alpha, int constrained,
                                                               double *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[2] = {0, 0};
    if (i < n) {
        const double4 pi = pos4[i];
        const double qi = tq[(int)pi.w];
        const double4 ci = com[mol[i]];
        const double a2 = alpha * alpha, a2pi = 2.0 * alpha / LU_SQRTPI;
        for (int k = 0; k < nnbr[i]; k++) {
            const int j = nbr[(size_t)k * n + i] & 0x7fffffff;
            const double4 pj = pos4[j];
            double dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
            lu_min(dx, dy, dz, box);
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (!(r2 < rc2)) continue;
            const double qij = qi * tq[(int)pj.w];
            double rr = r2;
            if (constrained) {
                const double4 cj = com[mol[j]];
                double mx = cj.x - ci.x, my = cj.y - ci.y, mz = cj.z - ci.z;
                lu_min(mx, my, mz, box);
                rr = dx * mx + dy * my + dz * mz;
            }
            const double r = sqrt(r2), ex = exp(-a2 * r2);
            const double f = (erfc(alpha * r) / r + a2pi * ex) / r2;
            v[0] += -qij * f * rr;
            v[1] += qij * (2.0 * f + 2.0 * a2pi * a2 * ex) * rr * rr / r2 + 2.0 * qij * f * rr;
        }
    }
    lu_block_out<2>(v, out);
}

// WolfForce::real_term's derivatives (WolfForce.cpp:200-244) over the full
// list of charge-site positions (the displaced O sites of "WAT" molecules
// where the sum puts them): with the sum shifted at the cutoff Rc,
//   f   = (erfc(a r)/r + a2pi e^{-a^2 r^2}) / r^2 - R / Rc,
//         R = erfc(a Rc)/Rc^2 + a2pi e^{-a^2 Rc^2} / Rc
//   dv2 = (2 dv + 2 a2pi a^2 e^{-a^2 r^2}) / r^2 - (2 R / Rc + 2 a2pi a^2 e^{-a^2 Rc^2}) / Rc^2
//   realDeriv    += -q_ij f (r_ij . R_ij)
//   realSecDeriv += q_ij dv2 (r_ij . R_ij)^2 + 2 q_ij f (r_ij . R_ij)
// with R_ij the molecules' centres' difference in every case.
__global__ void __launch_bounds__(LU_THREADS) k_lus_wolf(int n, const int *nbr, const int *nnbr,
                                                         const double4 *qpos4, const int *mol,
                                                         const double4 *com, const double *tq, Box box,
                                                         double rc, double alpha, double *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[2] = {0, 0};
    if (i < n) {
        const double4 pi = qpos4[i];
        const double qi = tq[(int)pi.w];
        const double4 ci = com[mol[i]];
        const double a2 = alpha * alpha, a2pi = 2.0 * alpha / LU_SQRTPI, rc2 = rc * rc;
        const double eR = erfc(alpha * rc) / rc;
        const double Rc = eR / rc + a2pi * exp(-a2 * rc2) / rc;
        const double d2c = (2.0 * Rc / rc + 2.0 * a2pi * a2 * exp(-a2 * rc2)) / rc2;
        for (int k = 0; k < nnbr[i]; k++) {
            const int j = nbr[(size_t)k * n + i] & 0x7fffffff;
            const double4 pj = qpos4[j];
            double dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
            lu_min(dx, dy, dz, box);
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (!(r2 < rc2)) continue;
            const double4 cj = com[mol[j]];
            double mx = cj.x - ci.x, my = cj.y - ci.y, mz = cj.z - ci.z;
            lu_min(mx, my, mz, box);
            const double rr = dx * mx + dy * my + dz * mz;
            const double qij = qi * tq[(int)pj.w];
            const double r = sqrt(r2), ex = exp(-a2 * r2);
            const double dv = (erfc(alpha * r) / r + a2pi * ex) / r2;
            const double f = dv - Rc / rc;
            const double dv2 = (2.0 * dv + 2.0 * a2pi * a2 * ex) / r2 - d2c;
            v[0] += -qij * f * rr;
            v[1] += qij * dv2 * rr * rr + 2.0 * qij * f * rr;
        }
    }
    lu_block_out<2>(v, out);
}

// EwaldForce::intraMolCorrect over each molecule's excluded pairs:
//   v0 = sum a2pi q_ij e^{-a^2 r^2}           (intravirCorrect = -v0)
//   v1 = sum q_ij (erf(a r)/r - a2pi e^{-a^2 r^2})   (molDeriv = v1 / 3V)
//   v2 = sum -2 q_ij d + q_ij (-2 d + 2 a2pi a^2 e^{-a^2 r^2} r^2)  (molSecDeriv = v2 / 9V^2)
__global__ void __launch_bounds__(LU_THREADS) k_lus_ewald_intra(int nmol, const int *mol_off, const int *mol_atoms,
                                                                const int *excl_off, const int *excl,
                                                                const double4 *pos4, const double *tq, Box box,
                                                                double alpha, double *out) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    double v[3] = {0, 0, 0};
    if (m < nmol) {
        const double a2 = alpha * alpha, a2pi = 2.0 * alpha / LU_SQRTPI;
        for (int p = mol_off[m]; p < mol_off[m + 1]; p++)
            for (int q = p + 1; q < mol_off[m + 1]; q++) {
                const int i = mol_atoms[p], j = mol_atoms[q];
                bool ex = false;
                for (int k = excl_off[i]; k < excl_off[i + 1]; k++)
                    if (excl[k] == j) { ex = true; break; }
                if (!ex) continue;
                const double4 pi = pos4[i], pj = pos4[j];
                double dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
                lu_min(dx, dy, dz, box);
                const double r2 = dx * dx + dy * dy + dz * dz, r = sqrt(r2);
                const double qij = tq[(int)pi.w] * tq[(int)pj.w];
                const double ex2 = exp(-a2 * r2);
                const double d = erf(alpha * r) / r - a2pi * ex2;
                v[0] += a2pi * qij * ex2;
                v[1] += qij * d;
                v[2] += -2.0 * qij * d + qij * (-2.0 * d + 2.0 * a2pi * a2 * ex2 * r2);
            }
    }
    lu_block_out<3>(v, out);
}

// site sums of the surface terms and of virialcorrect:
//   [0..2] q r, [3..5] q R (scaled charges), [6..8] q r, [9..11] q R
//   (charges / sqrt(ke)), [12..14] mu, [15..17] p, [18] mu.p, [19] p.p,
//   [20] f.(r - R) (force: Atom::force layout, may be null),
//   [21] 2 q tr(Q) - mu.mu (charges / sqrt(ke))
constexpr int LU_NSUM = 22;
__global__ void __launch_bounds__(LU_THREADS) k_lus_sites(int n, const double4 *pos4, const int *mol,
                                                          const double4 *com, const double *tq,
                                                          const double *mu, const double *qd,
                                                          const double *pind, const double *force,
                                                          double *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[LU_NSUM];
    for (int q = 0; q < LU_NSUM; q++) v[q] = 0;
    if (i < n) {
        const double4 p = pos4[i];
        const double4 R = com[mol[i]];
        const double qs = tq[(int)p.w], qu = qs / LU_SQC;
        const double r[3] = {p.x, p.y, p.z}, Rm[3] = {R.x, R.y, R.z};
        for (int d = 0; d < 3; d++) {
            v[d] = qs * r[d];
            v[3 + d] = qs * Rm[d];
            v[6 + d] = qu * r[d];
            v[9 + d] = qu * Rm[d];
        }
        double m[3] = {0, 0, 0}, pp[3] = {0, 0, 0};
        if (mu)
            for (int d = 0; d < 3; d++) m[d] = mu[(size_t)d * n + i];
        if (pind)
            for (int d = 0; d < 3; d++) pp[d] = pind[(size_t)d * n + i];
        for (int d = 0; d < 3; d++) {
            v[12 + d] = m[d];
            v[15 + d] = pp[d];
        }
        v[18] = m[0] * pp[0] + m[1] * pp[1] + m[2] * pp[2];
        v[19] = pp[0] * pp[0] + pp[1] * pp[1] + pp[2] * pp[2];
        if (force)
            for (int d = 0; d < 3; d++) v[20] += force[(size_t)3 * i + d] * (r[d] - Rm[d]);
        if (qd) {
            const double tr = qd[i] + qd[3 * (size_t)n + i] + qd[5 * (size_t)n + i];
            v[21] = 2.0 * qu * tr - (m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
        }
    }
    lu_block_out<LU_NSUM>(v, out);
}

// One block per k: the structure factors of the term, then (with
// constraints) the centre-of-mass sums Ff, Ffk2, d2UV1, d2UrR over the
// sites; out[2k] and out[2k + 1] take the k's share of longDeriv and
// longSecDeriv (or longPolDeriv and longSecPolDeriv).
//   KIND 0: point charges (EwaldForce::reciprocal_term)
//   KIND 1: permanent multipoles (Multipole::reciprocal_term)
//   KIND 2: induced dipoles (Induction::reciprocal_term, minimised dipoles)
template <int KIND>
__global__ void __launch_bounds__(LU_THREADS) k_lus_recip(int n, int nk, const double *kvec, const double *kcoef,
                                                          const double4 *pos4, const int *mol, const double4 *com,
                                                          const double *tq, const double *mu, const double *qd,
                                                          const double *pind, double alpha, int constrained,
                                                          double *out) {
    const int k = blockIdx.x;
    const double kx = kvec[k], ky = kvec[nk + k], kz = kvec[2 * (size_t)nk + k];
    const double k2 = kx * kx + ky * ky + kz * kz;
    const double kk[6] = {kx * kx, 2 * kx * ky, 2 * kx * kz, ky * ky, 2 * ky * kz, kz * kz};
    const double c = kcoef[k], b = 2.0 * c, x = k2 / (2.0 * alpha * alpha);
    // per site: weight of the charge-like sum, mu.k, p.k, 2 k.Q.k
    auto site = [&](int i, double &wq, double &wm, double &wp, double &w2, double &sn, double &cs, double d[3]) {
        const double4 p = pos4[i];
        const double4 R = com[mol[i]];
        d[0] = p.x - R.x; d[1] = p.y - R.y; d[2] = p.z - R.z;
        sincos(p.x * kx + p.y * ky + p.z * kz, &sn, &cs);
        wm = wp = w2 = 0;
        if (KIND == 0) {
            wq = tq[(int)p.w];
        } else {
            double qk = 0;
            for (int q = 0; q < 6; q++) qk += qd[(size_t)q * n + i] * kk[q];
            wq = tq[(int)p.w] / LU_SQC - qk;
            wm = mu[i] * kx + mu[n + i] * ky + mu[2 * (size_t)n + i] * kz;
            w2 = 2.0 * qk;
            if (KIND == 2) wp = pind[i] * kx + pind[n + i] * ky + pind[2 * (size_t)n + i] * kz;
        }
    };
    // [0,1] charge-like C S, [2,3] mu.k C S, [4,5] p.k C S, [6,7] 2kQk C S,
    // [8..10] sum C_i (r - R), [11..13] sum S_i (r - R)
    double s[14];
    for (int q = 0; q < 14; q++) s[q] = 0;
    for (int i = threadIdx.x; i < n; i += LU_THREADS) {
        double wq, wm, wp, w2, sn, cs, d[3];
        site(i, wq, wm, wp, w2, sn, cs, d);
        s[0] += wq * cs; s[1] += wq * sn;
        s[2] += wm * cs; s[3] += wm * sn;
        s[4] += wp * cs; s[5] += wp * sn;
        s[6] += w2 * cs; s[7] += w2 * sn;
        for (int q = 0; q < 3; q++) {
            s[8 + q] += wq * cs * d[q];
            s[11 + q] += wq * sn * d[q];
        }
    }
    lu_block_all<14>(s);
    const double Cq = s[0], Sq = s[1], Cm = s[2], Sm = s[3], Cp = s[4], Sp = s[5], C2 = s[6], S2 = s[7];
    double t[4] = {0, 0, 0, 0};   // Ff, Ffk2, d2UV1, d2UrR
    if (constrained) {
        for (int i = threadIdx.x; i < n; i += LU_THREADS) {
            double wq, wm, wp, w2, sn, cs, d[3];
            site(i, wq, wm, wp, w2, sn, cs, d);
            const double qc = wq * cs, qs = wq * sn, mc = wm * cs, ms = wm * sn, pc = wp * cs, ps = wp * sn;
            double val;
            if (KIND == 0)
                val = b * (qs * Cq - qc * Sq);
            else if (KIND == 1)
                val = LU_COU * b * ((qs * Cq - qc * Sq) + (mc * Cq + ms * Sq) - (qc * Cm + qs * Sm) + (ms * Cm - mc * Sm));
            else
                val = LU_COU * b * ((pc * Cq + ps * Sq) - (qc * Cp + qs * Sp) +
                                    (ps * (Cm + Cp) - pc * (Sm + Sp)) + (ms * Cp - mc * Sp));
            const double kd = kx * d[0] + ky * d[1] + kz * d[2];
            const double d2u1 = b * k2 * (qc * Cq + qs * Sq);
            const double d2u2 = b * k2 * ((qc * s[8] + qs * s[11]) * d[0] + (qc * s[9] + qs * s[12]) * d[1] +
                                          (qc * s[10] + qs * s[13]) * d[2]);
            t[0] += val * kd;
            t[1] += 2.0 * val * x * kd;
            t[2] += d2u1 * (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            t[3] += d2u2;
        }
        lu_block_all<4>(t);
    }
    if (threadIdx.x == 0) {
        double e, d1;
        if (KIND == 0) {
            e = c * (Cq * Cq + Sq * Sq);
            d1 = -e + e * x;
        } else if (KIND == 1) {
            const double UqQ = c * (Cq * Cq + Sq * Sq), UmqQ = c * (Sq * Cm - Cq * Sm), Umm = c * (Cm * Cm + Sm * Sm);
            e = (UqQ + 2.0 * UmqQ + Umm) * LU_COU;
            const double dqQ = b * (C2 * Cq + S2 * Sq), dqQm = b * (S2 * Cm - C2 * Sm);
            d1 = -e + e * x + (dqQ - 2.0 * UmqQ + dqQm - 2.0 * Umm) * LU_COU;
        } else {
            const double UmqQ = c * (Sq * Cp - Cq * Sp), Ump = c * (Cp * Cm + Sp * Sm);
            e = (UmqQ + Ump) * LU_COU;
            const double dpQ = c * (S2 * Cp - C2 * Sp), Upp = c * (Cp * Cp + Sp * Sp);
            const double Sk = 2.0 * UmqQ + 2.0 * Ump + Upp;
            d1 = (-Sk + Sk * x + (-2.0 * UmqQ + 2.0 * dpQ - 4.0 * Ump - 2.0 * Upp)) * LU_COU;
        }
        double d2 = 4.0 * e - 7.0 * e * x + e * x * x;
        if (constrained) {
            d1 += t[0];
            d2 += -6.0 * t[0] + t[1] - t[2] + t[3];
        }
        out[2 * (size_t)k] = d1;
        out[2 * (size_t)k + 1] = d2;
    }
}

// dU/dV of a set of torques as Multipole::torques2forces maps them
// (H sites: dU/du.u; O site: dU/du.u + dU/dv.v with half weight on the w
// rotation), one thread per site of each H O H molecule
__global__ void __launch_bounds__(LU_THREADS) k_lus_torque_dudv(int nmol, int n, const int *mol_off,
                                                                const int *mol_atoms, const double4 *pos4,
                                                                const long long *trq, double *out) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = g / 3, q = g - 3 * m;
    double v[1] = {0};
    if (m < nmol && mol_off[m + 1] - mol_off[m] == 3) {
        const int s = mol_off[m];
        const int h1 = mol_atoms[s], o = mol_atoms[s + 1], h2 = mol_atoms[s + 2];
        const double4 a = pos4[h1], bb = pos4[o], cc = pos4[h2];
        const V3 rh1 = v3(a.x, a.y, a.z), ro = v3(bb.x, bb.y, bb.z), rh2 = v3(cc.x, cc.y, cc.z);
        auto tq = [&](int id) {
            return v3((double)trq[id] * FRC_INV, (double)trq[n + id] * FRC_INV, (double)trq[2 * n + id] * FRC_INV);
        };
        if (q != 1) {
            const V3 rh = q == 0 ? rh1 : rh2;
            const V3 tau = tq(q == 0 ? h1 : h2);
            V3 u = rh - ro;
            const double ul = len(u);
            const V3 vv = fabs(u.x / ul) > 0.8666 ? v3(0, 1, 0) : v3(1, 0, 0);
            V3 w = crs(u, vv);
            const double wl = len(w);
            u = (1.0 / ul) * u;
            w = (1.0 / wl) * w;
            const V3 vxu = crs(vv, u), wxu = crs(w, u);
            const double vxuL = len(vxu), wxuL = len(wxu);
            const V3 dUdu = (-dot(vv, tau) / (vxuL * vxuL * ul)) * vxu + (-dot(w, tau) / (wxuL * wxuL * ul)) * wxu;
            v[0] = dot(dUdu, u) * ul;
        } else {
            const V3 tau = tq(o);
            V3 u = ro - rh1, vv = ro - rh2;
            V3 w = crs(u, vv);
            const double ul = len(u), vl = len(vv), wl = len(w);
            u = (1.0 / ul) * u;
            vv = (1.0 / vl) * vv;
            w = (1.0 / wl) * w;
            const V3 vxu = crs(vv, u), wxu = crs(w, u), wxv = crs(w, vv);
            const double vxuL = len(vxu), wxuL = len(wxu), wxvL = len(wxv);
            const V3 dUdu = (-dot(vv, tau) / (vxuL * vxuL * ul)) * vxu + (0.5 * -dot(w, tau) / (wxuL * wxuL * ul)) * wxu;
            const V3 dUdv = (-dot(u, tau) / (vxuL * vxuL * vl)) * (-vxu) + (0.5 * -dot(w, tau) / (wxvL * wxvL * vl)) * wxv;
            v[0] = dot(dUdu, u) * ul + dot(dUdv, vv) * vl;
        }
    }
    lu_block_out<1>(v, out);
}

// bonds: sum v r and sum (-2 r v + r^2 k) (BondForce.cpp:86-87, v = dU/dr;
// the second sum takes k itself for the AMOEBA form too); Urey-Bradley
// between the first and third site of every molecule, v = 2 kl (r - l0)
// (UreyBradleyForce.cpp:70-77)
__global__ void __launch_bounds__(LU_THREADS) k_lus_bonded(int nbond, const int4 *bonds, const double2 *bpar,
                                                           int amoeba, int nub, const int *mol_off,
                                                           const int *mol_atoms, double ub_k, double ub_l0,
                                                           const double4 *pos4, Box box, double *out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double v[4] = {0, 0, 0, 0};
    if (t < nbond) {
        const int4 bd = bonds[t];
        const double2 par = bpar[bd.z];
        const double4 p1 = pos4[bd.x], p2 = pos4[bd.y];
        double x = p1.x - p2.x, y = p1.y - p2.y, z = p1.z - p2.z;
        lu_min(x, y, z, box);
        const double r = sqrt(x * x + y * y + z * z), d = r - par.x, k = par.y;
        double val;
        if (amoeba) {
            const double c1 = 25.5, c2 = 379.3125;
            const double an = 1.0 - c1 * d + c2 * d * d;
            val = 2.0 * k * d * an + k * d * d * (-c1 + 2.0 * c2 * d);
        } else {
            val = k * d;
        }
        v[0] = val * r;
        v[1] = -2.0 * r * val + r * r * k;
    } else if (t < nbond + nub) {
        const int m = t - nbond;
        const int s0 = mol_off[m];
        if (mol_off[m + 1] - s0 >= 3) {
            const double4 p1 = pos4[mol_atoms[s0]], p2 = pos4[mol_atoms[s0 + 2]];
            double x = p1.x - p2.x, y = p1.y - p2.y, z = p1.z - p2.z;
            lu_min(x, y, z, box);
            const double r = sqrt(x * x + y * y + z * z);
            const double val = 2.0 * ub_k * (r - ub_l0);
            v[2] = val * r;
            v[3] = -2.0 * r * val + r * r * ub_k;
        }
    }
    lu_block_out<4>(v, out);
}

namespace {

// the first cnt * nv partials, summed per value in block order
int lus_fetch(Ctx &c, int cnt, int nv, double *tot) {
    std::vector<double> h((size_t)cnt * nv);
    if (cudaMemcpyAsync(h.data(), c.lus_buf, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c.stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(c.stream) != cudaSuccess)
        return SMD_ERR_CUDA;
    for (int q = 0; q < nv; q++) tot[q] = 0;
    for (int b = 0; b < cnt; b++)
        for (int q = 0; q < nv; q++) tot[q] += h[(size_t)b * nv + q];
    return SMD_OK;
}

// the intramolecular pass's per-molecule sums (at the start of the
// scratch), added in molecule order
int lus_fetch_mol(Ctx &c, double *tot) {
    std::vector<double> h(c.nmol);
    if (cudaMemcpyAsync(h.data(), c.lus_buf, c.nmol * sizeof(double), cudaMemcpyDeviceToHost, c.stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(c.stream) != cudaSuccess)
        return SMD_ERR_CUDA;
    *tot = 0;
    for (int m = 0; m < c.nmol; m++) *tot += h[m];
    return SMD_OK;
}

int lus_acc(Ctx &c, long long *h) {
    if (cudaMemcpyAsync(h, c.acc, ACC_COUNT * sizeof(long long), cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
        cudaStreamSynchronize(c.stream) != cudaSuccess)
        return SMD_ERR_CUDA;
    return SMD_OK;
}

int lus_clear(Ctx &c) {
    if (cudaMemsetAsync(c.acc, 0, ACC_COUNT * sizeof(long long), c.stream) != cudaSuccess ||
        cudaMemsetAsync(c.frc, 0, 3 * (size_t)c.n * sizeof(long long), c.stream) != cudaSuccess)
        return SMD_ERR_CUDA;
    if (c.trq && cudaMemsetAsync(c.trq, 0, 3 * (size_t)c.n * sizeof(long long), c.stream) != cudaSuccess)
        return SMD_ERR_CUDA;
    return SMD_OK;
}

// dU/dV of the torques now in c.trq
int lus_dudv(Ctx &c, double *dudv) {
    const int nb = (3 * c.nmol + LU_THREADS - 1) / LU_THREADS;
    k_lus_torque_dudv<<<nb, LU_THREADS, 0, c.stream>>>(c.nmol, c.n, c.mol_off, c.mol_atoms, c.pos4, c.trq, c.lus_buf);
    return lus_fetch(c, nb, 1, dudv);
}

double acc_trace(const long long *h) {
    return ((double)h[ACC_VIR] + (double)h[ACC_VIR + 4] + (double)h[ACC_VIR + 8]) * ACC_INV;
}

template <int KIND>
int lus_recip(Ctx &c, int constrained, double *d1, double *d2) {
    const int nk = c.rc.nk;
    *d1 = *d2 = 0;
    if (nk == 0) return SMD_OK;
    k_lus_recip<KIND><<<nk, LU_THREADS, 0, c.stream>>>(c.n, nk, c.rc.kvec, c.rc.kcoef, c.pos4, c.mol, c.lus_com,
                                                        c.type_q, c.mu, c.qd, c.pind, c.ew_alpha, constrained,
                                                        c.lus_buf);
    double t[2];
    int r = lus_fetch(c, nk, 2, t);
    *d1 = t[0];
    *d2 = t[1];
    return r;
}

}  // namespace

// out[SMD_LUSTIG_COUNT]: the fields of Ensemble::myLustig in declaration order
int lustig_all(Ctx &c, double *out) {
    for (int q = 0; q < SMD_LUSTIG_COUNT; q++) out[q] = 0;
    if ((c.vdw != VDW_NONE && c.vdw != VDW_LJ && c.vdw != VDW_BUFF) || c.rc.le) return SMD_ERR_ARG;
    // partials: 2 per k, LU_NSUM per site block, 4 per bond block, one per
    // molecule (the intramolecular pass)
    const size_t need = std::max<size_t>({(size_t)2 * std::max(c.rc.nk, 1),
                                          (size_t)LU_NSUM * ((c.n + LU_THREADS - 1) / LU_THREADS + 1),
                                          (size_t)4 * ((c.n + c.nmol + c.nbond + LU_THREADS - 1) / LU_THREADS + 1),
                                          (size_t)c.nmol});
    int r = lus_reserve(c, need);
    if (r) return r;
    const int save_prec = c.precision;
    c.precision = SMD_PREC_FP64;
    auto done = [&](int rc) {
        c.precision = save_prec;
        lus_clear(c);
        return rc;
    };
    const double V = c.box.L[0] * c.box.L[1] * c.box.L[2];
    const int constrained = c.clen2 != nullptr;
    const int nbs = (c.n + LU_THREADS - 1) / LU_THREADS;
    launch_nlist(c, !c.list_built);
    k_mol_com<<<(c.nmol + 127) / 128, 128, 0, c.stream>>>(c.nmol, c.mol_off, c.mol_atoms, c.pos4, c.mass, c.lus_com);
    long long h[ACC_COUNT];
    // ---- vdW
    if (c.vdw == VDW_LJ) {
        double lj[3];
        if ((r = lustig_lj(c, lj))) return done(r);
        out[SMD_LUS_LJ_U] = lj[0]; out[SMD_LUS_LJ_DU] = lj[1]; out[SMD_LUS_LJ_D2U] = lj[2];
    } else if (c.vdw == VDW_BUFF) {
        // BuffvdWForce: U, and sum (dU/dr) r over the virtual-site pairs,
        // minus the trace of the pass's share of Ensemble::virial
        const int ew = c.ewald_on, wf = c.wolf_on;
        c.ewald_on = 0; c.wolf_on = 0;
        if ((r = lus_clear(c))) return done(r);
        launch_pair(c);
        c.ewald_on = ew; c.wolf_on = wf;
        if ((r = lus_acc(c, h))) return done(r);
        out[SMD_LUS_LJ_U] = (double)h[ACC_E_VDW] * ACC_INV + c.e_lrc;
        out[SMD_LUS_LJ_DU] = -acc_trace(h) / (3.0 * V) + c.v_lrc / V;
    }
    // ---- site sums (surface terms): the multipoles and dipoles first
    if (c.mp_on) {
        launch_frames(c);
        if (c.ind_on) {
            launch_ind_solve(c);
            c.dip_version = c.cfg_version;
        }
    }
    double S[LU_NSUM];
    k_lus_sites<<<nbs, LU_THREADS, 0, c.stream>>>(c.n, c.pos4, c.mol, c.lus_com, c.type_q, c.mp_on ? c.mu : nullptr,
                                                   c.mp_on ? c.qd : nullptr, c.mp_on && c.ind_on ? c.pind : nullptr,
                                                   nullptr, c.lus_buf);
    if ((r = lus_fetch(c, nbs, LU_NSUM, S))) return done(r);
    auto dot3 = [](const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
    const double coeff = 2.0 * 3.14159265358979323846 / (3.0 * V), vr = 1.0 / V;
    // surfSecDeriv form of all three classes, from q r and q R sums
    auto surf2 = [&](const double *qr, const double *qR) {
        return constrained ? 2.0 * coeff * vr * vr * dot3(qr, qr) - 16.0 * coeff * vr * vr * dot3(qr, qR) / 9.0 +
                                 2.0 * coeff * vr * vr * dot3(qR, qR) / 9.0
                           : 4.0 * coeff * vr * vr * dot3(qr, qr) / 9.0;
    };
    // ---- point charges
    if (c.ewald_on) {
        k_lus_ewald_real<<<nbs, LU_THREADS, 0, c.stream>>>(c.n, c.pl.nbr, c.pl.nnbr, c.pos4, c.mol, c.lus_com,
                                                            c.type_q, c.box, c.ew_rc2, c.ew_alpha, constrained,
                                                            c.lus_buf);
        double t[3];
        if ((r = lus_fetch(c, nbs, 2, t))) return done(r);
        out[SMD_LUS_REAL] = 0.5 * t[0];
        out[SMD_LUS_REAL2] = 0.5 * t[1];
        const int nbm = (c.nmol + LU_THREADS - 1) / LU_THREADS;
        k_lus_ewald_intra<<<nbm, LU_THREADS, 0, c.stream>>>(c.nmol, c.mol_off, c.mol_atoms, c.excl_off, c.excl,
                                                             c.pos4, c.type_q, c.box, c.ew_alpha, c.lus_buf);
        if ((r = lus_fetch(c, nbm, 3, t))) return done(r);
        out[SMD_LUS_INTRAVIR] = -t[0];
        if (!constrained) {
            out[SMD_LUS_MOL] = t[1] / (3.0 * V);
            out[SMD_LUS_MOL2] = t[2] / (9.0 * V * V);
        }
        if (c.surface_on) {
            const double *qr = S, *qR = S + 3;
            out[SMD_LUS_SURF] = constrained ? -coeff * vr * dot3(qr, qr) + 2.0 * coeff * vr * dot3(qr, qR) / 3.0
                                            : -coeff * vr * dot3(qr, qr) / 3.0;
            out[SMD_LUS_SURF2] = surf2(qr, qR);
        }
        if ((r = lus_recip<0>(c, constrained, &out[SMD_LUS_LONG], &out[SMD_LUS_LONG2]))) return done(r);
    }
    // ---- the Wolf sum of the charges
    if (c.wolf_on) {
        const double4 *qp = c.pos4;
        if (c.wolf_msites) {
            launch_wolf_sites(c);
            qp = c.wpos4;
        }
        k_lus_wolf<<<nbs, LU_THREADS, 0, c.stream>>>(c.n, c.pl.nbr, c.pl.nnbr, qp, c.mol, c.lus_com, c.type_q, c.box,
                                                      c.wolf_rc, c.wolf_alpha, c.lus_buf);
        double t[2];
        if ((r = lus_fetch(c, nbs, 2, t))) return done(r);
        out[SMD_LUS_REAL] = 0.5 * t[0];
        out[SMD_LUS_REAL2] = 0.5 * t[1];
    }
    // ---- multipoles and induced dipoles (each part's torques on their own)
    if (c.mp_on) {
        double du;
        // real space: -ke sum f_ij.r_ij (r_ij = r_i - r_j) is ke times the trace
        // of the pass's share of Ensemble::virial (which subtracts f_ij r_ij)
        if ((r = lus_clear(c))) return done(r);
        launch_mp_real_only(c);
        if ((r = lus_acc(c, h)) || (r = lus_dudv(c, &du))) return done(r);
        out[SMD_LUS_REAL] = LU_COU * acc_trace(h) + du;
        // intramolecular correction: forces and torques of flexible molecules
        if (!constrained) {
            if ((r = lus_clear(c))) return done(r);
            launch_intra_flex_lus(c, true, false, c.lus_buf);
            double fr;
            if ((r = lus_fetch_mol(c, &fr)) || (r = lus_dudv(c, &du))) return done(r);
            out[SMD_LUS_MOL] = (-LU_COU * fr + du) / (3.0 * V);
        }
        if (c.surface_on) {
            if ((r = lus_clear(c))) return done(r);
            launch_surface(c, false, true, false);
            if ((r = lus_acc(c, h)) || (r = lus_dudv(c, &du))) return done(r);
            const double es = (double)h[ACC_E_SURF] * ACC_INV;
            const double *qr = S + 6, *qR = S + 9;
            const double qm[3] = {S[6] + S[12], S[7] + S[13], S[8] + S[14]};
            out[SMD_LUS_SURF] = -es * vr + 2.0 * coeff * vr * dot3(qm, qr) * LU_COU / 3.0 + du * vr / 3.0;
            out[SMD_LUS_SURF2] = surf2(qr, qR);
        }
        if ((r = lus_clear(c))) return done(r);
        launch_mp_long(c);
        if ((r = lus_dudv(c, &du))) return done(r);
        if ((r = lus_recip<1>(c, constrained, &out[SMD_LUS_LONG], &out[SMD_LUS_LONG2]))) return done(r);
        out[SMD_LUS_LONG] += du;
        if (c.ind_on) {
            if ((r = lus_clear(c))) return done(r);
            launch_ind_self_only(c);
            if ((r = lus_dudv(c, &du))) return done(r);
            out[SMD_LUS_POL_SELF] = du;
            if ((r = lus_clear(c))) return done(r);
            launch_ind_real_only(c);
            if ((r = lus_acc(c, h)) || (r = lus_dudv(c, &du))) return done(r);
            out[SMD_LUS_POL_REAL] = LU_COU * acc_trace(h) + du;
            if (!constrained) {
                if ((r = lus_clear(c))) return done(r);
                launch_intra_flex_lus(c, false, true, c.lus_buf);
                double fr;
                if ((r = lus_fetch_mol(c, &fr))) return done(r);
                out[SMD_LUS_POL_MOL] = -LU_COU * fr / (3.0 * V);
            }
            if (c.surface_on) {
                const double *qr = S + 6, *qR = S + 9, *ms = S + 12, *ps = S + 15;
                const double d1 = -coeff * vr * (2.0 * dot3(qr, ps) + 2.0 * dot3(ms, ps) + dot3(ps, ps) - 2.0 * S[18] - S[19]);
                const double d2 = 2.0 * coeff * vr * dot3(qr, ps) / 3.0;
                out[SMD_LUS_POL_SURF] = LU_COU * (d1 + d2);
                out[SMD_LUS_POL_SURF2] = surf2(qr, qR);
            }
            if ((r = lus_clear(c))) return done(r);
            launch_ind_long(c);
            if ((r = lus_dudv(c, &du))) return done(r);
            if ((r = lus_recip<2>(c, constrained, &out[SMD_LUS_POL_LONG], &out[SMD_LUS_POL_LONG2]))) return done(r);
            out[SMD_LUS_POL_LONG] += du;
        }
    }
    // ---- bonds and Urey-Bradley
    if (c.nbond > 0 || c.ub_on) {
        const int nub = c.ub_on ? c.nmol : 0;
        const int nb = (c.nbond + nub + LU_THREADS - 1) / LU_THREADS;
        k_lus_bonded<<<nb, LU_THREADS, 0, c.stream>>>(c.nbond, c.bonds, c.bond_par, c.bond_form == 2 ? 1 : 0, nub,
                                                       c.mol_off, c.mol_atoms, c.ub_k, c.ub_l0, c.pos4, c.box,
                                                       c.lus_buf);
        double t[4];
        if ((r = lus_fetch(c, nb, 4, t))) return done(r);
        out[SMD_LUS_BOND] = t[0]; out[SMD_LUS_BOND2] = t[1];
        out[SMD_LUS_UB] = t[2]; out[SMD_LUS_UB2] = t[3];
    }
    return done(SMD_OK);
}

}  // namespace smd
