// Nose-Hoover chain velocity-Verlet integrator (NVT), optionally with SLLOD
// planar Couette shear and Lees-Edwards images.
//
// Chain: NHIntegrator::chain (src/integrators/NHIntegrator.cpp:1814-1912),
// 4 links, nc = 5 multiple steps, Suzuki-Yoshida weights (1/(2 - 2^(1/3)),
// 1 - 2 w, w), Q_0 = Nf kT tau^2, Q_k = kT tau^2 (:113-119).  With the
// barostat (smd_set_barostat: the reference's NpT run) the chain carries the
// isotropic MTK degree of freedom vlog with mass W = (Nf + 1) kT tau_P^2
// (:119): G_0 = 2 K + W vlog^2 - (Nf + 1) kT, G_log = (2 K (1 + 3/Nf) +
// 3 V (P_vir - P)) / W, and the velocity scale exp(-(v_1 + (1 + 3/Nf) vlog)
// dt/2); the drift is r' = r e^(2h) + v e^h S(h) dt with h = vlog dt/2 and
// S the sinh(h)/h series to h^8, and the box edges scale by e^(2h)
// (:390-419).  P_vir is the reference's -molVirt of the previous forces
// (:382, :635): the Lustig volume derivative of the pair energy,
// sum r du/dr / 3V, minus that of the tail correction (LJForce.cpp:136-250,
// 297-327), the trace of the pair virial here.  Without the barostat vlog
// stays 0 and the first link sees Nf kT: constant volume.
// Step order as NHIntegrator::run (:380-408, :628-644):
//   k_nhc_chain   chain half step on the kinetic energy of v (one thread),
//                 Lees-Edwards offset delta += g Ly dt, the list test limit
//   k_nhc_first   v *= s; [SLLOD v_x -= g dt/2 v_y]; v += dt/2 F/m; drift
//                 x += dt v_x + g dt (y + dt v_y / 2), y, z += dt v; wrap
//                 (y first, moving x by -/+ delta); displacement test
//   pair list (if flagged), forces at t + dt
//   k_nhc_second  v += dt/2 F/m; [SLLOD half step]; kinetic sums; the last
//                 block runs the second chain half step, the observables and
//                 the pressure tensors (peculiar velocities under shear)
//   k_nhc_scale   v *= s
// SLLOD (no reference code; Evans and Morriss, Statistical Mechanics of
// Nonequilibrium Liquids, ch. 6): v is the peculiar velocity, the streaming
// and the -g v_y e_x term are integrated exactly over their sub-steps.
// The pair list stays valid while 2 max|displacement| + |delta - delta_build|
// < skin: the displacement limit of each step is ((skin - |d delta|)/2)^2 and
// a rebuild is forced when that is not positive.
#include "smd_ctx.cuh"

namespace smd {

constexpr double KB_N = 0.0083145112;  // BOLTZMAN, src/NEMD_defs.h:108
constexpr int NHC_BLOCK = 128;

enum { Q_KE = 0, Q_AP = 1 /*6*/, Q_KEM = 7, Q_MP = 8 /*6*/, Q_MC = 14 /*9*/, NQ = 23 };

struct NhcArgs {
    int n, nmol, nblocks;
    const int *mol_off, *mol_atoms;
    double4 *pos4, *vel4, *disp4;
    int4 *fixq;
    int write_fixq;
    const long long *frc;
    long long *acc;
    double *scal, *partials;
    unsigned int *ticket, *status;
    int *flags;
    smd_observables *obs;
    double *series;
    int series_cap;
    double *avg;           // running sums of the observables (may be null)
    double *wrap;          // [3][nmol] box shifts applied to each molecule since the last upload
    Box box;
    double dt, kT, nf, tau, gamma, skin, volume;
    int atom_ndf, mol_ndf;
    double e_lrc, v_lrc, e_self;
    // barostat (npt): the box on the device, target pressure, W, the tail
    // correction's energy times volume, the smallest box scale the cell
    // grid covers and the box it was built for
    int npt;
    Box *dbox;
    double press, wbar, lrc_k, smin, L0[3];
};

// one chain half step; returns the velocity scale (vnh in scal[SC_VNH..+3]);
// with the barostat also vlog, driven by the virial pressure pvir
__device__ double chain_half(double *vnh, double ekin, const NhcArgs &a, double &vlog, double pvir, double vol) {
    double qnh[4];
    for (int k = 0; k < 4; k++) qnh[k] = a.kT * a.tau * a.tau;
    qnh[0] *= a.nf;
    const double w0 = 1.0 / (2.0 - cbrt(2.0));
    const double wj[3] = {w0, 1.0 - 2.0 * w0, w0};
    const int nc = 5;
    const double gkt = a.npt ? (a.nf + 1.0) * a.kT : a.nf * a.kT;
    const double odnf = 1.0 + 3.0 / a.nf, diff = pvir - a.press;
    double scale = 1.0, g[4];
    for (int i = 0; i < nc; i++)
        for (int j = 0; j < 3; j++) {
            const double dts = wj[j] * a.dt / nc, dts2 = 0.5 * dts, dts4 = 0.25 * dts, dts8 = 0.125 * dts;
            double ex;
            g[3] = (qnh[2] * vnh[2] * vnh[2] - a.kT) / qnh[3];
            vnh[3] += g[3] * dts4;
            g[2] = (qnh[1] * vnh[1] * vnh[1] - a.kT) / qnh[2];
            ex = exp(-vnh[3] * dts8);
            vnh[2] = ex * (vnh[2] * ex + g[2] * dts4);
            g[1] = (qnh[0] * vnh[0] * vnh[0] - a.kT) / qnh[1];
            ex = exp(-vnh[2] * dts8);
            vnh[1] = ex * (vnh[1] * ex + g[1] * dts4);
            g[0] = (2.0 * ekin + (a.npt ? a.wbar * vlog * vlog : 0.0) - gkt) / qnh[0];
            ex = exp(-vnh[1] * dts8);
            vnh[0] = ex * (vnh[0] * ex + g[0] * dts4);
            if (a.npt) {
                const double glog = (2.0 * ekin * odnf + 3.0 * vol * diff) / a.wbar;
                ex = exp(-vnh[0] * dts8);
                vlog = ex * (vlog * ex + glog * dts4);
                ex = exp(-(vnh[0] + vlog * odnf) * dts2);
            } else {
                ex = exp(-vnh[0] * dts2);
            }
            scale *= ex;
            ekin = ekin * ex * ex;
            if (a.npt) {
                const double glog = (2.0 * ekin * odnf + 3.0 * vol * diff) / a.wbar;
                ex = exp(-vnh[0] * dts8);
                vlog = ex * (vlog * ex + glog * dts4);
            }
            g[0] = (2.0 * ekin + (a.npt ? a.wbar * vlog * vlog : 0.0) - gkt) / qnh[0];
            ex = exp(-vnh[1] * dts8);
            vnh[0] = ex * (vnh[0] * ex + g[0] * dts4);
            g[1] = (qnh[0] * vnh[0] * vnh[0] - a.kT) / qnh[1];
            ex = exp(-vnh[2] * dts8);
            vnh[1] = ex * (vnh[1] * ex + g[1] * dts4);
            g[2] = (qnh[1] * vnh[1] * vnh[1] - a.kT) / qnh[2];
            ex = exp(-vnh[3] * dts8);
            vnh[2] = ex * (vnh[2] * ex + g[2] * dts4);
            g[3] = (qnh[2] * vnh[2] * vnh[2] - a.kT) / qnh[3];
            vnh[3] += g[3] * dts4;
        }
    return scale;
}

__global__ void k_nhc_chain(NhcArgs a) {
    if (threadIdx.x != 0) return;
    double vnh[4];
    for (int k = 0; k < 4; k++) vnh[k] = a.scal[SC_VNH + k];
    double vlog = a.scal[SC_VLOG];
    const double s = chain_half(vnh, a.scal[SC_EKIN], a, vlog, -a.scal[SC_MOLVIRT], a.scal[SC_VOL]);
    for (int k = 0; k < 4; k++) a.scal[SC_VNH + k] = vnh[k];
    a.scal[SC_SCALE] = s;
    if (a.npt) {
        // the drift's factors and the scaled box (NHIntegrator.cpp:390-419)
        a.scal[SC_VLOG] = vlog;
        const double term = 0.5 * a.dt * vlog, ex = exp(term), ex2 = ex * ex, arg2 = term * term;
        const double e2 = 1.0 / 6.0, e4 = e2 / 20.0, e6 = e4 / 42.0, e8 = e6 / 72.0;
        const double poly = ex * (1.0 + arg2 * (e2 + arg2 * (e4 + arg2 * (e6 + arg2 * e8)))) * a.dt;
        a.scal[SC_X2] = ex2;
        a.scal[SC_POLY] = poly;
        Box b = *a.dbox;
        bool small = false;
        for (int d = 0; d < 3; d++) {
            b.L[d] *= ex2;
            b.half[d] = 0.5 * b.L[d];
            b.inv[d] = 1.0 / b.L[d];
            small |= b.L[d] < a.smin * a.L0[d];
        }
        *a.dbox = b;
        a.scal[SC_VOL] = b.L[0] * b.L[1] * b.L[2];
        if (small) atomicOr(a.status, ST_BOX);
    }
    double lim = 0.5 * a.skin;
    if (a.gamma != 0.0) {
        const double Lx = a.box.L[0];
        double d = fmod(a.scal[SC_LE] + a.gamma * a.box.L[1] * a.dt, Lx);
        if (d < 0) d += Lx;
        a.scal[SC_LE] = d;
        double dd = fabs(d - a.scal[SC_LE_B]);
        dd = fmin(dd, Lx - dd);
        lim = 0.5 * (a.skin - dd);
        if (!(lim > 0)) {
            a.flags[0] = 1;
            lim = 0;
        }
    }
    a.scal[SC_DRMAX] = lim * lim;
}

__device__ __forceinline__ double3 nhc_force(const long long *frc, int n, int i) {
    return make_double3((double)frc[i] * FRC_INV, (double)frc[n + i] * FRC_INV, (double)frc[2 * n + i] * FRC_INV);
}

// one thread per molecule: scale, kick, drift, wrap, list test, box fractions
__global__ void __launch_bounds__(NHC_BLOCK) k_nhc_first(NhcArgs a) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const double s = a.scal[SC_SCALE], delta = a.scal[SC_LE], drmax = a.scal[SC_DRMAX];
    const double hdt = 0.5 * a.dt, g = a.gamma;
    const Box bx = a.npt ? *a.dbox : a.box;
    const double x2 = a.npt ? a.scal[SC_X2] : 1.0, poly = a.npt ? a.scal[SC_POLY] : a.dt;
    bool rebuild = false, bad = false;
    if (m < a.nmol) {
        const int s0 = a.mol_off[m], s1 = a.mol_off[m + 1];
        double cx = 0, cy = 0, cz = 0, M = 0;
        for (int k = s0; k < s1; k++) {
            const int at = a.mol_atoms[k];
            double4 v = a.vel4[at];   // w: 1/m
            const double3 f = nhc_force(a.frc, a.n, at);
            v.x *= s; v.y *= s; v.z *= s;
            if (g != 0.0) v.x -= g * hdt * v.y;
            v.x += hdt * v.w * f.x; v.y += hdt * v.w * f.y; v.z += hdt * v.w * f.z;
            double4 p = a.pos4[at];
            double drx, dry, drz;
            if (a.npt) {
                // r' = r e^(2h) + v e^h S(h) dt
                drx = (p.x * x2 + v.x * poly) - p.x;
                dry = (p.y * x2 + v.y * poly) - p.y;
                drz = (p.z * x2 + v.z * poly) - p.z;
                p.x = p.x * x2 + v.x * poly; p.y = p.y * x2 + v.y * poly; p.z = p.z * x2 + v.z * poly;
            } else {
                drx = a.dt * v.x + g * a.dt * (p.y + hdt * v.y);
                dry = a.dt * v.y; drz = a.dt * v.z;
                p.x += drx; p.y += dry; p.z += drz;
            }
            double4 d = a.disp4[at];
            d.x += drx; d.y += dry; d.z += drz;
            if (d.x * d.x + d.y * d.y + d.z * d.z > drmax) rebuild = true;
            if (!isfinite(p.x + p.y + p.z)) bad = true;
            a.vel4[at] = v;
            a.disp4[at] = d;
            a.pos4[at] = p;
            const double mass = 1.0 / v.w;
            cx += mass * p.x; cy += mass * p.y; cz += mass * p.z;
            M += mass;
        }
        cx /= M; cy /= M; cz /= M;
        // wrap the centre of mass: y first (Lees-Edwards), then x and z
        double wx = 0, wy = 0;
        if (cy >= bx.half[1]) { wy = -bx.L[1]; wx = -delta; }
        else if (cy < -bx.half[1]) { wy = bx.L[1]; wx = delta; }
        if (g == 0.0) wx = 0;
        wx = pbc1(cx + wx, bx.L[0], bx.half[0]) - cx;
        const double wz = pbc1(cz, bx.L[2], bx.half[2]) - cz;
        // the shifts so far, per molecule: Atom::realPos = position - shift
        if (a.wrap && (wx != 0.0 || wy != 0.0 || wz != 0.0)) {
            a.wrap[m] += wx;
            a.wrap[a.nmol + m] += wy;
            a.wrap[2 * a.nmol + m] += wz;
        }
        for (int k = s0; k < s1; k++) {
            const int at = a.mol_atoms[k];
            double4 p = a.pos4[at];
            if (wx != 0.0 || wy != 0.0 || wz != 0.0) {
                p.x += wx; p.y += wy; p.z += wz;
                a.pos4[at] = p;
            }
            if (a.write_fixq) a.fixq[at] = site_frac(p, a.box, g != 0.0, delta);
        }
    }
    if (__any_sync(0xffffffffu, rebuild) && (threadIdx.x & 31) == 0) atomicOr(&a.flags[0], 1);
    if (bad) atomicOr(a.status, ST_NAN);
}

// one thread per molecule: second half kick, kinetic sums; last block:
// chain half step, observables, pressure tensors
__global__ void __launch_bounds__(NHC_BLOCK) k_nhc_second(NhcArgs a) {
    __shared__ double s_part[NHC_BLOCK / 32][NQ];
    __shared__ bool s_last;
    double part[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) part[q] = 0.0;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const double hdt = 0.5 * a.dt, g = a.gamma;
    if (m < a.nmol) {
        const int s0 = a.mol_off[m], s1 = a.mol_off[m + 1];
        double px = 0, py = 0, pz = 0, cx = 0, cy = 0, cz = 0, M = 0;
        for (int k = s0; k < s1; k++) {
            const int at = a.mol_atoms[k];
            double4 v = a.vel4[at];
            const double3 f = nhc_force(a.frc, a.n, at);
            v.x += hdt * v.w * f.x; v.y += hdt * v.w * f.y; v.z += hdt * v.w * f.z;
            if (g != 0.0) v.x -= g * hdt * v.y;
            a.vel4[at] = v;
            const double mass = 1.0 / v.w;
            const double mx = v.x * mass, my = v.y * mass, mz = v.z * mass;
            part[Q_KE] += (v.x * v.x + v.y * v.y + v.z * v.z) * mass;
            part[Q_AP + 0] += mx * v.x; part[Q_AP + 1] += mx * v.y; part[Q_AP + 2] += mx * v.z;
            part[Q_AP + 3] += my * v.y; part[Q_AP + 4] += my * v.z; part[Q_AP + 5] += mz * v.z;
            px += mx; py += my; pz += mz;
            const double4 p = a.pos4[at];
            cx += mass * p.x; cy += mass * p.y; cz += mass * p.z;
            M += mass;
        }
        cx /= M; cy /= M; cz /= M;
        part[Q_KEM] += (px * px + py * py + pz * pz) / M;
        part[Q_MP + 0] += px * px / M; part[Q_MP + 1] += px * py / M; part[Q_MP + 2] += px * pz / M;
        part[Q_MP + 3] += py * py / M; part[Q_MP + 4] += py * pz / M; part[Q_MP + 5] += pz * pz / M;
        for (int k = s0; k < s1; k++) {
            const int at = a.mol_atoms[k];
            const double3 f = nhc_force(a.frc, a.n, at);
            const double4 p = a.pos4[at];
            const double rx = p.x - cx, ry = p.y - cy, rz = p.z - cz;
            part[Q_MC + 0] += f.x * rx; part[Q_MC + 1] += f.y * rx; part[Q_MC + 2] += f.z * rx;
            part[Q_MC + 3] += f.x * ry; part[Q_MC + 4] += f.y * ry; part[Q_MC + 5] += f.z * ry;
            part[Q_MC + 6] += f.x * rz; part[Q_MC + 7] += f.y * rz; part[Q_MC + 8] += f.z * rz;
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NQ; q++) {
        const double v = warp_sum(part[q]);
        if (lane == 0) s_part[w][q] = v;
    }
    __syncthreads();
    if (threadIdx.x < NQ) {
        double v = 0;
        for (int q = 0; q < NHC_BLOCK / 32; q++) v += s_part[q][threadIdx.x];
        a.partials[(size_t)blockIdx.x * NQ + threadIdx.x] = v;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(a.ticket, 1u) == (unsigned)a.nblocks - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // last block: totals in a fixed order, then one thread finishes
    __shared__ double s_acc[NHC_BLOCK][NQ + 1];
    __shared__ double tot[NQ];
    for (int q = 0; q < NQ; q++) {
        double v = 0;
        for (int b = threadIdx.x; b < a.nblocks; b += NHC_BLOCK) v += __ldcg(&a.partials[(size_t)b * NQ + q]);
        s_acc[threadIdx.x][q] = v;
    }
    __syncthreads();
    for (int o = NHC_BLOCK / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int q = 0; q < NQ; q++) s_acc[threadIdx.x][q] += s_acc[threadIdx.x + o][q];
        __syncthreads();
    }
    if (threadIdx.x < NQ) tot[threadIdx.x] = s_acc[0][threadIdx.x];
    __syncthreads();
    if (threadIdx.x == 0) {
        double vnh[4];
        for (int k = 0; k < 4; k++) vnh[k] = a.scal[SC_VNH + k];
        double vlog = a.scal[SC_VLOG];
        const double vol = a.npt ? a.scal[SC_VOL] : a.volume;
        const double s = chain_half(vnh, 0.5 * tot[Q_KE], a, vlog, -a.scal[SC_MOLVIRT], vol);
        for (int k = 0; k < 4; k++) a.scal[SC_VNH + k] = vnh[k];
        a.scal[SC_SCALE] = s;
        // the tail correction of this volume (LJForce::long_range_correct,
        // recomputed every evaluation in NpT: E = K / V, virial -2 E, dU/dV = -2 E / V)
        const double e_lrc = a.npt ? a.lrc_k / vol : a.e_lrc;
        const double v_lrc = a.npt ? -2.0 * e_lrc : a.v_lrc;
        if (a.npt) {
            a.scal[SC_VLOG] = vlog;
            // molVirt = -(sum r du/dr) / 3V + dU_lrc/dV (NHIntegrator.cpp:635)
            double tr = 0.0;
            for (int q = 0; q < 9; q += 4)
                tr += ((double)__ldcg(&a.acc[ACC_VIR + q]) + (double)__ldcg(&a.acc[ACC_LVIR + q])) * ACC_INV;
            a.scal[SC_MOLVIRT] = -tr / (3.0 * vol) + v_lrc / vol;
        }
        const double s2 = s * s;
        const double keA = tot[Q_KE] * s2, keM = tot[Q_KEM] * s2;
        a.scal[SC_EKIN] = 0.5 * keA;
        smd_observables &o = *a.obs;
        o.zeta = vnh[0];
        o.ke_atom = 0.5 * keA;
        o.ke_mol = 0.5 * keM;
        o.t_atom = keA / (a.atom_ndf * KB_N);
        o.t_mol = keM / (a.mol_ndf * KB_N);
        const long long *acc = a.acc;
        long long accv[ACC_COUNT];
        for (int q = 0; q < ACC_COUNT; q++) accv[q] = __ldcg(&acc[q]);
        double en[SMD_E_COUNT];
        acc_energies(accv, e_lrc, a.e_self, en);
        double ep = 0;
        for (int q = 0; q < SMD_E_COUNT; q++) {
            o.energy[q] = en[q];
            ep += en[q];
        }
        o.e_potential = ep;
        const int sym[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
        for (int q = 0; q < 9; q++) {
            double vir = ((double)__ldcg(&acc[ACC_VIR + q]) + (double)__ldcg(&acc[ACC_LVIR + q])) * ACC_INV;
            if (q == 0 || q == 4 || q == 8) vir -= v_lrc;
            o.mol_pressure[q] = (tot[Q_MP + sym[q]] * s2 + vir - tot[Q_MC + q]) / vol;
            o.atom_pressure[q] = (tot[Q_AP + sym[q]] * s2 + vir) / vol;
            o.virial[q] = vir;
        }
        o.volume = vol;
        o.shear_offset = a.scal[SC_LE];
        o.step += 1;
        o.list_updates = a.flags[1];
        o.pairs_in_cutoff = __ldcg(&acc[ACC_NPAIR]) / 2;
        o.status = *a.status;
        if (a.series_cap > 0) {
            const long long slot = (o.step - 1) % a.series_cap;
            double *r = a.series + slot * 5;
            r[0] = o.e_potential; r[1] = o.ke_atom; r[2] = o.t_atom; r[3] = o.zeta;
            r[4] = o.atom_pressure[1];   // xy: the shear stress under SLLOD
        }
        accumulate_averages(a.avg, o);
        *a.ticket = 0;
    }
    __syncthreads();
    if (threadIdx.x < ACC_COUNT) a.acc[threadIdx.x] = 0;
}

__global__ void k_nhc_scale(int n, double4 *vel4, const double *scal) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double s = scal[SC_SCALE];
    double4 v = vel4[i];
    v.x *= s; v.y *= s; v.z *= s;
    vel4[i] = v;
}

// start: kinetic energy of the initial velocities, chain at rest, delta = 0
__global__ void k_nhc_start(int n, const double4 *vel4, double *scal, double skin, long long *acc) {
    __shared__ double s[256];
    double k = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double4 v = vel4[i];
        k += (v.x * v.x + v.y * v.y + v.z * v.z) / v.w;
    }
    s[threadIdx.x] = k;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        scal[SC_EKIN] = 0.5 * s[0];
        for (int q = 0; q < 4; q++) scal[SC_VNH + q] = 0.0;
        scal[SC_SCALE] = 1.0;
        scal[SC_LE] = 0.0;
        scal[SC_LE_B] = 0.0;
        scal[SC_DRMAX] = 0.25 * skin * skin;
    }
    __syncthreads();
    if (threadIdx.x < ACC_COUNT) acc[threadIdx.x] = 0;
}

namespace {
NhcArgs nhc_args(Ctx &c) {
    NhcArgs a;
    a.n = c.n; a.nmol = c.nmol;
    a.nblocks = (c.nmol + NHC_BLOCK - 1) / NHC_BLOCK;
    a.mol_off = c.mol_off; a.mol_atoms = c.mol_atoms;
    a.pos4 = c.pos4; a.vel4 = c.vel4; a.disp4 = c.disp4;
    a.fixq = c.fixq; a.write_fixq = c.precision == SMD_PREC_MIXED;
    a.frc = c.frc; a.acc = c.acc; a.scal = c.scal; a.partials = c.partials;
    a.ticket = c.ticket; a.status = c.status; a.flags = c.flags; a.obs = c.obs;
    a.series = c.series; a.series_cap = c.series_cap;
    a.avg = c.avg;
    a.wrap = c.wrap;
    a.box = c.box;
    a.dt = c.ip.timestep; a.kT = KB_N * c.ip.temperature; a.nf = c.ip.atom_ndf; a.tau = c.ip.coupl_const;
    a.gamma = c.ip.strain_rate; a.skin = c.cut_buffer;
    a.volume = c.box.L[0] * c.box.L[1] * c.box.L[2];
    a.atom_ndf = c.ip.atom_ndf; a.mol_ndf = c.ip.mol_ndf;
    a.e_lrc = c.e_lrc; a.v_lrc = c.v_lrc; a.e_self = c.e_self;
    a.npt = c.npt;
    a.dbox = c.dbox;
    a.press = c.npt_press;
    a.wbar = (c.ip.atom_ndf + 1.0) * a.kT * c.npt_tau * c.npt_tau;
    a.lrc_k = c.npt_lrc_k;
    a.smin = c.npt_smin;
    for (int d = 0; d < 3; d++) a.L0[d] = c.grid.L0[d];
    return a;
}
}  // namespace

void launch_nhc_first(Ctx &c) {
    NhcArgs a = nhc_args(c);
    k_nhc_chain<<<1, 32, 0, c.stream>>>(a);
    k_nhc_first<<<a.nblocks, NHC_BLOCK, 0, c.stream>>>(a);
}

void launch_nhc_second(Ctx &c) {
    NhcArgs a = nhc_args(c);
    k_nhc_second<<<a.nblocks, NHC_BLOCK, 0, c.stream>>>(a);
    k_nhc_scale<<<(c.n + 255) / 256, 256, 0, c.stream>>>(c.n, c.vel4, c.scal);
}

void launch_nhc_start(Ctx &c) {
    k_nhc_start<<<1, 256, 0, c.stream>>>(c.n, c.vel4, c.scal, c.cut_buffer, c.acc);
}

}  // namespace smd
