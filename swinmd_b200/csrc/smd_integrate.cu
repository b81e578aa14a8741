// Leap-frog Nose-Hoover integrator step, observables and thermostat update.
//
// One thread per molecule carries out, for the molecule's sites, the
// unconstrained update of LFIntegrator::run (src/integrators/LFIntegrator.cpp:
// 588-642): the implicit Nose-Hoover velocity iteration
//     v+ = v- + dt (F/m - zeta v),  v = (v+ + v-)/2     (to 1e-10, <= 10 passes)
// then r += dt v+, followed by the molecular centre of mass and momenta
// (:646-686), the pair-list displacement test (:307-315) and the molecule
// wrap into the box (:897-912).  The centre-of-mass drift removal the
// reference applies to v- at the start of the next step (:359-379) is
// applied here at the start of that step's update; forces do not depend on
// velocities, so the order is equivalent.
//
// Per-block partial sums (kinetic energies, kinetic pressure tensors, the
// molecular virial correction, sum m v-) are combined by the last block to
// finish (fixed summation order, so the result is deterministic); it then
// updates zeta (:688-722), temperatures, energies, the pressure tensors of
// Integrator::computePressure (src/Integrator.cpp:205-270), and clears the
// force accumulators for the next step.
#include "smd_ctx.cuh"

namespace smd {

// scal[] layout
enum {
    SC_FNH = 0,     // zeta used by the next velocity update
    SC_FNHMI = 1,   // zeta(t - dt/2)
    SC_VOM = 2,     // 3: centre-of-mass velocity of v- to remove
    SC_APPLY = 5,   // nonzero: remove SC_VOM at the next update
    SC_COUNT = 8
};

constexpr int NPART = 26;
constexpr int INT_BLOCK = 128;
constexpr double KB = 0.0083145112;  // BOLTZMAN, src/NEMD_defs.h:108

struct IntArgs {
    int n, nmol, nblocks;
    const int *mol_off, *mol_atoms;
    double4 *pos4, *vel4, *vtm4, *disp4;
    const long long *frc;
    long long *acc;
    double *scal, *partials;
    unsigned int *ticket, *status;
    int *flags;
    smd_observables *obs;
    double *series;
    int series_cap;
    Box box;
    double dt, temperature, tau, drmax, total_mass, volume;
    int thermostat, atom_thermo, atom_ndf, mol_ndf;
    double e_lrc, v_lrc, e_self;
};

__device__ __forceinline__ double3 fetch_force(const long long *frc, int n, int a) {
    return make_double3((double)frc[a] * FRC_INV, (double)frc[n + a] * FRC_INV,
                        (double)frc[2 * n + a] * FRC_INV);
}

__global__ void __launch_bounds__(INT_BLOCK) k_integrate(IntArgs a) {
    __shared__ double s_part[INT_BLOCK / 32][NPART];
    __shared__ bool s_last;
    double part[NPART];
#pragma unroll
    for (int q = 0; q < NPART; q++) part[q] = 0.0;

    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const double fnh = a.scal[SC_FNH];
    const bool apply_vom = a.scal[SC_APPLY] != 0.0;
    const double vomx = a.scal[SC_VOM], vomy = a.scal[SC_VOM + 1], vomz = a.scal[SC_VOM + 2];
    bool nh_fail = false, rebuild = false, bad = false;
    if (m < a.nmol) {
        const int s = a.mol_off[m], e = a.mol_off[m + 1];
        double cx = 0, cy = 0, cz = 0, px = 0, py = 0, pz = 0, M = 0;
        for (int k = s; k < e; k++) {
            const int at = a.mol_atoms[k];
            double4 vm = a.vtm4[at];   // w: mass
            double4 v = a.vel4[at];    // w: 1/mass
            if (apply_vom) {
                vm.x -= vomx; vm.y -= vomy; vm.z -= vomz;
                v.x -= vomx; v.y -= vomy; v.z -= vomz;
            }
            const double mass = vm.w, mr = v.w;
            const double3 f = fetch_force(a.frc, a.n, at);
            double vpx, vpy, vpz;
            if (a.thermostat == SMD_THERMO_NOSE_HOOVER) {
                double velcheck = 1.0;
                int cnt = 0;
                while (velcheck > 1e-10 && cnt < 11) {
                    vpx = vm.x + a.dt * (mr * f.x - fnh * v.x);
                    vpy = vm.y + a.dt * (mr * f.y - fnh * v.y);
                    vpz = vm.z + a.dt * (mr * f.z - fnh * v.z);
                    const double nx = (vpx + vm.x) * 0.5, ny = (vpy + vm.y) * 0.5,
                                 nz = (vpz + vm.z) * 0.5;
                    const double ddx = nx - v.x, ddy = ny - v.y, ddz = nz - v.z;
                    velcheck = sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
                    v.x = nx; v.y = ny; v.z = nz;
                    cnt++;
                }
                if (cnt == 10) nh_fail = true;  // the reference's (odd) failure test
            } else {
                vpx = vm.x + a.dt * mr * f.x;
                vpy = vm.y + a.dt * mr * f.y;
                vpz = vm.z + a.dt * mr * f.z;
            }
            const double drx = a.dt * vpx, dry = a.dt * vpy, drz = a.dt * vpz;
            double4 p = a.pos4[at];
            p.x += drx; p.y += dry; p.z += drz;
            double4 d = a.disp4[at];
            d.x += drx; d.y += dry; d.z += drz;
            if (d.x * d.x + d.y * d.y + d.z * d.z > a.drmax) rebuild = true;
            v.x = (vpx + vm.x) * 0.5; v.y = (vpy + vm.y) * 0.5; v.z = (vpz + vm.z) * 0.5;
            vm.x = vpx; vm.y = vpy; vm.z = vpz;
            a.vel4[at] = v;
            a.vtm4[at] = vm;
            a.disp4[at] = d;
            a.pos4[at] = p;
            if (!isfinite(p.x + p.y + p.z)) bad = true;
            // momenta, centre of mass, kinetic energy (LFIntegrator.cpp:668-676)
            const double mx = v.x * mass, my = v.y * mass, mz = v.z * mass;
            px += mx; py += my; pz += mz;
            cx += mass * p.x; cy += mass * p.y; cz += mass * p.z;
            M += mass;
            part[0] += (v.x * v.x + v.y * v.y + v.z * v.z) * mass;
            part[2] += mx * mx / mass; part[3] += mx * my / mass; part[4] += mx * mz / mass;
            part[5] += my * my / mass; part[6] += my * mz / mass; part[7] += mz * mz / mass;
            part[23] += vm.x * mass; part[24] += vm.y * mass; part[25] += vm.z * mass;
        }
        cx /= M; cy /= M; cz /= M;
        part[1] += (px * px + py * py + pz * pz) / M;
        part[8] += px * px / M; part[9] += px * py / M; part[10] += px * pz / M;
        part[11] += py * py / M; part[12] += py * pz / M; part[13] += pz * pz / M;
        // molecular virial correction sum_j f_j (r_j - R)  (Integrator.cpp:216-234)
        for (int k = s; k < e; k++) {
            const int at = a.mol_atoms[k];
            const double3 f = fetch_force(a.frc, a.n, at);
            const double4 p = a.pos4[at];
            const double rx = p.x - cx, ry = p.y - cy, rz = p.z - cz;
            part[14] += f.x * rx; part[15] += f.y * rx; part[16] += f.z * rx;
            part[17] += f.x * ry; part[18] += f.y * ry; part[19] += f.z * ry;
            part[20] += f.x * rz; part[21] += f.y * rz; part[22] += f.z * rz;
        }
        // wrap the molecule's centre of mass into the box
        const double wx = pbc1(cx, a.box.L[0], a.box.half[0]) - cx;
        const double wy = pbc1(cy, a.box.L[1], a.box.half[1]) - cy;
        const double wz = pbc1(cz, a.box.L[2], a.box.half[2]) - cz;
        if (wx != 0.0 || wy != 0.0 || wz != 0.0) {
            for (int k = s; k < e; k++) {
                const int at = a.mol_atoms[k];
                double4 p = a.pos4[at];
                p.x += wx; p.y += wy; p.z += wz;
                a.pos4[at] = p;
            }
        }
    }
    if (__any_sync(0xffffffffu, rebuild) && (threadIdx.x & 31) == 0) atomicOr(&a.flags[0], 1);
    if (nh_fail) atomicOr(a.status, ST_NH_ITER);
    if (bad) atomicOr(a.status, ST_NAN);

    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NPART; q++) {
        double v = warp_sum(part[q]);
        if (lane == 0) s_part[w][q] = v;
    }
    __syncthreads();
    if (threadIdx.x < NPART) {
        double v = 0;
        for (int q = 0; q < INT_BLOCK / 32; q++) v += s_part[q][threadIdx.x];
        a.partials[(size_t)blockIdx.x * NPART + threadIdx.x] = v;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int t = atomicAdd(a.ticket, 1u);
        s_last = (t == (unsigned)a.nblocks - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();

    // ---- last block: totals in fixed order -----------------------------
    __shared__ double tot[NPART];
    if (threadIdx.x < NPART) {
        double v = 0;
        for (int b = 0; b < a.nblocks; b++) v += ((volatile double *)a.partials)[(size_t)b * NPART + threadIdx.x];
        tot[threadIdx.x] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        smd_observables &o = *a.obs;
        const double keA = tot[0], keM = tot[1];
        // Nose-Hoover zeta update (LFIntegrator.cpp:688-722)
        if (a.thermostat == SMD_THERMO_NOSE_HOOVER) {
            const double ndf = a.atom_thermo ? a.atom_ndf : a.mol_ndf;
            const double qq = ndf * KB * a.temperature * a.tau * a.tau;
            const double invqq = 1.0 / qq;
            const double ke = a.atom_thermo ? keA : keM;
            const double fnhmi = a.scal[SC_FNHMI];
            const double fnhpl = fnhmi + a.dt * invqq * (ke - ndf * KB * a.temperature);
            a.scal[SC_FNH] = 0.5 * (fnhpl + fnhmi);
            a.scal[SC_FNHMI] = fnhpl;
        } else {
            a.scal[SC_FNH] = 0.0;
        }
        o.zeta = a.scal[SC_FNH];
        o.ke_atom = 0.5 * keA;
        o.ke_mol = 0.5 * keM;
        o.t_atom = keA / (a.atom_ndf * KB);
        o.t_mol = keM / (a.mol_ndf * KB);
        // energies
        volatile long long *acc = a.acc;
        o.energy[SMD_E_VDW] = (double)acc[ACC_E_VDW] * ACC_INV + a.e_lrc;
        o.energy[SMD_E_REAL] = (double)acc[ACC_E_REAL] * ACC_INV;
        o.energy[SMD_E_LONG] = (double)acc[ACC_E_LONG] * ACC_INV;
        o.energy[SMD_E_CORRECT] = a.e_self;
        o.energy[SMD_E_MOLCORRECT] = (double)acc[ACC_E_INTRA] * ACC_INV;
        o.energy[SMD_E_SURF] = (double)acc[ACC_E_SURF] * ACC_INV;
        double ep = 0;
        for (int q = 0; q < 6; q++) ep += o.energy[q];
        o.e_potential = ep;
        // virial and pressure tensors (Integrator::computePressure)
        const int sym[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
        for (int q = 0; q < 9; q++) {
            double vir = ((double)acc[ACC_VIR + q] + (double)acc[ACC_LVIR + q]) * ACC_INV;
            if (q == 0 || q == 4 || q == 8) vir -= a.v_lrc;
            o.virial[q] = vir;
            o.atom_pressure[q] = (tot[2 + sym[q]] + vir) / a.volume;
            o.mol_pressure[q] = (tot[8 + sym[q]] + vir - tot[14 + q]) / a.volume;
        }
        o.volume = a.volume;
        // centre-of-mass drift of v- for the next step (LFIntegrator.cpp:359-379)
        const double vx = tot[23] / a.total_mass, vy = tot[24] / a.total_mass,
                     vz = tot[25] / a.total_mass;
        a.scal[SC_VOM] = vx; a.scal[SC_VOM + 1] = vy; a.scal[SC_VOM + 2] = vz;
        a.scal[SC_APPLY] = (fabs(vx) > 1e-11 || fabs(vy) > 1e-11 || fabs(vz) > 1e-11) ? 1.0 : 0.0;
        o.step += 1;
        o.list_updates = a.flags[1];
        o.pairs_in_cutoff = acc[ACC_NPAIR] / 2;
        o.status = *a.status;
        if (a.series_cap > 0) {
            long long slot = (o.step - 1) % a.series_cap;
            double *r = a.series + slot * 5;
            r[0] = o.e_potential; r[1] = o.ke_atom; r[2] = o.t_atom; r[3] = o.zeta;
            r[4] = (o.atom_pressure[0] + o.atom_pressure[4] + o.atom_pressure[8]) / 3.0;
        }
        *a.ticket = 0;
    }
    __syncthreads();
    // clear the force-side accumulators for the next step
    if (threadIdx.x < ACC_COUNT) a.acc[threadIdx.x] = 0;
}

void launch_integrate(Ctx &c) {
    IntArgs a;
    a.n = c.n; a.nmol = c.nmol;
    a.nblocks = (c.nmol + INT_BLOCK - 1) / INT_BLOCK;
    a.mol_off = c.mol_off; a.mol_atoms = c.mol_atoms;
    a.pos4 = c.pos4; a.vel4 = c.vel4; a.vtm4 = c.vtm4; a.disp4 = c.disp4;
    a.frc = c.frc; a.acc = c.acc; a.scal = c.scal; a.partials = c.partials;
    a.ticket = c.ticket; a.status = c.status; a.flags = c.flags; a.obs = c.obs;
    a.series = c.series; a.series_cap = c.series_cap;
    a.box = c.box;
    a.dt = c.ip.timestep; a.temperature = c.ip.temperature; a.tau = c.ip.coupl_const;
    a.drmax = c.pl.drmax; a.total_mass = c.total_mass;
    a.volume = c.box.L[0] * c.box.L[1] * c.box.L[2];
    a.thermostat = c.ip.thermostat; a.atom_thermo = c.ip.atom_thermo;
    a.atom_ndf = c.ip.atom_ndf; a.mol_ndf = c.ip.mol_ndf;
    a.e_lrc = c.e_lrc; a.v_lrc = c.v_lrc; a.e_self = c.e_self;
    k_integrate<<<a.nblocks, INT_BLOCK, 0, c.stream>>>(a);
}

// LFIntegrator::start (LFIntegrator.cpp:1172-1173): vtMinus = v - dt/2 F/m.
__global__ void k_start(int n, double dt, const long long *frc, const double4 *vel4,
                        double4 *vtm4) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 v = vel4[i];
    double4 vm = vtm4[i];
    const double3 f = fetch_force(frc, n, i);
    vm.x = v.x - 0.5 * dt * v.w * f.x;
    vm.y = v.y - 0.5 * dt * v.w * f.y;
    vm.z = v.z - 0.5 * dt * v.w * f.z;
    vtm4[i] = vm;
}

// Centre-of-mass velocity of v- for the first step, one block, fixed order.
__global__ void k_vom(int n, const double4 *vtm4, double total_mass, double *scal,
                      long long *acc) {
    __shared__ double s[3][256];
    double x = 0, y = 0, z = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double4 v = vtm4[i];
        x += v.x * v.w; y += v.y * v.w; z += v.z * v.w;
    }
    s[0][threadIdx.x] = x; s[1][threadIdx.x] = y; s[2][threadIdx.x] = z;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int q = 0; q < 3; q++) s[q][threadIdx.x] += s[q][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double vx = s[0][0] / total_mass, vy = s[1][0] / total_mass, vz = s[2][0] / total_mass;
        scal[SC_VOM] = vx; scal[SC_VOM + 1] = vy; scal[SC_VOM + 2] = vz;
        scal[SC_APPLY] = (fabs(vx) > 1e-11 || fabs(vy) > 1e-11 || fabs(vz) > 1e-11) ? 1.0 : 0.0;
        scal[SC_FNH] = 0.0;
        scal[SC_FNHMI] = 0.0;
    }
    __syncthreads();
    if (threadIdx.x < ACC_COUNT) acc[threadIdx.x] = 0;
}

void launch_start_velocities(Ctx &c) {
    k_start<<<(c.n + 255) / 256, 256, 0, c.stream>>>(c.n, c.ip.timestep, c.frc, c.vel4, c.vtm4);
    k_vom<<<1, 256, 0, c.stream>>>(c.n, c.vtm4, c.total_mass, c.scal, c.acc);
}

// Fixed-point forces to the reference's per-atom FP64 Vector3 layout.
__global__ void k_forces_out(int n, const long long *frc, double *out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[3 * i] = (double)frc[i] * FRC_INV;
    out[3 * i + 1] = (double)frc[n + i] * FRC_INV;
    out[3 * i + 2] = (double)frc[2 * n + i] * FRC_INV;
}

void launch_finalize_forces(Ctx &c, double *f_out_dev) {
    k_forces_out<<<(c.n + 255) / 256, 256, 0, c.stream>>>(c.n, c.frc, f_out_dev);
}

}  // namespace smd
