// Leap-frog Nose-Hoover integrator step (optionally with SHAKE), observables
// and thermostat update.
//
// One thread per molecule carries out, for the molecule's sites:
//  - unconstrained (LFIntegrator::run, src/integrators/LFIntegrator.cpp:
//    588-642): the implicit Nose-Hoover velocity iteration
//        v+ = v- + dt (F/m - zeta v),  v = (v+ + v-)/2   (to 1e-10, <= 10 passes)
//    then r += dt v+;
//  - SHAKE (LFIntegrator::shake, :1678-1827, NVT branch): v+ = v- + dt/m
//    (F - zeta P_mol/ns), unconstrained r' = r + dt v+, then the cyclic
//    3-distance SHAKE iteration in FP64 until every squared distance is
//    within 2 tol of its target (<= maxCount passes), v+ = (r' - r)/dt and
//    the SHAKE virial sum factor r'_ij (x) r_ij / dt^2;
// followed by the molecular centre of mass and momenta (:646-686), the
// pair-list displacement test (:307-315) and the molecule wrap into the box
// (:897-912).  The centre-of-mass drift removal the reference applies to v-
// at the start of the next step (:359-379) is applied here at the start of
// that step's update; forces do not depend on velocities, so the order is
// equivalent.  In the FP32 path the same thread also writes the sites' new
// 32-bit box fractions for the next step's pair kernel.
//
// Per-block partial sums (kinetic energies, kinetic pressure tensors, the
// molecular virial correction, sum m v-, the SHAKE virial) are combined by
// the last block to finish in a fixed order (deterministic); it then updates
// zeta (:688-722), temperatures, energies, the pressure tensors of
// Integrator::computePressure (src/Integrator.cpp:205-270, SHAKE virial added
// to the atomic tensor as at LFIntegrator.cpp:805-814) and clears the force
// accumulators for the next step.
#include <type_traits>
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

// partial sums per block
enum {
    P_KEA = 0, P_KEM = 1, P_AP = 2 /*6*/, P_MP = 8 /*6*/, P_MC = 14 /*9*/, P_VM = 23 /*3*/,
    P_SV = 26 /*9*/, NPART = 35
};
constexpr int INT_BLOCK = 128;
constexpr double KB = 0.0083145112;  // BOLTZMAN, src/NEMD_defs.h:108

struct IntArgs {
    int n, nmol, nblocks;
    const int *mol_off, *mol_atoms;
    double4 *pos4, *vel4, *vtm4, *disp4;
    int4 *fixq;
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
    double dt, temperature, tau, drmax, total_mass, volume;
    int thermostat, atom_thermo, atom_ndf, mol_ndf, write_fixq;
    double e_lrc, v_lrc, e_self;
    const double *clen2;   // [nmol][3] squared constraint lengths
    double shake_tol;
    int shake_max;
};

__device__ __forceinline__ double3 fetch_force(const long long *frc, int n, int a) {
    return make_double3((double)frc[a] * FRC_INV, (double)frc[n + a] * FRC_INV,
                        (double)frc[2 * n + a] * FRC_INV);
}

__device__ __forceinline__ void pbc3(double &x, double &y, double &z, const Box &b) {
    x = pbc1(x, b.L[0], b.half[0]);
    y = pbc1(y, b.L[1], b.half[1]);
    z = pbc1(z, b.L[2], b.half[2]);
}

constexpr int MAX_MOL_SITES = 8;

// SHAKE step of one molecule (LFIntegrator::shake, NVT branch) and its
// contributions to the observables.  NS > 0 fixes the number of sites at
// compile time, so that every loop over sites and bonds unrolls and the
// per-site arrays stay in registers (three-site water); NS = 0 takes the
// count at run time (up to MAX_MOL_SITES sites, arrays in local memory).
template <int NS>
__device__ __forceinline__ void shake_mol(const IntArgs &a, int m, int s, int e, int ns_rt, double fnh,
                                          bool apply_vom, double vomx, double vomy, double vomz,
                                          double (&part)[NPART], bool &rebuild, bool &bad, bool &shake_fail,
                                          bool &shake_geom, double &cx, double &cy, double &cz, double &px,
                                          double &py, double &pz, double &M) {
    constexpr int CAP = NS ? NS : MAX_MOL_SITES;
    const int ns = NS ? NS : ns_rt;
    // molecular momentum of the previous step (Molecule::momenta)
    double Px = 0, Py = 0, Pz = 0;
    for (int k = s; k < e; k++) {
        const double4 v = a.vel4[a.mol_atoms[k]];
        const double mass = 1.0 / v.w;
        Px += v.x * mass; Py += v.y * mass; Pz += v.z * mass;
    }
    double ro[CAP][3], rn[CAP][3], mr[CAP];
    double4 vmv[CAP];
    for (int q = 0; q < ns; q++) {
        const int at = a.mol_atoms[s + q];
        double4 vm = a.vtm4[at];
        if (apply_vom) { vm.x -= vomx; vm.y -= vomy; vm.z -= vomz; }
        vmv[q] = vm;
        mr[q] = 1.0 / vm.w;
        const double3 f = fetch_force(a.frc, a.n, at);
        const double4 p = a.pos4[at];
        double vpx, vpy, vpz;
        if (a.thermostat == SMD_THERMO_NOSE_HOOVER) {
            vpx = vm.x + a.dt * mr[q] * (f.x - fnh * Px / ns);
            vpy = vm.y + a.dt * mr[q] * (f.y - fnh * Py / ns);
            vpz = vm.z + a.dt * mr[q] * (f.z - fnh * Pz / ns);
        } else {
            vpx = vm.x + a.dt * mr[q] * f.x;
            vpy = vm.y + a.dt * mr[q] * f.y;
            vpz = vm.z + a.dt * mr[q] * f.z;
        }
        ro[q][0] = p.x; ro[q][1] = p.y; ro[q][2] = p.z;
        rn[q][0] = p.x + a.dt * vpx; rn[q][1] = p.y + a.dt * vpy; rn[q][2] = p.z + a.dt * vpz;
    }
    const int nb = (ns == 3) ? 3 : ns - 1;
    const double tol2 = 2 * a.shake_tol;
    const double *bl = a.clen2 + (size_t)m * 3;
    // the old bond vectors stay fixed during the iteration: their
    // minimum images once, and the SHAKE virial sum_k f_k n_k (x) o
    // as (sum_k f_k n_k) (x) o per bond at the end
    double ob[CAP][3], sfn[CAP][3];
    for (int i = 0; i < nb; i++) {
        const int nx = i + 1 == ns ? 0 : i + 1;
        double ox = ro[i][0] - ro[nx][0], oy = ro[i][1] - ro[nx][1], oz = ro[i][2] - ro[nx][2];
        pbc3(ox, oy, oz, a.box);
        ob[i][0] = ox; ob[i][1] = oy; ob[i][2] = oz;
        sfn[i][0] = 0; sfn[i][1] = 0; sfn[i][2] = 0;
    }
    int count = 0;
    bool done = false;
    // the cyclic sweeps; PBC selects the minimum image of the new bond vectors
    auto sweeps = [&](auto pbc) {
        while (!done && count < a.shake_max) {
            done = true;
            for (int i = 0; i < nb; i++) {
                int nx = i + 1;
                if (nx == ns) nx = 0;
                double nx_ = rn[i][0] - rn[nx][0], ny_ = rn[i][1] - rn[nx][1], nz_ = rn[i][2] - rn[nx][2];
                if (decltype(pbc)::value) pbc3(nx_, ny_, nz_, a.box);
                const double r2 = nx_ * nx_ + ny_ * ny_ + nz_ * nz_;
                const double blen = bl[i < 3 ? i : 2];
                const double diff = blen - r2;
                if (fabs(diff) > blen * tol2) {
                    const double ox = ob[i][0], oy = ob[i][1], oz = ob[i][2];
                    const double rr = ox * nx_ + oy * ny_ + oz * nz_;
                    if (rr < blen * a.shake_tol) { shake_geom = true; done = true; count = a.shake_max; break; }
                    const double factor = diff / (2 * rr * (mr[i] + mr[nx]));
                    sfn[i][0] += factor * nx_; sfn[i][1] += factor * ny_; sfn[i][2] += factor * nz_;
                    rn[i][0] += factor * ox * mr[i]; rn[i][1] += factor * oy * mr[i]; rn[i][2] += factor * oz * mr[i];
                    rn[nx][0] -= factor * ox * mr[nx]; rn[nx][1] -= factor * oy * mr[nx];
                    rn[nx][2] -= factor * oz * mr[nx];
                    done = false;
                }
            }
            count++;
        }
    };
    // The minimum image leaves a bond vector unchanged while each component is
    // below half the box.  When every bond starts below a quarter of the box
    // the corrections (a small fraction of a bond length) cannot carry one
    // across half the box, so the sweeps skip the image test and give the
    // same numbers; a molecule split across the boundary takes the test.
    bool whole = true;
    for (int i = 0; i < nb; i++) {
        const int nx = i + 1 == ns ? 0 : i + 1;
        for (int d = 0; d < 3; d++) whole = whole && fabs(rn[i][d] - rn[nx][d]) < 0.5 * a.box.half[d];
    }
    if (whole)
        sweeps(std::integral_constant<bool, false>());
    else
        sweeps(std::integral_constant<bool, true>());
    if (!done) shake_fail = true;
    for (int i = 0; i < nb; i++)
        for (int p = 0; p < 3; p++)
            for (int q = 0; q < 3; q++) part[P_SV + 3 * p + q] += sfn[i][p] * ob[i][q];
    for (int q = 0; q < ns; q++) {
        const int at = a.mol_atoms[s + q];
        double4 p = a.pos4[at];
        const double drx = rn[q][0] - p.x, dry = rn[q][1] - p.y, drz = rn[q][2] - p.z;
        p.x += drx; p.y += dry; p.z += drz;
        double4 d = a.disp4[at];
        d.x += drx; d.y += dry; d.z += drz;
        if (d.x * d.x + d.y * d.y + d.z * d.z > a.drmax) rebuild = true;
        double4 vm = vmv[q];
        const double vpx = drx / a.dt, vpy = dry / a.dt, vpz = drz / a.dt;
        double4 v = a.vel4[at];
        v.x = (vpx + vm.x) * 0.5; v.y = (vpy + vm.y) * 0.5; v.z = (vpz + vm.z) * 0.5;
        vm.x = vpx; vm.y = vpy; vm.z = vpz;
        a.vel4[at] = v;
        a.vtm4[at] = vm;
        a.disp4[at] = d;
        a.pos4[at] = p;
        if (!isfinite(p.x + p.y + p.z)) bad = true;
        const double mass = vm.w;
        const double mx = v.x * mass, my = v.y * mass, mz = v.z * mass;
        px += mx; py += my; pz += mz;
        cx += mass * p.x; cy += mass * p.y; cz += mass * p.z;
        M += mass;
        part[P_KEA] += (v.x * v.x + v.y * v.y + v.z * v.z) * mass;
        part[P_AP + 0] += mx * mx / mass; part[P_AP + 1] += mx * my / mass; part[P_AP + 2] += mx * mz / mass;
        part[P_AP + 3] += my * my / mass; part[P_AP + 4] += my * mz / mass; part[P_AP + 5] += mz * mz / mass;
        part[P_VM + 0] += vm.x * mass; part[P_VM + 1] += vm.y * mass; part[P_VM + 2] += vm.z * mass;
    }
}

template <bool SHAKE>
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
    bool nh_fail = false, rebuild = false, bad = false, shake_fail = false, shake_geom = false;
    if (m < a.nmol) {
        const int s = a.mol_off[m], e = a.mol_off[m + 1];
        const int ns = e - s;
        double cx = 0, cy = 0, cz = 0, px = 0, py = 0, pz = 0, M = 0;
        if (SHAKE && ns == 3) {
            shake_mol<3>(a, m, s, e, ns, fnh, apply_vom, vomx, vomy, vomz, part, rebuild, bad, shake_fail,
                         shake_geom, cx, cy, cz, px, py, pz, M);
        } else if (SHAKE && ns > 1 && ns <= MAX_MOL_SITES) {
            shake_mol<0>(a, m, s, e, ns, fnh, apply_vom, vomx, vomy, vomz, part, rebuild, bad, shake_fail,
                         shake_geom, cx, cy, cz, px, py, pz, M);
        } else {
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
                    if (cnt == 10) nh_fail = true;  // the reference's failure test
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
                const double mx = v.x * mass, my = v.y * mass, mz = v.z * mass;
                px += mx; py += my; pz += mz;
                cx += mass * p.x; cy += mass * p.y; cz += mass * p.z;
                M += mass;
                part[P_KEA] += (v.x * v.x + v.y * v.y + v.z * v.z) * mass;
                part[P_AP + 0] += mx * mx / mass; part[P_AP + 1] += mx * my / mass; part[P_AP + 2] += mx * mz / mass;
                part[P_AP + 3] += my * my / mass; part[P_AP + 4] += my * mz / mass; part[P_AP + 5] += mz * mz / mass;
                part[P_VM + 0] += vm.x * mass; part[P_VM + 1] += vm.y * mass; part[P_VM + 2] += vm.z * mass;
            }
        }
        cx /= M; cy /= M; cz /= M;
        part[P_KEM] += (px * px + py * py + pz * pz) / M;
        part[P_MP + 0] += px * px / M; part[P_MP + 1] += px * py / M; part[P_MP + 2] += px * pz / M;
        part[P_MP + 3] += py * py / M; part[P_MP + 4] += py * pz / M; part[P_MP + 5] += pz * pz / M;
        // molecular virial correction sum_j f_j (r_j - R)  (Integrator.cpp:216-234)
        for (int k = s; k < e; k++) {
            const int at = a.mol_atoms[k];
            const double3 f = fetch_force(a.frc, a.n, at);
            const double4 p = a.pos4[at];
            const double rx = p.x - cx, ry = p.y - cy, rz = p.z - cz;
            part[P_MC + 0] += f.x * rx; part[P_MC + 1] += f.y * rx; part[P_MC + 2] += f.z * rx;
            part[P_MC + 3] += f.x * ry; part[P_MC + 4] += f.y * ry; part[P_MC + 5] += f.z * ry;
            part[P_MC + 6] += f.x * rz; part[P_MC + 7] += f.y * rz; part[P_MC + 8] += f.z * rz;
        }
        // wrap the molecule's centre of mass into the box
        const double wx = pbc1(cx, a.box.L[0], a.box.half[0]) - cx;
        const double wy = pbc1(cy, a.box.L[1], a.box.half[1]) - cy;
        const double wz = pbc1(cz, a.box.L[2], a.box.half[2]) - cz;
        // the shifts so far, per molecule: Atom::realPos = position - shift
        if (a.wrap && (wx != 0.0 || wy != 0.0 || wz != 0.0)) {
            a.wrap[m] += wx;
            a.wrap[a.nmol + m] += wy;
            a.wrap[2 * a.nmol + m] += wz;
        }
        for (int k = s; k < e; k++) {
            const int at = a.mol_atoms[k];
            double4 p = a.pos4[at];
            if (wx != 0.0 || wy != 0.0 || wz != 0.0) {
                p.x += wx; p.y += wy; p.z += wz;
                a.pos4[at] = p;
            }
            if (a.write_fixq)
                a.fixq[at] = make_int4(frac32(p.x, a.box.inv[0]), frac32(p.y, a.box.inv[1]),
                                       frac32(p.z, a.box.inv[2]), (int)p.w);
        }
    }
    if (__any_sync(0xffffffffu, rebuild) && (threadIdx.x & 31) == 0) atomicOr(&a.flags[0], 1);
    if (nh_fail) atomicOr(a.status, ST_NH_ITER);
    if (bad) atomicOr(a.status, ST_NAN);
    if (shake_fail) atomicOr(a.status, ST_SHAKE_ITER);
    if (shake_geom) atomicOr(a.status, ST_SHAKE_GEOM);

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

    // ---- last block: totals in a fixed order ---------------------------
    // warp w sums slots w, w + 4, ...: each lane a fixed strided subset of
    // the blocks, then the warp's butterfly (same order on every run)
    __shared__ double tot[NPART];
    for (int q = w; q < NPART; q += INT_BLOCK / 32) {
        double v = 0;
        for (int b = lane; b < a.nblocks; b += 32) v += __ldcg(&a.partials[(size_t)b * NPART + q]);
        v = warp_sum(v);
        if (lane == 0) tot[q] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // every accumulator into registers before the first store through o
        long long acc[ACC_COUNT];
#pragma unroll
        for (int q = 0; q < ACC_COUNT; q++) acc[q] = __ldcg(&a.acc[q]);
        const double fnhmi = a.scal[SC_FNHMI];
        const int list_updates = a.flags[1];
        const unsigned int status = *a.status;
        smd_observables &o = *a.obs;
        const double keA = tot[P_KEA], keM = tot[P_KEM];
        // Nose-Hoover zeta update (LFIntegrator.cpp:688-722)
        if (a.thermostat == SMD_THERMO_NOSE_HOOVER) {
            const double ndf = a.atom_thermo ? a.atom_ndf : a.mol_ndf;
            const double qq = ndf * KB * a.temperature * a.tau * a.tau;
            const double invqq = 1.0 / qq;
            const double ke = a.atom_thermo ? keA : keM;
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
        double en[SMD_E_COUNT];
        acc_energies(acc, a.e_lrc, a.e_self, en);
        double ep = 0;
        for (int q = 0; q < SMD_E_COUNT; q++) {
            o.energy[q] = en[q];
            ep += en[q];
        }
        o.e_potential = ep;
        // virial and pressure tensors (Integrator::computePressure; SHAKE
        // virial added afterwards to the atomic tensor, LFIntegrator.cpp:805-814)
        const int sym[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
        const double idt2 = 1.0 / (a.dt * a.dt);
        for (int q = 0; q < 9; q++) {
            double vir = ((double)acc[ACC_VIR + q] + (double)acc[ACC_LVIR + q]) * ACC_INV;
            if (q == 0 || q == 4 || q == 8) vir -= a.v_lrc;
            o.mol_pressure[q] = (tot[P_MP + sym[q]] + vir - tot[P_MC + q]) / a.volume;
            o.atom_pressure[q] = (tot[P_AP + sym[q]] + vir) / a.volume;
            if (SHAKE) {
                const double sv = tot[P_SV + q] * idt2;
                vir += sv;
                o.atom_pressure[q] += sv / a.volume;
            }
            o.virial[q] = vir;
        }
        o.volume = a.volume;
        // centre-of-mass drift of v- for the next step (LFIntegrator.cpp:359-379)
        const double vx = tot[P_VM] / a.total_mass, vy = tot[P_VM + 1] / a.total_mass,
                     vz = tot[P_VM + 2] / a.total_mass;
        a.scal[SC_VOM] = vx; a.scal[SC_VOM + 1] = vy; a.scal[SC_VOM + 2] = vz;
        a.scal[SC_APPLY] = (fabs(vx) > 1e-11 || fabs(vy) > 1e-11 || fabs(vz) > 1e-11) ? 1.0 : 0.0;
        o.step += 1;
        o.list_updates = list_updates;
        o.pairs_in_cutoff = acc[ACC_NPAIR] / 2;
        o.status = status;
        if (a.series_cap > 0) {
            long long slot = (o.step - 1) % a.series_cap;
            double *r = a.series + slot * 5;
            r[0] = o.e_potential; r[1] = o.ke_atom; r[2] = o.t_atom; r[3] = o.zeta;
            r[4] = (o.atom_pressure[0] + o.atom_pressure[4] + o.atom_pressure[8]) / 3.0;
        }
        accumulate_averages(a.avg, o);
        *a.ticket = 0;
    }
    __syncthreads();
    // clear the force-side accumulators for the next step
    if (threadIdx.x < ACC_COUNT) a.acc[threadIdx.x] = 0;
}

// Uploaded positions (staged in upload4, type in w) replace pos4; each
// site's minimum-image displacement adds to its displacement since the last
// list rebuild, and the rebuild flag is raised past half the skin.
__global__ void k_upload_positions(int n, const double4 *np, double4 *pos4, double4 *disp4, Box b, double drmax,
                                   int *flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 o = pos4[i], p = np[i];
    double4 d = disp4[i];
    d.x += pbc1(p.x - o.x, b.L[0], b.half[0]);
    d.y += pbc1(p.y - o.y, b.L[1], b.half[1]);
    d.z += pbc1(p.z - o.z, b.L[2], b.half[2]);
    disp4[i] = d;
    pos4[i] = p;
    if (d.x * d.x + d.y * d.y + d.z * d.z > drmax) atomicOr(&flags[0], 1);
}

void launch_upload_positions(Ctx &c) {
    k_upload_positions<<<(c.n + 255) / 256, 256, 0, c.stream>>>(c.n, c.upload4, c.pos4, c.disp4, c.box,
                                                               c.pl.drmax, c.flags);
}

void launch_integrate(Ctx &c) {
    IntArgs a;
    a.n = c.n; a.nmol = c.nmol;
    a.nblocks = (c.nmol + INT_BLOCK - 1) / INT_BLOCK;
    a.mol_off = c.mol_off; a.mol_atoms = c.mol_atoms;
    a.pos4 = c.pos4; a.vel4 = c.vel4; a.vtm4 = c.vtm4; a.disp4 = c.disp4;
    a.fixq = c.fixq; a.write_fixq = c.precision == SMD_PREC_MIXED;
    a.frc = c.frc; a.acc = c.acc; a.scal = c.scal; a.partials = c.partials;
    a.ticket = c.ticket; a.status = c.status; a.flags = c.flags; a.obs = c.obs;
    a.series = c.series; a.series_cap = c.series_cap;
    a.avg = c.avg;
    a.wrap = c.wrap;
    a.box = c.box;
    a.dt = c.ip.timestep; a.temperature = c.ip.temperature; a.tau = c.ip.coupl_const;
    a.drmax = c.pl.drmax; a.total_mass = c.total_mass;
    a.volume = c.box.L[0] * c.box.L[1] * c.box.L[2];
    a.thermostat = c.ip.thermostat; a.atom_thermo = c.ip.atom_thermo;
    a.atom_ndf = c.ip.atom_ndf; a.mol_ndf = c.ip.mol_ndf;
    a.e_lrc = c.e_lrc; a.v_lrc = c.v_lrc; a.e_self = c.e_self;
    a.clen2 = c.clen2; a.shake_tol = c.ip.shake_tol; a.shake_max = c.ip.shake_max_iter;
    if (c.ip.constraint == 2)
        k_integrate<true><<<a.nblocks, INT_BLOCK, 0, c.stream>>>(a);
    else
        k_integrate<false><<<a.nblocks, INT_BLOCK, 0, c.stream>>>(a);
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

// EwaldForce::intraMolCorrect (src/forces/EwaldForce.cpp:709-813): for
// every excluded site pair inside a molecule, -q_i q_j erf(a r)/r into the
// energy; with no constraints also the force q_i q_j (erf(a r)/r -
// 2a/sqrt(pi) exp(-a^2 r^2))/r^2 r_ij on i (and its negative on j), which
// the reference leaves out of the virial.  One thread per molecule owns its
// sites' forces.
__global__ void k_intra_ewald(int nmol, int n, const int *mol_off, const int *mol_atoms,
                              const int *excl_off, const int *excl, const double4 *pos4,
                              const double *tq, Box box, double alpha, int apply_force,
                              long long *frc, long long *acc) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    double en = 0;
    if (m < nmol) {
        const int s = mol_off[m], e = mol_off[m + 1];
        const double a2 = alpha * alpha, a2pi = 2.0 * alpha / 1.7724538509055160273;
        for (int p = s; p < e; p++) {
            const int i = mol_atoms[p];
            const double4 pi = pos4[i];
            const double qi = tq[(int)pi.w];
            for (int q = p + 1; q < e; q++) {
                const int j = mol_atoms[q];
                bool ex = false;
                for (int k = excl_off[i]; k < excl_off[i + 1]; k++)
                    if (excl[k] == j) { ex = true; break; }
                if (!ex) continue;
                const double4 pj = pos4[j];
                double dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
                pbc3(dx, dy, dz, box);
                const double r2 = dx * dx + dy * dy + dz * dz, r = sqrt(r2);
                const double qij = qi * tq[(int)pj.w];
                const double ee = erf(alpha * r) / r;
                en += qij * ee;
                if (apply_force) {
                    const double dudr = ee - a2pi * exp(-a2 * r2);
                    const double fs = qij * dudr / r2;
                    frc[i] += to_fix(fs * dx, FRC_SCALE);
                    frc[n + i] += to_fix(fs * dy, FRC_SCALE);
                    frc[2 * n + i] += to_fix(fs * dz, FRC_SCALE);
                    frc[j] -= to_fix(fs * dx, FRC_SCALE);
                    frc[n + j] -= to_fix(fs * dy, FRC_SCALE);
                    frc[2 * n + j] -= to_fix(fs * dz, FRC_SCALE);
                }
            }
        }
    }
    __shared__ double s_r[8];
    double t = warp_sum(en);
    if ((threadIdx.x & 31) == 0) s_r[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) v += s_r[q];
        if (v != 0.0) atomicAdd((unsigned long long *)&acc[ACC_E_INTRA], (unsigned long long)to_fix(-v, ACC_SCALE));
    }
}

void launch_intra(Ctx &c) {
    if (!c.ewald_on || !c.has_multisite) return;
    k_intra_ewald<<<(c.nmol + 127) / 128, 128, 0, c.stream>>>(
        c.nmol, c.n, c.mol_off, c.mol_atoms, c.excl_off, c.excl, c.pos4, c.type_q, c.box, c.ew_alpha,
        c.clen2 ? 0 : 1, c.frc, c.acc);  // constraints on: energy only
}

}  // namespace smd
