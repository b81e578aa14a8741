// Bonded terms of flexible molecules:
//
//   bond     BondForce::compute (src/forces/BondForce.cpp:37-110)
//            r12 = r1 - r2 (minimum image), d = |r12| - r0;
//            harmonic  U = k/2 d^2;  AMOEBA  U = k d^2 (1 - 25.5 d + 379.3125 d^2)
//   angle    AngleForce::compute (src/forces/AngleForce.cpp:34-130)
//            apex atom 2, cos t clamped at -0.9999999; harmonic U = k/2 (t - t0)^2;
//            AMOEBA in degrees D = (t - t0) 180/pi:
//            U = k D^2 (1 - 0.014 D + 5.6e-5 D^2 - 7e-7 D^3 + 2.2e-8 D^4) / (180/pi)^2
//   UB       UreyBradleyForce::compute (src/forces/UreyBradleyForce.cpp:39-100)
//            U = k (|r_H1 - r_H2| - l0)^2 between the first and third site of
//            every molecule
//
// One thread per bond, per angle and per molecule (UB) in one launch; forces
// and torque-free virials go into the fixed-point accumulators with integer
// atomics, so the sums do not depend on thread order.  The virials follow
// each reference class's own component order and sign: bond and angle add
// f_a r_b, Urey-Bradley -f_a r_b (UreyBradleyForce.cpp:77-85), and every
// class subtracts its sum from Ensemble::virial.
#include "smd_ctx.cuh"

namespace smd {

struct BondedArgs {
    int nbond, nangle, nub;          // nub: molecules with a UB term (0: off)
    const int4 *bonds, *angles;
    const double2 *bpar, *apar;
    const int *mol_off, *mol_atoms;
    const double4 *pos4;
    Box box;
    int amoeba;
    double ub_k, ub_l0;
    long long *frc, *acc;
};

__device__ __forceinline__ void add_frc(long long *frc, int n, int i, double fx, double fy, double fz) {
    atomicAdd((unsigned long long *)&frc[i], (unsigned long long)to_fix(fx, FRC_SCALE));
    atomicAdd((unsigned long long *)&frc[n + i], (unsigned long long)to_fix(fy, FRC_SCALE));
    atomicAdd((unsigned long long *)&frc[2 * n + i], (unsigned long long)to_fix(fz, FRC_SCALE));
}

__device__ __forceinline__ void min_d(const double4 &a, const double4 &b, const Box &bx, double &x, double &y,
                                      double &z) {
    x = pbc1(a.x - b.x, bx.L[0], bx.half[0]);
    y = pbc1(a.y - b.y, bx.L[1], bx.half[1]);
    z = pbc1(a.z - b.z, bx.L[2], bx.half[2]);
}

constexpr int BD_THREADS = 128;

// n: sites (the force arrays' stride)
__global__ void __launch_bounds__(BD_THREADS) k_bonded(BondedArgs a, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double e[3] = {0, 0, 0};   // bond, angle, UB
    double w[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};   // local virial, Ensemble gets -w
    if (t < a.nbond) {
        const int4 b = a.bonds[t];
        const double2 par = a.bpar[b.z];
        double x, y, z;
        min_d(a.pos4[b.x], a.pos4[b.y], a.box, x, y, z);
        const double r = sqrt(x * x + y * y + z * z);
        const double d = r - par.x, k = par.y;
        double u, v;
        if (a.amoeba) {
            const double c1 = 25.5, c2 = 379.3125;
            const double an = 1.0 - c1 * d + c2 * d * d;
            u = k * d * d * an;
            v = 2.0 * k * d * an + k * d * d * (-c1 + 2.0 * c2 * d);
        } else {
            u = 0.5 * k * d * d;
            v = k * d;
        }
        const double s = -v / r;
        const double f[3] = {s * x, s * y, s * z}, rr[3] = {x, y, z};
        e[0] = u;
        for (int p = 0; p < 3; p++)
            for (int q = 0; q < 3; q++) w[3 * p + q] += f[p] * rr[q];
        add_frc(a.frc, n, b.x, f[0], f[1], f[2]);
        add_frc(a.frc, n, b.y, -f[0], -f[1], -f[2]);
    } else if (t < a.nbond + a.nangle) {
        const int4 g = a.angles[t - a.nbond];
        const double2 par = a.apar[g.w];
        const double4 p1 = a.pos4[g.x], p2 = a.pos4[g.y], p3 = a.pos4[g.z];
        double x12, y12, z12, x32, y32, z32;
        min_d(p2, p1, a.box, x12, y12, z12);
        min_d(p2, p3, a.box, x32, y32, z32);
        const double d12r = 1.0 / sqrt(x12 * x12 + y12 * y12 + z12 * z12);
        const double d32r = 1.0 / sqrt(x32 * x32 + y32 * y32 + z32 * z32);
        double cs = (x12 * x32 + y12 * y32 + z12 * z32) * d12r * d32r;
        cs = fmax(cs, -0.9999999);
        const double sn = sqrt(1.0 - cs * cs), isn = 1.0 / sn;
        const double th = acos(cs);
        double diff = th - par.x;
        const double k = par.y;
        double u, v;
        if (a.amoeba) {
            const double deg = 180.0 / 3.14159265358979323846;
            const double c1 = 0.014, c2 = 5.6e-5, c3 = 7.0e-7, c4 = 2.2e-8;
            diff *= deg;
            const double d2 = diff * diff, d3 = d2 * diff, d4 = d2 * d2;
            const double an = 1.0 - c1 * diff + c2 * d2 - c3 * d3 + c4 * d4;
            u = k * d2 * an / (deg * deg);
            v = 2.0 * k * diff * an / deg + k * d2 * (-c1 + 2.0 * c2 * diff - 3.0 * c3 * d2 + 4.0 * c4 * d3) / deg;
        } else {
            u = 0.5 * k * diff * diff;
            v = k * diff;
        }
        const double u12[3] = {x12 * d12r, y12 * d12r, z12 * d12r}, u32[3] = {x32 * d32r, y32 * d32r, z32 * d32r};
        const double r12[3] = {x12, y12, z12}, r32[3] = {x32, y32, z32};
        double f1[3], f3[3];
        for (int p = 0; p < 3; p++) {
            f1[p] = v * d12r * isn * (u12[p] * cs - u32[p]);
            f3[p] = v * d32r * isn * (u32[p] * cs - u12[p]);
        }
        e[1] = u;
        for (int p = 0; p < 3; p++)
            for (int q = 0; q < 3; q++) w[3 * p + q] += f1[p] * r12[q] + f3[p] * r32[q];
        add_frc(a.frc, n, g.x, f1[0], f1[1], f1[2]);
        add_frc(a.frc, n, g.y, -(f1[0] + f3[0]), -(f1[1] + f3[1]), -(f1[2] + f3[2]));
        add_frc(a.frc, n, g.z, f3[0], f3[1], f3[2]);
    } else if (t < a.nbond + a.nangle + a.nub) {
        const int m = t - a.nbond - a.nangle;
        const int s0 = a.mol_off[m];
        if (a.mol_off[m + 1] - s0 >= 3) {
            const int i1 = a.mol_atoms[s0], i2 = a.mol_atoms[s0 + 2];
            double x, y, z;
            min_d(a.pos4[i1], a.pos4[i2], a.box, x, y, z);
            const double r = sqrt(x * x + y * y + z * z);
            const double d = r - a.ub_l0;
            const double v = 2.0 * a.ub_k * d;
            const double s = -v / r;
            const double f[3] = {s * x, s * y, s * z}, rr[3] = {x, y, z};
            e[2] = a.ub_k * d * d;
            for (int p = 0; p < 3; p++)
                for (int q = 0; q < 3; q++) w[3 * p + q] -= f[p] * rr[q];
            add_frc(a.frc, n, i1, f[0], f[1], f[2]);
            add_frc(a.frc, n, i2, -f[0], -f[1], -f[2]);
        }
    }
    __shared__ double s_r[BD_THREADS / 32][12];
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    double vals[12] = {e[0], e[1], e[2], w[0], w[1], w[2], w[3], w[4], w[5], w[6], w[7], w[8]};
    for (int q = 0; q < 12; q++) {
        const double sv = warp_sum(vals[q]);
        if (lane == 0) s_r[wp][q] = sv;
    }
    __syncthreads();
    if (threadIdx.x < 12) {
        double sv = 0;
        for (int q = 0; q < BD_THREADS / 32; q++) sv += s_r[q][threadIdx.x];
        const int q = threadIdx.x;
        const int slot = q == 0 ? ACC_E_BOND : (q == 1 ? ACC_E_ANGLE : (q == 2 ? ACC_E_UB : ACC_VIR + (q - 3)));
        if (q >= 3) sv = -sv;   // Ensemble::virial -= the local virial
        if (sv != 0.0) atomicAdd((unsigned long long *)&a.acc[slot], (unsigned long long)to_fix(sv, ACC_SCALE));
    }
}

void launch_bonded(Ctx &c, bool bond, bool angle, bool ub) {
    BondedArgs a;
    a.nbond = bond ? c.nbond : 0;
    a.nangle = angle ? c.nangle : 0;
    a.nub = ub && c.ub_on ? c.nmol : 0;
    const int total = a.nbond + a.nangle + a.nub;
    if (total == 0) return;
    a.bonds = c.bonds; a.angles = c.angles; a.bpar = c.bond_par; a.apar = c.angle_par;
    a.mol_off = c.mol_off; a.mol_atoms = c.mol_atoms; a.pos4 = c.pos4; a.box = c.box;
    a.amoeba = c.bond_form == 2 ? 1 : 0;
    a.ub_k = c.ub_k; a.ub_l0 = c.ub_l0;
    a.frc = c.frc; a.acc = c.acc;
    k_bonded<<<(total + BD_THREADS - 1) / BD_THREADS, BD_THREADS, 0, c.stream>>>(a, c.n);
}

}  // namespace smd
