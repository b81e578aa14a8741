// Shared device-side definitions of the SwinMD B200 force/integration path.
//
// Data layout in HBM (one system, N sites, M molecules):
//   pos4   double4[N]  x, y, z (nm) and the scaled charge q*sqrt(ke)   FP64 master
//   fixq   int4[N]     x, y, z as 32-bit fractions of the box edge and the
//                      site type: the FP32 pair kernels take exact integer
//                      minimum-image differences from it
//   vel4   double4[N]  on-step velocity, w = 1/m
//   vtm4   double4[N]  leap-frog half-step velocity v(t - dt/2), w = m
//   disp4  double4[N]  displacement since the last pair-list build,
//                      w = unwrapped-position offset bookkeeping (unused)
//   frc    long long[3][N]  forces, 64-bit fixed point (FRC_SCALE units),
//                      SoA so every kernel's owner-thread read-modify-write
//                      is coalesced; integer adds make the total independent
//                      of kernel and thread order
//   acc    long long[ACC_COUNT]  energies and virial, 64-bit fixed point
//   nbr    int[max_nbr][N] full (both directions) Verlet list, column-major
//                      so a warp of consecutive sites reads one row coalesced
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace smd {

// ---- fixed point -----------------------------------------------------------
// Forces: 2^32 units per kJ/mol/nm (resolution 2.3e-10, range +-2.1e9).
constexpr double FRC_SCALE = 4294967296.0;
constexpr double FRC_INV = 1.0 / 4294967296.0;
// Energies and virial terms: 2^28 units per kJ/mol (range +-3.4e10).
constexpr double ACC_SCALE = 268435456.0;
constexpr double ACC_INV = 1.0 / 268435456.0;

__device__ __forceinline__ long long to_fix(double v, double scale) {
    return __double2ll_rn(v * scale);
}

// ---- accumulator slots (acc[]) ---------------------------------------------
enum AccSlot {
    ACC_E_VDW = 0,      // LJ / Mie / BMH / buffered 14-7 pair energy
    ACC_E_REAL = 1,     // Ewald (point-charge or multipole) real-space energy
    ACC_E_LONG = 2,     // Ewald (point-charge or multipole) reciprocal energy
    ACC_E_INTRA = 3,    // Ewald intramolecular correction
    ACC_E_SURF = 4,     // surface-dipole correction
    ACC_E_SELF = 5,     // multipole self energy (point-charge self energy is a constant)
    ACC_E_POL_SELF = 6, // induced-dipole self energy
    ACC_E_POL_REAL = 7, // induced-dipole real-space energy
    ACC_VIR = 8,        // 9 short-range virial components (XX XY XZ YX .. ZZ)
    ACC_LVIR = 17,      // 9 long-range virial components
    ACC_NPAIR = 26,     // pairs inside the short-range cutoff (both directions)
    ACC_E_POL_LONG = 27,  // induced-dipole reciprocal energy
    ACC_E_POL_INTRA = 28, // induced-dipole intramolecular correction
    ACC_E_POL_SURF = 29,  // induced-dipole surface correction
    ACC_E_BOND = 30,      // bond stretching
    ACC_E_ANGLE = 31,     // angle bending
    ACC_E_UB = 32,        // Urey-Bradley
    ACC_COUNT = 33
};

// ---- status word bits (ctx->status on device) --------------------------------
enum StatusBits {
    ST_LIST_OVERFLOW = 1,    // a site had more neighbours than the list holds
    ST_NH_ITER = 2,          // Nose-Hoover implicit velocity iteration hit its cap
    ST_SHAKE_ITER = 4,       // SHAKE did not converge within maxCount
    ST_NAN = 8,              // non-finite force or position
    ST_CELL_RANGE = 16,      // site outside the cell grid after clamping
    ST_CG_ITER = 32,         // dipole solver did not converge
    ST_SHAKE_GEOM = 64,      // SHAKE geometric failure (reference LFIntegrator.cpp:1758)
    ST_WAIT_TIMEOUT = 128,   // a bounded device-side wait (the dipole solve's grid
                             // barrier, the network's tensor-core mbarrier) ran out:
                             // blocks not co-resident, one missing, or no commit
    ST_BOX = 256             // the barostat shrank the box below what the cell grid covers
};

// integrator scalars shared by several files (ctx->scal): 0-7 belong to the
// leap-frog integrator (smd_integrate.cu)
enum ScalShared {
    SC_VNH = 8,      // 4: chain thermostat velocities
    SC_EKIN = 12,    // kinetic energy of the current velocities (chain input)
    SC_SCALE = 13,   // last chain velocity scale
    SC_LE = 14,      // Lees-Edwards offset delta (nm), in [0, Lx)
    SC_LE_B = 15,    // delta at the last pair-list build
    SC_DRMAX = 16,   // displacement^2 limit of the current step's list test
    SC_VLOG = 17,    // barostat velocity vlog (NHIntegrator)
    SC_MOLVIRT = 18, // molVirt: minus the virial pressure of the last forces
    SC_X2 = 19,      // exp(dt vlog): position and box scale of the step
    SC_POLY = 20,    // exp(dt vlog / 2) sinh-series dt: velocity factor of the drift
    SC_VOL = 21,     // volume of the current box
    SC_NSCAL = 32
};

struct Box {
    double L[3];      // edges (nm)
    double half[3];   // L/2
    double inv[3];    // 1/L
};

// Minimum image as the reference's Ensemble::apply_pbc (src/Ensemble.h:319-334):
// while-loops on [-L/2, L/2); positions stay within one box of each other, so
// at most one correction per axis is ever taken.
// The loops are capped: a non-finite coordinate leaves them after a few
// passes instead of spinning (the integrator flags it as ST_NAN).
__device__ __forceinline__ double pbc1(double d, double L, double h) {
    for (int k = 0; k < 8 && d >= h; k++) d -= L;
    for (int k = 0; k < 8 && d < -h; k++) d += L;
    return d;
}

// Lees-Edwards minimum image (sliding images under planar Couette shear):
// the image one box up in y sits delta further in x, so y is reduced first,
// moving x by -/+ delta per crossing, then x and z as pbc1.
__device__ __forceinline__ void min_image_le(double &dx, double &dy, double &dz, const Box &b, double delta) {
    for (int k = 0; k < 8 && dy >= b.half[1]; k++) { dy -= b.L[1]; dx -= delta; }
    for (int k = 0; k < 8 && dy < -b.half[1]; k++) { dy += b.L[1]; dx += delta; }
    dx = pbc1(dx, b.L[0], b.half[0]);
    dz = pbc1(dz, b.L[2], b.half[2]);
}

// The same on 32-bit box fractions: the y difference's wrap count w (from
// the 64-bit difference) takes w Lees-Edwards offsets (as a fraction of Lx,
// modulo 2^32) off the x difference.  frac32 measures y from 0, the box
// from -Ly/2: flipping the top bit measures both from the box edge, so the
// 64-bit difference is the true y difference in units of Ly / 2^32.
__device__ __forceinline__ int le_dx_frac(int fxi, int fyi, int fxj, int fyj, unsigned dfrac) {
    const long long dy64 = (long long)((unsigned)fyj ^ 0x80000000u) - (long long)((unsigned)fyi ^ 0x80000000u);
    const int iy = (int)(unsigned)(dy64 & 0xffffffffLL);
    const long long w = (dy64 - iy) >> 32;
    return (int)((unsigned)fxj - (unsigned)fxi - (unsigned)(w * (long long)dfrac));
}

// Lees-Edwards offset as a fraction of the box edge, modulo 2^32
__device__ __forceinline__ unsigned le_frac(double delta, double invL) {
    double f = delta * invL;
    f -= floor(f);
    return (unsigned)(__double2ll_rn(f * 4294967296.0) & 0xffffffffLL);
}

// Box fraction of a coordinate as an unsigned 32-bit fixed-point number;
// the difference of two, read as a signed int, is the exact minimum image.
__device__ __forceinline__ int frac32(double x, double invL) {
    double f = x * invL;
    f -= floor(f);
    long long v = __double2ll_rn(f * 4294967296.0);
    return (int)(unsigned int)(v & 0xffffffffLL);
}

// Box fractions of a site for the FP32 path.  Under Lees-Edwards images (le)
// a site outside [-Ly/2, Ly/2) in y (molecules are wrapped whole, by their
// centre, so a site can stick out) is first taken to its image inside,
// which moves x by -/+ delta per box crossed in y: the fractions then belong
// to an image of the site, as le_dx_frac requires of both partners.
__device__ __forceinline__ int4 site_frac(double4 p, const Box &b, bool le, double delta) {
    if (le) {
        const double w = floor(p.y * b.inv[1] + 0.5);
        if (w != 0.0) {
            p.y -= w * b.L[1];
            p.x -= w * delta;
        }
    }
    return make_int4(frac32(p.x, b.inv[0]), frac32(p.y, b.inv[1]), frac32(p.z, b.inv[2]), (int)p.w);
}

// Warp helpers ---------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum over `width` consecutive lanes (power of two), result in every lane.
template <int width, typename T>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
    for (int o = width / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, width);
    return v;
}

}  // namespace smd
