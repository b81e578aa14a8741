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
#include <vector>
#include "smd_ctx.cuh"

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

int lustig_lj(Ctx &c, double *out) {
    if (c.vdw != VDW_LJ) return SMD_ERR_ARG;
    double *mass = nullptr;
    double4 *com = nullptr;
    long long *acc = nullptr;
    auto done = [&](int r) {
        cudaFree(mass); cudaFree(com); cudaFree(acc);
        return r;
    };
    if (cudaMalloc(&mass, c.n * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&com, c.nmol * sizeof(double4)) != cudaSuccess ||
        cudaMalloc(&acc, 3 * sizeof(long long)) != cudaSuccess)
        return done(SMD_ERR_CUDA);
    cudaMemcpyAsync(mass, c.h_mass.data(), c.n * sizeof(double), cudaMemcpyHostToDevice, c.stream);
    cudaMemsetAsync(acc, 0, 3 * sizeof(long long), c.stream);
    launch_nlist(c, !c.list_built);
    k_mol_com<<<(c.nmol + 127) / 128, 128, 0, c.stream>>>(c.nmol, c.mol_off, c.mol_atoms, c.pos4, mass, com);
    k_lustig_lj<<<(c.n + 127) / 128, 128, 0, c.stream>>>(c.n, c.pl.nbr, c.pl.nnbr, c.pos4, c.mol, com, c.pair_par,
                                                         c.ntypes, c.box, c.vdw_rc2, c.switch_on,
                                                         c.clen2 != nullptr, acc);
    long long h[3];
    if (cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
        cudaStreamSynchronize(c.stream) != cudaSuccess)
        return done(SMD_ERR_CUDA);
    const double V = c.box.L[0] * c.box.L[1] * c.box.L[2];
    const double su = 0.5 * (double)h[0] / LUS_SCALE, s1 = 0.5 * (double)h[1] / LUS_SCALE,
                 s2 = 0.5 * (double)h[2] / LUS_SCALE;
    out[0] = su + c.e_lrc;
    out[1] = -s1 / (3.0 * V) - 2.0 * c.e_lrc / V;
    out[2] = s2 / (9.0 * V * V) + 6.0 * c.e_lrc / (V * V);
    return done(SMD_OK);
}

}  // namespace smd
