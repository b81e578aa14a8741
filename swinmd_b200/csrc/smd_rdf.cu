// Radial distribution function on the device (RDF::sampling,
// src/observables/RDF.cpp:109-144): every pair of sites that is not
// excluded, minimum image, r^2 < maxR^2 with maxR the smallest half box
// edge, counted into bin (int)(nbins / maxR * r) of the histogram of its
// two types, in both type orders.  The distance arithmetic is written with
// round-to-nearest intrinsics (no fused multiply-adds), in the reference's
// order, so that every pair lands in the reference's bin.
//
// All pairs, tiled: a block takes RD_TILE sites i and walks every later
// site j in tiles of RD_TILE staged in shared memory; counts go to a
// shared-memory histogram (32-bit) and from there to the 64-bit global one
// with integer atomics.
#include "smd_ctx.cuh"

namespace smd {

constexpr int RD_TILE = 256;

// any_excl: some exclusion joins sites of different molecules, so every
// pair is looked up (otherwise only pairs of one molecule are)
__global__ void __launch_bounds__(RD_TILE) k_rdf(int n, int nt, int nbins, const double4 *pos4, const int *mol,
                                                 const int *excl_off, const int *excl, int any_excl, Box box,
                                                 double maxr2, double deltar_r, unsigned long long *hist) {
    extern __shared__ unsigned int s_hist[];   // [nt][nt][nbins]
    __shared__ double4 s_p[RD_TILE];
    __shared__ int s_m[RD_TILE];
    const int nh = nt * nt * nbins;
    for (int k = threadIdx.x; k < nh; k += RD_TILE) s_hist[k] = 0;
    const int i = blockIdx.x * RD_TILE + threadIdx.x;
    const bool own = i < n;
    double4 pi = make_double4(0, 0, 0, 0);
    int mi = -1, ti = 0;
    if (own) {
        pi = pos4[i];
        mi = mol[i];
        ti = (int)pi.w;
    }
    for (int j0 = blockIdx.x * RD_TILE; j0 < n; j0 += RD_TILE) {
        __syncthreads();
        const int jl = j0 + threadIdx.x;
        if (jl < n) {
            s_p[threadIdx.x] = pos4[jl];
            s_m[threadIdx.x] = mol[jl];
        }
        __syncthreads();
        if (!own) continue;
        const int cnt = min(RD_TILE, n - j0);
        for (int q = 0; q < cnt; q++) {
            const int j = j0 + q;
            if (j <= i) continue;
            const double4 pj = s_p[q];
            if (any_excl || s_m[q] == mi) {
                bool ex = false;
                for (int k = excl_off[i]; k < excl_off[i + 1]; k++)
                    if (excl[k] == j) { ex = true; break; }
                if (ex) continue;
            }
            const double x = pbc1(__dsub_rn(pi.x, pj.x), box.L[0], box.half[0]);
            const double y = pbc1(__dsub_rn(pi.y, pj.y), box.L[1], box.half[1]);
            const double z = pbc1(__dsub_rn(pi.z, pj.z), box.L[2], box.half[2]);
            const double r = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
            if (__dmul_rn(r, r) < maxr2) {
                int b = (int)__dmul_rn(deltar_r, r);
                b = b < nbins ? b : nbins - 1;
                const int tj = (int)pj.w;
                atomicAdd(&s_hist[(ti * nt + tj) * nbins + b], 1u);
                atomicAdd(&s_hist[(tj * nt + ti) * nbins + b], 1u);
            }
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nh; k += RD_TILE)
        if (s_hist[k]) atomicAdd(&hist[k], (unsigned long long)s_hist[k]);
}

int rdf_sample(Ctx &c) {
    const int nh = c.ntypes * c.ntypes * c.rdf_nbins;
    const size_t smem = (size_t)nh * sizeof(unsigned int);
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(k_rdf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return SMD_ERR_CUDA;
    k_rdf<<<(c.n + RD_TILE - 1) / RD_TILE, RD_TILE, smem, c.stream>>>(
        c.n, c.ntypes, c.rdf_nbins, c.pos4, c.mol, c.excl_off, c.excl, c.excl_intermol, c.box,
        c.rdf_maxr * c.rdf_maxr,
        c.rdf_nbins / c.rdf_maxr, c.rdf_hist);
    c.rdf_samples++;
    return SMD_OK;
}

}  // namespace smd
