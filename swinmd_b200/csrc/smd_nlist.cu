// Verlet pair list on the GPU.
//
// Same pair set as CellManager::update_pair_list (src/utils/CellManager.cpp:
// 216-314) and Ensemble::build_pairlist (src/Ensemble.cpp:492-525): all
// unordered pairs (i, j) not in the exclusion table whose minimum-image FP64
// distance squared, computed as the reference computes it, is below
// (cutoff + cutBuff)^2.  Sites are binned with the reference's cell formula
// (CellManager::find_cell, CellManager.h:75-102, clamping included), and the
// 27-cell stencil around each site's cell is the symmetric closure of the
// reference's own-cell + 13-cell half shell, so the list holds each pair in
// both directions ("full list"): every site's forces are then summed by the
// threads that own it, with no atomics.
//
// The list is rebuilt only when flags[0] is set (the integrate kernel raises
// it when a displacement since the last build exceeds cutBuff/2,
// LFIntegrator.cpp:307-341); every kernel here reads the flag and returns at
// once otherwise, so the step can run as one fixed CUDA graph.
#include "smd_ctx.cuh"

namespace smd {

// sc: the box edges over the ones the grid was laid out for (1 but under
// the barostat, which scales positions and box together)
__device__ __forceinline__ int ref_cell(const double4 &p, const CellGrid &g, const double (&sc)[3]) {
    int c[3];
    const double pp[3] = {p.x, p.y, p.z};
#pragma unroll
    for (int d = 0; d < 3; d++) {
        double delta = sc[d] == 1.0 ? pp[d] - g.origin[d] : pp[d] / sc[d] - g.origin[d];
        int x = (int)(delta * g.rlen[d]);
        if (x >= g.n[d]) x = g.n[d] - 1;
        else if (x < 0) x = 0;
        c[d] = x;
    }
    return (c[2] * g.n[1] + c[1]) * g.n[0] + c[0];
}

__global__ void k_bin(int n, const double4 *__restrict__ pos4, CellGrid g, int *cell_of,
                      int *cell_slot, int *cell_count, double4 *disp4, const int *flags, const Box *dbox) {
    if (!flags[0]) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (g.use_cells) {
        double sc[3] = {1.0, 1.0, 1.0};
        if (dbox)
            for (int d = 0; d < 3; d++) sc[d] = dbox->L[d] / g.L0[d];
        int c = ref_cell(pos4[i], g, sc);
        cell_of[i] = c;
        cell_slot[i] = atomicAdd(&cell_count[c], 1);
    }
    disp4[i] = make_double4(0, 0, 0, 0);
}

// Exclusive scan of the cell counts in one block; zeroes the counts for the
// next build.  ncell is small (a few thousand at most for one system).
__global__ void k_scan(int ncell, int *cell_count, int *cell_start, const int *flags) {
    if (!flags[0]) return;
    __shared__ int carry;
    __shared__ int warp_tot[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < ncell; base += blockDim.x) {
        int c = base + threadIdx.x;
        int v = c < ncell ? cell_count[c] : 0;
        int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_tot[w] = x;
        __syncthreads();
        if (w == 0) {
            int t = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            warp_tot[lane] = t;
        }
        __syncthreads();
        int excl = x - v + (w > 0 ? warp_tot[w - 1] : 0) + carry;
        if (c < ncell) {
            cell_start[c] = excl;
            cell_count[c] = 0;
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) cell_start[ncell] = carry;
}

__global__ void k_fill(int n, const int *cell_of, const int *cell_slot, const int *cell_start,
                       int *cell_atoms, const int *flags) {
    if (!flags[0]) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    cell_atoms[cell_start[cell_of[i]] + cell_slot[i]] = i;
}

// One warp per cell: order the cell's sites by index (rank sort), so the
// list rows, and with them every per-thread partial sum, come out the same
// on every run.
__global__ void k_sort_cells(int ncell, const int *cell_start, int *cell_atoms, int *scratch,
                             const int *flags) {
    if (!flags[0]) return;
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (warp >= ncell) return;
    int s = cell_start[warp], e = cell_start[warp + 1];
    for (int k = s + lane; k < e; k += 32) scratch[k] = cell_atoms[k];
    __syncwarp();
    for (int k = s + lane; k < e; k += 32) {
        int v = scratch[k], r = 0;
        for (int q = s; q < e; q++) r += scratch[q] < v;
        cell_atoms[s + r] = v;
    }
}

struct BuildArgs {
    int n, max_nbr;
    const double4 *pos4;
    const int *mol, *excl_off, *excl;
    const int *cell_of, *cell_start, *cell_atoms;
    CellGrid g;
    Box box;
    double rl2;
    int *nbr, *nnbr;
    unsigned int *status;
    const int *flags;
    const double *le;   // Lees-Edwards offset on the device, or null
    const Box *dbox;    // the box on the device (barostat), or null: box
};

// r^2 of the reference's pair test, without contraction into FMA
// (x86-64 -O2 builds of the reference use separate multiply and add).
__device__ __forceinline__ double ref_r2(const double4 &a, const double4 &b, const Box &bx,
                                         bool pbc, bool le, double delta) {
    double dx = __dsub_rn(b.x, a.x), dy = __dsub_rn(b.y, a.y), dz = __dsub_rn(b.z, a.z);
    if (le) {
        min_image_le(dx, dy, dz, bx, delta);
    } else if (pbc) {
        dx = pbc1(dx, bx.L[0], bx.half[0]);
        dy = pbc1(dy, bx.L[1], bx.half[1]);
        dz = pbc1(dz, bx.L[2], bx.half[2]);
    }
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// One warp per site i; candidates are tested 32 at a time and appended in
// candidate order (ballot + popc), so the row order is deterministic.
__device__ void build_site(const BuildArgs &a, int i, int lane) {
    const Box box = a.dbox ? *a.dbox : a.box;
    const double4 pi = a.pos4[i];
    const int mi = a.mol[i];
    const int e0 = a.excl_off[i], e1 = a.excl_off[i + 1];
    const bool le = a.le != nullptr;
    const double delta = le ? *a.le : 0.0;
    int count = 0;
    auto consider = [&](int j, bool pbc, bool valid) {
        bool take = valid && j != i;
        // the distance test first: only the few candidates inside the list
        // radius read the exclusion list
        if (take) take = ref_r2(pi, a.pos4[j], box, pbc, le && pbc, delta) < a.rl2;
        if (take) {
            for (int e = e0; e < e1; e++)
                if (a.excl[e] == j) { take = false; break; }
        }
        unsigned m = __ballot_sync(0xffffffffu, take);
        if (take) {
            int slot = count + __popc(m & ((1u << lane) - 1));
            int v = j | (a.mol[j] == mi ? (int)0x80000000 : 0);
            if (slot < a.max_nbr) a.nbr[(size_t)slot * a.n + i] = v;
        }
        count += __popc(m);
    };
    if (a.g.use_cells) {
        int c = a.cell_of[i];
        int cx = c % a.g.n[0], cy = (c / a.g.n[0]) % a.g.n[1], cz = c / (a.g.n[0] * a.g.n[1]);
        for (int dz = -1; dz <= 1; dz++) {
            int z = cz + dz; z = z < 0 ? z + a.g.n[2] : (z >= a.g.n[2] ? z - a.g.n[2] : z);
            for (int dy = -1; dy <= 1; dy++) {
                int y = cy + dy;
                // under shear, the images across the y boundary sit delta
                // further in x: the x window moves by delta and widens by a cell
                const int wy = y < 0 ? -1 : (y >= a.g.n[1] ? 1 : 0);
                y = y < 0 ? y + a.g.n[1] : (y >= a.g.n[1] ? y - a.g.n[1] : y);
                int sh = 0, dx1 = 1;
                if (le && wy != 0) {
                    sh = (int)floor((wy < 0 ? delta : -delta) * a.g.rlen[0]);
                    dx1 = 2;
                }
                for (int dx = -1; dx <= dx1; dx++) {
                    int x = (cx + sh + dx) % a.g.n[0];
                    x = x < 0 ? x + a.g.n[0] : x;
                    int nc = (z * a.g.n[1] + y) * a.g.n[0] + x;
                    // same-cell pairs are tested without minimum image, as the
                    // reference does (CellManager.cpp:246-262)
                    bool pbc = nc != c;
                    int s = a.cell_start[nc], e = a.cell_start[nc + 1];
                    for (int k = s; k < e; k += 32) {
                        int kk = k + lane;
                        consider(kk < e ? a.cell_atoms[kk] : -1, pbc, kk < e);
                    }
                }
            }
        }
    } else {
        for (int k = 0; k < a.n; k += 32) {
            int j = k + lane;
            consider(j < a.n ? j : -1, true, j < a.n);
        }
    }
    if (lane == 0) {
        if (count > a.max_nbr) {
            atomicOr(a.status, ST_LIST_OVERFLOW);
            count = a.max_nbr;
        }
        a.nnbr[i] = count;
    }
}

__global__ void k_build(BuildArgs a) {
    if (!a.flags[0]) return;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= a.n) return;
    build_site(a, i, threadIdx.x & 31);
}

// The same rows, with the candidates staged in shared memory: a block takes
// BS_SITES sites that are consecutive in cell order (one warp each).  When
// they all lie in one cell they share its 27-cell stencil: the stencil's
// candidates, in build_site's order (cells dz, dy, dx; sites in cell order),
// are staged BS_STAGE at a time with their positions, molecules and a
// same-cell flag, and every warp tests them from shared memory.  Blocks
// whose sites straddle a cell boundary take build_site.  Not for
// Lees-Edwards (sheared) boxes.
constexpr int BS_SITES = 16, BS_STAGE = 1024;
__global__ void __launch_bounds__(BS_SITES * 32) k_build_staged(BuildArgs a) {
    if (!a.flags[0]) return;
    const Box box = a.dbox ? *a.dbox : a.box;
    __shared__ double s_x[BS_STAGE], s_y[BS_STAGE], s_z[BS_STAGE];
    __shared__ int s_j[BS_STAGE], s_m[BS_STAGE];
    __shared__ int s_cell[BS_SITES], s_cs[27], s_off[28], s_nc[27];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int slot = blockIdx.x * BS_SITES + w;
    const bool has = slot < a.n;
    const int i = has ? a.cell_atoms[slot] : -1;
    if (lane == 0) s_cell[w] = has ? a.cell_of[i] : -1;
    __syncthreads();
    const int c = s_cell[0];
    bool same = true;
    for (int q = 1; q < BS_SITES; q++)
        if (s_cell[q] != c && s_cell[q] != -1) same = false;
    if (!same) {   // block-uniform: no barrier follows on this branch
        if (has) build_site(a, i, lane);
        return;
    }
    // the stencil's cells in build_site's order, their ranges and offsets
    if (threadIdx.x < 27) {
        const int t = threadIdx.x, dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
        const int cx = c % a.g.n[0], cy = (c / a.g.n[0]) % a.g.n[1], cz = c / (a.g.n[0] * a.g.n[1]);
        int z = cz + dz; z = z < 0 ? z + a.g.n[2] : (z >= a.g.n[2] ? z - a.g.n[2] : z);
        int y = cy + dy; y = y < 0 ? y + a.g.n[1] : (y >= a.g.n[1] ? y - a.g.n[1] : y);
        int x = (cx + dx) % a.g.n[0];
        x = x < 0 ? x + a.g.n[0] : x;
        const int nc = (z * a.g.n[1] + y) * a.g.n[0] + x;
        s_nc[t] = nc;
        s_cs[t] = a.cell_start[nc];
        s_off[t + 1] = a.cell_start[nc + 1] - a.cell_start[nc];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        s_off[0] = 0;
        for (int t = 0; t < 27; t++) s_off[t + 1] += s_off[t];
    }
    __syncthreads();
    const int total = s_off[27];
    double4 pi = make_double4(0, 0, 0, 0);
    int mi = 0, e0 = 0, e1 = 0, count = 0;
    if (has) {
        pi = a.pos4[i];
        mi = a.mol[i];
        e0 = a.excl_off[i];
        e1 = a.excl_off[i + 1];
    }
    for (int base = 0; base < total; base += BS_STAGE) {
        const int cnt = min(BS_STAGE, total - base);
        __syncthreads();
        for (int f = threadIdx.x; f < cnt; f += BS_SITES * 32) {
            const int g = base + f;
            int t = 0;
            while (s_off[t + 1] <= g) t++;
            const int j = a.cell_atoms[s_cs[t] + g - s_off[t]];
            const double4 pj = a.pos4[j];
            s_x[f] = pj.x; s_y[f] = pj.y; s_z[f] = pj.z;
            s_j[f] = j;
            // same-cell pairs without minimum image, as build_site (flag in bit 31)
            s_m[f] = a.mol[j] | (s_nc[t] == c ? (int)0x80000000 : 0);
        }
        __syncthreads();
        if (!has) continue;
        for (int k = 0; k < cnt; k += 32) {
            const int kk = k + lane;
            const bool valid = kk < cnt;
            const int j = valid ? s_j[kk] : -1;
            const int mj = valid ? s_m[kk] : 0;
            bool take = valid && j != i;
            if (take) {
                const double4 pj = make_double4(s_x[kk], s_y[kk], s_z[kk], 0.0);
                take = ref_r2(pi, pj, box, mj >= 0, false, 0.0) < a.rl2;
            }
            if (take)
                for (int q = e0; q < e1; q++)
                    if (a.excl[q] == j) { take = false; break; }
            const unsigned m = __ballot_sync(0xffffffffu, take);
            if (take) {
                const int at = count + __popc(m & ((1u << lane) - 1));
                if (at < a.max_nbr)
                    a.nbr[(size_t)at * a.n + i] = j | ((mj & 0x7fffffff) == mi ? (int)0x80000000 : 0);
            }
            count += __popc(m);
        }
    }
    if (has && lane == 0) {
        if (count > a.max_nbr) {
            atomicOr(a.status, ST_LIST_OVERFLOW);
            count = a.max_nbr;
        }
        a.nnbr[i] = count;
    }
}

__global__ void k_list_done(int *flags, double *scal_le) {
    if (flags[0]) {
        flags[1] += 1;
        flags[0] = 0;
        // the Lees-Edwards offset this list was built for
        if (scal_le) scal_le[SC_LE_B - SC_LE] = scal_le[0];
    }
}

void launch_nlist(Ctx &c, bool force_rebuild) {
    if (force_rebuild) {
        int one = 1;
        cudaMemcpyAsync(c.flags, &one, sizeof(int), cudaMemcpyHostToDevice, c.stream);
        c.list_built = 1;
    }
    const int T = 256;
    int nb = (c.n + T - 1) / T;
    if (c.grid.use_cells) {
        k_bin<<<nb, T, 0, c.stream>>>(c.n, c.pos4, c.grid, c.pl.cell_of, c.pl.cell_slot,
                                      c.pl.cell_count, c.disp4, c.flags, c.npt ? c.dbox : nullptr);
        k_scan<<<1, 1024, 0, c.stream>>>(c.grid.ncell, c.pl.cell_count, c.pl.cell_start, c.flags);
        k_fill<<<nb, T, 0, c.stream>>>(c.n, c.pl.cell_of, c.pl.cell_slot, c.pl.cell_start,
                                       c.pl.cell_atoms, c.flags);
        int nw = (c.grid.ncell * 32 + T - 1) / T;
        k_sort_cells<<<nw, T, 0, c.stream>>>(c.grid.ncell, c.pl.cell_start, c.pl.cell_atoms,
                                             c.pl.cell_slot /* reused as scratch after fill */,
                                             c.flags);
    } else {
        k_bin<<<nb, T, 0, c.stream>>>(c.n, c.pos4, c.grid, c.pl.cell_of, c.pl.cell_slot,
                                      c.pl.cell_count, c.disp4, c.flags, nullptr);
    }
    BuildArgs a;
    a.n = c.n; a.max_nbr = c.pl.max_nbr; a.pos4 = c.pos4; a.mol = c.mol;
    a.excl_off = c.excl_off; a.excl = c.excl; a.cell_of = c.pl.cell_of;
    a.cell_start = c.pl.cell_start; a.cell_atoms = c.pl.cell_atoms; a.g = c.grid; a.box = c.box;
    a.rl2 = c.pl.rl2; a.nbr = c.pl.nbr; a.nnbr = c.pl.nnbr; a.status = c.status; a.flags = c.flags;
    a.le = c.ip.strain_rate != 0.0 && c.integrator_ready ? c.scal + SC_LE : nullptr;
    a.dbox = c.npt ? c.dbox : nullptr;
    if (c.grid.use_cells && !a.le) {
        k_build_staged<<<(c.n + BS_SITES - 1) / BS_SITES, BS_SITES * 32, 0, c.stream>>>(a);
    } else {
        int nbw = (c.n * 32 + T - 1) / T;
        k_build<<<nbw, T, 0, c.stream>>>(a);
    }
    k_list_done<<<1, 1, 0, c.stream>>>(c.flags, a.le ? c.scal + SC_LE : nullptr);
}

}  // namespace smd
