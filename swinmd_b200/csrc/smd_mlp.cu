// Per-site network giving the initial guess of the induced dipoles.
//
// The induced dipoles are solved to the same tolerance from whatever start
// the solver is given; this guess only brings the start closer, so the solve
// needs fewer iterations.  The guess is the previous step's converged
// dipoles moved by the linear response to the change of the permanent field,
// pl = p(t-1) + alpha (E0(t) - E0(t-1)), plus a correction the network
// predicts (the mutual induction the first-order response leaves out).
// Each time step stores its converged dipoles and permanent field.
//
// Inputs (F = 20 per site, in the site's own axes u, v, w, so invariant under
// rotation of the system):
//   0-2   permanent field E0(t) at the site
//   3     |E0(t)|
//   4-6   E0(t) - E0(t-1)
//   7-12  E0(t) at the molecule's two other sites
//   13-15 p(t-1)
//   16-18 p(t-1) - p(t-2)
//   19    site type (O = 1, H = 0)
// Output (3): 1e5 (p - pl) in the site axes.
// Network: F -> 64 -> 64 -> 3, tanh hidden activations, FP32 weights.
// Training (on rows the solver itself produced): mean-squared error, Adam,
// forward and backward on the GPU with one thread per row; weight gradients
// are reduced within a warp by shuffles, then per block in shared memory,
// then over blocks in a fixed order by the Adam kernel.
#include <cmath>
#include <vector>
#include "smd_ctx.cuh"
#include "smd_polar.cuh"

namespace smd {

constexpr int MF = 20, MH = 64, MO = 3;
constexpr int OW1 = 0, OB1 = OW1 + MH * MF, OW2 = OB1 + MH, OB2 = OW2 + MH * MH, OW3 = OB2 + MH,
              OB3 = OW3 + MO * MH, MLP_NPARAM = OB3 + MO;
constexpr float TARGET_SCALE = 1.0e5f;
constexpr int MLP_THREADS = 256;
constexpr int MLP_MAX_BLOCKS = 64;

// ---------------------------------------------------------------------------
// features and targets
// ---------------------------------------------------------------------------
__device__ __forceinline__ V3 axis(const double *frame, int n, int i, int a) {
    return v3(frame[(size_t)(3 * a) * n + i], frame[(size_t)(3 * a + 1) * n + i], frame[(size_t)(3 * a + 2) * n + i]);
}
__device__ __forceinline__ V3 in_axes(const double *frame, int n, int i, V3 e) {
    return v3(dot(axis(frame, n, i, 0), e), dot(axis(frame, n, i, 1), e), dot(axis(frame, n, i, 2), e));
}

// stored step k = 1, 2 (most recent first): dipole and permanent field of
// site i; the ring holds [4][6][N] (p x y z, E0 x y z), flags[2] counts steps
__device__ __forceinline__ V3 hist_p(const double *ph, int n, int cnt, int k, int i) {
    const double *h = ph + (size_t)((cnt - k) & 3) * 6 * n;
    return v3(h[i], h[n + i], h[2 * n + i]);
}
__device__ __forceinline__ V3 hist_e(const double *ph, int n, int cnt, int k, int i) {
    const double *h = ph + (size_t)((cnt - k) & 3) * 6 * n + 3 * (size_t)n;
    return v3(h[i], h[n + i], h[2 * n + i]);
}

// first-order guess: the previous dipoles moved by dl, the response of the
// molecule's block to the change of the permanent field (k_blk_response;
// dl = M^-1 E0 when nothing is stored)
__device__ __forceinline__ V3 linear_guess(const double *ph, int n, int cnt, int i, const double *dl) {
    const V3 r = v3(dl[i], dl[n + i], dl[2 * n + i]);
    if (cnt < 1) return r;
    return hist_p(ph, n, cnt, 1, i) + r;
}

// the F inputs of site i (one thread)
__device__ __forceinline__ void site_features(int i, int n, int cnt, const int *mol, const int *mol_off,
                                              const int *mol_atoms, const double4 *pos4, const double *frame,
                                              const double *e0, const double *ph, float (&f)[MF]) {
    const V3 E = v3(e0[i], e0[n + i], e0[2 * n + i]);
    const V3 El = in_axes(frame, n, i, E);
    f[0] = (float)El.x; f[1] = (float)El.y; f[2] = (float)El.z;
    f[3] = (float)len(E);
    for (int q = 4; q < 19; q++) f[q] = 0.f;
    if (cnt >= 2) {
        const V3 dE = in_axes(frame, n, i, E - hist_e(ph, n, cnt, 1, i));
        const V3 p1 = hist_p(ph, n, cnt, 1, i);
        const V3 pl = in_axes(frame, n, i, p1), dp = in_axes(frame, n, i, p1 - hist_p(ph, n, cnt, 2, i));
        f[4] = (float)dE.x; f[5] = (float)dE.y; f[6] = (float)dE.z;
        f[13] = (float)pl.x; f[14] = (float)pl.y; f[15] = (float)pl.z;
        f[16] = (float)dp.x; f[17] = (float)dp.y; f[18] = (float)dp.z;
    }
    int q = 7;
    const int m = mol[i];
    for (int k = mol_off[m]; k < mol_off[m + 1] && q < 13; k++) {
        const int j = mol_atoms[k];
        if (j == i) continue;
        const V3 Ej = in_axes(frame, n, i, v3(e0[j], e0[n + j], e0[2 * n + j]));
        f[q++] = (float)Ej.x; f[q++] = (float)Ej.y; f[q++] = (float)Ej.z;
    }
    f[19] = (int)pos4[i].w == 0 ? 0.f : 1.f;
}

__global__ void k_mlp_features(int n, const int *mol, const int *mol_off, const int *mol_atoms,
                               const double4 *pos4, const double *frame, const double *e0, const double *ph,
                               const int *flags, float *x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float f[MF];
    site_features(i, n, flags[2], mol, mol_off, mol_atoms, pos4, frame, e0, ph, f);
    for (int k = 0; k < MF; k++) x[(size_t)i * MF + k] = f[k];
}

// appends (features, target) rows of the current configuration: the target
// is what the network should add to the first-order guess (needs 2 stored steps)
__global__ void k_mlp_collect(int n, const float *x, const double *frame, const double *p, const double *dl,
                              const double *ph, const int *flags, float *data, long long row0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float *row = data + (size_t)(row0 + i) * (MF + MO);
    for (int k = 0; k < MF; k++) row[k] = x[(size_t)i * MF + k];
    const V3 pl = linear_guess(ph, n, flags[2], i, dl);
    const V3 dt = in_axes(frame, n, i, v3(p[i], p[n + i], p[2 * n + i]) - pl);
    row[MF] = (float)dt.x * TARGET_SCALE;
    row[MF + 1] = (float)dt.y * TARGET_SCALE;
    row[MF + 2] = (float)dt.z * TARGET_SCALE;
}

// feature mean and 1/std over the collected rows (one block, fixed order)
__global__ void k_mlp_norm(long long rows, const float *data, float *norm) {
    __shared__ double s1[MF][8], s2[MF][8];
    const int f = threadIdx.x % MF, part = threadIdx.x / MF;  // 8 parts x 20 features = 160 threads
    double a = 0, b = 0;
    if (part < 8)
        for (long long r = part; r < rows; r += 8) {
            const double v = data[r * (MF + MO) + f];
            a += v;
            b += v * v;
        }
    if (part < 8) { s1[f][part] = a; s2[f][part] = b; }
    __syncthreads();
    if (threadIdx.x < MF) {
        double m = 0, q = 0;
        for (int p = 0; p < 8; p++) { m += s1[threadIdx.x][p]; q += s2[threadIdx.x][p]; }
        m /= (double)rows;
        double var = q / (double)rows - m * m;
        norm[threadIdx.x] = (float)m;
        norm[MF + threadIdx.x] = (float)(1.0 / sqrt(var > 1e-12 ? var : 1.0));
    }
}

// ---------------------------------------------------------------------------
// forward / backward
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mlp_forward(const float *W, const float *xn, float h1[MH], float y[MO]) {
    for (int k = 0; k < MH; k++) {
        float z = W[OB1 + k];
        for (int f = 0; f < MF; f++) z = fmaf(W[OW1 + k * MF + f], xn[f], z);
        h1[k] = tanhf(z);
    }
    for (int o = 0; o < MO; o++) y[o] = W[OB3 + o];
    for (int j = 0; j < MH; j++) {
        float z = W[OB2 + j];
        for (int k = 0; k < MH; k++) z = fmaf(W[OW2 + j * MH + k], h1[k], z);
        const float h2 = tanhf(z);
        for (int o = 0; o < MO; o++) y[o] = fmaf(W[OW3 + o * MH + j], h2, y[o]);
    }
}

// Inference with MLP_ITPP threads per site, features computed in the same
// kernel (one thread per site, while the block stages the weights).  Each
// thread computes MH / MLP_ITPP hidden units of each layer; weights and
// activations sit in shared memory in rows padded to a multiple of four
// floats, read as float4 with four partial sums per unit (the two operands
// of four multiply-adds in two 16-byte loads); the three outputs are summed
// over the site's threads by shuffles.
constexpr int MLP_ITPP = 4;
constexpr int MLP_IBLOCK = 128;
constexpr int MLP_ISITES = MLP_IBLOCK / MLP_ITPP;
constexpr int HP = MH + 4;   // padded row of hidden activations / of W2
static_assert(MF % 4 == 0 && MH % 4 == 0 && OW2 % 4 == 0, "float4 rows");
__device__ __forceinline__ float dot4(const float4 *w, const float4 *h, int cnt4, float z) {
    float z1 = 0.f, z2 = 0.f, z3 = 0.f;
#pragma unroll
    for (int k = 0; k < cnt4; k++) {
        const float4 a = w[k], b = h[k];
        z = fmaf(a.x, b.x, z); z1 = fmaf(a.y, b.y, z1); z2 = fmaf(a.z, b.z, z2); z3 = fmaf(a.w, b.w, z3);
    }
    return (z + z1) + (z2 + z3);
}
__global__ void __launch_bounds__(MLP_IBLOCK) k_mlp_infer(int n, const int *mol, const int *mol_off,
                                                          const int *mol_atoms, const double4 *pos4,
                                                          const double *e0, const float *norm, const float *Wg,
                                                          const double *frame, const double *dl,
                                                          const double *ph, const int *flags, double *p) {
    __shared__ __align__(16) float sW1[MH * MF];
    __shared__ __align__(16) float sW2[MH * HP];
    __shared__ __align__(16) float sX[MLP_ISITES][MF];
    __shared__ __align__(16) float sH1[MLP_ISITES][HP];
    __shared__ float sB1[MH], sB2[MH], sW3[MO * MH], sB3[MO];
    const int cnt = flags[2];
    {
        const float4 *g1 = (const float4 *)(Wg + OW1), *g2 = (const float4 *)(Wg + OW2);
        for (int k = threadIdx.x; k < MH * MF / 4; k += blockDim.x) ((float4 *)sW1)[k] = g1[k];
        for (int k = threadIdx.x; k < MH * MH / 4; k += blockDim.x) {
            const int j = k / (MH / 4), c4 = k - j * (MH / 4);
            *(float4 *)&sW2[j * HP + 4 * c4] = g2[k];
        }
    }
    for (int k = threadIdx.x; k < MO * MH; k += blockDim.x) sW3[k] = Wg[OW3 + k];
    for (int k = threadIdx.x; k < MH; k += blockDim.x) { sB1[k] = Wg[OB1 + k]; sB2[k] = Wg[OB2 + k]; }
    if (threadIdx.x < MO) sB3[threadIdx.x] = Wg[OB3 + threadIdx.x];
    if (threadIdx.x < MLP_ISITES) {
        const int is = blockIdx.x * MLP_ISITES + threadIdx.x;
        float f[MF];
        if (is < n) site_features(is, n, cnt, mol, mol_off, mol_atoms, pos4, frame, e0, ph, f);
#pragma unroll
        for (int k = 0; k < MF; k++) sX[threadIdx.x][k] = is < n ? (f[k] - norm[k]) * norm[MF + k] : 0.f;
    }
    const int ls = threadIdx.x / MLP_ITPP, t = threadIdx.x % MLP_ITPP;
    const int i = blockIdx.x * MLP_ISITES + ls;
    const bool own = i < n;
    __syncthreads();
    for (int j = t; j < MH; j += MLP_ITPP)
        sH1[ls][j] = tanhf(dot4((const float4 *)&sW1[j * MF], (const float4 *)sX[ls], MF / 4, sB1[j]));
    __syncthreads();
    float y0 = 0.f, y1 = 0.f, y2 = 0.f;
    for (int j = t; j < MH; j += MLP_ITPP) {
        const float h2 = tanhf(dot4((const float4 *)&sW2[j * HP], (const float4 *)sH1[ls], MH / 4, sB2[j]));
        y0 = fmaf(sW3[j], h2, y0);
        y1 = fmaf(sW3[MH + j], h2, y1);
        y2 = fmaf(sW3[2 * MH + j], h2, y2);
    }
    y0 = group_sum<MLP_ITPP>(y0) + sB3[0];
    y1 = group_sum<MLP_ITPP>(y1) + sB3[1];
    y2 = group_sum<MLP_ITPP>(y2) + sB3[2];
    if (!own || t != 0) return;
    V3 g = linear_guess(ph, n, cnt, i, dl);
    if (cnt >= 2) {
        const V3 u = axis(frame, n, i, 0), v = axis(frame, n, i, 1), w = axis(frame, n, i, 2);
        g = g + (y0 / TARGET_SCALE) * u + (y1 / TARGET_SCALE) * v + (y2 / TARGET_SCALE) * w;
    }
    p[i] = g.x;
    p[n + i] = g.y;
    p[2 * n + i] = g.z;
}

// gradient of the batch loss (1/(3B)) sum (y - t)^2 ; rows idx[r0 .. r0+B)
__device__ __forceinline__ void acc_grad(float *g, int k, float v) {
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) atomicAdd(&g[k], v);
}

__global__ void __launch_bounds__(MLP_THREADS) k_mlp_grad(long long r0, int batch, long long rows,
                                                          const unsigned int *perm, const float *data,
                                                          const float *norm, const float *Wg, float *part,
                                                          float *loss_part) {
    extern __shared__ float sm[];
    float *W = sm, *G = sm + MLP_NPARAM;
    for (int k = threadIdx.x; k < MLP_NPARAM; k += blockDim.x) { W[k] = Wg[k]; G[k] = 0.f; }
    __syncthreads();
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = r < batch;
    float xn[MF], h1[MH], dh1[MH], y[MO], dy[MO];
    float loss = 0.f;
    long long row = valid ? (long long)perm[(r0 + r) % rows] : 0;
    const float *d = data + row * (MF + MO);
    for (int f = 0; f < MF; f++) xn[f] = valid ? (d[f] - norm[f]) * norm[MF + f] : 0.f;
    mlp_forward(W, xn, h1, y);
    const float scale = 2.f / (3.f * (float)batch);
    for (int o = 0; o < MO; o++) {
        const float e = valid ? y[o] - d[MF + o] : 0.f;
        loss += e * e;
        dy[o] = scale * e;
        acc_grad(G, OB3 + o, dy[o]);
    }
    for (int k = 0; k < MH; k++) dh1[k] = 0.f;
    for (int j = 0; j < MH; j++) {
        float z = W[OB2 + j];
        for (int k = 0; k < MH; k++) z = fmaf(W[OW2 + j * MH + k], h1[k], z);
        const float h2 = tanhf(z);
        float dh2 = 0.f;
        for (int o = 0; o < MO; o++) {
            dh2 = fmaf(W[OW3 + o * MH + j], dy[o], dh2);
            acc_grad(G, OW3 + o * MH + j, dy[o] * h2);
        }
        const float dz2 = dh2 * (1.f - h2 * h2);
        acc_grad(G, OB2 + j, dz2);
        for (int k = 0; k < MH; k++) {
            acc_grad(G, OW2 + j * MH + k, dz2 * h1[k]);
            dh1[k] = fmaf(W[OW2 + j * MH + k], dz2, dh1[k]);
        }
    }
    for (int k = 0; k < MH; k++) {
        const float dz1 = dh1[k] * (1.f - h1[k] * h1[k]);
        acc_grad(G, OB1 + k, dz1);
        for (int f = 0; f < MF; f++) acc_grad(G, OW1 + k * MF + f, dz1 * xn[f]);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < MLP_NPARAM; k += blockDim.x) part[(size_t)blockIdx.x * MLP_NPARAM + k] = G[k];
    loss = warp_sum(loss);
    __shared__ float s_l[MLP_THREADS / 32];
    if ((threadIdx.x & 31) == 0) s_l[threadIdx.x >> 5] = loss;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0;
        for (int q = 0; q < MLP_THREADS / 32; q++) t += s_l[q];
        loss_part[blockIdx.x] = t / (3.f * (float)batch);
    }
}

// sums the block partials in a fixed order; Adam update
__global__ void k_mlp_adam(int nblocks, const float *part, float *W, float *m, float *v, float lr, int t,
                           float *grad_out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= MLP_NPARAM) return;
    float g = 0.f;
    for (int b = 0; b < nblocks; b++) g += part[(size_t)b * MLP_NPARAM + k];
    if (grad_out) { grad_out[k] = g; return; }
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    m[k] = b1 * m[k] + (1.f - b1) * g;
    v[k] = b2 * v[k] + (1.f - b2) * g * g;
    const float mh = m[k] / (1.f - powf(b1, (float)t)), vh = v[k] / (1.f - powf(b2, (float)t));
    W[k] -= lr * mh / (sqrtf(vh) + eps);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
void launch_mlp_features(Ctx &c) {
    k_mlp_features<<<(c.n + 127) / 128, 128, 0, c.stream>>>(c.n, c.mol, c.mol_off, c.mol_atoms, c.pos4, c.frame,
                                                            c.e0, c.phist, c.flags, c.mlp_x);
}

void launch_mlp_guess(Ctx &c) {
    double *dl = guess_response(c);
    // with the molecule blocks the block kernel has just formed it
    if (!(c.cg_precond == SMD_PRECOND_MOLECULE && c.cg_blk)) launch_blk_response(c, dl);
    k_mlp_infer<<<(c.n + MLP_ISITES - 1) / MLP_ISITES, MLP_IBLOCK, 0, c.stream>>>(
        c.n, c.mol, c.mol_off, c.mol_atoms, c.pos4, c.e0, c.mlp_norm, c.mlp_w, c.frame, dl, c.phist, c.flags,
        c.pind);
}

// The first-order guess alone, p = p(t-1) + M^-1 (E0(t) - E0(t-1)) (M^-1 E0
// with no stored step): the learned guess with the network's correction left
// out, the baseline that shows what the network adds.
__global__ void k_first_order_guess(int n, const double *dl, const double *ph, const int *flags, double *p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const V3 g = linear_guess(ph, n, flags[2], i, dl);
    p[i] = g.x;
    p[n + i] = g.y;
    p[2 * n + i] = g.z;
}

void launch_first_order_guess(Ctx &c) {
    double *dl = guess_response(c);
    // with the molecule blocks the block kernel has just formed it
    if (!(c.cg_precond == SMD_PRECOND_MOLECULE && c.cg_blk)) launch_blk_response(c, dl);
    k_first_order_guess<<<(c.n + 255) / 256, 256, 0, c.stream>>>(c.n, dl, c.phist, c.flags, c.pind);
}

int mlp_alloc(Ctx &c, long long cap_rows, unsigned int seed) {
    auto al = [](auto **p, size_t cnt) -> bool {
        if (*p) cudaFree(*p);
        *p = nullptr;
        return cudaMalloc((void **)p, (cnt ? cnt : 1) * sizeof(**p)) == cudaSuccess;
    };
    if (!al(&c.mlp_w, MLP_NPARAM) || !al(&c.mlp_m, MLP_NPARAM) || !al(&c.mlp_v, MLP_NPARAM) ||
        // block partials, per-block losses, then room for one gradient
        !al(&c.mlp_part, (size_t)(MLP_MAX_BLOCKS + 1) * MLP_NPARAM + MLP_MAX_BLOCKS) ||
        !al(&c.mlp_norm, 2 * MF) || !al(&c.mlp_x, (size_t)c.n * MF) ||
        !al(&c.mlp_data, (size_t)cap_rows * (MF + MO)))
        return SMD_ERR_CUDA;
    // Glorot-uniform weights from a 32-bit LCG (seeded), zero biases
    std::vector<float> w(MLP_NPARAM, 0.f);
    unsigned int s = seed * 2654435761u + 12345u;
    auto uni = [&]() {
        s = s * 1664525u + 1013904223u;
        return ((s >> 8) & 0xffffff) / 16777216.0f * 2.f - 1.f;
    };
    const float a1 = sqrtf(6.f / (MF + MH)), a2 = sqrtf(6.f / (MH + MH)), a3 = sqrtf(6.f / (MH + MO));
    for (int k = 0; k < MH * MF; k++) w[OW1 + k] = a1 * uni();
    for (int k = 0; k < MH * MH; k++) w[OW2 + k] = a2 * uni();
    for (int k = 0; k < MO * MH; k++) w[OW3 + k] = a3 * uni();
    std::vector<float> z(MLP_NPARAM, 0.f), nrm(2 * MF, 0.f);
    for (int k = 0; k < MF; k++) nrm[MF + k] = 1.f;
    cudaMemcpy(c.mlp_w, w.data(), w.size() * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(c.mlp_m, z.data(), z.size() * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(c.mlp_v, z.data(), z.size() * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(c.mlp_norm, nrm.data(), nrm.size() * 4, cudaMemcpyHostToDevice);
    c.mlp_cap = cap_rows;
    c.mlp_rows = 0;
    c.mlp_t = 0;
    return 0;
}

void launch_mlp_collect(Ctx &c) {
    launch_mlp_features(c);
    double *dl = guess_response(c);
    launch_blk_response(c, dl);   // the blocks of the solve that produced p
    k_mlp_collect<<<(c.n + 127) / 128, 128, 0, c.stream>>>(c.n, c.mlp_x, c.frame, c.pind, dl, c.phist, c.flags,
                                                           c.mlp_data, c.mlp_rows);
}

void launch_mlp_norm(Ctx &c) {
    k_mlp_norm<<<1, 160, 0, c.stream>>>(c.mlp_rows, c.mlp_data, c.mlp_norm);
}

// one optimisation step over rows perm[r0 .. r0 + batch); grad_only: write
// the batch gradient into grad_out instead of updating the weights
void launch_mlp_step(Ctx &c, const unsigned int *perm, long long r0, int batch, float lr, float *grad_out) {
    const int nb = (batch + MLP_THREADS - 1) / MLP_THREADS;
    const size_t smem = 2 * MLP_NPARAM * sizeof(float);
    k_mlp_grad<<<nb, MLP_THREADS, smem, c.stream>>>(r0, batch, c.mlp_rows, perm, c.mlp_data, c.mlp_norm,
                                                    c.mlp_w, c.mlp_part,
                                                    c.mlp_part + (size_t)MLP_MAX_BLOCKS * MLP_NPARAM);
    if (!grad_out) c.mlp_t++;
    k_mlp_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, c.stream>>>(nb, c.mlp_part, c.mlp_w, c.mlp_m, c.mlp_v, lr,
                                                               c.mlp_t, grad_out);
}

int mlp_nparam() { return MLP_NPARAM; }
int mlp_nfeat() { return MF; }
int mlp_max_batch() { return MLP_MAX_BLOCKS * MLP_THREADS; }

// network output for given feature rows (checker entry: x raw features)
__global__ void k_mlp_eval(int rows, const float *x, const float *norm, const float *W, float *y) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    float xn[MF], h1[MH], yy[MO];
    for (int f = 0; f < MF; f++) xn[f] = (x[(size_t)r * MF + f] - norm[f]) * norm[MF + f];
    mlp_forward(W, xn, h1, yy);
    for (int o = 0; o < MO; o++) y[(size_t)r * MO + o] = yy[o];
}

void launch_mlp_eval(Ctx &c, int rows, const float *x, float *y) {
    k_mlp_eval<<<(rows + 127) / 128, 128, 0, c.stream>>>(rows, x, c.mlp_norm, c.mlp_w, y);
}

}  // namespace smd
