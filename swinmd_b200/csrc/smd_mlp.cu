// Per-site network giving the initial guess of the induced dipoles.
//
// The induced dipoles are solved to the same tolerance from whatever start
// the solver is given; this network only supplies a better start than the
// first-order guess p0 = alpha E0, so the solve needs fewer iterations.
//
// Inputs (F = 20 per site, all invariant under rotation of the system):
//   0-2   permanent field E0 at the site in the site's own axes (u, v, w)
//   3     |E0|
//   4-9   E0 at the molecule's two other sites, in this site's axes
//   10-17 radial densities of the neighbours within the cutoff:
//         sum_j exp(-(r - R_k)^2 / 2s^2) fc(r), R_k = 0.22 + 0.09 k nm,
//         s = 0.05 nm, fc = (cos(pi r/rc) + 1)/2
//   18-19 site type (H, O) one-hot
// Output (3): 1000 (p - alpha E0) in the site axes; the guess is
//   p0 = alpha E0 + (u, v, w) y / 1000.
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
constexpr float TARGET_SCALE = 1000.0f;
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

// MLP_FTPP lanes per site split the neighbour row; the radial densities are
// combined by shuffles in a fixed order
constexpr int MLP_FTPP = 8;
__global__ void k_mlp_features(int n, const int *nbr, const int *nnbr, const int *mol, const int *mol_off,
                               const int *mol_atoms, const double4 *pos4, Box box, double rc,
                               const double *frame, const double *e0, float *x) {
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gt / MLP_FTPP, t = gt % MLP_FTPP;
    float g[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    double4 pi = make_double4(0, 0, 0, 0);
    if (i < n) {
        pi = pos4[i];
        const int cnt = nnbr[i];
        const float rcf = (float)rc, irc = 1.f / (float)rc;
        for (int k = t; k < cnt; k += MLP_FTPP) {
            const int j = nbr[(size_t)k * n + i] & 0x7fffffff;
            const double4 pj = pos4[j];
            const double dx = pbc1(pj.x - pi.x, box.L[0], box.half[0]);
            const double dy = pbc1(pj.y - pi.y, box.L[1], box.half[1]);
            const double dz = pbc1(pj.z - pi.z, box.L[2], box.half[2]);
            const float r = sqrtf((float)(dx * dx + dy * dy + dz * dz));
            if (r >= rcf) continue;
            const float fc = 0.5f * (cospif(r * irc) + 1.f);
            for (int b = 0; b < 8; b++) {
                const float d = r - (0.22f + 0.09f * b);
                g[b] += expf(-d * d * 200.f) * fc;   // 1 / (2 * 0.05^2)
            }
        }
    }
    for (int b = 0; b < 8; b++) g[b] = group_sum<MLP_FTPP>(g[b]);
    if (i >= n || t != 0) return;
    float f[MF];
    const V3 E = v3(e0[i], e0[n + i], e0[2 * n + i]);
    const V3 El = in_axes(frame, n, i, E);
    f[0] = (float)El.x; f[1] = (float)El.y; f[2] = (float)El.z;
    f[3] = (float)len(E);
    int q = 4;
    const int m = mol[i];
    for (int k = mol_off[m]; k < mol_off[m + 1] && q < 10; k++) {
        const int j = mol_atoms[k];
        if (j == i) continue;
        const V3 Ej = in_axes(frame, n, i, v3(e0[j], e0[n + j], e0[2 * n + j]));
        f[q++] = (float)Ej.x; f[q++] = (float)Ej.y; f[q++] = (float)Ej.z;
    }
    for (; q < 10; q++) f[q] = 0.f;
    for (int b = 0; b < 8; b++) f[10 + b] = g[b];
    const int ty = (int)pi.w;
    f[18] = ty == 0 ? 1.f : 0.f;
    f[19] = ty == 0 ? 0.f : 1.f;
    for (int k = 0; k < MF; k++) x[(size_t)i * MF + k] = f[k];
}

// appends (features, target) rows of the current configuration
__global__ void k_mlp_collect(int n, const float *x, const double *frame, const double *e0, const double *p,
                              const double4 *pos4, const double *polar, float *data, long long row0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float *row = data + (size_t)(row0 + i) * (MF + MO);
    for (int k = 0; k < MF; k++) row[k] = x[(size_t)i * MF + k];
    const double a = fmax(1e-8, polar[(int)pos4[i].w]);
    const V3 d = v3(p[i] - a * e0[i], p[n + i] - a * e0[n + i], p[2 * n + i] - a * e0[2 * n + i]);
    const V3 dl = in_axes(frame, n, i, d);
    row[MF] = (float)dl.x * TARGET_SCALE;
    row[MF + 1] = (float)dl.y * TARGET_SCALE;
    row[MF + 2] = (float)dl.z * TARGET_SCALE;
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

__global__ void k_mlp_infer(int n, const float *x, const float *norm, const float *Wg, const double *frame,
                            const double *e0, const double4 *pos4, const double *polar, double *p) {
    __shared__ float W[MLP_NPARAM];
    for (int k = threadIdx.x; k < MLP_NPARAM; k += blockDim.x) W[k] = Wg[k];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float xn[MF], h1[MH], y[MO];
    for (int f = 0; f < MF; f++) xn[f] = (x[(size_t)i * MF + f] - norm[f]) * norm[MF + f];
    mlp_forward(W, xn, h1, y);
    const double a = fmax(1e-8, polar[(int)pos4[i].w]);
    const V3 u = axis(frame, n, i, 0), v = axis(frame, n, i, 1), w = axis(frame, n, i, 2);
    const V3 d = (y[0] / TARGET_SCALE) * u + (y[1] / TARGET_SCALE) * v + (y[2] / TARGET_SCALE) * w;
    p[i] = a * e0[i] + d.x;
    p[n + i] = a * e0[n + i] + d.y;
    p[2 * n + i] = a * e0[2 * n + i] + d.z;
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
    k_mlp_features<<<(int)(((long long)c.n * MLP_FTPP + 127) / 128), 128, 0, c.stream>>>(c.n, c.pl.nbr, c.pl.nnbr, c.mol, c.mol_off,
                                                            c.mol_atoms, c.pos4, c.box, c.cutoff, c.frame,
                                                            c.e0, c.mlp_x);
}

void launch_mlp_guess(Ctx &c) {
    launch_mlp_features(c);
    k_mlp_infer<<<(c.n + 127) / 128, 128, 0, c.stream>>>(c.n, c.mlp_x, c.mlp_norm, c.mlp_w, c.frame, c.e0,
                                                         c.pos4, c.type_polar, c.pind);
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
    k_mlp_collect<<<(c.n + 127) / 128, 128, 0, c.stream>>>(c.n, c.mlp_x, c.frame, c.e0, c.pind, c.pos4,
                                                           c.type_polar, c.mlp_data, c.mlp_rows);
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
