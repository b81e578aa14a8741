// Per-site network giving the initial guess of the induced dipoles.
//
// The induced dipoles are solved to the same tolerance from whatever start
// the solver is given; this guess only brings the start closer, so the solve
// needs fewer iterations.  The guess is an extrapolation of the stored
// steps' dipoles (order 1-3, smd_mlp_set_base: the mutual part p - M^-1 E0 of
// the last steps carried forward, with the molecule blocks' response to this
// step's permanent field), plus a correction the network predicts from the
// site's own descriptors.  Each time step stores its converged dipoles and
// permanent field in a ring of four.
//
// Inputs (F = 24 per site, in the site's own axes u, v, w, so invariant under
// rotation of the system):
//   0-2   permanent field E0(t) at the site
//   3     |E0(t)|
//   4-6   E0(t) - E0(t-1)
//   7-12  E0(t) at the molecule's two other sites
//   13-15 p(t-1)
//   16-18 p(t-1) - p(t-2)
//   19-21 the mutual increment of the last step,
//         p(t-1) - p(t-2) - M^-1 (E0(t-1) - E0(t-2))
//   22    |E0(t) - E0(t-1)|
//   23    site type (O = 1, H = 0)
// Output (3): 1e5 (p - guess) in the site axes.
// Network: F -> 64 -> 64 -> 3, tanh hidden activations; FP32 master
// weights (Adam), BF16 operands of the two wide layers on the tensor cores
// (mma.sync m16n8k16, FP32 accumulation), the 64 -> 3 output layer in FP32.
//
// Every kernel works in warps of 16 rows (sites or training rows): a warp's
// 16 x 64 hidden activations stay in mma accumulator fragments, and the
// accumulator layout of one layer is the operand layout of the next, so the
// two hidden layers chain in registers.  Training runs the backward pass the
// same way (the input gradient of layer 2 is one more mma against W2^T) and
// forms the weight gradients as mma over the block's 64 rows, from
// transposed BF16 tiles in shared memory.  Every sum runs in a fixed order
// (fragments, then shuffles, then warps, then blocks in the Adam kernel), so
// training is deterministic.
#include <cmath>
#include <cstdint>
#include <vector>
#include <cuda_bf16.h>
#include "smd_ctx.cuh"
#include "smd_polar.cuh"

namespace smd {

constexpr int MF = 24, MH = 64, MO = 3;
constexpr int OW1 = 0, OB1 = OW1 + MH * MF, OW2 = OB1 + MH, OB2 = OW2 + MH * MH, OW3 = OB2 + MH,
              OB3 = OW3 + MO * MH, MLP_NPARAM = OB3 + MO;
constexpr float TARGET_SCALE = 1.0e5f;
constexpr int KP = 32;                        // input width padded to two k-steps of 16
constexpr int SX = KP + 8;                    // row stride (bf16) of 32-wide tiles
constexpr int SW = MH + 8;                    // row stride (bf16) of 64-wide tiles
constexpr int MLP_WARPS = 4, MLP_TB = 32 * MLP_WARPS;
constexpr int MLP_CHUNK = 16 * MLP_WARPS;     // rows per block pass
constexpr int MLP_MAX_BLOCKS = 128;
constexpr int MLP_MAX_BATCH = 65536;
static_assert(MF <= KP && MH % 16 == 0, "tile shapes");

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

// extrapolated guess of the given order: the stored dipoles' extrapolation
// plus dl, the molecule block's response to the permanent field's
// difference of the same order (k_blk_response; dl = M^-1 E0 when nothing is
// stored)
__device__ __forceinline__ V3 linear_guess(const double *ph, int n, int cnt, int i, const double *dl, int order) {
    return v3(dl[i] + hist_base_p(ph, n, cnt, order, i), dl[n + i] + hist_base_p(ph, n, cnt, order, n + i),
              dl[2 * n + i] + hist_base_p(ph, n, cnt, order, 2 * (size_t)n + i));
}

// the F inputs of site i (one thread); dlp = M^-1 (E0(t-1) - E0(t-2))
__device__ __forceinline__ void site_features(int i, int n, int cnt, const int *mol, const int *mol_off,
                                              const int *mol_atoms, const double4 *pos4, const double *frame,
                                              const double *e0, const double *ph, const double *dlp,
                                              float (&f)[MF]) {
    const V3 E = v3(e0[i], e0[n + i], e0[2 * n + i]);
    const V3 El = in_axes(frame, n, i, E);
    f[0] = (float)El.x; f[1] = (float)El.y; f[2] = (float)El.z;
    f[3] = (float)len(E);
#pragma unroll
    for (int q = 4; q < MF - 1; q++) f[q] = 0.f;
    if (cnt >= 1) {
        const V3 dE = E - hist_e(ph, n, cnt, 1, i);
        const V3 dEl = in_axes(frame, n, i, dE);
        const V3 p1 = in_axes(frame, n, i, hist_p(ph, n, cnt, 1, i));
        f[4] = (float)dEl.x; f[5] = (float)dEl.y; f[6] = (float)dEl.z;
        f[13] = (float)p1.x; f[14] = (float)p1.y; f[15] = (float)p1.z;
        f[22] = (float)len(dE);
    }
    if (cnt >= 2) {
        const V3 dp = hist_p(ph, n, cnt, 1, i) - hist_p(ph, n, cnt, 2, i);
        const V3 dpl = in_axes(frame, n, i, dp);
        const V3 mut = in_axes(frame, n, i, dp - v3(dlp[i], dlp[n + i], dlp[2 * n + i]));
        f[16] = (float)dpl.x; f[17] = (float)dpl.y; f[18] = (float)dpl.z;
        f[19] = (float)mut.x; f[20] = (float)mut.y; f[21] = (float)mut.z;
    }
    int q = 7;
    const int m = mol[i];
    for (int k = mol_off[m]; k < mol_off[m + 1] && q < 13; k++) {
        const int j = mol_atoms[k];
        if (j == i) continue;
        const V3 Ej = in_axes(frame, n, i, v3(e0[j], e0[n + j], e0[2 * n + j]));
        f[q++] = (float)Ej.x; f[q++] = (float)Ej.y; f[q++] = (float)Ej.z;
    }
    f[MF - 1] = (int)pos4[i].w == 0 ? 0.f : 1.f;
}

__global__ void k_mlp_features(int n, const int *mol, const int *mol_off, const int *mol_atoms,
                               const double4 *pos4, const double *frame, const double *e0, const double *ph,
                               const double *dlp, const int *flags, float *x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float f[MF];
    site_features(i, n, flags[2], mol, mol_off, mol_atoms, pos4, frame, e0, ph, dlp, f);
    for (int k = 0; k < MF; k++) x[(size_t)i * MF + k] = f[k];
}

// appends (features, target) rows of the current configuration: the target
// is what the network should add to the extrapolated guess (needs 2 stored
// steps)
__global__ void k_mlp_collect(int n, const float *x, const double *frame, const double *p, const double *dl,
                              const double *ph, const int *flags, float *data, long long row0, int order) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float *row = data + (size_t)(row0 + i) * (MF + MO);
    for (int k = 0; k < MF; k++) row[k] = x[(size_t)i * MF + k];
    const V3 pl = linear_guess(ph, n, flags[2], i, dl, order);
    const V3 dt = in_axes(frame, n, i, v3(p[i], p[n + i], p[2 * n + i]) - pl);
    row[MF] = (float)dt.x * TARGET_SCALE;
    row[MF + 1] = (float)dt.y * TARGET_SCALE;
    row[MF + 2] = (float)dt.z * TARGET_SCALE;
}

// feature mean and 1/std over the collected rows (one block, fixed order)
__global__ void k_mlp_norm(long long rows, const float *data, float *norm) {
    __shared__ double s1[MF][8], s2[MF][8];
    const int f = threadIdx.x % MF, part = threadIdx.x / MF;  // 8 parts x F features
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
// tensor-core building blocks
// ---------------------------------------------------------------------------
// two floats as one register of two BF16 (the lower index in the low half)
__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}
__device__ __forceinline__ uint32_t ld2(const __nv_bfloat16 *p) { return *reinterpret_cast<const uint32_t *>(p); }

// D += A (16 x 16, row) B (16 x 8, col), BF16 operands, FP32 accumulators.
// Fragments (g = lane / 4, t = lane % 4): a0 = A[g][2t..], a1 = A[g+8][2t..],
// a2 = A[g][2t+8..], a3 = A[g+8][2t+8..]; b0 = B[2t..][g], b1 = B[2t+8..][g];
// d0,d1 = D[g][2t, 2t+1], d2,d3 = D[g+8][2t, 2t+1].
__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// A fragments of 16-wide k-step ks from a row-major BF16 tile (stride ld)
__device__ __forceinline__ void frag_a(uint32_t (&a)[4], const __nv_bfloat16 *tile, int ld, int ks, int g, int t) {
    const __nv_bfloat16 *p = tile + g * ld + ks * 16 + 2 * t;
    a[0] = ld2(p);
    a[1] = ld2(p + 8 * ld);
    a[2] = ld2(p + 8);
    a[3] = ld2(p + 8 * ld + 8);
}
// A fragments of k-step kk taken from accumulator fragments of the previous
// layer (n-tiles 2 kk and 2 kk + 1): the layouts coincide
__device__ __forceinline__ void frag_chain(uint32_t (&a)[4], const float (&h)[8][4], int kk) {
    a[0] = pack2(h[2 * kk][0], h[2 * kk][1]);
    a[1] = pack2(h[2 * kk][2], h[2 * kk][3]);
    a[2] = pack2(h[2 * kk + 1][0], h[2 * kk + 1][1]);
    a[3] = pack2(h[2 * kk + 1][2], h[2 * kk + 1][3]);
}

// weights in shared memory: W1[j][f] (f zero-padded to KP), W2[j][k],
// FP32 biases and output layer
struct MlpW {
    __nv_bfloat16 w1[MH * SX];
    __nv_bfloat16 w2[MH * SW];
    float b1[MH], b2[MH], w3[MO * MH], b3[4];
};

// every thread of the block takes part; w2t (optional): W2^T[k][j]
__device__ __forceinline__ void load_weights(MlpW &S, const float *W, __nv_bfloat16 *w2t) {
    for (int k = threadIdx.x; k < MH * KP; k += blockDim.x) {
        const int j = k / KP, f = k - j * KP;
        S.w1[j * SX + f] = __float2bfloat16_rn(f < MF ? W[OW1 + j * MF + f] : 0.f);
    }
    for (int k = threadIdx.x; k < MH * MH; k += blockDim.x) {
        const int j = k / MH, q = k - j * MH;
        const __nv_bfloat16 v = __float2bfloat16_rn(W[OW2 + k]);
        S.w2[j * SW + q] = v;
        if (w2t) w2t[q * SW + j] = v;
    }
    for (int k = threadIdx.x; k < MH; k += blockDim.x) { S.b1[k] = W[OB1 + k]; S.b2[k] = W[OB2 + k]; }
    for (int k = threadIdx.x; k < MO * MH; k += blockDim.x) S.w3[k] = W[OW3 + k];
    if (threadIdx.x < MO) S.b3[threadIdx.x] = W[OB3 + threadIdx.x];
}

// the two hidden layers of one warp's 16 rows (normalised BF16 inputs in
// xs, row stride SX): h1, h2 after tanh, as accumulator fragments
// the hidden activation: tanhf, or with FAST the hardware approximation
// (tanh.approx.f32, relative error about 2^-11, below the BF16 rounding the
// next layer applies to it); training and the checker's entry use tanhf
template <bool FAST>
__device__ __forceinline__ float act(float x) {
    if (FAST) {
        float y;
        asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
        return y;
    }
    return tanhf(x);
}

template <bool FAST = false>
__device__ __forceinline__ void warp_hidden(const MlpW &S, const __nv_bfloat16 *xs, float (&h1)[8][4],
                                            float (&h2)[8][4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        const float b0 = S.b1[nt * 8 + 2 * t], b1 = S.b1[nt * 8 + 2 * t + 1];
        h1[nt][0] = b0; h1[nt][1] = b1; h1[nt][2] = b0; h1[nt][3] = b1;
    }
#pragma unroll
    for (int ks = 0; ks < KP / 16; ks++) {
        uint32_t a[4];
        frag_a(a, xs, SX, ks, g, t);
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            const __nv_bfloat16 *b = S.w1 + (nt * 8 + g) * SX + ks * 16 + 2 * t;
            mma16816(h1[nt], a, ld2(b), ld2(b + 8));
        }
    }
#pragma unroll
    for (int nt = 0; nt < 8; nt++)
#pragma unroll
        for (int q = 0; q < 4; q++) h1[nt][q] = act<FAST>(h1[nt][q]);
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        const float b0 = S.b2[nt * 8 + 2 * t], b1 = S.b2[nt * 8 + 2 * t + 1];
        h2[nt][0] = b0; h2[nt][1] = b1; h2[nt][2] = b0; h2[nt][3] = b1;
    }
#pragma unroll
    for (int kk = 0; kk < MH / 16; kk++) {
        uint32_t a[4];
        frag_chain(a, h1, kk);
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            const __nv_bfloat16 *b = S.w2 + (nt * 8 + g) * SW + kk * 16 + 2 * t;
            mma16816(h2[nt], a, ld2(b), ld2(b + 8));
        }
    }
#pragma unroll
    for (int nt = 0; nt < 8; nt++)
#pragma unroll
        for (int q = 0; q < 4; q++) h2[nt][q] = act<FAST>(h2[nt][q]);
}

// output layer in FP32: y of rows g (lo) and g + 8 (hi), in every lane of
// the row's quad
__device__ __forceinline__ void warp_out(const MlpW &S, const float (&h2)[8][4], float (&lo)[MO], float (&hi)[MO]) {
    const int t = threadIdx.x & 3;
#pragma unroll
    for (int o = 0; o < MO; o++) {
        float a = 0.f, b = 0.f;
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            const float w0 = S.w3[o * MH + nt * 8 + 2 * t], w1 = S.w3[o * MH + nt * 8 + 2 * t + 1];
            a = fmaf(w0, h2[nt][0], fmaf(w1, h2[nt][1], a));
            b = fmaf(w0, h2[nt][2], fmaf(w1, h2[nt][3], b));
        }
        a += __shfl_xor_sync(0xffffffffu, a, 1);
        a += __shfl_xor_sync(0xffffffffu, a, 2);
        b += __shfl_xor_sync(0xffffffffu, b, 1);
        b += __shfl_xor_sync(0xffffffffu, b, 2);
        lo[o] = a + S.b3[o];
        hi[o] = b + S.b3[o];
    }
}

// sum over the 8 row groups of a warp (lanes with equal t)
__device__ __forceinline__ float rows_sum(float v) {
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    v += __shfl_xor_sync(0xffffffffu, v, 8);
    v += __shfl_xor_sync(0xffffffffu, v, 16);
    return v;
}

// normalised input f of a raw feature row as BF16 (zero past the F inputs)
__device__ __forceinline__ __nv_bfloat16 norm_in(const float *row, const float *norm, int f, bool ok) {
    return __float2bfloat16_rn(ok && f < MF ? (row[f] - norm[f]) * norm[MF + f] : 0.f);
}

// ---------------------------------------------------------------------------
// inference: the start dipoles of the solve
// ---------------------------------------------------------------------------
// One block = 4 warps = 64 sites.  The first 64 threads compute one site's
// features each into a BF16 tile, the warps run the network on 16 sites
// each, and the same 64 threads add the correction to the extrapolated guess.
__global__ void __launch_bounds__(MLP_TB) k_mlp_infer(int n, const int *mol, const int *mol_off,
                                                      const int *mol_atoms, const double4 *pos4, const double *e0,
                                                      const float *norm, const float *Wg, const double *frame,
                                                      const double *dl, const double *dlp, const double *ph,
                                                      const int *flags, double *p, int order) {
    __shared__ __align__(16) MlpW S;
    __shared__ __align__(16) __nv_bfloat16 sX[MLP_CHUNK * SX];
    __shared__ float sY[MLP_CHUNK][MO];
    load_weights(S, Wg, nullptr);
    const int cnt = flags[2];
    const int i = blockIdx.x * MLP_CHUNK + threadIdx.x;
    if (threadIdx.x < MLP_CHUNK) {
        float f[MF];
        if (i < n) site_features(i, n, cnt, mol, mol_off, mol_atoms, pos4, frame, e0, ph, dlp, f);
#pragma unroll
        for (int k = 0; k < KP; k++) {
            float v = 0.f;
            if (k < MF && i < n) v = (f[k < MF ? k : 0] - norm[k < MF ? k : 0]) * norm[MF + (k < MF ? k : 0)];
            sX[threadIdx.x * SX + k] = __float2bfloat16_rn(v);
        }
    }
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    float h1[8][4], h2[8][4], lo[MO], hi[MO];
    warp_hidden<true>(S, sX + 16 * w * SX, h1, h2);
    warp_out(S, h2, lo, hi);
    if (t == 0)
        for (int o = 0; o < MO; o++) {
            sY[16 * w + g][o] = lo[o];
            sY[16 * w + g + 8][o] = hi[o];
        }
    __syncthreads();
    if (threadIdx.x >= MLP_CHUNK || i >= n) return;
    V3 gs = linear_guess(ph, n, cnt, i, dl, order);
    if (cnt >= 2) {
        const V3 u = axis(frame, n, i, 0), v = axis(frame, n, i, 1), ww = axis(frame, n, i, 2);
        const float *y = sY[threadIdx.x];
        gs = gs + (y[0] / TARGET_SCALE) * u + (y[1] / TARGET_SCALE) * v + (y[2] / TARGET_SCALE) * ww;
    }
    p[i] = gs.x;
    p[n + i] = gs.y;
    p[2 * n + i] = gs.z;
}

// network output for given raw feature rows (the checker's entry)
__global__ void __launch_bounds__(MLP_TB) k_mlp_eval(int rows, const float *x, const float *norm, const float *Wg,
                                                     float *y) {
    __shared__ __align__(16) MlpW S;
    __shared__ __align__(16) __nv_bfloat16 sX[MLP_CHUNK * SX];
    load_weights(S, Wg, nullptr);
    const int r0 = blockIdx.x * MLP_CHUNK;
    for (int k = threadIdx.x; k < MLP_CHUNK * KP; k += blockDim.x) {
        const int r = k / KP, f = k - r * KP;
        const bool ok = r0 + r < rows;
        sX[r * SX + f] = norm_in(x + (size_t)(ok ? r0 + r : 0) * MF, norm, f, ok);
    }
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    float h1[8][4], h2[8][4], lo[MO], hi[MO];
    warp_hidden(S, sX + 16 * w * SX, h1, h2);
    warp_out(S, h2, lo, hi);
    if (t != 0) return;
    const int ra = r0 + 16 * w + g, rb = ra + 8;
    for (int o = 0; o < MO; o++) {
        if (ra < rows) y[(size_t)ra * MO + o] = lo[o];
        if (rb < rows) y[(size_t)rb * MO + o] = hi[o];
    }
}

// ---------------------------------------------------------------------------
// training: gradient of the batch loss (1/(3B)) sum (y - t)^2
// ---------------------------------------------------------------------------
// Block b takes rows [b per, (b + 1) per) of the batch (per a multiple of 64)
// in passes of 64 rows.  Per pass each warp runs the forward and backward of
// its 16 rows in registers and writes the BF16 tiles the weight gradients
// need transposed (rows innermost) into shared memory; then warp w forms the
// gradient rows 16 w .. 16 w + 15 of W2 (64 x 64) and of W1 (64 x 32) as
// mma over the 64 rows, accumulating across passes in registers.  Bias and
// output-layer gradients are column sums (shuffles over a warp's rows, then
// per-warp slots in shared memory).  The block writes its partial gradient
// and loss; k_mlp_adam adds the blocks in order.
struct GradSmem {
    MlpW S;
    __nv_bfloat16 w2t[MH * SW];        // W2^T[k][j]
    __nv_bfloat16 x[MLP_CHUNK * SX];   // normalised inputs [row][f]
    __nv_bfloat16 xt[KP * SW];         // [f][row]
    __nv_bfloat16 h1t[MH * SW];        // [k][row]
    __nv_bfloat16 d2t[MH * SW];        // dL/dz2 [j][row]
    __nv_bfloat16 d1t[MH * SW];        // dL/dz1 [k][row]
    float tgt[MLP_CHUNK][4];           // targets, [3] = 1 for a row of the batch
    float acc[MLP_WARPS][2 * MH + MO * MH + 4];   // db1, db2, dW3, db3 per warp
    float loss[MLP_WARPS];
};
constexpr int GA_B1 = 0, GA_B2 = MH, GA_W3 = 2 * MH, GA_B3 = 2 * MH + MO * MH, GA_N = 2 * MH + MO * MH + 4;

__global__ void __launch_bounds__(MLP_TB) k_mlp_grad(long long r0, int batch, int per, long long rows,
                                                     const unsigned int *perm, const float *data, const float *norm,
                                                     const float *Wg, float *part, float *loss_part) {
    extern __shared__ __align__(16) unsigned char smraw[];
    GradSmem &G = *reinterpret_cast<GradSmem *>(smraw);
    load_weights(G.S, Wg, G.w2t);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    for (int k = lane; k < GA_N; k += 32) G.acc[w][k] = 0.f;
    float lsum = 0.f;
    float gW2[8][4], gW1[KP / 8][4];
#pragma unroll
    for (int nt = 0; nt < 8; nt++)
#pragma unroll
        for (int q = 0; q < 4; q++) gW2[nt][q] = 0.f;
#pragma unroll
    for (int nt = 0; nt < KP / 8; nt++)
#pragma unroll
        for (int q = 0; q < 4; q++) gW1[nt][q] = 0.f;
    const float scale = 2.f / (3.f * (float)batch);
    const int b0 = blockIdx.x * per, b1 = min(batch, b0 + per);
    for (int c0 = b0; c0 < b1; c0 += MLP_CHUNK) {
        __syncthreads();   // the previous pass's tiles have been read
        if (threadIdx.x < MLP_CHUNK) {
            const int r = c0 + threadIdx.x;
            const bool ok = r < b1;
            const float *d = data + (ok ? (size_t)perm[(r0 + r) % rows] : 0) * (MF + MO);
            for (int f = 0; f < KP; f++) {
                const __nv_bfloat16 v = norm_in(d, norm, f, ok);
                G.x[threadIdx.x * SX + f] = v;
                G.xt[f * SW + threadIdx.x] = v;
            }
            for (int o = 0; o < MO; o++) G.tgt[threadIdx.x][o] = ok ? d[MF + o] : 0.f;
            G.tgt[threadIdx.x][3] = ok ? 1.f : 0.f;
        }
        __syncthreads();
        const int ra = 16 * w + g, rb = ra + 8;   // this lane's rows in the pass
        float h1[8][4], h2[8][4], lo[MO], hi[MO];
        warp_hidden(G.S, G.x + 16 * w * SX, h1, h2);
        warp_out(G.S, h2, lo, hi);
        float da[MO], db[MO];   // dL/dy of rows ra, rb
        for (int o = 0; o < MO; o++) {
            const float ea = G.tgt[ra][3] != 0.f ? lo[o] - G.tgt[ra][o] : 0.f;
            const float eb = G.tgt[rb][3] != 0.f ? hi[o] - G.tgt[rb][o] : 0.f;
            if (t == 0) lsum += ea * ea + eb * eb;
            da[o] = scale * ea;
            db[o] = scale * eb;
        }
        // output layer: dW3[o][j] = sum_rows dy_o h2_j, db3 = sum_rows dy
#pragma unroll
        for (int nt = 0; nt < 8; nt++)
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const int col = nt * 8 + 2 * t + q;
                for (int o = 0; o < MO; o++) {
                    const float v = rows_sum(da[o] * h2[nt][q] + db[o] * h2[nt][q + 2]);
                    if (g == 0) G.acc[w][GA_W3 + o * MH + col] += v;
                }
            }
        for (int o = 0; o < MO; o++) {
            const float v = rows_sum(da[o] + db[o]);
            if (lane == 0) G.acc[w][GA_B3 + o] += v;
        }
        // dz2 = (W3^T dy) (1 - h2^2), in h2's fragments
#pragma unroll
        for (int nt = 0; nt < 8; nt++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int col = nt * 8 + 2 * t + (q & 1);
                float s = 0.f;
                for (int o = 0; o < MO; o++) s = fmaf(G.S.w3[o * MH + col], q < 2 ? da[o] : db[o], s);
                h2[nt][q] = s * (1.f - h2[nt][q] * h2[nt][q]);
            }
        // dz1 = (W2^T dz2) (1 - h1^2): one more mma per tile against W2^T
        float d1[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; nt++)
#pragma unroll
            for (int q = 0; q < 4; q++) d1[nt][q] = 0.f;
#pragma unroll
        for (int kk = 0; kk < MH / 16; kk++) {
            uint32_t a[4];
            frag_chain(a, h2, kk);
#pragma unroll
            for (int nt = 0; nt < 8; nt++) {
                const __nv_bfloat16 *b = G.w2t + (nt * 8 + g) * SW + kk * 16 + 2 * t;
                mma16816(d1[nt], a, ld2(b), ld2(b + 8));
            }
        }
        // bias gradients, and the transposed tiles of dz2, h1, dz1
#pragma unroll
        for (int nt = 0; nt < 8; nt++)
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const int col = nt * 8 + 2 * t + q;
                const float e1a = d1[nt][q] * (1.f - h1[nt][q] * h1[nt][q]);
                const float e1b = d1[nt][q + 2] * (1.f - h1[nt][q + 2] * h1[nt][q + 2]);
                const float s2 = rows_sum(h2[nt][q] + h2[nt][q + 2]);
                const float s1 = rows_sum(e1a + e1b);
                if (g == 0) {
                    G.acc[w][GA_B2 + col] += s2;
                    G.acc[w][GA_B1 + col] += s1;
                }
                G.d2t[col * SW + ra] = __float2bfloat16_rn(h2[nt][q]);
                G.d2t[col * SW + rb] = __float2bfloat16_rn(h2[nt][q + 2]);
                G.h1t[col * SW + ra] = __float2bfloat16_rn(h1[nt][q]);
                G.h1t[col * SW + rb] = __float2bfloat16_rn(h1[nt][q + 2]);
                G.d1t[col * SW + ra] = __float2bfloat16_rn(e1a);
                G.d1t[col * SW + rb] = __float2bfloat16_rn(e1b);
            }
        __syncthreads();
        // weight gradients over the pass's 64 rows: dW2 = dz2^T h1, dW1 = dz1^T x
#pragma unroll
        for (int ks = 0; ks < MLP_CHUNK / 16; ks++) {
            uint32_t a[4];
            frag_a(a, G.d2t + 16 * w * SW, SW, ks, g, t);
#pragma unroll
            for (int nt = 0; nt < 8; nt++) {
                const __nv_bfloat16 *b = G.h1t + (nt * 8 + g) * SW + ks * 16 + 2 * t;
                mma16816(gW2[nt], a, ld2(b), ld2(b + 8));
            }
            frag_a(a, G.d1t + 16 * w * SW, SW, ks, g, t);
#pragma unroll
            for (int nt = 0; nt < KP / 8; nt++) {
                const __nv_bfloat16 *b = G.xt + (nt * 8 + g) * SW + ks * 16 + 2 * t;
                mma16816(gW1[nt], a, ld2(b), ld2(b + 8));
            }
        }
    }
    // the block's partial gradient
    float *out = part + (size_t)blockIdx.x * MLP_NPARAM;
    const int ja = 16 * w + g, jb = ja + 8;
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        const int k = nt * 8 + 2 * t;
        out[OW2 + ja * MH + k] = gW2[nt][0];
        out[OW2 + ja * MH + k + 1] = gW2[nt][1];
        out[OW2 + jb * MH + k] = gW2[nt][2];
        out[OW2 + jb * MH + k + 1] = gW2[nt][3];
    }
#pragma unroll
    for (int nt = 0; nt < KP / 8; nt++) {
        const int f = nt * 8 + 2 * t;
        if (f < MF) {
            out[OW1 + ja * MF + f] = gW1[nt][0];
            out[OW1 + jb * MF + f] = gW1[nt][2];
        }
        if (f + 1 < MF) {
            out[OW1 + ja * MF + f + 1] = gW1[nt][1];
            out[OW1 + jb * MF + f + 1] = gW1[nt][3];
        }
    }
    lsum = rows_sum(lsum);
    if (lane == 0) G.loss[w] = lsum;
    __syncthreads();
    for (int k = threadIdx.x; k < GA_B3 + MO; k += blockDim.x) {
        float s = 0.f;
        for (int q = 0; q < MLP_WARPS; q++) s += G.acc[q][k];
        if (k < GA_B2) out[OB1 + k] = s;
        else if (k < GA_W3) out[OB2 + k - GA_B2] = s;
        else if (k < GA_B3) out[OW3 + k - GA_W3] = s;
        else out[OB3 + k - GA_B3] = s;
    }
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int q = 0; q < MLP_WARPS; q++) s += G.loss[q];
        loss_part[blockIdx.x] = s / (3.f * (float)batch);
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
// the two hidden layers on the 5th-generation tensor cores (tcgen05)
// ---------------------------------------------------------------------------
// One CTA of 128 threads takes 128 rows (sites or feature rows), thread r
// row r: one M = 128 tile.  The BF16 inputs, the layer-1 activations and
// both weight matrices sit in shared memory in the unswizzled K-major
// layout of the tensor cores' operands (8-row x 16-byte core matrices, the
// 8-row groups 128 B apart, the 8-element K chunks R x 16 B apart for an
// R-row tile); one elected thread issues tcgen05.mma (kind::f16: BF16
// operands, FP32 accumulation in tensor memory, N = 64, K = 16 per
// instruction) and commits to an mbarrier; every thread then reads its own
// row of the accumulator (tensor-memory lane r) with tcgen05.ld, adds the
// bias, applies the activation and writes the BF16 row the next layer
// reads.  Layer 1 takes tensor-memory columns 0-63, layer 2 64-127; the
// 64 -> 3 output layer runs in FP32 in registers.  The mbarrier waits are
// bounded: a wait that runs out sets ST_WAIT_TIMEOUT and the row's output is
// zero.
constexpr int TC_ROWS = 128;

// byte offset of element (row, k) of an R-row K-major tile
__host__ __device__ __forceinline__ uint32_t tc_ofs(int row, int k, int R) {
    return (uint32_t)(((k >> 3) * (R >> 3) + (row >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor (start, leading = K-chunk, stride = 8-row
// group byte offsets; version 1; no swizzle)
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr & 0x3FFFF) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}

struct TcSmem {
    __align__(1024) unsigned char x[TC_ROWS * KP * 2];   // inputs
    __align__(1024) unsigned char h[TC_ROWS * MH * 2];   // layer-1 activations
    __align__(1024) unsigned char w1[MH * KP * 2];
    __align__(1024) unsigned char w2[MH * MH * 2];
    float b1[MH], b2[MH], w3[MO * MH], b3[4];
    __align__(8) unsigned long long mbar;
    unsigned int tbase;
    // keeps the footprint above a fifth of the SM's shared memory: at most
    // four CTAs per SM, whose 4 x 128 tensor-memory columns all fit, so no
    // tcgen05.alloc has to wait for another CTA's release
    unsigned char pad[7 * 1024];
};

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                 "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

// waits for the mbarrier's given phase (bounded); false if it ran out
__device__ __forceinline__ bool tc_wait(uint32_t mb, uint32_t phase) {
    uint32_t done = 0;
    for (int it = 0; it < (1 << 22) && !done; it++)
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done) : "r"(mb), "r"(phase) : "memory");
    return done != 0;
}

// 16 consecutive FP32 columns of this thread's tensor-memory lane
__device__ __forceinline__ void tc_ld16(uint32_t addr, float (&v)[16]) {
    uint32_t u[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]), "=r"(u[7]),
                   "=r"(u[8]), "=r"(u[9]), "=r"(u[10]), "=r"(u[11]), "=r"(u[12]), "=r"(u[13]), "=r"(u[14]), "=r"(u[15])
                 : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; j++) v[j] = __uint_as_float(u[j]);
}

// 8 values as one 16-byte row of a core matrix (BF16, round to nearest)
__device__ __forceinline__ void tc_st8(unsigned char *dst, const float *v) {
    uint4 u;
    uint32_t *w = &u.x;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const __nv_bfloat162 b2 = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
        w[j] = *reinterpret_cast<const uint32_t *>(&b2);
    }
    *reinterpret_cast<uint4 *>(dst) = u;
}

// the weights of the network into the operand layouts
__device__ __forceinline__ void tc_load_weights(TcSmem &S, const float *W) {
    // one 16-byte core-matrix row (8 inputs of output j) per store
    for (int k = threadIdx.x; k < MH * (KP / 8); k += blockDim.x) {
        const int j = k / (KP / 8), f0 = 8 * (k - j * (KP / 8));
        float v[8];
#pragma unroll
        for (int e = 0; e < 8; e++) v[e] = f0 + e < MF ? W[OW1 + j * MF + f0 + e] : 0.f;
        tc_st8(S.w1 + tc_ofs(j, f0, MH), v);
    }
    for (int k = threadIdx.x; k < MH * (MH / 8); k += blockDim.x) {
        const int j = k / (MH / 8), q0 = 8 * (k - j * (MH / 8));
        float v[8];
#pragma unroll
        for (int e = 0; e < 8; e++) v[e] = W[OW2 + j * MH + q0 + e];
        tc_st8(S.w2 + tc_ofs(j, q0, MH), v);
    }
    for (int k = threadIdx.x; k < MH; k += blockDim.x) { S.b1[k] = W[OB1 + k]; S.b2[k] = W[OB2 + k]; }
    for (int k = threadIdx.x; k < MO * MH; k += blockDim.x) S.w3[k] = W[OW3 + k];
    if (threadIdx.x < MO) S.b3[threadIdx.x] = W[OB3 + threadIdx.x];
}

// S.x holds this CTA's 128 input rows; y = the network's output for the
// thread's row.  Every thread of the 128 calls it.
template <bool FAST>
__device__ void tc_forward(TcSmem &S, float (&y)[MO], unsigned int *status) {
    const int tid = threadIdx.x, w = tid >> 5;
    const uint32_t mb = (uint32_t)__cvta_generic_to_shared(&S.mbar);
    if (tid == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb));
    if (w == 0) {
        const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&S.tbase);
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(128));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    // the operand tiles written by the threads, visible to the tensor cores
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = S.tbase;
    // kind::f16: F32 accumulator, BF16 A and B, both K-major, N = 64, M = 128
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(MH >> 3) << 17) |
                           ((uint32_t)(TC_ROWS >> 4) << 24);
    const uint32_t x0 = (uint32_t)__cvta_generic_to_shared(S.x), h0 = (uint32_t)__cvta_generic_to_shared(S.h);
    const uint32_t w10 = (uint32_t)__cvta_generic_to_shared(S.w1), w20 = (uint32_t)__cvta_generic_to_shared(S.w2);
    constexpr uint32_t LA = (TC_ROWS / 8) * 128, LB = (MH / 8) * 128;   // K-chunk strides
    if (tid == 0) {
        for (int ks = 0; ks < KP / 16; ks++)
            tc_mma(tmem, tc_desc(x0 + ks * 2 * LA, LA, 128), tc_desc(w10 + ks * 2 * LB, LB, 128), idesc, ks > 0);
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mb)
                     : "memory");
    }
    bool ok = tc_wait(mb, 0);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t lane_base = tmem + ((uint32_t)(32 * w) << 16);
    if (ok)
        for (int c0 = 0; c0 < MH; c0 += 16) {
            float v[16];
            tc_ld16(lane_base + c0, v);
#pragma unroll
            for (int j = 0; j < 16; j++) v[j] = act<FAST>(v[j] + S.b1[c0 + j]);
            tc_st8(S.h + tc_ofs(tid, c0, TC_ROWS), v);
            tc_st8(S.h + tc_ofs(tid, c0 + 8, TC_ROWS), v + 8);
        }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
        for (int ks = 0; ks < MH / 16; ks++)
            tc_mma(tmem + MH, tc_desc(h0 + ks * 2 * LA, LA, 128), tc_desc(w20 + ks * 2 * LB, LB, 128), idesc, ks > 0);
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mb)
                     : "memory");
    }
    ok = tc_wait(mb, 1) && ok;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    for (int o = 0; o < MO; o++) y[o] = 0.f;
    if (ok) {
        for (int o = 0; o < MO; o++) y[o] = S.b3[o];
        for (int c0 = 0; c0 < MH; c0 += 16) {
            float v[16];
            tc_ld16(lane_base + MH + c0, v);
#pragma unroll
            for (int j = 0; j < 16; j++) {
                const float hj = act<FAST>(v[j] + S.b2[c0 + j]);
                for (int o = 0; o < MO; o++) y[o] = fmaf(S.w3[o * MH + c0 + j], hj, y[o]);
            }
        }
    } else if (tid == 0) {
        atomicOr(status, ST_WAIT_TIMEOUT);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (w == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128));
}

// the learned start on the tensor cores: k_mlp_infer's inputs and output
__global__ void __launch_bounds__(TC_ROWS) k_mlp_infer_tc(int n, const int *mol, const int *mol_off,
                                                          const int *mol_atoms, const double4 *pos4,
                                                          const double *e0, const float *norm, const float *Wg,
                                                          const double *frame, const double *dl, const double *dlp,
                                                          const double *ph, const int *flags, double *p, int order,
                                                          unsigned int *status) {
    __shared__ TcSmem S;
    tc_load_weights(S, Wg);
    const int cnt = flags[2];
    const int i = blockIdx.x * TC_ROWS + threadIdx.x;
    float f[MF];
    if (i < n) site_features(i, n, cnt, mol, mol_off, mol_atoms, pos4, frame, e0, ph, dlp, f);
    float v[KP];
#pragma unroll
    for (int k = 0; k < KP; k++)
        v[k] = (k < MF && i < n) ? (f[k < MF ? k : 0] - norm[k < MF ? k : 0]) * norm[MF + (k < MF ? k : 0)] : 0.f;
#pragma unroll
    for (int k = 0; k < KP; k += 8) tc_st8(S.x + tc_ofs(threadIdx.x, k, TC_ROWS), v + k);
    float y[MO];
    tc_forward<true>(S, y, status);
    if (i >= n) return;
    V3 gs = linear_guess(ph, n, cnt, i, dl, order);
    if (cnt >= 2) {
        const V3 u = axis(frame, n, i, 0), v = axis(frame, n, i, 1), ww = axis(frame, n, i, 2);
        gs = gs + (y[0] / TARGET_SCALE) * u + (y[1] / TARGET_SCALE) * v + (y[2] / TARGET_SCALE) * ww;
    }
    p[i] = gs.x;
    p[n + i] = gs.y;
    p[2 * n + i] = gs.z;
}

// the network's output for raw feature rows on the tensor cores (tanhf, as
// k_mlp_eval)
__global__ void __launch_bounds__(TC_ROWS) k_mlp_eval_tc(int rows, const float *x, const float *norm, const float *Wg,
                                                         float *y, unsigned int *status) {
    __shared__ TcSmem S;
    tc_load_weights(S, Wg);
    const int r = blockIdx.x * TC_ROWS + threadIdx.x;
    const bool ok = r < rows;
    for (int k = 0; k < KP; k++)
        *(__nv_bfloat16 *)(S.x + tc_ofs(threadIdx.x, k, TC_ROWS)) = norm_in(x + (size_t)(ok ? r : 0) * MF, norm, k, ok);
    float out[MO];
    tc_forward<false>(S, out, status);
    if (ok)
        for (int o = 0; o < MO; o++) y[(size_t)r * MO + o] = out[o];
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// the blocks' responses the guess and the features use: dl (the base order's
// field difference) and dlp (the last step's)
static void responses(Ctx &c, int order) {
    launch_blk_response(c, guess_response(c), order, guess_response_prev(c));
}

void launch_mlp_features(Ctx &c) {
    responses(c, c.mlp_base);
    k_mlp_features<<<(c.n + 127) / 128, 128, 0, c.stream>>>(c.n, c.mol, c.mol_off, c.mol_atoms, c.pos4, c.frame,
                                                            c.e0, c.phist, guess_response_prev(c), c.flags,
                                                            c.mlp_x);
}

void launch_mlp_guess(Ctx &c) {
    // with the molecule blocks the block kernel has just formed both
    if (!(c.cg_precond == SMD_PRECOND_MOLECULE && c.cg_blk)) responses(c, c.mlp_base);
    if (c.mlp_tc)
        k_mlp_infer_tc<<<(c.n + TC_ROWS - 1) / TC_ROWS, TC_ROWS, 0, c.stream>>>(
            c.n, c.mol, c.mol_off, c.mol_atoms, c.pos4, c.e0, c.mlp_norm, c.mlp_w, c.frame, guess_response(c),
            guess_response_prev(c), c.phist, c.flags, c.pind, c.mlp_base, c.status);
    else
        k_mlp_infer<<<(c.n + MLP_CHUNK - 1) / MLP_CHUNK, MLP_TB, 0, c.stream>>>(
            c.n, c.mol, c.mol_off, c.mol_atoms, c.pos4, c.e0, c.mlp_norm, c.mlp_w, c.frame, guess_response(c),
            guess_response_prev(c), c.phist, c.flags, c.pind, c.mlp_base);
}

// The extrapolated guess alone (order 1: p = p(t-1) + M^-1 (E0(t) - E0(t-1)),
// M^-1 E0 with no stored step): the learned guess with the network's
// correction left out, the baseline that shows what the network adds.
__global__ void k_first_order_guess(int n, const double *dl, const double *ph, const int *flags, double *p,
                                    int order) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const V3 g = linear_guess(ph, n, flags[2], i, dl, order);
    p[i] = g.x;
    p[n + i] = g.y;
    p[2 * n + i] = g.z;
}

void launch_first_order_guess(Ctx &c) {
    double *dl = guess_response(c);
    const int order = guess_order(c);
    // with the molecule blocks the block kernel has just formed it
    if (!(c.cg_precond == SMD_PRECOND_MOLECULE && c.cg_blk)) launch_blk_response(c, dl, order, nullptr);
    k_first_order_guess<<<(c.n + 255) / 256, 256, 0, c.stream>>>(c.n, dl, c.phist, c.flags, c.pind, order);
}

int mlp_alloc(Ctx &c, long long cap_rows, unsigned int seed) {
    auto al = [](auto **p, size_t cnt) -> bool {
        if (*p) cudaFree(*p);
        *p = nullptr;
        return cudaMalloc((void **)p, (cnt ? cnt : 1) * sizeof(**p)) == cudaSuccess;
    };
    if (!al(&c.mlp_w, MLP_NPARAM) || !al(&c.mlp_m, MLP_NPARAM) || !al(&c.mlp_v, MLP_NPARAM) ||
        // block partials, per-block losses
        !al(&c.mlp_part, (size_t)MLP_MAX_BLOCKS * MLP_NPARAM + MLP_MAX_BLOCKS) ||
        !al(&c.mlp_norm, 2 * MF) || !al(&c.mlp_x, (size_t)c.n * MF) ||
        !al(&c.mlp_data, (size_t)cap_rows * (MF + MO)))
        return SMD_ERR_CUDA;
    if (cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(GradSmem)) !=
        cudaSuccess)
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
    launch_mlp_features(c);   // also the responses, from the blocks of the solve that produced p
    k_mlp_collect<<<(c.n + 127) / 128, 128, 0, c.stream>>>(c.n, c.mlp_x, c.frame, c.pind, guess_response(c),
                                                           c.phist, c.flags, c.mlp_data, c.mlp_rows, c.mlp_base);
}

void launch_mlp_norm(Ctx &c) {
    k_mlp_norm<<<1, 8 * MF, 0, c.stream>>>(c.mlp_rows, c.mlp_data, c.mlp_norm);
}

// blocks of one optimisation step over a batch, and the rows each takes (a
// multiple of the 64-row pass)
static int step_blocks(int batch, int &per) {
    int nb = (batch + MLP_CHUNK - 1) / MLP_CHUNK;
    if (nb > MLP_MAX_BLOCKS) nb = MLP_MAX_BLOCKS;
    per = (batch + nb - 1) / nb;
    per = (per + MLP_CHUNK - 1) / MLP_CHUNK * MLP_CHUNK;
    return (batch + per - 1) / per;
}

// one optimisation step over rows perm[r0 .. r0 + batch); grad_out: write
// the batch gradient there instead of updating the weights
void launch_mlp_step(Ctx &c, const unsigned int *perm, long long r0, int batch, float lr, float *grad_out) {
    int per = 0;
    const int nb = step_blocks(batch, per);
    k_mlp_grad<<<nb, MLP_TB, sizeof(GradSmem), c.stream>>>(r0, batch, per, c.mlp_rows, perm, c.mlp_data,
                                                          c.mlp_norm, c.mlp_w, c.mlp_part,
                                                          c.mlp_part + (size_t)MLP_MAX_BLOCKS * MLP_NPARAM);
    if (!grad_out) c.mlp_t++;
    k_mlp_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, c.stream>>>(nb, c.mlp_part, c.mlp_w, c.mlp_m, c.mlp_v, lr,
                                                               c.mlp_t, grad_out);
}

// mean-squared error of the rows perm[0 .. batch) (weights unchanged)
int mlp_batch_loss(Ctx &c, const unsigned int *perm, int batch, double *loss) {
    int per = 0;
    const int nb = step_blocks(batch, per);
    float *lpart = c.mlp_part + (size_t)MLP_MAX_BLOCKS * MLP_NPARAM;
    k_mlp_grad<<<nb, MLP_TB, sizeof(GradSmem), c.stream>>>(0, batch, per, c.mlp_rows, perm, c.mlp_data,
                                                          c.mlp_norm, c.mlp_w, c.mlp_part, lpart);
    std::vector<float> lp(nb);
    if (cudaMemcpyAsync(lp.data(), lpart, nb * sizeof(float), cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
        cudaStreamSynchronize(c.stream) != cudaSuccess)
        return SMD_ERR_CUDA;
    double t = 0;
    for (int q = 0; q < nb; q++) t += lp[q];
    *loss = t;
    return 0;
}

int mlp_nparam() { return MLP_NPARAM; }
int mlp_nfeat() { return MF; }
int mlp_max_batch() { return MLP_MAX_BATCH; }

void launch_mlp_eval(Ctx &c, int rows, const float *x, float *y) {
    if (c.mlp_tc)
        k_mlp_eval_tc<<<(rows + TC_ROWS - 1) / TC_ROWS, TC_ROWS, 0, c.stream>>>(rows, x, c.mlp_norm, c.mlp_w, y,
                                                                              c.status);
    else
        k_mlp_eval<<<(rows + MLP_CHUNK - 1) / MLP_CHUNK, MLP_TB, 0, c.stream>>>(rows, x, c.mlp_norm, c.mlp_w, y);
}

}  // namespace smd
