// Ewald reciprocal-space sum for point charges (EwaldForce::set_up and
// EwaldForce::reciprocal_term, src/forces/EwaldForce.cpp:198-257, 529-698).
//
//   k set : n = (nx, ny, nz), half space (nx > 0, or nx = 0 and ny > 0, or
//           nx = ny = 0 and nz > 0), k = 2 pi n / L, k^2 < kCut^2
//   S(k)  = sum_i q_i exp(i k.r_i)                  (q: scaled charges)
//   E     = sum_k 4 pi/V exp(-k^2/4a^2)/k^2 |S(k)|^2
//   F_i  += k 8 pi/V exp(-k^2/4a^2)/k^2 (q_i sin(k.r_i) Re S - q_i cos(k.r_i) Im S)
//   W_ab += E_k (delta_ab - 2 (1/4a^2 + 1/k^2) k_a k_b)  (long virial)
//
// Three kernels: partial structure factors over (k tile x site chunk)
// blocks, a fixed-order reduction over chunks that also forms the energy and
// virial, and a per-site force pass.  In the FP32 path the phase k.r is an
// exact 32-bit integer sum of n_a times the sites' 32-bit box fractions (the
// wrap mod 2^32 is the wrap mod 2 pi), so the FP32 sine and cosine see an
// argument in [-pi, pi) with no reduction error.
//
// Sheared cell (SLLOD with Lees-Edwards images; no reference code): the
// images of the box with offset d form the lattice a1 = (Lx, 0, 0),
// a2 = (d, Ly, 0), a3 = (0, 0, Lz), whose reciprocal vectors give
// k(n) = 2 pi (nx / Lx, (ny - nx t) / Ly, nz / Lz), t = d / Lx, with d
// reduced to [-Lx/2, Lx/2] (d and d + Lx are the same lattice).  The sums are
// those above over the half space of n with |k| < kcut for that lattice, so
// the k list changes with d: k_le_kset rebuilds it on the device before every
// evaluation, in the order of the unsheared list (nx, ny, nz ascending), and
// the passes read the live count from the device.  The phase is
// n.(fractional coordinates): x's fraction becomes (x - d y / Ly) / Lx.
#include <cmath>
#include <vector>
#include <algorithm>
#include <cstdlib>
#include "smd_ctx.cuh"

namespace smd {

constexpr int RK_THREADS = 128;   // k vectors per structure-factor block
constexpr int RK_CHUNKS = 16;     // site chunks (partial sums per k)
constexpr int RF_TPS = 4;         // threads per site in the force pass

// sin and cos of 2 pi ph / 2^32 for a 32-bit phase: the top 24 bits go
// through sincospif exactly (they fit a float), the low 8 bits (an angle
// below 4e-7 rad) are added to first order, so the argument carries no
// rounding at all.
__device__ __forceinline__ void sincos_phase(int ph, float &s, float &c) {
    const int hi = ph & ~0xff;
    const float b = (float)(ph & 0xff) * 1.4629180792671596e-09f;  // pi / 2^31
    float sh, ch;
    sincospif((float)hi * 4.656612873077393e-10f, &sh, &ch);
    s = fmaf(b, ch, sh);
    c = fmaf(-b, sh, ch);
}

// the Lees-Edwards offset reduced to [-Lx/2, Lx/2]
__device__ __forceinline__ double le_reduced(const double *le, const Box &b) {
    const double d = le ? *le : 0.0;
    return d - b.L[0] * floor(d * b.inv[0] + 0.5);
}

// sheared cell: the 32-bit fraction of x - dd y / Ly along a1
__device__ __forceinline__ int le_xfrac(const double4 &p, double dd, const Box &b) {
    return frac32(p.x - dd * (p.y * b.inv[1]), b.inv[0]);
}

// The k list of the sheared cell (one block): candidates (nx, m, nz) with
// nx in [0, nxm], m in [-nyr, nyr], nz in [-nzm, nzm] and ny = m + rint(nx t)
// cover every n with |k| < kcut (|ny - nx t| <= kcut Ly / 2 pi and
// |nx t - rint(nx t)| <= 1/2).  Each thread takes a contiguous run of
// candidates, counts its members, and after a block-wide exclusive scan
// writes them in candidate order: nx, then ny, then nz ascending.
constexpr int KSET_THREADS = 1024;
__global__ void __launch_bounds__(KSET_THREADS) k_le_kset(int nxm, int nyr, int nzm, Box box, const double *le,
                                                          double kc2, double aR4, double pi4V, int cap, int *kn,
                                                          double *kvec, double *kcoef, int *nk_out) {
    __shared__ int s_w[KSET_THREADS / 32];
    const double PI2 = 6.283185307179586476925;
    const double t = le_reduced(le, box) * box.inv[0];
    const int nys = 2 * nyr + 1, nzs = 2 * nzm + 1;
    const int total = (nxm + 1) * nys * nzs;
    const int per = (total + KSET_THREADS - 1) / KSET_THREADS;
    const int c0 = min(total, (int)threadIdx.x * per), c1 = min(total, c0 + per);
    auto member = [&](int ci, int &nx, int &ny, int &nz, double &kx, double &ky, double &kz, double &k2) {
        nx = ci / (nys * nzs);
        const int r = ci - nx * nys * nzs;
        const int m = r / nzs - nyr;
        nz = r - (m + nyr) * nzs - nzm;
        ny = m + (int)rint(nx * t);
        if (!(nx > 0 || (nx == 0 && ny > 0) || (nx == 0 && ny == 0 && nz > 0))) return false;
        kx = PI2 * nx * box.inv[0];
        ky = PI2 * (ny - nx * t) * box.inv[1];
        kz = PI2 * nz * box.inv[2];
        k2 = kx * kx + ky * ky + kz * kz;
        return k2 < kc2;
    };
    int cnt = 0;
    for (int ci = c0; ci < c1; ci++) {
        int nx, ny, nz;
        double kx, ky, kz, k2;
        if (member(ci, nx, ny, nz, kx, ky, kz, k2)) cnt++;
    }
    // exclusive scan of cnt over the block
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int inc = cnt;
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += v;
    }
    if (lane == 31) s_w[w] = inc;
    __syncthreads();
    if (w == 0) {
        int v = s_w[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += u;
        }
        s_w[lane] = v;   // inclusive totals per warp
    }
    __syncthreads();
    int k = inc - cnt + (w > 0 ? s_w[w - 1] : 0);
    if (threadIdx.x == KSET_THREADS - 1) *nk_out = k + cnt;
    for (int ci = c0; ci < c1 && k < cap; ci++) {
        int nx, ny, nz;
        double kx, ky, kz, k2;
        if (!member(ci, nx, ny, nz, kx, ky, kz, k2)) continue;
        kn[k] = nx; kn[cap + k] = ny; kn[2 * cap + k] = nz;
        kvec[k] = kx; kvec[cap + k] = ky; kvec[2 * cap + k] = kz;
        kcoef[k] = pi4V * (exp(-k2 * aR4) / k2);
        k++;
    }
}

// partial[ch][2][nk]; nk is the stride of the k arrays, *nkd (when given)
// the live count; le (sheared cell) the device offset
template <typename R>
__global__ void __launch_bounds__(RK_THREADS) k_sk_partial(int n, int nk, const int *nkd, const double4 *pos4,
                                                           const int4 *fixq, const int *kn,
                                                           const double *kvec, const double *tq,
                                                           Box box, const double *le, double *partial) {
    __shared__ double4 s_p[RK_THREADS];
    __shared__ int4 s_f[RK_THREADS];
    const int k = blockIdx.x * RK_THREADS + threadIdx.x;
    const int nkv = nkd ? *nkd : nk;
    if ((int)(blockIdx.x * RK_THREADS) >= nkv) return;   // block-uniform: no k of this block is live
    const int ch = blockIdx.y;
    const int per = (n + RK_CHUNKS - 1) / RK_CHUNKS;
    const int s0 = ch * per, s1 = min(n, s0 + per);
    const double dd = le ? le_reduced(le, box) : 0.0;
    int nx = 0, ny = 0, nz = 0;
    double kx = 0, ky = 0, kz = 0;
    if (k < nkv) {
        nx = kn[k]; ny = kn[nk + k]; nz = kn[2 * nk + k];
        kx = kvec[k]; ky = kvec[nk + k]; kz = kvec[2 * nk + k];
    }
    double cs = 0, sn = 0;
    for (int base = s0; base < s1; base += RK_THREADS) {
        const int i = base + threadIdx.x;
        __syncthreads();
        if (i < s1) {
            if (sizeof(R) == 8) {
                s_p[threadIdx.x] = pos4[i];
            } else {
                int4 f = fixq[i];
                if (le) f.x = le_xfrac(pos4[i], dd, box);
                s_f[threadIdx.x] = f;
            }
        }
        __syncthreads();
        const int cnt = min(RK_THREADS, s1 - base);
        if (k < nkv) {
            for (int q = 0; q < cnt; q++) {
                R s, c, qi;
                if (sizeof(R) == 8) {
                    const double4 p = s_p[q];
                    const double a = p.x * kx + p.y * ky + p.z * kz;
                    double sd, cd;
                    sincos(a, &sd, &cd);
                    s = (R)sd; c = (R)cd;
                    qi = (R)tq[(int)p.w];
                } else {
                    const int4 f = s_f[q];
                    const int ph = (int)((unsigned)nx * (unsigned)f.x + (unsigned)ny * (unsigned)f.y +
                                         (unsigned)nz * (unsigned)f.z);
                    float sf, cf;
                    sincos_phase(ph, sf, cf);
                    s = sf; c = cf;
                    qi = (R)tq[f.w];
                }
                cs += (double)(qi * c);
                sn += (double)(qi * s);
            }
        }
    }
    if (k < nkv) {
        partial[(size_t)ch * 2 * nk + k] = cs;
        partial[(size_t)ch * 2 * nk + nk + k] = sn;
    }
}

// S(k) in fixed chunk order; energy and long virial per k.
__global__ void k_sk_reduce(int nk, const int *nkd, const double *partial, const double *kcoef, const double *kvec,
                            double alphaR4, double *sk, long long *acc) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int nkv = nkd ? *nkd : nk;
    if ((int)(blockIdx.x * blockDim.x) >= nkv) return;   // block-uniform
    double e = 0, vxx = 0, vxy = 0, vxz = 0, vyy = 0, vyz = 0, vzz = 0;
    if (k < nkv) {
        double cs = 0, sn = 0;
        for (int ch = 0; ch < RK_CHUNKS; ch++) {
            cs += partial[(size_t)ch * 2 * nk + k];
            sn += partial[(size_t)ch * 2 * nk + nk + k];
        }
        sk[k] = cs;
        sk[nk + k] = sn;
        const double kx = kvec[k], ky = kvec[nk + k], kz = kvec[2 * nk + k];
        const double k2 = kx * kx + ky * ky + kz * kz;
        e = kcoef[k] * (sn * sn + cs * cs);
        const double coeff = 2.0 * (alphaR4 + 1.0 / k2);
        vxx = e - e * coeff * kx * kx;
        vyy = e - e * coeff * ky * ky;
        vzz = e - e * coeff * kz * kz;
        vxy = -e * coeff * kx * ky;
        vxz = -e * coeff * kx * kz;
        vyz = -e * coeff * ky * kz;
    }
    __shared__ double s_r[7][8];
    double v[7] = {e, vxx, vxy, vxz, vyy, vyz, vzz};
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int q = 0; q < 7; q++) {
        double t = warp_sum(v[q]);
        if (lane == 0) s_r[q][w] = t;
    }
    __syncthreads();
    if (threadIdx.x < 7) {
        double t = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) t += s_r[threadIdx.x][q];
        const int slots[7][2] = {{ACC_E_LONG, -1},       {ACC_LVIR + 0, -1},
                                 {ACC_LVIR + 1, ACC_LVIR + 3}, {ACC_LVIR + 2, ACC_LVIR + 6},
                                 {ACC_LVIR + 4, -1},     {ACC_LVIR + 5, ACC_LVIR + 7},
                                 {ACC_LVIR + 8, -1}};
        long long fx = to_fix(t, ACC_SCALE);
        atomicAdd((unsigned long long *)&acc[slots[threadIdx.x][0]], (unsigned long long)fx);
        if (slots[threadIdx.x][1] >= 0)
            atomicAdd((unsigned long long *)&acc[slots[threadIdx.x][1]], (unsigned long long)fx);
    }
}

// Per-site reciprocal force; RF_TPS threads split the k set.
template <typename R>
__global__ void __launch_bounds__(256) k_recip_force(int n, int nk, const int *nkd, const double4 *pos4,
                                                     const int4 *fixq, const int *kn,
                                                     const double *kvec, const double *kcoef,
                                                     const double *sk, const double *tq, Box box,
                                                     const double *le, long long *frc) {
    __shared__ int s_n[3][256];
    // k vectors, prefactors and S(k) stay FP64; only the phase and its
    // sine/cosine follow R (the FP32 path's cost is in sincospif)
    __shared__ double s_k[3][256];
    __shared__ double s_b[256], s_c[256], s_s[256];
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gt / RF_TPS, t = gt % RF_TPS;
    double4 p64 = make_double4(0, 0, 0, 0);
    int4 pf = make_int4(0, 0, 0, 0);
    R qi = 0;
    if (i < n) {
        if (sizeof(R) == 8) { p64 = pos4[i]; qi = (R)tq[(int)p64.w]; }
        else {
            pf = fixq[i];
            if (le) pf.x = le_xfrac(pos4[i], le_reduced(le, box), box);
            qi = (R)tq[pf.w];
        }
    }
    const int nkv = nkd ? *nkd : nk;
    double fx = 0, fy = 0, fz = 0;
    for (int base = 0; base < nkv; base += 256) {
        __syncthreads();
        const int k = base + threadIdx.x;
        if (k < nkv) {
            s_n[0][threadIdx.x] = kn[k]; s_n[1][threadIdx.x] = kn[nk + k]; s_n[2][threadIdx.x] = kn[2 * nk + k];
            s_k[0][threadIdx.x] = kvec[k]; s_k[1][threadIdx.x] = kvec[nk + k];
            s_k[2][threadIdx.x] = kvec[2 * nk + k];
            s_b[threadIdx.x] = 2.0 * kcoef[k];
            s_c[threadIdx.x] = sk[k];
            s_s[threadIdx.x] = sk[nk + k];
        }
        __syncthreads();
        const int cnt = min(256, nkv - base);
        if (i < n) {
            double ax = 0, ay = 0, az = 0;
            for (int q = t; q < cnt; q += RF_TPS) {
                R s, c;
                if (sizeof(R) == 8) {
                    const double a = p64.x * s_k[0][q] + p64.y * s_k[1][q] + p64.z * s_k[2][q];
                    double sd, cd;
                    sincos(a, &sd, &cd);
                    s = (R)sd; c = (R)cd;
                } else {
                    const int ph = (int)((unsigned)s_n[0][q] * (unsigned)pf.x +
                                         (unsigned)s_n[1][q] * (unsigned)pf.y +
                                         (unsigned)s_n[2][q] * (unsigned)pf.z);
                    float sf, cf;
                    sincos_phase(ph, sf, cf);
                    s = sf; c = cf;
                }
                const double qs = (double)(qi * s), qc = (double)(qi * c);
                const double val = s_b[q] * (qs * s_c[q] - qc * s_s[q]);
                ax += s_k[0][q] * val;
                ay += s_k[1][q] * val;
                az += s_k[2][q] * val;
            }
            fx += ax; fy += ay; fz += az;
        }
    }
    fx = group_sum<RF_TPS>(fx);
    fy = group_sum<RF_TPS>(fy);
    fz = group_sum<RF_TPS>(fz);
    if (i < n && t == 0) {
        frc[i] += to_fix(fx, FRC_SCALE);
        frc[n + i] += to_fix(fy, FRC_SCALE);
        frc[2 * n + i] += to_fix(fz, FRC_SCALE);
    }
}

// sheared cell: capacity for every candidate of k_le_kset
static int setup_recip_le(Ctx &c) {
    const double PI = 3.14159265358979323846;
    const double kCut = c.ew_kcut;
    c.rc.le_nx = (int)(kCut * c.box.L[0] / (2 * PI));
    c.rc.le_ny = (int)(kCut * c.box.L[1] / (2 * PI)) + 1;
    c.rc.le_nz = (int)(kCut * c.box.L[2] / (2 * PI));
    const long long cap = (long long)(c.rc.le_nx + 1) * (2 * c.rc.le_ny + 1) * (2 * c.rc.le_nz + 1);
    if (cap > (1 << 26)) return SMD_ERR_ARG;
    const int nk = (int)cap;
    c.rc.nk = nk;
    c.rc.nmax = std::max(c.rc.le_nx + c.rc.le_ny, c.rc.le_nz);
    auto realloc = [](auto **p, size_t cnt) -> bool {
        if (*p) cudaFree(*p);
        *p = nullptr;
        return cudaMalloc((void **)p, (cnt ? cnt : 1) * sizeof(**p)) == cudaSuccess;
    };
    if (!realloc(&c.rc.kn, 3 * (size_t)nk) || !realloc(&c.rc.kvec, 3 * (size_t)nk) ||
        !realloc(&c.rc.kcoef, (size_t)nk) || !realloc(&c.rc.sk, 6 * (size_t)nk * RK_CHUNKS + 6 * (size_t)nk) ||
        !realloc(&c.rc.nk_dev, 1))
        return SMD_ERR_CUDA;
    if (cudaMemset(c.rc.nk_dev, 0, sizeof(int)) != cudaSuccess) return SMD_ERR_CUDA;
    c.rc.le = 1;
    c.graph_dirty = 1;
    return 0;
}

int setup_recip(Ctx &c) {
    const double PI = 3.14159265358979323846;
    if (!(c.ewald_on || c.mp_on) || c.box.L[0] <= 0) return 0;
    // SLLOD shear with the point-charge sum: the k list follows the offset
    if (c.ewald_on && !c.mp_on && c.integrator_ready && c.ip.strain_rate != 0.0) return setup_recip_le(c);
    c.rc.le = 0;
    const double kCut = c.ew_kcut, kCut2 = kCut * kCut;
    const double alpha2 = c.ew_alpha * c.ew_alpha, alphaR4 = 1.0 / (4.0 * alpha2);
    const int nxMax = (int)(kCut * c.box.L[0] / (2 * PI));
    const int nyMax = (int)(kCut * c.box.L[1] / (2 * PI));
    const int nzMax = (int)(kCut * c.box.L[2] / (2 * PI));
    const double vx = 2.0 * PI / c.box.L[0], vy = 2.0 * PI / c.box.L[1], vz = 2.0 * PI / c.box.L[2];
    std::vector<int> nxs, nys, nzs;
    std::vector<double> kxs, kys, kzs, coef;
    const double vol = c.box.L[0] * c.box.L[1] * c.box.L[2];
    const double pi4Volumer = 4.0 * PI * (1.0 / vol);
    for (int nx = 0; nx <= nxMax; nx++) {
        double kx = nx * vx;
        for (int ny = (nx == 0 ? 0 : -nyMax); ny <= nyMax; ny++) {
            double ky = ny * vy;
            for (int nz = ((nx == 0 && ny == 0) ? 1 : -nzMax); nz <= nzMax; nz++) {
                double kz = nz * vz;
                double k2 = kx * kx + ky * ky + kz * kz;
                if (k2 < kCut2) {
                    nxs.push_back(nx); nys.push_back(ny); nzs.push_back(nz);
                    kxs.push_back(kx); kys.push_back(ky); kzs.push_back(kz);
                    coef.push_back(pi4Volumer * (exp(-k2 * alphaR4) / k2));
                }
            }
        }
    }
    const int nk = (int)nxs.size();
    c.rc.nk = nk;
    c.rc.nmax = 0;
    for (int k = 0; k < nk; k++)
        c.rc.nmax = std::max(c.rc.nmax, std::max(std::abs(nxs[k]), std::max(std::abs(nys[k]), std::abs(nzs[k]))));
    std::vector<int> kn(3 * (size_t)nk);
    std::vector<double> kv(3 * (size_t)nk);
    for (int k = 0; k < nk; k++) {
        kn[k] = nxs[k]; kn[nk + k] = nys[k]; kn[2 * nk + k] = nzs[k];
        kv[k] = kxs[k]; kv[nk + k] = kys[k]; kv[2 * nk + k] = kzs[k];
    }
    auto realloc = [](auto **p, size_t cnt) -> bool {
        if (*p) cudaFree(*p);
        *p = nullptr;
        return cudaMalloc((void **)p, (cnt ? cnt : 1) * sizeof(**p)) == cudaSuccess;
    };
    if (!realloc(&c.rc.kn, 3 * (size_t)nk) || !realloc(&c.rc.kvec, 3 * (size_t)nk) ||
        !realloc(&c.rc.kcoef, (size_t)nk) || !realloc(&c.rc.sk, 6 * (size_t)nk * RK_CHUNKS + 6 * (size_t)nk))
        return SMD_ERR_CUDA;
    if (nk) {
        cudaMemcpy(c.rc.kn, kn.data(), kn.size() * sizeof(int), cudaMemcpyHostToDevice);
        cudaMemcpy(c.rc.kvec, kv.data(), kv.size() * sizeof(double), cudaMemcpyHostToDevice);
        cudaMemcpy(c.rc.kcoef, coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice);
    }
    c.graph_dirty = 1;
    return c.mp_on ? mp_recip_prepare(c) : 0;
}

// the live k count (the sheared cell's list is built on the device)
int recip_nk(Ctx &c, int *nk) {
    if (!c.rc.le) {
        *nk = c.rc.nk;
        return 0;
    }
    if (cudaStreamSynchronize(c.stream) != cudaSuccess) return SMD_ERR_CUDA;
    return cudaMemcpy(nk, c.rc.nk_dev, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : SMD_ERR_CUDA;
}

void launch_recip(Ctx &c) {
    const int nk = c.rc.nk;
    if (nk == 0) return;
    // rc.sk holds: [RK_CHUNKS][2][nk] partials, then S(k) as [2][nk]
    double *partial = (double *)c.rc.sk;
    double *sk = partial + (size_t)2 * nk * RK_CHUNKS;
    const double alphaR4 = 1.0 / (4.0 * c.ew_alpha * c.ew_alpha);
    // sheared cell: the offset is the integrator's (zero before it starts)
    const bool le = c.rc.le && c.integrator_ready && c.ip.strain_rate != 0.0;
    const double *led = le ? c.scal + SC_LE : nullptr;
    const int *nkd = c.rc.le ? c.rc.nk_dev : nullptr;
    if (c.rc.le) {
        const double vol = c.box.L[0] * c.box.L[1] * c.box.L[2];
        k_le_kset<<<1, KSET_THREADS, 0, c.stream>>>(c.rc.le_nx, c.rc.le_ny, c.rc.le_nz, c.box, led,
                                                    c.ew_kcut * c.ew_kcut, alphaR4,
                                                    4.0 * 3.14159265358979323846 * (1.0 / vol), nk, c.rc.kn,
                                                    c.rc.kvec, c.rc.kcoef, c.rc.nk_dev);
    }
    dim3 g1((nk + RK_THREADS - 1) / RK_THREADS, RK_CHUNKS);
    const bool mixed = c.precision == SMD_PREC_MIXED;
    if (mixed) {
        k_sk_partial<float><<<g1, RK_THREADS, 0, c.stream>>>(c.n, nk, nkd, c.pos4, c.fixq, c.rc.kn,
                                                             c.rc.kvec, c.type_q, c.box, led, partial);
    } else {
        k_sk_partial<double><<<g1, RK_THREADS, 0, c.stream>>>(c.n, nk, nkd, c.pos4, c.fixq, c.rc.kn,
                                                              c.rc.kvec, c.type_q, c.box, led, partial);
    }
    k_sk_reduce<<<(nk + 255) / 256, 256, 0, c.stream>>>(nk, nkd, partial, c.rc.kcoef, c.rc.kvec,
                                                        alphaR4, sk, c.acc);
    const int nb = (int)(((long long)c.n * RF_TPS + 255) / 256);
    if (mixed) {
        k_recip_force<float><<<nb, 256, 0, c.stream>>>(c.n, nk, nkd, c.pos4, c.fixq, c.rc.kn, c.rc.kvec,
                                                       c.rc.kcoef, sk, c.type_q, c.box, led, c.frc);
    } else {
        k_recip_force<double><<<nb, 256, 0, c.stream>>>(c.n, nk, nkd, c.pos4, c.fixq, c.rc.kn,
                                                        c.rc.kvec, c.rc.kcoef, sk, c.type_q, c.box, led, c.frc);
    }
}

}  // namespace smd
