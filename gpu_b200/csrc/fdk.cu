// fdk.cu -- FDK reconstruction and ellipsoid phantom utilities.
//
// FDK restates Reconstruction_FDK (V63/host_FDK.cpp:4-57):
//   1. cosine pre-weight, kernel_FDK_projection_adjust (V63/FDK/kernel_FDK.cu:1-14);
//   2. ramp filter.  The reference zero-pads each row to 2R, runs a cuFFT C2C,
//      multiplies by |k|*F_step*0.5 and inverts (V63/FDK/FFT_1d_GPU.h:241-287),
//      i.e. a linear convolution with h[n] = (1/2R) sum_k H[k] cos(pi k n / R),
//      |n| < R.  Here h is computed once in FP64 on the host and the rows are
//      convolved directly in a register-tiled Toeplitz kernel;
//   3. voxel-driven bilinear backprojection, kernel_FDK_reconstruction
//      (V63/FDK/kernel_FDK.cu:16-62), with a batch of views per launch held in
//      registers (each view's update is still applied with the reference's
//      float/double steps, so the sum is the reference's to the bit).
#include <cmath>
#include <vector>

#include "ctr_device.cuh"

namespace ctr {

__global__ void k_fdk_weight(const DevGeom g, const float* __restrict__ in, float* __restrict__ out)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y;
    const int w = blockIdx.z;
    if (u >= g.R) return;
    const long long p = ((long long)w * g.ZP + v) * g.R + u;
    const float x1 = g.dso;
    const float dd = fs(g.dso, g.dod);
    const float x2 = fdv(fm(fa(g.ymin, fm((float)u, g.du)), g.dso), dd);
    const float x3 = fdv(fm(fa(g.zmin, fm((float)v, g.dv)), g.dso), dd);
    out[p] = fdv(fm(in[p], g.dso), __fsqrt_rn(fa(fa(fm(x1, x1), fm(x2, x2)), fm(x3, x3))));
}

// Toeplitz row convolution out[r][j] = sum_m in[r][m] * h[j - m + R - 1].
// Block tile: 32 rows x 128 outputs; a thread owns 8 rows x 4 consecutive
// outputs and slides a 4-tap register window along m.
static constexpr int RP_COLS = 128, RP_ROWS = 32, RP_MC = 32, RP_TR = 8;
__global__ void __launch_bounds__(128)
k_ramp(const float* __restrict__ in, float* __restrict__ out, const float* __restrict__ h, int R, long long nrows)
{
    __shared__ float sg[RP_ROWS][RP_MC + 1];
    __shared__ float sh[RP_COLS + RP_MC + 4];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int j0 = blockIdx.x * RP_COLS;
    const long long r0 = (long long)blockIdx.y * RP_ROWS;
    const int jt = j0 + 4 * lane;          // first of this thread's 4 outputs
    float acc[RP_TR][4];
#pragma unroll
    for (int a = 0; a < RP_TR; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = 0.f;
    for (int m0 = 0; m0 < R; m0 += RP_MC) {
        __syncthreads();
        for (int t = threadIdx.x; t < RP_ROWS * RP_MC; t += 128) {
            const int rr = t / RP_MC, mm = t % RP_MC;
            const long long row = r0 + rr;
            sg[rr][mm] = (row < nrows && m0 + mm < R) ? in[row * R + m0 + mm] : 0.f;
        }
        // taps h[j - m + R - 1] for j in [j0, j0+128), m in [m0, m0+MC):
        // index e = j - m + R - 1 - (j0 - m0 - MC + 1 + R - 1) in [0, 128+MC-1)
        const int ebase = j0 - m0 - RP_MC + 1 + R - 1;
        for (int t = threadIdx.x; t < RP_COLS + RP_MC + 4; t += 128) {
            const int e = ebase + t;
            sh[t] = (e >= 0 && e < 2 * R - 1) ? h[e] : 0.f;
        }
        __syncthreads();
        // for output jt+b and m = m0+mm the tap is sh[jt + b - j0 - mm + MC - 1]
        const int hb = 4 * lane + RP_MC - 1;
        float w0 = sh[hb + 0], w1 = sh[hb + 1], w2 = sh[hb + 2], w3 = sh[hb + 3];
#pragma unroll 8
        for (int mm = 0; mm < RP_MC; ++mm) {
#pragma unroll
            for (int a = 0; a < RP_TR; ++a) {
                const float gv = sg[warp * RP_TR + a][mm];
                acc[a][0] = fmaf(gv, w0, acc[a][0]);
                acc[a][1] = fmaf(gv, w1, acc[a][1]);
                acc[a][2] = fmaf(gv, w2, acc[a][2]);
                acc[a][3] = fmaf(gv, w3, acc[a][3]);
            }
            // slide: next m needs taps one lower
            w3 = w2; w2 = w1; w1 = w0;
            w0 = sh[hb - mm - 1 >= 0 ? hb - mm - 1 : 0];
        }
    }
#pragma unroll
    for (int a = 0; a < RP_TR; ++a) {
        const long long row = r0 + warp * RP_TR + a;
        if (row >= nrows) continue;
#pragma unroll
        for (int b = 0; b < 4; ++b)
            if (jt + b < R) out[row * R + jt + b] = acc[a][b];
    }
}

static constexpr int FB_BX = 32, FB_BY = 4, FB_K = 4;

// floor(x) and (int)floor(x) for 0 <= x < 2^22 without conversion
// instructions (the backprojection is bound by the pipe that executes them):
// adding 1.5*2^23 rounds x to an integer m held in the low mantissa bits, and
// m - 1 when m > x.  Both results are exact, so they equal the reference's
// an = floor(ksi) and (float)an.
__device__ __forceinline__ float floor_small(float x, int& n)
{
    const float C = 12582912.0f;   // 1.5 * 2^23
    const float t = __fadd_rn(x, C);
    float r = __fsub_rn(t, C);
    n = __float_as_int(t) - 0x4B400000;
    if (r > x) {
        r = __fsub_rn(r, 1.0f);
        n -= 1;
    }
    return r;
}
__global__ void __launch_bounds__(FB_BX * FB_BY)
k_fdk_bp(const DevGeom g, float* __restrict__ vol, const float* __restrict__ proj, int view0, int nview)
{
    const int i = blockIdx.x * FB_BX + (threadIdx.x % FB_BX);
    const int j = blockIdx.y * FB_BY + (threadIdx.x / FB_BX);
    const int k0 = blockIdx.z * FB_K;
    if (i >= g.M || j >= g.N) return;
    const long long MN = (long long)g.M * g.N;
    const int R = g.R, ZP = g.ZP;
    const float DSO = g.dso, DOD = g.dod;
    // kernel_FDK.cu:86-88
    const float x = fa(fa(g.bx, fm(g.vx, 0.5f)), fm((float)i, g.vx));
    const float y = fa(fa(g.by, fm(g.vy, 0.5f)), fm((float)j, g.vy));
    float acc[FB_K], zc[FB_K];
#pragma unroll
    for (int kk = 0; kk < FB_K; ++kk) {
        const int k = min(k0 + kk, g.Z - 1);
        acc[kk] = vol[(long long)k * MN + (long long)j * g.M + i];
        zc[kk] = fa(fa(g.bz, fm(g.vz, 0.5f)), fm((float)k, g.vz));
    }
    for (int w = 0; w < nview; ++w) {
        const float2 scv = g.trig_fdk[view0 + w];
        const float sn = scv.x, cs = scv.y;
        const float t = fa(fm(x, cs), fm(y, sn));
        const float s = fa(fm(-x, sn), fm(y, cs));
        const float ds = fs(DSO, s);
        const float temp1 = fdv(fm(DSO, DSO), fm(ds, ds));
        float p = fdv(fm(DSO, t), ds);
        p = fdv(fs(fdv(fm(p, fs(DSO, DOD)), DSO), g.ymin), g.du);
        const float* __restrict__ pv = proj + (long long)w * R * ZP;
#pragma unroll
        for (int kk = 0; kk < FB_K; ++kk) {
            float ksi = fdv(fm(DSO, zc[kk]), ds);
            ksi = fdv(fs(fdv(fm(ksi, fs(DSO, DOD)), DSO), g.zmin), g.dv);
            float temp2;
            if ((0 <= ksi) && (fa(ksi, 1.0f) < (float)ZP) && (0 <= p) && (fa(p, 1.0f) < (float)R)) {
                int an, bn;
                const float an0 = fs(ksi, floor_small(ksi, an));   // ksi - an, an = floor(ksi)
                const float bn0 = fs(p, floor_small(p, bn));
                const float* q0 = pv + (long long)R * an + bn;
                const float* q1 = q0 + R;
                const float t00 = fm(fm(fs(1.0f, an0), fs(1.0f, bn0)), __ldg(q0));
                const float t01 = fm(fm(fs(1.0f, an0), bn0), __ldg(q0 + 1));
                const float t10 = fm(fm(an0, fs(1.0f, bn0)), __ldg(q1));
                const float t11 = fm(fm(an0, bn0), __ldg(q1 + 1));
                temp2 = fa(fa(fa(t00, t01), t10), t11);
            } else {
                temp2 = 0.0f;
            }
            // vol += temp1*temp2*(us_rate*PI/180.0f)*360.0/(us_rate*Nviews)  (float*float*float, then double)
            const float fprod = fm(fm(temp1, temp2), g.fdk_ang);
            if (g.fdk_full) {
                // a full circle (us_rate*Nviews == 360): (double)fprod*360.0 is exact
                // (24 + 6 significant bits) and dividing it by 360 gives fprod back; and
                // the FP64 sum of two floats rounded to float is their float sum (when
                // the FP64 sum is inexact the smaller term is below 2^-28 of the larger,
                // far under half a float ulp), so the update is one float add
                acc[kk] = fa(acc[kk], fprod);
            } else {
                const double dv = __ddiv_rn(__dmul_rn((double)fprod, 360.0), (double)g.fdk_usn);
                acc[kk] = (float)__dadd_rn((double)acc[kk], dv);
            }
        }
    }
#pragma unroll
    for (int kk = 0; kk < FB_K; ++kk) {
        const int k = k0 + kk;
        if (k < g.Z) vol[(long long)k * MN + (long long)j * g.M + i] = acc[kk];
    }
}

// h[n + R - 1], |n| < R, of the reference's padded-DFT ramp (FP64, as the oracle).
static void ramp_taps(const ctr_geometry_desc& d, std::vector<float>& taps)
{
    const int R = d.nu, P = 2 * R;
    const float DSO = d.dso, DOD = d.dod;
    const float F_max = (float)(1.0 / 2.0 / (double)(d.du * DSO / (DSO - DOD)));   // FFT_1d_GPU.h:246
    const float F_step = F_max / (float)(P / 2);
    std::vector<float> H(P);
    for (int i = 0; i < P; ++i) {
        const int k = (i >= P / 2) ? i - P : i;
        float hv = (float)std::abs(k) * F_step;
        hv *= 0.5f;
        H[i] = hv;
    }
    taps.assign(2 * R - 1, 0.f);
    for (int n = -(R - 1); n <= R - 1; ++n) {
        double acc = 0.0;
        const long long an = n < 0 ? -n : n;
        for (int i = 0; i < P; ++i) {
            const long long m = ((long long)i * an) % P;
            acc += (double)H[i] * std::cos(2.0 * M_PI * (double)m / (double)P);
        }
        taps[n + R - 1] = (float)(acc / (double)P);
    }
}

ctr_status launch_fdk(Geometry& G, const float* sino, float* vol, cudaStream_t st)
{
    const DevGeom& g = G.dg;
    const int nv = g.nviews;
    const long long P = G.npix();
    if (!G.d_ramp) {
        std::vector<float> taps;
        ramp_taps(G.desc, taps);
        CTR_CUDA_TRY(cudaMalloc(&G.d_ramp, taps.size() * sizeof(float)));
        CTR_CUDA_TRY(cudaMemcpy(G.d_ramp, taps.data(), taps.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    const size_t need = (size_t)P * nv * 2;
    if (G.fdk_cap < need) {
        if (G.d_fdk) cudaFree(G.d_fdk);
        G.d_fdk = nullptr;
        G.fdk_cap = 0;
        CTR_CUDA_TRY(cudaMalloc(&G.d_fdk, need * sizeof(float)));
        G.fdk_cap = need;
    }
    float* wsino = G.d_fdk;
    float* fsino = G.d_fdk + (size_t)P * nv;
    for (int v0 = 0; v0 < nv; v0 += 65535) {
        const int cnt = std::min(65535, nv - v0);
        k_fdk_weight<<<dim3((g.R + 127) / 128, g.ZP, cnt), 128, 0, st>>>(g, sino + (size_t)P * v0, wsino + (size_t)P * v0);
    }
    const long long nrows = (long long)nv * g.ZP;
    for (long long r0 = 0; r0 < nrows; r0 += 65535LL * RP_ROWS) {
        const long long cnt = std::min<long long>(65535LL * RP_ROWS, nrows - r0);
        dim3 grd((g.R + RP_COLS - 1) / RP_COLS, (unsigned)((cnt + RP_ROWS - 1) / RP_ROWS));
        k_ramp<<<grd, 128, 0, st>>>(wsino + r0 * g.R, fsino + r0 * g.R, G.d_ramp, g.R, cnt);
    }
    CTR_CUDA_TRY(cudaGetLastError());
    return launch_fdk_bp(G, fsino, 0, nv, vol, st);
}

// In-place exchange of x and y in every z slice of a square (nx == ny) volume.
__global__ void k_swap_xy(int n, int Z, float* __restrict__ vol)
{
    const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, k = blockIdx.z;
    if (i >= n || j >= n || i >= j) return;
    float* sl = vol + (long long)k * n * n;
    const float a = sl[(long long)j * n + i];
    sl[(long long)j * n + i] = sl[(long long)i * n + j];
    sl[(long long)i * n + j] = a;
}

ctr_status launch_swap_xy(const Geometry& G, float* vol, cudaStream_t st)
{
    const int n = G.desc.nx, Z = G.desc.nz;
    k_swap_xy<<<dim3((n + 31) / 32, (n + 7) / 8, Z), dim3(32, 8), 0, st>>>(n, Z, vol);
    CTR_CUDA_TRY(cudaGetLastError());
    return CTR_OK;
}

ctr_status launch_fdk_bp(const Geometry& G, const float* fsino, int view0, int nview, float* vol, cudaStream_t st)
{
    const DevGeom& g = G.dg;
    const long long P = G.npix();
    dim3 grd((g.M + FB_BX - 1) / FB_BX, (g.N + FB_BY - 1) / FB_BY, (g.Z + FB_K - 1) / FB_K);
    const int VB = 32;
    for (int w = 0; w < nview; w += VB)
        k_fdk_bp<<<grd, FB_BX * FB_BY, 0, st>>>(g, vol, fsino + (size_t)P * w, view0 + w, std::min(VB, nview - w));
    CTR_CUDA_TRY(cudaGetLastError());
    return CTR_OK;
}

// ---------------------------------------------------------------- phantoms
// Per ellipsoid: centre(3), rotation R (row major, 9), semi-axes(3), mu.
struct Ell { double c[3], R[9], ax[3], mu; };

__global__ void k_phantom(const DevGeom g, const Ell* __restrict__ e, int n, float* __restrict__ vol, double bx,
                          double by, double bz)
{
    const long long MN = (long long)g.M * g.N, V = MN * g.Z;
    for (long long q = blockIdx.x * 256LL + threadIdx.x; q < V; q += (long long)gridDim.x * 256) {
        const int i = (int)(q % g.M), j = (int)((q / g.M) % g.N), k = (int)(q / MN);
        const double p0 = __dadd_rn(bx, __dmul_rn((double)g.vx, (double)i + 0.5));
        const double p1 = __dadd_rn(by, __dmul_rn((double)g.vy, (double)j + 0.5));
        const double p2 = __dadd_rn(bz, __dmul_rn((double)g.vz, (double)k + 0.5));
        double acc = 0.0;
        for (int a = 0; a < n; ++a) {
            const Ell& E = e[a];
            const double d0 = __dsub_rn(p0, E.c[0]), d1 = __dsub_rn(p1, E.c[1]), d2 = __dsub_rn(p2, E.c[2]);
            double r2 = 0.0;
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const double l = __ddiv_rn(__dadd_rn(__dadd_rn(__dmul_rn(E.R[b], d0), __dmul_rn(E.R[3 + b], d1)),
                                                     __dmul_rn(E.R[6 + b], d2)),
                                           E.ax[b]);
                r2 = __dadd_rn(r2, __dmul_rn(l, l));
            }
            if (r2 <= 1.0) acc = __dadd_rn(acc, E.mu);
        }
        vol[q] = (float)__dadd_rn((double)vol[q], acc);
    }
}

static void euler_zxz(const double* e, double Rm[9])
{
    const double cp = std::cos(e[0]), sp = std::sin(e[0]), ct = std::cos(e[1]), st = std::sin(e[1]),
                 cs = std::cos(e[2]), ss = std::sin(e[2]);
    Rm[0] = cp * cs - sp * ct * ss; Rm[1] = -cp * ss - sp * ct * cs; Rm[2] = sp * st;
    Rm[3] = sp * cs + cp * ct * ss; Rm[4] = -sp * ss + cp * ct * cs; Rm[5] = -cp * st;
    Rm[6] = st * ss;                Rm[7] = st * cs;                 Rm[8] = ct;
}

ctr_status launch_phantom(const Geometry& G, const double* params, int n, float* vol, cudaStream_t st)
{
    std::vector<Ell> h(n);
    for (int a = 0; a < n; ++a) {
        const double* q = params + 10 * a;
        for (int b = 0; b < 3; ++b) { h[a].c[b] = q[b]; h[a].ax[b] = q[3 + b]; }
        euler_zxz(q + 6, h[a].R);
        h[a].mu = q[9];
    }
    Ell* d = nullptr;
    CTR_CUDA_TRY(cudaMalloc(&d, sizeof(Ell) * (n > 0 ? n : 1)));
    cudaError_t e = cudaMemcpyAsync(d, h.data(), sizeof(Ell) * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        const ctr_geometry_desc& D = G.desc;
        const double bx = -(double)D.vx * ((double)D.nx / 2.0 + (double)D.m_offset);
        const double by = -(double)D.vy * ((double)D.ny / 2.0);
        const double bz = -(double)D.vz * ((double)D.nz / 2.0);
        k_phantom<<<148 * 16, 256, 0, st>>>(G.dg, d, n, vol, bx, by, bz);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d);
    CTR_CUDA_TRY(e);
    return CTR_OK;
}

}  // namespace ctr
