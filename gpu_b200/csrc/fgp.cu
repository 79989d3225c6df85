// fgp.cu -- FGP total-variation prox, FISTA momentum, objective reductions.
//
// FGP restates FGP_denoise_GPUx7_exact (V63/host_FGP_Denoise_GPUx7.c:1-111)
// and its kernels FGP_operator_L_Pc / FGP_operator_LT_Pp
// (V63/kernel_FGP_Denoise_GPUx7.cu:2-88) with the same float operations.  The
// duals are stored in the volume's storage type; L stays FP32.
//
// Dual layout: volume-sized arrays; r[p] belongs to the edge (x, x+1) and is 0
// at x = nx-1 (the reference's zero-padded d_r[x+1], V63/host_FGP_Denoise_
// GPUx7.c:8-38); likewise s along y and t along z.
#include "ctr_device.cuh"

namespace ctr {

static constexpr int FG_BX = 32, FG_BY = 8;

// f may be stored in another type than the duals (the refinement solver's
// FP32 sum y_k + d against 16-bit duals).
template <typename T, typename TF = T>
__device__ __forceinline__ float fgp_L(const TF* __restrict__ f, const T* __restrict__ r, const T* __restrict__ s,
                                       const T* __restrict__ t, int x, int y, int z, long long p, int M, long long MN,
                                       float lambda)
{
    const float rv = Store<T>::ld(r + p), rm = x > 0 ? Store<T>::ld(r + p - 1) : 0.0f;
    const float sv = Store<T>::ld(s + p), sm = y > 0 ? Store<T>::ld(s + p - M) : 0.0f;
    const float tv = Store<T>::ld(t + p), tm = z > 0 ? Store<T>::ld(t + p - MN) : 0.0f;
    const float tl = fa(fa(fs(rv, rm), fs(sv, sm)), fs(tv, tm));       // L_Pc :14
    return fs(Store<TF>::ld(f + p), fm(lambda, tl));                   // :17
}

// One inner iteration in two passes, as the reference's x7 form: k_fgp_L
// writes L = f - lambda*div(r,s,t) (FP32, as the reference keeps it) for every
// voxel; k_fgp_dual reads L at the voxel and its +x, +y, +z neighbours and
// updates the voxel's own duals in place (no voxel reads another's duals in
// this pass, so no double buffer is needed).  One thread per voxel, a 3-D
// grid of 32x8 tiles: both passes stream at close to the copy bandwidth.
template <typename T, typename TF = T>
__global__ void __launch_bounds__(FG_BX * FG_BY)
k_fgp_L(int M, int N, int Z, const TF* __restrict__ f, const T* __restrict__ r, const T* __restrict__ s,
        const T* __restrict__ t, float* __restrict__ L, float lambda)
{
    const int x = blockIdx.x * FG_BX + threadIdx.x;
    const int y = blockIdx.y * FG_BY + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= M || y >= N) return;
    const long long MN = (long long)M * N;
    const long long p = (long long)z * MN + (long long)y * M + x;
    L[p] = fgp_L<T, TF>(f, r, s, t, x, y, z, p, M, MN, lambda);          // L_Pc, GPUx7.cu:2-24
}

template <typename T>
__global__ void __launch_bounds__(FG_BX * FG_BY)
k_fgp_dual(int M, int N, int Z, const float* __restrict__ L, T* __restrict__ r, T* __restrict__ s,
           T* __restrict__ t, T* __restrict__ o, T* __restrict__ pd, T* __restrict__ q, float alpha12, float gam)
{
    const int x = blockIdx.x * FG_BX + threadIdx.x;
    const int y = blockIdx.y * FG_BY + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= M || y >= N) return;
    const long long MN = (long long)M * N;
    const long long p = (long long)z * MN + (long long)y * M + x;
    const float Lc = __ldg(L + p);
    const float Lx = (x < M - 1) ? __ldg(L + p + 1) : 0.0f;
    const float Ly = (y < N - 1) ? __ldg(L + p + M) : 0.0f;
    const float Lz = (z < Z - 1) ? __ldg(L + p + MN) : 0.0f;
    // LT_Pp (V63/kernel_FGP_Denoise_GPUx7.cu:52-86)
    float tr = Store<T>::ldw(r + p), ts = Store<T>::ldw(s + p), tt = Store<T>::ldw(t + p);
    if (x < M - 1) tr = fa(tr, fm(alpha12, fs(Lc, Lx)));
    if (y < N - 1) ts = fa(ts, fm(alpha12, fs(Lc, Ly)));
    if (z < Z - 1) tt = fa(tt, fm(alpha12, fs(Lc, Lz)));
    const float rst = __fsqrt_rn(fa(fa(fm(tr, tr), fm(ts, ts)), fm(tt, tt)));
    const float den = fmaxf(1.0f, rst);
    if (x < M - 1) {
        const float on = fdv(tr, den);
        Store<T>::st(r + p, fa(on, fm(gam, fs(on, Store<T>::ldw(o + p)))));
        Store<T>::st(o + p, on);
    }
    if (y < N - 1) {
        const float pn = fdv(ts, den);
        Store<T>::st(s + p, fa(pn, fm(gam, fs(pn, Store<T>::ldw(pd + p)))));
        Store<T>::st(pd + p, pn);
    }
    if (z < Z - 1) {
        const float qn = fdv(tt, den);
        Store<T>::st(t + p, fa(qn, fm(gam, fs(qn, Store<T>::ldw(q + p)))));
        Store<T>::st(q + p, qn);
    }
}

// x* = f - lambda*div(o,p,q) (the final L_Pc, V63/host_FGP_Denoise_GPUx7.c:83);
// with FISTA fused: y = x* + gam*(x* - xprev), xprev = x* (V63/main_recon.cu:375-382).
template <typename T, bool FISTA>
__global__ void __launch_bounds__(256)
k_fgp_final(int M, int N, int Z, T* __restrict__ vol, const T* __restrict__ o, const T* __restrict__ pd,
            const T* __restrict__ q, float lambda, T* __restrict__ xprev, float gam, const float* __restrict__ gam_dev)
{
    if (FISTA && gam_dev) gam = *gam_dev;
    const long long MN = (long long)M * N;
    const long long n = MN * Z;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(p % M);
        const int y = (int)((p / M) % N);
        const int z = (int)(p / MN);
        const float xs = fgp_L<T>(vol, o, pd, q, x, y, z, p, M, MN, lambda);
        if (FISTA) {
            const float xp = Store<T>::ldw(xprev + p);
            // the stored x_k is what the momentum step sees
            T xs_t;
            Store<T>::st(&xs_t, xs);
            const float xk = Store<T>::ldw(&xs_t);
            Store<T>::st(vol + p, fa(xk, fm(gam, fs(xk, xp))));
            xprev[p] = xs_t;
        } else {
            Store<T>::st(vol + p, xs);
        }
    }
}

// Refinement solver: the FP32 input of the prox, y_k + d = (1+g) x_k - g x_(k-1) + d,
// written over x_(k-1) (which is not needed after it).  d is read in the
// projectors' tiled layout.
// Refinement solver: the start d0 of the correction volume, the storage
// rounding of y_k - y~_k = (1+g)(x_k - x~_k) - g (x_(k-1) - x~_(k-1)), where
// x~ are the projectors' round-to-nearest copies of the FP32 iterates (the
// pass projects y~_k through the copy of x_k and A x~_(k-1)).  With d
// starting there, A (y~_k + d) is the projection of the FP32 y_k up to the
// rounding of that small difference, so the copies' rounding does not bias
// the fixed point.  T: the copies' type; TD: the correction's (T, or FP32).
// Zero for FP32 copies.
template <typename T, typename TD>
__device__ __forceinline__ float refine_d0(float xk, float xm, float gm)
{
    const float e = fs(fm(fa(1.0f, gm), fs(xk, Store<T>::rn(xk))), fm(gm, fs(xm, Store<T>::rn(xm))));
    return Store<TD>::rn(e);
}

// d = d0 in the tiled layout, one thread per tiled element (padding zero).
template <typename T, typename TD>
__global__ void __launch_bounds__(256)
k_refine_start(const DevGeom g, const float* __restrict__ xk, const float* __restrict__ xm,
               const float* __restrict__ gdev, TD* __restrict__ d)
{
    const float gm = *gdev;
    const long long n = tiled_count(g);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int w = (int)(t & 63);
        const long long tile = t >> 6;
        const int tx = (int)(tile % g.Mt);
        const long long r = tile / g.Mt;
        const int ty = (int)(r % g.Nt);
        const int k = (int)(r / g.Nt);
        const int i = tx * 8 + (w & 7), j = ty * 8 + (w >> 3);
        float v = 0.0f;
        if (i < g.M && j < g.N) {
            const long long p = ((long long)k * g.N + j) * g.M + i;
            v = refine_d0<T, TD>(xk[p], xm[p], gm);
        }
        Store<TD>::st(d + t, v);
    }
}

// z = y_k + (d - d0) in FP32 into xm (FGP's input).
template <typename T, typename TD>
__global__ void __launch_bounds__(256)
k_refine_sum(const DevGeom g, const float* __restrict__ xk, float* __restrict__ xm, const TD* __restrict__ d,
             const float* __restrict__ gdev)
{
    const float gm = *gdev;
    const long long MN = (long long)g.M * g.N, n = MN * g.Z;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(p % g.M), y = (int)((p / g.M) % g.N), z = (int)(p / MN);
        const float xkv = xk[p], xmv = xm[p];
        const float yk = fs(fm(fa(1.0f, gm), xkv), fm(gm, xmv));
        xm[p] = fa(yk, fs(Store<TD>::ld(d + tile_index(g, x, y, z)), refine_d0<T, TD>(xkv, xmv, gm)));
    }
}

// Refinement solver: x* = the prox f - lambda*div(o,p,q) of f = xm (FGP), or
// f itself; then the rotation x_(k-1) = x_k, x_k = x*, and the projectors'
// 16-bit copy of x* in the tiled layout (round to nearest).
template <typename T, bool FGP>
__global__ void __launch_bounds__(256)
k_refine_final(const DevGeom g, float* __restrict__ xk, float* __restrict__ xm, const T* __restrict__ o,
               const T* __restrict__ pd, const T* __restrict__ q, float lambda, T* __restrict__ xt)
{
    const int M = g.M;
    const long long MN = (long long)g.M * g.N, n = MN * g.Z;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(p % M), y = (int)((p / M) % g.N), z = (int)(p / MN);
        const float xs = FGP ? fgp_L<T, float>(xm, o, pd, q, x, y, z, p, M, MN, lambda) : xm[p];
        xm[p] = xk[p];
        xk[p] = xs;
        Store<T>::st(xt + tile_index(g, x, y, z), xs);
    }
}

__global__ void k_set_scalar(float* p, float v) { *p = v; }

template <typename T>
__global__ void __launch_bounds__(256)
k_momentum(long long n, T* __restrict__ y, T* __restrict__ xprev, const T* __restrict__ x, float gam,
           const float* __restrict__ gam_dev)
{
    if (gam_dev) gam = *gam_dev;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const float xv = Store<T>::ldw(x + p);
        const float xp = Store<T>::ldw(xprev + p);
        Store<T>::st(y + p, fa(xv, fm(gam, fs(xv, xp))));        // main_recon.cu:378
        Store<T>::st(xprev + p, xv);                              // :380
    }
}

static int grid_for(long long n, int threads)
{
    long long b = (n + threads - 1) / threads;
    if (b > 148LL * 64) b = 148LL * 64;
    return (int)(b < 1 ? 1 : b);
}

// t_k = (1 + sqrt(1 + 4 t^2))/2 in float (V63/host_FGP_Denoise_GPUx7.c:161)
static float next_t(float t) { return (1.0f + sqrtf(1.0f + 4.0f * t * t)) / 2.0f; }

ctr_status launch_fgp(Geometry& G, void* vol, ctr_dtype dt, float lambda, int iters, void* fista_y,
                      void* fista_xprev, float fista_gamma, cudaStream_t st, const float* gamma_dev)
{
    const int M = G.desc.nx, N = G.desc.ny, Z = G.desc.nz;
    const long long V = G.nvox();
    const size_t es = dtype_size(dt);
    CTR_TRY(ensure_fgp(&G, fgp_workspace_bytes(V, dt)));
    CTR_CUDA_TRY(cudaMemsetAsync(G.d_fgp, 0, 6 * (size_t)V * es, st));
    const float alpha12 = 1.0f / (lambda * 12.0f);                 // :166
    const dim3 blk(FG_BX, FG_BY), grd((M + FG_BX - 1) / FG_BX, (N + FG_BY - 1) / FG_BY, Z);
    CTR_DISPATCH_DTYPE(dt, T, {
        T* base = (T*)G.d_fgp;
        T* D[6] = {base, base + V, base + 2 * V, base + 3 * V, base + 4 * V, base + 5 * V};   // r s t o p q
        float* L = (float*)((char*)G.d_fgp + 6 * (size_t)V * es);
        float t_k_1 = 1.0f;
        for (int it = 0; it < iters; ++it) {
            const float t_k = next_t(t_k_1);
            const float gam = (t_k_1 - 1.0f) / t_k;
            k_fgp_L<T><<<grd, blk, 0, st>>>(M, N, Z, (const T*)vol, D[0], D[1], D[2], L, lambda);
            k_fgp_dual<T><<<grd, blk, 0, st>>>(M, N, Z, L, D[0], D[1], D[2], D[3], D[4], D[5], alpha12, gam);
            t_k_1 = t_k;
        }
        if (fista_y) {
            if (fista_y != vol) return set_error(CTR_ERR_INVALID_ARGUMENT, "fused FISTA output must alias the volume");
            k_fgp_final<T, true><<<grid_for(V, 256), 256, 0, st>>>(M, N, Z, (T*)vol, D[3], D[4], D[5], lambda,
                                                                    (T*)fista_xprev, fista_gamma, gamma_dev);
        } else {
            k_fgp_final<T, false><<<grid_for(V, 256), 256, 0, st>>>(M, N, Z, (T*)vol, D[3], D[4], D[5], lambda,
                                                                     nullptr, 0.0f, nullptr);
        }
    });
    CTR_CUDA_TRY(cudaGetLastError());
    return CTR_OK;
}

ctr_status launch_momentum(const Geometry& G, void* y, void* xprev, const void* x, ctr_dtype dt, float gam,
                           cudaStream_t st, const float* gamma_dev)
{
    const long long V = G.nvox();
    CTR_DISPATCH_DTYPE(dt, T, {
        k_momentum<T><<<grid_for(V, 256), 256, 0, st>>>(V, (T*)y, (T*)xprev, (const T*)x, gam, gamma_dev);
    });
    CTR_CUDA_TRY(cudaGetLastError());
    return CTR_OK;
}

ctr_status launch_refine_update(Geometry& G, float* xk, float* xm, const void* d_tiled, ctr_dtype ddt, void* xt_tiled,
                                ctr_dtype dt, float lam, int iters, const float* gdev, cudaStream_t st)
{
    const int M = G.desc.nx, N = G.desc.ny, Z = G.desc.nz;
    const long long V = G.nvox();
    const size_t es = dtype_size(dt);
    const bool fgp = lam > 0.f && iters >= 0;
    if (ddt != dt && ddt != CTR_F32) return set_error(CTR_ERR_INVALID_ARGUMENT, "correction type");
    if (fgp) CTR_TRY(ensure_fgp(&G, fgp_workspace_bytes(V, dt)));
    const int nb = grid_for(V, 256);
    CTR_DISPATCH_DTYPE(dt, T, {
        if (ddt == CTR_F32) k_refine_sum<T, float><<<nb, 256, 0, st>>>(G.dg, xk, xm, (const float*)d_tiled, gdev);
        else k_refine_sum<T, T><<<nb, 256, 0, st>>>(G.dg, xk, xm, (const T*)d_tiled, gdev);
        if (fgp) {
            CTR_CUDA_TRY(cudaMemsetAsync(G.d_fgp, 0, 6 * (size_t)V * es, st));
            const float alpha12 = 1.0f / (lam * 12.0f);
            const dim3 blk(FG_BX, FG_BY), grd((M + FG_BX - 1) / FG_BX, (N + FG_BY - 1) / FG_BY, Z);
            T* base = (T*)G.d_fgp;
            T* D[6] = {base, base + V, base + 2 * V, base + 3 * V, base + 4 * V, base + 5 * V};   // r s t o p q
            float* L = (float*)((char*)G.d_fgp + 6 * (size_t)V * es);
            float t_k_1 = 1.0f;
            for (int it = 0; it < iters; ++it) {
                const float t_k = next_t(t_k_1);
                const float gam = (t_k_1 - 1.0f) / t_k;
                k_fgp_L<T, float><<<grd, blk, 0, st>>>(M, N, Z, xm, D[0], D[1], D[2], L, lam);
                k_fgp_dual<T><<<grd, blk, 0, st>>>(M, N, Z, L, D[0], D[1], D[2], D[3], D[4], D[5], alpha12, gam);
                t_k_1 = t_k;
            }
            k_refine_final<T, true><<<nb, 256, 0, st>>>(G.dg, xk, xm, D[3], D[4], D[5], lam, (T*)xt_tiled);
        } else {
            k_refine_final<T, false><<<nb, 256, 0, st>>>(G.dg, xk, xm, nullptr, nullptr, nullptr, 0.f, (T*)xt_tiled);
        }
    });
    CTR_CUDA_TRY(cudaGetLastError());
    return CTR_OK;
}

ctr_status launch_refine_start(Geometry& G, const float* xk, const float* xm, void* d_tiled, ctr_dtype ddt,
                               ctr_dtype dt, const float* gdev, cudaStream_t st)
{
    if (ddt != dt && ddt != CTR_F32) return set_error(CTR_ERR_INVALID_ARGUMENT, "correction type");
    const int nb = grid_for(tiled_count(G.dg), 256);
    CTR_DISPATCH_DTYPE(dt, T, {
        if (ddt == CTR_F32) k_refine_start<T, float><<<nb, 256, 0, st>>>(G.dg, xk, xm, gdev, (float*)d_tiled);
        else k_refine_start<T, T><<<nb, 256, 0, st>>>(G.dg, xk, xm, gdev, (T*)d_tiled);
    });
    CTR_CUDA_TRY(cudaGetLastError());
    return CTR_OK;
}

ctr_status launch_set_scalar(float* p, float v, cudaStream_t st)
{
    k_set_scalar<<<1, 1, 0, st>>>(p, v);
    CTR_CUDA_TRY(cudaGetLastError());
    return CTR_OK;
}

// ---------------------------------------------------------------- reductions

// Sum of part[0..n) in a fixed order: block b sums the contiguous segment
// [b*seg, (b+1)*seg) into out[b].  Repeated runs give identical bits.
__global__ void __launch_bounds__(1024) k_reduce(const double* __restrict__ part, long long n, long long seg,
                                                 double* __restrict__ out)
{
    __shared__ double sh[32];
    const long long lo = blockIdx.x * seg, hi = min(n, lo + seg);
    double v = 0.0;
    for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) v += part[i];
    const double t = block_sum(v, sh);
    if (threadIdx.x == 0) out[blockIdx.x] = t;
}

// Needs 1024 doubles of scratch after part[n].
ctr_status launch_reduce(const double* partial, size_t n, double* out, cudaStream_t st)
{
    if (n > 16384) {
        double* mid = const_cast<double*>(partial) + n;
        const long long seg = ((long long)n + 1023) / 1024;
        k_reduce<<<1024, 1024, 0, st>>>(partial, (long long)n, seg, mid);
        k_reduce<<<1, 1024, 0, st>>>(mid, 1024, 1024, out);
    } else {
        k_reduce<<<1, 1024, 0, st>>>(partial, (long long)n, (long long)n, out);
    }
    CTR_CUDA_TRY(cudaGetLastError());
    return CTR_OK;
}

template <int OP>   // 0: a*b, 1: (a-b)^2 in float
__global__ void __launch_bounds__(256)
k_pairsum(const float* __restrict__ a, const float* __restrict__ b, long long n, double* __restrict__ part)
{
    __shared__ double sh[8];
    double v = 0.0;
    for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) {
        if (OP == 0) v += (double)a[i] * (double)b[i];
        else {
            const float e = fs(a[i], b[i]);
            v += (double)fm(e, e);
        }
    }
    const double t = block_sum(v, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

ctr_status launch_dot(const float* a, const float* b, long long n, double* partial, size_t cap, double* out,
                      cudaStream_t st)
{
    int nb = grid_for(n, 256);
    if ((size_t)nb > cap) nb = (int)cap;
    k_pairsum<0><<<nb, 256, 0, st>>>(a, b, n, partial);
    CTR_CUDA_TRY(cudaGetLastError());
    return launch_reduce(partial, nb, out, st);
}

ctr_status launch_l2(const float* a, const float* b, long long n, double* partial, size_t cap, double* out,
                     cudaStream_t st)
{
    int nb = grid_for(n, 256);
    if ((size_t)nb > cap) nb = (int)cap;
    k_pairsum<1><<<nb, 256, 0, st>>>(a, b, n, partial);
    CTR_CUDA_TRY(cudaGetLastError());
    return launch_reduce(partial, nb, out, st);
}

// TV_norm_kernel (V63/kernel_tool_functions.cu:39-65) with an FP64 block sum.
template <typename T>
__global__ void __launch_bounds__(256)
k_tv(int M, int N, int Z, const T* __restrict__ d, double* __restrict__ part)
{
    __shared__ double sh[8];
    const long long MN = (long long)M * N, n = MN * Z;
    double acc = 0.0;
    for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) {
        const int x = (int)(i % M), y = (int)((i / M) % N), z = (int)(i / MN);
        const float c = Store<T>::ld(d + i);
        const float dj = x < M - 1 ? fs(c, Store<T>::ld(d + i + 1)) : 0.f;
        const float dk = y < N - 1 ? fs(c, Store<T>::ld(d + i + M)) : 0.f;
        const float dl = z < Z - 1 ? fs(c, Store<T>::ld(d + i + MN)) : 0.f;
        float tv = 0.0f;
        const bool bx = x < M - 1, by = y < N - 1, bz = z < Z - 1;
        if (bx && by && bz) tv = __fsqrt_rn(fa(fa(fm(dj, dj), fm(dk, dk)), fm(dl, dl)));
        else if (!bx && by && bz) tv = __fsqrt_rn(fa(fm(dk, dk), fm(dl, dl)));
        else if (bx && !by && bz) tv = __fsqrt_rn(fa(fm(dj, dj), fm(dl, dl)));
        else if (bx && by && !bz) tv = __fsqrt_rn(fa(fm(dj, dj), fm(dk, dk)));
        else if (!bx && !by && bz) tv = fabsf(dl);
        else if (!bx && by && !bz) tv = fabsf(dk);
        else if (bx && !by && !bz) tv = fabsf(dj);
        acc += (double)tv;
    }
    const double t = block_sum(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

ctr_status launch_tv(const Geometry& G, const void* vol, ctr_dtype dt, double* partial, size_t cap, double* out,
                     cudaStream_t st)
{
    const long long V = G.nvox();
    int nb = grid_for(V, 256);
    if ((size_t)nb > cap) nb = (int)cap;
    CTR_DISPATCH_DTYPE(dt, T, { k_tv<T><<<nb, 256, 0, st>>>(G.desc.nx, G.desc.ny, G.desc.nz, (const T*)vol, partial); });
    CTR_CUDA_TRY(cudaGetLastError());
    return launch_reduce(partial, nb, out, st);
}

template <typename S, typename D>
__global__ void k_convert(const S* __restrict__ s, D* __restrict__ d, long long n)
{
    for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256)
        Store<D>::st(d + i, Store<S>::ld(s + i));
}

ctr_status launch_convert(const void* src, ctr_dtype sdt, void* dst, ctr_dtype ddt, long long n, cudaStream_t st)
{
    const int nb = grid_for(n, 256);
    CTR_DISPATCH_DTYPE(sdt, S, {
        CTR_DISPATCH_DTYPE(ddt, D, { k_convert<S, D><<<nb, 256, 0, st>>>((const S*)src, (D*)dst, n); });
    });
    CTR_CUDA_TRY(cudaGetLastError());
    return CTR_OK;
}

}  // namespace ctr
