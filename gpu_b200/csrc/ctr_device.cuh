// ctr_device.cuh -- device helpers shared by the kernels.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "ctr_internal.h"

namespace ctr {

// IEEE single-precision operations that the compiler never contracts into FMA.
// The geometric expressions of the projectors use these so that every alpha,
// plane index and chord length is bit-identical to the reference arithmetic.
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fdv(float a, float b) { return __fdiv_rn(a, b); }

// storage <-> FP32
template <typename T> struct Store;
// ld: the read-only path (data no thread of the launch writes); ldc: a
// coherent load (ld.global.ca) for data that other blocks of the same launch
// wrote before an acquire (the batch's persistent pass).
template <> struct Store<float> {
    static __device__ __forceinline__ float ld(const float* p) { return __ldg(p); }
    static __device__ __forceinline__ float ldc(const float* p) { return __ldca(p); }
    static __device__ __forceinline__ float ldw(const float* p) { return *p; }
    static __device__ __forceinline__ void st(float* p, float v) { *p = v; }
    static __device__ __forceinline__ float rn(float v) { return v; }
};
template <> struct Store<__nv_bfloat16> {
    static __device__ __forceinline__ float ld(const __nv_bfloat16* p) { return __bfloat162float(__ldg(p)); }
    static __device__ __forceinline__ float ldc(const __nv_bfloat16* p) { return __bfloat162float(__ldca(p)); }
    static __device__ __forceinline__ float ldw(const __nv_bfloat16* p) { return __bfloat162float(*p); }
    static __device__ __forceinline__ void st(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
    static __device__ __forceinline__ float rn(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }
};
template <> struct Store<__half> {
    static __device__ __forceinline__ float ld(const __half* p) { return __half2float(__ldg(p)); }
    static __device__ __forceinline__ float ldc(const __half* p) { return __half2float(__ldca(p)); }
    static __device__ __forceinline__ float ldw(const __half* p) { return __half2float(*p); }
    static __device__ __forceinline__ void st(__half* p, float v) { *p = __float2half_rn(v); }
    static __device__ __forceinline__ float rn(float v) { return __half2float(__float2half_rn(v)); }
};

// Stochastic rounding of an FP32 value to the storage type: add uniform random
// bits below the kept mantissa, then truncate.  The expected stored value
// equals the FP32 value, so SART increments below half an ulp are not lost on
// average.
__device__ __forceinline__ uint32_t hash32(uint32_t x)
{
    x ^= x >> 16; x *= 0x7feb352dU; x ^= x >> 15; x *= 0x846ca68bU; x ^= x >> 16;
    return x;
}
template <typename T> __device__ __forceinline__ void st_sr(T* p, float v, uint32_t rnd);
template <> __device__ __forceinline__ void st_sr<float>(float* p, float v, uint32_t) { *p = v; }
template <> __device__ __forceinline__ void st_sr<__nv_bfloat16>(__nv_bfloat16* p, float v, uint32_t rnd)
{
    uint32_t b = __float_as_uint(v);
    if ((b & 0x7f800000u) != 0x7f800000u) b += (rnd & 0xffffu);   // finite only
    *p = __ushort_as_bfloat16((unsigned short)(b >> 16));
}
template <> __device__ __forceinline__ void st_sr<__half>(__half* p, float v, uint32_t rnd)
{
    // FP16 keeps 10 mantissa bits; dither by a uniform fraction of one FP16 ulp
    // of |v| and round toward zero.
    const float av = fabsf(v);
    if (!(av < 65504.f) || av < 6.103515625e-05f) { *p = __float2half_rn(v); return; }
    int ex;
    frexpf(av, &ex);                                   // av in [2^(ex-1), 2^ex)
    const float ulp = ldexpf(1.0f, ex - 11);
    const float d = ulp * ((float)(rnd & 0xffffffu) * (1.0f / 16777216.0f));
    *p = __float2half_rz(v >= 0.f ? v + d : v - d);
}

template <typename T> struct DT;
template <> struct DT<float> { static constexpr ctr_dtype v = CTR_F32; };
template <> struct DT<__nv_bfloat16> { static constexpr ctr_dtype v = CTR_BF16; };
template <> struct DT<__half> { static constexpr ctr_dtype v = CTR_F16; };

__device__ __forceinline__ float ld_any(const void* p, long long i, int dt)
{
    if (dt == CTR_F32) return __ldg((const float*)p + i);
    if (dt == CTR_BF16) return __bfloat162float(__ldg((const __nv_bfloat16*)p + i));
    return __half2float(__ldg((const __half*)p + i));
}
__device__ __forceinline__ void st_any(void* p, long long i, int dt, float v)
{
    if (dt == CTR_F32) ((float*)p)[i] = v;
    else if (dt == CTR_BF16) ((__nv_bfloat16*)p)[i] = __float2bfloat16_rn(v);
    else ((__half*)p)[i] = __float2half_rn(v);
}

// Block-wide FP64 sum (blockDim.x a multiple of 32, at most 1024); result in
// thread 0.  Fixed order, so repeated runs are bit-identical.
__device__ __forceinline__ double block_sum(double v, double* sh)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r += sh[i];
    return r;
}

// Index of voxel (i, j, k) in the 8x8-tiled layout.
__device__ __forceinline__ int tile_index(const DevGeom& g, int i, int j, int k)
{
    return (((k * g.Nt) + (j >> 3)) * g.Mt + (i >> 3)) * 64 + ((j & 7) << 3) + (i & 7);
}

// Source X2 and detector pixel centre X1 of the ray through pixel (u, v) at
// view angle (s, c) (V63/kernel_IterativeRecon_universal.cu:21-45): one source
// (cone beam), the source at the row's height (multi-slice fan beam), or a
// source opposite each pixel (parallel beam); the tetrahedron beam's row v is
// row v % nvr of source v / nvr's band (T42/...TBCT_voxel.cu:23-40).
struct RayEnds {
    float x1x, x1y, x1z, x2x, x2y, x2z;
};
__device__ __forceinline__ RayEnds ray_ends(const DevGeom& g, float s, float c, int u, int v)
{
    RayEnds e;
    const float pu = fa(g.ymin, fm((float)u, g.du));
    const float sy_ = g.ct_style == 2 ? pu : g.srcy;
    e.x2x = fs(fm(g.srcx, c), fm(sy_, s));
    e.x2y = fa(fm(g.srcx, s), fm(sy_, c));
    e.x1x = fs(fm(g.dod, c), fm(pu, s));
    e.x1y = fa(fm(g.dod, s), fm(pu, c));
    const int src = g.ct_style == 3 ? v / g.nvr : 0;
    e.x1z = fa(g.zmin, fm((float)(v - src * g.nvr), g.dv));
    e.x2z = g.ct_style == 3 ? fa(g.zsrc0, fm((float)src, g.zsrc_dz)) : (g.ct_style == 0 ? g.srcz : e.x1z);
    return e;
}
// d12 = |X2 - X1| (universal.cu:290)
__device__ __forceinline__ float ray_d12(const RayEnds& e)
{
    const float dx = fs(e.x2x, e.x1x), dy = fs(e.x2y, e.x1y), dz = fs(e.x2z, e.x1z);
    return __fsqrt_rn(fa(fa(fm(dx, dx), fm(dy, dy)), fm(dz, dz)));
}

// The tetrahedron-beam backprojector's voxel centre: b + v*(0.5f + i) along x
// and y, bz + vz*(0.5f + k) (T42/voxel/kernel_IterativeRecon_TBCT_voxel.cu:
// 568-570); in a slab of its multi-GPU build b + v*0.5f + i*v and
// boundary_voxel_z + vz*(ZETA/D*s + 0.5f) + k*vz (T42/voxel/..._multiGPU.cu:1140-1142).
__device__ __forceinline__ float tb_centre_xy(const DevGeom& g, float b, float v, int i)
{
    return g.slab_n > 1 ? fa(fa(b, fm(v, 0.5f)), fm((float)i, v)) : fa(b, fm(v, fa(0.5f, (float)i)));
}
__device__ __forceinline__ float tb_centre_z(const DevGeom& g, int k)
{
    return g.slab_n > 1 ? fa(fa(g.bz_ref, g.cz_off), fm((float)k, g.vz)) : fa(g.bz, fm(g.vz, fa(0.5f, (float)k)));
}

// Dispatch a runtime ctr_dtype to a storage type.
#define CTR_DISPATCH_DTYPE(dt, T, ...)                      \
    switch (dt) {                                           \
    case CTR_F32: { using T = float; __VA_ARGS__; } break;  \
    case CTR_BF16: { using T = __nv_bfloat16; __VA_ARGS__; } break; \
    case CTR_F16: { using T = __half; __VA_ARGS__; } break; \
    default: return set_error(CTR_ERR_INVALID_ARGUMENT, "bad dtype %d", (int)(dt)); \
    }

}  // namespace ctr
