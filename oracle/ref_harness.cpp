/*
 * ref_harness.cpp -- runs the reference's own CUDA kernel sources on the CPU.
 *
 * TEST INFRASTRUCTURE ONLY (the checker and the CPU baseline, never the
 * product).  The Makefile compiles this file with -DREF_DIR pointing at the
 * reference's CBCT v6.3 snapshot; the reference sources are #included from
 * where they lie and are not copied.  Output: oracle/_ref/libctref.so.
 *
 * CUDA keywords are defined away, threadIdx/blockIdx/blockDim/gridDim become
 * thread-local variables that the launch loops below set, and the reference's
 * compile-time geometry constants (V63/main_recon.cu:54-111) become mutable
 * globals set by ref_set_geometry() with the same float/double steps.
 *
 * With -DREF_TBCT the same harness runs the tetrahedron-beam program's
 * projector, backprojector and update kernels instead
 * (TBCT/TBCT_1024V_1024P_v4.2_20171012/voxel/kernel_IterativeRecon_TBCT_voxel.cu,
 * abbreviated T42/, read from REF_TBCT_DIR; output oracle/_ref/libctref_tbct.so);
 * with -DREF_TBCT -DREF_TBCT_MULTI its multi-GPU build's kernels
 * (T42/voxel/kernel_IterativeRecon_TBCT_voxel_multiGPU.cu) with its host
 * sequence (T42/voxel/host_IterativeRecon_TBCT_voxel_multiGPU.c), the devices
 * a loop over the slabs (oracle/_ref/libctref_tbct_multi.so).
 * Its atomicAdd becomes a plain add: a voxel's sources are launched in
 * ascending order by one thread.
 *
 * The CBCT builds also run the multi-GPU build's kernels
 * (V63/kernel_IterativeRecon_universal_multiGPU.cu) with its host sequence
 * (V63/host_IterativeRecon_CBCT_multiGPU.c): the devices become a loop over
 * the slabs in device order, Number_of_Devices a global set per call.
 */
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
using namespace std;

struct ref_dim3 { unsigned x, y, z; };
static thread_local ref_dim3 tl_threadIdx, tl_blockIdx, tl_blockDim, tl_gridDim;
#define threadIdx tl_threadIdx
#define blockIdx tl_blockIdx
#define blockDim tl_blockDim
#define gridDim tl_gridDim
#define __global__
#define __device__
#define __host__
#define __shared__
static inline void __syncthreads() {}
float sdata[1];   /* satisfies the never-called shared-memory reduction kernels */

#ifndef CT_style
#define CT_style 0   /* the Makefile builds one library per style */
#endif
#define MAX_infi (1.0 / 0.0)

/* geometry globals with the reference's names */
static int M, N, ZETA, NO_X, NO_Y, NO_Z, NO_VOXEL, R, Z_prj, M_Offset, Nviews;
static float DSO, DOD, Offset, Detector_pixel_x, Detector_Ymin, Detector_Zmin;
static float volumn_x, inv_volumn_x, boundary_voxel_x;
static float volumn_y, inv_volumn_y, boundary_voxel_y;
static float volumn_z, inv_volumn_z, boundary_voxel_z;
static float Source_x, Source_y, Source_z;
static float us_rate, initialAngle, shiftAngle;
static const float PI = 3.141592653589793f;

#define REF_STR2(x) #x
#define REF_STR(x) REF_STR2(x)
#ifdef REF_TBCT
/* T42/main_recon.cu:76-108 */
static float boundary_voxel_z_upper, Detector_Zmax, Source_z_min, Source_interval;
static int N_source;
static inline float atomicAdd(float* p, float v)
{
    const float o = *p;
    *p = o + v;
    return o;
}
#ifdef REF_TBCT_MULTI
/* the multi-GPU build's device count (T42/main_recon.cu:17), set per call */
static int Number_of_Devices = 1;
#include REF_STR(REF_TBCT_DIR/voxel/kernel_IterativeRecon_TBCT_voxel_multiGPU.cu)
#else
#include REF_STR(REF_TBCT_DIR/voxel/kernel_IterativeRecon_TBCT_voxel.cu)
#endif
#else
/* the multi-GPU build's device count (V63/main_recon.cu:23), set per call */
static int Number_of_Devices = 1;
#include REF_STR(REF_DIR/kernel_IterativeRecon_universal.cu)
#include REF_STR(REF_DIR/kernel_IterativeRecon_universal_multiGPU.cu)
#include REF_STR(REF_DIR/kernel_FGP_Denoise_GPUx7.cu)
#include REF_STR(REF_DIR/kernel_tool_functions.cu)
#include REF_STR(REF_DIR/FDK/kernel_FDK.cu)
#include REF_STR(REF_DIR/FDK/FFT1d.h)
#endif

#include "ct_oracle.h"

extern "C" {

/* V63/main_recon.cu:60-111 with the constants taken from the description. */
int ref_set_geometry(const og_desc* d)
{
    if (d->vy > 0.f && d->vy != d->vx) return -1;   /* the reference has one voxel pitch */
    /* volumn_z = (CT_style == 0) ? volumn_x : Detector_pixel_x (V63/main_recon.cu:96);
     * T42/main_recon.cu:73 volumn_z = volumn_x */
    const float vz_ref = CT_style == 0 ? d->vx : d->du;
#ifdef REF_TBCT
    if (d->ct_style != 3 || d->n_sources < 1) return -1;
#else
    if (d->ct_style != CT_style) return -1;
#endif
    if (d->vz > 0.f && d->vz != vz_ref) return -1;
    if (d->dv > 0.f && d->dv != d->du) return -1;   /* and one detector pitch */
    M = d->nx; N = d->ny; ZETA = d->nz;
    NO_X = M; NO_Y = N; NO_Z = ZETA; NO_VOXEL = M * N * ZETA;
    R = d->nu; Z_prj = d->nv; Nviews = d->nviews;
    DSO = d->dso; DOD = d->dod; Offset = d->offset; M_Offset = d->m_offset;
    Detector_pixel_x = d->du;
    Detector_Ymin = -Detector_pixel_x * (float(R) / 2.0f - 0.5f) + Offset;
    Detector_Zmin = -Detector_pixel_x * (float(Z_prj) / 2.0f - 0.5f);
    volumn_x = d->vx;
    inv_volumn_x = 1.0 / volumn_x;
    boundary_voxel_x = -volumn_x * (float(M) / 2.0f + M_Offset);
    volumn_y = volumn_x;
    inv_volumn_y = 1.0 / volumn_y;
    boundary_voxel_y = -volumn_y * (float(N) / 2.0f);
    volumn_z = CT_style == 0 ? volumn_x : Detector_pixel_x;
    inv_volumn_z = 1.0 / volumn_z;
    boundary_voxel_z = -volumn_z * (float(ZETA) / 2.0f);
    Source_x = DSO; Source_y = Offset; Source_z = 0;
    us_rate = d->us_rate; initialAngle = d->initial_angle; shiftAngle = d->shift_angle;
#ifdef REF_TBCT
    /* T42/main_recon.cu:76, :93, :96-108 */
    boundary_voxel_z_upper = -volumn_z * (float(ZETA) / 2.0f) + ZETA * volumn_z;
    Detector_Zmax = +Detector_pixel_x * ((Z_prj) / 2.0f - 0.5f);
    N_source = d->n_sources;
    if (N_source == 1) {
        Source_z_min = 0.0f;
        Source_interval = 0.0f;
    } else {
        const float Source_z_max = (boundary_voxel_z_upper - Detector_Zmax) * (DSO - DOD) / DSO + Detector_Zmax;
        Source_z_min = (boundary_voxel_z - Detector_Zmin) * (DSO - DOD) / DSO + Detector_Zmin;
        Source_interval = (Source_z_max - Source_z_min) / (N_source - 1);
    }
#endif
    return 0;
}

/* V63/host_IterativeRecon_CBCT.c:34-41 */
void ref_view_trig(int j, int fdk, float* s_out, float* c_out)
{
    float t_theta = (float)(j * us_rate + initialAngle);
    t_theta = (t_theta + shiftAngle) * PI / 180.0f;
    if (!fdk) t_theta = -t_theta;
    *s_out = sin(t_theta);
    *c_out = cos(t_theta);
}

#if defined(REF_TBCT) && defined(REF_TBCT_MULTI)
static int ref_devices(int D)
{
    if (D < 1 || ZETA % D != 0 || Z_prj % D != 0) return -1;
    Number_of_Devices = D;
    return 0;
}

/* forward_ray_driven_3d_kernel_correction_separate over grid (1, Z_prj, N_source) x
 * block R on slab sub (T42/voxel/host_IterativeRecon_TBCT_voxel_multiGPU.c:78-82) */
int ref_slab_forward_view(int D, int sub, const float* vol_slab, float* sumLen, float* weightedLen, float s, float c)
{
    if (ref_devices(D) != 0) return -1;
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (int src = 0; src < N_source; ++src)
        for (int v = 0; v < Z_prj; ++v) {
            tl_blockDim = {(unsigned)R, 1, 1};
            tl_gridDim = {1, (unsigned)Z_prj, (unsigned)N_source};
            for (int u = 0; u < R; ++u) {
                tl_blockIdx = {0, (unsigned)v, (unsigned)src};
                tl_threadIdx = {(unsigned)u, 0, 0};
                forward_ray_driven_3d_kernel_correction_separate((float*)vol_slab, sumLen, weightedLen, s, c, sub);
            }
        }
    return 0;
}

/* the host's combination (multiGPU.c:89-101): memset, kernel_add_proj per device
 * in order (weighted, then lengths), kernel_divide_proj; parts [D][N_source*Z_prj*R] */
int ref_combine_view(int D, const float* sumLen, const float* weightedLen, const float* b, float* corr)
{
    if (ref_devices(D) != 0) return -1;
    const long long P = (long long)R * Z_prj * N_source;
    float* hs = (float*)calloc(P, sizeof(float));
    float* hw = (float*)calloc(P, sizeof(float));
    auto grid = [&](auto&& fn) {
        tl_blockDim = {(unsigned)R, 1, 1};
        tl_gridDim = {1, (unsigned)Z_prj, (unsigned)N_source};
        for (int src = 0; src < N_source; ++src)
            for (int v = 0; v < Z_prj; ++v)
                for (int u = 0; u < R; ++u) {
                    tl_blockIdx = {0, (unsigned)v, (unsigned)src};
                    tl_threadIdx = {(unsigned)u, 0, 0};
                    fn();
                }
    };
    for (int i = 0; i < D; ++i) {
        grid([&] { kernel_add_proj(hw, (float*)weightedLen + P * i); });
        grid([&] { kernel_add_proj(hs, (float*)sumLen + P * i); });
    }
    grid([&] { kernel_divide_proj(corr, (float*)b, hs, hw); });
    free(hs);
    free(hw);
    return 0;
}

/* backprj_ray_driven_3d_kernel_multiGPU into zeroed slab volumes (a voxel's
 * sources in ascending order), then update (multiGPU.c:119-135); command is
 * ignored, as the kernels have none */
int ref_slab_backproject_view(int D, int sub, float* vol_slab, const float* corr, float beta, float s, float c,
                              int command)
{
    (void)command;
    if (ref_devices(D) != 0) return -1;
    const int Zs = ZETA / D;
    const long long V = (long long)M * N * Zs;
    float* ws = (float*)calloc(V, sizeof(float));
    float* len = (float*)calloc(V, sizeof(float));
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
    for (int k = 0; k < Zs; ++k)
        for (int j = 0; j < N; ++j) {
            tl_blockDim = {(unsigned)M, 1, 1};
            tl_gridDim = {(unsigned)N, (unsigned)Zs, (unsigned)N_source};
            for (int src = 0; src < N_source; ++src)
                for (int i = 0; i < M; ++i) {
                    tl_blockIdx = {(unsigned)j, (unsigned)k, (unsigned)src};
                    tl_threadIdx = {(unsigned)i, 0, 0};
                    backprj_ray_driven_3d_kernel_multiGPU(ws, len, (float*)corr, s, c, sub);
                }
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < Zs; ++k)
        for (int j = 0; j < N; ++j) {
            tl_blockDim = {(unsigned)M, 1, 1};
            for (int i = 0; i < M; ++i) {
                tl_blockIdx = {(unsigned)j, (unsigned)k, 0};
                tl_threadIdx = {(unsigned)i, 0, 0};
                update(vol_slab, ws, len, beta);
            }
        }
    free(ws);
    free(len);
    return 0;
}

/* Reconstruction_3D_ray_driven_TBCT of the multi-GPU build (multiGPU.c:1-183) for
 * the views [v0, v0+nv); the volume is the D slabs back to back (:44-48) */
int ref_sart_views_slabs(int D, float* vol, const float* sino, float beta, int v0, int nv)
{
    if (ref_devices(D) != 0) return -1;
    const long long P = (long long)R * Z_prj * N_source, Vs = (long long)M * N * (ZETA / D);
    float* sl = (float*)calloc(P * D, sizeof(float));
    float* wl = (float*)calloc(P * D, sizeof(float));
    float* corr = (float*)malloc(sizeof(float) * P);
    for (int j = v0; j < v0 + nv; ++j) {
        float s, c;
        ref_view_trig(j, 0, &s, &c);
        for (int i = 0; i < D; ++i) ref_slab_forward_view(D, i, vol + Vs * i, sl + P * i, wl + P * i, s, c);
        ref_combine_view(D, sl, wl, sino + P * j, corr);
        for (int i = 0; i < D; ++i) ref_slab_backproject_view(D, i, vol + Vs * i, corr, beta, s, c, 1);
    }
    free(sl);
    free(wl);
    free(corr);
    return 0;
}

/* Forward_3D_ray_driven_siddon_TBCT of the multi-GPU build, one view
 * (multiGPU.c:185-306): device i projects rows [Z_prj/D*i, Z_prj/D*(i+1)) of
 * every source's band with forward_ray_driven_3d_kernel_correction_multiGPU,
 * command 0, into [src][row][col] portions copied back per source (:264-267) */
int ref_forward_view_split(int D, const float* vol, float* out, float s, float c)
{
    if (ref_devices(D) != 0) return -1;
    const int rows = Z_prj / D;
    float* part = (float*)malloc(sizeof(float) * (size_t)R * rows * N_source);
    for (int i = 0; i < D; ++i) {
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
        for (int src = 0; src < N_source; ++src)
            for (int v = 0; v < rows; ++v) {
                tl_blockDim = {(unsigned)R, 1, 1};
                tl_gridDim = {1, (unsigned)rows, (unsigned)N_source};
                for (int u = 0; u < R; ++u) {
                    tl_blockIdx = {0, (unsigned)v, (unsigned)src};
                    tl_threadIdx = {(unsigned)u, 0, 0};
                    forward_ray_driven_3d_kernel_correction_multiGPU((float*)vol, part, part, s, c, i, 0);
                }
            }
        for (int k = 0; k < N_source; ++k)
            memcpy(out + (size_t)R * Z_prj * k + (size_t)R * rows * i, part + (size_t)R * rows * k,
                   sizeof(float) * R * rows);
    }
    free(part);
    return 0;
}
#elif defined(REF_TBCT)
/* forward_ray_driven_3d_kernel_correction over grid (1, Z_prj, N_source) x block R
 * (T42/voxel/host_IterativeRecon_TBCT_voxel.c:48-49, one block row per launch here) */
void ref_forward_view(const float* vol, float* out, const float* b, float s, float c, int command)
{
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (int src = 0; src < N_source; ++src)
        for (int v = 0; v < Z_prj; ++v) {
            tl_blockDim = {(unsigned)R, 1, 1};
            tl_gridDim = {1, (unsigned)Z_prj, (unsigned)N_source};
            for (int u = 0; u < R; ++u) {
                tl_blockIdx = {0, (unsigned)v, (unsigned)src};
                tl_threadIdx = {(unsigned)u, 0, 0};
                forward_ray_driven_3d_kernel_correction((float*)vol, out, (float*)b, s, c, (float)command);
            }
        }
}

/* The TBCT SART update of one view (T42/voxel/host_IterativeRecon_TBCT_voxel.c:67-75):
 * zeroed weighted-sum and length volumes, backprj_ray_driven_3d_kernel over
 * every voxel and source (sources of a voxel in ascending order), then
 * update.  The kernel has no command: command is ignored. */
void ref_backproject_view(float* vol, const float* corr, float beta, float s, float c, int command)
{
    (void)command;
    const long long V = (long long)M * N * ZETA;
    float* ws = (float*)calloc(V, sizeof(float));
    float* len = (float*)calloc(V, sizeof(float));
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
    for (int k = 0; k < ZETA; ++k)
        for (int j = 0; j < N; ++j) {
            tl_blockDim = {(unsigned)M, 1, 1};
            tl_gridDim = {(unsigned)N, (unsigned)ZETA, (unsigned)N_source};
            for (int src = 0; src < N_source; ++src)
                for (int i = 0; i < M; ++i) {
                    tl_blockIdx = {(unsigned)j, (unsigned)k, (unsigned)src};
                    tl_threadIdx = {(unsigned)i, 0, 0};
                    backprj_ray_driven_3d_kernel(ws, len, (float*)corr, s, c);
                }
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < ZETA; ++k)
        for (int j = 0; j < N; ++j) {
            tl_blockDim = {(unsigned)M, 1, 1};
            for (int i = 0; i < M; ++i) {
                tl_blockIdx = {(unsigned)j, (unsigned)k, 0};
                tl_threadIdx = {(unsigned)i, 0, 0};
                update(vol, ws, len, beta);
            }
        }
    free(ws);
    free(len);
}

/* Reconstruction_3D_ray_driven_TBCT (T42/voxel/host_IterativeRecon_TBCT_voxel.c:1-92)
 * for the views [v0, v0+nv) */
void ref_sart_views(float* vol, const float* sino, float beta, int v0, int nv)
{
    const long long P = (long long)R * Z_prj * N_source;
    float* corr = (float*)malloc(sizeof(float) * P);
    for (int j = v0; j < v0 + nv; ++j) {
        float s, c;
        ref_view_trig(j, 0, &s, &c);
        ref_forward_view(vol, corr, sino + P * j, s, c, 1);
        ref_backproject_view(vol, corr, beta, s, c, 1);
    }
    free(corr);
}
#else
/* forward_ray_driven_3d_kernel_correction over grid (1, Z_prj) x block R */
void ref_forward_view(const float* vol, float* out, const float* b, float s, float c, int command)
{
#pragma omp parallel for schedule(dynamic, 1)
    for (int v = 0; v < Z_prj; ++v) {
        tl_blockDim = {(unsigned)R, 1, 1};
        tl_gridDim = {1, (unsigned)Z_prj, 1};
        for (int u = 0; u < R; ++u) {
            tl_blockIdx = {0, (unsigned)v, 0};
            tl_threadIdx = {(unsigned)u, 0, 0};
            forward_ray_driven_3d_kernel_correction((float*)vol, out, (float*)b, s, c, command);
        }
    }
}

/* backprj_ray_driven_3d_kernel over grid (1, N, ZETA) x block M */
void ref_backproject_view(float* vol, const float* corr, float beta, float s, float c, int command)
{
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
    for (int k = 0; k < ZETA; ++k)
        for (int j = 0; j < N; ++j) {
            tl_blockDim = {(unsigned)M, 1, 1};
            tl_gridDim = {1, (unsigned)N, (unsigned)ZETA};
            for (int i = 0; i < M; ++i) {
                tl_blockIdx = {0, (unsigned)j, (unsigned)k};
                tl_threadIdx = {(unsigned)i, 0, 0};
                backprj_ray_driven_3d_kernel(vol, (float*)corr, beta, s, c, command);
            }
        }
}

/* Reconstruction_3D_ray_driven_CBCT (V63/host_IterativeRecon_CBCT.c:1-67) for
 * the views [v0, v0+nv): FP command 1 then BP command 1, strictly in order. */
void ref_sart_views(float* vol, const float* sino, float beta, int v0, int nv)
{
    const long long P = (long long)R * Z_prj;
    float* corr = (float*)malloc(sizeof(float) * P);
    for (int j = v0; j < v0 + nv; ++j) {
        float s, c;
        ref_view_trig(j, 0, &s, &c);
        ref_forward_view(vol, corr, sino + P * j, s, c, 1);
        ref_backproject_view(vol, corr, beta, s, c, 1);
    }
    free(corr);
}

/* ---- the multi-GPU build (Number_of_Devices = D > 1) ---- */
static int ref_devices(int D)
{
    if (D < 1 || ZETA % D != 0 || Z_prj % D != 0) return -1;
    Number_of_Devices = D;
    return 0;
}

/* forward_ray_driven_3d_kernel_correction_separate over grid (1, Z_prj) x block R
 * on the slab volume sub (V63/host_IterativeRecon_CBCT_multiGPU.c:71-75) */
int ref_slab_forward_view(int D, int sub, const float* vol_slab, float* sumLen, float* weightedLen, float s, float c)
{
    if (ref_devices(D) != 0) return -1;
#pragma omp parallel for schedule(dynamic, 1)
    for (int v = 0; v < Z_prj; ++v) {
        tl_blockDim = {(unsigned)R, 1, 1};
        tl_gridDim = {1, (unsigned)Z_prj, 1};
        for (int u = 0; u < R; ++u) {
            tl_blockIdx = {0, (unsigned)v, 0};
            tl_threadIdx = {(unsigned)u, 0, 0};
            forward_ray_driven_3d_kernel_correction_separate((float*)vol_slab, sumLen, weightedLen, s, c, sub);
        }
    }
    return 0;
}

/* the host's combination of the D parts, [D][Z_prj*R] each
 * (V63/host_IterativeRecon_CBCT_multiGPU.c:82-95): memset, kernel_add_proj per
 * device in order (weighted, then lengths), kernel_divide_proj */
int ref_combine_view(int D, const float* sumLen, const float* weightedLen, const float* b, float* corr)
{
    if (ref_devices(D) != 0) return -1;
    const long long P = (long long)R * Z_prj;
    float* hs = (float*)calloc(P, sizeof(float));
    float* hw = (float*)calloc(P, sizeof(float));
    auto grid = [&](auto&& fn) {
        tl_blockDim = {(unsigned)R, 1, 1};
        tl_gridDim = {1, (unsigned)Z_prj, 1};
        for (int v = 0; v < Z_prj; ++v)
            for (int u = 0; u < R; ++u) {
                tl_blockIdx = {0, (unsigned)v, 0};
                tl_threadIdx = {(unsigned)u, 0, 0};
                fn();
            }
    };
    for (int i = 0; i < D; ++i) {
        grid([&] { kernel_add_proj(hw, (float*)weightedLen + P * i); });
        grid([&] { kernel_add_proj(hs, (float*)sumLen + P * i); });
    }
    grid([&] { kernel_divide_proj(corr, (float*)b, hs, hw); });
    free(hs);
    free(hw);
    return 0;
}

/* backprj_ray_driven_3d_kernel_multiGPU over grid (1, N, ZETA/D) x block M */
int ref_slab_backproject_view(int D, int sub, float* vol_slab, const float* corr, float beta, float s, float c,
                              int command)
{
    if (ref_devices(D) != 0) return -1;
    const int Zs = ZETA / D;
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
    for (int k = 0; k < Zs; ++k)
        for (int j = 0; j < N; ++j) {
            tl_blockDim = {(unsigned)M, 1, 1};
            tl_gridDim = {1, (unsigned)N, (unsigned)Zs};
            for (int i = 0; i < M; ++i) {
                tl_blockIdx = {0, (unsigned)j, (unsigned)k};
                tl_threadIdx = {(unsigned)i, 0, 0};
                backprj_ray_driven_3d_kernel_multiGPU(vol_slab, (float*)corr, beta, s, c, sub, command);
            }
        }
    return 0;
}

/* Reconstruction_3D_ray_driven_CBCT of the multi-GPU build
 * (V63/host_IterativeRecon_CBCT_multiGPU.c:1-161) for the views [v0, v0+nv):
 * the volume is the D slabs back to back (:40-44) */
int ref_sart_views_slabs(int D, float* vol, const float* sino, float beta, int v0, int nv)
{
    if (ref_devices(D) != 0) return -1;
    const long long P = (long long)R * Z_prj, Vs = (long long)M * N * (ZETA / D);
    float* sl = (float*)calloc(P * D, sizeof(float));
    float* wl = (float*)calloc(P * D, sizeof(float));
    float* corr = (float*)malloc(sizeof(float) * P);
    for (int j = v0; j < v0 + nv; ++j) {
        float s, c;
        ref_view_trig(j, 0, &s, &c);
        for (int i = 0; i < D; ++i) ref_slab_forward_view(D, i, vol + Vs * i, sl + P * i, wl + P * i, s, c);
        ref_combine_view(D, sl, wl, sino + P * j, corr);
        for (int i = 0; i < D; ++i) ref_slab_backproject_view(D, i, vol + Vs * i, corr, beta, s, c, 1);
    }
    free(sl);
    free(wl);
    free(corr);
    return 0;
}

/* Forward_3D_ray_driven_siddon of the multi-GPU build, one view
 * (V63/host_IterativeRecon_CBCT_multiGPU.c:171-258): device i projects rows
 * [Z_prj/D*i, Z_prj/D*(i+1)) of the whole volume with
 * forward_ray_driven_3d_kernel_correction_multiGPU, command 0 */
int ref_forward_view_split(int D, const float* vol, float* out, float s, float c)
{
    if (ref_devices(D) != 0) return -1;
    const int rows = Z_prj / D;
    for (int i = 0; i < D; ++i) {
        float* part = out + (long long)R * rows * i;
#pragma omp parallel for schedule(dynamic, 1)
        for (int v = 0; v < rows; ++v) {
            tl_blockDim = {(unsigned)R, 1, 1};
            tl_gridDim = {1, (unsigned)rows, 1};
            for (int u = 0; u < R; ++u) {
                tl_blockIdx = {0, (unsigned)v, 0};
                tl_threadIdx = {(unsigned)u, 0, 0};
                forward_ray_driven_3d_kernel_correction_multiGPU((float*)vol, part, part, s, c, i, 0);
            }
        }
    }
    return 0;
}

/* FGP_denoise_GPUx7_exact (V63/host_FGP_Denoise_GPUx7.c:1-111), in place */
void ref_fgp(float* f, float lambda, int niter)
{
    const long long V = (long long)M * N * ZETA;
    const long long nr = (long long)ZETA * N * (M + 1), ns = (long long)ZETA * (N + 1) * M,
                    nt = (long long)(ZETA + 1) * N * M;
    float* r = (float*)calloc(nr, 4); float* o = (float*)calloc(nr, 4);
    float* s = (float*)calloc(ns, 4); float* p = (float*)calloc(ns, 4);
    float* t = (float*)calloc(nt, 4); float* q = (float*)calloc(nt, 4);
    float* L = (float*)calloc(V, 4);
    float t_k_1 = 1.0f, t_k;
    auto launch = [&](int which) {
#pragma omp parallel for collapse(2) schedule(static)
        for (int z = 0; z < ZETA; ++z)
            for (int y = 0; y < N; ++y) {
                tl_blockDim = {(unsigned)M, 1, 1};
                tl_gridDim = {(unsigned)N, (unsigned)ZETA, 1};
                for (int x = 0; x < M; ++x) {
                    tl_blockIdx = {(unsigned)y, (unsigned)z, 0};
                    tl_threadIdx = {(unsigned)x, 0, 0};
                    if (which == 0) FGP_operator_L_Pc(f, r, s, t, L, lambda);
                    else if (which == 1) FGP_operator_LT_Pp(r, s, t, L, o, p, q, t_k_1, t_k, 1.0f / (lambda * 12.0f));
                    else FGP_operator_L_Pc(f, o, p, q, L, lambda);
                }
            }
    };
    for (int i = 0; i < niter; ++i) {
        t_k = (1.0f + sqrt(1.0f + 4.0f * t_k_1 * t_k_1)) / 2.0f;
        launch(0);
        launch(1);
        t_k_1 = t_k;
    }
    launch(2);
    memcpy(f, L, sizeof(float) * V);
    free(r); free(o); free(s); free(p); free(t); free(q); free(L);
}

/* TV_norm_kernel into a zeroed buffer, summed in double (the reference's
 * alternative CPU summation, V63/host_tool_functions.cu:81-87) */
double ref_tv_norm(const float* vol)
{
    const long long V = (long long)M * N * ZETA;
    float* tv = (float*)calloc(V, 4);
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < ZETA; ++z)
        for (int y = 0; y < N; ++y) {
            tl_blockDim = {(unsigned)M, 1, 1};
            for (int x = 0; x < M; ++x) {
                tl_blockIdx = {0, (unsigned)y, (unsigned)z};
                tl_threadIdx = {(unsigned)x, 0, 0};
                TV_norm_kernel(tv, (float*)vol);
            }
        }
    double acc = 0.0;
    for (long long i = 0; i < V; ++i) acc += (double)tv[i];
    free(tv);
    return acc;
}

/* L2_norm_kernel over (nviews, Z_prj, R), summed in double (the reference's
 * CPU summation, V63/host_tool_functions.cu:37-44); a is overwritten. */
double ref_l2_norm(float* a, const float* b, int nviews)
{
#pragma omp parallel for collapse(2) schedule(static)
    for (int w = 0; w < nviews; ++w)
        for (int v = 0; v < Z_prj; ++v) {
            tl_blockDim = {(unsigned)R, 1, 1};
            tl_gridDim = {1, (unsigned)Z_prj, (unsigned)nviews};
            for (int u = 0; u < R; ++u) {
                tl_blockIdx = {0, (unsigned)v, (unsigned)w};
                tl_threadIdx = {(unsigned)u, 0, 0};
                L2_norm_kernel(a, (float*)b);
            }
        }
    double acc = 0.0;
    const long long n = (long long)nviews * R * Z_prj;
    for (long long i = 0; i < n; ++i) acc += (double)a[i];
    return acc;
}

/* kernel_FDK_projection_adjust over (1, Z_prj, nviews) x R */
void ref_fdk_weight(const float* in, float* out, int nviews)
{
#pragma omp parallel for collapse(2) schedule(static)
    for (int w = 0; w < nviews; ++w)
        for (int v = 0; v < Z_prj; ++v) {
            tl_blockDim = {(unsigned)R, 1, 1};
            for (int u = 0; u < R; ++u) {
                tl_blockIdx = {0, (unsigned)v, (unsigned)w};
                tl_threadIdx = {(unsigned)u, 0, 0};
                kernel_FDK_projection_adjust((float*)in, out);
            }
        }
}

/* RampFiltering_GPU (V63/FDK/FFT_1d_GPU.h:241-287) with the reference's own
 * CPU mixed-radix FFT (V63/FDK/FFT1d.h) in place of cuFFT.  Serial: FFT1d.h
 * keeps its state in file-scope statics. */
void ref_ramp_filter(const float* in, float* out, int nrows)
{
    const int pad_size = R * 2;
    float F_max = 1.0 / 2.0 / (Detector_pixel_x * DSO / (DSO - DOD));
    float F_step = F_max / (pad_size / 2);
    float* H = (float*)malloc(sizeof(float) * pad_size);
    for (int i = 0; i < pad_size; i++) {
        const int k = (i >= pad_size / 2) ? i - pad_size : i;
        H[i] = abs(k) * F_step;
        H[i] *= 0.5f;
    }
    complex<double>* x = new complex<double>[pad_size];
    for (int r = 0; r < nrows; ++r) {
        for (int i = 0; i < pad_size; ++i) x[i] = complex<double>(i < R ? in[(long long)r * R + i] : 0.0, 0.0);
        FFT(x, pad_size, 1);
        for (int i = 0; i < pad_size; ++i) x[i] *= (double)H[i];
        FFT(x, pad_size, -1);          /* FLAG=-1 divides by n, like the reference's /pad_size */
        for (int j = 0; j < R; ++j) out[(long long)r * R + j] = (float)x[j].real();
    }
    delete[] x;
    free(H);
}

/* kernel_FDK_reconstruction over (1, N, ZETA) x M, one view */
void ref_fdk_bp_view(float* vol, const float* proj, float s, float c)
{
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < ZETA; ++k)
        for (int j = 0; j < N; ++j) {
            tl_blockDim = {(unsigned)M, 1, 1};
            for (int i = 0; i < M; ++i) {
                tl_blockIdx = {0, (unsigned)j, (unsigned)k};
                tl_threadIdx = {(unsigned)i, 0, 0};
                kernel_FDK_reconstruction(vol, (float*)proj, s, c);
            }
        }
}

#endif  /* REF_TBCT */

}  /* extern "C" */
