/*
 * ref_gpu_bench.cu -- the reference's own GPU path timed on this GPU.
 *
 * MEASUREMENT INFRASTRUCTURE ONLY (never the product, never linked by it).
 * The Makefile compiles this file with nvcc for sm_100a with the reference's
 * own flags (-use_fast_math, OpenMP), -DREF_DIR pointing at the reference's
 * CBCT v6.3 snapshot; the reference's kernels and host functions are
 * #included from where they lie and are not copied.  Output:
 * oracle/_ref/ref_gpu_bench.
 *
 * The reference fixes its geometry as compile-time constants
 * (V63/main_recon.cu:54-111); they are set here to the 512^3 / 1024-view
 * benchmark scan (0.5 mm voxels, 1024x768 detector of 0.4 mm, DSO 1000 mm,
 * DOD -500 mm), in the reference's names and formulas.  main() follows the
 * reference's driver for FISTA == 1 (V63/main_recon.cu:142-430): the sinogram
 * is the reference's own forward projection of a phantom (:247), each
 * iteration copies y into the pinned volume, runs the reference's SART pass
 * (Reconstruction_3D_ray_driven_CBCT), its FGP-TV (FGP_denoise_GPUx7_exact,
 * 20 iterations), the OpenMP FISTA step on the host and the objective
 * (Forward_3D_ray_driven_siddon + L2_norm_gpu + TV_norm_gpu).  The saving
 * section (file writes) is left out.  Prints one JSON line.
 *
 *   ref_gpu_bench [timed iterations = 2] [warm-up iterations = 1]
 */
#include <cmath>
#include <fstream>
#include <time.h>
#include <iostream>
#include <stddef.h>
#include <stdlib.h>
#include <stdio.h>
#include <string.h>
#include <math.h>
#include <sys/time.h>
#include <assert.h>
#include <omp.h>
using namespace std;

#define Default_GPU 0
#define Number_of_Devices (1)
#define CT_style 0
#define FISTA (1)
#define DenoiseOption (1)
#define DEBUG (1)
#define CT_TOMO (0)
#define MAX_infi (1.0 / 0.0)
#define pixelDriven (0)

/* SART relaxation 2/Lip_con = 0.8 and lambda_denoise_TV = 2*lambda_TV/Lip_con
 * = 0.8 * 2e-4, the benchmark's parameters (V63/main_recon.cu:161-162) */
const float lambda_TV = 2e-4f;
const float lambda_L1 = 0.00f;
const float Lip_con = 2.5f;
const float initialAngle = 0.0f;
const float shiftAngle = 0.0f;

/* geometry in the reference's names and formulas (V63/main_recon.cu:60-111), in mm */
const float DSO = 1000.0f;
const float DOD = -500.0f;
const float Offset = 0;
const int M = 512;
const int N = 512;
const int ZETA = 512;
const int NO_X = M;
const int NO_Y = N;
const int NO_Z = ZETA;
const int NO_VOXEL = M * N * ZETA;
const float Detector_pixel_x = 0.4f;
const int R = 1024;
const int Z_prj = 768;
const float Detector_Ymin = -Detector_pixel_x * (float(R) / 2.0f - 0.5f) + Offset;
const float Detector_Zmin = -Detector_pixel_x * (float(Z_prj) / 2.0f - 0.5f);
const float volumn_x = 0.5f;
const float inv_volumn_x = 1.0 / volumn_x;
const int M_Offset = 0;
const float boundary_voxel_x = -volumn_x * (float(M) / 2.0f + M_Offset);
const float volumn_y = volumn_x;
const float inv_volumn_y = 1.0 / volumn_y;
const float boundary_voxel_y = -volumn_y * (float(N) / 2.0f);
const float volumn_z = volumn_x;
const float inv_volumn_z = 1.0 / volumn_z;
const float boundary_voxel_z = -volumn_z * (float(ZETA) / 2.0f);
const float Source_x = DSO;
const float Source_y = Offset;
const float Source_z = 0;
const float PI = 3.141592653589793f;
const int Nviews = 1024;
const float us_rate = 360.0f / 1024.0f;

#define REF_STR2(x) #x
#define REF_STR(x) REF_STR2(x)
#include REF_STR(REF_DIR/kernel_tool_functions.cu)
#include REF_STR(REF_DIR/host_tool_functions.cu)
#include REF_STR(REF_DIR/kernel_IterativeRecon_universal.cu)
#include REF_STR(REF_DIR/host_IterativeRecon_CBCT.c)
#include REF_STR(REF_DIR/kernel_FGP_Denoise_GPUx7.cu)
#include REF_STR(REF_DIR/host_FGP_Denoise_GPUx7.c)

static double now_s()
{
    struct timeval t;
    gettimeofday(&t, NULL);
    return t.tv_sec + 1e-6 * t.tv_usec;
}

/* a fixed phantom: four ellipsoids (mm), attenuation per mm */
static void phantom(float* f)
{
    const float E[4][7] = {{0, 0, 0, 90, 70, 80, 0.02f}, {20, -15, 10, 30, 20, 25, 0.01f},
                           {-30, 25, -20, 15, 15, 40, 0.015f}, {10, 30, 35, 8, 8, 8, 0.03f}};
#pragma omp parallel for
    for (int k = 0; k < ZETA; ++k)
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < M; ++i) {
                const float x = boundary_voxel_x + (i + 0.5f) * volumn_x;
                const float y = boundary_voxel_y + (j + 0.5f) * volumn_y;
                const float z = boundary_voxel_z + (k + 0.5f) * volumn_z;
                float v = 0.f;
                for (int e = 0; e < 4; ++e) {
                    const float dx = (x - E[e][0]) / E[e][3], dy = (y - E[e][1]) / E[e][4], dz = (z - E[e][2]) / E[e][5];
                    if (dx * dx + dy * dy + dz * dz <= 1.f) v += E[e][6];
                }
                f[(size_t)k * M * N + (size_t)j * M + i] = v;
            }
}

int main(int argc, char** argv)
{
    const int iters = argc > 1 ? atoi(argv[1]) : 2;
    const int warm = argc > 2 ? atoi(argv[2]) : 1;
    cudaSetDevice(Default_GPU);
    const int Niter_denoise = 20;
    float step_size = 2.0f / Lip_con;
    float lambda_denoise_TV = 2.0f * lambda_TV / Lip_con;
    size_t size_proj_data = sizeof(float) * R * Z_prj * Nviews;
    size_t size_volume = sizeof(float) * M * N * ZETA;
    float* F_Y_k = new float[(size_t)M * N * ZETA];
    float* F_X_k_1 = new float[(size_t)M * N * ZETA];
    memset(F_Y_k, 0, size_volume);
    memset(F_X_k_1, 0, size_volume);
    float *F_recon, *h_proj_data;
    if (cudaHostAlloc((void**)&F_recon, size_volume, cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc((void**)&h_proj_data, size_proj_data, cudaHostAllocDefault) != cudaSuccess) {
        printf("{\"impl\": \"reference-gpu\", \"error\": \"pinned allocation failed\"}\n");
        return 1;
    }
    phantom(F_recon);
    double t = now_s();
    Forward_3D_ray_driven_siddon(F_recon, h_proj_data);   /* V63/main_recon.cu:247 */
    const double t_sino = now_s() - t;
    memset(F_recon, 0, size_volume);
    float t_k, t_k_1 = 1.0f;
    double sum_sart = 0, sum_fgp = 0, sum_fista = 0, sum_obj = 0, sum_iter = 0;
    double data_fidelity = 0, tv_value = 0;
    for (int k = 1; k <= warm + iters; ++k) {
        const double t0 = now_s();
#pragma omp parallel for
        for (int i = 0; i < NO_VOXEL; i++) F_recon[i] = F_Y_k[i];
        Reconstruction_3D_ray_driven_CBCT(F_recon, h_proj_data, step_size);
        const double t1 = now_s();
        FGP_denoise_GPUx7_exact(F_recon, lambda_denoise_TV, Niter_denoise);
        const double t2 = now_s();
        t_k = (1.0f + sqrt(1.0f + 4.0f * t_k_1 * t_k_1)) / 2.0f;
#pragma omp parallel for
        for (int i = 0; i < NO_VOXEL; i++) {
            F_Y_k[i] = F_recon[i] + (t_k_1 - 1.0f) / t_k * (F_recon[i] - F_X_k_1[i]);
            F_X_k_1[i] = F_recon[i];
        }
        t_k_1 = t_k;
        const double t3 = now_s();
        /* objective (V63/main_recon.cu:390-430) */
        float* d_proj_forward = NULL;
        cudaMalloc((void**)&d_proj_forward, size_proj_data);
        Forward_3D_ray_driven_siddon(F_recon, d_proj_forward);
        data_fidelity = L2_norm_gpu(d_proj_forward, h_proj_data);
        cudaFree(d_proj_forward);
        float* d_recon;
        cudaMalloc((void**)&d_recon, size_volume);
        cudaMemcpyAsync(d_recon, F_recon, size_volume, cudaMemcpyDefault);
        tv_value = TV_norm_gpu(d_recon);
        cudaFree(d_recon);
        cudaDeviceSynchronize();
        const double t4 = now_s();
        fprintf(stderr, "iteration %d: SART %.3f s, FGP %.3f s, FISTA %.3f s, objective %.3f s (TV %g, fidelity %g)\n",
                k, t1 - t0, t2 - t1, t3 - t2, t4 - t3, tv_value, data_fidelity);
        if (k > warm) {
            sum_sart += t1 - t0;
            sum_fgp += t2 - t1;
            sum_fista += t3 - t2;
            sum_obj += t4 - t3;
            sum_iter += t4 - t0;
        }
    }
    const cudaError_t e = cudaGetLastError();
    printf("{\"impl\": \"reference-gpu\", \"seconds_per_iteration\": %.6f, \"iter_per_s\": %.6f, "
           "\"parts_s\": {\"sart\": %.6f, \"fgp\": %.6f, \"fista_host\": %.6f, \"objective\": %.6f}, "
           "\"iterations\": %d, \"warmup\": %d, \"sinogram_s\": %.3f, \"cuda_error\": \"%s\", "
           "\"objective_last\": [%.9g, %.9g]}\n",
           sum_iter / iters, iters / sum_iter, sum_sart / iters, sum_fgp / iters, sum_fista / iters,
           sum_obj / iters, iters, warm, t_sino, cudaGetErrorString(e), tv_value, data_fidelity);
    cudaFreeHost(F_recon);
    cudaFreeHost(h_proj_data);
    delete[] F_Y_k;
    delete[] F_X_k_1;
    return e == cudaSuccess ? 0 : 2;
}
