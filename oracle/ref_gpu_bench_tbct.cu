/*
 * ref_gpu_bench_tbct.cu -- the tetrahedron-beam program's own GPU path timed
 * on this GPU.
 *
 * MEASUREMENT INFRASTRUCTURE ONLY (never the product, never linked by it).
 * The Makefile compiles this file with nvcc for sm_100a with the reference's
 * own flags (-use_fast_math, OpenMP), -DREF_TBCT_DIR pointing at
 * TBCT/TBCT_1024V_1024P_v4.2_20171012 (T42/ below); its kernels and host
 * functions are #included from where they lie and are not copied.  Output:
 * oracle/_ref/ref_gpu_bench_tbct.
 *
 * The constants are T42's own sample configuration (T42/main_recon.cu:41-120,
 * metres): 512^3 voxels of 0.1 mm, K = 64 sources with 16 detector rows of
 * 1024 columns each (1.2e-4 m pixels), DSO 0.2 m, DOD -0.2 m, 360 views 1
 * degree apart, Lip_con 32, lambda_TV 0 (no TV prox).  main() follows T42's
 * driver for FISTA == 1 (T42/main_recon.cu:270-430): each iteration copies y
 * into the pinned volume, runs the SART pass (Reconstruction_3D_ray_driven_TBCT,
 * whose kernels read the pinned host sinogram), the OpenMP FISTA step and the
 * objective (Forward_3D_ray_driven_siddon_TBCT into device memory,
 * L2_norm_gpu, TV_norm_gpu).  The sinogram is T42's own forward projection of
 * a phantom.  Prints one JSON line.
 *
 *   ref_gpu_bench_tbct [timed iterations = 1] [warm-up iterations = 1]
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
#include <omp.h>
using namespace std;

#define Default_GPU (0)
#define Number_of_Devices (1)
#define pixelDriven (0)
#define MAX_infi (1.0 / 0.0)
#define FISTA (1)
#define DenoiseOption (1)

/* T42/main_recon.cu:41-120 */
const float Lip_con = 32.0f;
const float lambda_TV = 0.00f;
const float lambda_L1 = 0.00f;
const float DSO = 0.2f;
const float DOD = -0.2f;
const int M = 512;
const int N = 512;
const int ZETA = 512;
const int NO_X = M;
const int NO_Y = N;
const int NO_Z = ZETA;
const int NO_VOXEL = NO_X * NO_Y * NO_Z;
const float volumn_x = 1.0e-4;
const float inv_volumn_x = 1.0 / volumn_x;
const int M_Offset = 0;
const float boundary_voxel_x = -volumn_x * (float(M) / 2.0f + M_Offset);
const float volumn_y = volumn_x;
const float inv_volumn_y = 1.0 / volumn_y;
const float boundary_voxel_y = -volumn_y * (float(N) / 2.0f);
const float volumn_z = volumn_x;
const float inv_volumn_z = 1.0 / volumn_z;
const float boundary_voxel_z = -volumn_z * (float(ZETA) / 2.0f);
const float boundary_voxel_z_upper = -volumn_z * (float(ZETA) / 2.0f) + ZETA * volumn_z;
const float Offset = 0;
const float PI = 3.141592653589793f;
#define K (64)
const float Detector_pixel_x = 1.2e-4;
const float inv_Detector_pixel_x = 1.0f / Detector_pixel_x;
const int R = 1024;
const int Z_prj = 1024 / K;
const float Detector_Ymin = -Detector_pixel_x * ((R) / 2.0f - 0.5f) + Offset;
const float Detector_Zmin = -Detector_pixel_x * ((Z_prj) / 2.0f - 0.5f);
const float Detector_Zmax = +Detector_pixel_x * ((Z_prj) / 2.0f - 0.5f);
const int N_source = K;
const float Source_z_max = (boundary_voxel_z_upper - Detector_Zmax) * (DSO - DOD) / DSO + Detector_Zmax;
const float Source_z_min = (boundary_voxel_z - Detector_Zmin) * (DSO - DOD) / DSO + Detector_Zmin;
const float Source_interval = (Source_z_max - Source_z_min) / (K - 1);
const float Source_y = Offset;
const float Source_x = DSO;
const int Nviews = 360;
const float us_rate = 1.00f;
const float initialAngle = 0.00f;
const float shiftAngle = 0.0f;

#define REF_STR2(x) #x
#define REF_STR(x) REF_STR2(x)
#include REF_STR(REF_TBCT_DIR/kernel_tool_functions.cu)
#include REF_STR(REF_TBCT_DIR/host_tool_functions.cu)
#include REF_STR(REF_TBCT_DIR/voxel/kernel_IterativeRecon_TBCT_voxel.cu)
#include REF_STR(REF_TBCT_DIR/voxel/host_IterativeRecon_TBCT_voxel.c)

static double now_s()
{
    struct timeval t;
    gettimeofday(&t, NULL);
    return t.tv_sec + 1e-6 * t.tv_usec;
}

/* a fixed phantom: four ellipsoids (metres), attenuation per metre */
static void phantom(float* f)
{
    const float E[4][7] = {{0, 0, 0, 0.018f, 0.014f, 0.016f, 100.f}, {0.004f, -0.003f, 0.002f, 0.006f, 0.004f, 0.005f, 50.f},
                           {-0.006f, 0.005f, -0.004f, 0.003f, 0.003f, 0.008f, 75.f},
                           {0.002f, 0.006f, 0.007f, 0.0016f, 0.0016f, 0.0016f, 150.f}};
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
    const int iters = argc > 1 ? atoi(argv[1]) : 1;
    const int warm = argc > 2 ? atoi(argv[2]) : 1;
    cudaSetDevice(Default_GPU);
    float step_size = 2.0f / Lip_con;
    size_t size_proj_data = sizeof(float) * R * Z_prj * N_source * Nviews;
    size_t size_volume = sizeof(float) * M * N * ZETA;
    float* F_Y_k = new float[(size_t)M * N * ZETA];
    float* F_X_k_1 = new float[(size_t)M * N * ZETA];
    memset(F_Y_k, 0, size_volume);
    memset(F_X_k_1, 0, size_volume);
    float *F_recon, *h_proj_data;
    if (cudaHostAlloc((void**)&F_recon, size_volume, cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc((void**)&h_proj_data, size_proj_data, cudaHostAllocDefault) != cudaSuccess) {
        printf("{\"impl\": \"reference-gpu-tbct\", \"error\": \"pinned allocation failed\"}\n");
        return 1;
    }
    phantom(F_recon);
    double t = now_s();
    Forward_3D_ray_driven_siddon_TBCT(F_recon, h_proj_data);   /* the sinogram: T42's own projection */
    cudaDeviceSynchronize();
    const double t_sino = now_s() - t;
    memset(F_recon, 0, size_volume);
    float t_k, t_k_1 = 1.0f;
    double sum_sart = 0, sum_fista = 0, sum_obj = 0, sum_iter = 0;
    double data_fidelity = 0, tv_value = 0;
    for (int k = 1; k <= warm + iters; ++k) {
        const double t0 = now_s();
#pragma omp parallel for
        for (int i = 0; i < NO_VOXEL; i++) F_recon[i] = F_Y_k[i];
        Reconstruction_3D_ray_driven_TBCT(F_recon, h_proj_data, step_size);
        const double t1 = now_s();
        t_k = (1.0f + sqrt(1.0f + 4.0f * t_k_1 * t_k_1)) / 2.0f;
#pragma omp parallel for
        for (int i = 0; i < NO_VOXEL; i++) {
            F_Y_k[i] = F_recon[i] + (t_k_1 - 1.0f) / t_k * (F_recon[i] - F_X_k_1[i]);
            F_X_k_1[i] = F_recon[i];
        }
        t_k_1 = t_k;
        const double t2 = now_s();
        /* objective */
        float* d_proj_forward = NULL;
        cudaMalloc((void**)&d_proj_forward, size_proj_data);
        Forward_3D_ray_driven_siddon_TBCT(F_recon, d_proj_forward);
        data_fidelity = L2_norm_gpu(d_proj_forward, h_proj_data);
        cudaFree(d_proj_forward);
        float* d_recon;
        cudaMalloc((void**)&d_recon, size_volume);
        cudaMemcpyAsync(d_recon, F_recon, size_volume, cudaMemcpyDefault);
        tv_value = TV_norm_gpu(d_recon);
        cudaFree(d_recon);
        cudaDeviceSynchronize();
        const double t3 = now_s();
        fprintf(stderr, "iteration %d: SART %.3f s, FISTA %.3f s, objective %.3f s (TV %g, fidelity %g)\n", k, t1 - t0,
                t2 - t1, t3 - t2, tv_value, data_fidelity);
        if (k > warm) {
            sum_sart += t1 - t0;
            sum_fista += t2 - t1;
            sum_obj += t3 - t2;
            sum_iter += t3 - t0;
        }
    }
    const cudaError_t e = cudaGetLastError();
    printf("{\"impl\": \"reference-gpu-tbct\", \"seconds_per_iteration\": %.6f, \"iter_per_s\": %.6f, "
           "\"parts_s\": {\"sart\": %.6f, \"fista_host\": %.6f, \"objective\": %.6f}, "
           "\"iterations\": %d, \"warmup\": %d, \"sinogram_s\": %.3f, \"cuda_error\": \"%s\", "
           "\"objective_last\": [%.9g, %.9g]}\n",
           sum_iter / iters, iters / sum_iter, sum_sart / iters, sum_fista / iters, sum_obj / iters, iters, warm,
           t_sino, cudaGetErrorString(e), tv_value, data_fidelity);
    cudaFreeHost(F_recon);
    cudaFreeHost(h_proj_data);
    delete[] F_Y_k;
    delete[] F_X_k_1;
    return e == cudaSuccess ? 0 : 2;
}
