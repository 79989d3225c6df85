// drop_in_main.cpp -- the reference's FISTA driver loop (V63/main_recon.cu:286-430,
// FISTA == 1) written against libctrecon's reference-compatible entry points,
// as a maintainer of the reference would after replacing its host and kernel
// includes by ctrecon.h: the same host arrays, the same host function names
// and the same call order; only the geometry comes from
// ctr_set_default_geometry instead of compile-time constants.
//
//   drop_in_main nx ny nz vx nu nv du dso dod n_views iterations step_size
//                lambda_TV Niter_denoise sinogram.raw out_volume.raw [Number_of_Devices]
//
// Number_of_Devices (default 1) is that of the build being replaced
// (V63/main_recon.cu:23; the stock file has 4).
//
// Prints one line per iteration: "k tv fidelity objective" (%.17g), like the
// reference's object_func array (V63/main_recon.cu:419-425).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ctrecon.h"

int main(int argc, char** argv)
{
    if (argc != 17 && argc != 18) {
        std::fprintf(stderr, "usage: %s nx ny nz vx nu nv du dso dod n_views iters step lambda_tv niter_fgp sino out "
                     "[devices]\n", argv[0]);
        return 2;
    }
    const int Number_of_Devices = argc == 18 ? std::atoi(argv[17]) : 1;
    ctr_geometry_desc d;
    std::memset(&d, 0, sizeof(d));
    d.nx = std::atoi(argv[1]); d.ny = std::atoi(argv[2]); d.nz = std::atoi(argv[3]);
    d.vx = (float)std::atof(argv[4]);
    d.nu = std::atoi(argv[5]); d.nv = std::atoi(argv[6]);
    d.du = (float)std::atof(argv[7]);
    d.dso = (float)std::atof(argv[8]); d.dod = (float)std::atof(argv[9]);
    d.n_views = std::atoi(argv[10]);
    d.us_rate = 360.0f / (float)d.n_views;
    const int iters = std::atoi(argv[11]);
    const float step_size = (float)std::atof(argv[12]);
    const float lambda_TV = (float)std::atof(argv[13]);
    const int Niter_denoise = std::atoi(argv[14]);
    if (ctr_set_default_geometry(&d) != CTR_OK || ctr_set_default_devices(Number_of_Devices) != CTR_OK) {
        std::fprintf(stderr, "ctrecon: %s\n", ctr_last_error_string());
        return 1;
    }
    const size_t NO_VOXEL = (size_t)d.nx * d.ny * d.nz;
    const size_t n_proj = (size_t)d.nu * d.nv * d.n_views;
    std::vector<float> h_proj_data(n_proj), F_recon(NO_VOXEL), F_Y_k(NO_VOXEL, 0.f), F_X_k_1(NO_VOXEL, 0.f);
    std::vector<float> proj_forward(n_proj);
    FILE* fp = std::fopen(argv[15], "rb");
    if (!fp || std::fread(h_proj_data.data(), sizeof(float), n_proj, fp) != n_proj) {
        std::fprintf(stderr, "cannot read %s\n", argv[15]);
        return 1;
    }
    std::fclose(fp);

    // lambda_denoise_TV = 2*lambda_TV/Lip_con with step_size = 2/Lip_con (:161-162)
    const float lambda_denoise_TV = lambda_TV * step_size;
    float t_k, t_k_1 = 1.0f;
    for (int k = 1; k <= iters; ++k) {
        for (size_t i = 0; i < NO_VOXEL; i++) F_recon[i] = F_Y_k[i];                   // :346-348
        Reconstruction_3D_ray_driven_CBCT(F_recon.data(), h_proj_data.data(), step_size);   // :352
        if (lambda_TV > 0.0f) FGP_denoise_GPUx7_exact(F_recon.data(), lambda_denoise_TV, Niter_denoise);   // :360
        t_k = (1.0f + std::sqrt(1.0f + 4.0f * t_k_1 * t_k_1)) / 2.0f;                   // :372
        for (size_t i = 0; i < NO_VOXEL; i++) {                                          // :375-381
            F_Y_k[i] = F_recon[i] + (t_k_1 - 1.0f) / t_k * (F_recon[i] - F_X_k_1[i]);
            F_X_k_1[i] = F_recon[i];
        }
        t_k_1 = t_k;
        Forward_3D_ray_driven_siddon(F_recon.data(), proj_forward.data());              // :405
        const double data_fidelity = L2_norm_gpu(proj_forward.data(), h_proj_data.data());   // :407
        const double tv_value = TV_norm_gpu(F_recon.data());                             // :417
        const char* err = ctr_last_error_string();
        if (err && err[0]) {
            std::fprintf(stderr, "ctrecon: %s\n", err);
            return 1;
        }
        std::printf("%d %.17g %.17g %.17g\n", k, tv_value, data_fidelity,
                    data_fidelity + 2.0 * (double)lambda_TV * tv_value);                // :423
    }
    fp = std::fopen(argv[16], "wb");
    if (!fp || std::fwrite(F_X_k_1.data(), sizeof(float), NO_VOXEL, fp) != NO_VOXEL) return 1;
    std::fclose(fp);
    return 0;
}
