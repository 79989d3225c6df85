// slabs.cu -- the combination step of the multi-GPU build's z-slab SART.
//
// Per view the reference's multi-GPU build (V63/host_IterativeRecon_CBCT_
// multiGPU.c:69-118) has every device project its z-slab of the volume into
// partial ray sums (Sum(len*f), Sum(len)) without threshold, adds the parts on
// the host in device order starting from zero (kernel_add_proj, twice per
// device), and divides (kernel_divide_proj,
// V63/kernel_IterativeRecon_universal_multiGPU.cu:1-19) before each device
// backprojects the one correction into its slab.  k_combine is that host
// step on the device: it reads the D parts of a ray -- gathered into one
// [D][P] buffer by the exchange, or the slabs' own outputs on one GPU -- adds
// them in slab order with the reference's float operations, and writes the
// ray record the backprojectors read: (correction, d12).
#include "ctr_device.cuh"

namespace ctr {

// b == nullptr: only the weighted sums, as floats into rays (the multi-GPU
// CheckMatchedJointOperator's y, V63/host_IterativeRecon_CBCT_multiGPU.c:368-376)
__global__ void k_combine(const DevGeom g, const float2* __restrict__ parts, int n_parts, long long P, int view,
                          const void* __restrict__ b, int b_dt, float2* __restrict__ rays)
{
    const float2 sc = g.trig[view];
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
        float w = 0.0f, l = 0.0f;                          // memset(h_proj_*, 0), multiGPU.c:82-83
        for (int i = 0; i < n_parts; ++i) {                // kernel_add_proj per device in order, :86-91
            const float2 t = __ldg(parts + (long long)i * P + p);
            w = fa(w, t.x);
            l = fa(l, t.y);
        }
        if (!b) {
            reinterpret_cast<float*>(rays)[p] = w;
            continue;
        }
        // kernel_divide_proj: 0 below volumn_z*1e-6f (T42: 1e-3f), else (b - w)*1.0f/l (x*1.0f is x)
        const float corr = l < g.thr_comb ? 0.0f : fdv(fs(ld_any(b, p, b_dt), w), l);
        const int v = (int)(p / g.R), u = (int)(p - (long long)v * g.R);
        rays[p] = make_float2(corr, ray_d12(ray_ends(g, sc.x, sc.y, u, v)));
    }
}

ctr_status launch_combine(const Geometry& G, const float2* parts, int n_parts, int view, const void* b,
                          ctr_dtype b_dt, float2* rays, cudaStream_t st)
{
    const long long P = (long long)G.dg.R * G.dg.ZP;
    const int blocks = (int)std::min<long long>((P + 255) / 256, 148LL * 8);
    k_combine<<<blocks, 256, 0, st>>>(G.dg, parts, n_parts, P, view, b, (int)b_dt, rays);
    CTR_CUDA_TRY(cudaGetLastError());
    return CTR_OK;
}

}  // namespace ctr
