// fp.cu -- the forward projector's launcher and the matched adjoint's ray
// records.  The kernels are templates in fp_kernels.cuh, instantiated per
// storage type in fp_f32.cu, fp_bf16.cu and fp_f16.cu.
#include "fp_kernels.cuh"

namespace ctr {

ctr_status launch_forward(const Geometry& G, const FpArgs& a, cudaStream_t st, size_t* nblocks_out)
{
    static_assert(kFpShapes[1].rows == FP_BY && kFpShapes[1].cpm == 0, "shape 1 is the fixed shape");
    const DevGeom& g = G.dg;
    if (a.nview <= 0) return CTR_OK;
    if (a.nview > 65535) return set_error(CTR_ERR_INVALID_ARGUMENT, "too many views in one launch");
    const bool refine = a.kind == FP_SART_REFINE || a.kind == FP_SART_REFINE32;
    if (a.tiled && a.kind != FP_SART && a.kind != FP_OBJECTIVE && a.kind != FP_SART_OBJ && a.kind != FP_PARTIAL &&
        !refine)
        return set_error(CTR_ERR_UNSUPPORTED, "the tiled layout is for SART and objective projections");
    if (a.kind == FP_SART_REFINE32 && !a.tiled)
        return set_error(CTR_ERR_UNSUPPORTED, "SART_REFINE32 takes tiled volumes");
    if (a.kind == FP_SART_OBJ && !a.vol2) return set_error(CTR_ERR_INVALID_ARGUMENT, "SART_OBJ needs vol2");
    if (refine && (!a.vol2 || !a.ax || !a.gdev || !a.partial))
        return set_error(CTR_ERR_INVALID_ARGUMENT, "SART_REFINE needs vol2, ax, gdev and partial");
    // the dot product keeps the fixed shape: its block partial sums, and so
    // the rounding of the total, do not depend on the tuned shape
    if (nblocks_out)
        *nblocks_out = (a.kind == FP_OBJECTIVE || a.kind == FP_SART_OBJ || refine)
                           ? objective_partials_per_view(g) * a.nview
                           : (size_t)((g.R + FP_BX - 1) / FP_BX) * ((g.ZP + FP_BY - 1) / FP_BY) * a.nview;
    const size_t smem = plane_tables_bytes(g);
    switch (a.vol_dtype) {
    case CTR_F32: launch_forward_f32(G, a, smem, st); break;
    case CTR_BF16: launch_forward_bf16(G, a, smem, st); break;
    case CTR_F16: launch_forward_f16(G, a, smem, st); break;
    default: return set_error(CTR_ERR_INVALID_ARGUMENT, "bad dtype %d", (int)a.vol_dtype);
    }
    CTR_CUDA_TRY(cudaGetLastError());
    return CTR_OK;
}

// Ray records for the matched adjoint: the value, the chord length d12 (:290),
// the alpha interval the forward traversal covers, the voxel it starts in and
// the axes it treats as parallel.  With these the gather backprojector
// reproduces the traversal's own cell intervals, so it stays the exact
// adjoint where the reference traversal drops a ray at a volume edge or
// starts a nearly axis-parallel ray one cell over.
template <bool E64>
__global__ void __launch_bounds__(FP_THREADS)
k_ray_prep(const DevGeom g, const float* __restrict__ y, int view0, AdjRay* __restrict__ rays)
{
    extern __shared__ float sp[];
    float* PX;
    float* PY;
    float* PZ;
    float* PINF;
    plane_tables_layout(g, sp, PX, PY, PZ, PINF);
    for (int t = threadIdx.x; t < g.M + 3; t += FP_THREADS) PX[t] = g.px[t];
    for (int t = threadIdx.x; t < g.N + 3; t += FP_THREADS) PY[t] = g.py[t];
    for (int t = threadIdx.x; t < g.Z + 3; t += FP_THREADS) PZ[t] = g.pz[t];
    if (threadIdx.x == 0) PINF[0] = __int_as_float(0x7f800000);
    __syncthreads();
    const int u = blockIdx.x * FP_BX + (threadIdx.x % FP_BX);
    const int v = blockIdx.y * FP_BY + (threadIdx.x / FP_BX);
    const int w = blockIdx.z;
    if (u >= g.R || v >= g.ZP) return;
    const float2 sc = g.trig[view0 + w];
    const RayResult rr = siddon<float, E64, false, false>(g, PX, PY, PZ, PINF, nullptr, sc.x, sc.y, u, v);
    const long long p = ((long long)w * g.ZP + v) * g.R + u;
    AdjRay a;
    a.f = make_float4(y[p], rr.d12, rr.a_lo, rr.a_hi);
    a.i = make_int4(rr.vi0, rr.vj0, rr.vk0, rr.par);
    rays[p] = a;
}

ctr_status launch_ray_prep(const Geometry& G, const float* y, int view0, int nview, AdjRay* rays, cudaStream_t st)
{
    const DevGeom& g = G.dg;
    if (nview <= 0) return CTR_OK;
    dim3 grid((g.R + FP_BX - 1) / FP_BX, (g.ZP + FP_BY - 1) / FP_BY, nview);
    const size_t smem = plane_tables_bytes(g);
    if (g.entry64) k_ray_prep<true><<<grid, FP_THREADS, smem, st>>>(g, y, view0, rays);
    else k_ray_prep<false><<<grid, FP_THREADS, smem, st>>>(g, y, view0, rays);
    CTR_CUDA_TRY(cudaGetLastError());
    return CTR_OK;
}

}  // namespace ctr
