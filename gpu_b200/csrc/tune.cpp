// tune.cpp -- launch shapes of the SART projectors and their tuner.
//
// The forward projector runs 32 x {2, 4, 8} rays per block, with plane
// coordinates read from shared memory or computed; the SART backprojector
// runs either the fixed-shape kernel (8 voxels of a column per thread) or the
// column walk with {4, 8} voxel rows per block, a z run of {8, 32, 128}
// voxels, registers capped for 8 or 10 blocks per SM, and one or two detector
// rows per batch of loads.  Every shape computes each ray and each voxel with
// the same operations in the same order, so the shape changes the speed and
// never the result.  ctr_geometry_autotune times each shape on a few views
// spread over the scan and keeps the fastest, on the tiled layout the solver
// projects (CTR_SART_TILED).
#include <cstring>
#include <vector>

#include "ctr_internal.h"

using namespace ctr;

namespace {

Geometry* GE(const ctr_geometry* g) { return reinterpret_cast<Geometry*>(const_cast<ctr_geometry*>(g)); }

struct Events {
    std::vector<cudaEvent_t> e;
    explicit Events(size_t n) : e(n, nullptr) {}
    ~Events()
    {
        for (auto x : e)
            if (x) cudaEventDestroy(x);
    }
    ctr_status create()
    {
        for (auto& x : e) CTR_CUDA_TRY(cudaEventCreate(&x));
        return CTR_OK;
    }
};

struct DevMem {
    void* p = nullptr;
    ~DevMem() { cudaFree(p); }
};

ctr_status fp_sart(Geometry* g, void* vol, ctr_dtype vdt, const float* view_sino, int j, cudaStream_t st,
                   bool tiled = true)
{
    FpArgs a{};
    a.vol = vol; a.vol_dtype = vdt; a.view0 = j; a.nview = 1; a.kind = FP_SART; a.tiled = tiled;
    a.out = g->d_rays; a.b = view_sino; a.b_dtype = CTR_F32;
    return launch_forward(*g, a, st, nullptr);
}

ctr_status bp_sart(Geometry* g, void* vol, ctr_dtype vdt, int j, cudaStream_t st, bool tiled = true)
{
    BpArgs b{};
    b.vol = vol; b.vol_dtype = vdt; b.rays = g->d_rays; b.view0 = j; b.nview = 1; b.sart = 1; b.beta = 0.5f;
    b.tiled = tiled;
    return launch_backproject(*g, b, st);
}

}  // namespace

extern "C" ctr_status ctr_geometry_set_shapes(ctr_geometry* geom, int fp_shape, int bp_shape)
{
    clear_error();
    if (!geom) return set_error(CTR_ERR_INVALID_ARGUMENT, "geometry is NULL");
    if (fp_shape < 0 || fp_shape >= FP_SHAPES) return set_error(CTR_ERR_INVALID_ARGUMENT, "fp_shape %d out of range", fp_shape);
    if (bp_shape < -1 || bp_shape >= BP_SHAPES) return set_error(CTR_ERR_INVALID_ARGUMENT, "bp_shape %d out of range", bp_shape);
    Geometry* g = GE(geom);
    g->fp_shape = fp_shape;
    g->bp_shape = bp_shape;
    return CTR_OK;
}

extern "C" ctr_status ctr_geometry_get_shapes(const ctr_geometry* geom, int* fp_shape, int* bp_shape)
{
    clear_error();
    if (!geom) return set_error(CTR_ERR_INVALID_ARGUMENT, "geometry is NULL");
    if (fp_shape) *fp_shape = GE(geom)->fp_shape;
    if (bp_shape) *bp_shape = GE(geom)->bp_shape;
    return CTR_OK;
}

extern "C" ctr_status ctr_geometry_autotune(ctr_geometry* geom, ctr_dtype vdt, int n_views, float* fp_ms,
                                            float* bp_ms, void* stream)
{
    clear_error();
    if (!geom) return set_error(CTR_ERR_INVALID_ARGUMENT, "geometry is NULL");
    if (vdt != CTR_F32 && vdt != CTR_BF16 && vdt != CTR_F16) return set_error(CTR_ERR_INVALID_ARGUMENT, "bad vol_dtype");
    Geometry* g = GE(geom);
    if (n_views < 1 || n_views > g->desc.n_views)
        return set_error(CTR_ERR_INVALID_ARGUMENT, "n_views must be in [1, %d]", g->desc.n_views);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t P = (size_t)g->npix();
    CTR_TRY(ensure_rays(g, P * sizeof(float2)));
    DevMem vol, sino;
    const size_t vbytes = (size_t)tiled_count(g->dg) * dtype_size(vdt);   // tiled (>= linear)
    CTR_CUDA_TRY(cudaMalloc(&vol.p, vbytes));
    CTR_CUDA_TRY(cudaMalloc(&sino.p, P * sizeof(float)));
    CTR_CUDA_TRY(cudaMemsetAsync(vol.p, 0, vbytes, st));
    CTR_CUDA_TRY(cudaMemsetAsync(sino.p, 0, P * sizeof(float), st));
    const float* view_sino = (const float*)sino.p;
    std::vector<int> views(n_views);
    // spread over the scan, off the axis-aligned angles where rays run along the planes
    for (int q = 0; q < n_views; ++q) views[q] = (int)(((double)q + 0.3) * g->desc.n_views / n_views);
    Events ev(2 * (size_t)n_views);
    CTR_TRY(ev.create());
    auto elapsed = [&](float& total) -> ctr_status {
        CTR_CUDA_TRY(cudaStreamSynchronize(st));
        total = 0.f;
        for (int q = 0; q < n_views; ++q) {
            float t = 0.f;
            CTR_CUDA_TRY(cudaEventElapsedTime(&t, ev.e[2 * q], ev.e[2 * q + 1]));
            total += t;
        }
        total /= (float)n_views;
        return CTR_OK;
    };
    const int fp0 = g->fp_shape, bp0 = g->bp_shape;
    ctr_status r = CTR_OK;

    // forward projector shapes (the SART kind: the ray sums and chords)
    int best_fp = fp0;
    float best_t = 0.f;
    for (int s = 0; s < FP_SHAPES && r == CTR_OK; ++s) {
        g->fp_shape = s;
        r = fp_sart(g, vol.p, vdt, view_sino, views[0], st);   // warm-up
        for (int q = 0; q < n_views && r == CTR_OK; ++q) {
            if (cudaEventRecord(ev.e[2 * q], st) != cudaSuccess) r = set_error(CTR_ERR_CUDA, "cudaEventRecord");
            if (r == CTR_OK) r = fp_sart(g, vol.p, vdt, view_sino, views[q], st);
            if (r == CTR_OK && cudaEventRecord(ev.e[2 * q + 1], st) != cudaSuccess) r = set_error(CTR_ERR_CUDA, "cudaEventRecord");
        }
        float t = 0.f;
        if (r == CTR_OK) r = elapsed(t);
        if (r == CTR_OK) {
            if (fp_ms) fp_ms[s] = t;
            if (s == 0 || t < best_t) { best_t = t; best_fp = s; }
        }
    }
    if (r == CTR_OK) g->fp_shape = best_fp;

    // SART backprojector shapes.  Index 0 of bp_ms is the fixed-shape kernel,
    // which serves the linear layout only: timed there for reference, never
    // chosen; the column walks are timed on the tiled layout.
    int best_bp = bp0;
    for (int s = -1; s < BP_SHAPES && r == CTR_OK; ++s) {
        const bool tl = s >= 0;
        g->bp_shape = s;
        r = fp_sart(g, vol.p, vdt, view_sino, views[0], st, tl);
        if (r == CTR_OK) r = bp_sart(g, vol.p, vdt, views[0], st, tl);   // warm-up
        for (int q = 0; q < n_views && r == CTR_OK; ++q) {
            r = fp_sart(g, vol.p, vdt, view_sino, views[q], st, tl);
            if (r == CTR_OK && cudaEventRecord(ev.e[2 * q], st) != cudaSuccess) r = set_error(CTR_ERR_CUDA, "cudaEventRecord");
            if (r == CTR_OK) r = bp_sart(g, vol.p, vdt, views[q], st, tl);
            if (r == CTR_OK && cudaEventRecord(ev.e[2 * q + 1], st) != cudaSuccess) r = set_error(CTR_ERR_CUDA, "cudaEventRecord");
        }
        float t = 0.f;
        if (r == CTR_OK) r = elapsed(t);
        if (r == CTR_OK) {
            if (bp_ms) bp_ms[s + 1] = t;
            if (s == 0 || (s > 0 && t < best_t)) { best_t = t; best_bp = s; }
        }
    }
    if (r == CTR_OK) {
        g->bp_shape = best_bp;
    } else {
        g->fp_shape = fp0;
        g->bp_shape = bp0;
    }
    return r;
}
