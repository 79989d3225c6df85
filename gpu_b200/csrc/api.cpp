// api.cpp -- the C ABI: argument checks, drivers for the reference's call
// sequence (SART pass, SART+FISTA+TV iteration, FDK, objective) and the
// reference-compatible host entry points.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>

#include "ctr_internal.h"

using namespace ctr;

namespace {

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }
inline Geometry* GE(const ctr_geometry* g) { return const_cast<Geometry*>(reinterpret_cast<const Geometry*>(g)); }

ctr_status check_views(const Geometry* g, int v0, int n)
{
    if (v0 < 0 || n < 0 || (long long)v0 + n > g->desc.n_views)
        return set_error(CTR_ERR_INVALID_ARGUMENT, "view range [%d, %d) outside [0, %d)", v0, v0 + n, g->desc.n_views);
    return CTR_OK;
}

ctr_status need(const void* p, const char* what)
{
    if (!p) return set_error(CTR_ERR_INVALID_ARGUMENT, "%s is NULL", what);
    return CTR_OK;
}

ctr_status need_dtype(int dt, const char* what)
{
    if (!dtype_ok(dt)) return set_error(CTR_ERR_INVALID_ARGUMENT, "%s: unknown dtype %d", what, dt);
    return CTR_OK;
}

// views per adjoint pass: bounded so the ray records stay under ~256 MB
int adjoint_batch(const Geometry* g)
{
    long long b = (256LL << 20) / ((long long)sizeof(AdjRay) * g->npix());
    if (b < 1) b = 1;
    if (b > 32) b = 32;
    return (int)b;
}

// forward over [v0, v0+n) in launches of at most 65535 views
ctr_status forward_chunks(Geometry* g, FpArgs a, cudaStream_t st)
{
    const long long P = g->npix();
    const int v0 = a.view0, n = a.nview;
    for (int c = 0; c < n; c += 65535) {
        FpArgs b = a;
        b.view0 = v0 + c;
        b.nview = std::min(65535, n - c);
        if (a.out) b.out = (char*)a.out + (size_t)c * P * (a.kind == FP_SART ? sizeof(float2) : dtype_size(a.out_dtype));
        if (a.b) b.b = (const char*)a.b + (size_t)c * P * dtype_size(a.b_dtype);
        CTR_TRY(launch_forward(*g, b, st, nullptr));
    }
    return CTR_OK;
}

// SART pass: per view FP command 1 -> ray records, then BP command 1.
// With ev (3 events per view) the launches are bracketed for timing.
// With tiled (a scratch of tiled_count elements) the views run on an 8x8-tiled
// copy of the volume, copied in before and out after; the result is the same.
// With obj_tiled (a tiled volume) each view's forward projection also writes
// the objective partials of that volume, [view][row][u/32] into obj_partial:
// the objective's projection rides on the SART traversal.
ctr_status sart_views(Geometry* g, void* vol, ctr_dtype vdt, const void* sino, ctr_dtype sdt, float beta,
                      unsigned flags, uint32_t seed, int v0, int nv, cudaStream_t st, cudaEvent_t* ev,
                      const uint32_t* pass_seed = nullptr, void* tiled = nullptr, const void* obj_tiled = nullptr,
                      double* obj_partial = nullptr)
{
    if (obj_tiled && (!tiled || !obj_partial)) return set_error(CTR_ERR_INVALID_ARGUMENT, "fused objective needs tiled");
    const size_t per_view = objective_partials_per_view(g->dg);
    const long long P = g->npix();
    CTR_TRY(ensure_rays(g, (size_t)P * sizeof(float2)));
    void* pv = tiled ? tiled : vol;
    if (tiled) CTR_TRY(launch_tiling(*g, vol, tiled, vdt, true, st));
    for (int j = v0; j < v0 + nv; ++j) {
        if (ev) CTR_CUDA_TRY(cudaEventRecord(ev[3 * (j - v0)], st));
        FpArgs a{};
        a.vol = pv; a.vol_dtype = vdt; a.view0 = j; a.nview = 1; a.kind = FP_SART; a.tiled = tiled != nullptr;
        a.out = g->d_rays; a.b = (const char*)sino + (size_t)j * P * dtype_size(sdt); a.b_dtype = sdt;
        if (obj_tiled) {
            a.kind = FP_SART_OBJ;
            a.vol2 = obj_tiled;
            a.partial = obj_partial + (size_t)j * per_view;
        }
        CTR_TRY(launch_forward(*g, a, st, nullptr));
        if (ev) CTR_CUDA_TRY(cudaEventRecord(ev[3 * (j - v0) + 1], st));
        BpArgs b{};
        b.vol = pv; b.vol_dtype = vdt; b.rays = g->d_rays; b.view0 = j; b.nview = 1; b.sart = 1;
        b.flags = flags; b.beta = beta; b.seed = seed * 0x9E3779B9u + (uint32_t)j; b.pass_seed = pass_seed;
        b.tiled = tiled != nullptr;
        CTR_TRY(launch_backproject(*g, b, st));
        if (ev) CTR_CUDA_TRY(cudaEventRecord(ev[3 * (j - v0) + 2], st));
    }
    if (tiled) CTR_TRY(launch_tiling(*g, tiled, vol, vdt, false, st));
    return CTR_OK;
}

ctr_status sart_pass(Geometry* g, void* vol, ctr_dtype vdt, const void* sino, ctr_dtype sdt, float beta,
                     unsigned flags, uint32_t seed, cudaStream_t st, const uint32_t* pass_seed = nullptr,
                     void* tiled = nullptr, const void* obj_tiled = nullptr, double* obj_partial = nullptr)
{
    return sart_views(g, vol, vdt, sino, sdt, beta, flags, seed, 0, g->desc.n_views, st, nullptr, pass_seed, tiled,
                      obj_tiled, obj_partial);
}

// Fidelity ||A x - b||^2 (FP64 partials per warp of 32 rays, summed in index
// order by a two-level reduction) and TV of x.  With tiled, the projection
// reads an 8x8-tiled copy of x made there.
ctr_status objective_async(Geometry* g, const void* vol, ctr_dtype vdt, const void* sino, ctr_dtype sdt,
                           double* d_fid, double* d_tv, cudaStream_t st, void* tiled = nullptr)
{
    const DevGeom& q = g->dg;
    const size_t per_view = objective_partials_per_view(q);
    const size_t nblk = per_view * g->desc.n_views;
    const size_t tvcap = 148 * 64;
    CTR_TRY(ensure_partial(g, std::max(nblk, tvcap) + 2048));
    if (d_fid) {
        if (tiled) CTR_TRY(launch_tiling(*g, vol, tiled, vdt, true, st));
        FpArgs a{};
        a.vol = tiled ? tiled : vol; a.vol_dtype = vdt; a.view0 = 0; a.nview = g->desc.n_views;
        a.kind = FP_OBJECTIVE; a.tiled = tiled != nullptr;
        a.b = sino; a.b_dtype = sdt; a.partial = g->d_partial;
        const long long P = g->npix();
        for (int c = 0; c < g->desc.n_views; c += 65535) {
            FpArgs b = a;
            b.view0 = c;
            b.nview = std::min(65535, g->desc.n_views - c);
            b.b = (const char*)sino + (size_t)c * P * dtype_size(sdt);
            b.partial = g->d_partial + (size_t)c * per_view;
            CTR_TRY(launch_forward(*g, b, st, nullptr));
        }
        CTR_TRY(launch_reduce(g->d_partial, nblk, d_fid, st));
    }
    if (d_tv) CTR_TRY(launch_tv(*g, vol, vdt, g->d_partial, tvcap, d_tv, st));
    return CTR_OK;
}

}  // namespace

// ------------------------------------------------------------------ projectors

extern "C" ctr_status ctr_forward(const ctr_geometry* geom, const void* vol, ctr_dtype vdt, void* sino,
                                  ctr_dtype sdt, int v0, int n, void* stream)
{
    clear_error();
    CTR_TRY(need(geom, "geometry"));
    CTR_TRY(need(vol, "vol"));
    CTR_TRY(need(sino, "sino"));
    CTR_TRY(need_dtype(vdt, "vol_dtype"));
    CTR_TRY(need_dtype(sdt, "sino_dtype"));
    Geometry* g = GE(geom);
    CTR_TRY(check_views(g, v0, n));
    FpArgs a{};
    a.vol = vol; a.vol_dtype = vdt; a.view0 = v0; a.nview = n; a.kind = FP_FORWARD; a.out = sino; a.out_dtype = sdt;
    return forward_chunks(g, a, S(stream));
}

extern "C" ctr_status ctr_backproject(const ctr_geometry* geom, const float* sino, int v0, int n, void* vol,
                                      ctr_dtype vdt, unsigned flags, void* stream)
{
    clear_error();
    CTR_TRY(need(geom, "geometry"));
    CTR_TRY(need(sino, "sino"));
    CTR_TRY(need(vol, "vol"));
    CTR_TRY(need_dtype(vdt, "vol_dtype"));
    Geometry* g = GE(geom);
    CTR_TRY(check_views(g, v0, n));
    cudaStream_t st = S(stream);
    const long long P = g->npix();
    const bool masked = (flags & CTR_BP_FOV_MASK) != 0;
    const int batch = masked ? 1 : adjoint_batch(g);
    if (n == 0) {
        if (!(flags & CTR_BP_ACCUMULATE)) CTR_CUDA_TRY(cudaMemsetAsync(vol, 0, g->nvox() * dtype_size(vdt), st));
        return CTR_OK;
    }
    CTR_TRY(ensure_rays(g, (size_t)P * batch * sizeof(AdjRay)));
    for (int c = 0; c < n; c += batch) {
        const int cnt = std::min(batch, n - c);
        CTR_TRY(launch_ray_prep(*g, sino + (size_t)c * P, v0 + c, cnt, (AdjRay*)g->d_rays, st));
        BpArgs b{};
        b.vol = vol; b.vol_dtype = vdt; b.rays = g->d_rays; b.view0 = v0 + c; b.nview = cnt; b.sart = 0;
        b.flags = (flags & CTR_BP_FOV_MASK) | ((c > 0 || (flags & CTR_BP_ACCUMULATE)) ? CTR_BP_ACCUMULATE : 0u);
        CTR_TRY(launch_backproject(*g, b, st));
    }
    return CTR_OK;
}

extern "C" ctr_status ctr_sart_pass(const ctr_geometry* geom, void* vol, ctr_dtype vdt, const void* sino,
                                    ctr_dtype sdt, float beta, unsigned flags, uint32_t seed, void* stream)
{
    clear_error();
    CTR_TRY(need(geom, "geometry"));
    CTR_TRY(need(vol, "vol"));
    CTR_TRY(need(sino, "sino"));
    CTR_TRY(need_dtype(vdt, "vol_dtype"));
    CTR_TRY(need_dtype(sdt, "sino_dtype"));
    if (!std::isfinite(beta)) return set_error(CTR_ERR_INVALID_ARGUMENT, "beta must be finite");
    Geometry* g = GE(geom);
    void* tiled = nullptr;
    if (flags & CTR_SART_TILED) {
        CTR_TRY(ensure_tiled(g, (size_t)tiled_count(g->dg) * dtype_size(vdt)));
        tiled = g->d_tiled;
    }
    return sart_pass(g, vol, vdt, sino, sdt, beta, flags, seed, S(stream), nullptr, tiled);
}

extern "C" ctr_status ctr_sart_views(const ctr_geometry* geom, void* vol, ctr_dtype vdt, const void* sino,
                                     ctr_dtype sdt, float beta, unsigned flags, uint32_t seed, int v0, int n,
                                     float* fp_ms, float* bp_ms, void* stream)
{
    clear_error();
    CTR_TRY(need(geom, "geometry"));
    CTR_TRY(need(vol, "vol"));
    CTR_TRY(need(sino, "sino"));
    CTR_TRY(need_dtype(vdt, "vol_dtype"));
    CTR_TRY(need_dtype(sdt, "sino_dtype"));
    Geometry* g = GE(geom);
    CTR_TRY(check_views(g, v0, n));
    if (!std::isfinite(beta)) return set_error(CTR_ERR_INVALID_ARGUMENT, "beta must be finite");
    cudaStream_t st = S(stream);
    void* tiled = nullptr;
    if (flags & CTR_SART_TILED) {
        CTR_TRY(ensure_tiled(g, (size_t)tiled_count(g->dg) * dtype_size(vdt)));
        tiled = g->d_tiled;
    }
    if (!fp_ms && !bp_ms)
        return sart_views(g, vol, vdt, sino, sdt, beta, flags, seed, v0, n, st, nullptr, nullptr, tiled);
    std::vector<cudaEvent_t> ev(3 * (size_t)n, nullptr);
    ctr_status r = CTR_OK;
    for (auto& e : ev)
        if (r == CTR_OK && cudaEventCreate(&e) != cudaSuccess) r = set_error(CTR_ERR_CUDA, "cudaEventCreate");
    if (r == CTR_OK) r = sart_views(g, vol, vdt, sino, sdt, beta, flags, seed, v0, n, st, ev.data(), nullptr, tiled);
    if (r == CTR_OK && cudaStreamSynchronize(st) != cudaSuccess) r = set_error(CTR_ERR_CUDA, "cudaStreamSynchronize");
    float tf = 0.f, tb = 0.f;
    for (int j = 0; r == CTR_OK && j < n; ++j) {
        float a = 0.f, b = 0.f;
        cudaEventElapsedTime(&a, ev[3 * j], ev[3 * j + 1]);
        cudaEventElapsedTime(&b, ev[3 * j + 1], ev[3 * j + 2]);
        tf += a;
        tb += b;
    }
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    if (fp_ms) *fp_ms = tf;
    if (bp_ms) *bp_ms = tb;
    return r;
}

extern "C" ctr_status ctr_forward_trace(const ctr_geometry* geom, const float* vol, int view, int* nseg,
                                        uint64_t* hash, float* len, void* stream)
{
    clear_error();
    CTR_TRY(need(geom, "geometry"));
    CTR_TRY(need(vol, "vol"));
    CTR_TRY(need(nseg, "nseg"));
    CTR_TRY(need(hash, "hash"));
    CTR_TRY(need(len, "len"));
    Geometry* g = GE(geom);
    CTR_TRY(check_views(g, view, 1));
    FpArgs a{};
    a.vol = vol; a.vol_dtype = CTR_F32; a.view0 = view; a.nview = 1; a.kind = FP_TRACE;
    a.nseg = nseg; a.hash = hash; a.len = len;
    return launch_forward(*g, a, S(stream), nullptr);
}

// ------------------------------------------------------------- TV and FISTA

// ------------------------------------------------ z-slab SART (multi-GPU build)

namespace {

ctr_status need_slab(const Geometry* g)
{
    if (g->dg.slab_n > 1) return set_error(CTR_ERR_UNSUPPORTED, "not for a slab geometry");
    return CTR_OK;
}

// the slab geometries of g (a whole-volume geometry) for an n-way split, built on first use
ctr_status slab_geoms(Geometry* g, int n, std::vector<Geometry*>& out)
{
    CTR_TRY(need_slab(g));
    if ((int)g->slab_geoms.size() != n) {
        for (Geometry* sg : g->slab_geoms) ctr_geometry_destroy(reinterpret_cast<ctr_geometry*>(sg));
        g->slab_geoms.clear();
        for (int i = 0; i < n; ++i) {
            ctr_geometry* sg = nullptr;
            const ctr_status st = ctr_geometry_create_slab(&g->desc, n, i, &sg);
            if (st != CTR_OK) {
                for (Geometry* q : g->slab_geoms) ctr_geometry_destroy(reinterpret_cast<ctr_geometry*>(q));
                g->slab_geoms.clear();
                return st;
            }
            g->slab_geoms.push_back(GE(sg));
        }
    }
    if (g->dg.ct_style == 3 && !g->split_geom) {
        // the tetrahedron beam's n-device build projects whole views with V63's
        // traversal rules (T42/voxel/kernel_IterativeRecon_TBCT_voxel_multiGPU.cu:22-576);
        // for the other scanners its row-split projector is the one-device one
        ctr_geometry* sg = nullptr;
        CTR_TRY(ctr_geometry_create_slab(&g->desc, n, -1, &sg));
        g->split_geom = GE(sg);
    }
    for (Geometry* sg : g->slab_geoms) {   // the parent's tuned launch shapes
        sg->fp_shape = g->fp_shape;
        sg->bp_shape = g->bp_shape;
    }
    if (g->split_geom) {
        g->split_geom->fp_shape = g->fp_shape;
        g->split_geom->bp_shape = g->bp_shape;
    }
    if ((int)g->slab_streams.size() != n || (int)g->slab_events.size() != n + 2) {   // also after a failed build
        for (cudaStream_t q : g->slab_streams) cudaStreamDestroy(q);
        for (cudaEvent_t e : g->slab_events) cudaEventDestroy(e);
        g->slab_streams.clear();
        g->slab_events.clear();
        for (int i = 0; i < n; ++i) {
            cudaStream_t q = nullptr;
            CTR_CUDA_TRY(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking));
            g->slab_streams.push_back(q);
        }
        for (int i = 0; i < n + 2; ++i) {
            cudaEvent_t e = nullptr;
            CTR_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            g->slab_events.push_back(e);
        }
    }
    out = g->slab_geoms;
    return CTR_OK;
}

ctr_status ensure_parts(Geometry* g, size_t bytes)
{
    if (bytes <= g->parts_cap) return CTR_OK;
    if (g->d_parts) cudaFree(g->d_parts);
    g->d_parts = nullptr;
    g->parts_cap = 0;
    CTR_CUDA_TRY(cudaMalloc(&g->d_parts, bytes));
    g->parts_cap = bytes;
    return CTR_OK;
}

// Views [v0, v0+nv) of the D-slab SART on one GPU; pv the whole volume
// (linear or tiled).  The slabs are independent between the combinations --
// slab s's projection reads and its update writes only slab s -- so each
// slab runs on its own stream: its projection of view j, then (after the
// combination of view j on st, which waits for every slab's projection) its
// update, then its projection of view j+1.  A slab's short launches then
// share the GPU with the others' instead of running one after another.  The
// ray records and parts are safe to reuse: view j+1's combination waits for
// every slab's projection of j+1, each of which follows that slab's update
// of j.
ctr_status sart_views_slabs(Geometry* g, const std::vector<Geometry*>& sl, void* pv, ctr_dtype vdt, bool tiled,
                            const void* sino, ctr_dtype sdt, float beta, unsigned flags, uint32_t seed, int v0, int nv,
                            cudaStream_t st)
{
    const int D = (int)sl.size();
    const long long P = g->npix();
    const long long per_slab = tiled ? tiled_count(sl[0]->dg) : sl[0]->nvox();
    const size_t es = dtype_size(vdt);
    CTR_TRY(ensure_rays(g, (size_t)P * sizeof(float2)));
    CTR_TRY(ensure_parts(g, (size_t)P * D * sizeof(float2)));
    float2* parts = (float2*)g->d_parts;
    const std::vector<cudaStream_t>& ss = g->slab_streams;
    const std::vector<cudaEvent_t>& ev = g->slab_events;
    cudaEvent_t ev_comb = ev[D], ev_start = ev[D + 1];
    CTR_CUDA_TRY(cudaEventRecord(ev_start, st));
    for (int i = 0; i < D; ++i) CTR_CUDA_TRY(cudaStreamWaitEvent(ss[i], ev_start, 0));
    ctr_status r = CTR_OK;
    for (int j = v0; j < v0 + nv && r == CTR_OK; ++j) {
        for (int i = 0; i < D && r == CTR_OK; ++i) {   // multiGPU.c:71-75
            FpArgs a{};
            a.vol = (const char*)pv + (size_t)per_slab * i * es; a.vol_dtype = vdt; a.view0 = j; a.nview = 1;
            a.kind = FP_PARTIAL; a.out = parts + (size_t)P * i; a.tiled = tiled;
            r = launch_forward(*sl[i], a, ss[i], nullptr);
            if (r == CTR_OK && cudaEventRecord(ev[i], ss[i]) != cudaSuccess) r = set_error(CTR_ERR_CUDA, "cudaEventRecord");
            if (r == CTR_OK && cudaStreamWaitEvent(st, ev[i], 0) != cudaSuccess)
                r = set_error(CTR_ERR_CUDA, "cudaStreamWaitEvent");
        }
        if (r == CTR_OK)
            r = launch_combine(*g, parts, D, j, (const char*)sino + (size_t)j * P * dtype_size(sdt), sdt,
                               (float2*)g->d_rays, st);   // :82-95
        if (r == CTR_OK && cudaEventRecord(ev_comb, st) != cudaSuccess) r = set_error(CTR_ERR_CUDA, "cudaEventRecord");
        for (int i = 0; i < D && r == CTR_OK; ++i) {   // :103-112
            if (cudaStreamWaitEvent(ss[i], ev_comb, 0) != cudaSuccess) {
                r = set_error(CTR_ERR_CUDA, "cudaStreamWaitEvent");
                break;
            }
            BpArgs b{};
            b.vol = (char*)pv + (size_t)per_slab * i * es; b.vol_dtype = vdt; b.rays = g->d_rays; b.view0 = j;
            b.nview = 1; b.sart = 1; b.flags = flags; b.beta = beta; b.seed = seed * 0x9E3779B9u + (uint32_t)j;
            b.tiled = tiled;
            r = launch_backproject(*sl[i], b, ss[i]);
        }
    }
    // st resumes after every slab's last launch, also on an error
    for (int i = 0; i < D; ++i) {
        cudaEventRecord(ev[i], ss[i]);
        cudaStreamWaitEvent(st, ev[i], 0);
    }
    return r;
}

}  // namespace

extern "C" ctr_status ctr_forward_partial(const ctr_geometry* geom, const void* vol, ctr_dtype vdt, int view,
                                          float* part, unsigned flags, void* stream)
{
    clear_error();
    CTR_TRY(need(geom, "geometry"));
    CTR_TRY(need(vol, "vol"));
    CTR_TRY(need(part, "part"));
    CTR_TRY(need_dtype(vdt, "vol_dtype"));
    Geometry* g = GE(geom);
    CTR_TRY(check_views(g, view, 1));
    FpArgs a{};
    a.vol = vol; a.vol_dtype = vdt; a.view0 = view; a.nview = 1; a.kind = FP_PARTIAL; a.out = part;
    a.tiled = (flags & CTR_VOLUME_TILED) != 0;
    return launch_forward(*g, a, S(stream), nullptr);
}

extern "C" ctr_status ctr_combine_partials(const ctr_geometry* geom, const float* parts, int n_parts, int view,
                                           const void* b_view, ctr_dtype bdt, float* rays, void* stream)
{
    clear_error();
    CTR_TRY(need(geom, "geometry"));
    CTR_TRY(need(parts, "parts"));
    CTR_TRY(need(b_view, "b_view"));
    CTR_TRY(need(rays, "rays"));
    CTR_TRY(need_dtype(bdt, "b_dtype"));
    if (n_parts < 1) return set_error(CTR_ERR_INVALID_ARGUMENT, "n_parts must be >= 1");
    Geometry* g = GE(geom);
    CTR_TRY(check_views(g, view, 1));
    return launch_combine(*g, (const float2*)parts, n_parts, view, b_view, bdt, (float2*)rays, S(stream));
}

extern "C" ctr_status ctr_sart_update(const ctr_geometry* geom, void* vol, ctr_dtype vdt, const float* rays, int view,
                                      float beta, unsigned flags, uint32_t seed, void* stream)
{
    clear_error();
    CTR_TRY(need(geom, "geometry"));
    CTR_TRY(need(vol, "vol"));
    CTR_TRY(need(rays, "rays"));
    CTR_TRY(need_dtype(vdt, "vol_dtype"));
    if (!std::isfinite(beta)) return set_error(CTR_ERR_INVALID_ARGUMENT, "beta must be finite");
    Geometry* g = GE(geom);
    CTR_TRY(check_views(g, view, 1));
    BpArgs b{};
    b.vol = vol; b.vol_dtype = vdt; b.rays = rays; b.view0 = view; b.nview = 1; b.sart = 1;
    b.flags = flags & (CTR_SART_STOCHASTIC_ROUND | CTR_SART_REFERENCE_BP); b.beta = beta;
    b.seed = seed * 0x9E3779B9u + (uint32_t)view; b.tiled = (flags & CTR_VOLUME_TILED) != 0;
    CTR_TRY(launch_backproject(*g, b, S(stream)));
    return CTR_OK;
}

extern "C" ctr_status ctr_sart_pass_slabs(const ctr_geometry* geom, int n_slabs, void* vol, ctr_dtype vdt,
                                          const void* sino, ctr_dtype sdt, float beta, unsigned flags, uint32_t seed,
                                          int v0, int n, void* stream)
{
    clear_error();
    CTR_TRY(need(geom, "geometry"));
    CTR_TRY(need(vol, "vol"));
    CTR_TRY(need(sino, "sino"));
    CTR_TRY(need_dtype(vdt, "vol_dtype"));
    CTR_TRY(need_dtype(sdt, "sino_dtype"));
    if (!std::isfinite(beta)) return set_error(CTR_ERR_INVALID_ARGUMENT, "beta must be finite");
    if (n_slabs < 1) return set_error(CTR_ERR_INVALID_ARGUMENT, "n_slabs must be >= 1");
    Geometry* g = GE(geom);
    CTR_TRY(check_views(g, v0, n));
    std::vector<Geometry*> sl;
    CTR_TRY(slab_geoms(g, n_slabs, sl));
    cudaStream_t st = S(stream);
    const bool tiled = (flags & CTR_SART_TILED) != 0;
    void* pv = vol;
    if (tiled) {
        CTR_TRY(ensure_tiled(g, (size_t)tiled_count(g->dg) * dtype_size(vdt)));
        pv = g->d_tiled;
        CTR_TRY(launch_tiling(*g, vol, pv, vdt, true, st));
    }
    CTR_TRY(sart_views_slabs(g, sl, pv, vdt, tiled, sino, sdt, beta, flags & ~CTR_SART_TILED, seed, v0, n, st));
    if (tiled) CTR_TRY(launch_tiling(*g, pv, vol, vdt, false, st));
    return CTR_OK;
}

extern "C" ctr_status ctr_volume_tiling(const ctr_geometry* geom, const void* src, void* dst, ctr_dtype dt,
                                        int to_tiled, void* stream)
{
    clear_error();
    CTR_TRY(need(geom, "geometry"));
    CTR_TRY(need(src, "src"));
    CTR_TRY(need(dst, "dst"));
    CTR_TRY(need_dtype(dt, "dtype"));
    return launch_tiling(*GE(geom), src, dst, dt, to_tiled != 0, S(stream));
}

extern "C" ctr_status ctr_volume_tiled_count(const ctr_geometry* geom, int64_t* count)
{
    clear_error();
    CTR_TRY(need(geom, "geometry"));
    CTR_TRY(need(count, "count"));
    *count = tiled_count(GE(geom)->dg);
    return CTR_OK;
}


extern "C" ctr_status ctr_fgp_tv(const ctr_geometry* geom, void* vol, ctr_dtype dt, float lambda, int n_iter,
                                 void* stream)
{
    clear_error();
    CTR_TRY(need(geom, "geometry"));
    CTR_TRY(need(vol, "vol"));
    CTR_TRY(need_dtype(dt, "dtype"));
    if (!(lambda > 0.f) || !std::isfinite(lambda)) return set_error(CTR_ERR_INVALID_ARGUMENT, "lambda must be positive");
    if (n_iter < 0) return set_error(CTR_ERR_INVALID_ARGUMENT, "n_iter must be >= 0");
    return launch_fgp(*GE(geom), vol, dt, lambda, n_iter, nullptr, nullptr, 0.f, S(stream));
}

extern "C" ctr_status ctr_fista_momentum(const ctr_geometry* geom, void* y, void* xprev, const void* x,
                                         ctr_dtype dt, float t_prev, float t_k, void* stream)
{
    clear_error();
    CTR_TRY(need(geom, "geometry"));
    CTR_TRY(need(y, "y"));
    CTR_TRY(need(xprev, "x_prev"));
    CTR_TRY(need(x, "x"));
    CTR_TRY(need_dtype(dt, "dtype"));
    if (!(t_k != 0.f)) return set_error(CTR_ERR_INVALID_ARGUMENT, "t_k must be non-zero");
    const float gam = (t_prev - 1.0f) / t_k;
    return launch_momentum(*GE(geom), y, xprev, x, dt, gam, S(stream));
}

// ---------------------------------------------------------------- objective

extern "C" ctr_status ctr_objective(const ctr_geometry* geom, const void* vol, ctr_dtype vdt, const void* sino,
                                    ctr_dtype sdt, double* fid, double* tv, void* stream)
{
    clear_error();
    CTR_TRY(need(geom, "geometry"));
    CTR_TRY(need(vol, "vol"));
    CTR_TRY(need(sino, "sino"));
    CTR_TRY(need_dtype(vdt, "vol_dtype"));
    CTR_TRY(need_dtype(sdt, "sino_dtype"));
    Geometry* g = GE(geom);
    cudaStream_t st = S(stream);
    CTR_TRY(objective_async(g, vol, vdt, sino, sdt, g->d_result, g->d_result + 1, st));
    double h[2];
    CTR_CUDA_TRY(cudaMemcpyAsync(h, g->d_result, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CTR_TRY(check_device_errors(g, st));
    if (fid) *fid = h[0];
    if (tv) *tv = h[1];
    return CTR_OK;
}

extern "C" ctr_status ctr_tv_norm(const ctr_geometry* geom, const void* vol, ctr_dtype dt, double* out, void* stream)
{
    clear_error();
    CTR_TRY(need(geom, "geometry"));
    CTR_TRY(need(vol, "vol"));
    CTR_TRY(need(out, "out"));
    CTR_TRY(need_dtype(dt, "dtype"));
    Geometry* g = GE(geom);
    cudaStream_t st = S(stream);
    CTR_TRY(ensure_partial(g, 148 * 64 + 2048));
    CTR_TRY(launch_tv(*g, vol, dt, g->d_partial, 148 * 64, g->d_result, st));
    CTR_CUDA_TRY(cudaMemcpyAsync(out, g->d_result, sizeof(double), cudaMemcpyDeviceToHost, st));
    CTR_CUDA_TRY(cudaStreamSynchronize(st));
    return CTR_OK;
}

extern "C" ctr_status ctr_l2_norm(const float* a, const float* b, int64_t n, double* out, void* stream)
{
    clear_error();
    CTR_TRY(need(a, "a"));
    CTR_TRY(need(b, "b"));
    CTR_TRY(need(out, "out"));
    if (n < 0) return set_error(CTR_ERR_INVALID_ARGUMENT, "n < 0");
    cudaStream_t st = S(stream);
    double* buf = nullptr;
    const size_t cap = 148 * 64;
    CTR_CUDA_TRY(cudaMalloc(&buf, (cap + 2048 + 1) * sizeof(double)));
    ctr_status s = launch_l2(a, b, n, buf, cap, buf + cap + 2048, st);
    if (s == CTR_OK) {
        cudaError_t e = cudaMemcpyAsync(out, buf + cap + 2048, sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) s = cuda_error(e, "ctr_l2_norm");
    }
    cudaFree(buf);
    return s;
}

// --------------------------------------------------------------------- FDK

extern "C" ctr_status ctr_fdk(const ctr_geometry* geom, const float* sino, float* vol, void* stream)
{
    clear_error();
    CTR_TRY(need(geom, "geometry"));
    CTR_TRY(need(sino, "sino"));
    CTR_TRY(need(vol, "vol"));
    CTR_TRY(need_slab(GE(geom)));
    if (GE(geom)->dg.ct_style != 0) return set_error(CTR_ERR_UNSUPPORTED, "FDK is for the cone-beam geometry");
    return launch_fdk(*GE(geom), sino, vol, S(stream));
}

extern "C" ctr_status ctr_fdk_projector_frame(const ctr_geometry* geom, const float* sino, float* vol, void* stream)
{
    clear_error();
    CTR_TRY(need(geom, "geometry"));
    CTR_TRY(need(sino, "sino"));
    CTR_TRY(need(vol, "vol"));
    Geometry* g = GE(geom);
    CTR_TRY(need_slab(g));
    const ctr_geometry_desc& d = g->desc;
    if (g->dg.ct_style != 0) return set_error(CTR_ERR_UNSUPPORTED, "FDK is for the cone-beam geometry");
    if (d.nx != d.ny || g->dg.vx != g->dg.vy || d.m_offset != 0 || d.offset != 0.0f)
        return set_error(CTR_ERR_UNSUPPORTED, "the projector frame of FDK needs nx == ny, vx == vy and no offsets");
    // the FDK frame at angle +theta is the projector's frame at -theta with x and y exchanged
    cudaStream_t st = S(stream);
    CTR_TRY(launch_swap_xy(*g, vol, st));
    CTR_TRY(launch_fdk(*g, sino, vol, st));
    return launch_swap_xy(*g, vol, st);
}

extern "C" ctr_status ctr_fdk_backproject(const ctr_geometry* geom, const float* filtered, int v0, int n, float* vol,
                                          void* stream)
{
    clear_error();
    CTR_TRY(need(geom, "geometry"));
    CTR_TRY(need(filtered, "filtered"));
    CTR_TRY(need(vol, "vol"));
    Geometry* g = GE(geom);
    CTR_TRY(check_views(g, v0, n));
    CTR_TRY(need_slab(g));
    if (g->dg.ct_style != 0) return set_error(CTR_ERR_UNSUPPORTED, "FDK is for the cone-beam geometry");
    return launch_fdk_bp(*g, filtered, v0, n, vol, S(stream));
}

// -------------------------------------------------------------- dot product

extern "C" ctr_status ctr_dot_test(const ctr_geometry* geom, const float* x, const float* y, int v0, int n,
                                   double* ax_y, double* x_aty, void* stream)
{
    clear_error();
    CTR_TRY(need(geom, "geometry"));
    CTR_TRY(need(x, "x"));
    CTR_TRY(need(y, "y"));
    Geometry* g = GE(geom);
    CTR_TRY(check_views(g, v0, n));
    cudaStream_t st = S(stream);
    const long long V = g->nvox();
    const DevGeom& q = g->dg;
    const size_t per_view = (size_t)((q.R + 31) / 32) * ((q.ZP + 3) / 4);
    const size_t nblk = per_view * (n > 0 ? n : 1);
    const size_t cap = 148 * 64;
    CTR_TRY(ensure_partial(g, std::max(nblk, cap) + 2048));
    // <A x, y>: the projector's segments, each ray summed in FP64
    if (n > 0) {
        FpArgs a{};
        a.vol = x; a.vol_dtype = CTR_F32; a.view0 = v0; a.nview = n; a.kind = FP_DOT;
        a.b = y; a.b_dtype = CTR_F32; a.partial = g->d_partial;
        CTR_TRY(launch_forward(*g, a, st, nullptr));
        CTR_TRY(launch_reduce(g->d_partial, nblk, g->d_result, st));
    } else {
        CTR_CUDA_TRY(cudaMemsetAsync(g->d_result, 0, sizeof(double), st));
    }
    double h0 = 0.0;
    CTR_CUDA_TRY(cudaMemcpyAsync(&h0, g->d_result, sizeof(double), cudaMemcpyDeviceToHost, st));
    CTR_CUDA_TRY(cudaStreamSynchronize(st));
    // <x, A^T y>: the matched adjoint (FP64 accumulation, rounded to float per voxel)
    float* aty = nullptr;
    CTR_CUDA_TRY(cudaMalloc(&aty, sizeof(float) * (size_t)V));
    ctr_status s = ctr_backproject(geom, y, v0, n, aty, CTR_F32, 0, stream);
    if (s == CTR_OK) s = launch_dot(x, aty, V, g->d_partial, cap, g->d_result + 1, st);
    double h1 = 0.0;
    if (s == CTR_OK) {
        cudaError_t e = cudaMemcpyAsync(&h1, g->d_result + 1, sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) s = cuda_error(e, "cudaMemcpyAsync");
    }
    if (s == CTR_OK) s = check_device_errors(g, st);
    cudaFree(aty);
    if (s == CTR_OK) {
        if (ax_y) *ax_y = h0;
        if (x_aty) *x_aty = h1;
    }
    return s;
}

// ---------------------------------------------------------------- utilities

extern "C" ctr_status ctr_convert(const void* src, ctr_dtype sdt, void* dst, ctr_dtype ddt, int64_t n, void* stream)
{
    clear_error();
    CTR_TRY(need(src, "src"));
    CTR_TRY(need(dst, "dst"));
    CTR_TRY(need_dtype(sdt, "src_dtype"));
    CTR_TRY(need_dtype(ddt, "dst_dtype"));
    if (n < 0) return set_error(CTR_ERR_INVALID_ARGUMENT, "n < 0");
    if (n == 0) return CTR_OK;
    return launch_convert(src, sdt, dst, ddt, n, S(stream));
}

extern "C" ctr_status ctr_phantom_voxelize(const ctr_geometry* geom, const double* params, int n, float* vol,
                                           void* stream)
{
    clear_error();
    CTR_TRY(need(geom, "geometry"));
    CTR_TRY(need(vol, "vol"));
    if (n < 0 || (n > 0 && !params)) return set_error(CTR_ERR_INVALID_ARGUMENT, "bad ellipsoid list");
    for (int a = 0; a < n; ++a)
        for (int b = 3; b < 6; ++b)
            if (!(params[10 * a + b] > 0.0)) return set_error(CTR_ERR_INVALID_ARGUMENT, "ellipsoid %d: semi-axes must be > 0", a);
    if (n == 0) return CTR_OK;
    return launch_phantom(*GE(geom), params, n, vol, S(stream));
}

// ------------------------------------------------------------------ solver

struct ctr_solver {
    Geometry* g = nullptr;
    ctr_dtype vdt = CTR_F32;
    ctr_solver_params p{};
    const void* sino = nullptr;
    ctr_dtype sdt = CTR_F32;
    void* y = nullptr;       // working volume: y_k, then x_k during an iteration
    void* xprev = nullptr;   // x_(k-1); after an iteration with FISTA, x_k
    void* yt = nullptr;      // 8x8-tiled scratch copy for the projections
    void* xt = nullptr;      // 8x8-tiled copy of x_(k-1) for the objective fused into the SART pass
    float t = 1.0f;          // t_(k-1) of V63/main_recon.cu:177
    int k = 0;
    // SART pass: plain, with the fused objective, the refinement pass
    cudaGraph_t graph[3] = {nullptr, nullptr, nullptr};
    cudaGraphExec_t exec[3] = {nullptr, nullptr, nullptr};
    const void* graph_ws[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};   // workspaces captured with
    double* d_obj = nullptr; // [2] fid, tv
    // Objective history on the device, row k-1 = (fidelity, TV) of x_k.  The
    // objective of the latest x_k is "pending" until the next SART pass
    // projects it in the same traversal, or until someone asks for it.
    double* d_hist = nullptr;
    int hist_cap = 0;
    std::vector<unsigned char> hist_valid;
    bool obj_pending = false;
    int slabs = 1;           // > 1: the SART pass of the reference's slabs-device build (ctr_solver_set_slabs)
    // Refinement solver (p.refine): FP32 x_k and x_(k-1); xt is the 16-bit
    // copy of x_k the projectors read (tiled) and yt the correction volume d
    // (tiled); ax holds A x~ of the previous copy, one FP32 value per ray of
    // every view; gm is the FISTA factor of the coming pass (device: d_gm).
    bool refine = false;
    ctr_dtype ddt = CTR_F32;   // the correction volume's type: vol_dtype, or FP32 (refine = 2)
    float* xk32 = nullptr;
    float* xm32 = nullptr;
    float* ax = nullptr;
    float* d_gm = nullptr;
    float gm = 0.0f;
    // the FP64 reference solver (vol_dtype CTR_F64, f64.cu)
    F64Solver* f64 = nullptr;
};

extern "C" ctr_status ctr_solver_create(const ctr_geometry* geom, ctr_dtype vdt, const ctr_solver_params* p,
                                        ctr_solver** out)
{
    clear_error();
    CTR_TRY(need(geom, "geometry"));
    CTR_TRY(need(p, "params"));
    CTR_TRY(need(out, "out"));
    *out = nullptr;
    if (vdt != CTR_F64) CTR_TRY(need_dtype(vdt, "vol_dtype"));
    CTR_TRY(need_slab(GE(geom)));
    if (!std::isfinite(p->beta) || !std::isfinite(p->lambda_tv) || p->lambda_tv < 0.f || p->fgp_iters < 0)
        return set_error(CTR_ERR_INVALID_ARGUMENT, "bad solver parameters");
    if (p->refine < 0 || p->refine > 2) return set_error(CTR_ERR_INVALID_ARGUMENT, "refine must be 0, 1 or 2");
    ctr_solver* s = new (std::nothrow) ctr_solver();
    if (!s) return set_error(CTR_ERR_OUT_OF_MEMORY, "host allocation");
    s->g = GE(geom);
    s->vdt = vdt;
    s->p = *p;
    if (vdt == CTR_F64) {   // the FP64 reference solver
        ctr_status st = f64_create(s->g, *p, &s->f64);
        if (st != CTR_OK) {
            delete s;
            return st;
        }
        *out = s;
        return CTR_OK;
    }
    s->refine = p->refine != 0;
    s->ddt = p->refine == 2 ? CTR_F32 : vdt;
    const size_t bytes = s->g->nvox() * dtype_size(vdt);
    cudaError_t e;
    if (s->refine) {
        const size_t b32 = s->g->nvox() * sizeof(float);
        const size_t nax = (size_t)s->g->npix() * s->g->desc.n_views * sizeof(float);
        if ((e = cudaMalloc(&s->xk32, b32)) != cudaSuccess || (e = cudaMalloc(&s->xm32, b32)) != cudaSuccess ||
            (e = cudaMalloc(&s->ax, nax)) != cudaSuccess || (e = cudaMalloc(&s->d_gm, sizeof(float))) != cudaSuccess ||
            (e = cudaMemset(s->xk32, 0, b32)) != cudaSuccess || (e = cudaMemset(s->xm32, 0, b32)) != cudaSuccess ||
            (e = cudaMemset(s->ax, 0, nax)) != cudaSuccess || (e = cudaMemset(s->d_gm, 0, sizeof(float))) != cudaSuccess) {
            ctr_status st = cuda_error(e, "refinement solver allocation");
            ctr_solver_destroy(s);
            return st;
        }
    }
    if ((e = cudaMalloc(&s->y, bytes)) != cudaSuccess || (e = cudaMalloc(&s->xprev, bytes)) != cudaSuccess ||
        (e = cudaMalloc(&s->yt, (size_t)tiled_count(s->g->dg) * dtype_size(s->refine ? s->ddt : vdt))) != cudaSuccess ||
        (e = cudaMalloc(&s->xt, (size_t)tiled_count(s->g->dg) * dtype_size(vdt))) != cudaSuccess ||
        (e = cudaMalloc(&s->d_obj, 4 * sizeof(double))) != cudaSuccess || (e = cudaMemset(s->y, 0, bytes)) != cudaSuccess ||
        (e = cudaMemset(s->xprev, 0, bytes)) != cudaSuccess ||
        (e = cudaMemset(s->xt, 0, (size_t)tiled_count(s->g->dg) * dtype_size(vdt))) != cudaSuccess) {
        ctr_status st = cuda_error(e, "solver allocation");
        ctr_solver_destroy(s);
        return st;
    }
    *out = s;
    return CTR_OK;
}

static void drop_graph(ctr_solver* s)
{
    for (int i = 0; i < 3; ++i) {
        if (s->exec[i]) cudaGraphExecDestroy(s->exec[i]);
        if (s->graph[i]) cudaGraphDestroy(s->graph[i]);
        s->exec[i] = nullptr;
        s->graph[i] = nullptr;
    }
}

extern "C" ctr_status ctr_solver_destroy(ctr_solver* s)
{
    if (!s) return CTR_OK;
    drop_graph(s);
    cudaFree(s->y);
    cudaFree(s->xprev);
    cudaFree(s->yt);
    cudaFree(s->xt);
    cudaFree(s->d_obj);
    cudaFree(s->d_hist);
    cudaFree(s->xk32);
    cudaFree(s->xm32);
    cudaFree(s->ax);
    cudaFree(s->d_gm);
    if (s->f64) f64_destroy(s->f64);
    delete s;
    return CTR_OK;
}

static ctr_status flush_objective(ctr_solver* s, cudaStream_t st);

extern "C" ctr_status ctr_solver_set_sinogram(ctr_solver* s, const void* sino, ctr_dtype sdt)
{
    clear_error();
    CTR_TRY(need(s, "solver"));
    CTR_TRY(need(sino, "sino"));
    CTR_TRY(need_dtype(sdt, "sino_dtype"));
    if (s->sino != sino || s->sdt != sdt) {
        CTR_TRY(flush_objective(s, nullptr));   // the pending objective belongs to the old sinogram
        drop_graph(s);
    }
    s->sino = sino;
    s->sdt = sdt;
    return CTR_OK;
}

extern "C" ctr_status ctr_solver_set_volume(ctr_solver* s, const void* vol, void* stream)
{
    clear_error();
    CTR_TRY(need(s, "solver"));
    cudaStream_t st = S(stream);
    if (s->f64) return f64_set_volume(s->f64, (const double*)vol, st);
    const size_t bytes = s->g->nvox() * dtype_size(s->vdt);
    if (vol) {
        CTR_CUDA_TRY(cudaMemcpyAsync(s->y, vol, bytes, cudaMemcpyDefault, st));
        CTR_CUDA_TRY(cudaMemcpyAsync(s->xprev, vol, bytes, cudaMemcpyDefault, st));
    } else {
        CTR_CUDA_TRY(cudaMemsetAsync(s->y, 0, bytes, st));
        CTR_CUDA_TRY(cudaMemsetAsync(s->xprev, 0, bytes, st));
    }
    if (s->refine) {   // x_k = x_(k-1) = the estimate in FP32, its 16-bit copy, no previous projection
        const size_t b32 = s->g->nvox() * sizeof(float);
        CTR_TRY(launch_convert(s->y, s->vdt, s->xk32, CTR_F32, s->g->nvox(), st));
        CTR_CUDA_TRY(cudaMemcpyAsync(s->xm32, s->xk32, b32, cudaMemcpyDeviceToDevice, st));
        CTR_TRY(launch_tiling(*s->g, s->y, s->xt, s->vdt, true, st));
        CTR_CUDA_TRY(cudaMemsetAsync(s->ax, 0, (size_t)s->g->npix() * s->g->desc.n_views * sizeof(float), st));
        s->gm = 0.0f;
    }
    s->t = 1.0f;
    s->k = 0;
    s->obj_pending = false;
    s->hist_valid.clear();
    return CTR_OK;
}

// The refinement projection kind: the correction in the copies' type, or in
// FP32 (refine = 2) while the copies are 16-bit.
static FpKind refine_kind(const ctr_solver* s)
{
    return (s->ddt == CTR_F32 && s->vdt != CTR_F32) ? FP_SART_REFINE32 : FP_SART_REFINE;
}

// The refinement solver's SART pass: d = d0 (the copies' rounding of y_k),
// then per view the projection of the copy xt and of d (FP_SART_REFINE: the
// residual against y_k, A x~_k into ax, the objective partials of x~_k) and
// the SART update of d (in its own type: FP32 d takes no stochastic rounding).
static ctr_status refine_pass(ctr_solver* s, uint32_t seed, const uint32_t* pass_seed, const float* gdev,
                              cudaStream_t st)
{
    Geometry* g = s->g;
    const long long P = g->npix();
    const size_t per_view = objective_partials_per_view(g->dg);
    CTR_TRY(ensure_rays(g, (size_t)P * sizeof(float2)));
    CTR_TRY(launch_refine_start(*g, s->xk32, s->xm32, s->yt, s->ddt, s->vdt, gdev, st));
    const unsigned flags = s->ddt == CTR_F32 ? (s->p.sart_flags & ~CTR_SART_STOCHASTIC_ROUND) : s->p.sart_flags;
    for (int j = 0; j < g->desc.n_views; ++j) {
        FpArgs a{};
        a.vol = s->xt; a.vol_dtype = s->vdt; a.view0 = j; a.nview = 1; a.kind = refine_kind(s); a.tiled = 1;
        a.out = g->d_rays; a.b = (const char*)s->sino + (size_t)j * P * dtype_size(s->sdt); a.b_dtype = s->sdt;
        a.vol2 = s->yt; a.ax = s->ax + (size_t)j * P; a.gdev = gdev; a.partial = g->d_partial + (size_t)j * per_view;
        CTR_TRY(launch_forward(*g, a, st, nullptr));
        BpArgs b{};
        b.vol = s->yt; b.vol_dtype = s->ddt; b.rays = g->d_rays; b.view0 = j; b.nview = 1; b.sart = 1;
        b.flags = flags; b.beta = s->p.beta; b.seed = seed * 0x9E3779B9u + (uint32_t)j;
        b.pass_seed = pass_seed; b.tiled = 1;
        CTR_TRY(launch_backproject(*g, b, st));
    }
    return CTR_OK;
}

// Replay graph gi of the solver, capturing issue(stream) first if it has none
// or if a workspace it used (ws0, ws1) was reallocated by another call.
template <typename F>
static ctr_status solver_graph(ctr_solver* s, int gi, const void* ws0, const void* ws1, cudaStream_t st, F issue)
{
    if (s->exec[gi] && (s->graph_ws[gi][0] != ws0 || s->graph_ws[gi][1] != ws1)) {
        cudaGraphExecDestroy(s->exec[gi]);
        cudaGraphDestroy(s->graph[gi]);
        s->exec[gi] = nullptr;
        s->graph[gi] = nullptr;
    }
    if (!s->exec[gi]) {
        cudaStream_t cs;
        CTR_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        ctr_status r = CTR_OK;
        if (e != cudaSuccess) r = cuda_error(e, "cudaStreamBeginCapture");
        if (r == CTR_OK) r = issue(cs);
        cudaGraph_t gr = nullptr;
        e = cudaStreamEndCapture(cs, &gr);
        if (r == CTR_OK && e != cudaSuccess) r = cuda_error(e, "cudaStreamEndCapture");
        if (r == CTR_OK) {
            e = cudaGraphInstantiate(&s->exec[gi], gr, 0);
            if (e != cudaSuccess) r = cuda_error(e, "cudaGraphInstantiate");
        }
        s->graph[gi] = gr;
        s->graph_ws[gi][0] = ws0;
        s->graph_ws[gi][1] = ws1;
        cudaStreamDestroy(cs);
        if (r != CTR_OK) {
            if (s->exec[gi]) cudaGraphExecDestroy(s->exec[gi]);
            if (s->graph[gi]) cudaGraphDestroy(s->graph[gi]);
            s->exec[gi] = nullptr;
            s->graph[gi] = nullptr;
            return r;
        }
    }
    CTR_CUDA_TRY(cudaGraphLaunch(s->exec[gi], st));
    return CTR_OK;
}

// The refinement pass of ctr_solver_iterate: the FISTA factor of the pass
// goes to device memory first, so the captured graph reads it.
static ctr_status solver_refine_pass(ctr_solver* s, uint32_t seed, cudaStream_t st)
{
    Geometry* g = s->g;
    CTR_TRY(ensure_rays(g, (size_t)g->npix() * sizeof(float2)));
    CTR_TRY(ensure_partial(g, objective_partials_per_view(g->dg) * g->desc.n_views + 2048));
    CTR_TRY(launch_set_scalar(s->d_gm, s->gm, st));
    const bool stoch = (s->p.sart_flags & CTR_SART_STOCHASTIC_ROUND) != 0;
    if (!s->p.use_graph || stoch) return refine_pass(s, seed, nullptr, s->d_gm, st);
    return solver_graph(s, 2, g->d_rays, g->d_partial, st,
                        [&](cudaStream_t cs) { return refine_pass(s, 0, nullptr, s->d_gm, cs); });
}

// The refinement solver's objective of x_k by its own projection: the
// fidelity of the copy xt (tiled) that the passes project, the TV of the
// FP32 x_k, into d_obj.
static ctr_status refine_objective(ctr_solver* s, cudaStream_t st)
{
    Geometry* g = s->g;
    const size_t per_view = objective_partials_per_view(g->dg);
    const size_t nblk = per_view * g->desc.n_views;
    CTR_TRY(ensure_partial(g, std::max(nblk, (size_t)148 * 64) + 2048));
    const long long P = g->npix();
    for (int c = 0; c < g->desc.n_views; c += 65535) {
        FpArgs a{};
        a.vol = s->xt; a.vol_dtype = s->vdt; a.view0 = c; a.nview = std::min(65535, g->desc.n_views - c);
        a.kind = FP_OBJECTIVE; a.tiled = 1;
        a.b = (const char*)s->sino + (size_t)c * P * dtype_size(s->sdt); a.b_dtype = s->sdt;
        a.partial = g->d_partial + (size_t)c * per_view;
        CTR_TRY(launch_forward(*g, a, st, nullptr));
    }
    CTR_TRY(launch_reduce(g->d_partial, nblk, s->d_obj, st));
    return launch_tv(*g, s->xk32, CTR_F32, g->d_partial, 148 * 64, s->d_obj + 1, st);
}

// One SART pass (fused: also the objective partials of xt), captured once per
// form as a CUDA graph (2 launches per view) and replayed.
static ctr_status solver_sart(ctr_solver* s, uint32_t seed, cudaStream_t st, bool fused)
{
    Geometry* g = s->g;
    const void* xt = fused ? s->xt : nullptr;
    CTR_TRY(ensure_rays(g, (size_t)g->npix() * sizeof(float2)));
    if (fused) CTR_TRY(ensure_partial(g, objective_partials_per_view(g->dg) * g->desc.n_views + 2048));
    double* part = fused ? g->d_partial : nullptr;
    const bool stoch = (s->p.sart_flags & CTR_SART_STOCHASTIC_ROUND) != 0;
    if (!s->p.use_graph || stoch)   // the seed changes every pass: issue directly
        return sart_pass(g, s->y, s->vdt, s->sino, s->sdt, s->p.beta, s->p.sart_flags, seed, st, nullptr, s->yt, xt,
                         part);
    return solver_graph(s, fused ? 1 : 0, g->d_rays, part, st, [&](cudaStream_t cs) {
        return sart_pass(g, s->y, s->vdt, s->sino, s->sdt, s->p.beta, s->p.sart_flags, 0, cs, nullptr, s->yt, xt,
                         part);
    });
}

// The SART pass of the reference's D-device build on the solver's tiled
// volume: its slab sequence, each slab on its own stream between the
// combinations (sart_views_slabs), issued directly.
static ctr_status solver_sart_slabs(ctr_solver* s, uint32_t seed, cudaStream_t st)
{
    Geometry* g = s->g;
    std::vector<Geometry*> sl;
    CTR_TRY(slab_geoms(g, s->slabs, sl));
    CTR_TRY(launch_tiling(*g, s->y, s->yt, s->vdt, true, st));
    CTR_TRY(sart_views_slabs(g, sl, s->yt, s->vdt, true, s->sino, s->sdt, s->p.beta, s->p.sart_flags & ~CTR_SART_TILED,
                             seed, 0, g->desc.n_views, st));
    return launch_tiling(*g, s->yt, s->y, s->vdt, false, st);
}

extern "C" ctr_status ctr_solver_set_slabs(ctr_solver* s, int n_slabs)
{
    clear_error();
    CTR_TRY(need(s, "solver"));
    if (n_slabs < 1) return set_error(CTR_ERR_INVALID_ARGUMENT, "n_slabs must be >= 1");
    if (n_slabs > 1 && (s->refine || s->f64))
        return set_error(CTR_ERR_UNSUPPORTED, "the slab pass is not available to the %s solver",
                         s->f64 ? "FP64" : "refinement");
    if (n_slabs > 1) {
        std::vector<Geometry*> sl;
        CTR_TRY(slab_geoms(s->g, n_slabs, sl));   // the slab geometries, streams, events
        CTR_TRY(ensure_rays(s->g, (size_t)s->g->npix() * sizeof(float2)));
        CTR_TRY(ensure_parts(s->g, (size_t)s->g->npix() * n_slabs * sizeof(float2)));
    }
    s->slabs = n_slabs;
    return CTR_OK;
}

// history rows for iterations 1..k (allocated outside any capture)
static ctr_status hist_reserve(ctr_solver* s, int k, cudaStream_t st)
{
    if ((int)s->hist_valid.size() < k) s->hist_valid.resize(k, 0);
    if (k <= s->hist_cap) return CTR_OK;
    const int cap = std::max(k, 2 * s->hist_cap + 16);
    double* d = nullptr;
    CTR_CUDA_TRY(cudaMalloc(&d, sizeof(double) * 2 * cap));
    if (s->d_hist) {
        cudaError_t e = cudaMemcpyAsync(d, s->d_hist, sizeof(double) * 2 * s->hist_cap, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) { cudaFree(d); return cuda_error(e, "objective history"); }
        cudaFree(s->d_hist);
    }
    s->d_hist = d;
    s->hist_cap = cap;
    return CTR_OK;
}

// d_obj (fid, tv) -> history row of iteration k
static ctr_status hist_store(ctr_solver* s, int k, cudaStream_t st)
{
    CTR_CUDA_TRY(cudaMemcpyAsync(s->d_hist + 2 * (size_t)(k - 1), s->d_obj, 2 * sizeof(double),
                                 cudaMemcpyDeviceToDevice, st));
    s->hist_valid[k - 1] = 1;
    return CTR_OK;
}

// the pending objective of the current x_k, by its own projection
static ctr_status flush_objective(ctr_solver* s, cudaStream_t st)
{
    if (!s->obj_pending) return CTR_OK;
    const void* xk = s->p.fista ? s->xprev : s->y;
    CTR_TRY(hist_reserve(s, s->k, st));
    if (s->refine) {   // the fidelity of the projectors' copy of x_k, the TV of the FP32 x_k
        CTR_TRY(refine_objective(s, st));
        CTR_TRY(hist_store(s, s->k, st));
        s->obj_pending = false;
        return CTR_OK;
    }
    // with the slab pass, the n-device build's projector (its own for the tetrahedron beam)
    Geometry* og = (s->slabs > 1 && s->g->split_geom) ? s->g->split_geom : s->g;
    CTR_TRY(objective_async(og, xk, s->vdt, s->sino, s->sdt, s->d_obj, s->d_obj + 1, st, s->yt));
    CTR_TRY(hist_store(s, s->k, st));
    s->obj_pending = false;
    return CTR_OK;
}

// history rows of iterations first..first+count-1 as [TV, fidelity, objective]
static ctr_status read_history(ctr_solver* s, int first, int count, double* out, cudaStream_t st)
{
    std::vector<double> h(2 * (size_t)count);
    CTR_CUDA_TRY(cudaMemcpyAsync(h.data(), s->d_hist + 2 * (size_t)(first - 1), sizeof(double) * 2 * count,
                                 cudaMemcpyDeviceToHost, st));
    CTR_CUDA_TRY(cudaStreamSynchronize(st));
    for (int i = 0; i < count; ++i) {
        if (!s->hist_valid[first - 1 + i]) {
            out[3 * i + 0] = out[3 * i + 1] = out[3 * i + 2] = NAN;
            continue;
        }
        out[3 * i + 0] = h[2 * i + 1];
        out[3 * i + 1] = h[2 * i];
        out[3 * i + 2] = h[2 * i] + 2.0 * (double)s->p.lambda_tv * h[2 * i + 1];   // V63/main_recon.cu:423
    }
    return CTR_OK;
}

extern "C" ctr_status ctr_solver_iterate(ctr_solver* s, int n, double* obj_out, void* stream)
{
    clear_error();
    CTR_TRY(need(s, "solver"));
    if (!s->sino) return set_error(CTR_ERR_INVALID_ARGUMENT, "no sinogram set");
    if (n < 0) return set_error(CTR_ERR_INVALID_ARGUMENT, "n < 0");
    cudaStream_t st = S(stream);
    Geometry* g = s->g;
    if (s->f64) return f64_iterate(s->f64, s->sino, s->sdt, n, obj_out, st);
    const int k0 = s->k;
    CTR_TRY(hist_reserve(s, k0 + n, st));
    if (s->refine) {
        for (int it = 0; it < n; ++it) {
            // y_k = (1+g) x_k - g x_(k-1) stays implicit: the pass projects the
            // copy of x_k and the correction d, and the objective of x_k rides
            // on it (V63/main_recon.cu:344-386, 390-430)
            const bool pending = s->obj_pending;
            if (pending) CTR_TRY(launch_tv(*g, s->xk32, CTR_F32, g->d_partial, 148 * 64, s->d_obj + 1, st));
            CTR_TRY(solver_refine_pass(s, (uint32_t)(s->k + 1), st));
            if (pending) {
                CTR_TRY(launch_reduce(g->d_partial, objective_partials_per_view(g->dg) * g->desc.n_views, s->d_obj,
                                      st));
                CTR_TRY(hist_store(s, s->k, st));
                s->obj_pending = false;
            }
            const float lam = s->p.lambda_tv > 0.f ? s->p.beta * s->p.lambda_tv : 0.f;
            CTR_TRY(launch_refine_update(*g, s->xk32, s->xm32, s->yt, s->ddt, s->xt, s->vdt, lam, s->p.fgp_iters, s->d_gm,
                                         st));
            const float t_k = (1.0f + sqrtf(1.0f + 4.0f * s->t * s->t)) / 2.0f;   // :372
            if (s->p.fista) {
                s->gm = (s->t - 1.0f) / t_k;                                     // the next pass's y_k
                s->t = t_k;
            }
            s->k++;
            s->obj_pending = s->p.objective != 0;
        }
        if (obj_out && n > 0) {
            CTR_TRY(flush_objective(s, st));
            CTR_TRY(read_history(s, k0 + 1, n, obj_out, st));
        }
        return check_device_errors(g, st);
    }
    for (int it = 0; it < n; ++it) {
        // The objective of x_(k-1), the previous iteration's result (V63/main_recon.cu:390-430),
        // is projected in this iteration's SART traversal: x_(k-1) is xprev with
        // FISTA and the volume the pass starts from without.  With the slab
        // pass it is projected on its own with the one-device projector, whose
        // sums the D-device build's row-split projector gives
        // (V63/host_IterativeRecon_CBCT_multiGPU.c:171-258).
        const bool slabbed = s->slabs > 1;
        if (slabbed && s->obj_pending) CTR_TRY(flush_objective(s, st));
        const bool fused = s->obj_pending;
        if (fused) {
            const void* xk1 = s->p.fista ? s->xprev : s->y;
            CTR_TRY(launch_tiling(*g, xk1, s->xt, s->vdt, true, st));
            CTR_TRY(objective_async(g, xk1, s->vdt, s->sino, s->sdt, nullptr, s->d_obj + 1, st));   // TV
        }
        // V63/main_recon.cu:344-386 (FISTA == 1) / :316-341 (FISTA == 0)
        if (slabbed) CTR_TRY(solver_sart_slabs(s, (uint32_t)(s->k + 1), st));
        else CTR_TRY(solver_sart(s, (uint32_t)(s->k + 1), st, fused));
        if (fused) {
            CTR_TRY(launch_reduce(g->d_partial, objective_partials_per_view(g->dg) * g->desc.n_views, s->d_obj, st));
            CTR_TRY(hist_store(s, s->k, st));
            s->obj_pending = false;
        }
        const float lam = s->p.beta * s->p.lambda_tv;     // lambda_denoise_TV = 2*lambda_TV/Lip
        const float t_k = (1.0f + sqrtf(1.0f + 4.0f * s->t * s->t)) / 2.0f;   // :372
        const float gam = (s->t - 1.0f) / t_k;
        if (s->p.fista) {
            if (s->p.lambda_tv > 0.f && s->p.fgp_iters >= 0)
                CTR_TRY(launch_fgp(*g, s->y, s->vdt, lam, s->p.fgp_iters, s->y, s->xprev, gam, st));
            else
                CTR_TRY(launch_momentum(*g, s->y, s->xprev, s->y, s->vdt, gam, st));
            s->t = t_k;
        } else if (s->p.lambda_tv > 0.f) {
            CTR_TRY(launch_fgp(*g, s->y, s->vdt, lam, s->p.fgp_iters, nullptr, nullptr, 0.f, st));
        }
        s->k++;
        s->obj_pending = s->p.objective != 0;
    }
    if (obj_out && n > 0) {
        CTR_TRY(flush_objective(s, st));
        CTR_TRY(read_history(s, k0 + 1, n, obj_out, st));
    }
    return check_device_errors(g, st);
}

extern "C" ctr_status ctr_solver_objectives(ctr_solver* s, int first, int count, double* out, void* stream)
{
    clear_error();
    CTR_TRY(need(s, "solver"));
    CTR_TRY(need(out, "out"));
    if (s->f64)
        return set_error(CTR_ERR_UNSUPPORTED, "the FP64 solver returns its objectives from ctr_solver_iterate only");
    if (first < 1 || count < 0 || first + count - 1 > s->k)
        return set_error(CTR_ERR_INVALID_ARGUMENT, "iterations %d..%d not run (k = %d)", first, first + count - 1, s->k);
    if (count == 0) return CTR_OK;
    cudaStream_t st = S(stream);
    CTR_TRY(hist_reserve(s, s->k, st));
    if (first + count - 1 == s->k) CTR_TRY(flush_objective(s, st));
    return read_history(s, first, count, out, st);
}

extern "C" ctr_status ctr_solver_get_volume(ctr_solver* s, void* dst, void* stream)
{
    clear_error();
    CTR_TRY(need(s, "solver"));
    CTR_TRY(need(dst, "dst"));
    if (s->f64) return f64_get_volume(s->f64, dst, false, S(stream));
    const void* xk = (s->p.fista && s->k > 0) ? s->xprev : s->y;
    if (s->refine) {   // the storage rounding of the FP32 x_k (the projectors' copy, untiled)
        CTR_TRY(launch_convert(s->xk32, CTR_F32, s->y, s->vdt, s->g->nvox(), S(stream)));
        xk = s->y;
    }
    CTR_CUDA_TRY(cudaMemcpyAsync(dst, xk, s->g->nvox() * dtype_size(s->vdt), cudaMemcpyDefault, S(stream)));
    CTR_CUDA_TRY(cudaStreamSynchronize(S(stream)));
    return CTR_OK;
}

extern "C" ctr_status ctr_solver_get_volume_f32(ctr_solver* s, float* dst, void* stream)
{
    clear_error();
    CTR_TRY(need(s, "solver"));
    CTR_TRY(need(dst, "dst"));
    cudaStream_t st = S(stream);
    if (s->f64) return f64_get_volume(s->f64, dst, true, st);
    const size_t b32 = s->g->nvox() * sizeof(float);
    if (s->refine) {
        CTR_CUDA_TRY(cudaMemcpyAsync(dst, s->xk32, b32, cudaMemcpyDefault, st));
        CTR_CUDA_TRY(cudaStreamSynchronize(st));
        return CTR_OK;
    }
    const void* xk = (s->p.fista && s->k > 0) ? s->xprev : s->y;
    if (s->vdt == CTR_F32) {
        CTR_CUDA_TRY(cudaMemcpyAsync(dst, xk, b32, cudaMemcpyDefault, st));
        CTR_CUDA_TRY(cudaStreamSynchronize(st));
        return CTR_OK;
    }
    float* tmp = nullptr;   // widened on the device, then copied to dst (which may be host memory)
    CTR_CUDA_TRY(cudaMalloc(&tmp, b32));
    ctr_status r = launch_convert(xk, s->vdt, tmp, CTR_F32, s->g->nvox(), st);
    cudaError_t e = cudaSuccess;
    if (r == CTR_OK) e = cudaMemcpyAsync(dst, tmp, b32, cudaMemcpyDefault, st);
    if (r == CTR_OK && e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(tmp);
    if (r != CTR_OK) return r;
    CTR_CUDA_TRY(e);
    return CTR_OK;
}

extern "C" ctr_status ctr_solver_iteration_count(const ctr_solver* s, int* k)
{
    if (!s || !k) return set_error(CTR_ERR_INVALID_ARGUMENT, "NULL argument");
    *k = s->f64 ? f64_iteration(s->f64) : s->k;
    return CTR_OK;
}

static uint64_t geom_hash(const ctr_geometry_desc& d)
{
    uint64_t h = 1469598103934665603ULL;
    const unsigned char* b = reinterpret_cast<const unsigned char*>(&d);
    for (size_t i = 0; i < sizeof(d); ++i) h = (h ^ b[i]) * 1099511628211ULL;
    return h;
}

struct CkptHeader {
    char magic[8];
    uint32_t version, dtype;
    uint64_t geom;
    int32_t k, fista;
    float t, pad;
    uint64_t nvox;
};

extern "C" ctr_status ctr_solver_save(ctr_solver* s, const char* path, void* stream)
{
    clear_error();
    CTR_TRY(need(s, "solver"));
    CTR_TRY(need(path, "path"));
    if (s->f64) return set_error(CTR_ERR_UNSUPPORTED, "the FP64 solver has no checkpoint");
    // refinement solver: the FP32 x_k and x_(k-1) (its copies and A x~_(k-1) are rebuilt on load)
    const size_t bytes = s->g->nvox() * (s->refine ? sizeof(float) : dtype_size(s->vdt));
    std::vector<char> buf(2 * bytes);
    CTR_CUDA_TRY(cudaMemcpyAsync(buf.data(), s->refine ? (void*)s->xk32 : s->y, bytes, cudaMemcpyDeviceToHost,
                                 S(stream)));
    CTR_CUDA_TRY(cudaMemcpyAsync(buf.data() + bytes, s->refine ? (void*)s->xm32 : s->xprev, bytes,
                                 cudaMemcpyDeviceToHost, S(stream)));
    CTR_CUDA_TRY(cudaStreamSynchronize(S(stream)));
    CkptHeader h{};
    memcpy(h.magic, "CTRCKPT1", 8);
    h.version = s->refine ? 2 : 1; h.dtype = s->vdt; h.geom = geom_hash(s->g->desc); h.k = s->k;
    h.fista = s->p.fista; h.t = s->t; h.pad = s->refine ? s->gm : 0.0f; h.nvox = s->g->nvox();
    FILE* f = fopen(path, "wb");
    if (!f) return set_error(CTR_ERR_IO, "cannot open %s for writing", path);
    const bool ok = fwrite(&h, sizeof(h), 1, f) == 1 && fwrite(buf.data(), 1, buf.size(), f) == buf.size();
    const bool closed = fclose(f) == 0;
    if (!ok || !closed) return set_error(CTR_ERR_IO, "short write to %s", path);
    return CTR_OK;
}

extern "C" ctr_status ctr_solver_load(ctr_solver* s, const char* path, void* stream)
{
    clear_error();
    CTR_TRY(need(s, "solver"));
    CTR_TRY(need(path, "path"));
    if (s->f64) return set_error(CTR_ERR_UNSUPPORTED, "the FP64 solver has no checkpoint");
    FILE* f = fopen(path, "rb");
    if (!f) return set_error(CTR_ERR_IO, "cannot open %s", path);
    CkptHeader h{};
    const size_t bytes = s->g->nvox() * (s->refine ? sizeof(float) : dtype_size(s->vdt));
    std::vector<char> buf(2 * bytes);
    const bool ok = fread(&h, sizeof(h), 1, f) == 1 && fread(buf.data(), 1, buf.size(), f) == buf.size();
    fclose(f);
    if (!ok || memcmp(h.magic, "CTRCKPT1", 8) != 0) return set_error(CTR_ERR_IO, "%s is not a solver checkpoint", path);
    if (h.geom != geom_hash(s->g->desc) || h.dtype != (uint32_t)s->vdt || h.nvox != (uint64_t)s->g->nvox())
        return set_error(CTR_ERR_INVALID_ARGUMENT, "checkpoint %s was written for another geometry or dtype", path);
    if (h.version != (s->refine ? 2u : 1u))
        return set_error(CTR_ERR_INVALID_ARGUMENT, "checkpoint %s was written by a %s solver", path,
                         h.version == 2 ? "refinement" : "non-refinement");
    cudaStream_t st = S(stream);
    if (s->refine) {
        // x_k, x_(k-1) in FP32; the copy of x_k (tiled) and A x~_(k-1) of the
        // copy of x_(k-1), as the passes left them (a forward projection of
        // the linear copy gives the same sums, with the same zero rule)
        Geometry* g = s->g;
        CTR_CUDA_TRY(cudaMemcpyAsync(s->xk32, buf.data(), bytes, cudaMemcpyHostToDevice, st));
        CTR_CUDA_TRY(cudaMemcpyAsync(s->xm32, buf.data() + bytes, bytes, cudaMemcpyHostToDevice, st));
        CTR_TRY(launch_convert(s->xk32, CTR_F32, s->y, s->vdt, g->nvox(), st));
        CTR_TRY(launch_tiling(*g, s->y, s->xt, s->vdt, true, st));
        CTR_TRY(launch_convert(s->xm32, CTR_F32, s->xprev, s->vdt, g->nvox(), st));
        FpArgs a{};
        a.vol = s->xprev; a.vol_dtype = s->vdt; a.view0 = 0; a.nview = g->desc.n_views; a.kind = FP_FORWARD;
        a.out = s->ax; a.out_dtype = CTR_F32;
        CTR_TRY(forward_chunks(g, a, st));
        CTR_CUDA_TRY(cudaStreamSynchronize(st));
        s->gm = h.pad;
    } else {
        CTR_CUDA_TRY(cudaMemcpyAsync(s->y, buf.data(), bytes, cudaMemcpyHostToDevice, st));
        CTR_CUDA_TRY(cudaMemcpyAsync(s->xprev, buf.data() + bytes, bytes, cudaMemcpyHostToDevice, st));
        CTR_CUDA_TRY(cudaStreamSynchronize(st));
    }
    s->k = h.k;
    s->t = h.t;
    s->obj_pending = false;                       // objectives before the checkpoint are not known here
    s->hist_valid.assign((size_t)std::max(h.k, 0), 0);
    return CTR_OK;
}

// ------------------------------------------------------------ batched scans

// Workspace a solver's iteration needs, allocated before graph capture.
static ctr_status solver_reserve(ctr_solver* s)
{
    Geometry* g = s->g;
    CTR_TRY(ensure_rays(g, (size_t)g->npix() * sizeof(float2)));
    if (s->p.lambda_tv > 0.f) CTR_TRY(ensure_fgp(g, fgp_workspace_bytes(g->nvox(), s->vdt)));
    const size_t nblk = objective_partials_per_view(g->dg) * g->desc.n_views;
    CTR_TRY(ensure_partial(g, std::max(nblk, (size_t)148 * 64) + 2048));
    return CTR_OK;
}

// FGP-TV with the fused FISTA step (or the momentum alone), the FISTA factor
// read from device memory (V63/main_recon.cu:360-384).
static ctr_status solver_prox(ctr_solver* s, cudaStream_t st, const float* gam_dev)
{
    Geometry* g = s->g;
    const float lam = s->p.beta * s->p.lambda_tv;
    if (s->p.fista) {
        if (s->p.lambda_tv > 0.f)
            CTR_TRY(launch_fgp(*g, s->y, s->vdt, lam, s->p.fgp_iters, s->y, s->xprev, 0.f, st, gam_dev));
        else
            CTR_TRY(launch_momentum(*g, s->y, s->xprev, s->y, s->vdt, 0.f, st, gam_dev));
    } else if (s->p.lambda_tv > 0.f) {
        CTR_TRY(launch_fgp(*g, s->y, s->vdt, lam, s->p.fgp_iters, nullptr, nullptr, 0.f, st));
    }
    return CTR_OK;
}

// One outer iteration of V63/main_recon.cu:344-386 for one scan on stream st;
// the FISTA factor and the stochastic-rounding seed of the pass are read from
// device memory so the launches can be replayed.  fused: the SART traversal
// also projects the objective of x_(k-1) (into d_obj), as ctr_solver_iterate
// does from the second iteration of a call on.
static ctr_status solver_issue(ctr_solver* s, cudaStream_t st, const float* gam_dev, const uint32_t* seed_dev,
                               bool fused)
{
    Geometry* g = s->g;
    if (s->refine) {   // as ctr_solver_iterate's refinement iteration, with g from gam_dev
        if (fused) CTR_TRY(launch_tv(*g, s->xk32, CTR_F32, g->d_partial, 148 * 64, s->d_obj + 1, st));
        CTR_TRY(refine_pass(s, 0, seed_dev, gam_dev, st));
        if (fused)
            CTR_TRY(launch_reduce(g->d_partial, objective_partials_per_view(g->dg) * g->desc.n_views, s->d_obj, st));
        const float lam = s->p.lambda_tv > 0.f ? s->p.beta * s->p.lambda_tv : 0.f;
        return launch_refine_update(*g, s->xk32, s->xm32, s->yt, s->ddt, s->xt, s->vdt, lam, s->p.fgp_iters, gam_dev, st);
    }
    if (fused) {
        const void* xk1 = s->p.fista ? s->xprev : s->y;
        CTR_TRY(launch_tiling(*g, xk1, s->xt, s->vdt, true, st));
        CTR_TRY(objective_async(g, xk1, s->vdt, s->sino, s->sdt, nullptr, s->d_obj + 1, st));   // TV
    }
    CTR_TRY(sart_pass(g, s->y, s->vdt, s->sino, s->sdt, s->p.beta, s->p.sart_flags, 0, st, seed_dev, s->yt,
                      fused ? s->xt : nullptr, fused ? g->d_partial : nullptr));
    if (fused)
        CTR_TRY(launch_reduce(g->d_partial, objective_partials_per_view(g->dg) * g->desc.n_views, s->d_obj, st));
    return solver_prox(s, st, gam_dev);
}

// The batch's persistent form of solver_issue: the steps before and after
// the SART pass's views, which the persistent pass runs for every scan in
// one launch between them.
static ctr_status batch_pre(ctr_solver* s, cudaStream_t st, bool fused, const float* gam_dev)
{
    Geometry* g = s->g;
    if (s->refine) {
        if (fused) CTR_TRY(launch_tv(*g, s->xk32, CTR_F32, g->d_partial, 148 * 64, s->d_obj + 1, st));
        return launch_refine_start(*g, s->xk32, s->xm32, s->yt, s->ddt, s->vdt, gam_dev, st);
    }
    if (fused) {
        const void* xk1 = s->p.fista ? s->xprev : s->y;
        CTR_TRY(launch_tiling(*g, xk1, s->xt, s->vdt, true, st));
        CTR_TRY(objective_async(g, xk1, s->vdt, s->sino, s->sdt, nullptr, s->d_obj + 1, st));   // TV
    }
    return launch_tiling(*g, s->y, s->yt, s->vdt, true, st);
}

static ctr_status batch_post(ctr_solver* s, cudaStream_t st, const float* gam_dev, bool fused)
{
    Geometry* g = s->g;
    if (!s->refine) CTR_TRY(launch_tiling(*g, s->yt, s->y, s->vdt, false, st));
    if (fused)
        CTR_TRY(launch_reduce(g->d_partial, objective_partials_per_view(g->dg) * g->desc.n_views, s->d_obj, st));
    if (s->refine) {
        const float lam = s->p.lambda_tv > 0.f ? s->p.beta * s->p.lambda_tv : 0.f;
        return launch_refine_update(*g, s->xk32, s->xm32, s->yt, s->ddt, s->xt, s->vdt, lam, s->p.fgp_iters, gam_dev, st);
    }
    return solver_prox(s, st, gam_dev);
}

struct ctr_batch {
    std::vector<ctr_solver*> scans;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> joins;
    cudaEvent_t fork = nullptr;
    float* d_gam = nullptr;                 // per scan FISTA factor of the coming iteration
    uint32_t* d_seed = nullptr;             // per scan stochastic-rounding seed of the coming pass
    std::vector<float> h_gam;
    std::vector<uint32_t> h_seed;
    // one iteration of every scan: [0] plain, [1] with the previous objective fused
    cudaGraph_t graph[2] = {nullptr, nullptr};
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    std::vector<const void*> ws[2];         // workspaces each graph was captured with, 3 per scan
    // the persistent pass (ctr_batch_set_persistent): the SART views of every
    // scan in one launch per iteration
    bool persistent = false;
    int pass_blocks = 0;                    // CTAs of the launch (its occupancy x SMs)
    size_t pass_smem = 0;
    BatchScan* d_scans[2] = {nullptr, nullptr};   // per graph: the scans' pass descriptions
    void* d_flow = nullptr;                 // the pass's work counters (batch_flow_bytes)
    unsigned* d_err = nullptr;              // ERR_BARRIER
};

static std::vector<const void*> batch_workspaces(const ctr_batch* b)
{
    std::vector<const void*> w;
    for (const auto* s : b->scans) {
        w.push_back(s->g->d_rays);
        w.push_back(s->g->d_partial);
        w.push_back(s->g->d_fgp);
    }
    return w;
}

static void batch_drop_graph(ctr_batch* b, int which = -1)
{
    for (int i = 0; i < 2; ++i) {
        if (which >= 0 && which != i) continue;
        if (b->exec[i]) cudaGraphExecDestroy(b->exec[i]);
        if (b->graph[i]) cudaGraphDestroy(b->graph[i]);
        b->exec[i] = nullptr;
        b->graph[i] = nullptr;
    }
}

// The forward kind of the scans' passes in graph gi (the same for all scans).
static int batch_pass_kind(const ctr_batch* b, int gi)
{
    return b->scans[0]->refine ? refine_kind(b->scans[0]) : (gi == 1 ? FP_SART_OBJ : FP_SART);
}

// The scans' descriptions for the persistent pass of graph gi, and the
// split of the launch's CTAs: each scan gets CTAs in proportion to the
// instructions of its pass (ray steps of the forward projections, voxels
// of the updates), at least one.
static ctr_status batch_describe(ctr_batch* b, int gi)
{
    const int ns = (int)b->scans.size();
    const int T = b->pass_blocks;
    if (ns > T) return set_error(CTR_ERR_UNSUPPORTED, "%d scans exceed the persistent pass's %d resident blocks", ns, T);
    std::vector<double> cost(ns);
    double total = 0.0;
    for (int i = 0; i < ns; ++i) {
        const DevGeom& g = b->scans[i]->g->dg;
        cost[i] = (double)g.nviews * ((double)g.R * g.ZP * (g.M + g.N + g.Z) * 21.0 + (double)g.M * g.N * g.Z * 170.0);
        total += cost[i];
    }
    std::vector<int> nc(ns);
    int used = 0;
    for (int i = 0; i < ns; ++i) {
        nc[i] = std::max(1, (int)std::floor(T * cost[i] / total));
        used += nc[i];
    }
    while (used > T) {   // trim the scans with the most CTAs per unit of work
        int k = -1;
        for (int i = 0; i < ns; ++i)
            if (nc[i] > 1 && (k < 0 || nc[i] / cost[i] > nc[k] / cost[k])) k = i;
        --nc[k];
        --used;
    }
    while (used < T) {   // give the rest to the scans with the most work per CTA
        int k = 0;
        for (int i = 1; i < ns; ++i)
            if (cost[i] / nc[i] > cost[k] / nc[k]) k = i;
        ++nc[k];
        ++used;
    }
    const int kind = batch_pass_kind(b, gi);
    std::vector<BatchScan> h(ns);
    int c0 = 0;
    for (int i = 0; i < ns; ++i) {
        ctr_solver* s = b->scans[i];
        Geometry* G = s->g;
        BatchScan& q = h[i];
        q.g = G->dg;
        if (s->refine) {
            q.fp_vol = s->xt; q.fp_vol2 = s->yt; q.bp_vol = s->yt;
            q.partial = G->d_partial; q.ax = s->ax; q.gdev = b->d_gam + i;
        } else {
            q.fp_vol = s->yt; q.fp_vol2 = kind == FP_SART_OBJ ? s->xt : nullptr; q.bp_vol = s->yt;
            q.partial = kind == FP_SART_OBJ ? G->d_partial : nullptr; q.ax = nullptr; q.gdev = nullptr;
        }
        q.b = s->sino;
        q.b_dt = s->sdt;
        q.rays = (float2*)G->d_rays;
        q.pass_seed = b->d_seed + i;
        q.beta = s->p.beta;
        q.nviews = G->desc.n_views;
        q.c0 = c0;
        q.nc = nc[i];
        c0 += nc[i];
        q.fp_gx = (G->dg.R + 31) / 32;
        q.fp_gy = (G->dg.ZP + 3) / 4;
        // the full z run of 32 voxels: the scans fill the GPU together, so a
        // small scan's run is not shortened to make blocks (fewer blocks to
        // hand out, each column's setup shared by more voxels)
        q.zl = std::min(32, G->dg.Z);
        q.bp_gx = (G->dg.M + 31) / 32;
        q.bp_gy = (G->dg.N + 3) / 4;
        q.bp_gz = (G->dg.Z + q.zl - 1) / q.zl;
    }
    if (!b->d_scans[gi]) CTR_CUDA_TRY(cudaMalloc(&b->d_scans[gi], sizeof(BatchScan) * ns));
    CTR_CUDA_TRY(cudaMemcpy(b->d_scans[gi], h.data(), sizeof(BatchScan) * ns, cudaMemcpyHostToDevice));
    return CTR_OK;
}

static ctr_status batch_capture(ctr_batch* b, int gi)
{
    const int ns = (int)b->scans.size();
    for (auto* s : b->scans) CTR_TRY(solver_reserve(s));
    if (b->persistent) CTR_TRY(batch_describe(b, gi));
    CTR_CUDA_TRY(cudaDeviceSynchronize());
    cudaStream_t cs;
    CTR_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    ctr_status r = CTR_OK;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) r = cuda_error(e, "cudaStreamBeginCapture");
    if (r == CTR_OK && (e = cudaEventRecord(b->fork, cs)) != cudaSuccess) r = cuda_error(e, "cudaEventRecord");
    if (!b->persistent) {
        for (int i = 0; i < ns && r == CTR_OK; ++i) {
            if ((e = cudaStreamWaitEvent(b->streams[i], b->fork, 0)) != cudaSuccess) { r = cuda_error(e, "fork"); break; }
            r = solver_issue(b->scans[i], b->streams[i], b->d_gam + i, b->d_seed + i, gi == 1);
            if (r == CTR_OK && (e = cudaEventRecord(b->joins[i], b->streams[i])) != cudaSuccess) r = cuda_error(e, "join");
            if (r == CTR_OK && (e = cudaStreamWaitEvent(cs, b->joins[i], 0)) != cudaSuccess) r = cuda_error(e, "join");
        }
    } else {
        // every scan's steps before its views (parallel branches), the one
        // persistent pass, every scan's steps after them
        for (int i = 0; i < ns && r == CTR_OK; ++i) {
            if ((e = cudaStreamWaitEvent(b->streams[i], b->fork, 0)) != cudaSuccess) { r = cuda_error(e, "fork"); break; }
            r = batch_pre(b->scans[i], b->streams[i], gi == 1, b->d_gam + i);
            if (r == CTR_OK && (e = cudaEventRecord(b->joins[i], b->streams[i])) != cudaSuccess) r = cuda_error(e, "join");
            if (r == CTR_OK && (e = cudaStreamWaitEvent(cs, b->joins[i], 0)) != cudaSuccess) r = cuda_error(e, "join");
        }
        const bool stoch = (b->scans[0]->p.sart_flags & CTR_SART_STOCHASTIC_ROUND) != 0;
        if (r == CTR_OK && (e = cudaMemsetAsync(b->d_flow, 0, batch_flow_bytes(ns), cs)) != cudaSuccess)
            r = cuda_error(e, "cudaMemsetAsync");
        if (r == CTR_OK)
            r = launch_batch_pass(b->d_scans[gi], ns, b->pass_blocks, b->scans[0]->vdt, batch_pass_kind(b, gi), stoch,
                                  b->d_flow, b->d_err, b->pass_smem, cs);
        if (r == CTR_OK && (e = cudaEventRecord(b->fork, cs)) != cudaSuccess) r = cuda_error(e, "cudaEventRecord");
        for (int i = 0; i < ns && r == CTR_OK; ++i) {
            if ((e = cudaStreamWaitEvent(b->streams[i], b->fork, 0)) != cudaSuccess) { r = cuda_error(e, "fork"); break; }
            r = batch_post(b->scans[i], b->streams[i], b->d_gam + i, gi == 1);
            if (r == CTR_OK && (e = cudaEventRecord(b->joins[i], b->streams[i])) != cudaSuccess) r = cuda_error(e, "join");
            if (r == CTR_OK && (e = cudaStreamWaitEvent(cs, b->joins[i], 0)) != cudaSuccess) r = cuda_error(e, "join");
        }
    }
    cudaGraph_t gr = nullptr;
    e = cudaStreamEndCapture(cs, &gr);
    if (r == CTR_OK && e != cudaSuccess) r = cuda_error(e, "cudaStreamEndCapture");
    if (r == CTR_OK && (e = cudaGraphInstantiate(&b->exec[gi], gr, 0)) != cudaSuccess) r = cuda_error(e, "cudaGraphInstantiate");
    b->graph[gi] = gr;
    b->ws[gi] = batch_workspaces(b);
    cudaStreamDestroy(cs);
    if (r != CTR_OK) batch_drop_graph(b, gi);
    return r;
}

extern "C" ctr_status ctr_batch_destroy(ctr_batch* b)
{
    if (!b) return CTR_OK;
    batch_drop_graph(b);
    for (auto* s : b->scans) ctr_solver_destroy(s);
    for (auto st : b->streams) if (st) cudaStreamDestroy(st);
    for (auto e : b->joins) if (e) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    cudaFree(b->d_gam);
    cudaFree(b->d_seed);
    cudaFree(b->d_scans[0]);
    cudaFree(b->d_scans[1]);
    cudaFree(b->d_flow);
    cudaFree(b->d_err);
    delete b;
    return CTR_OK;
}

extern "C" ctr_status ctr_batch_set_persistent(ctr_batch* b, int on)
{
    clear_error();
    CTR_TRY(need(b, "batch"));
    batch_drop_graph(b);
    if (!on) {
        b->persistent = false;
        return CTR_OK;
    }
    const int ns = (int)b->scans.size();
    size_t smem = 0;
    for (int i = 0; i < ns; ++i) {
        const ctr_solver* s = b->scans[i];
        const DevGeom& g = s->g->dg;
        if ((s->p.sart_flags & CTR_SART_REFERENCE_BP) || s->slabs > 1 || g.entry64 || g.fast_sums || g.slab_n > 1)
            return set_error(CTR_ERR_UNSUPPORTED,
                             "scan %d: the persistent pass runs the engine's update with FP32 entry and the "
                             "reference's sums (no CTR_SART_REFERENCE_BP, slabs, CTR_GEOM_ENTRY_F64 or "
                             "CTR_GEOM_FAST_SUMS)", i);
        smem = std::max(smem, batch_pass_smem(g));
    }
    if (smem > 227 * 1024) return set_error(CTR_ERR_UNSUPPORTED, "persistent pass: tables exceed shared memory");
    const ctr_dtype vdt = b->scans[0]->vdt;
    const bool stoch = (b->scans[0]->p.sart_flags & CTR_SART_STOCHASTIC_ROUND) != 0;
    int per_sm = 0;
    if (b->scans[0]->refine) {
        const FpKind k = refine_kind(b->scans[0]);
        per_sm = batch_pass_blocks_per_sm(vdt, k, stoch && k == FP_SART_REFINE, smem);
    } else {
        per_sm = std::min(batch_pass_blocks_per_sm(vdt, FP_SART, stoch, smem),
                          batch_pass_blocks_per_sm(vdt, FP_SART_OBJ, stoch, smem));
    }
    int dev = 0, sms = 0;
    CTR_CUDA_TRY(cudaGetDevice(&dev));
    CTR_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (per_sm <= 0 || per_sm * sms < ns)
        return set_error(CTR_ERR_UNSUPPORTED, "persistent pass: %d resident blocks for %d scans", per_sm * sms, ns);
    if (!b->d_flow) CTR_CUDA_TRY(cudaMalloc(&b->d_flow, batch_flow_bytes(ns)));
    if (!b->d_err) CTR_CUDA_TRY(cudaMalloc(&b->d_err, sizeof(unsigned)));
    CTR_CUDA_TRY(cudaMemset(b->d_err, 0, sizeof(unsigned)));
    b->pass_blocks = per_sm * sms;
    b->pass_smem = smem;
    b->persistent = true;
    return CTR_OK;
}

extern "C" ctr_status ctr_batch_create(const ctr_geometry* const* geoms, int n, ctr_dtype vdt,
                                       const ctr_solver_params* p, ctr_batch** out)
{
    clear_error();
    CTR_TRY(need(geoms, "geometries"));
    CTR_TRY(need(p, "params"));
    CTR_TRY(need(out, "out"));
    *out = nullptr;
    if (n <= 0) return set_error(CTR_ERR_INVALID_ARGUMENT, "need at least one scan");
    if (vdt == CTR_F64) return set_error(CTR_ERR_UNSUPPORTED, "the FP64 solver runs one scan at a time");
    for (int i = 0; i < n; ++i) {
        if (!geoms[i]) return set_error(CTR_ERR_INVALID_ARGUMENT, "geometry %d is NULL", i);
        for (int j = 0; j < i; ++j)
            if (geoms[j] == geoms[i])
                return set_error(CTR_ERR_INVALID_ARGUMENT, "scans %d and %d share a geometry (workspaces would race)", j, i);
    }
    ctr_batch* b = new (std::nothrow) ctr_batch();
    if (!b) return set_error(CTR_ERR_OUT_OF_MEMORY, "host allocation");
    ctr_status st = CTR_OK;
    for (int i = 0; i < n && st == CTR_OK; ++i) {
        ctr_solver* s = nullptr;
        st = ctr_solver_create(geoms[i], vdt, p, &s);
        if (st == CTR_OK) {
            s->p.sart_flags |= BP_FULL_RUNS;   // the scans fill the GPU together
            b->scans.push_back(s);
        }
        cudaStream_t cs = nullptr;
        cudaEvent_t ev = nullptr;
        if (st == CTR_OK && cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess)
            st = set_error(CTR_ERR_CUDA, "cudaStreamCreate");
        b->streams.push_back(cs);
        if (st == CTR_OK && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
            st = set_error(CTR_ERR_CUDA, "cudaEventCreate");
        b->joins.push_back(ev);
    }
    if (st == CTR_OK && cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess)
        st = set_error(CTR_ERR_CUDA, "cudaEventCreate");
    if (st == CTR_OK && (cudaMalloc(&b->d_gam, sizeof(float) * n) != cudaSuccess ||
                         cudaMalloc(&b->d_seed, sizeof(uint32_t) * n) != cudaSuccess))
        st = set_error(CTR_ERR_OUT_OF_MEMORY, "cudaMalloc");
    b->h_gam.assign(n, 0.f);
    b->h_seed.assign(n, 0u);
    if (st != CTR_OK) {
        ctr_batch_destroy(b);
        return st;
    }
    *out = b;
    return CTR_OK;
}

extern "C" ctr_status ctr_batch_set_sinogram(ctr_batch* b, int scan, const void* sino, ctr_dtype sdt)
{
    clear_error();
    CTR_TRY(need(b, "batch"));
    if (scan < 0 || scan >= (int)b->scans.size()) return set_error(CTR_ERR_INVALID_ARGUMENT, "scan %d out of range", scan);
    const void* old = b->scans[scan]->sino;
    CTR_TRY(ctr_solver_set_sinogram(b->scans[scan], sino, sdt));
    if (old != sino) batch_drop_graph(b);
    return CTR_OK;
}

extern "C" ctr_status ctr_batch_reset(ctr_batch* b, void* stream)
{
    clear_error();
    CTR_TRY(need(b, "batch"));
    for (auto* s : b->scans) CTR_TRY(ctr_solver_set_volume(s, nullptr, stream));
    return CTR_OK;
}

extern "C" ctr_status ctr_batch_iterate(ctr_batch* b, int n, double* obj_out, void* stream)
{
    clear_error();
    CTR_TRY(need(b, "batch"));
    if (n < 0) return set_error(CTR_ERR_INVALID_ARGUMENT, "n < 0");
    const int ns = (int)b->scans.size();
    for (int i = 0; i < ns; ++i)
        if (!b->scans[i]->sino) return set_error(CTR_ERR_INVALID_ARGUMENT, "scan %d has no sinogram", i);
    cudaStream_t st = S(stream);
    const bool objective = b->scans[0]->p.objective != 0;
    // the objective of iteration it is projected in iteration it+1's SART
    // traversal (graph 1); the last one of the call separately
    auto obj_rows = [&](int it) -> ctr_status {
        if (!obj_out) return CTR_OK;
        std::vector<double> h(2 * (size_t)ns);
        for (int i = 0; i < ns; ++i)
            CTR_CUDA_TRY(cudaMemcpyAsync(&h[2 * i], b->scans[i]->d_obj, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
        CTR_CUDA_TRY(cudaStreamSynchronize(st));
        for (int i = 0; i < ns; ++i) {
            const ctr_solver* s = b->scans[i];
            double* o = obj_out + ((size_t)i * n + it) * 3;
            o[0] = h[2 * i + 1];
            o[1] = h[2 * i];
            o[2] = h[2 * i] + 2.0 * (double)s->p.lambda_tv * h[2 * i + 1];   // V63/main_recon.cu:423
        }
        return CTR_OK;
    };
    for (int it = 0; it < n; ++it) {
        const int gi = (objective && it > 0) ? 1 : 0;
        if (b->exec[gi] && b->ws[gi] != batch_workspaces(b)) batch_drop_graph(b, gi);   // grown by another call
        if (!b->exec[gi]) CTR_TRY(batch_capture(b, gi));
        for (int i = 0; i < ns; ++i) {
            ctr_solver* s = b->scans[i];
            const float t_k = (1.0f + sqrtf(1.0f + 4.0f * s->t * s->t)) / 2.0f;   // V63/main_recon.cu:372
            // the momentum of this iteration, or for a refinement solver the
            // factor of y_k that its pass projects (set by the previous iteration)
            b->h_gam[i] = s->refine ? s->gm : (s->t - 1.0f) / t_k;
            b->h_seed[i] = (uint32_t)(s->k + 1);   // the single-scan solver's seed of this pass
        }
        CTR_CUDA_TRY(cudaMemcpyAsync(b->d_gam, b->h_gam.data(), sizeof(float) * ns, cudaMemcpyHostToDevice, st));
        CTR_CUDA_TRY(cudaMemcpyAsync(b->d_seed, b->h_seed.data(), sizeof(uint32_t) * ns, cudaMemcpyHostToDevice, st));
        CTR_CUDA_TRY(cudaGraphLaunch(b->exec[gi], st));
        for (auto* s : b->scans) {
            if (s->p.fista) {
                const float t_k = (1.0f + sqrtf(1.0f + 4.0f * s->t * s->t)) / 2.0f;
                if (s->refine) s->gm = (s->t - 1.0f) / t_k;
                s->t = t_k;
            }
            s->k++;
        }
        if (gi == 1) CTR_TRY(obj_rows(it - 1));
    }
    if (n > 0) {
        if (objective) {
            for (auto* s : b->scans) {
                const void* xk = s->p.fista ? s->xprev : s->y;
                if (s->refine) CTR_TRY(refine_objective(s, st));
                else CTR_TRY(objective_async(s->g, xk, s->vdt, s->sino, s->sdt, s->d_obj, s->d_obj + 1, st, s->yt));
            }
            CTR_TRY(obj_rows(n - 1));
        } else if (obj_out) {
            for (size_t i = 0; i < (size_t)ns * n * 3; ++i) obj_out[i] = NAN;
        }
    }
    for (auto* s : b->scans) CTR_TRY(check_device_errors(s->g, st));
    if (b->persistent) {   // a barrier wait of the persistent pass that gave up
        unsigned h = 0;
        CTR_CUDA_TRY(cudaMemcpyAsync(&h, b->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        CTR_CUDA_TRY(cudaStreamSynchronize(st));
        if (h) {
            CTR_CUDA_TRY(cudaMemset(b->d_err, 0, sizeof(unsigned)));
            return set_error(CTR_ERR_TIMEOUT, "the persistent pass's barrier wait gave up (error word %u)", h);
        }
    }
    return CTR_OK;
}

extern "C" ctr_status ctr_batch_get_volume(ctr_batch* b, int scan, void* dst, void* stream)
{
    clear_error();
    CTR_TRY(need(b, "batch"));
    if (scan < 0 || scan >= (int)b->scans.size()) return set_error(CTR_ERR_INVALID_ARGUMENT, "scan %d out of range", scan);
    return ctr_solver_get_volume(b->scans[scan], dst, stream);
}

extern "C" ctr_status ctr_batch_get_volume_f32(ctr_batch* b, int scan, float* dst, void* stream)
{
    clear_error();
    CTR_TRY(need(b, "batch"));
    if (scan < 0 || scan >= (int)b->scans.size()) return set_error(CTR_ERR_INVALID_ARGUMENT, "scan %d out of range", scan);
    return ctr_solver_get_volume_f32(b->scans[scan], dst, stream);
}

// -------------------------------------------- reference-compatible entry points

namespace {
std::mutex g_default_mu;
Geometry* g_default = nullptr;
int g_default_devices = 1;   // Number_of_Devices of the replaced build

// device copy of a host or device buffer
struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
};

ctr_status in_dev(DevBuf& b, const void* src, size_t bytes)
{
    CTR_CUDA_TRY(cudaMalloc(&b.p, bytes));
    if (src) CTR_CUDA_TRY(cudaMemcpy(b.p, src, bytes, cudaMemcpyDefault));
    return CTR_OK;
}
}  // namespace

extern "C" ctr_status ctr_set_default_geometry(const ctr_geometry_desc* desc)
{
    std::lock_guard<std::mutex> lk(g_default_mu);
    ctr_geometry* g = nullptr;
    CTR_TRY(ctr_geometry_create(desc, &g));
    if (g_default) ctr_geometry_destroy(reinterpret_cast<ctr_geometry*>(g_default));
    g_default = GE(g);
    return CTR_OK;
}

extern "C" ctr_status ctr_set_default_devices(int n)
{
    clear_error();
    if (n < 1) return set_error(CTR_ERR_INVALID_ARGUMENT, "Number_of_Devices must be >= 1");
    std::lock_guard<std::mutex> lk(g_default_mu);
    g_default_devices = n;
    return CTR_OK;
}

static Geometry* default_geom()
{
    if (!g_default) set_error(CTR_ERR_INVALID_ARGUMENT, "ctr_set_default_geometry() has not been called");
    return g_default;
}

extern "C" void Forward_3D_ray_driven_siddon(float* h_volume, float* h_proj_data)
{
    clear_error();
    Geometry* g = default_geom();
    if (!g || !h_volume || !h_proj_data) { if (g) set_error(CTR_ERR_INVALID_ARGUMENT, "NULL argument"); return; }
    const size_t vb = g->nvox() * 4, pb = (size_t)g->npix() * g->desc.n_views * 4;
    DevBuf v, p;
    if (in_dev(v, h_volume, vb) != CTR_OK || in_dev(p, nullptr, pb) != CTR_OK) return;
    Geometry* fg = g;
    if (g_default_devices > 1 && g->dg.ct_style == 3) {
        // the tetrahedron beam's n-device build projects with its row-split projector
        // (T42/voxel/host_IterativeRecon_TBCT_voxel_multiGPU.c:185-306)
        std::vector<Geometry*> sl;
        if (slab_geoms(g, g_default_devices, sl) != CTR_OK) return;
        fg = g->split_geom;
    }
    ctr_geometry* gg = reinterpret_cast<ctr_geometry*>(fg);
    if (ctr_forward(gg, v.p, CTR_F32, p.p, CTR_F32, 0, g->desc.n_views, nullptr) != CTR_OK) return;
    cudaError_t e = cudaMemcpy(h_proj_data, p.p, pb, cudaMemcpyDefault);
    if (e != cudaSuccess) cuda_error(e, "Forward_3D_ray_driven_siddon");
}

extern "C" void Reconstruction_3D_ray_driven_CBCT(float* h_volume, float* h_proj_data, float beta)
{
    clear_error();
    Geometry* g = default_geom();
    if (!g || !h_volume || !h_proj_data) { if (g) set_error(CTR_ERR_INVALID_ARGUMENT, "NULL argument"); return; }
    const size_t vb = g->nvox() * 4, pb = (size_t)g->npix() * g->desc.n_views * 4;
    DevBuf v, p;
    if (in_dev(v, h_volume, vb) != CTR_OK || in_dev(p, h_proj_data, pb) != CTR_OK) return;
    // the reference's own backprojection arithmetic: the drop-in returns the reference's numbers;
    // for an n-device build its z-slab sequence (V63/host_IterativeRecon_CBCT_multiGPU.c:1-161)
    ctr_geometry* gg = reinterpret_cast<ctr_geometry*>(g);
    const ctr_status st = g_default_devices > 1
                              ? ctr_sart_pass_slabs(gg, g_default_devices, v.p, CTR_F32, p.p, CTR_F32, beta,
                                                    CTR_SART_REFERENCE_BP, 0, 0, g->desc.n_views, nullptr)
                              : ctr_sart_pass(gg, v.p, CTR_F32, p.p, CTR_F32, beta, CTR_SART_REFERENCE_BP, 0, nullptr);
    if (st != CTR_OK) return;
    cudaError_t e = cudaMemcpy(h_volume, v.p, vb, cudaMemcpyDefault);
    if (e != cudaSuccess) { cuda_error(e, "Reconstruction_3D_ray_driven_CBCT"); return; }
    if (check_device_errors(g, nullptr) != CTR_OK || g_default_devices <= 1) return;
    for (Geometry* sg : g->slab_geoms)   // the slabs' projectors keep their own error words
        if (check_device_errors(sg, nullptr) != CTR_OK) return;
}

extern "C" void CheckMatchedJointOperator(float* h_volume)
{
    clear_error();
    Geometry* g = default_geom();
    if (!g || !h_volume) { if (g) set_error(CTR_ERR_INVALID_ARGUMENT, "NULL argument"); return; }
    const size_t vb = g->nvox() * 4, pb = (size_t)g->npix() * 4;
    DevBuf v, p, bp;
    if (in_dev(v, h_volume, vb) != CTR_OK || in_dev(p, nullptr, pb) != CTR_OK || in_dev(bp, nullptr, vb) != CTR_OK) return;
    ctr_geometry* gg = reinterpret_cast<ctr_geometry*>(g);
    if (cudaMemset(bp.p, 0, vb) != cudaSuccess) return;
    if (g_default_devices > 1) {
        // the n-device build (V63/host_IterativeRecon_CBCT_multiGPU.c:296-412): y = the slabs'
        // weighted sums added in order (no threshold), then each slab's command-0 backprojection
        std::vector<Geometry*> sl;
        if (slab_geoms(g, g_default_devices, sl) != CTR_OK) return;
        const int D = (int)sl.size();
        const long long P = g->npix();
        if (ensure_parts(g, (size_t)P * D * sizeof(float2)) != CTR_OK) return;
        for (int i = 0; i < D; ++i)
            if (ctr_forward_partial(reinterpret_cast<ctr_geometry*>(sl[i]), (const float*)v.p + sl[0]->nvox() * i,
                                    CTR_F32, 0, (float*)g->d_parts + 2 * P * i, 0, nullptr) != CTR_OK)
                return;
        if (launch_combine(*g, (const float2*)g->d_parts, D, 0, nullptr, CTR_F32, (float2*)p.p, nullptr) != CTR_OK)
            return;
        for (int i = 0; i < D; ++i)
            if (ctr_backproject(reinterpret_cast<ctr_geometry*>(sl[i]), (const float*)p.p, 0, 1,
                                (float*)bp.p + sl[0]->nvox() * i, CTR_F32, CTR_BP_FOV_MASK, nullptr) != CTR_OK)
                return;
    } else {
        // view 0: y = A x (command 0), z = A^T y with the reference's masked command-0 BP
        if (ctr_forward(gg, v.p, CTR_F32, p.p, CTR_F32, 0, 1, nullptr) != CTR_OK) return;
        if (ctr_backproject(gg, (const float*)p.p, 0, 1, bp.p, CTR_F32, CTR_BP_FOV_MASK, nullptr) != CTR_OK) return;
    }
    std::vector<float> hy(g->npix()), hz(g->nvox());
    if (cudaMemcpy(hy.data(), p.p, pb, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(hz.data(), bp.p, vb, cudaMemcpyDeviceToHost) != cudaSuccess) return;
    double ip1 = 0.0, ip2 = 0.0;   // V63/host_IterativeRecon_CBCT.c:186-197
    for (size_t i = 0; i < hy.size(); ++i) ip1 += (double)hy[i] * (double)hy[i];
    for (size_t i = 0; i < hz.size(); ++i) ip2 += (double)h_volume[i] * (double)hz[i];
    printf("The 1st inner product = %f\n", ip1);
    printf("The 2nd inner product = %f\n", ip2);
}

extern "C" void FGP_denoise_GPUx7_exact(float* h_f, float lambda, int niter)
{
    clear_error();
    Geometry* g = default_geom();
    if (!g || !h_f) { if (g) set_error(CTR_ERR_INVALID_ARGUMENT, "NULL argument"); return; }
    const size_t vb = g->nvox() * 4;
    DevBuf v;
    if (in_dev(v, h_f, vb) != CTR_OK) return;
    if (ctr_fgp_tv(reinterpret_cast<ctr_geometry*>(g), v.p, CTR_F32, lambda, niter, nullptr) != CTR_OK) return;
    cudaError_t e = cudaMemcpy(h_f, v.p, vb, cudaMemcpyDefault);
    if (e != cudaSuccess) cuda_error(e, "FGP_denoise_GPUx7_exact");
}

extern "C" void Reconstruction_FDK(float* h_volume, float* h_proj)
{
    clear_error();
    Geometry* g = default_geom();
    if (!g || !h_volume || !h_proj) { if (g) set_error(CTR_ERR_INVALID_ARGUMENT, "NULL argument"); return; }
    const size_t vb = g->nvox() * 4, pb = (size_t)g->npix() * g->desc.n_views * 4;
    DevBuf v, p;
    if (in_dev(v, h_volume, vb) != CTR_OK || in_dev(p, h_proj, pb) != CTR_OK) return;
    if (ctr_fdk(reinterpret_cast<ctr_geometry*>(g), (const float*)p.p, (float*)v.p, nullptr) != CTR_OK) return;
    cudaError_t e = cudaMemcpy(h_volume, v.p, vb, cudaMemcpyDefault);
    if (e != cudaSuccess) cuda_error(e, "Reconstruction_FDK");
}

extern "C" double L2_norm_gpu(float* d_a, float* d_b)
{
    clear_error();
    Geometry* g = default_geom();
    if (!g || !d_a || !d_b) { if (g) set_error(CTR_ERR_INVALID_ARGUMENT, "NULL argument"); return NAN; }
    const size_t n = (size_t)g->npix() * g->desc.n_views;
    DevBuf a, b;
    if (in_dev(a, d_a, n * 4) != CTR_OK || in_dev(b, d_b, n * 4) != CTR_OK) return NAN;
    double r = NAN;
    if (ctr_l2_norm((const float*)a.p, (const float*)b.p, (int64_t)n, &r, nullptr) != CTR_OK) return NAN;
    return r;
}

extern "C" double TV_norm_gpu(float* d_volume)
{
    clear_error();
    Geometry* g = default_geom();
    if (!g || !d_volume) { if (g) set_error(CTR_ERR_INVALID_ARGUMENT, "NULL argument"); return NAN; }
    DevBuf v;
    if (in_dev(v, d_volume, g->nvox() * 4) != CTR_OK) return NAN;
    double r = NAN;
    if (ctr_tv_norm(reinterpret_cast<ctr_geometry*>(g), v.p, CTR_F32, &r, nullptr) != CTR_OK) return NAN;
    return r;
}
