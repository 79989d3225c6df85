// geometry.cpp -- scan geometry: validation, the reference's derived float
// constants, per-view and per-plane tables, error reporting and workspace.
//
// Compiled with -ffp-contract=off: every float expression here rounds as
// written, matching the reference's host and kernel arithmetic.
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <mutex>

#include "ctr_internal.h"

namespace ctr {

static thread_local std::string g_last_error;

ctr_status set_error(ctr_status st, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return st;
}

ctr_status cuda_error(cudaError_t e, const char* what)
{
    if (e == cudaErrorMemoryAllocation)
        return set_error(CTR_ERR_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
    return set_error(CTR_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

void clear_error() { g_last_error.clear(); }

static const float kPi = 3.141592653589793f;   // const float PI (V63/main_recon.cu:105)

// View angle of V63/host_IterativeRecon_CBCT.c:34-41 (fdk=false, negated) and
// V63/host_FDK.cpp:35-40 (fdk=true).
static void view_trig(const ctr_geometry_desc& d, int j, bool fdk, float* s, float* c)
{
    float t = (float)(j * d.us_rate + d.initial_angle);
    t = (t + d.shift_angle) * kPi / 180.0f;
    if (!fdk) t = -t;
    *s = std::sin(t);
    *c = std::cos(t);
}

// Voxel index the forward projector keeps along an axis to which a ray is
// (nearly) parallel: floor((x1 - b) * inv_v), the reference's i_max / i_min-1
// with the alpha_min*(x2-x1) term, which is exactly 0 for an exactly parallel
// ray (V63/kernel_IterativeRecon_universal.cu:131-143,178-183,271-284).
static int parallel_voxel(float x1, float b, float inv_v)
{
    return (int)std::floor((x1 - b) * inv_v);
}

static float plane(float v, int n, float b) { return v * (float)n + b; }

ctr_status ensure_rays(Geometry* g, size_t bytes)
{
    if (bytes <= g->rays_cap) return CTR_OK;
    if (g->d_rays) cudaFree(g->d_rays);
    g->d_rays = nullptr;
    g->rays_cap = 0;
    CTR_CUDA_TRY(cudaMalloc(&g->d_rays, bytes));
    g->rays_cap = bytes;
    return CTR_OK;
}

ctr_status ensure_partial(Geometry* g, size_t n)
{
    if (n <= g->partial_cap) return CTR_OK;
    if (g->d_partial) cudaFree(g->d_partial);
    g->d_partial = nullptr;
    g->partial_cap = 0;
    CTR_CUDA_TRY(cudaMalloc(&g->d_partial, n * sizeof(double)));
    g->partial_cap = n;
    return CTR_OK;
}

ctr_status ensure_fgp(Geometry* g, size_t bytes)
{
    if (bytes <= g->fgp_bytes) return CTR_OK;
    if (g->d_fgp) cudaFree(g->d_fgp);
    g->d_fgp = nullptr;
    g->fgp_bytes = 0;
    CTR_CUDA_TRY(cudaMalloc(&g->d_fgp, bytes));
    g->fgp_bytes = bytes;
    return CTR_OK;
}

ctr_status ensure_tiled(Geometry* g, size_t bytes)
{
    if (bytes <= g->tiled_bytes) return CTR_OK;
    if (g->d_tiled) cudaFree(g->d_tiled);
    g->d_tiled = nullptr;
    g->tiled_bytes = 0;
    CTR_CUDA_TRY(cudaMalloc(&g->d_tiled, bytes));
    g->tiled_bytes = bytes;
    return CTR_OK;
}

ctr_status check_device_errors(Geometry* g, cudaStream_t st)
{
    unsigned h = 0;
    CTR_CUDA_TRY(cudaMemcpyAsync(&h, g->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CTR_CUDA_TRY(cudaStreamSynchronize(st));
    if (h & ERR_TRAVERSAL) {
        CTR_CUDA_TRY(cudaMemsetAsync(g->d_err, 0, sizeof(unsigned), st));
        return set_error(CTR_ERR_TRAVERSAL_BOUND,
                         "a ray exceeded the Siddon step bound nx+ny+nz+3 (non-finite geometry?)");
    }
    return CTR_OK;
}

static ctr_status validate(const ctr_geometry_desc* d)
{
    if (!d) return set_error(CTR_ERR_INVALID_ARGUMENT, "geometry description is NULL");
    if (d->nx <= 0 || d->ny <= 0 || d->nz <= 0 || d->nu <= 0 || d->nv <= 0 || d->n_views <= 0)
        return set_error(CTR_ERR_BAD_GEOMETRY, "sizes must be positive (nx=%d ny=%d nz=%d nu=%d nv=%d views=%d)",
                         d->nx, d->ny, d->nz, d->nu, d->nv, d->n_views);
    const double vox = (double)((d->nx + 7) / 8 * 8) * ((d->ny + 7) / 8 * 8) * d->nz;   // tiled layout
    if (vox > 2147483647.0)
        return set_error(CTR_ERR_BAD_GEOMETRY, "volume of %.0f voxels exceeds the 2^31-1 index range", vox);
    const bool tbct = (d->flags & CTR_GEOM_TBCT) != 0;
    if (tbct && d->n_sources < 1) return set_error(CTR_ERR_BAD_GEOMETRY, "CTR_GEOM_TBCT needs n_sources >= 1");
    const double rows = (double)d->nv * (tbct ? d->n_sources : 1);
    if ((double)d->nu * rows > 2147483647.0)
        return set_error(CTR_ERR_BAD_GEOMETRY, "detector too large");
    if (!(d->vx > 0.f) || !(d->du > 0.f) || !std::isfinite(d->vx) || !std::isfinite(d->du))
        return set_error(CTR_ERR_BAD_GEOMETRY, "voxel and detector pitch must be positive and finite");
    // vy, vz, dv: 0 or below selects the x / u pitch; a given one must be finite
    if (!std::isfinite(d->vy) || !std::isfinite(d->vz) || !std::isfinite(d->dv))
        return set_error(CTR_ERR_BAD_GEOMETRY, "vy, vz and dv must be finite (0 selects the x or u pitch)");
    // the projector's and the update's thresholds are 1e-6 of a voxel pitch
    // (universal.cu:554, :785, :799); a pitch whose threshold rounds to 0 in
    // float would let a ray or a voxel with no chord divide by zero
    const float vz_used = d->vz > 0.f ? d->vz : d->vx;
    if (!(d->vx * 1e-6f > 0.f) || !(vz_used * 1e-6f > 0.f))
        return set_error(CTR_ERR_BAD_GEOMETRY, "voxel pitch too small: 1e-6 of it rounds to 0 in float");
    if (!(d->dso > 0.f) || !std::isfinite(d->dso) || !std::isfinite(d->dod) || !(d->dod < d->dso))
        return set_error(CTR_ERR_BAD_GEOMETRY, "need 0 < dso and dod < dso (detector opposite the source)");
    if (!std::isfinite(d->us_rate) || !std::isfinite(d->initial_angle) || !std::isfinite(d->shift_angle) ||
        !std::isfinite(d->offset))
        return set_error(CTR_ERR_BAD_GEOMETRY, "angles and offset must be finite");
    // the volume must sit strictly between source and detector planes along every view
    const double vy = d->vy > 0.f ? d->vy : d->vx;
    const double half_diag = 0.5 * std::sqrt((double)d->nx * d->vx * d->nx * d->vx + (double)d->ny * vy * d->ny * vy) +
                             std::fabs((double)d->m_offset * d->vx);
    if (half_diag >= d->dso || half_diag >= -d->dod)
        return set_error(CTR_ERR_BAD_GEOMETRY, "volume (half-diagonal %.4g) reaches the source or detector", half_diag);
    const int styles = ((d->flags & CTR_GEOM_FAN_SLICES) ? 1 : 0) + ((d->flags & CTR_GEOM_PARALLEL) ? 1 : 0) +
                       (tbct ? 1 : 0);
    if (styles > 1)
        return set_error(CTR_ERR_BAD_GEOMETRY, "CTR_GEOM_FAN_SLICES, CTR_GEOM_PARALLEL and CTR_GEOM_TBCT exclude each other");
    if (tbct && ((d->vz > 0.f && d->vz != d->vx) || (d->dv > 0.f && d->dv != d->du)))
        return set_error(CTR_ERR_BAD_GEOMETRY, "CTR_GEOM_TBCT needs vz = vx and dv = du (the reference's single pitches)");
    if (d->nx > 65535 || d->ny > 65535 * 8 || d->nz > 65535 || rows > 65535.0 * 4)
        return set_error(CTR_ERR_BAD_GEOMETRY, "dimension exceeds the launch limits");
    return CTR_OK;
}

}  // namespace ctr

using namespace ctr;

// The whole volume (n_slabs = 1) or slab `slab` of the n_slabs-way z split of
// the multi-GPU build.
static ctr_status create(const ctr_geometry_desc* din, int n_slabs, int slab, ctr_geometry** out)
{
    clear_error();
    if (!out) return set_error(CTR_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    CTR_TRY(validate(din));
    if (n_slabs < 1 || slab < (n_slabs > 1 ? -1 : 0) || slab >= n_slabs)
        return set_error(CTR_ERR_INVALID_ARGUMENT, "slab %d of %d", slab, n_slabs);
    if (n_slabs > 1) {
        // V63/main_recon.cu:24, T42/main_recon.cu:18: volume height and detector rows split evenly
        if (din->nz % n_slabs != 0 || din->nv % n_slabs != 0)
            return set_error(CTR_ERR_BAD_GEOMETRY, "nz=%d and nv=%d must both split into %d slabs", din->nz, din->nv,
                             n_slabs);
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return set_error(CTR_ERR_NO_DEVICE, "no CUDA device");
    Geometry* g = new (std::nothrow) Geometry();
    if (!g) return set_error(CTR_ERR_OUT_OF_MEMORY, "host allocation");
    ctr_geometry_desc d = *din;
    if (!(d.vy > 0.f)) d.vy = d.vx;
    if (!(d.vz > 0.f)) d.vz = d.vx;
    if (!(d.dv > 0.f)) d.dv = d.du;
    g->desc = d;
    cudaGetDevice(&g->device);

    DevGeom& q = g->dg;
    const bool tbct = (d.flags & CTR_GEOM_TBCT) != 0;
    if (!tbct) d.n_sources = 0;
    g->desc.n_sources = d.n_sources;
    q.nsrc = tbct ? d.n_sources : 1;
    q.nvr = d.nv;
    q.M = d.nx; q.N = d.ny; q.Z = d.nz; q.R = d.nu; q.ZP = d.nv * q.nsrc; q.nviews = d.n_views;
    q.max_steps = d.nx + d.ny + d.nz + 3;
    q.Mt = (d.nx + 7) / 8;
    q.Nt = (d.ny + 7) / 8;
    {
        // alpha of a point = its distance from the detector plane / (DSO - DOD);
        // the volume's nearest point is at least -DOD - (half-diagonal) away
        const double half_diag = 0.5 * std::sqrt((double)d.nx * d.vx * d.nx * d.vx + (double)d.ny * d.vy * d.ny * d.vy) +
                                 std::fabs((double)d.m_offset * d.vx);
        // (the tetrahedron beam's loop test, alpha_max - alpha_c > 1e-6f, has no one-comparison
        // form; its multi-GPU build's projectors test against 1e-16f, as V63's)
        const bool inside = (-(double)d.dod - half_diag) / ((double)d.dso - (double)d.dod) >= 1e-6;
        q.fast_exit = ((!tbct || n_slabs > 1) && inside) ? 1 : 0;
    }
    q.entry64 = (d.flags & CTR_GEOM_ENTRY_F64) ? 1 : 0;
    q.fast_sums = (d.flags & CTR_GEOM_FAST_SUMS) ? 1 : 0;
    q.ct_style = tbct ? 3 : ((d.flags & CTR_GEOM_FAN_SLICES) ? 1 : ((d.flags & CTR_GEOM_PARALLEL) ? 2 : 0));
    // T42/...TBCT_voxel.cu:282, V63/...universal.cu:291, T42/..._multiGPU.cu:303,853
    q.loop_eps = (tbct && n_slabs == 1) ? 1e-6f : 1e-16f;
    q.vx = d.vx; q.vy = d.vy; q.vz = d.vz;
    // inv_volumn_x = 1.0/volumn_x (double division stored as float), main_recon.cu:88
    q.inv_vx = (float)(1.0 / (double)d.vx);
    q.inv_vy = (float)(1.0 / (double)d.vy);
    q.inv_vz = (float)(1.0 / (double)d.vz);
    // boundary_voxel_* (main_recon.cu:90,94,98)
    q.bx = -d.vx * ((float)d.nx / 2.0f + (float)d.m_offset);
    q.by = -d.vy * ((float)d.ny / 2.0f);
    q.bz = -d.vz * ((float)d.nz / 2.0f);
    // the slab of the multi-GPU build (V63/kernel_IterativeRecon_universal_multiGPU.cu):
    // BOUNDARY_VOXEL_Z = boundary_voxel_z + volumn_z*ZETA/D*subVolIdx and ZETA/D
    // slices in the projector (:636-637), the backprojector's voxel centre
    // boundary_voxel_z + volumn_z*(ZETA/D*subVolIdx + 0.5f) + k*volumn_z (:1179)
    q.slab_n = n_slabs;
    q.slab_i = slab;
    q.bz_ref = q.bz;
    q.cz_off = d.vz * 0.5f;
    q.ref_plus0 = 1;
    q.zpar_kr = tbct ? 0 : 1;
    q.row_lo = 0;
    q.row_hi = q.ZP;
    q.thr_comb = tbct ? d.vz * 1e-3f : d.vz * 1e-6f;
    if (n_slabs > 1 && slab == -1) {
        // the whole volume as the n-device build's row-split projector traverses it
        // (V63/..._multiGPU.cu:21-590, T42/voxel/..._multiGPU.cu:22-576): V63's rules,
        // so the tetrahedron beam gains the z-parallel k range; a whole-volume geometry otherwise
        q.zpar_kr = 1;
        q.slab_n = 1;
        q.slab_i = 0;
    } else if (n_slabs > 1) {
        const int zs = d.nz / n_slabs, k0 = zs * slab;
        q.bz = q.bz_ref + d.vz * (float)d.nz / (float)n_slabs * (float)slab;
        q.cz_off = d.vz * ((float)k0 + 0.5f);
        q.ref_plus0 = 0;   // :1388-1391
        q.zpar_kr = 0;     // :775-800
        if (q.ct_style == 1 || q.ct_style == 2) {   // :663
            q.row_lo = d.nv / n_slabs * slab;
            q.row_hi = d.nv / n_slabs * (slab + 1);
        } else if (q.ct_style == 0) {
            // Cone beam: the rows whose rays can reach the slab at any view.  A
            // point at alpha of a ray lies at DOD + alpha*(DSO-DOD) along the
            // view's axis and at height x1z*(1-alpha) (the source at z = 0), and
            // the volume lies within its xy half-diagonal of the axis, so inside
            // the volume alpha is in [a_lo, a_hi].  Rows whose heights over that
            // range stay a voxel clear of the slab miss it geometrically and the
            // projector gives them (0, 0); the band keeps two rows of margin.
            const double rv = 0.5 * std::sqrt((double)d.nx * d.vx * d.nx * d.vx + (double)d.ny * d.vy * d.ny * d.vy) +
                              std::fabs((double)d.m_offset * d.vx);
            const double a_lo = (-rv - d.dod) / ((double)d.dso - d.dod), a_hi = (rv - d.dod) / ((double)d.dso - d.dod);
            const double zlo = (double)q.bz - d.vz, zhi = (double)q.bz + (double)zs * d.vz + d.vz;
            const float zmin = -d.dv * ((float)d.nv / 2.0f - 0.5f);   // Detector_Zmin, set below
            int lo = d.nv, hi = -1;
            for (int v = 0; v < d.nv; ++v) {
                const double x1z = (double)zmin + (double)v * d.dv;
                const double z0 = x1z * (1.0 - a_hi), z1 = x1z * (1.0 - a_lo);
                if (std::max(z0, z1) >= zlo && std::min(z0, z1) <= zhi) {
                    lo = std::min(lo, v);
                    hi = v;
                }
            }
            q.row_lo = lo <= hi ? std::max(0, lo - 2) : 0;
            q.row_hi = lo <= hi ? std::min(d.nv, hi + 3) : 0;
        }
        d.nz = zs;
        g->desc.nz = zs;
        q.Z = zs;
        q.max_steps = d.nx + d.ny + zs + 3;
    }
    // Detector_Ymin / Detector_Zmin (main_recon.cu:83-84)
    q.ymin = -d.du * ((float)d.nu / 2.0f - 0.5f) + d.offset;
    q.zmin = -d.dv * ((float)d.nv / 2.0f - 0.5f);
    q.du = d.du; q.dv = d.dv;
    q.inv_du = 1.0f / d.du;        // inv_Detector_pixel (universal.cu:615)
    q.inv_dv = 1.0f / d.dv;
    q.dso = d.dso; q.dod = d.dod;
    q.srcx = d.dso; q.srcy = d.offset; q.srcz = 0.0f;   // main_recon.cu:101-103
    q.dsod = d.dso - d.dod;
    q.zmax = +d.du * ((float)d.nv / 2.0f - 0.5f);        // T42/main_recon.cu:93
    q.zsrc0 = 0.0f;
    q.zsrc_dz = 0.0f;
    if (tbct && d.n_sources > 1) {                        // T42/main_recon.cu:76, :104-107
        // placed from the whole volume's faces (din->nz, bz_ref), also for a slab
        const float bzu = -d.vz * ((float)din->nz / 2.0f) + (float)din->nz * d.vz;
        const float zsmax = (bzu - q.zmax) * (d.dso - d.dod) / d.dso + q.zmax;
        q.zsrc0 = (q.bz_ref - q.zmin) * (d.dso - d.dod) / d.dso + q.zmin;
        q.zsrc_dz = (zsmax - q.zsrc0) / (float)(d.n_sources - 1);
        if (!(q.zsrc_dz > 0.f)) {
            delete g;
            return set_error(CTR_ERR_BAD_GEOMETRY, "CTR_GEOM_TBCT: the source spacing is not positive "
                                                   "(detector band taller than the magnified volume)");
        }
    }
    {
        // T42/...TBCT_voxel.cu:772 compares the float sum with the double
        // volumn_x*1e-3: the same as comparing with the largest float <= it
        const double t = (double)d.vx * 1e-3;
        float f = (float)t;
        if ((double)f > t) f = std::nextafter(f, -INFINITY);
        q.thr_upd = f;
    }
    q.thr_fp = d.vz * 1e-6f;       // universal.cu:554
    q.thr_bp = d.vx * 1e-6f;       // universal.cu:785,799
    q.fov_h_x = (float)d.nx * 0.5f - 0.5f;
    q.fov_h_y = (float)d.ny * 0.5f - 0.5f;
    q.fov_r2 = q.fov_h_x * d.vx * q.fov_h_y * d.vy;   // universal.cu:628
    q.m_off = (float)d.m_offset;
    q.fdk_ang = d.us_rate * kPi / 180.0f;
    q.fdk_usn = d.us_rate * (float)d.n_views;
    q.fdk_full = q.fdk_usn == 360.0f ? 1 : 0;

    // plane tables: px[n+1] = volumn_x*n + boundary_voxel_x, n = -1..M+1
    g->h_px.resize(d.nx + 3);
    g->h_py.resize(d.ny + 3);
    g->h_pz.resize(d.nz + 3);
    for (int n = -1; n <= d.nx + 1; ++n) g->h_px[n + 1] = plane(d.vx, n, q.bx);
    for (int n = -1; n <= d.ny + 1; ++n) g->h_py[n + 1] = plane(d.vy, n, q.by);
    for (int n = -1; n <= d.nz + 1; ++n) g->h_pz[n + 1] = plane(d.vz, n, q.bz);

    g->h_trig.resize(d.n_views);
    g->h_trig_fdk.resize(d.n_views);
    for (int j = 0; j < d.n_views; ++j) {
        view_trig(d, j, false, &g->h_trig[j].x, &g->h_trig[j].y);
        view_trig(d, j, true, &g->h_trig_fdk[j].x, &g->h_trig_fdk[j].y);
    }

    // BP column table: per view and detector column the forward projector's
    // own x1 and 1/(x2-x1) for x and y.  An axis to which the ray is parallel
    // (|x1-x2| < v*1e-6, where the projector keeps alpha = inf and a fixed voxel)
    // is encoded as x1 = centre of that voxel, 1/d = +inf, so that the gather
    // backprojector sees the interval (-inf, +inf) for that voxel only.
    const float INF = INFINITY;
    std::vector<float4> colt((size_t)d.n_views * d.nu);
    for (int j = 0; j < d.n_views; ++j) {
        const float s = g->h_trig[j].x, c = g->h_trig[j].y;
        for (int u = 0; u < d.nu; ++u) {
            const float pu = q.ymin + (float)u * q.du;
            const float sy = q.ct_style == 2 ? pu : q.srcy;   // parallel beam: a source per column
            const float x2x = q.srcx * c - sy * s;
            const float x2y = q.srcx * s + sy * c;
            const float x1x = q.dod * c - pu * s;
            const float x1y = q.dod * s + pu * c;
            float4 e;
            if (std::fabs(x1x - x2x) < q.vx * 1e-6f) {
                const int iv = parallel_voxel(x1x, q.bx, q.inv_vx);
                e.x = plane(q.vx, iv, q.bx) + 0.5f * q.vx;
                e.y = INF;
            } else {
                e.x = x1x;
                e.y = 1.0f / (x2x - x1x);
            }
            if (std::fabs(x1y - x2y) < q.vy * 1e-6f) {
                const int jv = parallel_voxel(x1y, q.by, q.inv_vy);
                e.z = plane(q.vy, jv, q.by) + 0.5f * q.vy;
                e.w = INF;
            } else {
                e.z = x1y;
                e.w = 1.0f / (x2y - x1y);
            }
            colt[(size_t)j * d.nu + u] = e;
        }
    }
    // BP row table: x1z and 1/(x2z-x1z) per detector row, same encoding.
    std::vector<float2> rowt(q.ZP);
    for (int v = 0; v < q.ZP; ++v) {
        const int src = v / q.nvr, vr = v - src * q.nvr;
        const float x1z = q.zmin + (float)vr * q.dv;
        // fan slices, parallel beam: rows parallel to xy; tetrahedron beam: the band's source
        const float x2z = q.ct_style == 3 ? q.zsrc0 + (float)src * q.zsrc_dz : (q.ct_style == 0 ? q.srcz : x1z);
        if (std::fabs(x1z - x2z) < q.vz * 1e-6f) {
            const int kv = parallel_voxel(x1z, q.bz, q.inv_vz);
            rowt[v].x = plane(q.vz, kv, q.bz) + 0.5f * q.vz;
            rowt[v].y = INF;
        } else {
            rowt[v].x = x1z;
            rowt[v].y = 1.0f / (x2z - x1z);
        }
    }

    // one device block for the small tables
    const size_t n_px = g->h_px.size(), n_py = g->h_py.size(), n_pz = g->h_pz.size();
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t o_px = 0, o_py = o_px + al(n_px * 4), o_pz = o_py + al(n_py * 4),
                 o_tr = o_pz + al(n_pz * 4), o_tf = o_tr + al(d.n_views * 8),
                 o_row = o_tf + al(d.n_views * 8), total = o_row + al((size_t)q.ZP * 8);
    ctr_status st = CTR_OK;
    char* base = nullptr;
    cudaError_t e;
    if ((e = cudaMalloc(&g->d_tables, total)) != cudaSuccess) { st = cuda_error(e, "cudaMalloc(tables)"); goto fail; }
    base = (char*)g->d_tables;
    if ((e = cudaMemcpy(base + o_px, g->h_px.data(), n_px * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(base + o_py, g->h_py.data(), n_py * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(base + o_pz, g->h_pz.data(), n_pz * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(base + o_tr, g->h_trig.data(), d.n_views * 8, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(base + o_tf, g->h_trig_fdk.data(), d.n_views * 8, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(base + o_row, rowt.data(), (size_t)q.ZP * 8, cudaMemcpyHostToDevice)) != cudaSuccess) {
        st = cuda_error(e, "cudaMemcpy(tables)");
        goto fail;
    }
    if ((e = cudaMalloc(&g->d_colt, colt.size() * sizeof(float4))) != cudaSuccess) { st = cuda_error(e, "cudaMalloc(colt)"); goto fail; }
    if ((e = cudaMemcpy(g->d_colt, colt.data(), colt.size() * sizeof(float4), cudaMemcpyHostToDevice)) != cudaSuccess) {
        st = cuda_error(e, "cudaMemcpy(colt)");
        goto fail;
    }
    if ((e = cudaMalloc(&g->d_err, 256)) != cudaSuccess) { st = cuda_error(e, "cudaMalloc(err)"); goto fail; }
    if ((e = cudaMemset(g->d_err, 0, 256)) != cudaSuccess) { st = cuda_error(e, "cudaMemset(err)"); goto fail; }
    if ((e = cudaMalloc(&g->d_result, 8 * sizeof(double))) != cudaSuccess) { st = cuda_error(e, "cudaMalloc(result)"); goto fail; }
    q.px = (const float*)(base + o_px);
    q.py = (const float*)(base + o_py);
    q.pz = (const float*)(base + o_pz);
    q.trig = (const float2*)(base + o_tr);
    q.trig_fdk = (const float2*)(base + o_tf);
    q.rowt = (const float2*)(base + o_row);
    q.colt = g->d_colt;
    q.err = g->d_err;
    if ((e = cudaMalloc(&g->d_zcell, sizeof(float2) * (size_t)d.nz * q.ZP)) != cudaSuccess) {
        st = cuda_error(e, "cudaMalloc(zcell)");
        goto fail;
    }
    if ((st = launch_zcell(*g, g->d_zcell, 0)) != CTR_OK) goto fail;
    if ((e = cudaMalloc(&g->d_zref, sizeof(float2) * (size_t)d.nz * q.ZP)) != cudaSuccess) {
        st = cuda_error(e, "cudaMalloc(zref)");
        goto fail;
    }
    if ((st = launch_zref(*g, g->d_zref, 0)) != CTR_OK) goto fail;
    q.zref = g->d_zref;
    if ((e = cudaStreamSynchronize(0)) != cudaSuccess) { st = cuda_error(e, "zcell"); goto fail; }
    q.zcell = g->d_zcell;
    *out = reinterpret_cast<ctr_geometry*>(g);
    return CTR_OK;
fail:
    ctr_geometry_destroy(reinterpret_cast<ctr_geometry*>(g));
    return st;
}

extern "C" ctr_status ctr_geometry_create(const ctr_geometry_desc* din, ctr_geometry** out)
{
    return create(din, 1, 0, out);
}

extern "C" ctr_status ctr_geometry_create_slab(const ctr_geometry_desc* din, int n_slabs, int slab,
                                               ctr_geometry** out)
{
    return create(din, n_slabs, slab, out);
}

extern "C" ctr_status ctr_geometry_slab(const ctr_geometry* geom, int* n_slabs, int* slab, int* k0)
{
    if (!geom) return set_error(CTR_ERR_INVALID_ARGUMENT, "geometry is NULL");
    const Geometry* g = reinterpret_cast<const Geometry*>(geom);
    if (n_slabs) *n_slabs = g->dg.slab_n;
    if (slab) *slab = g->dg.slab_i;
    if (k0) *k0 = g->dg.Z * g->dg.slab_i;
    return CTR_OK;
}

extern "C" ctr_status ctr_geometry_destroy(ctr_geometry* geom)
{
    if (!geom) return CTR_OK;
    Geometry* g = reinterpret_cast<Geometry*>(geom);
    cudaFree(g->d_tables);
    cudaFree(g->d_colt);
    cudaFree(g->d_zcell);
    cudaFree(g->d_zref);
    cudaFree(g->d_err);
    cudaFree(g->d_rays);
    cudaFree(g->d_partial);
    cudaFree(g->d_result);
    cudaFree(g->d_fgp);
    cudaFree(g->d_fdk);
    cudaFree(g->d_tiled);
    cudaFree(g->d_ramp);
    cudaFree(g->d_parts);
    if (g->split_geom) ctr_geometry_destroy(reinterpret_cast<ctr_geometry*>(g->split_geom));
    for (cudaStream_t q : g->slab_streams) cudaStreamDestroy(q);
    for (cudaEvent_t e : g->slab_events) cudaEventDestroy(e);
    for (Geometry* sg : g->slab_geoms) ctr_geometry_destroy(reinterpret_cast<ctr_geometry*>(sg));
    delete g;
    return CTR_OK;
}

extern "C" ctr_status ctr_geometry_view_trig(const ctr_geometry* geom, int view, float* s, float* c)
{
    if (!geom || !s || !c) return set_error(CTR_ERR_INVALID_ARGUMENT, "NULL argument");
    const Geometry* g = reinterpret_cast<const Geometry*>(geom);
    if (view < 0 || view >= g->desc.n_views) return set_error(CTR_ERR_INVALID_ARGUMENT, "view %d out of range", view);
    *s = g->h_trig[view].x;
    *c = g->h_trig[view].y;
    return CTR_OK;
}

extern "C" const char* ctr_last_error_string(void) { return ctr::g_last_error.c_str(); }
