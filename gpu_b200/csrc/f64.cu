// f64.cu -- the FP64 reference solver.
//
// The solver's iteration -- a SART pass over all views in order, FGP-TV,
// FISTA momentum, the objective -- with every step in double precision on the
// device, for stating the error of the FP32 and mixed-precision solvers at
// full size.  The steps follow the reference's call sequence
// (V63/main_recon.cu:344-430, V63/host_IterativeRecon_CBCT.c:1-67) with exact
// geometry instead of the reference's float rounding:
//   * forward projection: a Siddon traversal per ray with FP64 alphas, from
//     the detector pixel centre (alpha = 0) to the source (alpha = 1), the
//     geometry of V63/kernel_IterativeRecon_universal.cu:21-45 and 77-104;
//     the SART correction (b - sum)/len, zero below vx*1e-6 (:554-562);
//   * SART update: per voxel inside the reconstruction cylinder (:626-628),
//     every detector pixel in the bounding rectangle of the voxel's corner
//     projections (:639-706) contributes the geometric chord of its ray
//     through the voxel (slab intersection in FP64), f += beta*Sum(w c)/Sum(w)
//     where Sum(w) >= vx*1e-6 (:799-807).  The chord is the traversal's
//     segment in exact arithmetic, so the update is the projector's adjoint;
//   * FGP-TV (V63/kernel_FGP_Denoise_GPUx7.cu:2-88), FISTA (main_recon.cu:
//     372-382, t in FP64) and the objective (host_tool_functions.cu:28-101)
//     in FP64.
// Cone beam only.  Rays lying exactly on a voxel plane are counted in
// neither neighbour (a measure-zero case of odd detectors at axis angles).
#include <algorithm>
#include <new>

#include "ctr_device.cuh"

namespace ctr {

// Geometry in FP64 from the description (V63/main_recon.cu:60-111 without the
// float rounding).
struct G64 {
    int M, N, Z, R, ZP, nviews;
    double vx, vy, vz, bx, by, bz;
    double du, dv, ymin, zmin, dso, dod, srcy;
    double thr;            // vx*1e-6: the zero-length thresholds
    double us, a0, shift;  // degrees
};

// The projector frame's view angle -(j*us_rate + initial + shift) in radians,
// evaluated on the host (V63/host_IterativeRecon_CBCT.c:34-41 in FP64).
static void view_sc(const G64& h, int j, double& s, double& c)
{
    const double t = -((j * h.us + h.a0) + h.shift) * (3.14159265358979323846 / 180.0);
    s = std::sin(t);
    c = std::cos(t);
}

// Ray of pixel (u, v): detector pixel centre X1 and the direction X2 - X1.
struct Ray64 {
    double x1[3], d[3];
};
__device__ __forceinline__ Ray64 ray64(const G64& h, double s, double c, int u, int v)
{
    Ray64 r;
    const double pu = h.ymin + u * h.du;
    r.x1[0] = h.dod * c - pu * s;
    r.x1[1] = h.dod * s + pu * c;
    r.x1[2] = h.zmin + v * h.dv;
    const double x2x = h.dso * c - h.srcy * s, x2y = h.dso * s + h.srcy * c;
    r.d[0] = x2x - r.x1[0];
    r.d[1] = x2y - r.x1[1];
    r.d[2] = 0.0 - r.x1[2];
    return r;
}

// Siddon traversal of one ray over vol (FP64): returns Sum(len*f), len in *len_out.
__device__ double traverse64(const G64& h, const Ray64& r, const double* __restrict__ vol, double* len_out)
{
    const double P0[3] = {h.bx, h.by, h.bz};
    const double VV[3] = {h.vx, h.vy, h.vz};
    const int NN[3] = {h.M, h.N, h.Z};
    double amin = -INFINITY, amax = INFINITY;
    double inv[3];
    int dir[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        dir[a] = r.d[a] > 0.0 ? 1 : (r.d[a] < 0.0 ? -1 : 0);
        if (fabs(r.d[a]) < VV[a] * 1e-12) {   // parallel to the axis's planes
            dir[a] = 0;
            inv[a] = 0.0;
            if (r.x1[a] <= P0[a] || r.x1[a] >= P0[a] + VV[a] * NN[a]) { *len_out = 0.0; return 0.0; }
            continue;
        }
        inv[a] = 1.0 / r.d[a];
        const double t0 = (P0[a] - r.x1[a]) * inv[a], t1 = (P0[a] + VV[a] * NN[a] - r.x1[a]) * inv[a];
        amin = fmax(amin, fmin(t0, t1));
        amax = fmin(amax, fmax(t0, t1));
    }
    double sum = 0.0, len = 0.0;
    if (amax > amin) {
        const double d12 = sqrt(r.d[0] * r.d[0] + r.d[1] * r.d[1] + r.d[2] * r.d[2]);
        int vox[3];
        double an[3];
        // the voxel holding the entry point, taken just inside the volume
        const double ain = amin + 1e-9 * (amax - amin);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double x = r.x1[a] + ain * r.d[a];
            int iv = (int)floor((x - P0[a]) / VV[a]);
            iv = min(max(iv, 0), NN[a] - 1);
            vox[a] = iv;
            an[a] = dir[a] == 0 ? INFINITY : (P0[a] + VV[a] * (iv + (dir[a] > 0)) - r.x1[a]) * inv[a];
        }
        double ac = amin;
        const long long MN = (long long)h.M * h.N;
        for (int step = 0; step < h.M + h.N + h.Z + 3 && ac < amax; ++step) {
            double m = fmin(fmin(an[0], an[1]), an[2]);
            if (m > amax) m = amax;
            const double seg = d12 * (m - ac);
            len += seg;
            if (vol) sum += seg * vol[(long long)vox[2] * MN + (long long)vox[1] * h.M + vox[0]];
            ac = m;
            bool out = false;
#pragma unroll
            for (int a = 0; a < 3; ++a)
                if (an[a] == m) {
                    vox[a] += dir[a];
                    out |= vox[a] < 0 || vox[a] >= NN[a];
                    an[a] = (P0[a] + VV[a] * (vox[a] + (dir[a] > 0)) - r.x1[a]) * inv[a];
                }
            if (out) break;
        }
    }
    *len_out = len;
    return sum;
}

// MODE 0: SART correction and chord length per ray, rays[p] = (c, d12).
// MODE 1: objective partials, one per warp of 32 rays: Sum((Ax - b)^2).
template <int MODE>
__global__ void __launch_bounds__(128)
k64_forward(const G64 h, const double* __restrict__ vol, double s, double c, const void* __restrict__ b, int b_dt,
            double2* __restrict__ rays, double* __restrict__ partial)
{
    const int u = blockIdx.x * 32 + (threadIdx.x & 31);
    const int v = blockIdx.y * 4 + (threadIdx.x >> 5);
    double e2 = 0.0;
    if (u < h.R && v < h.ZP) {
        const Ray64 r = ray64(h, s, c, u, v);
        double len;
        const double sum = traverse64(h, r, vol, &len);
        const long long p = (long long)v * h.R + u;
        const double bv = (double)ld_any(b, p, b_dt);
        if (MODE == 0) {
            const double d12 = sqrt(r.d[0] * r.d[0] + r.d[1] * r.d[1] + r.d[2] * r.d[2]);
            rays[p] = make_double2(len < h.thr ? 0.0 : (bv - sum) / len, d12);
        } else {
            const double e = (len < h.thr ? 0.0 : sum) - bv;
            e2 = e * e;
        }
    }
    if (MODE == 1) {
        for (int o = 16; o > 0; o >>= 1) e2 += __shfl_down_sync(0xffffffffu, e2, o);
        if ((threadIdx.x & 31) == 0) partial[((size_t)v) * gridDim.x + blockIdx.x] = e2;
    }
}

// Per detector column u of a view: the pixel centre's x and y and the
// reciprocals of the ray's x and y extents (0 for an extent below 1e-12 of a
// voxel: a ray parallel to those planes); per detector row v (the same for
// every view): the pixel centre's z and 1/(z extent), 0 likewise.
__global__ void k64_columns(const G64 h, double s, double c, double4* __restrict__ col)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= h.R) return;
    const double pu = h.ymin + u * h.du;
    const double x1x = h.dod * c - pu * s, x1y = h.dod * s + pu * c;
    const double dx = (h.dso * c - h.srcy * s) - x1x, dy = (h.dso * s + h.srcy * c) - x1y;
    col[u] = make_double4(x1x, x1y, fabs(dx) < h.vx * 1e-12 ? 0.0 : 1.0 / dx, fabs(dy) < h.vy * 1e-12 ? 0.0 : 1.0 / dy);
}
__global__ void k64_rows(const G64 h, double2* __restrict__ row)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= h.ZP) return;
    const double x1z = h.zmin + v * h.dv, dz = 0.0 - x1z;
    row[v] = make_double2(x1z, fabs(dz) < h.vz * 1e-12 ? 0.0 : 1.0 / dz);
}

// The alpha interval of a ray inside the slab [lo, hi] of one axis (x1 the
// ray's start on that axis, inv 1/extent, 0 for a ray parallel to the slab):
// (-inf, inf) inside, empty (returned false) outside.
__device__ __forceinline__ bool slab64(double lo, double hi, double x1, double inv, double& a, double& b)
{
    if (inv == 0.0) {
        a = -INFINITY;
        b = INFINITY;
        return x1 > lo && x1 < hi;
    }
    const double t0 = (lo - x1) * inv, t1 = (hi - x1) * inv;
    a = fmin(t0, t1);
    b = fmax(t0, t1);
    return true;
}

constexpr int F64_RUN = 4;    // detector columns of a voxel column kept in registers
constexpr int F64_ZRUN = 16;  // voxels of a column per thread

// SART update of one view (gather, no atomics): a thread walks F64_ZRUN
// voxels of one (x, y) column.  Per column: the reconstruction cylinder test
// (the reference's float test, universal.cu:626-628), the detector columns
// between the corner projections (rounded to the nearest pixel, a superset
// of the pixel centres the column projects to) and their rays' xy alpha
// intervals; per voxel: the detector rows between its corner projections
// (the magnification's extremes over the column) and, per (row, column), the
// geometric chord d12*(exit - entry).  f += beta*Sum(w c)/Sum(w) where
// Sum(w) >= vx*1e-6.
__global__ void __launch_bounds__(128)
k64_update(const G64 h, const DevGeom g, double* __restrict__ vol, const double2* __restrict__ rays, double s,
           double c, const double4* __restrict__ col, const double2* __restrict__ row, double beta)
{
    const int i = blockIdx.x * 32 + (threadIdx.x & 31);
    const int j = blockIdx.y * 4 + (threadIdx.x >> 5);
    if (i >= h.M || j >= h.N) return;
    const float ex = fs(fs((float)i, g.fov_h_x), g.m_off);
    const float ey = fs((float)j, g.fov_h_y);
    if (fa(fm(fm(fm(ex, g.vx), ex), g.vx), fm(fm(fm(ey, g.vy), ey), g.vy)) >= g.fov_r2) return;
    const double xl = h.bx + i * h.vx, xh = xl + h.vx;
    const double yl = h.by + j * h.vy, yh = yl + h.vy;
    double umin = INFINITY, umax = -INFINITY, mlo = INFINITY, mhi = -INFINITY;
    const double sdd = h.dso - h.dod;
#pragma unroll
    for (int cc = 0; cc < 4; ++cc) {
        const double x = (cc & 1) ? xh : xl, y = (cc >> 1) ? yh : yl;
        const double t = x * c + y * s, ss = -x * s + y * c;
        const double mag = sdd / (h.dso - t);
        const double up = h.srcy + (ss - h.srcy) * mag;
        umin = fmin(umin, up); umax = fmax(umax, up);
        mlo = fmin(mlo, mag); mhi = fmax(mhi, mag);
    }
    const int ulo = max((int)floor((umin - h.ymin) / h.du + 0.5), 0);
    const int uhi = min((int)floor((umax - h.ymin) / h.du + 0.5), h.R - 1);
    if (ulo > uhi) return;
    const int nrun = uhi - ulo + 1;
    double ra[F64_RUN], rb[F64_RUN];
#pragma unroll
    for (int q = 0; q < F64_RUN; ++q) {
        ra[q] = 1.0; rb[q] = 0.0;   // empty
        if (q < nrun) {
            const double4 ct = col[ulo + q];
            double a0, b0, a1, b1;
            const bool in = slab64(xl, xh, ct.x, ct.z, a0, b0) & slab64(yl, yh, ct.y, ct.w, a1, b1);
            if (in) { ra[q] = fmax(a0, a1); rb[q] = fmin(b0, b1); }
        }
    }
    const int kb = blockIdx.z * F64_ZRUN, ke = min(h.Z, kb + F64_ZRUN);
    const double vscale = 1.0 / h.dv;
    for (int k = kb; k < ke; ++k) {
        const double zl = h.bz + k * h.vz, zh = zl + h.vz;
        const double vmin = fmin(fmin(zl * mlo, zl * mhi), fmin(zh * mlo, zh * mhi));
        const double vmax = fmax(fmax(zl * mlo, zl * mhi), fmax(zh * mlo, zh * mhi));
        const int vlo = max((int)floor((vmin - h.zmin) * vscale + 0.5), 0);
        const int vhi = min((int)floor((vmax - h.zmin) * vscale + 0.5), h.ZP - 1);
        double W = 0.0, L = 0.0;
        for (int v = vlo; v <= vhi; ++v) {
            const double2 rt = row[v];
            double za, zb;
            if (!slab64(zl, zh, rt.x, rt.y, za, zb)) continue;
            const double2* __restrict__ rr = rays + (long long)v * h.R + ulo;
            for (int q = 0; q < nrun; ++q) {
                double a, b;
                if (q < F64_RUN) {
                    a = ra[q]; b = rb[q];
                } else {
                    const double4 ct = col[ulo + q];
                    double a0, b0, a1, b1;
                    const bool in = slab64(xl, xh, ct.x, ct.z, a0, b0) & slab64(yl, yh, ct.y, ct.w, a1, b1);
                    a = in ? fmax(a0, a1) : 1.0;
                    b = in ? fmin(b0, b1) : 0.0;
                }
                const double lo = fmax(a, za), hi = fmin(b, zb);
                if (!(hi > lo)) continue;
                const double2 rc = rr[q];
                const double w = rc.y * (hi - lo);
                W += w * rc.x;
                L += w;
            }
        }
        if (L >= h.thr) vol[((long long)k * h.N + j) * h.M + i] += beta * W / L;
    }
}

// FGP-TV in FP64 on one-voxel duals (r, s, t, o, p, q): r[p] belongs to the
// edge (x, x+1) and is 0 at x = nx-1, likewise s along y and t along z
// (V63/host_FGP_Denoise_GPUx7.c:8-38's zero-padded duals).
__device__ __forceinline__ double fgp_L64(const double* __restrict__ f, const double* __restrict__ r,
                                          const double* __restrict__ s, const double* __restrict__ t, int x, int y,
                                          int z, long long p, int M, long long MN, double lambda)
{
    const double tl = (r[p] - (x > 0 ? r[p - 1] : 0.0)) + (s[p] - (y > 0 ? s[p - M] : 0.0)) +
                      (t[p] - (z > 0 ? t[p - MN] : 0.0));
    return f[p] - lambda * tl;
}

__global__ void __launch_bounds__(256)
k64_fgp_L(int M, int N, int Z, const double* __restrict__ f, const double* __restrict__ r,
          const double* __restrict__ s, const double* __restrict__ t, double* __restrict__ L, double lambda)
{
    const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    if (x >= M || y >= N) return;
    const long long MN = (long long)M * N, p = (long long)z * MN + (long long)y * M + x;
    L[p] = fgp_L64(f, r, s, t, x, y, z, p, M, MN, lambda);
}

__global__ void __launch_bounds__(256)
k64_fgp_dual(int M, int N, int Z, const double* __restrict__ L, double* __restrict__ r, double* __restrict__ s,
             double* __restrict__ t, double* __restrict__ o, double* __restrict__ pd, double* __restrict__ q,
             double alpha12, double gam)
{
    const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    if (x >= M || y >= N) return;
    const long long MN = (long long)M * N, p = (long long)z * MN + (long long)y * M + x;
    const double Lc = L[p];
    double tr = r[p], ts = s[p], tt = t[p];
    if (x < M - 1) tr += alpha12 * (Lc - L[p + 1]);
    if (y < N - 1) ts += alpha12 * (Lc - L[p + M]);
    if (z < Z - 1) tt += alpha12 * (Lc - L[p + MN]);
    const double den = fmax(1.0, sqrt(tr * tr + ts * ts + tt * tt));
    if (x < M - 1) { const double on = tr / den; r[p] = on + gam * (on - o[p]); o[p] = on; }
    if (y < N - 1) { const double pn = ts / den; s[p] = pn + gam * (pn - pd[p]); pd[p] = pn; }
    if (z < Z - 1) { const double qn = tt / den; t[p] = qn + gam * (qn - q[p]); q[p] = qn; }
}

// x* = the prox (FGP) or x itself; with FISTA y = x* + gam (x* - xprev),
// xprev = x*; without, y = x*.
template <bool FGP>
__global__ void __launch_bounds__(256)
k64_final(long long n, int M, int N, double* __restrict__ y, double* __restrict__ xprev, const double* __restrict__ o,
          const double* __restrict__ pd, const double* __restrict__ q, double lambda, int fista, double gam)
{
    const long long MN = (long long)M * N;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(p % M), yy = (int)((p / M) % N), z = (int)(p / MN);
        const double xs = FGP ? fgp_L64(y, o, pd, q, x, yy, z, p, M, MN, lambda) : y[p];
        if (fista) {
            y[p] = xs + gam * (xs - xprev[p]);
            xprev[p] = xs;
        } else {
            y[p] = xs;
        }
    }
}

// TV_norm_kernel (V63/kernel_tool_functions.cu:39-65) in FP64, block partials.
__global__ void __launch_bounds__(256) k64_tv(int M, int N, int Z, const double* __restrict__ d, double* __restrict__ part)
{
    __shared__ double sh[8];
    const long long MN = (long long)M * N, n = MN * Z;
    double acc = 0.0;
    for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) {
        const int x = (int)(i % M), y = (int)((i / M) % N), z = (int)(i / MN);
        const bool bx = x < M - 1, by = y < N - 1, bz = z < Z - 1;
        const double dj = bx ? d[i] - d[i + 1] : 0.0, dk = by ? d[i] - d[i + M] : 0.0, dl = bz ? d[i] - d[i + MN] : 0.0;
        const int nb = (int)bx + (int)by + (int)bz;
        if (nb >= 2) acc += sqrt(dj * dj + dk * dk + dl * dl);
        else if (nb == 1) acc += fabs(dj + dk + dl);
    }
    const double t = block_sum(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

template <typename S>
__global__ void k64_convert(const S* __restrict__ src, double* __restrict__ dst, long long n)
{
    for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) dst[i] = (double)src[i];
}
__global__ void k64_to_f32(const double* __restrict__ src, float* __restrict__ dst, long long n)
{
    for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) dst[i] = (float)src[i];
}

struct F64Solver {
    Geometry* g = nullptr;
    ctr_solver_params p{};
    G64 h{};
    double* y = nullptr;       // working volume: y_k, then x_k during an iteration
    double* xprev = nullptr;   // x_(k-1); after an iteration with FISTA, x_k
    double* work = nullptr;    // FGP: six duals and L (7 volumes)
    double2* rays = nullptr;   // one view's (c, d12)
    double4* col = nullptr;    // one view's column table (k64_columns)
    double2* row = nullptr;    // the row table (k64_rows)
    double* partial = nullptr;
    size_t partial_cap = 0;
    double t = 1.0;
    int k = 0;
};

static int grid64(long long n)
{
    long long b = (n + 255) / 256;
    if (b > 148LL * 32) b = 148LL * 32;
    return (int)(b < 1 ? 1 : b);
}

ctr_status f64_create(Geometry* g, const ctr_solver_params& p, F64Solver** out)
{
    const ctr_geometry_desc& d = g->desc;
    if (g->dg.ct_style != 0 || g->dg.slab_n > 1)
        return set_error(CTR_ERR_UNSUPPORTED, "the FP64 solver supports the whole-volume cone beam only");
    F64Solver* s = new (std::nothrow) F64Solver();
    if (!s) return set_error(CTR_ERR_OUT_OF_MEMORY, "host allocation");
    s->g = g;
    s->p = p;
    G64& h = s->h;
    h.M = d.nx; h.N = d.ny; h.Z = d.nz; h.R = d.nu; h.ZP = d.nv; h.nviews = d.n_views;
    h.vx = g->dg.vx; h.vy = g->dg.vy; h.vz = g->dg.vz;   // the pitches as given (floats)
    h.bx = -h.vx * ((double)d.nx / 2.0 + (double)d.m_offset);
    h.by = -h.vy * ((double)d.ny / 2.0);
    h.bz = -h.vz * ((double)d.nz / 2.0);
    h.du = g->dg.du; h.dv = g->dg.dv;
    h.ymin = -h.du * ((double)d.nu / 2.0 - 0.5) + (double)d.offset;
    h.zmin = -h.dv * ((double)d.nv / 2.0 - 0.5);
    h.dso = d.dso; h.dod = d.dod; h.srcy = d.offset;
    h.thr = h.vx * 1e-6;
    h.us = d.us_rate; h.a0 = d.initial_angle; h.shift = d.shift_angle;
    const long long V = g->nvox();
    const size_t P = (size_t)g->npix();
    // objective: one partial per warp of a padded 4-row block grid; TV: block partials
    s->partial_cap = std::max<size_t>((size_t)(h.ZP + 4) * ((h.R + 31) / 32), 148 * 32) + 2048;
    cudaError_t e;
    if ((e = cudaMalloc(&s->y, V * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&s->xprev, V * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&s->rays, P * sizeof(double2))) != cudaSuccess ||
        (e = cudaMalloc(&s->col, (size_t)h.R * sizeof(double4))) != cudaSuccess ||
        (e = cudaMalloc(&s->row, (size_t)h.ZP * sizeof(double2))) != cudaSuccess ||
        (e = cudaMalloc(&s->partial, s->partial_cap * sizeof(double))) != cudaSuccess ||
        (e = cudaMemset(s->y, 0, V * sizeof(double))) != cudaSuccess ||
        (e = cudaMemset(s->xprev, 0, V * sizeof(double))) != cudaSuccess) {
        f64_destroy(s);
        return cuda_error(e, "FP64 solver allocation");
    }
    k64_rows<<<(h.ZP + 127) / 128, 128>>>(h, s->row);
    if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaDeviceSynchronize()) != cudaSuccess) {
        f64_destroy(s);
        return cuda_error(e, "FP64 solver row table");
    }
    *out = s;
    return CTR_OK;
}

void f64_destroy(F64Solver* s)
{
    if (!s) return;
    cudaFree(s->y);
    cudaFree(s->xprev);
    cudaFree(s->work);
    cudaFree(s->rays);
    cudaFree(s->col);
    cudaFree(s->row);
    cudaFree(s->partial);
    delete s;
}

ctr_status f64_set_volume(F64Solver* s, const double* vol, cudaStream_t st)
{
    const size_t bytes = s->g->nvox() * sizeof(double);
    if (vol) {
        CTR_CUDA_TRY(cudaMemcpyAsync(s->y, vol, bytes, cudaMemcpyDefault, st));
        CTR_CUDA_TRY(cudaMemcpyAsync(s->xprev, vol, bytes, cudaMemcpyDefault, st));
    } else {
        CTR_CUDA_TRY(cudaMemsetAsync(s->y, 0, bytes, st));
        CTR_CUDA_TRY(cudaMemsetAsync(s->xprev, 0, bytes, st));
    }
    s->t = 1.0;
    s->k = 0;
    return CTR_OK;
}

int f64_iteration(const F64Solver* s) { return s->k; }

// Sum(Ax - b)^2 and TV of x, both FP64, synchronised.
static ctr_status f64_objective(F64Solver* s, const double* x, const void* sino, ctr_dtype sdt, double* fid,
                                double* tv, cudaStream_t st)
{
    const G64& h = s->h;
    const dim3 grid((h.R + 31) / 32, (h.ZP + 3) / 4);
    const size_t per_view = (size_t)grid.x * grid.y * 4;
    const long long P = (long long)h.R * h.ZP;
    std::vector<double> part(per_view);
    double f = 0.0;
    for (int j = 0; j < h.nviews; ++j) {
        double vs, vc;
        view_sc(h, j, vs, vc);
        k64_forward<1><<<grid, 128, 0, st>>>(h, x, vs, vc, (const char*)sino + (size_t)j * P * dtype_size(sdt), sdt,
                                             nullptr, s->partial);
        CTR_CUDA_TRY(cudaGetLastError());
        CTR_CUDA_TRY(cudaMemcpyAsync(part.data(), s->partial, per_view * sizeof(double), cudaMemcpyDeviceToHost, st));
        CTR_CUDA_TRY(cudaStreamSynchronize(st));
        for (int r = 0; r < h.ZP; ++r)   // the warps of each row, in order
            for (unsigned b = 0; b < grid.x; ++b) f += part[(size_t)r * grid.x + b];
    }
    const long long V = s->g->nvox();
    const int nb = grid64(V);
    k64_tv<<<nb, 256, 0, st>>>(h.M, h.N, h.Z, x, s->partial);
    CTR_CUDA_TRY(cudaGetLastError());
    std::vector<double> tp(nb);
    CTR_CUDA_TRY(cudaMemcpyAsync(tp.data(), s->partial, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
    CTR_CUDA_TRY(cudaStreamSynchronize(st));
    double t = 0.0;
    for (int b = 0; b < nb; ++b) t += tp[b];
    *fid = f;
    *tv = t;
    return CTR_OK;
}

ctr_status f64_iterate(F64Solver* s, const void* sino, ctr_dtype sdt, int n, double* obj_out, cudaStream_t st)
{
    const G64& h = s->h;
    Geometry* g = s->g;
    const long long V = g->nvox();
    const long long P = (long long)h.R * h.ZP;
    const double beta = s->p.beta;
    const double lam = (double)s->p.beta * (double)s->p.lambda_tv;   // lambda_denoise_TV = 2*lambda_TV/Lip
    const bool fgp = s->p.lambda_tv > 0.f && s->p.fgp_iters >= 0;
    if (fgp && !s->work) CTR_CUDA_TRY(cudaMalloc(&s->work, 7 * (size_t)V * sizeof(double)));
    const dim3 fgrid((h.R + 31) / 32, (h.ZP + 3) / 4);
    const dim3 bgrid((h.M + 31) / 32, (h.N + 3) / 4, (h.Z + F64_ZRUN - 1) / F64_ZRUN);
    const dim3 vblk(32, 8), vgrid((h.M + 31) / 32, (h.N + 7) / 8, h.Z);
    for (int it = 0; it < n; ++it) {
        // SART pass on y (V63/host_IterativeRecon_CBCT.c:1-67)
        for (int j = 0; j < h.nviews; ++j) {
            double vs, vc;
            view_sc(h, j, vs, vc);
            k64_forward<0><<<fgrid, 128, 0, st>>>(h, s->y, vs, vc, (const char*)sino + (size_t)j * P * dtype_size(sdt),
                                                  sdt, s->rays, nullptr);
            k64_columns<<<(h.R + 127) / 128, 128, 0, st>>>(h, vs, vc, s->col);
            k64_update<<<bgrid, 128, 0, st>>>(h, g->dg, s->y, s->rays, vs, vc, s->col, s->row, beta);
        }
        CTR_CUDA_TRY(cudaGetLastError());
        const double t_k = (1.0 + sqrt(1.0 + 4.0 * s->t * s->t)) / 2.0;   // V63/main_recon.cu:372
        const double gam = (s->t - 1.0) / t_k;
        const int fista = s->p.fista ? 1 : 0;
        if (fgp) {
            double* D[7];
            for (int q = 0; q < 7; ++q) D[q] = s->work + (size_t)q * V;   // r s t o p q L
            CTR_CUDA_TRY(cudaMemsetAsync(s->work, 0, 6 * (size_t)V * sizeof(double), st));
            const double alpha12 = 1.0 / (lam * 12.0);
            double tk1 = 1.0;
            for (int q = 0; q < s->p.fgp_iters; ++q) {
                const double tk = (1.0 + sqrt(1.0 + 4.0 * tk1 * tk1)) / 2.0;
                k64_fgp_L<<<vgrid, vblk, 0, st>>>(h.M, h.N, h.Z, s->y, D[0], D[1], D[2], D[6], lam);
                k64_fgp_dual<<<vgrid, vblk, 0, st>>>(h.M, h.N, h.Z, D[6], D[0], D[1], D[2], D[3], D[4], D[5], alpha12,
                                                     (tk1 - 1.0) / tk);
                tk1 = tk;
            }
            k64_final<true><<<grid64(V), 256, 0, st>>>(V, h.M, h.N, s->y, s->xprev, D[3], D[4], D[5], lam, fista, gam);
        } else {
            k64_final<false><<<grid64(V), 256, 0, st>>>(V, h.M, h.N, s->y, s->xprev, nullptr, nullptr, nullptr, 0.0,
                                                        fista, gam);
        }
        CTR_CUDA_TRY(cudaGetLastError());
        if (fista) s->t = t_k;
        s->k++;
        if (obj_out) {
            double* o = obj_out + 3 * (size_t)it;
            if (s->p.objective) {
                double fid = 0.0, tv = 0.0;
                CTR_TRY(f64_objective(s, fista ? s->xprev : s->y, sino, sdt, &fid, &tv, st));
                o[0] = tv;
                o[1] = fid;
                o[2] = fid + 2.0 * (double)s->p.lambda_tv * tv;   // V63/main_recon.cu:423
            } else {
                o[0] = o[1] = o[2] = NAN;
            }
        }
    }
    return CTR_OK;
}

ctr_status f64_get_volume(F64Solver* s, void* dst, bool as_f32, cudaStream_t st)
{
    const long long V = s->g->nvox();
    const double* x = (s->p.fista && s->k > 0) ? s->xprev : s->y;
    if (!as_f32) {
        CTR_CUDA_TRY(cudaMemcpyAsync(dst, x, V * sizeof(double), cudaMemcpyDefault, st));
    } else {
        float* tmp = nullptr;
        CTR_CUDA_TRY(cudaMalloc(&tmp, V * sizeof(float)));
        k64_to_f32<<<grid64(V), 256, 0, st>>>(x, tmp, V);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(dst, tmp, V * sizeof(float), cudaMemcpyDefault, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaFree(tmp);
        CTR_CUDA_TRY(e);
    }
    CTR_CUDA_TRY(cudaStreamSynchronize(st));
    return CTR_OK;
}

}  // namespace ctr
