// fp_kernels.cuh -- Siddon ray-driven forward projector for sm_100a (the
// kernel templates; fp.cu holds the launcher, fp_<type>.cu the instances).
//
// One ray per thread.  The traversal restates forward_ray_driven_3d_kernel_
// correction (V63/kernel_IterativeRecon_universal.cu:7-567) with IEEE float
// operations in the reference's order, so the voxel index sequence of every
// ray and its float ray sum are bit-identical to the reference compiled for
// the CPU.  Differences from the reference kernel are in organisation only:
//   * the seven tie branches become "advance every axis whose next-plane
//     alpha equals the minimum" (the same rule for non-NaN alphas), executed
//     branch-free, which keeps the 32 lanes of a warp converged;
//   * the plane coordinates volumn*n+boundary come from shared-memory tables;
//   * the loop also ends when a voxel index leaves the volume.  Every step
//     moves at least one index one voxel in its fixed direction (the minimum
//     of non-NaN alphas equals one of them; all-NaN alphas end the loop), so
//     a ray takes at most nx+ny+nz+1 steps: the reference's endless loop on
//     NaN alphas cannot occur.  After the first step the whole test is one
//     comparison of alpha against a per-ray limit (see the loop);
//   * blocks are issued centre-out over the detector, so the long rays
//     through the middle of the volume start first and the last wave holds
//     short ones;
//   * the epilogue also writes the chord length of every ray (for the gather
//     backprojector), or reduces the squared residual in FP64 (objective).
#pragma once

#include <type_traits>

#include "ctr_device.cuh"

namespace ctr {

static constexpr int FP_BX = 32;   // rays along a detector row per block
static constexpr int FP_BY = 4;    // detector rows per block of the fixed-shape kernels
static constexpr int FP_THREADS = FP_BX * FP_BY;

// Tile t of n in centre-out order: c, c+1, c-1, c+2, c-2, ... (c = (n-1)/2),
// a bijection of [0, n).
__device__ __forceinline__ int centre_out(int t, int n)
{
    const int c = (n - 1) >> 1, d = (t + 1) >> 1;
    return (t & 1) ? c + d : c - d;
}
static constexpr uint64_t kFnvOffset = 1469598103934665603ULL;
static constexpr uint64_t kFnvPrime = 1099511628211ULL;

struct RayResult {
    float sum, len, d12;
    float sum2;         // the same segments over a second volume (DUAL only)
    double dsum;        // the same segments summed in FP64 (ACC64 only)
    float a_lo, a_hi;   // alpha interval the traversal covered (empty when it dropped the ray)
    int vi0, vj0, vk0;  // voxel the traversal starts in
    int par;            // axes the traversal treats as parallel (bit 0 x, 1 y, 2 z)
    int nseg;
    uint64_t hash;
};

// Shared plane tables with one padding entry before and after each table,
// then the +inf slot: 1 + (M+3) + 2 + (N+3) + 2 + (Z+3) + 1 + 1 floats.
__device__ __forceinline__ void plane_tables_addr(const DevGeom& g, float* sp, float*& PX, float*& PY, float*& PZ,
                                                  float*& PINF)
{
    PX = sp + 1;
    PY = PX + (g.M + 3) + 2;
    PZ = PY + (g.N + 3) + 2;
    PINF = PZ + (g.Z + 3) + 1;
}
__device__ __forceinline__ void plane_tables_layout(const DevGeom& g, float* sp, float*& PX, float*& PY, float*& PZ,
                                                    float*& PINF)
{
    plane_tables_addr(g, sp, PX, PY, PZ, PINF);
    for (int t = threadIdx.x; t < g.M + g.N + g.Z + 16; t += blockDim.x) sp[t] = 0.f;
    __syncthreads();
}
static size_t plane_tables_bytes(const DevGeom& g) { return sizeof(float) * (size_t)(g.M + g.N + g.Z + 16); }

// Floor of the position along an axis at parameter a, as a plane index
// (the reference's floor((a*(x2-x1) + x1 - b)*inv_v)).
__device__ __forceinline__ float pos_floor(float a, float d, float x1, float b, float inv_v)
{
    return floorf(fm(fs(fa(fm(a, d), x1), b), inv_v));
}

// LOAD=false walks the rays without reading the volume: it yields the chord
// lengths' support (a_lo, a_hi) for the matched adjoint.
// PINF points at a shared +inf: the next-plane table of an axis the ray is
// parallel to, so every axis can recompute its alpha unconditionally.
// CPM (bit 0 x, 1 y, 2 z): axes whose next plane is computed as
// volumn*n + boundary from a float plane counter instead of read from the
// shared table -- the same two roundings as the table entries, so the same
// alphas; it trades shared-memory traffic for arithmetic.  CPM == 8: every
// axis keeps the plane after its next one loaded ahead, so no shared-memory
// read sits between choosing a step and the next alpha.  The tables carry a
// padding entry at each end for those reads one plane past the volume.
// The voxel value loaded in a step is accumulated in the next step, so the
// load's latency overlaps the following traversal step; the sum is the same
// sequence of roundings.
// FAST (geometry flag CTR_GEOM_FAST_SUMS): the ray sum accumulates
// alpha-step x value with fused multiply-adds and applies d12 once at the
// end, and the chord length is d12 times the alpha span, three instructions
// fewer per step (four with a second volume); alphas, plane indices and the
// step rule are the same code, so every ray visits the same voxels.  The sums
// round differently from the reference's sequence (within 1e-5 relative).
template <typename VT, bool E64, bool TRACE, bool LOAD = true, bool ACC64 = false, int CPM = 0, bool TL = false,
          bool DUAL = false, bool FAST = false, bool COH = false, typename VT2 = VT>
__device__ __forceinline__ RayResult siddon(const DevGeom& g, const float* __restrict__ PX,
                                            const float* __restrict__ PY, const float* __restrict__ PZ,
                                            const float* __restrict__ PINF, const VT* __restrict__ vol, float s,
                                            float c, int u, int v, const VT2* __restrict__ vol2 = nullptr)
{
    const int M = g.M, N = g.N, Z = g.Z;
    RayResult r;
    r.sum = 0.f; r.sum2 = 0.f; r.len = 0.f; r.dsum = 0.0; r.nseg = 0; r.hash = kFnvOffset;
    r.a_lo = 1.0f; r.a_hi = 0.0f;
    r.vi0 = r.vj0 = r.vk0 = -1; r.par = 0;

    // source X2 and detector pixel centre X1 (universal.cu:21-45)
    const RayEnds re = ray_ends(g, s, c, u, v);
    const float x1x = re.x1x, x1y = re.x1y, x1z = re.x1z, x2x = re.x2x, x2y = re.x2y, x2z = re.x2z;
    const float dx = fs(x2x, x1x), dy = fs(x2y, x1y), dz = fs(x2z, x1z);
    const float ix = fdv(1.0f, dx), iy = fdv(1.0f, dy), iz = fdv(1.0f, dz);
    r.d12 = ray_d12(re);   // :290

    // alpha_min / alpha_max (:77-104); PX[n+1] is plane n
    float a0, a1;
    a0 = fm(fs(PX[1], x1x), ix); a1 = fm(fs(PX[M + 1], x1x), ix);
    const float axmin = fminf(a0, a1), axmax = fmaxf(a0, a1);
    a0 = fm(fs(PY[1], x1y), iy); a1 = fm(fs(PY[N + 1], x1y), iy);
    const float aymin = fminf(a0, a1), aymax = fmaxf(a0, a1);
    a0 = fm(fs(PZ[1], x1z), iz); a1 = fm(fs(PZ[Z + 1], x1z), iz);
    const float azmin = fminf(a0, a1), azmax = fmaxf(a0, a1);
    float amin = fmaxf(fmaxf(axmin, aymin), fmaxf(aymin, azmin));
    float amax = fminf(fminf(axmax, aymax), fminf(aymax, azmax));

    int i_min, i_max, j_min, j_max, k_min, k_max;
    bool hit;
    const bool zpar = fabsf(fs(x1z, x2z)) < fm(g.vz, 1e-6f);
    // T42 (T42/...TBCT_voxel.cu:171) and the multi-GPU build's slab projector
    // (V63/kernel_IterativeRecon_universal_multiGPU.cu:775-800) have no
    // z-parallel k range
    const bool zpar_k = zpar && g.zpar_kr;
    if (!E64) {
        hit = !(amax <= amin);
        if (!hit) return r;
        // first/last plane index per axis (:113-209)
        if (x1x < x2x) {
            i_min = (amin == axmin) ? 1 : __float2int_rz(fa(pos_floor(amin, dx, x1x, g.bx, g.inv_vx), 1.0f));
            i_max = (amax == axmax) ? M : __float2int_rz(pos_floor(amax, dx, x1x, g.bx, g.inv_vx));
        } else {
            i_max = (amin == axmin) ? M - 1 : __float2int_rz(pos_floor(amin, dx, x1x, g.bx, g.inv_vx));
            i_min = (amax == axmax) ? 0 : __float2int_rz(fa(pos_floor(amax, dx, x1x, g.bx, g.inv_vx), 1.0f));
        }
        if (x1y < x2y) {
            j_min = (amin == aymin) ? 1 : __float2int_rz(fa(pos_floor(amin, dy, x1y, g.by, g.inv_vy), 1.0f));
            j_max = (amax == aymax) ? N : __float2int_rz(pos_floor(amax, dy, x1y, g.by, g.inv_vy));
        } else {
            j_max = (amin == aymin) ? N - 1 : __float2int_rz(pos_floor(amin, dy, x1y, g.by, g.inv_vy));
            j_min = (amax == aymax) ? 0 : __float2int_rz(fa(pos_floor(amax, dy, x1y, g.by, g.inv_vy), 1.0f));
        }
        if (zpar_k) {
            const float fz = floorf(fm(fs(x1z, g.bz), g.inv_vz));
            k_min = __float2int_rz(fa(fz, 1.0f));
            k_max = __float2int_rz(fz);
        } else if (x1z < x2z) {
            k_min = (amin == azmin) ? 1 : __float2int_rz(fa(pos_floor(amin, dz, x1z, g.bz, g.inv_vz), 1.0f));
            k_max = (amax == azmax) ? Z : __float2int_rz(pos_floor(amax, dz, x1z, g.bz, g.inv_vz));
        } else {
            k_max = (amin == azmin) ? Z - 1 : __float2int_rz(pos_floor(amin, dz, x1z, g.bz, g.inv_vz));
            k_min = (amax == azmax) ? 0 : __float2int_rz(fa(pos_floor(amax, dz, x1z, g.bz, g.inv_vz), 1.0f));
        }
    } else {
        // FP64 ray-box entry/exit on the float positions; traversal stays float.
        const double X1x = x1x, X1y = x1y, X1z = x1z;
        const double Dx = (double)x2x - X1x, Dy = (double)x2y - X1y, Dz = (double)x2z - X1z;
        const double Ix = 1.0 / Dx, Iy = 1.0 / Dy, Iz = 1.0 / Dz;
        const double IVx = 1.0 / (double)g.vx, IVy = 1.0 / (double)g.vy, IVz = 1.0 / (double)g.vz;
        double b0, b1;
        b0 = ((double)PX[1] - X1x) * Ix; b1 = ((double)PX[M + 1] - X1x) * Ix;
        const double Axmin = fmin(b0, b1), Axmax = fmax(b0, b1);
        b0 = ((double)PY[1] - X1y) * Iy; b1 = ((double)PY[N + 1] - X1y) * Iy;
        const double Aymin = fmin(b0, b1), Aymax = fmax(b0, b1);
        b0 = ((double)PZ[1] - X1z) * Iz; b1 = ((double)PZ[Z + 1] - X1z) * Iz;
        const double Azmin = fmin(b0, b1), Azmax = fmax(b0, b1);
        const double Amin = fmax(fmax(Axmin, Aymin), Azmin);
        const double Amax = fmin(fmin(Axmax, Aymax), Azmax);
        hit = !(Amax <= Amin);
        if (!hit) return r;
        const double Bx = g.bx, By = g.by, Bz = g.bz;
        if (x1x < x2x) {
            i_min = (Amin == Axmin) ? 1 : (int)floor(__dmul_rn(__dsub_rn(__dadd_rn(__dmul_rn(Amin, Dx), X1x), Bx), IVx)) + 1;
            i_max = (Amax == Axmax) ? M : (int)floor(__dmul_rn(__dsub_rn(__dadd_rn(__dmul_rn(Amax, Dx), X1x), Bx), IVx));
        } else {
            i_max = (Amin == Axmin) ? M - 1 : (int)floor(__dmul_rn(__dsub_rn(__dadd_rn(__dmul_rn(Amin, Dx), X1x), Bx), IVx));
            i_min = (Amax == Axmax) ? 0 : (int)floor(__dmul_rn(__dsub_rn(__dadd_rn(__dmul_rn(Amax, Dx), X1x), Bx), IVx)) + 1;
        }
        if (x1y < x2y) {
            j_min = (Amin == Aymin) ? 1 : (int)floor(__dmul_rn(__dsub_rn(__dadd_rn(__dmul_rn(Amin, Dy), X1y), By), IVy)) + 1;
            j_max = (Amax == Aymax) ? N : (int)floor(__dmul_rn(__dsub_rn(__dadd_rn(__dmul_rn(Amax, Dy), X1y), By), IVy));
        } else {
            j_max = (Amin == Aymin) ? N - 1 : (int)floor(__dmul_rn(__dsub_rn(__dadd_rn(__dmul_rn(Amin, Dy), X1y), By), IVy));
            j_min = (Amax == Aymax) ? 0 : (int)floor(__dmul_rn(__dsub_rn(__dadd_rn(__dmul_rn(Amax, Dy), X1y), By), IVy)) + 1;
        }
        if (zpar_k) {
            k_min = (int)floor(__dmul_rn(__dsub_rn(X1z, Bz), IVz)) + 1;
            k_max = (int)floor(__dmul_rn(__dsub_rn(X1z, Bz), IVz));
        } else if (x1z < x2z) {
            k_min = (Amin == Azmin) ? 1 : (int)floor(__dmul_rn(__dsub_rn(__dadd_rn(__dmul_rn(Amin, Dz), X1z), Bz), IVz)) + 1;
            k_max = (Amax == Azmax) ? Z : (int)floor(__dmul_rn(__dsub_rn(__dadd_rn(__dmul_rn(Amax, Dz), X1z), Bz), IVz));
        } else {
            k_max = (Amin == Azmin) ? Z - 1 : (int)floor(__dmul_rn(__dsub_rn(__dadd_rn(__dmul_rn(Amin, Dz), X1z), Bz), IVz));
            k_min = (Amax == Azmax) ? 0 : (int)floor(__dmul_rn(__dsub_rn(__dadd_rn(__dmul_rn(Amax, Dz), X1z), Bz), IVz)) + 1;
        }
        amin = (float)Amin;
        amax = (float)Amax;
    }

    // initial next-plane alphas (:218-266) and voxel indices (:271-284)
    const float INF = __int_as_float(0x7f800000);
    float ax, ay, az;
    if (fabsf(fs(x1x, x2x)) < fm(g.vx, 1e-6f)) ax = INF;
    else ax = fm(fs(fa(fm(g.vx, (float)(x1x < x2x ? i_min : i_max)), g.bx), x1x), ix);
    if (fabsf(fs(x1y, x2y)) < fm(g.vy, 1e-6f)) ay = INF;
    else ay = fm(fs(fa(fm(g.vy, (float)(x1y < x2y ? j_min : j_max)), g.by), x1y), iy);
    if (zpar) az = INF;
    else az = fm(fs(fa(fm(g.vz, (float)(x1z < x2z ? k_min : k_max)), g.bz), x1z), iz);
    int vi = (x1x < x2x) ? i_min - 1 : i_max;
    int vj = (x1y < x2y) ? j_min - 1 : j_max;
    int vk = (x1z < x2z) ? k_min - 1 : k_max;
    r.vi0 = vi; r.vj0 = vj; r.vk0 = vk;
    r.par = (ax == INF ? 1 : 0) | (ay == INF ? 2 : 0) | (az == INF ? 4 : 0);
    // Per axis: direction, and the table PXo with PXo[voxel] = the next plane
    // after the move (the reference's next_alpha_index): plane vi+1 when
    // increasing, vi when decreasing.  A parallel axis never moves and reads
    // +inf through (x1 = 0, 1/d = 1).
    int sx = (x1x < x2x) ? 1 : ((x1x > x2x) ? -1 : 0);
    int sy = (x1y < x2y) ? 1 : ((x1y > x2y) ? -1 : 0);
    int sz = (x1z < x2z) ? 1 : ((x1z > x2z) ? -1 : 0);
    const float* PXo = PX + 1 + (sx > 0);
    const float* PYo = PY + 1 + (sy > 0);
    const float* PZo = PZ + 1 + (sz > 0);
    float ex1x = x1x, eix = ix, ex1y = x1y, eiy = iy, ex1z = x1z, eiz = iz;
    // computed planes: counter fn = index of the next plane, plane = v*fn + b;
    // a parallel axis uses v = 0, b = +inf
    float fnx = (float)(vi + (sx > 0)), fny = (float)(vj + (sy > 0)), fnz = (float)(vk + (sz > 0));
    float vxe = g.vx, bxe = g.bx, vye = g.vy, bye = g.by, vze = g.vz, bze = g.bz;
    if (ax == INF) { sx = 0; PXo = PINF - vi; ex1x = 0.f; eix = 1.f; vxe = 0.f; bxe = INF; }
    if (ay == INF) { sy = 0; PYo = PINF - vj; ex1y = 0.f; eiy = 1.f; vye = 0.f; bye = INF; }
    if (az == INF) { sz = 0; PZo = PINF - vk; ex1z = 0.f; eiz = 1.f; vze = 0.f; bze = INF; }
    const float fsx = (float)sx, fsy = (float)sy, fsz = (float)sz;
    // prefetch mode: current next-plane coordinate and the one after it
    float cxp = 0.f, nxp = 0.f, cyp = 0.f, nyp = 0.f, czp = 0.f, nzp = 0.f;
    if (CPM == 8) {
        const int ci = min(max(vi, -1), M), cj = min(max(vj, -1), N), ck = min(max(vk, -1), Z);
        cxp = PXo[ci]; nxp = PXo[ci + sx];
        cyp = PYo[cj]; nyp = PYo[cj + sy];
        czp = PZo[ck]; nzp = PZo[ck + sz];
    }
    const int MN = M * N;
    const int syM = sy * M, szMN = sz * MN;
    int idx = TL ? tile_index(g, vi, vj, vk) : vk * MN + vj * M + vi;
    const float d12 = r.d12;
    float ac = amin, sum = 0.f, len = 0.f;
    double dsum = 0.0;
    float seg_p = 0.f, f_p = 0.f;   // the previous step's segment and voxel value
    float sum2 = 0.f, f2_p = 0.f;
    bool any = false;
    // Loop condition after the first step.  Every next-plane alpha is at
    // least ac and grows along its axis, so an index leaves the volume
    // exactly when ac reaches the alpha of that axis's last plane in index
    // space (aex*: the next plane of the last voxel); and when every alpha of
    // the volume is >= 1e-6 (geometry flag fast_exit, never set for the
    // tetrahedron beam's test against 1e-6), amax - ac > 1e-16 is
    // ac < amax (distinct floats >= 2^-28 differ by more than 2^-51).  The
    // first step keeps the reference's own test, which also covers a start
    // voxel whose next plane lies behind the entry point.
    float alim = amax;
    if (g.fast_exit) {
        const float aex = sx > 0 ? fm(fs(PXo[M - 1], ex1x), eix) : (sx < 0 ? fm(fs(PXo[0], ex1x), eix) : INF);
        const float aey = sy > 0 ? fm(fs(PYo[N - 1], ex1y), eiy) : (sy < 0 ? fm(fs(PYo[0], ex1y), eiy) : INF);
        const float aez = sz > 0 ? fm(fs(PZo[Z - 1], ex1z), eiz) : (sz < 0 ? fm(fs(PZo[0], ex1z), eiz) : INF);
        alim = fminf(amax, fminf(aex, fminf(aey, aez)));
    }
    // :297-551.  Branch-free step: every axis re-evaluates its next-plane
    // alpha from its (possibly unchanged) index, which reproduces the current
    // value bit for bit when the axis did not move.
    bool go = (fs(amax, ac) > g.loop_eps) & ((unsigned)vi < (unsigned)M) & ((unsigned)vj < (unsigned)N) &
              ((unsigned)vk < (unsigned)Z);
    while (go) {
        const float m = fminf(fminf(ax, ay), az);
        if (FAST && LOAD) {   // alpha steps, d12 applied after the loop
            const float da = fs(m, ac);
            const float f = COH ? Store<VT>::ldc(vol + idx) : Store<VT>::ld(vol + idx);
            sum = __fmaf_rn(seg_p, f_p, sum);                          // +0 on the first step
            if (DUAL) {
                const float f2 = COH ? Store<VT2>::ldc(vol2 + idx) : Store<VT2>::ld(vol2 + idx);
                sum2 = __fmaf_rn(seg_p, f2_p, sum2);
                f2_p = f2;
            }
            seg_p = da;
            f_p = f;
        } else {
            const float seg = fm(d12, fs(m, ac));
            len = fa(len, seg);
            if (LOAD) {
                const float f = COH ? Store<VT>::ldc(vol + idx) : Store<VT>::ld(vol + idx);
                if (ACC64) dsum = __fma_rn((double)seg_p, (double)f_p, dsum);   // +0 on the first step
                else sum = fa(sum, fm(seg_p, f_p));
                if (DUAL) {
                    const float f2 = COH ? Store<VT2>::ldc(vol2 + idx) : Store<VT2>::ld(vol2 + idx);
                    sum2 = fa(sum2, fm(seg_p, f2_p));
                    f2_p = f2;
                }
                seg_p = seg;
                f_p = f;
            }
        }
        any = true;
        if (TRACE) {
            r.nseg++;
            r.hash = (r.hash ^ (uint64_t)(uint32_t)idx) * kFnvPrime;
        }
        ac = m;
        const int mx = (ax == m) ? 1 : 0, my = (ay == m) ? 1 : 0, mz = (az == m) ? 1 : 0;
        vi += mx * sx;
        vj += my * sy;
        vk += mz * sz;
        if (TL) idx = tile_index(g, vi, vj, vk);
        else idx += mx * sx + my * syM + mz * szMN;
        if (CPM == 8) {
            cxp = mx ? nxp : cxp;
            cyp = my ? nyp : cyp;
            czp = mz ? nzp : czp;
            ax = fm(fs(cxp, ex1x), eix);
            ay = fm(fs(cyp, ex1y), eiy);
            az = fm(fs(czp, ex1z), eiz);
            nxp = PXo[vi + sx];   // in [-2, M+1]: padded
            nyp = PYo[vj + sy];
            nzp = PZo[vk + sz];
        } else {
            if (CPM & 1) {
                fnx = fa(fnx, mx ? fsx : 0.f);
                ax = fm(fs(fa(fm(vxe, fnx), bxe), ex1x), eix);
            } else {
                ax = fm(fs(PXo[vi], ex1x), eix);
            }
            if (CPM & 2) {
                fny = fa(fny, my ? fsy : 0.f);
                ay = fm(fs(fa(fm(vye, fny), bye), ex1y), eiy);
            } else {
                ay = fm(fs(PYo[vj], ex1y), eiy);
            }
            if (CPM & 4) {
                fnz = fa(fnz, mz ? fsz : 0.f);
                az = fm(fs(fa(fm(vze, fnz), bze), ex1z), eiz);
            } else {
                az = fm(fs(PZo[vk], ex1z), eiz);
            }
        }
        if (g.fast_exit) go = ac < alim;
        else go = (fs(amax, ac) > g.loop_eps) & ((unsigned)vi < (unsigned)M) & ((unsigned)vj < (unsigned)N) &
                  ((unsigned)vk < (unsigned)Z);
    }
    if (FAST && LOAD) {
        if (any) {
            sum = fm(__fmaf_rn(seg_p, f_p, sum), d12);
            if (DUAL) sum2 = fm(__fmaf_rn(seg_p, f2_p, sum2), d12);
            len = fm(d12, fs(ac, amin));
        }
    } else if (LOAD && any) {
        if (ACC64) dsum = __fma_rn((double)seg_p, (double)f_p, dsum);
        else sum = fa(sum, fm(seg_p, f_p));
        if (DUAL) sum2 = fa(sum2, fm(seg_p, f2_p));
    }
    r.sum = sum;
    r.sum2 = sum2;
    r.dsum = dsum;
    r.len = len;
    if (any) {
        r.a_lo = amin;
        r.a_hi = ac;
    }
    return r;
}

// BY detector rows of 32 rays per block.  The objective's partial sums are
// one per warp (the 32 rays of one detector row segment, a fixed shuffle
// tree), stored by (view, row, segment), so the totals do not depend on the
// launch shape or the issue order; the dot product's are per block of the
// fixed 32x4 shape.
// The plane tables of the forward kernels in shared memory (the caller syncs).
__device__ __forceinline__ void fp_tables(const DevGeom& g, float* sp, float*& PX, float*& PY, float*& PZ,
                                          float*& PINF)
{
    plane_tables_layout(g, sp, PX, PY, PZ, PINF);
    for (int t = threadIdx.x; t < g.M + 3; t += blockDim.x) PX[t] = g.px[t];
    for (int t = threadIdx.x; t < g.N + 3; t += blockDim.x) PY[t] = g.py[t];
    for (int t = threadIdx.x; t < g.Z + 3; t += blockDim.x) PZ[t] = g.pz[t];
    if (threadIdx.x == 0) PINF[0] = __int_as_float(0x7f800000);
}

// One block of the forward projection: block (bx, by, bz) of a (gx, gy, *)
// grid of FP_BX x BY rays (bz: the view offset), with the plane tables in
// shared memory.  k_forward runs it as its own block; the batch's persistent
// pass runs the blocks of every scan's view in turn, with coherent volume
// loads (COH: the volumes were written by other blocks of that launch).
template <typename VT, int KIND, bool E64, int BY, int CPM, bool TL, bool FAST, bool COH = false>
__device__ __forceinline__ void fp_block(const DevGeom& g, const float* __restrict__ PX, const float* __restrict__ PY,
                                         const float* __restrict__ PZ, const float* __restrict__ PINF, int bx, int by,
                                         int bz, int gx, int gy, const VT* __restrict__ vol, int view0,
                                         void* __restrict__ out, int out_dt, const void* __restrict__ b, int b_dt,
                                         double* __restrict__ partial, int* __restrict__ nseg,
                                         uint64_t* __restrict__ hash, float* __restrict__ lens,
                                         const void* __restrict__ vol2_any, float* __restrict__ ax,
                                         const float* __restrict__ gdev)
{
    constexpr bool REFINE = KIND == FP_SART_REFINE || KIND == FP_SART_REFINE32;
    constexpr bool DUAL = KIND == FP_SART_OBJ || REFINE;
    using VT2 = typename std::conditional<KIND == FP_SART_REFINE32, float, VT>::type;   // the second volume's type
    const VT2* __restrict__ vol2 = (const VT2*)vol2_any;
    const int tx = centre_out(bx, gx), ty = centre_out(by, gy);
    const int u = tx * FP_BX + (threadIdx.x % FP_BX);
    const int v = ty * BY + (threadIdx.x / FP_BX);
    const int w = bz;
    const bool active = (u < g.R) && (v < g.ZP);
    const long long P = (long long)g.R * g.ZP;
    const long long p = (long long)w * P + (long long)v * g.R + u;
    double e2 = 0.0;
    if (KIND == FP_PARTIAL && active && (v < g.row_lo || v >= g.row_hi)) {
        // a fan-slice / parallel-beam slab traces only its band's rows (multiGPU.cu:663-667);
        // a cone-beam slab's other rows miss it, and their sums are (0, 0)
        ((float2*)out)[p] = make_float2(0.0f, 0.0f);
    } else if (active) {
        const float2 sc = g.trig[view0 + w];
        const RayResult rr = siddon<VT, E64, KIND == FP_TRACE, true, KIND == FP_DOT, CPM, TL, DUAL, FAST, COH, VT2>(
            g, PX, PY, PZ, PINF, vol, sc.x, sc.y, u, v, vol2);
        const bool zero = rr.len < g.thr_fp;                       // :554
        if (KIND == FP_PARTIAL) {
            ((float2*)out)[p] = make_float2(rr.sum, rr.len);           // multiGPU.cu:1146-1147, no threshold
        } else if (KIND == FP_FORWARD) {
            st_any(out, p, out_dt, zero ? 0.0f : rr.sum);
        } else if (KIND == FP_SART || KIND == FP_SART_OBJ) {
            const float bv = ld_any(b, p, b_dt);
            const float cv = zero ? 0.0f : fdv(fs(bv, rr.sum), rr.len);   // :562
            ((float2*)out)[p] = make_float2(cv, rr.d12);
            if (KIND == FP_SART_OBJ) {
                const float e = fs(zero ? 0.0f : rr.sum2, bv);
                e2 = (double)fm(e, e);                                 // L2_norm_kernel, tool_functions.cu:35
            }
        } else if (REFINE) {
            // the residual against y_k = (1+g) x_k - g x_(k-1) and the correction d so far
            const float bv = ld_any(b, p, b_dt);
            const float sx = zero ? 0.0f : rr.sum;                     // A x_k, the objective's rule
            const float sp = ax[p];                                    // A x_(k-1), from the previous pass
            const float gm = *gdev;
            const float ay = fs(fm(fa(1.0f, gm), sx), fm(gm, sp));
            const float cv = zero ? 0.0f : fdv(fs(fs(bv, ay), rr.sum2), rr.len);
            ((float2*)out)[p] = make_float2(cv, rr.d12);
            ax[p] = sx;
            const float e = fs(sx, bv);
            e2 = (double)fm(e, e);
        } else if (KIND == FP_OBJECTIVE) {
            const float ax = zero ? 0.0f : rr.sum;
            const float bv = ld_any(b, p, b_dt);
            const float e = fs(ax, bv);
            e2 = (double)fm(e, e);                                     // L2_norm_kernel, tool_functions.cu:35
        } else if (KIND == FP_DOT) {
            e2 = zero ? 0.0 : rr.dsum * (double)ld_any(b, p, b_dt);   // <A x, y> with FP64 ray sums
        } else {
            nseg[p] = rr.nseg;
            hash[p] = rr.hash;
            lens[p] = rr.len;
        }
    }
    if (KIND == FP_OBJECTIVE || KIND == FP_SART_OBJ || REFINE) {
        double t = e2;
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if ((threadIdx.x & 31) == 0 && v < g.ZP) partial[((size_t)w * g.ZP + v) * gx + tx] = t;
    } else if (KIND == FP_DOT) {
        __shared__ double sh[BY];
        const double t = block_sum(e2, sh);
        if (threadIdx.x == 0) partial[((size_t)bz * gy + ty) * gx + tx] = t;
    }
}

template <typename VT, int KIND, bool E64, int BY, int CPM = 0, bool TL = false, int MINB = 1, bool FAST = false>
__global__ void __launch_bounds__(FP_BX * BY, MINB)
k_forward(const DevGeom g, const VT* __restrict__ vol, int view0, void* __restrict__ out, int out_dt,
          const void* __restrict__ b, int b_dt, double* __restrict__ partial, int* __restrict__ nseg,
          uint64_t* __restrict__ hash, float* __restrict__ lens, const void* __restrict__ vol2,
          float* __restrict__ ax, const float* __restrict__ gdev)
{
    extern __shared__ float sp[];
    float* PX;
    float* PY;
    float* PZ;
    float* PINF;
    fp_tables(g, sp, PX, PY, PZ, PINF);
    __syncthreads();
    fp_block<VT, KIND, E64, BY, CPM, TL, FAST>(g, PX, PY, PZ, PINF, blockIdx.x, blockIdx.y, blockIdx.z, gridDim.x,
                                               gridDim.y, vol, view0, out, out_dt, b, b_dt, partial, nseg, hash,
                                               lens, vol2, ax, gdev);
}

template <typename VT, int KIND, int BY, int CPM, bool TL, int MINB, bool FAST = false>
static void launch_fp_tl(const Geometry& G, const FpArgs& a, int nview, size_t smem, cudaStream_t st)
{
    const DevGeom& g = G.dg;
    const dim3 grid((g.R + FP_BX - 1) / FP_BX, (g.ZP + BY - 1) / BY, nview);
    const VT* vol = (const VT*)a.vol;
    if (g.entry64)
        k_forward<VT, KIND, true, BY, CPM, TL, MINB, FAST><<<grid, FP_BX * BY, smem, st>>>(
            g, vol, a.view0, a.out, a.out_dtype, a.b, a.b_dtype, a.partial, a.nseg, a.hash, a.len, a.vol2,
            a.ax, a.gdev);
    else
        k_forward<VT, KIND, false, BY, CPM, TL, MINB, FAST><<<grid, FP_BX * BY, smem, st>>>(
            g, vol, a.view0, a.out, a.out_dtype, a.b, a.b_dtype, a.partial, a.nseg, a.hash, a.len, a.vol2,
            a.ax, a.gdev);
}

template <typename VT, int KIND, int BY, int CPM = 0, int MINB = 1, bool FAST = false>
static void launch_fp_t(const Geometry& G, const FpArgs& a, int nview, size_t smem, cudaStream_t st)
{
    if constexpr (KIND == FP_SART_REFINE32) {   // the refinement solver's volumes are always tiled
        launch_fp_tl<VT, KIND, BY, CPM, true, MINB, FAST>(G, a, nview, smem, st);
    } else {
        if constexpr (KIND == FP_SART || KIND == FP_OBJECTIVE || KIND == FP_SART_OBJ || KIND == FP_PARTIAL ||
                      KIND == FP_SART_REFINE) {
            if (a.tiled) {
                launch_fp_tl<VT, KIND, BY, CPM, true, MINB, FAST>(G, a, nview, smem, st);
                return;
            }
        }
        launch_fp_tl<VT, KIND, BY, CPM, false, MINB, FAST>(G, a, nview, smem, st);
    }
}

// Projector shapes the tuner chooses from: (rows per block, plane mode --
// 0 table, 7 computed, 8 table read ahead --, blocks per SM the registers
// are capped for).
struct FpShape { int rows, cpm, minb; };
static constexpr FpShape kFpShapes[FP_SHAPES] = {{2, 0, 1}, {4, 0, 1}, {8, 0, 1}, {4, 0, 16},
                                                 {4, 0, 12}, {4, 8, 1}, {4, 7, 1}};

template <typename VT, int KIND, bool FAST>
static void launch_fp_shape_t(const Geometry& G, const FpArgs& a, size_t smem, cudaStream_t st)
{
    switch (G.fp_shape) {
    case 0: launch_fp_t<VT, KIND, 2, 0, 1, FAST>(G, a, a.nview, smem, st); break;
    case 2: launch_fp_t<VT, KIND, 8, 0, 1, FAST>(G, a, a.nview, smem, st); break;
    case 3: launch_fp_t<VT, KIND, 4, 0, 16, FAST>(G, a, a.nview, smem, st); break;
    case 4: launch_fp_t<VT, KIND, 4, 0, 12, FAST>(G, a, a.nview, smem, st); break;
    case 5: launch_fp_t<VT, KIND, 4, 8, 1, FAST>(G, a, a.nview, smem, st); break;
    case 6: launch_fp_t<VT, KIND, 4, 7, 1, FAST>(G, a, a.nview, smem, st); break;
    default: launch_fp_t<VT, KIND, 4, 0, 1, FAST>(G, a, a.nview, smem, st); break;
    }
}

// The projections whose sums the solver and ctr_forward use take the fused
// accumulation when the geometry asks for it; the traces, dot products and
// slab partial sums keep the reference's sequence.
template <typename VT, int KIND>
static void launch_fp_shape(const Geometry& G, const FpArgs& a, size_t smem, cudaStream_t st)
{
    if constexpr (KIND == FP_FORWARD || KIND == FP_SART || KIND == FP_OBJECTIVE || KIND == FP_SART_OBJ ||
                  KIND == FP_SART_REFINE || KIND == FP_SART_REFINE32) {
        if (G.dg.fast_sums) {
            launch_fp_shape_t<VT, KIND, true>(G, a, smem, st);
            return;
        }
    }
    launch_fp_shape_t<VT, KIND, false>(G, a, smem, st);
}

// Every projection kind of one storage type (instantiated once per type, in
// fp_f32.cu, fp_bf16.cu and fp_f16.cu, so the three compile in parallel).
template <typename VT>
void launch_forward_kinds(const Geometry& G, const FpArgs& a, size_t smem, cudaStream_t st)
{
    switch (a.kind) {
    case FP_FORWARD: launch_fp_shape<VT, FP_FORWARD>(G, a, smem, st); break;
    case FP_SART: launch_fp_shape<VT, FP_SART>(G, a, smem, st); break;
    case FP_OBJECTIVE: launch_fp_shape<VT, FP_OBJECTIVE>(G, a, smem, st); break;
    case FP_SART_OBJ: launch_fp_shape<VT, FP_SART_OBJ>(G, a, smem, st); break;
    case FP_SART_REFINE: launch_fp_shape<VT, FP_SART_REFINE>(G, a, smem, st); break;
    case FP_SART_REFINE32:   // an FP32 copy with an FP32 correction is FP_SART_REFINE
        if constexpr (std::is_same<VT, float>::value) launch_fp_shape<VT, FP_SART_REFINE>(G, a, smem, st);
        else launch_fp_shape<VT, FP_SART_REFINE32>(G, a, smem, st);
        break;
    case FP_PARTIAL: launch_fp_shape<VT, FP_PARTIAL>(G, a, smem, st); break;
    case FP_TRACE: launch_fp_t<VT, FP_TRACE, FP_BY>(G, a, a.nview, smem, st); break;
    case FP_DOT: launch_fp_t<VT, FP_DOT, FP_BY>(G, a, a.nview, smem, st); break;
    }
}

void launch_forward_f32(const Geometry& G, const FpArgs& a, size_t smem, cudaStream_t st);
void launch_forward_bf16(const Geometry& G, const FpArgs& a, size_t smem, cudaStream_t st);
void launch_forward_f16(const Geometry& G, const FpArgs& a, size_t smem, cudaStream_t st);

}  // namespace ctr
