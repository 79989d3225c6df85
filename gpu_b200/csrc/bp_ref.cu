// bp_ref.cu -- the SART update with the reference backprojector's own
// arithmetic (CTR_SART_REFERENCE_BP).
//
// backprj_ray_driven_3d_kernel (V63/kernel_IterativeRecon_universal.cu:571-810)
// evaluates, per voxel, the bounding rectangle of its 8 corner projections
// (floor(x + 0.5), clamped), and for every detector pixel in it, row by row
// and column by column, the ray's slab alphas by division
// ((c -+ v/2) - q)/(s - q), the chord d12*(alpha_max - alpha_min) when
// positive, kept above vx*1e-6; then f += beta*sum(w c)/sum(w), or f += 0 when
// the summed length is below vx*1e-6.  This kernel evaluates the same
// expressions in the same order, so with the forward projector's correction
// (itself the reference's to the bit) a SART pass equals the reference's bit
// for bit.  Organisation (the values are unchanged):
//   * a thread walks a run of voxels of one (i, j) column: the rectangle's
//     columns do not depend on z (the corner magnification (t-DOD)/(DSO-t)
//     depends on the corner's x, y only), so each column's x and y alphas --
//     four divisions -- are computed once per run;
//   * the z alphas of (cell k, detector row) do not depend on the view (the
//     source height and the rows do not turn): a table per geometry;
//   * alpha_min = max(tx, ty, tz) and alpha_max = min(...) regroup the
//     reference's fmax/fmin chains, which never see a NaN operand (each t is
//     the min or max of two alphas that cannot both be 0/0), so the grouping
//     does not matter; a column whose x-y interval is empty contributes nothing
//     for any z and is skipped;
//   * d12 of a cone-beam ray is the forward projector's (the same expression
//     of the same endpoints), read from the ray record; for the fan-slice and
//     parallel beams the reference's source sits at the voxel's height, so the
//     chord length is recomputed per pair;
//   * "f += 0" turns a stored -0 into +0; done as such.
#include "ctr_device.cuh"

namespace ctr {

// zref[k][v] = (min, max) of the reference's z alphas of cell k for detector
// row v (universal.cu:717-718 with :592-594 and :711-735; for the tetrahedron
// beam T42/...TBCT_voxel.cu:717-718 with its voxel centre :568-570 and row v's
// source, :615).
__global__ void k_zref(const DevGeom g, float2* __restrict__ zref)
{
    const long long n = (long long)g.Z * g.ZP;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t / g.ZP), v = (int)(t % g.ZP);
        const int src = v / g.nvr;
        const float cz = g.ct_style == 3 ? tb_centre_z(g, k) : fa(fa(g.bz_ref, g.cz_off), fm((float)k, g.vz));
        const float qz = fa(g.zmin, fm((float)(v - src * g.nvr), g.dv));
        const float sz = g.ct_style == 3 ? fa(g.zsrc0, fm((float)src, g.zsrc_dz)) : (g.ct_style == 0 ? g.srcz : cz);
        const float az0 = fdv(fs(fs(cz, fm(0.5f, g.vz)), qz), fs(sz, qz));
        const float az1 = fdv(fs(fa(cz, fm(0.5f, g.vz)), qz), fs(sz, qz));
        zref[t] = make_float2(fminf(az0, az1), fmaxf(az0, az1));
    }
}

ctr_status launch_zref(const Geometry& G, float2* zref, cudaStream_t st)
{
    const long long n = (long long)G.dg.Z * G.dg.ZP;
    k_zref<<<(int)std::min<long long>((n + 255) / 256, 148LL * 64), 256, 0, st>>>(G.dg, zref);
    CTR_CUDA_TRY(cudaGetLastError());
    return CTR_OK;
}

constexpr int REF_COLS = 4;   // rectangle columns whose x-y alphas a thread keeps in registers

template <typename VT>
__device__ __forceinline__ void plus_zero(const DevGeom& g, VT* p)
{
    // the reference's "d_volumn_kernel[idx] += 0.0f": only a stored -0 changes
    // (the multi-GPU build's slab kernel has the line commented out, multiGPU.cu:1388-1391)
    if (g.ref_plus0 && __float_as_uint(Store<VT>::ldw(p)) == 0x80000000u) Store<VT>::st(p, 0.0f);
}

// CONE: CT_style 0 (the source's height fixed; d12 from the ray record)
template <typename VT, bool STOCH, int BY, int MINB, bool TL, bool CONE>
__global__ void __launch_bounds__(32 * BY, MINB)
k_sart_ref(const DevGeom g, VT* __restrict__ vol, const float2* __restrict__ rays, int view, float beta,
           uint32_t seed, const uint32_t* __restrict__ pass_seed, int zl)
{
    if (STOCH && pass_seed) seed = *pass_seed * 0x9E3779B9u + (uint32_t)view;
    const int i = blockIdx.x * 32 + (threadIdx.x & 31);
    const int j = blockIdx.y * BY + (threadIdx.x >> 5);
    if (i >= g.M || j >= g.N) return;
    const int kb = blockIdx.z * zl, ke = min(g.Z, kb + zl);
    const long long MN = (long long)g.M * g.N;
    const long long vstep = TL ? 64LL * g.Mt * g.Nt : MN;
    VT* const pv0 = vol + (TL ? (long long)tile_index(g, i, j, kb) : (long long)kb * MN + (long long)j * g.M + i);

    // FOV cylinder (universal.cu:626-632): no rays, the "+= 0" branch
    const float ex = fs(fs((float)i, g.fov_h_x), g.m_off);
    const float ey = fs((float)j, g.fov_h_y);
    if (fa(fm(fm(fm(ex, g.vx), ex), g.vx), fm(fm(fm(ey, g.vy), ey), g.vy)) >= g.fov_r2) {
        VT* pv = pv0;
        for (int k = kb; k < ke; ++k, pv += vstep) plus_zero(g, pv);
        return;
    }

    const float cx = fa(fa(g.bx, fm(g.vx, 0.5f)), fm((float)i, g.vx));   // :592-594
    const float cy = fa(fa(g.by, fm(g.vy, 0.5f)), fm((float)j, g.vy));
    const float2 sc = g.trig[view];
    const float s = sc.x, c = sc.y;
    const float DSO = g.dso, DOD = g.dod;

    // corner projections (:639-678): u per corner, and the z magnification
    // (t-DOD)/(DSO-t) of the corners, of which the z projections
    // m*(pz - srcz) + pz take their extremes at the extreme m (rounding is
    // monotone), so 4 of the 8 vertices give the rectangle's rows
    float mlo = __int_as_float(0x7f800000), mhi = -mlo;
    float minY = mlo, maxY = mhi;
#pragma unroll
    for (int cc = 0; cc < 4; ++cc) {
        const float px = fs(fa(cx, fm((float)(cc & 1), g.vx)), fm(0.5f, g.vx));
        const float py = fs(fa(cy, fm((float)(cc >> 1), g.vy)), fm(0.5f, g.vy));
        const float t = fa(fm(px, c), fm(py, s));
        const float ss = fa(fm(-px, s), fm(py, c));
        const float mg = fdv(fs(t, DOD), fs(DSO, t));
        const float ou = g.ct_style == 2 ? ss : fa(fm(mg, fs(ss, g.srcy)), ss);
        minY = fminf(minY, ou);
        maxY = fmaxf(maxY, ou);
        mlo = fminf(mlo, mg);
        mhi = fmaxf(mhi, mg);
    }
    int minYi = __float2int_rd(fa(fm(fs(minY, g.ymin), g.inv_du), 0.5f));   // :680-681
    int maxYi = __float2int_rd(fa(fm(fs(maxY, g.ymin), g.inv_du), 0.5f));
    const bool u_out = (minYi < 0 && maxYi < 0) || (minYi > g.R - 1 && maxYi > g.R - 1);
    minYi = max(minYi, 0);                                                   // :699-702
    maxYi = min(maxYi, g.R - 1);

    // per rectangle column: max of the x and y entry alphas, min of the exits
    // (:760-777), and for the fan-slice / parallel beams the x-y part of d12
    const float sx0 = fs(fm(g.srcx, c), fm(g.srcy, s));                     // :711-712
    const float sy0 = fa(fm(g.srcx, s), fm(g.srcy, c));
    const float xlo = fs(cx, fm(0.5f, g.vx)), xhi = fa(cx, fm(0.5f, g.vx));
    const float ylo = fs(cy, fm(0.5f, g.vy)), yhi = fa(cy, fm(0.5f, g.vy));
    auto column = [&](int ir, float& lo, float& hi, float& q2) {
        const float pu = fa(g.ymin, fm((float)ir, g.du));
        const float qx = fs(fm(DOD, c), fm(pu, s));                          // :733-734
        const float qy = fa(fm(DOD, s), fm(pu, c));
        const float sx = g.ct_style == 2 ? fs(fm(g.srcx, c), fm(pu, s)) : sx0;   // :737-742
        const float sy = g.ct_style == 2 ? fa(fm(g.srcx, s), fm(pu, c)) : sy0;
        const float ax0 = fdv(fs(xlo, qx), fs(sx, qx)), ax1 = fdv(fs(xhi, qx), fs(sx, qx));
        const float ay0 = fdv(fs(ylo, qy), fs(sy, qy)), ay1 = fdv(fs(yhi, qy), fs(sy, qy));
        lo = fmaxf(fminf(ax0, ax1), fminf(ay0, ay1));
        hi = fminf(fmaxf(ax0, ax1), fmaxf(ay0, ay1));
        if (!CONE) q2 = fa(fm(fs(sx, qx), fs(sx, qx)), fm(fs(sy, qy), fs(sy, qy)));
    };
    float clo[REF_COLS], chi[REF_COLS], cq2[REF_COLS];
    unsigned live = 0;
    const int ncol = maxYi - minYi + 1;
#pragma unroll
    for (int q = 0; q < REF_COLS; ++q) {
        clo[q] = 0.f; chi[q] = 0.f; cq2[q] = 0.f;
        if (!u_out && q < ncol) {
            column(minYi + q, clo[q], chi[q], cq2[q]);
            if (chi[q] > clo[q]) live |= 1u << q;   // an empty x-y interval is empty for every z
        }
    }

    const int R = g.R;
    VT* pv = pv0;
    for (int k = kb; k < ke; ++k, pv += vstep) {
        const float cz = fa(fa(g.bz_ref, g.cz_off), fm((float)k, g.vz));   // :594; a slab's, multiGPU.cu:1179
        // detector rows of the rectangle (:655-683)
        float minZ, maxZ;
        if (CONE) {
            minZ = __int_as_float(0x7f800000);
            maxZ = -minZ;
#pragma unroll
            for (int kk = 0; kk < 2; ++kk) {
                const float pz = fs(fa(cz, fm((float)kk, g.vz)), fm(0.5f, g.vz));
                const float dz = fs(pz, g.srcz);
                const float a0 = fa(fm(dz >= 0.f ? mlo : mhi, dz), pz);   // the smallest of the 4 corners
                const float a1 = fa(fm(dz >= 0.f ? mhi : mlo, dz), pz);   // and the largest
                minZ = fminf(minZ, a0);
                maxZ = fmaxf(maxZ, a1);
            }
        } else {
            minZ = cz;
            maxZ = cz;
        }
        int minZi = __float2int_rd(fa(fm(fs(minZ, g.zmin), g.inv_dv), 0.5f));
        int maxZi = __float2int_rd(fa(fm(fs(maxZ, g.zmin), g.inv_dv), 0.5f));
        float sw = 0.f, sl = 0.f;
        if (!(u_out || (minZi < 0 && maxZi < 0) || (minZi > g.ZP - 1 && maxZi > g.ZP - 1))) {
            minZi = max(minZi, 0);
            maxZi = min(maxZi, g.ZP - 1);
            const float2* __restrict__ zr = g.zref + (long long)k * g.ZP;
            auto pair = [&](float lo, float hi, float q2, float2 zc, float qzd, float2 rec) {
                const float amin = fmaxf(lo, zc.x), amax = fminf(hi, zc.y);
                const float dl = fs(amax, amin);
                if (dl > 0.f) {                                              // :780
                    // cone beam: the projector's d12; fan slices / parallel beam: source at the voxel's height
                    const float d12 = CONE ? rec.y : __fsqrt_rn(fa(q2, fm(qzd, qzd)));
                    const float temp = fm(d12, dl);
                    if (temp > g.thr_bp) {                                   // :785-791
                        sw = fa(sw, fm(temp, rec.x));
                        sl = fa(sl, temp);
                    }
                }
            };
            for (int jr = minZi; jr <= maxZi; ++jr) {
                const float2 zc = __ldg(zr + jr);
                const float qzd = CONE ? 0.f : fs(cz, fa(g.zmin, fm((float)jr, g.dv)));   // sz - qz, sz = cz
                const float2* __restrict__ rrow = rays + (long long)jr * R + minYi;
#pragma unroll
                for (int q = 0; q < REF_COLS; ++q)
                    if (live & (1u << q)) pair(clo[q], chi[q], cq2[q], zc, qzd, __ldg(rrow + q));
                for (int q = REF_COLS; q < ncol; ++q) {   // wide rectangles: the rest per row
                    float lo, hi, q2;
                    column(minYi + q, lo, hi, q2);
                    if (hi > lo) pair(lo, hi, q2, zc, qzd, __ldg(rrow + q));
                }
            }
        }
        if (sl < g.thr_bp) {                                                 // :799-807
            plus_zero(g, pv);
        } else {
            const float nv = fa(Store<VT>::ldw(pv), fdv(fm(beta, sw), sl));
            if (STOCH) st_sr<VT>(pv, nv, hash32(seed ^ hash32((uint32_t)(k * MN + j * g.M + i))));
            else Store<VT>::st(pv, nv);
        }
    }
}

// The tetrahedron beam (T42/voxel/kernel_IterativeRecon_TBCT_voxel.cu:546-775):
// per voxel (T42's centre, boundary + v*(0.5 + index)), the sources that pass
// its source_lower/source_upper test (:620-627), each with the bounding
// rectangle of the voxel's corners projected from that source (:631-685), its
// pixels row by row, column by column, the slab alphas by division
// (:713-731), chords above vx*1e-6 (:733-747); the sources' sums added in
// ascending order (one of the orders of the reference's atomicAdd), and
// f += beta*sum/length where the length exceeds vx*1e-3 (:772-773), nothing
// otherwise.  The same regroupings as k_sart_ref; the chord length is the
// projector's (source and pixel are the projector's endpoints).
template <typename VT, bool STOCH, int BY, int MINB, bool TL>
__global__ void __launch_bounds__(32 * BY, MINB)
k_sart_ref_tb(const DevGeom g, VT* __restrict__ vol, const float2* __restrict__ rays, int view, float beta,
              uint32_t seed, const uint32_t* __restrict__ pass_seed, int zl)
{
    if (STOCH && pass_seed) seed = *pass_seed * 0x9E3779B9u + (uint32_t)view;
    const int i = blockIdx.x * 32 + (threadIdx.x & 31);
    const int j = blockIdx.y * BY + (threadIdx.x >> 5);
    if (i >= g.M || j >= g.N) return;
    const int kb = blockIdx.z * zl, ke = min(g.Z, kb + zl);
    const long long MN = (long long)g.M * g.N;
    const long long vstep = TL ? 64LL * g.Mt * g.Nt : MN;

    const float ex = fs(fs((float)i, g.fov_h_x), g.m_off);                   // :600-602
    const float ey = fs((float)j, g.fov_h_y);
    if (fa(fm(fm(fm(ex, g.vx), ex), g.vx), fm(fm(fm(ey, g.vy), ey), g.vy)) >= g.fov_r2) return;

    const float cx = tb_centre_xy(g, g.bx, g.vx, i);                        // :568-569
    const float cy = tb_centre_xy(g, g.by, g.vy, j);
    const float2 sc = g.trig[view];
    const float s = sc.x, c = sc.y;
    const float DSO = g.dso, DOD = g.dod;
    const float tden = fs(fa(fm(cx, c), fm(cy, s)), DOD);                    // :620, t - DOD

    float mlo = __int_as_float(0x7f800000), mhi = -mlo;
    float minY = mlo, maxY = mhi;
#pragma unroll
    for (int cc = 0; cc < 4; ++cc) {                                          // :631-655
        const float px = fs(fa(cx, fm((float)(cc & 1), g.vx)), fm(0.5f, g.vx));
        const float py = fs(fa(cy, fm((float)(cc >> 1), g.vy)), fm(0.5f, g.vy));
        const float t = fa(fm(px, c), fm(py, s));
        const float ss = fa(fm(-px, s), fm(py, c));
        const float mg = fdv(fs(t, DOD), fs(DSO, t));
        const float ou = fa(fm(mg, fs(ss, g.srcy)), ss);
        minY = fminf(minY, ou);
        maxY = fmaxf(maxY, ou);
        mlo = fminf(mlo, mg);
        mhi = fmaxf(mhi, mg);
    }
    int minYi = __float2int_rd(fa(fm(fs(minY, g.ymin), g.inv_du), 0.5f));   // :659-660
    int maxYi = __float2int_rd(fa(fm(fs(maxY, g.ymin), g.inv_du), 0.5f));
    if ((minYi < 0 && maxYi < 0) || (minYi > g.R - 1 && maxYi > g.R - 1)) return;   // :668: nothing added
    minYi = max(minYi, 0);
    maxYi = min(maxYi, g.R - 1);

    const float sx = fs(fm(g.srcx, c), fm(g.srcy, s));                      // :613-614
    const float sy = fa(fm(g.srcx, s), fm(g.srcy, c));
    const float xlo = fs(cx, fm(0.5f, g.vx)), xhi = fa(cx, fm(0.5f, g.vx));
    const float ylo = fs(cy, fm(0.5f, g.vy)), yhi = fa(cy, fm(0.5f, g.vy));
    auto column = [&](int ir, float& lo, float& hi) {                        // :693-731
        const float pu = fa(g.ymin, fm((float)ir, g.du));
        const float qx = fs(fm(DOD, c), fm(pu, s));
        const float qy = fa(fm(DOD, s), fm(pu, c));
        const float ax0 = fdv(fs(xlo, qx), fs(sx, qx)), ax1 = fdv(fs(xhi, qx), fs(sx, qx));
        const float ay0 = fdv(fs(ylo, qy), fs(sy, qy)), ay1 = fdv(fs(yhi, qy), fs(sy, qy));
        lo = fmaxf(fminf(ax0, ax1), fminf(ay0, ay1));
        hi = fminf(fmaxf(ax0, ax1), fmaxf(ay0, ay1));
    };
    float clo[REF_COLS], chi[REF_COLS];
    unsigned live = 0;
    const int ncol = maxYi - minYi + 1;
#pragma unroll
    for (int q = 0; q < REF_COLS; ++q) {
        clo[q] = 0.f; chi[q] = 0.f;
        if (q < ncol) {
            column(minYi + q, clo[q], chi[q]);
            if (chi[q] > clo[q]) live |= 1u << q;
        }
    }

    const int R = g.R, nv = g.nvr;
    auto zsrc = [&](int q) { return fa(g.zsrc0, fm((float)q, g.zsrc_dz)); };
    int s0 = 0, s1 = -1;
    bool s_est = true;
    VT* pv = vol + (TL ? (long long)tile_index(g, i, j, kb) : (long long)kb * MN + (long long)j * g.M + i);
    for (int k = kb; k < ke; ++k, pv += vstep) {
        const float cz = tb_centre_z(g, k);                                 // :570
        const float upper = fa(fdv(fm(fs(fa(cz, g.vz), g.zmin), g.dsod), tden), g.zmin);   // :623
        const float lower = fa(fdv(fm(fs(fs(cz, g.vz), g.zmax), g.dsod), tden), g.zmax);   // :624
        if (s_est) {   // the kept sources: one range growing with k (see k_sart_walk's TB form)
            s_est = false;
            s0 = 0;
            s1 = g.nsrc - 1;
            if (g.nsrc > 1) {
                s0 = (int)fminf(fmaxf(ceilf(__fdividef(fs(lower, g.zsrc0), g.zsrc_dz)), 0.f), (float)g.nsrc);
                s1 = (int)fminf(fmaxf(floorf(__fdividef(fs(upper, g.zsrc0), g.zsrc_dz)), -1.f), (float)(g.nsrc - 1));
            }
        }
        while (s0 > 0 && !(zsrc(s0 - 1) < lower)) --s0;
        while (s0 < g.nsrc && zsrc(s0) < lower) ++s0;
        while (s1 < g.nsrc - 1 && !(zsrc(s1 + 1) > upper)) ++s1;
        while (s1 >= 0 && zsrc(s1) > upper) --s1;
        const float2* __restrict__ zr = g.zref + (long long)k * g.ZP;
        float WS = 0.f, L = 0.f;
        for (int sq = s0; sq <= s1; ++sq) {
            const float zs = zsrc(sq);
            // rows of the rectangle projected from this source (:649, :661-662)
            float minZ = __int_as_float(0x7f800000), maxZ = -minZ;
#pragma unroll
            for (int kk = 0; kk < 2; ++kk) {
                const float pz = fs(fa(cz, fm((float)kk, g.vz)), fm(0.5f, g.vz));
                const float dz = fs(pz, zs);
                minZ = fminf(minZ, fa(fm(dz >= 0.f ? mlo : mhi, dz), pz));
                maxZ = fmaxf(maxZ, fa(fm(dz >= 0.f ? mhi : mlo, dz), pz));
            }
            int minZi = __float2int_rd(fa(fm(fs(minZ, g.zmin), g.inv_du), 0.5f));
            int maxZi = __float2int_rd(fa(fm(fs(maxZ, g.zmin), g.inv_du), 0.5f));
            float sw = 0.f, sl = 0.f;
            if (!((minZi < 0 && maxZi < 0) || (minZi > nv - 1 && maxZi > nv - 1))) {
                minZi = max(minZi, 0);
                maxZi = min(maxZi, nv - 1);
                for (int jr = sq * nv + minZi; jr <= sq * nv + maxZi; ++jr) {
                    const float2 zc = __ldg(zr + jr);
                    const float2* __restrict__ rrow = rays + (long long)jr * R + minYi;
                    auto pair = [&](float lo, float hi, float2 rec) {
                        const float dl = fs(fminf(hi, zc.y), fmaxf(lo, zc.x));
                        if (dl > 0.f) {                                          // :733
                            const float temp = fm(rec.y, dl);
                            if (temp > g.thr_bp) {                              // :738-744
                                sw = fa(sw, fm(temp, rec.x));
                                sl = fa(sl, temp);
                            }
                        }
                    };
#pragma unroll
                    for (int q = 0; q < REF_COLS; ++q)
                        if (live & (1u << q)) pair(clo[q], chi[q], __ldg(rrow + q));
                    for (int q = REF_COLS; q < ncol; ++q) {
                        float lo, hi;
                        column(minYi + q, lo, hi);
                        if (hi > lo) pair(lo, hi, __ldg(rrow + q));
                    }
                }
            }
            WS = fa(WS, sw);                                                    // :754-755
            L = fa(L, sl);
        }
        if (L > g.thr_upd) {                                                    // :772-773
            const float nvl = fa(Store<VT>::ldw(pv), fdv(fm(beta, WS), L));
            if (STOCH) st_sr<VT>(pv, nvl, hash32(seed ^ hash32((uint32_t)(k * MN + j * g.M + i))));
            else Store<VT>::st(pv, nvl);
        }
    }
}

// launch shapes: the column walk's table (rows per block, z run, register cap)
template <typename VT, bool STOCH, bool TL>
ctr_status launch_sart_ref_t(const Geometry& G, const BpArgs& a, cudaStream_t st)
{
    const DevGeom& g = G.dg;
    const int shape = (G.bp_shape >= 0 && G.bp_shape < BP_SHAPES) ? G.bp_shape : 1;
    static constexpr int kRows[BP_SHAPES] = {4, 4, 4, 8, 4, 4};
    static constexpr int kZl[BP_SHAPES] = {8, 32, 32, 32, 128, 32};
    int zl = kZl[shape];
    const long long cols = (long long)g.M * g.N;
    while (zl > 1 && cols * ((g.Z + zl - 1) / zl) < 148LL * 2048) zl >>= 1;
    const int rows = kRows[shape];
    const dim3 grid((g.M + 31) / 32, (g.N + rows - 1) / rows, (g.Z + zl - 1) / zl);
    if (grid.z > 65535) return set_error(CTR_ERR_UNSUPPORTED, "too many z runs");
    const float2* rays = (const float2*)a.rays;
    const bool cone = g.ct_style == 0;
    if (g.ct_style == 3) {
        if (rows == 8)
            k_sart_ref_tb<VT, STOCH, 8, 4, TL><<<grid, 256, 0, st>>>(g, (VT*)a.vol, rays, a.view0, a.beta, a.seed,
                                                                      a.pass_seed, zl);
        else
            k_sart_ref_tb<VT, STOCH, 4, 8, TL><<<grid, 128, 0, st>>>(g, (VT*)a.vol, rays, a.view0, a.beta, a.seed,
                                                                      a.pass_seed, zl);
    } else if (rows == 8) {
        if (cone)
            k_sart_ref<VT, STOCH, 8, 4, TL, true><<<grid, 256, 0, st>>>(g, (VT*)a.vol, rays, a.view0, a.beta, a.seed,
                                                                        a.pass_seed, zl);
        else
            k_sart_ref<VT, STOCH, 8, 4, TL, false><<<grid, 256, 0, st>>>(g, (VT*)a.vol, rays, a.view0, a.beta, a.seed,
                                                                         a.pass_seed, zl);
    } else if (cone) {
        k_sart_ref<VT, STOCH, 4, 8, TL, true><<<grid, 128, 0, st>>>(g, (VT*)a.vol, rays, a.view0, a.beta, a.seed,
                                                                    a.pass_seed, zl);
    } else {
        k_sart_ref<VT, STOCH, 4, 8, TL, false><<<grid, 128, 0, st>>>(g, (VT*)a.vol, rays, a.view0, a.beta, a.seed,
                                                                     a.pass_seed, zl);
    }
    return CTR_OK;
}

ctr_status launch_sart_ref(const Geometry& G, const BpArgs& a, cudaStream_t st)
{
    const bool sr = (a.flags & CTR_SART_STOCHASTIC_ROUND) != 0;
    CTR_DISPATCH_DTYPE(a.vol_dtype, VT, {
        if (a.tiled) {
            if (sr) CTR_TRY((launch_sart_ref_t<VT, true, true>(G, a, st)));
            else CTR_TRY((launch_sart_ref_t<VT, false, true>(G, a, st)));
        } else if (sr) {
            CTR_TRY((launch_sart_ref_t<VT, true, false>(G, a, st)));
        } else {
            CTR_TRY((launch_sart_ref_t<VT, false, false>(G, a, st)));
        }
    });
    CTR_CUDA_TRY(cudaGetLastError());
    return CTR_OK;
}

}  // namespace ctr
