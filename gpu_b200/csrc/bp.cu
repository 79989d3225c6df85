// bp.cu -- voxel-driven gather backprojector (matched adjoint and SART update).
//
// Restates backprj_ray_driven_3d_kernel (V63/kernel_IterativeRecon_universal.cu:
// 571-810): for each voxel, every detector pixel in the bounding rectangle of
// its corner projections is a candidate ray, and the ray's chord through the
// voxel is d12 * (min of exit alphas - max of entry alphas).
//
// Where the reference recomputes each alpha as ((c +- v/2) - x1)/(x2 - x1),
// this kernel evaluates the alphas exactly as the forward projector does,
// (plane_n - x1) * (1/(x2 - x1)) with the projector's own x1, 1/(x2-x1) and
// d12, so every (voxel, ray) chord equals the projector's Siddon segment
// bit for bit and the adjoint is matched.  Two further changes:
//   * the alphas of a ray split into an xy part, fixed by the detector column
//     (x1x, x1y, 1/dx, 1/dy do not depend on the row), and a z part fixed by
//     the row.  A thread owns K voxels of one z column: the column's
//     detector-column range and its xy entry/exit interval per column are
//     computed once and reused for all K voxels;
//   * the adjoint accumulates several views per pass in registers, so the
//     volume is read and written once per batch.
#include "ctr_device.cuh"

namespace ctr {

static constexpr int BP_BX = 32;   // voxels along x per block (one warp row)
static constexpr int BP_BY = 4;    // voxel rows along y per block
static constexpr int BP_THREADS = BP_BX * BP_BY;
static constexpr int BP_K = 4;     // z voxels per thread

// Ray records: REC = float2 (c, d12) for the SART update and the reference's
// command-0 backprojection, whose chords are purely geometric like the
// reference BP's; REC = float4 (y, d12, alpha_lo, alpha_hi) for the matched
// adjoint, whose chords are clipped to the interval the forward traversal
// covered (empty where the reference traversal drops a ray at a volume edge).
template <typename VT, typename REC, bool SART, bool MASK, bool STOCH>
__global__ void __launch_bounds__(BP_THREADS)
k_backproject(const DevGeom g, VT* __restrict__ vol, const REC* __restrict__ rays, int view0, int nview,
              int accumulate, float beta, uint32_t seed)
{
    constexpr bool WINDOW = sizeof(REC) == sizeof(float4) && !SART && !MASK;
    extern __shared__ float sp[];
    float* PX = sp;
    float* PY = PX + (g.M + 3);
    float* PZ = PY + (g.N + 3);
    float2* RT = reinterpret_cast<float2*>(PZ + ((g.Z + 3 + 1) & ~1));
    for (int t = threadIdx.x; t < g.M + 3; t += BP_THREADS) PX[t] = g.px[t];
    for (int t = threadIdx.x; t < g.N + 3; t += BP_THREADS) PY[t] = g.py[t];
    for (int t = threadIdx.x; t < g.Z + 3; t += BP_THREADS) PZ[t] = g.pz[t];
    for (int t = threadIdx.x; t < g.ZP; t += BP_THREADS) RT[t] = g.rowt[t];
    __syncthreads();

    const int i = blockIdx.x * BP_BX + (threadIdx.x % BP_BX);
    const int j = blockIdx.y * BP_BY + (threadIdx.x / BP_BX);
    const int k0 = blockIdx.z * BP_K;
    if (i >= g.M || j >= g.N) return;
    const int R = g.R, ZP = g.ZP;

    // FOV cylinder (universal.cu:626-628)
    bool masked = false;
    if (MASK) {
        const float ex = fs(fs((float)i, g.fov_h_x), g.m_off);
        const float ey = fs((float)j, g.fov_h_y);
        masked = fa(fm(fm(fm(ex, g.vx), ex), g.vx), fm(fm(fm(ey, g.vy), ey), g.vy)) >= g.fov_r2;
    }

    float sw[BP_K], sl[BP_K];
#pragma unroll
    for (int kk = 0; kk < BP_K; ++kk) { sw[kk] = 0.f; sl[kk] = 0.f; }

    if (!masked) {
        // voxel centre (universal.cu:592-594) and its bounding planes
        const float cx = fa(fa(g.bx, fm(g.vx, 0.5f)), fm((float)i, g.vx));
        const float cy = fa(fa(g.by, fm(g.vy, 0.5f)), fm((float)j, g.vy));
        const float xlo = PX[i + 1], xhi = PX[i + 2];
        const float ylo = PY[j + 1], yhi = PY[j + 2];
        for (int w = 0; w < nview; ++w) {
            const int view = view0 + w;
            const float2 sc = g.trig[view];
            const float s = sc.x, c = sc.y;
            // corner projections onto the detector (universal.cu:639-683):
            // u depends on the corner's x,y only; the z projection scales by
            // 1 + (t-DOD)/(DSO-t), bounded by its extremes over the 4 corners.
            float umin = __int_as_float(0x7f800000), umax = -umin, mlo = umin, mhi = -umin;
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) {
                const float pxc = fs(fa(cx, fm((float)(cc & 1), g.vx)), fm(0.5f, g.vx));
                const float pyc = fs(fa(cy, fm((float)(cc >> 1), g.vy)), fm(0.5f, g.vy));
                const float t = fa(fm(pxc, c), fm(pyc, s));
                const float ss = fa(fm(-pxc, s), fm(pyc, c));
                const float mt = fdv(fs(t, g.dod), fs(g.dso, t));
                const float ou = fa(fm(mt, fs(ss, g.srcy)), ss);
                umin = fminf(umin, ou); umax = fmaxf(umax, ou);
                mlo = fminf(mlo, mt); mhi = fmaxf(mhi, mt);
            }
            int ulo = __float2int_rd(fa(fm(fs(umin, g.ymin), g.inv_du), 0.5f));
            int uhi = __float2int_rd(fa(fm(fs(umax, g.ymin), g.inv_du), 0.5f));
            if ((ulo < 0 && uhi < 0) || (ulo > R - 1 && uhi > R - 1)) continue;
            ulo = max(ulo, 0);
            uhi = min(uhi, R - 1);
            // detector-row range of each of the K voxels
            int vlo[BP_K], vhi[BP_K];
#pragma unroll
            for (int kk = 0; kk < BP_K; ++kk) {
                const int k = k0 + kk;
                vlo[kk] = 1; vhi[kk] = 0;
                if (k < g.Z) {
                    const float zlo = fs(PZ[k + 1], g.srcz), zhi = fs(PZ[k + 2], g.srcz);
                    const float a0 = fa(fm(mlo, zlo), PZ[k + 1]), a1 = fa(fm(mhi, zlo), PZ[k + 1]);
                    const float b0 = fa(fm(mlo, zhi), PZ[k + 2]), b1 = fa(fm(mhi, zhi), PZ[k + 2]);
                    const float zmn = fminf(fminf(a0, a1), fminf(b0, b1));
                    const float zmx = fmaxf(fmaxf(a0, a1), fmaxf(b0, b1));
                    int lo = __float2int_rd(fa(fm(fs(zmn, g.zmin), g.inv_dv), 0.5f));
                    int hi = __float2int_rd(fa(fm(fs(zmx, g.zmin), g.inv_dv), 0.5f));
                    if (!((lo < 0 && hi < 0) || (lo > ZP - 1 && hi > ZP - 1))) {
                        vlo[kk] = max(lo, 0);
                        vhi[kk] = min(hi, ZP - 1);
                    }
                }
            }
            const float4* __restrict__ colt = g.colt + (long long)view * R;
            const REC* __restrict__ rw = rays + (long long)w * R * ZP;
            for (int uu = ulo; uu <= uhi; ++uu) {
                const float4 ct = __ldg(colt + uu);
                // xy entry/exit of this ray column through the voxel column
                const float ax0 = fm(fs(xlo, ct.x), ct.y), ax1 = fm(fs(xhi, ct.x), ct.y);
                const float ay0 = fm(fs(ylo, ct.z), ct.w), ay1 = fm(fs(yhi, ct.z), ct.w);
                const float a = fmaxf(fminf(ax0, ax1), fminf(ay0, ay1));
                const float bb = fminf(fmaxf(ax0, ax1), fmaxf(ay0, ay1));
                if (!(bb > a)) continue;
#pragma unroll
                for (int kk = 0; kk < BP_K; ++kk) {
                    const int kc = min(k0 + kk, g.Z - 1);
                    const float zl = PZ[kc + 1], zh = PZ[kc + 2];
                    for (int vv = vlo[kk]; vv <= vhi[kk]; ++vv) {
                        const float2 rt = RT[vv];
                        const float az0 = fm(fs(zl, rt.x), rt.y), az1 = fm(fs(zh, rt.x), rt.y);
                        float lo = fmaxf(a, fminf(az0, az1));
                        float hi = fminf(bb, fmaxf(az0, az1));
                        const REC rec = __ldg(rw + (long long)vv * R + uu);
                        if constexpr (WINDOW) {
                            lo = fmaxf(lo, rec.z);
                            hi = fminf(hi, rec.w);
                        }
                        const float temp = fm(rec.y, fs(hi, lo));
                        if (SART || MASK) {
                            if (temp > g.thr_bp) {                        // :785-791
                                sw[kk] = fa(sw[kk], fm(temp, rec.x));
                                sl[kk] = fa(sl[kk], temp);
                            }
                        } else if (temp > 0.0f) {
                            sw[kk] = __fmaf_rn(temp, rec.x, sw[kk]);
                        }
                    }
                }
            }
        }
    }

    const long long MN = (long long)g.M * g.N;
#pragma unroll
    for (int kk = 0; kk < BP_K; ++kk) {
        const int k = k0 + kk;
        if (k >= g.Z) break;
        VT* p = vol + (long long)k * MN + (long long)j * g.M + i;
        if (SART) {
            if (!(sl[kk] < g.thr_bp)) {                                  // :799-806
                const float nv = fa(Store<VT>::ldw(p), fdv(fm(beta, sw[kk]), sl[kk]));
                if (STOCH) st_sr<VT>(p, nv, hash32(seed ^ hash32((uint32_t)(k * MN + j * g.M + i))));
                else Store<VT>::st(p, nv);
            }
        } else if (MASK) {
            // reference command 0: assignment where the summed length passes
            if (!(sl[kk] < g.thr_bp)) Store<VT>::st(p, accumulate ? fa(Store<VT>::ldw(p), sw[kk]) : sw[kk]);
            else if (!accumulate) Store<VT>::st(p, 0.0f);
        } else {
            Store<VT>::st(p, accumulate ? fa(Store<VT>::ldw(p), sw[kk]) : sw[kk]);
        }
    }
}

template <typename VT, typename REC, bool SART, bool MASK, bool STOCH>
static void launch_bp_t(const Geometry& G, const BpArgs& a, cudaStream_t st)
{
    const DevGeom& g = G.dg;
    dim3 grid((g.M + BP_BX - 1) / BP_BX, (g.N + BP_BY - 1) / BP_BY, (g.Z + BP_K - 1) / BP_K);
    const size_t smem = sizeof(float) * (size_t)(g.M + 3 + g.N + 3 + ((g.Z + 3 + 1) & ~1)) + sizeof(float2) * g.ZP;
    k_backproject<VT, REC, SART, MASK, STOCH><<<grid, BP_THREADS, smem, st>>>(
        g, (VT*)a.vol, (const REC*)a.rays, a.view0, a.nview, (a.flags & CTR_BP_ACCUMULATE) ? 1 : 0, a.beta, a.seed);
}

ctr_status launch_backproject(const Geometry& G, const BpArgs& a, cudaStream_t st)
{
    if (a.nview <= 0) return CTR_OK;
    const size_t smem = sizeof(float) * (size_t)(G.dg.M + G.dg.N + G.dg.Z + 10) + sizeof(float2) * G.dg.ZP;
    if (smem > 48 * 1024) return set_error(CTR_ERR_UNSUPPORTED, "plane tables exceed 48 KB of shared memory");
    CTR_DISPATCH_DTYPE(a.vol_dtype, VT, {
        if (a.sart) {
            if (a.flags & CTR_SART_STOCHASTIC_ROUND) launch_bp_t<VT, float2, true, true, true>(G, a, st);
            else launch_bp_t<VT, float2, true, true, false>(G, a, st);
        } else {
            if (a.flags & CTR_BP_FOV_MASK) launch_bp_t<VT, float4, false, true, false>(G, a, st);
            else launch_bp_t<VT, float4, false, false, false>(G, a, st);
        }
    });
    CTR_CUDA_TRY(cudaGetLastError());
    return CTR_OK;
}

}  // namespace ctr
