// bp.cu -- voxel-driven gather backprojectors (SART update, matched adjoint).
//
// Both restate backprj_ray_driven_3d_kernel (V63/kernel_IterativeRecon_
// universal.cu:571-810): for each voxel, every detector pixel in the bounding
// rectangle of its corner projections is a candidate ray, and the ray's chord
// through the voxel is d12 * (min of exit alphas - max of entry alphas).
//
// Where the reference recomputes each alpha as ((c +- v/2) - x1)/(x2 - x1),
// these kernels evaluate the alphas exactly as the forward projector does,
// (plane_n - x1) * (1/(x2 - x1)) with the projector's own x1, 1/(x2-x1) and
// d12, so every (voxel, ray) chord is the projector's Siddon segment bit for
// bit.  Organisation:
//   * the alphas of a ray split into an xy part fixed by the detector column
//     (x1x, x1y, 1/dx, 1/dy do not depend on the row) and a z part fixed by
//     the row.  A thread owns BP_K voxels of one z column: the column's
//     detector-column range and the xy entry/exit alphas per detector column
//     are computed once and reused for all of them;
//   * writes are coalesced: the 32 lanes of a warp own 32 consecutive x.
//
// k_backproject: the SART update (command 1) and the reference's command 0,
// with the reference BP's geometric chords, FOV mask and thresholds.
// k_adjoint: the exact adjoint of the forward projector.  Each ray record
// carries the alpha interval, start voxel and parallel axes of the forward
// traversal, and the chord of a voxel is taken over the traversal's own cell
// intervals: the start cell opens at -inf, cells behind the start are never
// visited, a parallel axis keeps its start cell.  That is what the reference
// traversal does where its floor-based start index differs from the geometry
// (rays through volume edges, nearly axis-parallel rays).  Several views are
// accumulated per pass in FP64 registers (a float*float product is exact in
// FP64), so the volume is read and written once per batch.
#include "ctr_device.cuh"
#include "fp_kernels.cuh"   // the forward blocks of the batch's persistent pass

namespace ctr {

static constexpr int BP_BX = 32;   // voxels along x per block (one warp row)
static constexpr int BP_BY = 4;    // voxel rows along y per block
static constexpr int BP_THREADS = BP_BX * BP_BY;
static constexpr int BP_K = 8;     // z voxels per thread

struct SharedTables {
    float* PX;
    float* PY;
    float* PZ;
    float2* RT;
};

__device__ __forceinline__ SharedTables load_tables(const DevGeom& g, float* sp)
{
    SharedTables t;
    t.PX = sp;
    t.PY = t.PX + (g.M + 3);
    t.PZ = t.PY + (g.N + 3);
    t.RT = reinterpret_cast<float2*>(t.PZ + ((g.Z + 3 + 1) & ~1));
    for (int q = threadIdx.x; q < g.M + 3; q += BP_THREADS) t.PX[q] = g.px[q];
    for (int q = threadIdx.x; q < g.N + 3; q += BP_THREADS) t.PY[q] = g.py[q];
    for (int q = threadIdx.x; q < g.Z + 3; q += BP_THREADS) t.PZ[q] = g.pz[q];
    for (int q = threadIdx.x; q < g.ZP; q += BP_THREADS) t.RT[q] = g.rowt[q];
    __syncthreads();
    return t;
}

// Candidate detector columns of voxel column (i, j) and candidate rows of
// its BP_K voxels: the reference's bounding rectangle of the corner
// projections (universal.cu:639-706).  u depends on the corner's x, y only;
// the z projection scales by 1 + (t-DOD)/(DSO-t), bounded by its extremes
// over the 4 xy corners.  The rows are those of the band of nvr rows from
// row0 seen from a source at height zs (one band for every style but the
// tetrahedron beam).  Returns false when the column misses the detector.
__device__ __forceinline__ bool candidate_rect(const DevGeom& g, const SharedTables& T, float cx, float cy, int k0,
                                               float s, float c, float zs, int row0, int& ulo, int& uhi, int* vlo,
                                               int* vhi)
{
    float umin = __int_as_float(0x7f800000), umax = -umin, mlo = umin, mhi = -umin;
#pragma unroll
    for (int cc = 0; cc < 4; ++cc) {
        const float pxc = fs(fa(cx, fm((float)(cc & 1), g.vx)), fm(0.5f, g.vx));
        const float pyc = fs(fa(cy, fm((float)(cc >> 1), g.vy)), fm(0.5f, g.vy));
        const float t = fa(fm(pxc, c), fm(pyc, s));
        const float ss = fa(fm(-pxc, s), fm(pyc, c));
        // magnification of the corner (universal.cu:655-670); a parallel beam has none
        const float mt = g.ct_style == 2 ? 0.0f : fdv(fs(t, g.dod), fs(g.dso, t));
        const float ou = fa(fm(mt, fs(ss, g.srcy)), ss);
        umin = fminf(umin, ou); umax = fmaxf(umax, ou);
        mlo = fminf(mlo, mt); mhi = fmaxf(mhi, mt);
    }
    // rays parallel to the xy plane: rows in the voxel's z span
    if (g.ct_style == 1 || g.ct_style == 2) { mlo = 0.0f; mhi = 0.0f; }
    ulo = __float2int_rd(fa(fm(fs(umin, g.ymin), g.inv_du), 0.5f));
    uhi = __float2int_rd(fa(fm(fs(umax, g.ymin), g.inv_du), 0.5f));
    if ((ulo < 0 && uhi < 0) || (ulo > g.R - 1 && uhi > g.R - 1)) return false;
    ulo = max(ulo, 0);
    uhi = min(uhi, g.R - 1);
#pragma unroll
    for (int kk = 0; kk < BP_K; ++kk) {
        const int k = k0 + kk;
        vlo[kk] = 1; vhi[kk] = 0;
        if (k < g.Z) {
            const float z0 = T.PZ[k + 1], z1 = T.PZ[k + 2];
            const float zlo = fs(z0, zs), zhi = fs(z1, zs);
            const float a0 = fa(fm(mlo, zlo), z0), a1 = fa(fm(mhi, zlo), z0);
            const float b0 = fa(fm(mlo, zhi), z1), b1 = fa(fm(mhi, zhi), z1);
            const float zmn = fminf(fminf(a0, a1), fminf(b0, b1));
            const float zmx = fmaxf(fmaxf(a0, a1), fmaxf(b0, b1));
            const int lo = __float2int_rd(fa(fm(fs(zmn, g.zmin), g.inv_dv), 0.5f));
            const int hi = __float2int_rd(fa(fm(fs(zmx, g.zmin), g.inv_dv), 0.5f));
            if (!((lo < 0 && hi < 0) || (lo > g.nvr - 1 && hi > g.nvr - 1))) {
                vlo[kk] = row0 + max(lo, 0);
                vhi[kk] = row0 + min(hi, g.nvr - 1);
            }
        }
    }
    return true;
}

__device__ __forceinline__ float rec_value(const float2& r) { return r.x; }
__device__ __forceinline__ float rec_d12(const float2& r) { return r.y; }
__device__ __forceinline__ float rec_value(const AdjRay& r) { return r.f.x; }
__device__ __forceinline__ float rec_d12(const AdjRay& r) { return r.f.y; }

// SART update (SART=true) or the reference's command 0 (SART=false).
template <typename VT, typename REC, bool SART, bool STOCH>
__global__ void __launch_bounds__(BP_THREADS)
k_backproject(const DevGeom g, VT* __restrict__ vol, const REC* __restrict__ rays, int view0, int accumulate,
              float beta, uint32_t seed, const uint32_t* __restrict__ pass_seed)
{
    if (STOCH && pass_seed) seed = *pass_seed * 0x9E3779B9u + (uint32_t)view0;
    extern __shared__ float sp[];
    const SharedTables T = load_tables(g, sp);
    const int i = blockIdx.x * BP_BX + (threadIdx.x % BP_BX);
    const int j = blockIdx.y * BP_BY + (threadIdx.x / BP_BX);
    const int k0 = blockIdx.z * BP_K;
    if (i >= g.M || j >= g.N) return;
    const int R = g.R;

    // FOV cylinder (universal.cu:626-628)
    const float ex = fs(fs((float)i, g.fov_h_x), g.m_off);
    const float ey = fs((float)j, g.fov_h_y);
    const bool masked = fa(fm(fm(fm(ex, g.vx), ex), g.vx), fm(fm(fm(ey, g.vy), ey), g.vy)) >= g.fov_r2;

    float sw[BP_K], sl[BP_K];
#pragma unroll
    for (int kk = 0; kk < BP_K; ++kk) { sw[kk] = 0.f; sl[kk] = 0.f; }

    if (!masked) {
        const float cx = fa(fa(g.bx, fm(g.vx, 0.5f)), fm((float)i, g.vx));   // :592-594
        const float cy = fa(fa(g.by, fm(g.vy, 0.5f)), fm((float)j, g.vy));
        const float xlo = T.PX[i + 1], xhi = T.PX[i + 2];
        const float ylo = T.PY[j + 1], yhi = T.PY[j + 2];
        const float2 sc = g.trig[view0];
        int ulo, uhi, vlo[BP_K], vhi[BP_K];
        if (candidate_rect(g, T, cx, cy, k0, sc.x, sc.y, g.srcz, 0, ulo, uhi, vlo, vhi)) {
            const float4* __restrict__ colt = g.colt + (long long)view0 * R;
            // the detector columns whose ray column crosses this voxel column
            // form one run; find it first so that lanes loop over it in step
            int ua = uhi + 1, ub = ulo - 1;
            for (int uu = ulo; uu <= uhi; ++uu) {
                const float4 ct = __ldg(colt + uu);
                const float ax0 = fm(fs(xlo, ct.x), ct.y), ax1 = fm(fs(xhi, ct.x), ct.y);
                const float ay0 = fm(fs(ylo, ct.z), ct.w), ay1 = fm(fs(yhi, ct.z), ct.w);
                if (fminf(fmaxf(ax0, ax1), fmaxf(ay0, ay1)) > fmaxf(fminf(ax0, ax1), fminf(ay0, ay1))) {
                    ua = min(ua, uu);
                    ub = uu;
                }
            }
            // per voxel, row by row (rows ascending), the columns of the run
            // ascending: the walk's and the oracle's order
#pragma unroll
            for (int kk = 0; kk < BP_K; ++kk) {
                const int kc = min(k0 + kk, g.Z - 1);
                const float zl = T.PZ[kc + 1], zh = T.PZ[kc + 2];
                for (int vv = vlo[kk]; vv <= vhi[kk]; ++vv) {
                    const float2 rt = T.RT[vv];
                    const float az0 = fm(fs(zl, rt.x), rt.y), az1 = fm(fs(zh, rt.x), rt.y);
                    for (int uu = ua; uu <= ub; ++uu) {
                        const float4 ct = __ldg(colt + uu);
                        const float ax0 = fm(fs(xlo, ct.x), ct.y), ax1 = fm(fs(xhi, ct.x), ct.y);
                        const float ay0 = fm(fs(ylo, ct.z), ct.w), ay1 = fm(fs(yhi, ct.z), ct.w);
                        const float a = fmaxf(fminf(ax0, ax1), fminf(ay0, ay1));
                        const float bb = fminf(fmaxf(ax0, ax1), fmaxf(ay0, ay1));
                        if (!(bb > a)) continue;
                        const float lo = fmaxf(a, fminf(az0, az1));
                        const float hi = fminf(bb, fmaxf(az0, az1));
                        const REC rec = rays[(long long)vv * R + uu];
                        const float temp = fm(rec_d12(rec), fs(hi, lo));
                        if (temp > g.thr_bp) {                                 // :785-791
                            sw[kk] = fa(sw[kk], fm(temp, rec_value(rec)));
                            sl[kk] = fa(sl[kk], temp);
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
            if (!(sl[kk] < g.thr_bp)) {                                         // :799-806
                const float nv = fa(Store<VT>::ldw(p), fdv(fm(beta, sw[kk]), sl[kk]));
                if (STOCH) st_sr<VT>(p, nv, hash32(seed ^ hash32((uint32_t)(k * MN + j * g.M + i))));
                else Store<VT>::st(p, nv);
            }
        } else {
            // command 0: assignment where the summed length passes
            if (!(sl[kk] < g.thr_bp)) Store<VT>::st(p, accumulate ? fa(Store<VT>::ldw(p), sw[kk]) : sw[kk]);
            else if (!accumulate) Store<VT>::st(p, 0.0f);
        }
    }
}

// z alphas of every (cell k, detector row v) pair, ordered: the values the
// gather backprojectors otherwise compute per pair from the row table,
// (plane - x1z) * (1/dz) for the cell's two planes.
__global__ void k_zcell(const DevGeom g, float2* __restrict__ zcell)
{
    const long long n = (long long)g.Z * g.ZP;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t / g.ZP), v = (int)(t % g.ZP);
        const float2 rt = g.rowt[v];
        const float az0 = fm(fs(g.pz[k + 1], rt.x), rt.y), az1 = fm(fs(g.pz[k + 2], rt.x), rt.y);
        zcell[t] = make_float2(fminf(az0, az1), fmaxf(az0, az1));
    }
}

ctr_status launch_zcell(const Geometry& G, float2* zcell, cudaStream_t st)
{
    const long long n = (long long)G.dg.Z * G.dg.ZP;
    k_zcell<<<(int)std::min<long long>((n + 255) / 256, 148LL * 64), 256, 0, st>>>(G.dg, zcell);
    CTR_CUDA_TRY(cudaGetLastError());
    return CTR_OK;
}

// SART update by voxel-column walk.  A thread owns a run of up to zl voxels
// of one (i, j) column: the column's xy work -- FOV test, detector-column
// bounds from the corner projections, the run of detector columns whose
// rays cross the column and their xy entry/exit alphas -- is done once and
// kept in registers while the thread walks down its voxels; per voxel only
// the candidate detector rows and the z alphas of each (column, row) pair
// remain.  Every voxel sums its rays in the same order as k_backproject
// (detector column ascending, then row ascending) with the same
// arithmetic, so the two give bit-identical volumes.
//
// TB: the tetrahedron beam (T42/voxel/kernel_IterativeRecon_TBCT_voxel.cu:
// 546-775).  Per voxel, the sources whose band can see it
// (source_lower <= z_src <= source_upper, evaluated as T42 does at :620-627)
// each contribute the sums over their own rows (column, then row, as
// above); the sources are added in ascending order, and the update applies
// where the summed length exceeds vx*1e-3 (:772).
constexpr int WALK_RUN = 4;   // detector columns of the run kept in registers
constexpr float ROW_EPS = 1.0f / 32.0f;   // margin of the alpha-range row estimate, in rows

// The walk's plane and row tables in shared memory: their addresses, and the
// tables themselves (the caller syncs).
__device__ __forceinline__ void walk_tables_addr(const DevGeom& g, float* sp, float*& PX, float*& PY, float*& PZ,
                                                 float2*& RT)
{
    PX = sp;
    PY = PX + (g.M + 3);
    PZ = PY + (g.N + 3);
    RT = reinterpret_cast<float2*>(PZ + ((g.Z + 3 + 1) & ~1));
}
__device__ __forceinline__ void walk_tables(const DevGeom& g, float* sp, float*& PX, float*& PY, float*& PZ,
                                            float2*& RT)
{
    walk_tables_addr(g, sp, PX, PY, PZ, RT);
    for (int q = threadIdx.x; q < g.M + 3; q += blockDim.x) PX[q] = g.px[q];
    for (int q = threadIdx.x; q < g.N + 3; q += blockDim.x) PY[q] = g.py[q];
    for (int q = threadIdx.x; q < g.Z + 3; q += blockDim.x) PZ[q] = g.pz[q];
    for (int q = threadIdx.x; q < g.ZP; q += blockDim.x) RT[q] = g.rowt[q];
}

// One block of the walk: voxel rows by*BY.. and x voxels bx*32.. of z run bz
// (zl voxels).  k_sart_walk runs it as its own block; the batch's persistent
// pass runs the blocks of every scan's view in turn, with coherent loads of
// the ray records (COH: written by other blocks of that launch).
template <typename VT, bool STOCH, int BY, bool TL, int UNR, bool TB, bool COH = false>
__device__ __forceinline__ void walk_block(const DevGeom& g, const float* __restrict__ PX,
                                           const float* __restrict__ PY, const float* __restrict__ PZ,
                                           const float2* __restrict__ RT, int bx, int by, int bz,
                                           VT* __restrict__ vol, const float2* __restrict__ rays, int view,
                                           float beta, uint32_t seed, int zl)
{
    // A warp leaves together or not at all: the lanes of a warp that stays
    // and have nothing to do (past the volume's x edge, outside the FOV
    // cylinder, missing the detector) run on as idle lanes with no columns
    // and no rows, so that the warp-wide reductions below always have all
    // 32 lanes.  Idle lanes read only in-range addresses and store nothing.
    const int i = bx * 32 + (threadIdx.x & 31);
    const int j = by * BY + (threadIdx.x >> 5);
    if (j >= g.N) return;   // the whole warp
    const int ic = min(i, g.M - 1);
    const int kb = bz * zl, ke = min(g.Z, kb + zl);

    // FOV cylinder (universal.cu:626-628): masked voxels keep their value
    const float ex = fs(fs((float)i, g.fov_h_x), g.m_off);
    const float ey = fs((float)j, g.fov_h_y);
    bool live = i < g.M && fa(fm(fm(fm(ex, g.vx), ex), g.vx), fm(fm(fm(ey, g.vy), ey), g.vy)) < g.fov_r2;

    const float cx = fa(fa(g.bx, fm(g.vx, 0.5f)), fm((float)ic, g.vx));   // :592-594
    const float cy = fa(fa(g.by, fm(g.vy, 0.5f)), fm((float)j, g.vy));
    const float xlo = PX[ic + 1], xhi = PX[ic + 2];
    const float ylo = PY[j + 1], yhi = PY[j + 2];
    const float2 sc = g.trig[view];
    const float s = sc.x, c = sc.y;

    // detector-column bounds of the corner projections (universal.cu:639-706)
    float umin = __int_as_float(0x7f800000), umax = -umin, mlo = umin, mhi = -umin;
#pragma unroll
    for (int cc = 0; cc < 4; ++cc) {
        const float pxc = fs(fa(cx, fm((float)(cc & 1), g.vx)), fm(0.5f, g.vx));
        const float pyc = fs(fa(cy, fm((float)(cc >> 1), g.vy)), fm(0.5f, g.vy));
        const float t = fa(fm(pxc, c), fm(pyc, s));
        const float ss = fa(fm(-pxc, s), fm(pyc, c));
        // magnification of the corner (universal.cu:655-670); a parallel beam has none
        const float mt = g.ct_style == 2 ? 0.0f : fdv(fs(t, g.dod), fs(g.dso, t));
        const float ou = fa(fm(mt, fs(ss, g.srcy)), ss);
        umin = fminf(umin, ou); umax = fmaxf(umax, ou);
        mlo = fminf(mlo, mt); mhi = fmaxf(mhi, mt);
    }
    // rays parallel to the xy plane: rows in the voxel's z span
    if (g.ct_style == 1 || g.ct_style == 2) { mlo = 0.0f; mhi = 0.0f; }
    int ulo = __float2int_rd(fa(fm(fs(umin, g.ymin), g.inv_du), 0.5f));
    int uhi = __float2int_rd(fa(fm(fs(umax, g.ymin), g.inv_du), 0.5f));
    if ((ulo < 0 && uhi < 0) || (ulo > g.R - 1 && uhi > g.R - 1)) live = false;
    ulo = max(ulo, 0);
    uhi = min(uhi, g.R - 1);
    if (!live) { ulo = 1; uhi = 0; }   // an idle lane searches no column

    // the run of detector columns whose ray column crosses this voxel column
    const float4* __restrict__ colt = g.colt + (long long)view * g.R;
    int ua = uhi + 1, ub = ulo - 1;
    float amin = 1.0f, bmax = 0.0f;   // the run's alpha range inside the voxel column
    for (int uu = ulo; uu <= uhi; ++uu) {
        const float4 ct = __ldg(colt + uu);
        const float ax0 = fm(fs(xlo, ct.x), ct.y), ax1 = fm(fs(xhi, ct.x), ct.y);
        const float ay0 = fm(fs(ylo, ct.z), ct.w), ay1 = fm(fs(yhi, ct.z), ct.w);
        const float a = fmaxf(fminf(ax0, ax1), fminf(ay0, ay1)), bb = fminf(fmaxf(ax0, ax1), fmaxf(ay0, ay1));
        if (bb > a) {
            ua = min(ua, uu);
            ub = uu;
            amin = fminf(amin, a);
            bmax = fmaxf(bmax, bb);
        }
    }
    if (ua > ub) live = false;
    if (__all_sync(0xffffffffu, !live)) return;   // the whole warp is idle
    // every column of the run crosses the voxel column (bb > a); an idle lane
    // keeps a run of one column (0) whose alpha interval is empty (below)
    if (!live) { ua = 0; ub = 0; }
    const int nrun = ub - ua + 1;

    // Candidate detector rows.  A cone-beam ray from source height zs meets
    // height z at alpha where z = x1z + alpha (zs - x1z), so the ray of the
    // row centred at x1z is inside the cell [z0, z1] at some alpha of the
    // run's range [amin, bmax] iff x1z lies between the least of
    // zs + (z0 - zs) / (1 - alpha) and the greatest of zs + (z1 - zs) / (1 - alpha)
    // over alpha = amin, bmax (both bounds are monotone in alpha).  Written
    // as z + (z - zs) m, m = alpha / (1 - alpha), it is the corner estimate's
    // form with the corners' magnifications replaced by the run's alpha
    // range.  The rows whose centre lies in that span widened by ROW_EPS rows
    // (the float error of the span is below 1e-3 rows; a row the projector
    // takes as level, |x1z - zs| < 1e-6 vz, sits inside it) are a superset of
    // the rows with a positive chord; the corner estimate rounds to the
    // nearest row instead, half a row of margin each side.  Both are bounds,
    // not sums: they use fused multiply-adds (their rounding, below 1e-4
    // rows, is inside either margin), and a detector height z maps to the
    // row position z * inv_dv - zmin * inv_dv, offset by the margin.
    float row_off = 0.5f;
    if ((g.ct_style == 0 || g.ct_style == 3) && live && amin > 0.0f && bmax < 1.0f) {
        mlo = __fdividef(amin, fs(1.0f, amin));
        mhi = __fdividef(bmax, fs(1.0f, bmax));
        row_off = ROW_EPS;
    }
    const float zrow0 = -fm(g.zmin, g.inv_dv);
    // an idle lane's lowest row lies far above the table (its corner bounds
    // are finite, for a column of the volume): it has no rows
    const float zrow_lo = live ? fs(zrow0, row_off) : 1e7f, zrow_hi = fa(zrow0, row_off);
    // the warp's longest run: the pair slots every detector row executes
    const int nq = __reduce_max_sync(0xffffffffu, nrun);
    // the run's alpha intervals; a slot beyond the run gets the empty interval
    // [1, 0] (no chord with any row: hi - lo <= -1), so every thread of the
    // warp runs the same pair slots without a test
    float ra[WALK_RUN], rb[WALK_RUN];
#pragma unroll
    for (int q = 0; q < WALK_RUN; ++q) {
        ra[q] = 1.f; rb[q] = 0.f;
        if (live && ua + q <= ub) {
            const float4 ct = __ldg(colt + ua + q);
            const float ax0 = fm(fs(xlo, ct.x), ct.y), ax1 = fm(fs(xhi, ct.x), ct.y);
            const float ay0 = fm(fs(ylo, ct.z), ct.w), ay1 = fm(fs(yhi, ct.z), ct.w);
            ra[q] = fmaxf(fminf(ax0, ax1), fminf(ay0, ay1));
            rb[q] = fminf(fmaxf(ax0, ax1), fmaxf(ay0, ay1));
        }
    }

    const int R = g.R;
    const long long MN = (long long)g.M * g.N;
    // projections of the lower plane of voxel kb; each voxel's upper plane is
    // the next voxel's lower one, so its pair is carried (min and max of
    // four finite values do not depend on the grouping)
    float cmn = 0.f, cmx = 0.f;
    if (!TB) {
        const float z0 = PZ[kb + 1], zlo = fs(z0, g.srcz);
        const float a0 = __fmaf_rn(mlo, zlo, z0), a1 = __fmaf_rn(mhi, zlo, z0);
        cmn = fminf(a0, a1);
        cmx = fmaxf(a0, a1);
    }
    // TB: the depth of the column centre as T42 evaluates it (:568-569, :620)
    float tden = 0.f;
    if (TB) {
        const float cxr = tb_centre_xy(g, g.bx, g.vx, i);
        const float cyr = tb_centre_xy(g, g.by, g.vy, j);
        tden = fs(fa(fm(cxr, c), fm(cyr, s)), g.dod);
    }
    // TB: the range [s0, s1] of sources kept for the current voxel.  Both
    // bounds only grow with k (source_lower and source_upper grow with the
    // voxel's height), so after an estimate at the first voxel each voxel
    // settles them with a comparison or two.
    int s0 = 0, s1 = -1;
    bool s_est = TB;
    // voxel and z-cell row addresses advance by a constant per z step
    const long long vstep = TL ? 64LL * g.Mt * g.Nt : MN;
    // (ic: an idle lane past the x edge loads its neighbour's value and stores nothing)
    VT* pv = vol + (TL ? (long long)tile_index(g, ic, j, kb) : (long long)kb * MN + (long long)j * g.M + ic);
    const float2* __restrict__ zrow = g.zcell + (long long)kb * g.ZP;
    // the z run with NQ pair slots per detector row (NQ = the warp's longest
    // run, at most WALK_RUN; longer runs take the rest from the column table)
    auto z_run = [&](auto nq_c) {
    constexpr int NQ = decltype(nq_c)::value;
    for (int k = kb; k < ke; ++k, pv += vstep, zrow += g.ZP) {
        int vlo = 0, vhi = -1;   // candidate rows (absolute row indices)
        float sw = 0.f, sl = 0.f;
        // selects, not a branch: the sums take the pair only above the
        // threshold (:785-791); the product is formed either way
        auto pair = [&](float a, float bb, float2 zc, float2 rec) {
            const float lo = fmaxf(a, zc.x);
            const float hi = fminf(bb, zc.y);
            const float temp = fm(rec.y, fs(hi, lo));
            const bool on = temp > g.thr_bp;
            const float w = fa(sw, fm(temp, rec.x)), l = fa(sl, temp);
            sw = on ? w : sw;
            sl = on ? l : sl;
        };
        // the pairs of one detector row: its z-cell interval is loaded once and
        // met with every column of the run (columns ascending)
        auto rec = [&](const float2* p) { return COH ? __ldca(p) : __ldg(p); };
        auto row_pairs = [&](int vv, float2 zc) {
            const float2* __restrict__ rr = rays + (long long)vv * R + ua;
#pragma unroll
            for (int q = 0; q < NQ; ++q)   // a slot beyond the run reads the run's last record (no chord)
                pair(ra[q], rb[q], zc, rec(rr + min(q, nrun - 1)));
            if (NQ == WALK_RUN)
                for (int q = WALK_RUN; q < nrun; ++q) {   // runs longer than the registers hold
                    // the column's planes re-read from the shared tables (rare: not kept live)
                    const float4 ct = __ldg(colt + ua + q);
                    const float x0 = PX[i + 1], x1 = PX[i + 2], y0 = PY[j + 1], y1 = PY[j + 2];
                    const float ax0 = fm(fs(x0, ct.x), ct.y), ax1 = fm(fs(x1, ct.x), ct.y);
                    const float ay0 = fm(fs(y0, ct.z), ct.w), ay1 = fm(fs(y1, ct.z), ct.w);
                    pair(fmaxf(fminf(ax0, ax1), fminf(ay0, ay1)), fminf(fmaxf(ax0, ax1), fmaxf(ay0, ay1)), zc,
                         rec(rr + q));
                }
        };
        // every pair of the voxel, row by row (rows ascending), the order the
        // oracle's gather sums them
        // Every lane runs the warp's largest row count (no divergent loop):
        // a lane past its own rows meets the empty z interval [1, 0] (no
        // chord with any column) at a row clamped into the table.  (The
        // tetrahedron beam calls this per source, inside a loop whose trip
        // count differs across lanes; there each lane runs its own rows.)
        auto all_pairs = [&]() {   // vlo..vhi: this lane's rows (none when vlo > vhi)
            if constexpr (TB) {   // this lane's rows, the next row's z-cell load ahead (vlo <= vhi here)
                int vv = vlo;
                float2 zn = __ldg(zrow + vv);
                for (; vv < vhi; ++vv) {
                    const float2 zc = zn;
                    zn = __ldg(zrow + vv + 1);
                    row_pairs(vv, zc);
                }
                row_pairs(vhi, zn);
                return;
            }
            const int nrows = max(vhi - vlo + 1, 0);
            const int wrows = __reduce_max_sync(0xffffffffu, nrows);
            const float2 none = make_float2(1.0f, 0.0f);
            auto row = [&](int r) { return min(max(vlo + r, 0), g.ZP - 1); };
            if (UNR == 2) {   // two rows' z-cell loads in flight, then their pairs in row order
                for (int r = 0; r < wrows; r += 2) {
                    const float2 z0c = __ldg(zrow + row(r)), z1c = __ldg(zrow + row(r + 1));
                    row_pairs(row(r), r < nrows ? z0c : none);
                    if (r + 1 < wrows) row_pairs(row(r + 1), r + 1 < nrows ? z1c : none);
                }
            } else {          // the next row's z-cell load issued before this row's pairs
                float2 zn = __ldg(zrow + row(0));
                for (int r = 0; r < wrows; ++r) {
                    const float2 zc = r < nrows ? zn : none;
                    zn = __ldg(zrow + row(r + 1));
                    row_pairs(row(r), zc);
                }
            }
        };
        // candidate rows of the band [row0, row0 + nvr) seen from height zs
        // through the cell between planes z0 and z1
        auto band_rows = [&](float z0, float z1, float zs, int row0) -> bool {
            const float zlo = fs(z0, zs), zhi = fs(z1, zs);
            const float a0 = __fmaf_rn(mlo, zlo, z0), a1 = __fmaf_rn(mhi, zlo, z0);
            const float b0 = __fmaf_rn(mlo, zhi, z1), b1 = __fmaf_rn(mhi, zhi, z1);
            const float zmn = fminf(fminf(a0, a1), fminf(b0, b1)), zmx = fmaxf(fmaxf(a0, a1), fmaxf(b0, b1));
            const int lo = max(__float2int_ru(__fmaf_rn(zmn, g.inv_dv, zrow_lo)), 0);
            const int hi = min(__float2int_rd(__fmaf_rn(zmx, g.inv_dv, zrow_hi)), g.nvr - 1);
            if (lo > hi) return false;
            vlo = row0 + lo;
            vhi = row0 + hi;
            return true;
        };
        if (!TB) {
            // candidate detector rows of voxel k
            const float z1 = PZ[k + 2], zhi = fs(z1, g.srcz);
            const float b0 = __fmaf_rn(mlo, zhi, z1), b1 = __fmaf_rn(mhi, zhi, z1);
            const float bmn = fminf(b0, b1), bmx = fmaxf(b0, b1);
            const float zmn = fminf(cmn, bmn), zmx = fmaxf(cmx, bmx);
            cmn = bmn;
            cmx = bmx;
            vlo = max(__float2int_ru(__fmaf_rn(zmn, g.inv_dv, zrow_lo)), 0);
            vhi = min(__float2int_rd(__fmaf_rn(zmx, g.inv_dv, zrow_hi)), g.ZP - 1);
            // (a voxel with no rows, an idle lane's included, stays in step with
            // the warp: its sums stay 0, below thr_bp > 0, so it is not updated)
            const float old = Store<VT>::ldw(pv);   // loaded ahead: its latency overlaps the pairs
            all_pairs();
            if (!(sl < g.thr_bp)) {                                            // :799-806
                VT* p = pv;
                const float nv = fa(old, fdv(fm(beta, sw), sl));
                if (STOCH) st_sr<VT>(p, nv, hash32(seed ^ hash32((uint32_t)(k * MN + j * g.M + i))));
                else Store<VT>::st(p, nv);
            }
        } else if (live) {   // no warp-wide step here: an idle lane skips the voxel
            // the sources T42 keeps for this voxel (:620-627): source_lower <= z <= source_upper
            const float czr = tb_centre_z(g, k);
            const float upper = fa(fdv(fm(fs(fa(czr, g.vz), g.zmin), g.dsod), tden), g.zmin);
            const float lower = fa(fdv(fm(fs(fs(czr, g.vz), g.zmax), g.dsod), tden), g.zmax);
            auto zsrc = [&](int q) { return fa(g.zsrc0, fm((float)q, g.zsrc_dz)); };
            // the source heights increase with the index (zsrc_dz > 0), so the
            // kept sources are one range [s0, s1]: estimated by division at the
            // first voxel, then settled by T42's own comparisons
            if (s_est) {
                s_est = false;
                s0 = 0;
                s1 = g.nsrc - 1;
                if (g.nsrc > 1) {
                    s0 = (int)fminf(fmaxf(ceilf(__fdividef(fs(lower, g.zsrc0), g.zsrc_dz)), 0.f), (float)g.nsrc);
                    s1 = (int)fminf(fmaxf(floorf(__fdividef(fs(upper, g.zsrc0), g.zsrc_dz)), -1.f),
                                    (float)(g.nsrc - 1));
                }
            }
            while (s0 > 0 && !(zsrc(s0 - 1) < lower)) --s0;
            while (s0 < g.nsrc && zsrc(s0) < lower) ++s0;
            while (s1 < g.nsrc - 1 && !(zsrc(s1 + 1) > upper)) ++s1;
            while (s1 >= 0 && zsrc(s1) > upper) --s1;
            const float z0 = PZ[k + 1], z1 = PZ[k + 2];
            float WS = 0.f, L = 0.f;
            for (int q = s0; q <= s1; ++q) {
                if (!band_rows(z0, z1, zsrc(q), q * g.nvr)) continue;
                sw = 0.f;
                sl = 0.f;
                all_pairs();
                WS = fa(WS, sw);                                               // :754-755
                L = fa(L, sl);
            }
            if (L > g.thr_upd) {                                               // :772-773
                VT* p = pv;
                const float nv = fa(Store<VT>::ldw(p), fdv(fm(beta, WS), L));
                if (STOCH) st_sr<VT>(p, nv, hash32(seed ^ hash32((uint32_t)(k * MN + j * g.M + i))));
                else Store<VT>::st(p, nv);
            }
        }
    }
    };
    if (nq <= 2) {
        if (nq <= 1) z_run(std::integral_constant<int, 1>());
        else z_run(std::integral_constant<int, 2>());
    } else {
        if (nq == 3) z_run(std::integral_constant<int, 3>());
        else z_run(std::integral_constant<int, WALK_RUN>());
    }
}

template <typename VT, bool STOCH, int BY, int MINB, bool TL, int UNR, bool TB>
__global__ void __launch_bounds__(32 * BY, MINB)
k_sart_walk(const DevGeom g, VT* __restrict__ vol, const float2* __restrict__ rays, int view, float beta,
            uint32_t seed, const uint32_t* __restrict__ pass_seed, int zl)
{
    extern __shared__ float sp[];
    float *PX, *PY, *PZ;
    float2* RT;
    walk_tables(g, sp, PX, PY, PZ, RT);
    __syncthreads();
    if (STOCH && pass_seed) seed = *pass_seed * 0x9E3779B9u + (uint32_t)view;
    walk_block<VT, STOCH, BY, TL, UNR, TB>(g, PX, PY, PZ, RT, blockIdx.x, blockIdx.y, blockIdx.z, vol, rays, view,
                                           beta, seed, zl);
}

// Linear <-> 8x8-tiled copies of a volume (same storage type).  One thread
// per tiled element; padding elements are written as zero.
template <typename T, bool TO_TILED>
__global__ void k_tiling(const DevGeom g, const T* __restrict__ src, T* __restrict__ dst)
{
    const long long n = tiled_count(g);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int w = (int)(t & 63);
        const long long tile = t >> 6;
        const int tx = (int)(tile % g.Mt);
        const long long r = tile / g.Mt;
        const int ty = (int)(r % g.Nt);
        const int k = (int)(r / g.Nt);
        const int i = tx * 8 + (w & 7), j = ty * 8 + (w >> 3);
        const bool in = i < g.M && j < g.N;
        const long long lin = ((long long)k * g.N + j) * g.M + i;
        if (TO_TILED) dst[t] = in ? src[lin] : T(0.0f);
        else if (in) dst[lin] = src[t];
    }
}

ctr_status launch_tiling(const Geometry& G, const void* src, void* dst, ctr_dtype dt, bool to_tiled, cudaStream_t st)
{
    const long long n = tiled_count(G.dg);
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 32);
    CTR_DISPATCH_DTYPE(dt, T, {
        if (to_tiled) k_tiling<T, true><<<blocks, 256, 0, st>>>(G.dg, (const T*)src, (T*)dst);
        else k_tiling<T, false><<<blocks, 256, 0, st>>>(G.dg, (const T*)src, (T*)dst);
    });
    CTR_CUDA_TRY(cudaGetLastError());
    return CTR_OK;
}

// SART backprojector launch shapes the tuner chooses from: voxel rows per
// block, the longest z run per thread (shortened for small volumes so that
// the grid still fills the GPU) and the blocks per SM the registers are
// capped for.
struct BpShape { int rows, zl, minb, unroll; };
static constexpr BpShape kBpShapes[BP_SHAPES] = {{4, 8, 8, 1}, {4, 32, 8, 1}, {4, 32, 8, 2}, {8, 32, 4, 1},
                                                 {4, 128, 8, 1}, {4, 32, 10, 1}};

template <typename VT, bool STOCH, bool TL, bool TB>
static ctr_status launch_sart_walk(const Geometry& G, const BpArgs& a, cudaStream_t st, size_t smem)
{
    const DevGeom& g = G.dg;
    const BpShape sh = kBpShapes[(G.bp_shape >= 0 && G.bp_shape < BP_SHAPES) ? G.bp_shape : 1];
    int zl = sh.zl;
    const long long cols = (long long)g.M * g.N;
    if (!(a.flags & BP_FULL_RUNS))
        while (zl > 1 && cols * ((g.Z + zl - 1) / zl) < 148LL * 2048) zl >>= 1;   // about two waves at least
    const dim3 grid((g.M + 31) / 32, (g.N + sh.rows - 1) / sh.rows, (g.Z + zl - 1) / zl);
    if (grid.z > 65535) return set_error(CTR_ERR_UNSUPPORTED, "too many z runs");
    const float2* rays = (const float2*)a.rays;
    if (sh.rows == 8)
        k_sart_walk<VT, STOCH, 8, 4, TL, 1, TB><<<grid, 256, smem, st>>>(g, (VT*)a.vol, rays, a.view0, a.beta, a.seed,
                                                                     a.pass_seed, zl);
    else if (sh.minb == 10)
        k_sart_walk<VT, STOCH, 4, 10, TL, 1, TB><<<grid, 128, smem, st>>>(g, (VT*)a.vol, rays, a.view0, a.beta, a.seed,
                                                                      a.pass_seed, zl);
    else if (sh.unroll == 2)
        k_sart_walk<VT, STOCH, 4, 8, TL, 2, TB><<<grid, 128, smem, st>>>(g, (VT*)a.vol, rays, a.view0, a.beta, a.seed,
                                                                     a.pass_seed, zl);
    else
        k_sart_walk<VT, STOCH, 4, 8, TL, 1, TB><<<grid, 128, smem, st>>>(g, (VT*)a.vol, rays, a.view0, a.beta, a.seed,
                                                                     a.pass_seed, zl);
    return CTR_OK;
}

// Interval of cell n along one axis under the forward traversal: geometric
// [min(a0,a1), max(a0,a1)], opened at -inf for the start cell, empty behind
// the start; for a parallel axis (-inf, +inf) at the start cell only.
__device__ __forceinline__ bool traversal_cell(int n, int n0, bool par, float a0, float a1, float dirsign,
                                               float& lo, float& hi)
{
    const float INF = __int_as_float(0x7f800000);
    if (par) {
        lo = -INF;
        hi = INF;
        return n == n0;
    }
    const int d = n - n0;
    if ((dirsign > 0.f && d < 0) || (dirsign < 0.f && d > 0)) return false;
    lo = d == 0 ? -INF : fminf(a0, a1);
    hi = fmaxf(a0, a1);
    return true;
}

template <typename VT>
__global__ void __launch_bounds__(BP_THREADS)
k_adjoint(const DevGeom g, VT* __restrict__ vol, const AdjRay* __restrict__ rays, int view0, int nview,
          int accumulate)
{
    extern __shared__ float sp[];
    const SharedTables T = load_tables(g, sp);
    const int i = blockIdx.x * BP_BX + (threadIdx.x % BP_BX);
    const int j = blockIdx.y * BP_BY + (threadIdx.x / BP_BX);
    const int k0 = blockIdx.z * BP_K;
    if (i >= g.M || j >= g.N) return;
    const int R = g.R, ZP = g.ZP;
    double acc[BP_K];
#pragma unroll
    for (int kk = 0; kk < BP_K; ++kk) acc[kk] = 0.0;
    const float cx = fa(fa(g.bx, fm(g.vx, 0.5f)), fm((float)i, g.vx));
    const float cy = fa(fa(g.by, fm(g.vy, 0.5f)), fm((float)j, g.vy));
    const float xlo = T.PX[i + 1], xhi = T.PX[i + 2];
    const float ylo = T.PY[j + 1], yhi = T.PY[j + 2];
    for (int w = 0; w < nview; ++w)
    for (int src = 0; src < g.nsrc; ++src) {   // each source's band of rows (one band but for TBCT)
        const int view = view0 + w;
        const float2 sc = g.trig[view];
        const float zs = g.ct_style == 3 ? fa(g.zsrc0, fm((float)src, g.zsrc_dz)) : g.srcz;
        int ulo, uhi, vlo[BP_K], vhi[BP_K];
        if (!candidate_rect(g, T, cx, cy, k0, sc.x, sc.y, zs, src * g.nvr, ulo, uhi, vlo, vhi)) break;
        bool rows = false;
#pragma unroll
        for (int kk = 0; kk < BP_K; ++kk) rows |= vlo[kk] <= vhi[kk];
        if (!rows) continue;
        const float4* __restrict__ colt = g.colt + (long long)view * R;
        const AdjRay* __restrict__ rw = rays + (long long)w * R * ZP;
        for (int uu = ulo; uu <= uhi; ++uu) {
            const float4 ct = __ldg(colt + uu);
            const float ax0 = fm(fs(xlo, ct.x), ct.y), ax1 = fm(fs(xhi, ct.x), ct.y);
            const float ay0 = fm(fs(ylo, ct.z), ct.w), ay1 = fm(fs(yhi, ct.z), ct.w);
#pragma unroll
            for (int kk = 0; kk < BP_K; ++kk) {
                const int k = k0 + kk;
                const int kc = min(k, g.Z - 1);
                const float zl = T.PZ[kc + 1], zh = T.PZ[kc + 2];
                for (int vv = vlo[kk]; vv <= vhi[kk]; ++vv) {
                    const AdjRay rec = rw[(long long)vv * R + uu];
                    const float2 rt = T.RT[vv];
                    const float az0 = fm(fs(zl, rt.x), rt.y), az1 = fm(fs(zh, rt.x), rt.y);
                    float exl, exh, eyl, eyh, ezl, ezh;
                    if (!traversal_cell(i, rec.i.x, rec.i.w & 1, ax0, ax1, ct.y, exl, exh)) continue;
                    if (!traversal_cell(j, rec.i.y, rec.i.w & 2, ay0, ay1, ct.w, eyl, eyh)) continue;
                    if (!traversal_cell(k, rec.i.z, rec.i.w & 4, az0, az1, rt.y, ezl, ezh)) continue;
                    const float lo = fmaxf(fmaxf(exl, eyl), fmaxf(ezl, rec.f.z));
                    const float hi = fminf(fminf(exh, eyh), fminf(ezh, rec.f.w));
                    const float temp = fm(rec.f.y, fs(hi, lo));
                    const bool start = (i == rec.i.x) && (j == rec.i.y) && (k == rec.i.z);
                    // the traversal's first segment may be a rounding-size negative length
                    if (temp > 0.0f || (start && rec.f.z <= rec.f.w))
                        acc[kk] = __fma_rn((double)temp, (double)rec.f.x, acc[kk]);
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
        const double v = accumulate ? (double)Store<VT>::ldw(p) + acc[kk] : acc[kk];
        Store<VT>::st(p, (float)v);
    }
}

static size_t bp_smem(const DevGeom& g)
{
    return sizeof(float) * (size_t)(g.M + 3 + g.N + 3 + ((g.Z + 3 + 1) & ~1)) + sizeof(float2) * g.ZP;
}

// ------------------------------------------------- the batch's persistent pass

int walk_z_run(const DevGeom& g)
{
    int zl = kBpShapes[1].zl;
    const long long cols = (long long)g.M * g.N;
    while (zl > 1 && cols * ((g.Z + zl - 1) / zl) < 148LL * 2048) zl >>= 1;
    return zl;
}

// forward tables (rounded to 8 bytes), then the walk's
__host__ __device__ __forceinline__ size_t fp_table_floats(const DevGeom& g)
{
    return ((size_t)(g.M + g.N + g.Z + 16) + 1) & ~(size_t)1;
}
size_t batch_pass_smem(const DevGeom& g) { return sizeof(float) * fp_table_floats(g) + bp_smem(g); }

constexpr unsigned long long kIdleNs = 4000000000ull;   // a block idles at most 4 s (by the global timer)

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// blocks of phase ph of a scan: view ph/2's forward projection (even) or walk (odd)
__device__ __forceinline__ unsigned flow_blocks(const BatchScan& S, unsigned ph)
{
    return (ph & 1u) ? (unsigned)(S.bp_gx * S.bp_gy * S.bp_gz) : (unsigned)(S.fp_gx * S.fp_gy);
}

// Thread 0 of a block: claim one block of work, from the home scan first,
// then round the other scans; returns the scan (phase and block in ph, blk),
// or -1 once every scan is done or an error was flagged.  With nothing to
// claim (every scan's current phase handed out, its last blocks still
// running) it polls again after a sleep that doubles up to 4 us; idle past
// kIdleNs it flags ERR_BARRIER and returns -1.
__device__ __forceinline__ int flow_claim(const BatchScan* __restrict__ scans, int nscans, int home,
                                          BatchFlow* flow, unsigned* finished, unsigned* err, unsigned& ph, int& blk,
                                          int& cnt)
{
    unsigned sleep_ns = 64;
    const unsigned long long t0 = global_ns();
    for (;;) {
        if (*(volatile unsigned*)err != 0u || *(volatile unsigned*)finished >= (unsigned)nscans) return -1;
        for (int t = 0; t < nscans; ++t) {
            const int s = home + t < nscans ? home + t : home + t - nscans;
            const BatchScan& S = scans[s];
            const unsigned last = 2u * (unsigned)S.nviews;
            const unsigned long long w = *(volatile unsigned long long*)&flow[s].claim;
            const unsigned p = (unsigned)(w >> 32), nb = flow_blocks(S, p);
            if (p >= last || (unsigned)w >= nb) continue;
            // a chunk of up to 8 blocks per claim (1 per 128 of the phase):
            // one claim's latency serves several blocks
            const unsigned k = max(1u, min(8u, nb / 128u));
            const unsigned long long o = atomicAdd(&flow[s].claim, (unsigned long long)k);
            const unsigned p2 = (unsigned)(o >> 32), nb2 = flow_blocks(S, p2), c2 = (unsigned)o;
            if (p2 < last && c2 < nb2) {
                ph = p2;
                blk = (int)c2;
                cnt = (int)min(k, nb2 - c2);
                return s;
            }
        }
        if (global_ns() - t0 > kIdleNs) {
            atomicOr(err, ERR_BARRIER);
            return -1;
        }
        __nanosleep(sleep_ns);
        sleep_ns = min(2u * sleep_ns, 4096u);
    }
}

// The SART pass of every scan of a batch in one launch, scheduled as a data
// flow.  A scan's phases run in order (view j's forward projection, its
// walk, view j+1's forward projection, ...); the blocks of a phase run in any
// order on any CTA.  A CTA takes the next chunk of blocks (1-8) of its home
// scan's current phase, else of any other scan's, so no CTA waits while some
// scan has a block to give.  The phase's last chunk to finish opens the next
// phase: each chunk releases its writes (fence, then its count), the last
// one resets the count and moves the claim word on (fence first); a CTA that
// claims a chunk fences before reading (acquire), and reads the ray records
// and volumes the launch writes with coherent loads.  Each block runs the
// per-ray and per-voxel code of k_forward (shape 1) and k_sart_walk (shape
// 1), every voxel sees its views in order, so every scan's result equals
// its solver's.  No block waits for a particular other block, so the CTAs
// need not be co-resident; an idle CTA's wait is bounded (flow_claim).
// 5 blocks per SM: 96 registers hold the forward and walk code without
// spills (80, at 6 per SM, spilled 250-400 bytes a thread).
template <typename VT, int KIND, bool STOCH>
__global__ void __launch_bounds__(128, 5)
k_batch_pass(const BatchScan* __restrict__ scans, int nscans, BatchFlow* __restrict__ flow,
             unsigned* __restrict__ finished, unsigned* __restrict__ err)
{
    extern __shared__ float sp[];
    __shared__ int s_scan, s_blk, s_cnt;
    __shared__ unsigned s_ph;
    int home = 0;
    {   // the last scan whose first home CTA is at or before this one
        int lo = 0, hi = nscans - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (scans[mid].c0 <= (int)blockIdx.x) lo = mid;
            else hi = mid - 1;
        }
        home = lo;
    }
    int cur = -1;   // the scan whose tables are in shared memory
    for (;;) {
        if (threadIdx.x == 0) {
            unsigned ph = 0;
            int blk = 0, cnt = 0;
            const int s = flow_claim(scans, nscans, home, flow, finished, err, ph, blk, cnt);
            __threadfence();   // acquire: the phase before ph is complete
            s_scan = s;
            s_ph = ph;
            s_blk = blk;
            s_cnt = cnt;
        }
        __syncthreads();
        const int s = s_scan;
        if (s < 0) return;
        const BatchScan& S = scans[s];
        const DevGeom& g = S.g;
        float *PX, *PY, *PZ, *PINF, *WX, *WY, *WZ;   // recomputed per block, not kept live across blocks
        float2* RT;
        if (s != cur) {   // this scan's plane tables
            fp_tables(g, sp, PX, PY, PZ, PINF);
            walk_tables(g, sp + fp_table_floats(g), WX, WY, WZ, RT);
            __syncthreads();
            cur = s;
        }
        plane_tables_addr(g, sp, PX, PY, PZ, PINF);
        walk_tables_addr(g, sp + fp_table_floats(g), WX, WY, WZ, RT);
        const unsigned ph = s_ph;
        const int j = (int)(ph >> 1), cnt = s_cnt;
        for (int vb = s_blk; vb < s_blk + cnt; ++vb) {   // the claimed chunk of the phase
            if ((ph & 1u) == 0u) {
                const long long P = (long long)g.R * g.ZP;
                const size_t per_view = (size_t)g.ZP * S.fp_gx;
                const size_t bsz = S.b_dt == CTR_F32 ? 4 : 2;
                fp_block<VT, KIND, false, 4, 0, true, false, true>(
                    g, PX, PY, PZ, PINF, vb % S.fp_gx, vb / S.fp_gx, 0, S.fp_gx, S.fp_gy, (const VT*)S.fp_vol, j,
                    S.rays, 0, (const char*)S.b + (size_t)j * P * bsz, S.b_dt,
                    S.partial ? S.partial + (size_t)j * per_view : nullptr, nullptr, nullptr, nullptr, S.fp_vol2,
                    S.ax ? S.ax + (size_t)j * P : nullptr, S.gdev);
            } else {
                // the updated volume: the FP32 correction of FP_SART_REFINE32, else the storage type
                using WT = typename std::conditional<KIND == FP_SART_REFINE32, float, VT>::type;
                constexpr bool WSTOCH = STOCH && !std::is_same<WT, float>::value;
                const uint32_t seed = WSTOCH ? *S.pass_seed * 0x9E3779B9u + (uint32_t)j : 0u;
                const int bx = vb % S.bp_gx, r = vb / S.bp_gx, by = r % S.bp_gy, bz = r / S.bp_gy;
                if (g.ct_style == 3)
                    walk_block<WT, WSTOCH, 4, true, 1, true, true>(g, WX, WY, WZ, RT, bx, by, bz, (WT*)S.bp_vol,
                                                                   S.rays, j, S.beta, seed, S.zl);
                else
                    walk_block<WT, WSTOCH, 4, true, 1, false, true>(g, WX, WY, WZ, RT, bx, by, bz, (WT*)S.bp_vol,
                                                                    S.rays, j, S.beta, seed, S.zl);
            }
        }
        __syncthreads();   // the chunk's writes are issued
        if (threadIdx.x == 0) {
            __threadfence();   // release them
            const unsigned d = atomicAdd(&flow[s].done, (unsigned)cnt) + (unsigned)cnt;
            if (d == flow_blocks(S, ph)) {   // the phase's last chunk opens the next
                atomicExch(&flow[s].done, 0u);
                __threadfence();
                atomicExch(&flow[s].claim, (unsigned long long)(ph + 1u) << 32);
                if (ph + 1u == 2u * (unsigned)S.nviews) atomicAdd(finished, 1u);
            }
        }
    }
}

template <typename VT, int KIND, bool STOCH>
static const void* batch_pass_fn()
{
    return reinterpret_cast<const void*>(&k_batch_pass<VT, KIND, STOCH>);
}

static const void* batch_pass_kernel(ctr_dtype vdt, int kind, bool stoch)
{
    const void* f = nullptr;
    auto pick = [&](auto tag) {
        using VT = decltype(tag);
        if (kind == FP_SART) f = stoch ? batch_pass_fn<VT, FP_SART, true>() : batch_pass_fn<VT, FP_SART, false>();
        else if (kind == FP_SART_OBJ)
            f = stoch ? batch_pass_fn<VT, FP_SART_OBJ, true>() : batch_pass_fn<VT, FP_SART_OBJ, false>();
        else if (kind == FP_SART_REFINE)
            f = stoch ? batch_pass_fn<VT, FP_SART_REFINE, true>() : batch_pass_fn<VT, FP_SART_REFINE, false>();
        else if (kind == FP_SART_REFINE32) {   // FP32 correction: no stochastic rounding
            if constexpr (std::is_same<VT, float>::value) f = batch_pass_fn<VT, FP_SART_REFINE, false>();
            else f = batch_pass_fn<VT, FP_SART_REFINE32, false>();
        }
    };
    if (vdt == CTR_F32) pick(float());
    else if (vdt == CTR_BF16) pick(__nv_bfloat16());
    else if (vdt == CTR_F16) pick(__half());
    return f;
}

int batch_pass_blocks_per_sm(ctr_dtype vdt, int kind, bool stoch, size_t smem)
{
    const void* f = batch_pass_kernel(vdt, kind, stoch);
    if (!f) return 0;
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, 128, smem) != cudaSuccess) return 0;
    return n;
}

ctr_status launch_batch_pass(const BatchScan* d_scans, int nscans, int nblocks, ctr_dtype vdt, int kind, bool stoch,
                             void* flow, unsigned* err, size_t smem, cudaStream_t st)
{
    const void* f = batch_pass_kernel(vdt, kind, stoch);
    if (!f) return set_error(CTR_ERR_UNSUPPORTED, "persistent pass: storage type or kind not supported");
    BatchFlow* fl = (BatchFlow*)flow;
    unsigned* finished = (unsigned*)(fl + nscans);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nblocks);
    cfg.blockDim = dim3(128);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    void* args[] = {(void*)&d_scans, (void*)&nscans, (void*)&fl, (void*)&finished, (void*)&err};
    CTR_CUDA_TRY(cudaLaunchKernelExC(&cfg, f, args));
    return CTR_OK;
}

ctr_status launch_backproject(const Geometry& G, const BpArgs& a, cudaStream_t st)
{
    const DevGeom& g = G.dg;
    if (a.nview <= 0) return CTR_OK;
    const size_t smem = bp_smem(g);
    if (smem > 48 * 1024) return set_error(CTR_ERR_UNSUPPORTED, "plane tables exceed 48 KB of shared memory");
    dim3 grid((g.M + BP_BX - 1) / BP_BX, (g.N + BP_BY - 1) / BP_BY, (g.Z + BP_K - 1) / BP_K);
    const int acc = (a.flags & CTR_BP_ACCUMULATE) ? 1 : 0;
    CTR_DISPATCH_DTYPE(a.vol_dtype, VT, {
        if (a.sart) {
            if (a.nview != 1) return set_error(CTR_ERR_INVALID_ARGUMENT, "SART updates one view at a time");
            const bool sr = (a.flags & CTR_SART_STOCHASTIC_ROUND) != 0;
            if (a.flags & CTR_SART_REFERENCE_BP) {   // the reference backprojector's arithmetic (bp_ref.cu)
                CTR_TRY(launch_sart_ref(G, a, st));
            } else if (g.ct_style == 3) {   // the tetrahedron beam: column walks only (bp_shape -1 runs walk shape 1)
                if (a.tiled) {
                    if (sr) CTR_TRY((launch_sart_walk<VT, true, true, true>(G, a, st, smem)));
                    else CTR_TRY((launch_sart_walk<VT, false, true, true>(G, a, st, smem)));
                } else if (sr) {
                    CTR_TRY((launch_sart_walk<VT, true, false, true>(G, a, st, smem)));
                } else {
                    CTR_TRY((launch_sart_walk<VT, false, false, true>(G, a, st, smem)));
                }
            } else if (a.tiled) {
                if (sr) CTR_TRY((launch_sart_walk<VT, true, true, false>(G, a, st, smem)));
                else CTR_TRY((launch_sart_walk<VT, false, true, false>(G, a, st, smem)));
            } else if (G.bp_shape < 0) {   // the fixed-shape kernel: 8 voxels of a column per thread
                if (a.flags & CTR_SART_STOCHASTIC_ROUND)
                    k_backproject<VT, float2, true, true><<<grid, BP_THREADS, smem, st>>>(
                        g, (VT*)a.vol, (const float2*)a.rays, a.view0, 0, a.beta, a.seed, a.pass_seed);
                else
                    k_backproject<VT, float2, true, false><<<grid, BP_THREADS, smem, st>>>(
                        g, (VT*)a.vol, (const float2*)a.rays, a.view0, 0, a.beta, a.seed, nullptr);
            } else if (sr) {
                CTR_TRY((launch_sart_walk<VT, true, false, false>(G, a, st, smem)));
            } else {
                CTR_TRY((launch_sart_walk<VT, false, false, false>(G, a, st, smem)));
            }
        } else if (a.flags & CTR_BP_FOV_MASK) {
            if (g.ct_style == 3)
                return set_error(CTR_ERR_UNSUPPORTED, "CTR_BP_FOV_MASK (command 0): not defined for the tetrahedron "
                                                      "beam, whose backprojector has no command argument");
            for (int w = 0; w < a.nview; ++w)
                k_backproject<VT, AdjRay, false, false><<<grid, BP_THREADS, smem, st>>>(
                    g, (VT*)a.vol, (const AdjRay*)a.rays + (size_t)w * G.npix(), a.view0 + w, (acc || w > 0) ? 1 : 0,
                    0.f, 0u, nullptr);
        } else {
            k_adjoint<VT><<<grid, BP_THREADS, smem, st>>>(g, (VT*)a.vol, (const AdjRay*)a.rays, a.view0, a.nview, acc);
        }
    });
    CTR_CUDA_TRY(cudaGetLastError());
    return CTR_OK;
}

}  // namespace ctr
