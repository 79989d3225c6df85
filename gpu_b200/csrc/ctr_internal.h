// ctr_internal.h -- types shared by the host library and the CUDA kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/ctrecon.h"

namespace ctr {

// Geometry as the kernels see it (passed by value, lives in the constant bank).
// Every float is derived on the host with the reference's float/double steps
// (V63/main_recon.cu:60-111).
struct DevGeom {
    int M, N, Z;            // volume
    int R, ZP;              // detector columns, rows of a view (all sources' bands for TBCT)
    int nviews;
    int max_steps;          // Siddon step bound nx+ny+nz+3
    int Mt, Nt;             // 8x8 (x, y) tiles per row / column of the tiled layout
    int fast_exit;          // every alpha inside the volume >= 1e-6: the Siddon loop test is one comparison
    int entry64;            // FP64 ray-box entry/exit
    int fast_sums;          // CTR_GEOM_FAST_SUMS: fused ray-sum accumulation in the solver's projections
    int ct_style;           // 0 cone beam, 1 multi-slice fan beam, 2 parallel beam (the reference's CT_style),
                            // 3 tetrahedron beam (CTR_GEOM_TBCT)
    int nvr;                // detector rows of one source's band (= ZP unless TBCT)
    int nsrc;               // sources (1 unless TBCT)
    float vx, vy, vz, inv_vx, inv_vy, inv_vz;
    float bx, by, bz;       // boundary_voxel_*
    float ymin, zmin;       // Detector_Ymin/Zmin
    float du, dv, inv_du, inv_dv;
    float dso, dod;
    float srcx, srcy, srcz;
    float zmax;             // TBCT: Detector_Zmax (T42/main_recon.cu:93)
    float zsrc0, zsrc_dz;   // TBCT: Source_z_min, Source_interval (T42/main_recon.cu:96-108)
    float dsod;             // DSO - DOD in float
    float loop_eps;         // Siddon loop test alpha_max - alpha_c > loop_eps: 1e-16f, TBCT 1e-6f
    float thr_upd;          // TBCT update threshold: L > thr_upd <=> (double)L > (double)vx*1e-3
    float thr_fp;           // volumn_z*1e-6f: FP zero-length threshold
    float thr_bp;           // volumn_x*1e-6f: BP pair and sum thresholds
    float fov_h_x, fov_h_y; // float(M)*0.5f-0.5f, float(N)*0.5f-0.5f
    float fov_r2;           // (hx*vx)*hy*vy
    float m_off;            // (float)M_Offset
    float fdk_ang;          // us_rate*PI/180.0f        (V63/FDK/kernel_FDK.cu:117)
    float fdk_usn;          // us_rate*Nviews in float  (same line)
    int fdk_full;           // fdk_usn == 360: the FP64 factor 360.0/fdk_usn is exactly 1
    // z-slab of the multi-GPU build (V63/kernel_IterativeRecon_universal_multiGPU.cu:591-1402):
    // Z is the slab's ZETA/D slices, bz its BOUNDARY_VOXEL_Z; the whole volume otherwise
    int slab_n, slab_i;     // D (1: no split) and this slab's index (subVolIdx)
    int zpar_kr;            // the single-GPU z-parallel k range applies (not T42's, not a slab's)
    int row_lo, row_hi;     // partial forward: rows traced (a fan-slice / parallel slab: its band; a
                            // cone-beam slab: a conservative band of the rows that can reach it)
    float bz_ref, cz_off;   // reference BP voxel centre z = (bz_ref + cz_off) + k*vz (universal.cu:594,
                            // multiGPU.cu:1179): bz and vz*0.5f, or the whole volume's bz and vz*(k0+0.5f)
    int ref_plus0;          // the reference BP's "+= 0.0f" on voxels without rays (not in a slab's)
    float thr_comb;         // the slab combination's zero-length threshold: volumn_z*1e-6f (V63),
                            // volumn_z*1e-3f (T42/voxel/kernel_IterativeRecon_TBCT_voxel_multiGPU.cu:14)
    const float* px;        // plane coordinates vx*n+bx for n = -1..M+1 at px[n+1]
    const float* py;
    const float* pz;
    const float2* trig;     // [view] (sin, cos) of the FP/SART frame angle
    const float2* trig_fdk; // [view] (sin, cos) of the FDK frame angle
    const float4* colt;     // [view][u] (x1x, 1/dx, x1y, 1/dy), parallel axes encoded
    const float2* rowt;     // [v] (x1z, 1/dz) of every row of a view, parallel rows encoded
    const float2* zcell;    // [k][v] (min, max) of the z alphas of cell k's planes for row v
    const float2* zref;     // [k][v] (min, max) of the reference backprojector's z alphas (CTR_SART_REFERENCE_BP)
    unsigned int* err;      // device error bits (ERR_*)
};

enum : unsigned { ERR_TRAVERSAL = 1u };
constexpr int FP_SHAPES = 7;
constexpr int BP_SHAPES = 6;

struct Geometry {
    ctr_geometry_desc desc{};
    DevGeom dg{};
    int device = 0;
    std::vector<float> h_px, h_py, h_pz;
    std::vector<float2> h_trig, h_trig_fdk;
    // device allocations
    void* d_tables = nullptr;  // px,py,pz,trig,trig_fdk,rowt
    float4* d_colt = nullptr;
    float2* d_zcell = nullptr;
    float2* d_zref = nullptr;
    unsigned* d_err = nullptr;
    // workspace
    void* d_rays = nullptr;  size_t rays_cap = 0;       // ray records (float2 SART / AdjRay adjoint)
    double* d_partial = nullptr; size_t partial_cap = 0;
    double* d_result = nullptr;                        // 8 doubles
    void* d_fgp = nullptr; size_t fgp_bytes = 0;       // 9 dual arrays
    float* d_fdk = nullptr; size_t fdk_cap = 0;
    void* d_tiled = nullptr; size_t tiled_bytes = 0;   // tiled copy for CTR_SART_TILED
    float* d_ramp = nullptr;                           // 2R-1 taps
    // slab geometries of the one-GPU slab SART (ctr_sart_pass_slabs), built on first use,
    // with a stream per slab and the events that order them around the combination
    std::vector<Geometry*> slab_geoms;
    std::vector<cudaStream_t> slab_streams;
    std::vector<cudaEvent_t> slab_events;              // [0, D): per slab; D: combination; D+1: start
    Geometry* split_geom = nullptr;                    // tetrahedron beam: the D-device build's row-split
                                                       // projector (ctr_geometry_create_slab, slab -1)
    void* d_parts = nullptr; size_t parts_cap = 0;     // [D][P] float2 partial ray sums
    // launch shapes (indices into the tuner's tables; results do not depend on them)
    int fp_shape = 1;                                  // FP: see kFpShapes in fp.cu
    int bp_shape = 1;                                  // SART BP: see kBpShapes in bp.cu
    long long nvox() const { return (long long)desc.nx * desc.ny * desc.nz; }
    long long npix() const { return (long long)dg.R * dg.ZP; }
};

// error reporting (thread-local message)
ctr_status set_error(ctr_status st, const char* fmt, ...);
ctr_status cuda_error(cudaError_t e, const char* what);
void clear_error();

#define CTR_CUDA_TRY(call)                                         \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return ::ctr::cuda_error(e_, #call); \
    } while (0)
#define CTR_TRY(call)                          \
    do {                                       \
        ctr_status s_ = (call);                \
        if (s_ != CTR_OK) return s_;           \
    } while (0)

inline size_t dtype_size(ctr_dtype t) { return t == CTR_F32 ? 4 : 2; }
inline bool dtype_ok(int t) { return t == CTR_F32 || t == CTR_BF16 || t == CTR_F16; }

// workspace helpers (geometry.cpp)
ctr_status ensure_rays(Geometry* g, size_t bytes);
ctr_status ensure_partial(Geometry* g, size_t n);
ctr_status ensure_fgp(Geometry* g, size_t bytes);
// FGP workspace: six duals in the storage type and L in FP32
inline size_t fgp_workspace_bytes(long long V, ctr_dtype dt) { return (size_t)V * (6 * dtype_size(dt) + 4); }
ctr_status ensure_tiled(Geometry* g, size_t bytes);
ctr_status check_device_errors(Geometry* g, cudaStream_t st);

// ---- kernel launchers (implemented in the .cu files) ----
// FP_SART_OBJ: the SART correction of vol and, in the same traversal, the
// objective residual (A vol2 - b)^2 of a second volume.
// FP_PARTIAL: a slab's (Sum(len*f), Sum(len)) per ray as float2, no threshold.
// FP_SART_REFINE: the refinement solver's pass.  vol is the 16-bit copy of
// x_k, vol2 the correction volume d; per ray c = (b - ((1+g)Ax_k - g Ax_(k-1))
// - Ad)/len with g = *gdev and Ax_(k-1) read from ax[p], which is then
// overwritten with Ax_k; the objective partials of x_k as FP_SART_OBJ.
// FP_SART_REFINE32: FP_SART_REFINE with the correction volume (vol2) in FP32
// while vol is a 16-bit copy.
enum FpKind { FP_FORWARD = 0, FP_SART = 1, FP_OBJECTIVE = 2, FP_TRACE = 3, FP_DOT = 4, FP_SART_OBJ = 5,
              FP_PARTIAL = 6, FP_SART_REFINE = 7, FP_SART_REFINE32 = 8 };
struct FpArgs {
    const void* vol; ctr_dtype vol_dtype;
    int view0, nview;
    FpKind kind;
    void* out; ctr_dtype out_dtype;       // FORWARD: sino; SART: float2 rays
    const void* b; ctr_dtype b_dtype;     // SART/OBJECTIVE: measured sinogram; DOT: y (offset to view0)
    double* partial;                      // OBJECTIVE, SART_OBJ: one double per warp (32 rays of a row),
                                          // [view - view0][v][u/32]; DOT: one per block
    const void* vol2 = nullptr;           // SART_OBJ: the volume of the objective (same dtype, layout);
                                          // SART_REFINE: the correction d (vol_dtype; FP32 for SART_REFINE32)
    int* nseg; uint64_t* hash; float* len;  // TRACE
    int tiled = 0;                        // vol in the 8x8-tiled layout (FORWARD, SART, OBJECTIVE)
    float* ax = nullptr;                  // SART_REFINE: FP32 ray sums of the previous x copy, this view
    const float* gdev = nullptr;          // SART_REFINE: the FISTA factor g (device)
};
ctr_status launch_forward(const Geometry& g, const FpArgs& a, cudaStream_t st, size_t* nblocks_out);
// objective partials per view: one per warp of 32 rays
inline size_t objective_partials_per_view(const DevGeom& g) { return (size_t)g.ZP * ((g.R + 31) / 32); }

// Internal SART flag (not in the public header): the walk keeps its full z
// runs instead of shortening them to fill the GPU with one scan's blocks (a
// batch's scans fill it together).  The sums do not depend on the runs.
constexpr unsigned BP_FULL_RUNS = 0x40000000u;
struct BpArgs {
    void* vol; ctr_dtype vol_dtype;
    const void* rays;                     // [nview][ZP][R]: float2 (c, d12) for SART and the
                                          // masked (reference command 0) form, AdjRay otherwise
    int view0, nview;
    int sart;                             // 1: SART update; 0: adjoint
    unsigned flags;                       // CTR_BP_* / CTR_SART_*
    float beta;
    uint32_t seed;                        // stochastic rounding: per-view seed
    const uint32_t* pass_seed = nullptr;  // if set, the seed is *pass_seed * 0x9E3779B9 + view (device)
    int tiled = 0;                        // vol in the 8x8-tiled layout (SART only)
};
ctr_status launch_backproject(const Geometry& g, const BpArgs& a, cudaStream_t st);
// The tiled volume layout of the solver's projections: 8x8 tiles in (x, y),
// tile-major within a z slice, so the 32 rays of a warp, which lie side by
// side across the beam, touch a few 128-byte lines instead of one per ray.
// Voxels of the padding (x >= nx or y >= ny in the last tiles) are never read
// or written by the projectors.
__host__ __device__ inline long long tiled_count(const DevGeom& g) { return (long long)g.Z * g.Nt * g.Mt * 64; }
ctr_status launch_tiling(const Geometry& g, const void* src, void* dst, ctr_dtype dt, bool to_tiled, cudaStream_t st);
// fills dg.zcell (view-independent: the rows' z and the source height do not turn)
ctr_status launch_zcell(const Geometry& g, float2* zcell, cudaStream_t st);
// the reference backprojector's z alphas per (cell, row), and its SART update (bp_ref.cu)
ctr_status launch_zref(const Geometry& g, float2* zref, cudaStream_t st);
ctr_status launch_sart_ref(const Geometry& g, const BpArgs& a, cudaStream_t st);
// Matched-adjoint ray record: f = (value, chord length d12, alpha_lo, alpha_hi),
// i = (start voxel i, j, k, parallel-axis bits).
struct __align__(16) AdjRay {
    float4 f;
    int4 i;
};
ctr_status launch_ray_prep(const Geometry& g, const float* y, int view0, int nview, AdjRay* rays,
                           cudaStream_t st);

// slab SART: the slabs' partial sums [n_parts][P] added in slab order, the
// SART correction of view `view` and the ray's d12 -> rays (slabs.cu); with
// b == nullptr the weighted sums alone, as floats
ctr_status launch_combine(const Geometry& g, const float2* parts, int n_parts, int view, const void* b,
                          ctr_dtype b_dt, float2* rays, cudaStream_t st);
ctr_status launch_reduce(const double* partial, size_t n, double* out, cudaStream_t st);
ctr_status launch_dot(const float* a, const float* b, long long n, double* partial, size_t cap,
                      double* out, cudaStream_t st);
ctr_status launch_l2(const float* a, const float* b, long long n, double* partial, size_t cap,
                     double* out, cudaStream_t st);
ctr_status launch_tv(const Geometry& g, const void* vol, ctr_dtype dt, double* partial, size_t cap,
                     double* out, cudaStream_t st);
// gamma_dev (optional): read the FISTA factor (t_prev-1)/t_k from device
// memory instead of the argument, so a captured graph can be replayed.
ctr_status launch_fgp(Geometry& g, void* vol, ctr_dtype dt, float lambda, int iters,
                      void* fista_y, void* fista_xprev, float fista_gamma, cudaStream_t st,
                      const float* gamma_dev = nullptr);
ctr_status launch_momentum(const Geometry& g, void* y, void* xprev, const void* x, ctr_dtype dt,
                           float gam, cudaStream_t st, const float* gamma_dev = nullptr);
// Refinement solver, before its SART pass (fgp.cu): the correction volume d
// (tiled, ddt storage: dt or FP32) = d0, the ddt rounding of
// (1+g)(xk - x~k) - g(xm - x~m) with x~ the round-to-nearest dt copies (zero
// for FP32 copies).
ctr_status launch_refine_start(Geometry& g, const float* xk, const float* xm, void* d_tiled, ctr_dtype ddt,
                               ctr_dtype dt, const float* gdev, cudaStream_t st);
// Refinement solver, after its SART pass (fgp.cu): xm = (1+g) xk - g xm + (d - d0)
// (d tiled, ddt storage), then with lam > 0 and iters >= 0 the FGP-TV prox of
// that FP32 volume (duals in dt storage), and x* (the prox, or the sum when
// lam == 0) rotated in: xm = xk, xk = x*, xt = the dt copy of x* (tiled).
ctr_status launch_refine_update(Geometry& g, float* xk, float* xm, const void* d_tiled, ctr_dtype ddt, void* xt_tiled,
                                ctr_dtype dt, float lam, int iters, const float* gdev, cudaStream_t st);
// *p = v on the device (a per-iteration scalar that graphs read)
ctr_status launch_set_scalar(float* p, float v, cudaStream_t st);

// One scan of the batch's persistent SART pass (bp.cu): view after view, the
// blocks of its forward projection (fp_gx x fp_gy blocks of 32 x 4 rays),
// then the blocks of its walk (bp_gx x bp_gy x bp_gz blocks of 32 x 4 voxel
// columns, z runs of zl).  CTAs [c0, c0 + nc) take this scan's blocks first
// (its home CTAs, a share proportional to its work) and any other scan's
// when it has none to give.
struct BatchScan {
    DevGeom g;
    const void* fp_vol;          // the volume the projection reads (tiled)
    const void* fp_vol2;         // SART_OBJ: the objective's volume; SART_REFINE: the correction d
    void* bp_vol;                // the volume the update writes (tiled)
    const void* b;               // measured sinogram
    int b_dt;
    float2* rays;                // the scan's ray records (one view)
    double* partial;             // SART_OBJ, SART_REFINE: objective partials, [view][row][u/32]
    float* ax;                   // SART_REFINE
    const float* gdev;           // SART_REFINE
    const uint32_t* pass_seed;   // stochastic rounding (device)
    float beta;
    int nviews;
    int c0, nc;
    int fp_gx, fp_gy;
    int bp_gx, bp_gy, bp_gz, zl;
};
// The persistent pass's work counters of one scan: claim = (phase << 32) |
// the next block of the phase to hand out, done = the phase's blocks
// finished; phase 2j is view j's forward projection, 2j + 1 its walk.
struct BatchFlow {
    unsigned long long claim;
    unsigned done;
    unsigned pad;
};
// bytes of the persistent pass's zeroed state: one BatchFlow per scan and
// the count of finished scans
inline size_t batch_flow_bytes(int nscans) { return sizeof(BatchFlow) * (size_t)nscans + 16; }
constexpr unsigned ERR_BARRIER = 2u;   // a persistent pass's block found no work for too long
// Blocks per SM the persistent pass runs at (its occupancy), or 0.
int batch_pass_blocks_per_sm(ctr_dtype vdt, int kind, bool stoch, size_t smem);
// The persistent pass over every scan: one launch of nblocks CTAs.  flow:
// batch_flow_bytes(nscans) zeroed bytes; err: the device error word
// (ERR_BARRIER when a block idles past its bound).
ctr_status launch_batch_pass(const BatchScan* d_scans, int nscans, int nblocks, ctr_dtype vdt, int kind, bool stoch,
                             void* flow, unsigned* err, size_t smem, cudaStream_t st);
// shared memory of the persistent pass for one scan's geometry
size_t batch_pass_smem(const DevGeom& g);
// the walk's z run for a geometry (launch shape 1, shortened for small volumes)
int walk_z_run(const DevGeom& g);

// The FP64 reference solver (f64.cu): the solver's iteration with every step
// in FP64.  obj_out (host, may be NULL): [TV, fidelity, objective] per
// iteration, evaluated when params.objective is set (NaN otherwise).
struct F64Solver;
ctr_status f64_create(Geometry* g, const ctr_solver_params& p, F64Solver** out);
void f64_destroy(F64Solver* s);
ctr_status f64_set_volume(F64Solver* s, const double* vol, cudaStream_t st);
ctr_status f64_iterate(F64Solver* s, const void* sino, ctr_dtype sdt, int n, double* obj_out, cudaStream_t st);
ctr_status f64_get_volume(F64Solver* s, void* dst, bool as_f32, cudaStream_t st);
int f64_iteration(const F64Solver* s);
ctr_status launch_convert(const void* src, ctr_dtype sdt, void* dst, ctr_dtype ddt, long long n,
                          cudaStream_t st);
ctr_status launch_fdk(Geometry& g, const float* sino, float* vol, cudaStream_t st);
// exchange x and y of every z slice in place (nx == ny)
ctr_status launch_swap_xy(const Geometry& g, float* vol, cudaStream_t st);
// the backprojection stage: vol += views [view0, view0+nview) of the filtered sinogram (fsino[0] = view0)
ctr_status launch_fdk_bp(const Geometry& g, const float* fsino, int view0, int nview, float* vol, cudaStream_t st);
ctr_status launch_phantom(const Geometry& g, const double* dparams, int n, float* vol,
                          cudaStream_t st);

}  // namespace ctr
