/*
 * ctrecon.h -- C ABI of the B200 cone-beam CT reconstruction engine.
 *
 * One process, one GPU.  Every entry point returns a ctr_status (0 = OK);
 * ctr_last_error_string() gives the calling thread's last message.  Nothing
 * in the library calls exit() or assert().
 *
 * Units: any consistent length unit (the reference uses metres, the scan
 * descriptions used by the tests use millimetres).
 *
 * Layouts are the reference's:
 *   volume    vol[k*nx*ny + j*nx + i]         (k = z slice, j = y row, i = x)
 *   view      view[row*nu + col]              (row = detector z, col = detector u)
 *   sinogram  views stacked: sino[view*nu*nv + row*nu + col]
 *
 * Native API: device pointers, an explicit CUDA stream (cudaStream_t passed
 * as void*; NULL = the legacy default stream), asynchronous unless stated.
 * Reference-compatible API (bottom of this file): the reference's host
 * function names and signatures, host pointers, synchronous.
 *
 * Reference interface citations use CBCT/CBCT_1024V_1024P_multiGPU_v6.3_20170823/
 * (abbreviated V63/).
 */
#ifndef CTRECON_H
#define CTRECON_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CTRECON_ABI_VERSION 3

typedef enum ctr_status {
    CTR_OK = 0,
    CTR_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad size, bad dtype, bad view range      */
    CTR_ERR_BAD_GEOMETRY = 2,     /* geometry description rejected                         */
    CTR_ERR_OUT_OF_MEMORY = 3,    /* a device or host allocation failed                     */
    CTR_ERR_CUDA = 4,             /* a CUDA runtime call failed (message has the CUDA text)  */
    CTR_ERR_TRAVERSAL_BOUND = 5,  /* a ray took more than nx+ny+nz+3 Siddon steps            */
    CTR_ERR_TIMEOUT = 6,          /* a device-side wait gave up                              */
    CTR_ERR_UNSUPPORTED = 7,      /* combination not implemented                             */
    CTR_ERR_NO_DEVICE = 8,        /* no CUDA device, or not an sm_100 device                 */
    CTR_ERR_IO = 9                /* file could not be read or written                       */
} ctr_status;

/* storage type of a volume or sinogram buffer; arithmetic is always FP32
 * (FP64 for the norm reductions).  CTR_F64 is accepted only as the volume
 * type of ctr_solver_create: the FP64 reference solver. */
typedef enum ctr_dtype { CTR_F32 = 0, CTR_BF16 = 1, CTR_F16 = 2, CTR_F64 = 3 } ctr_dtype;

/* Scan geometry: the reference's compile-time constants (V63/main_recon.cu:54-111)
 * as a run-time description.  Circular orbit; source at (dso, offset, 0) and
 * the detector plane at x = dod (< 0), both rotated by the view angle. */
typedef struct ctr_geometry_desc {
    int   nx, ny, nz;          /* M, N, ZETA: voxels                                   */
    float vx, vy, vz;          /* voxel pitch (volumn_x/y/z); vy, vz <= 0 mean = vx     */
    int   nu, nv;              /* R (detector columns), Z_prj (detector rows)           */
    float du, dv;              /* detector pitch (Detector_pixel_x); dv <= 0 means = du */
    float dso;                 /* DSO: source to isocentre                              */
    float dod;                 /* DOD: detector plane position (negative)               */
    float offset;              /* Offset: half-detector shift (source y and detector u) */
    int   m_offset;            /* M_Offset: volume x shift in voxels                    */
    int   n_views;             /* Nviews                                                */
    float us_rate;             /* degrees between views                                 */
    float initial_angle;       /* degrees                                               */
    float shift_angle;         /* degrees                                               */
    unsigned flags;            /* CTR_GEOM_* below                                      */
    int   n_sources;           /* CTR_GEOM_TBCT: N_source (>= 1); ignored otherwise     */
} ctr_geometry_desc;

/* Compute the ray-box entry/exit parameters and the first plane indices in
 * FP64 (the traversal itself stays FP32). */
#define CTR_GEOM_ENTRY_F64 0x1u
/* Scanner geometry, the reference's CT_style (V63/main_recon.cu:29): cone
 * beam by default; CTR_GEOM_FAN_SLICES (CT_style 1): a fan beam per detector
 * row, the source at the row's height; CTR_GEOM_PARALLEL (CT_style 2): a
 * parallel beam, every ray perpendicular to the detector.  In both the rays
 * are parallel to the xy plane, and the reference sets vz to the detector
 * pitch.  FDK supports the cone beam only. */
#define CTR_GEOM_FAN_SLICES 0x2u
#define CTR_GEOM_PARALLEL 0x4u
/* Tetrahedron-beam CT (TBCT/TBCT_1024V_1024P_v4.2_20171012, abbreviated
 * T42/): n_sources sources stacked along z on the orbit, placed as the
 * reference places them (T42/main_recon.cu:95-108: the first source sees the
 * volume's bottom face from the detector's bottom row, the last its top face
 * from the top row), each with its own band of nv detector rows.  A view is
 * n_sources bands of nv rows, view[(src*nv + row)*nu + col]
 * (T42/voxel/kernel_IterativeRecon_TBCT_voxel.cu:27): every "row" count of
 * this API is n_sources*nv.  The projector is T42's (its loop test
 * alpha_max - alpha_c > 1e-6f and k range); the SART update is T42's
 * backprojection + update (a voxel's rays summed per source, sources whose
 * band cannot see the voxel skipped, update where the summed length exceeds
 * vx*1e-3) with the projector's chords.  Requires vz = vx and dv = du (the
 * reference's single pitches).  Not with CTR_GEOM_FAN_SLICES/PARALLEL, FDK or
 * CTR_BP_FOV_MASK (V63's command 0; T42's backprojector has no command
 * argument). */
#define CTR_GEOM_TBCT 0x8u
/* Fused ray sums: the solver's, the SART calls' and ctr_forward's
 * projections accumulate (alpha step) x (voxel value) with fused
 * multiply-adds and apply the chord factor |X2 - X1| once per ray (the chord
 * length is that factor times the alpha span), three instructions fewer
 * per Siddon step.  The traversal -- alphas, plane indices, the voxels each
 * ray visits -- is the same code; the sums round differently from the
 * reference's step-by-step sequence, within 1e-5 relative.  Traces, dot
 * tests and slab partial sums keep the reference's sequence. */
#define CTR_GEOM_FAST_SUMS 0x10u

typedef struct ctr_geometry ctr_geometry;

/* Validate the description, derive the reference's float constants, and
 * upload the per-view and per-plane tables to the current device.
 * Replaces the compile-time globals of V63/main_recon.cu:60-111. */
ctr_status ctr_geometry_create(const ctr_geometry_desc* desc, ctr_geometry** out);
ctr_status ctr_geometry_destroy(ctr_geometry* geom);
/* Per-view sin/cos of the FP frame angle -(j*us_rate+initial+shift)*pi/180
 * (V63/host_IterativeRecon_CBCT.c:34-41), as the kernels use them. */
ctr_status ctr_geometry_view_trig(const ctr_geometry* geom, int view, float* sin_out, float* cos_out);

/* Launch shapes of the SART projectors.  fp_shape 0..6: (rows of 32 rays per
 * block, plane coordinates, blocks per SM the registers are capped for) =
 * (2, table, -) (4, table, -) (8, table, -) (4, table, 16) (4, table, 12)
 * (4, table read one plane ahead, -) (4, computed, -).  bp_shape -1: the fixed-shape backprojector (8 voxels of a
 * column per thread); 0..5: the column walk with (voxel rows per block, z
 * run, blocks per SM the registers are capped for, detector rows loaded
 * together) = (4,8,8,1) (4,32,8,1) (4,32,8,2) (8,32,4,1) (4,128,8,1)
 * (4,32,10,1).  Results never depend on
 * the shape.  Defaults: fp_shape 1, bp_shape 1.  Not thread-safe against
 * launches on the same geometry. */
ctr_status ctr_geometry_set_shapes(ctr_geometry* geom, int fp_shape, int bp_shape);
ctr_status ctr_geometry_get_shapes(const ctr_geometry* geom, int* fp_shape, int* bp_shape);
/* Time every shape on n_views views spread over the scan (SART forward
 * projection, then SART backprojection into a scratch volume of vol_dtype in
 * the tiled layout the solver projects) and keep the fastest.  fp_ms[7] and
 * bp_ms[7] (may be NULL) receive the mean milliseconds per view of each
 * shape; bp_ms[0] is bp_shape -1 on the linear layout (reported, not chosen).  Allocates a
 * scratch volume and one sinogram view; synchronises the stream. */
ctr_status ctr_geometry_autotune(ctr_geometry* geom, ctr_dtype vol_dtype, int n_views, float* fp_ms, float* bp_ms,
                                 void* stream);

/* ---------------------------------------------------------------- projectors */

/* sino[w] = A_(view_begin+w) vol for w < view_count (Siddon ray sums, command 0
 * of V63/kernel_IterativeRecon_universal.cu:7-567).  Replaces the per-view
 * launches of Forward_3D_ray_driven_siddon (V63/host_IterativeRecon_CBCT.c:70-128). */
ctr_status ctr_forward(const ctr_geometry* geom, const void* vol, ctr_dtype vol_dtype,
                       void* sino, ctr_dtype sino_dtype, int view_begin, int view_count,
                       void* stream);

/* Matched adjoint: vol = sum_w A_(view_begin+w)^T sino[w] (FP32 sino), with the
 * forward projector's own Siddon chord lengths (gather form, no atomics).
 * CTR_BP_ACCUMULATE adds into vol instead of overwriting; CTR_BP_FOV_MASK skips
 * voxels outside the reconstruction cylinder and keeps the reference's
 * thresholds, i.e. command 0 of backprj_ray_driven_3d_kernel
 * (V63/kernel_IterativeRecon_universal.cu:571-810) as used by
 * CheckMatchedJointOperator (V63/host_IterativeRecon_CBCT.c:131-204). */
#define CTR_BP_ACCUMULATE 0x1u
#define CTR_BP_FOV_MASK 0x2u
ctr_status ctr_backproject(const ctr_geometry* geom, const float* sino, int view_begin,
                           int view_count, void* vol, ctr_dtype vol_dtype, unsigned flags,
                           void* stream);

/* One SART pass over all views in order: per view, FP command 1 (correction
 * (b - Af)/len) then BP command 1 (f += beta * sum(w c)/sum(w) inside the FOV
 * cylinder).  Replaces Reconstruction_3D_ray_driven_CBCT
 * (V63/host_IterativeRecon_CBCT.c:1-67) on device buffers.
 * CTR_SART_STOCHASTIC_ROUND rounds BF16/F16 voxel updates stochastically.
 * CTR_SART_TILED runs the views on an 8x8-tiled copy of the volume (a
 * geometry workspace, copied in before and out after): the same result,
 * fewer cache lines per projector load.  The solver always does this. */
#define CTR_SART_STOCHASTIC_ROUND 0x1u
#define CTR_SART_TILED 0x2u
/* CTR_SART_REFERENCE_BP: the backprojection with the reference kernel's own
 * arithmetic (backprj_ray_driven_3d_kernel command 1,
 * V63/kernel_IterativeRecon_universal.cu:571-810: the bounding rectangle of
 * the voxel's corner projections, the slab alphas by division, the pixels
 * row by row, "f += 0" where the summed length is below vx*1e-6), so that a
 * FP32 SART pass equals the reference's bit for bit (CT_style 0, 1, 2; for
 * CTR_GEOM_TBCT the tetrahedron-beam program's backprojection and update,
 * T42/voxel/kernel_IterativeRecon_TBCT_voxel.cu:546-775, its sources added in
 * ascending order).  Default (flag clear): the gather backprojector with
 * the forward projector's own chords, the exact transpose of the projector,
 * which differs from the reference's alphas in rounding (and keeps the rays
 * lying on a voxel plane that the reference's 0/0 drops). */
#define CTR_SART_REFERENCE_BP 0x4u
ctr_status ctr_sart_pass(const ctr_geometry* geom, void* vol, ctr_dtype vol_dtype,
                         const void* sino, ctr_dtype sino_dtype, float beta, unsigned flags,
                         uint32_t seed, void* stream);

/* The SART pass restricted to views [view_begin, view_begin+view_count), in
 * order.  When fp_ms / bp_ms are non-NULL the library records CUDA events
 * around every forward and backprojection launch on the stream, synchronises,
 * and returns the summed kernel times in milliseconds (profiling hook). */
ctr_status ctr_sart_views(const ctr_geometry* geom, void* vol, ctr_dtype vol_dtype, const void* sino,
                          ctr_dtype sino_dtype, float beta, unsigned flags, uint32_t seed,
                          int view_begin, int view_count, float* fp_ms, float* bp_ms, void* stream);

/* ctr_sart_views without any device allocation, for callers that cannot
 * allocate while they reconstruct: a host whose memory pool has reserved the
 * GPU up front, or a real-time loop that must not stall on cudaMalloc/cudaFree.
 * No counterpart in the reference (its host functions cudaMalloc and cudaFree
 * on every call).  The ray records live in a fixed 8 MiB device array inside
 * the library, so the detector may have at most 1,048,576 pixels (larger ones
 * are rejected with CTR_ERR_INVALID_ARGUMENT).  The geometry's device must be
 * current.  The first call on a device looks the array up (no allocation),
 * and so does the first call in a new context of that device (after
 * cudaDeviceReset, or with another context current); make those calls before
 * any stream capture.  CTR_SART_TILED is refused (its tiled copy would be a
 * workspace); the other flags act as in ctr_sart_views.  All calls share the
 * array: calls that overlap on the GPU (other streams, other threads) race. */
ctr_status ctr_sart_views_noalloc(const ctr_geometry* geom, void* vol, ctr_dtype vol_dtype, const void* sino,
                                  ctr_dtype sino_dtype, float beta, unsigned flags, uint32_t seed,
                                  int view_begin, int view_count, void* stream);

/* ------------------------------------------- z-slab SART of the multi-GPU build */

/* The reference's default build (V63/main_recon.cu:23, Number_of_Devices 4)
 * splits the volume into D z-slabs, one per device, and runs each SART view
 * as (V63/host_IterativeRecon_CBCT_multiGPU.c:1-161, kernels
 * V63/kernel_IterativeRecon_universal_multiGPU.cu):
 *   1. every slab projects its own voxels: partial ray sums (Sum(len*f),
 *      Sum(len)), no threshold (forward_ray_driven_3d_kernel_correction_
 *      separate, :591-1149), with the slab's own z planes
 *      boundary_voxel_z + volumn_z*ZETA/D*s + n*volumn_z and ZETA/D slices;
 *   2. the parts are added in slab order from zero and divided:
 *      c = (b - Sum(len*f))/Sum(len), 0 below volumn_z*1e-6 (:1-19);
 *   3. every slab backprojects c into its voxels (:1156-1402).
 * The rounding differs from the one-device pass (a ray's sum is the sum of
 * its slabs' sums; the slab planes are computed from the slab's boundary), so
 * these calls reproduce the D-device build, not the one-device one.  ZETA and
 * Z_prj must split evenly into D (V63/main_recon.cu:24).  The tetrahedron-beam
 * program's default build is its multi-GPU one too (T42/main_recon.cu:17,
 * T42/voxel/kernel_IterativeRecon_TBCT_voxel_multiGPU.cu): the same sequence with its sources, its
 * projectors testing alpha_max - alpha_c > 1e-16f (its one-device one: 1e-6f),
 * its combination zeroing below volumn_z*1e-3f, and its slab backprojector's
 * voxel centres; CTR_GEOM_TBCT geometries get those.
 *
 * Slab s of D of a scan: a geometry of nz/D slices.  Volumes passed with it
 * are that slab's nx*ny*(nz/D) voxels; its z planes, voxel centres and (for
 * CTR_GEOM_FAN_SLICES / CTR_GEOM_PARALLEL) traced detector rows are the
 * multi-GPU build's.  s = -1: the whole volume as the D-device build's
 * row-split projector (its Forward_3D_ray_driven_siddon) traverses it -- for
 * the tetrahedron beam V63's traversal rules, otherwise the one-device
 * projector.  Not for the solver or FDK. */
ctr_status ctr_geometry_create_slab(const ctr_geometry_desc* desc, int n_slabs, int slab, ctr_geometry** out);
/* D (1 for a whole-volume geometry, s = -1 included), s, and the slab's first slice in the volume. */
ctr_status ctr_geometry_slab(const ctr_geometry* geom, int* n_slabs, int* slab, int* first_slice);

/* Per-view calls of one slab, for a host that holds one slab per GPU and
 * exchanges the parts itself (e.g. an all-gather over NCCL):
 * ctr_forward_partial: part[p] = (Sum(len*f), Sum(len)) of ray p (2 floats per
 *   ray, rows*nu rays) for view `view` of the slab volume;
 * ctr_combine_partials: parts = n_parts such arrays back to back, in slab
 *   order; writes the ray records rays[p] = (c, d12) (2 floats per ray) from
 *   the view's measured data b_view (rows*nu values of b_dtype); any geometry
 *   of the scan;
 * ctr_sart_update: the slab's SART backprojection of those records,
 *   vol += beta*Sum(w c)/Sum(w) (CTR_SART_REFERENCE_BP: the multi-GPU
 *   backprojector's arithmetic, bit-exact with it; clear: the gather update
 *   with the slab projector's own chords).
 * CTR_VOLUME_TILED: vol is stored in the 8x8-tiled layout (ctr_volume_tiling)
 * instead of [z][y][x]; the result is the same. */
#define CTR_VOLUME_TILED 0x8u
ctr_status ctr_forward_partial(const ctr_geometry* slab_geom, const void* vol, ctr_dtype vol_dtype, int view,
                               float* part, unsigned flags, void* stream);
ctr_status ctr_combine_partials(const ctr_geometry* geom, const float* parts, int n_parts, int view,
                                const void* b_view, ctr_dtype b_dtype, float* rays, void* stream);
ctr_status ctr_sart_update(const ctr_geometry* slab_geom, void* vol, ctr_dtype vol_dtype, const float* rays,
                           int view, float beta, unsigned flags, uint32_t seed, void* stream);
/* The D-slab SART over views [view_begin, view_begin+view_count) on one GPU:
 * geom is the whole-volume geometry, vol the whole volume ([z][y][x], the D
 * slabs back to back); flags as ctr_sart_pass.  Its slab geometries are kept
 * with geom. */
ctr_status ctr_sart_pass_slabs(const ctr_geometry* geom, int n_slabs, void* vol, ctr_dtype vol_dtype,
                               const void* sino, ctr_dtype sino_dtype, float beta, unsigned flags, uint32_t seed,
                               int view_begin, int view_count, void* stream);
/* Layout conversion between [z][y][x] and the 8x8-tiled layout of the
 * projectors (to_tiled = 1: src linear, dst tiled); dst holds
 * ctr_volume_tiled_count elements when tiled. */
ctr_status ctr_volume_tiling(const ctr_geometry* geom, const void* src, void* dst, ctr_dtype dtype, int to_tiled,
                             void* stream);
ctr_status ctr_volume_tiled_count(const ctr_geometry* geom, int64_t* count);

/* Trace one view: per ray, the number of Siddon segments, an FNV-1a hash of
 * the visited voxel index sequence and the summed chord length.  For parity
 * checks of the traversal (the voxel index set of every ray). */
ctr_status ctr_forward_trace(const ctr_geometry* geom, const float* vol, int view, int* nseg,
                             uint64_t* hash, float* len, void* stream);

/* ----------------------------------------------------- TV prox and FISTA */

/* In-place FGP TV prox: vol = argmin 0.5||x - vol||^2 + lambda TV_iso(x), n_iter
 * Beck-Teboulle FGP steps with dual step 1/(12 lambda).  Replaces
 * FGP_denoise_GPUx7_exact (V63/host_FGP_Denoise_GPUx7.c:1-111, kernels
 * V63/kernel_FGP_Denoise_GPUx7.cu:2-88).  Workspace: 9 volume-sized dual arrays
 * of vol_dtype, allocated on first use and kept with the geometry. */
ctr_status ctr_fgp_tv(const ctr_geometry* geom, void* vol, ctr_dtype vol_dtype, float lambda,
                      int n_iter, void* stream);

/* FISTA outer step (V63/main_recon.cu:372-384):
 *   y = x + (t_prev - 1)/t_k * (x - x_prev);  x_prev = x.
 * y may alias x.  t_k = (1 + sqrt(1 + 4 t_prev^2))/2 is the caller's. */
ctr_status ctr_fista_momentum(const ctr_geometry* geom, void* y, void* x_prev, const void* x,
                              ctr_dtype dtype, float t_prev, float t_k, void* stream);

/* ---------------------------------------------------------------- objective */

/* sum over all views of (A vol - sino)^2 and the isotropic TV of vol, both
 * reduced in FP64.  Synchronises the stream.  Replaces L2_norm_gpu and
 * TV_norm_gpu (V63/host_tool_functions.cu:28-101) after the objective's
 * Forward_3D_ray_driven_siddon (V63/main_recon.cu:401-417). */
ctr_status ctr_objective(const ctr_geometry* geom, const void* vol, ctr_dtype vol_dtype,
                         const void* sino, ctr_dtype sino_dtype, double* fidelity, double* tv,
                         void* stream);
/* TV_norm_gpu (V63/host_tool_functions.cu:61-101): FP64 sum of the per-voxel
 * forward-difference TV terms.  Synchronises the stream. */
ctr_status ctr_tv_norm(const ctr_geometry* geom, const void* vol, ctr_dtype dtype, double* tv,
                       void* stream);
/* L2_norm_gpu (V63/host_tool_functions.cu:28-58) without its in-place side
 * effect: FP64 sum of float (a - b)^2 over n elements.  Synchronises. */
ctr_status ctr_l2_norm(const float* a, const float* b, int64_t n, double* out, void* stream);

/* --------------------------------------------------------------------- FDK */

/* FDK: cosine pre-weight, spatial-domain ramp (the exact kernel of the
 * reference's padded-DFT filter |k|*F_step*0.5 on a 2R grid), then voxel-driven
 * bilinear backprojection in the +theta frame, accumulated into vol (FP32).
 * Replaces Reconstruction_FDK (V63/host_FDK.cpp:4-57; kernels
 * V63/FDK/kernel_FDK.cu:1-62; ramp V63/FDK/FFT_1d_GPU.h:241-287).
 * Frame: the reference's FDK rotates its voxels by +theta
 * (V63/FDK/kernel_FDK.cu:33-34, V63/host_FDK.cpp:37) where the projectors use
 * -theta, so its volume is the projector frame's volume with x and y
 * exchanged: vol[k][j][i] here is voxel (x = j, y = i) of ctr_forward's volume.
 * This call keeps the reference's frame (its output bit for bit);
 * ctr_fdk_projector_frame returns the projector's frame, e.g. to start the
 * iterative solver from FDK.  Workspace: two FP32 sinogram copies, allocated
 * on first use and kept with the geometry. */
ctr_status ctr_fdk(const ctr_geometry* geom, const float* sino, float* vol, void* stream);
/* ctr_fdk with the result in the projectors' frame: vol (projector frame) +=
 * FDK with x and y exchanged, done in place (vol is exchanged, FDK
 * accumulates, vol is exchanged back).  Needs nx == ny, vx == vy, offset 0
 * and m_offset 0, where the exchange maps the volume onto itself. */
ctr_status ctr_fdk_projector_frame(const ctr_geometry* geom, const float* sino, float* vol, void* stream);
/* The backprojection stage of FDK alone: vol += the bilinear voxel-driven
 * backprojection of the already weighted and filtered views
 * [view_begin, view_begin+view_count) (filtered[w] is view view_begin+w,
 * FP32), view by view in order, each view's update rounded as the
 * reference's kernel_FDK_reconstruction (V63/FDK/kernel_FDK.cu:16-62) rounds
 * it, the per-view launch loop of V63/host_FDK.cpp:33-50.  No workspace. */
ctr_status ctr_fdk_backproject(const ctr_geometry* geom, const float* filtered, int view_begin, int view_count,
                               float* vol, void* stream);

/* ------------------------------------------------------------ dot product */

/* <A x, y> and <x, A^T y> over views [view_begin, view_begin+view_count):
 * FP64 inner products; A x sums the projector's Siddon segments of each ray
 * in FP64 and A^T y is the matched adjoint (FP64 accumulation, float result),
 * so the two agree to float rounding of A^T y.  Synchronises.  The matched-
 * adjoint check of CheckMatchedJointOperator (V63/host_IterativeRecon_CBCT.c:131-204). */
ctr_status ctr_dot_test(const ctr_geometry* geom, const float* x, const float* y, int view_begin,
                        int view_count, double* ax_dot_y, double* x_dot_aty, void* stream);

/* ------------------------------------------------------- iterative solver */

/* SART + FISTA + FGP-TV outer loop of V63/main_recon.cu:286-484 (FISTA == 1)
 * on device buffers.  One iteration: x = SART(y); x = FGP(x, beta*lambda_tv);
 * t_k = (1+sqrt(1+4 t^2))/2; y = x + (t-1)/t_k (x - x_prev); x_prev = x; and,
 * when requested, the objective [TV, fidelity, fidelity + 2 lambda_tv TV].
 *
 * refine = 1, mixed-precision iterative refinement (vol_dtype BF16 or F16;
 * allowed with F32): the FISTA state x_k, x_(k-1) stays in FP32 and is
 * touched once per iteration.  The projectors read the round-to-nearest
 * vol_dtype copies x~ of the iterates and accumulate the SART pass into a
 * vol_dtype correction volume d: per view j, c = (b_j - A_j y~_k - A_j d)/len,
 * where A_j y~_k = (1+g) A_j x~_k - g A_j x~_(k-1) (g the FISTA factor
 * (t-1)/t_k), A_j x~_k is summed in the same traversal as A_j d, and
 * A_j x~_(k-1) is kept from the previous pass in an FP32 sinogram.  d starts
 * at d0, the vol_dtype rounding of y_k - y~_k (the copies' own rounding
 * errors, each at most half a vol_dtype ulp), so that y~_k + d is the FP32 y_k to
 * within the rounding of that small difference: the residual is formed in
 * FP32 against the estimate itself, and no per-view update is rounded
 * against the (large) stored estimate, only against d (the iteration's
 * change).  After the pass x_(k+1) = FGP(y_k + (d - d0)) in FP32.  In
 * exact arithmetic this is the same iteration as refine = 0.  The fidelity of
 * the objective is that of the vol_dtype copy of x_k the pass projects, the TV
 * that of the FP32 x_k.  Workspace: two FP32 volumes and one FP32 sinogram.
 * Not with ctr_solver_set_slabs.  refine = 2 keeps d in FP32 (its per-view
 * updates are then not rounded to 16 bits; a 16-bit d's rounding noise is
 * the error floor of refine = 1, about 2e-3 of the maximum with BF16 at
 * 1024^3): the projectors read the 16-bit copy and the FP32 d, the update
 * writes FP32 d, stochastic rounding does not apply to it.
 *
 * vol_dtype CTR_F64: the FP64 reference solver.  The same iteration with every
 * step in FP64 on the device: a Siddon traversal per ray with FP64 alphas,
 * the SART update summing the geometric chord of every (voxel, ray) pair
 * (gather form), FGP-TV, FISTA (t in FP64) and the objective.  It states the
 * error of the FP32 and mixed-precision solvers at full size.  Cone beam
 * only (not CTR_GEOM_FAN_SLICES, CTR_GEOM_PARALLEL or CTR_GEOM_TBCT); the
 * sinogram may be any storage type (widened); set_volume / get_volume take
 * FP64 volumes; sart_flags, refine and use_graph are ignored, and
 * ctr_solver_set_slabs, ctr_solver_save/load and ctr_batch_create refuse it. */
typedef struct ctr_solver_params {
    float beta;            /* SART relaxation, the reference's 2/Lip_con               */
    float lambda_tv;       /* lambda_TV; the FGP weight is beta*lambda_tv (main:162)     */
    int   fgp_iters;       /* Niter_denoise (20)                                         */
    int   fista;           /* 1: FISTA momentum (FISTA == 1); 0: SART + TV only          */
    int   objective;       /* 1: evaluate the objective every iteration                  */
    int   use_graph;       /* 1: capture one iteration as a CUDA graph and replay it     */
    unsigned sart_flags;   /* CTR_SART_*                                                 */
    int   refine;          /* 1: mixed-precision iterative refinement (above); 2: the    */
                           /* same with the correction volume d in FP32                  */
} ctr_solver_params;

typedef struct ctr_solver ctr_solver;

ctr_status ctr_solver_create(const ctr_geometry* geom, ctr_dtype vol_dtype,
                             const ctr_solver_params* params, ctr_solver** out);
ctr_status ctr_solver_destroy(ctr_solver* s);
/* Borrow the measured sinogram (device, n_views*nv*nu of sino_dtype); it must
 * stay valid while the solver iterates. */
ctr_status ctr_solver_set_sinogram(ctr_solver* s, const void* sino, ctr_dtype sino_dtype);
/* Set the estimate (device, vol_dtype; NULL = zeros) and restart FISTA (t = 1). */
ctr_status ctr_solver_set_volume(ctr_solver* s, const void* vol, void* stream);
/* Run n outer iterations.  objective_out (host, may be NULL) receives 3 doubles
 * per iteration: TV, fidelity, objective.  Synchronises the stream. */
ctr_status ctr_solver_iterate(ctr_solver* s, int n, double* objective_out, void* stream);
/* Copy the current estimate x_k (vol_dtype) to dst (device or host). */
ctr_status ctr_solver_get_volume(ctr_solver* s, void* dst, void* stream);
/* The current estimate as FP32 (device or host): the FP32 x_k of a
 * refinement solver, the stored x_k widened otherwise, the FP64 x_k rounded
 * for the FP64 solver.  Synchronises. */
ctr_status ctr_solver_get_volume_f32(ctr_solver* s, float* dst, void* stream);
ctr_status ctr_solver_iteration_count(const ctr_solver* s, int* k);

/* The SART pass of the reference's n_slabs-device build (its z-slab sequence,
 * ctr_sart_pass_slabs) instead of the one-device pass, from the next
 * ctr_solver_iterate on; 1 restores the one-device pass.  With n_slabs > 1
 * every iteration's objective is projected on its own with the one-device
 * projector (the sums the n-device build's row-split projector gives) rather
 * than inside the next pass, and the pass is issued without a CUDA graph.
 * With sart_flags = CTR_SART_REFERENCE_BP and FP32 storage the SART + FISTA +
 * FGP-TV loop and its objectives equal that build's (for CTR_GEOM_TBCT the
 * objective's projector is that build's row-split one).  ZETA and Z_prj must
 * split into n_slabs. */
ctr_status ctr_solver_set_slabs(ctr_solver* s, int n_slabs);
/* Objective history [TV, fidelity, objective] of iterations first..first+count-1
 * (1-based, at most the iterations run).  With objective_out == NULL,
 * ctr_solver_iterate leaves the objective of its last x_k pending and projects
 * it inside the next call's first SART traversal; asking for it here
 * projects it at once.  Rows the solver never evaluated (before a checkpoint
 * load) are NaN.  Synchronises. */
ctr_status ctr_solver_objectives(ctr_solver* s, int first, int count, double* out, void* stream);
/* Exact checkpoint of the FISTA state (x_k, y_k, t_k, k and a geometry hash),
 * raw little-endian, and its restore. */
ctr_status ctr_solver_save(ctr_solver* s, const char* path, void* stream);
ctr_status ctr_solver_load(ctr_solver* s, const char* path, void* stream);

/* ------------------------------------------------------------ batched scans */

/* Many independent scans of uneven sizes iterated together: one CUDA graph
 * launch runs one outer iteration (SART pass, FGP-TV, FISTA, objective) of
 * every scan, the scans as parallel branches.  Each scan needs its own
 * geometry handle (workspaces are per geometry).  Per-iteration scalars (the
 * FISTA factor, the stochastic-rounding seed of the pass) are read from device
 * memory, so every scan's result is bit-identical to ctr_solver_iterate on the
 * same inputs.  No counterpart in the reference, which reconstructs one scan
 * per process. */
typedef struct ctr_batch ctr_batch;
ctr_status ctr_batch_create(const ctr_geometry* const* geoms, int n_scans, ctr_dtype vol_dtype,
                            const ctr_solver_params* params, ctr_batch** out);
ctr_status ctr_batch_destroy(ctr_batch* b);
ctr_status ctr_batch_set_sinogram(ctr_batch* b, int scan, const void* sino, ctr_dtype sino_dtype);
/* zero every estimate and restart FISTA */
ctr_status ctr_batch_reset(ctr_batch* b, void* stream);
/* n iterations of every scan; objective_out (host, may be NULL) receives
 * [scan][iteration][TV, fidelity, objective].  Synchronises. */
ctr_status ctr_batch_iterate(ctr_batch* b, int n, double* objective_out, void* stream);
ctr_status ctr_batch_get_volume(ctr_batch* b, int scan, void* dst, void* stream);
/* ctr_solver_get_volume_f32 of one scan. */
ctr_status ctr_batch_get_volume_f32(ctr_batch* b, int scan, float* dst, void* stream);
/* on = 1: from the next ctr_batch_iterate, the SART views of every scan run
 * in one persistent launch per iteration, as many blocks as the GPU holds at
 * once, scheduled as a data flow: each scan's phases (view j's forward
 * projection, then its update, then view j+1's projection, ...) run in
 * order, the blocks of a phase on any block of the launch; a block takes
 * work from its home scan (the blocks are split among the scans in
 * proportion to their work) and from any other scan when its own has none to
 * give, and the last block of a phase to finish opens the next.  The per-ray
 * and per-voxel code is the single-scan kernels' (launch shape 1), so every
 * scan's result is unchanged.  A block that finds no work for 4 s (nothing
 * legitimate takes that long) stops the pass, and ctr_batch_iterate returns
 * CTR_ERR_TIMEOUT.  Refused (CTR_ERR_UNSUPPORTED) for scans with
 * CTR_SART_REFERENCE_BP, slabs, CTR_GEOM_ENTRY_F64 or CTR_GEOM_FAST_SUMS, or
 * more scans than resident blocks.  on = 0: one kernel per view and scan, the
 * scans as parallel graph branches (the default). */
ctr_status ctr_batch_set_persistent(ctr_batch* b, int on);

/* ------------------------------------------------------------- utilities */

/* Thread-local text of the last failure on this thread ("" if none). */
const char* ctr_last_error_string(void);
/* Convert between storage types on the device (n elements). */
ctr_status ctr_convert(const void* src, ctr_dtype src_dtype, void* dst, ctr_dtype dst_dtype,
                       int64_t n, void* stream);
/* Add seeded ellipsoids to a device volume: params is n x 10 host doubles
 * (cx,cy,cz, ax,ay,az, phi,theta,psi (z-x-z Euler, radians), attenuation). */
ctr_status ctr_phantom_voxelize(const ctr_geometry* geom, const double* params, int n,
                                float* vol, void* stream);

/* ------------------------------------------------------------- file formats */

/* The reference driver's files (V63/main_recon.cu:197-266, 434-477), host only.
 * View files hold one view as raw little-endian float [nv][nu]; volumes are raw
 * float [nz][ny][nx]; the objective file holds 3 doubles per iteration. */
/* "View_%.02f.dat" for view j, with the reference's angle rule (tomosynthesis
 * split at n_views/2, negative angles + 360), V63/main_recon.cu:203-212. */
ctr_status ctr_io_view_filename(char* out, size_t n, int view, float us_rate, float initial_angle, int tomo,
                                int n_views);
/* The reconstruction file names of V63/main_recon.cu:438 (iteration < 0) and
 * :452 (numbered copy); voxel_um is the voxel pitch in micrometres. */
ctr_status ctr_io_recon_filename(char* out, size_t n, const char* object, int nx, int ny, int nz, float voxel_um,
                                 int n_views, float initial_angle, float end_angle, float lambda_tv,
                                 float lambda_l1, float lip, int iteration);
/* object_func_<...>.bin of V63/main_recon.cu:468. */
ctr_status ctr_io_objective_filename(char* out, size_t n, const char* object, int n_views, float initial_angle,
                                     float end_angle, float lambda_tv, float lip);
ctr_status ctr_io_write_raw(const char* path, const void* data, size_t bytes);
ctr_status ctr_io_read_raw(const char* path, void* data, size_t bytes, size_t offset);
/* All views from dir/View_<angle>.dat into h_proj [n_views][nv][nu], skipping
 * row_offset rows at the start of each file (the reference's fseek, :221). */
ctr_status ctr_io_read_views(const char* dir, int nu, int nv, int n_views, float us_rate, float initial_angle,
                             int tomo, int row_offset, float* h_proj);
ctr_status ctr_io_write_views(const char* dir, int nu, int nv, int n_views, float us_rate, float initial_angle,
                              int tomo, const float* h_proj);

/* ------------------------------------------- reference-compatible entry points */

/* The reference's host functions keep their geometry in compile-time globals;
 * these names take it from the default geometry set here.  All take host
 * (pinned or pageable) or device pointers, copy in and out like the reference,
 * and report failures through ctr_last_error_string(). */
ctr_status ctr_set_default_geometry(const ctr_geometry_desc* desc);
/* Number_of_Devices of the reference build being replaced (V63/main_recon.cu:23,
 * T42/main_recon.cu:17; default 1).  With n > 1 Reconstruction_3D_ray_driven_CBCT
 * and CheckMatchedJointOperator compute what the n-device build computes (the
 * z-slab sequence above, on the current GPU); Forward_3D_ray_driven_siddon
 * projects as its row-split projector (V63's is the one-device one; the
 * tetrahedron beam's follows V63's traversal rules). */
ctr_status ctr_set_default_devices(int n);

/* V63/host_IterativeRecon_CBCT.c:70-128: A x for all views into h_proj_data. */
void Forward_3D_ray_driven_siddon(float* h_volume, float* h_proj_data);
/* V63/host_IterativeRecon_CBCT.c:1-67: one SART pass, h_volume updated in place,
 * with the reference backprojector's arithmetic (CTR_SART_REFERENCE_BP), so
 * the result is the reference's bit for bit; for a tetrahedron-beam geometry
 * that of Reconstruction_3D_ray_driven_TBCT
 * (TBCT/TBCT_1024V_1024P_v4.2_20171012/voxel/host_IterativeRecon_TBCT_voxel.c:1-92). */
void Reconstruction_3D_ray_driven_CBCT(float* h_volume, float* h_proj_data, float beta_temp);
/* V63/host_IterativeRecon_CBCT.c:131-204: prints <Ax,Ax> and <x,A^T A x> for view 0. */
void CheckMatchedJointOperator(float* h_volume);
/* V63/host_FGP_Denoise_GPUx7.c:1-111: TV prox of h_f_noise in place. */
void FGP_denoise_GPUx7_exact(float* h_f_noise, float lambda, int Niter_denoise);
/* V63/host_FDK.cpp:4-57: FDK of h_proj_data accumulated into h_volume. */
void Reconstruction_FDK(float* h_volume, float* h_proj_data);
/* V63/host_tool_functions.cu:28-58: sum over all views of (a-b)^2; unlike the
 * reference, d_a is not overwritten. */
double L2_norm_gpu(float* d_a, float* d_b);
/* V63/host_tool_functions.cu:61-101 */
double TV_norm_gpu(float* d_volume);

#ifdef __cplusplus
}
#endif
#endif /* CTRECON_H */
