/*
 * ct_oracle.h -- CPU restatement of the reference CBCT reconstruction path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (gpu_b200/, include/)
 * links, loads or calls this code.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg use it, and only as the checker.
 *
 * Each function restates one reference function or kernel of
 * CBCT/CBCT_1024V_1024P_multiGPU_v6.3_20170823 (abbreviated V63/ below) as
 * scalar C, with the same float operation order, so that it can be pinned
 * bit-for-bit against the reference's own kernel sources compiled for the
 * CPU (oracle/ref_harness.cpp -> oracle/_ref/libctref.so).
 *
 * Layouts (the reference's):
 *   volume    f[k*M*N + j*M + i]      (V63/kernel_IterativeRecon_universal.cu:10)
 *   view      p[row*R + col]          (V63/kernel_IterativeRecon_universal.cu:17)
 *   sinogram  views stacked: p[view*R*Z_prj + row*R + col]
 *
 * ct_style 3 restates the tetrahedron-beam program TBCT/TBCT_1024V_1024P_
 * v4.2_20171012 (abbreviated T42/): N_source sources stacked along z share
 * the orbit, each with its own band of Z_prj detector rows, so one view is
 * p[src*R*Z_prj + row*R + col] (T42/voxel/kernel_IterativeRecon_TBCT_voxel.cu:27)
 * and every function below that loops over "rows" takes the N_source*Z_prj
 * rows of og_geom.rows, row r belonging to source r / Z_prj.
 */
#ifndef CT_ORACLE_H
#define CT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Scan description: the reference's compile-time constants
 * (V63/main_recon.cu:54-111) as run-time fields. */
typedef struct og_desc {
    int   nx, ny, nz;        /* M, N, ZETA                                  */
    int   nu, nv;            /* R (detector columns), Z_prj (rows)          */
    int   nviews;            /* Nviews                                      */
    float vx, vy, vz;        /* volumn_x, volumn_y, volumn_z                */
    float du, dv;            /* detector pitch (Detector_pixel_x, both axes)*/
    float dso, dod;          /* DSO, DOD (detector plane at x = DOD < 0)    */
    float offset;            /* Offset (half-detector shift)                */
    int   m_offset;          /* M_Offset                                    */
    float us_rate;           /* degrees per view                            */
    float initial_angle;     /* degrees                                     */
    float shift_angle;       /* degrees                                     */
    int   ct_style;          /* CT_style: 0 cone beam, 1 multi-slice fan     */
                             /* beam, 2 parallel beam (V63/main_recon.cu:29) */
                             /* 3: tetrahedron beam (TBCT v4.2, below)       */
    int   n_sources;         /* ct_style 3: N_source, sources along z, each  */
                             /* with its own band of nv detector rows        */
    int   n_slabs;           /* > 1: the z-slab split of the multi-GPU SART  */
                             /* (V63 Number_of_Devices): this description is */
    int   slab;              /* slab `slab` (subVolIdx) of n_slabs, nz/n_slabs*/
                             /* slices of the nz-slice volume; 0/1: no split; */
                             /* -1: the whole volume as the n_slabs-device    */
                             /* build's row-split projector traverses it      */
} og_desc;

/* Derived constants, computed with the reference's float/double steps. */
typedef struct og_geom {
    og_desc d;
    float inv_vx, inv_vy, inv_vz;   /* inv_volumn_*  = (float)(1.0/v)      */
    float bx, by, bz;               /* boundary_voxel_*                     */
    float ymin, zmin;               /* Detector_Ymin, Detector_Zmin         */
    float srcx, srcy, srcz;         /* Source_x/y/z                         */
    float zmax;                     /* Detector_Zmax (T42/main_recon.cu:91)   */
    float zsrc0, zsrc_dz;           /* Source_z_min, Source_interval (:95-108) */
    int   rows;                     /* detector rows of one view: nv, or     */
                                    /* nv * n_sources for ct_style 3          */
    /* Slab geometry (n_slabs > 1): d.nz is the slab's ZETA/D slices, bz its
     * BOUNDARY_VOXEL_Z = boundary_voxel_z + volumn_z*ZETA/D*subVolIdx
     * (V63/kernel_IterativeRecon_universal_multiGPU.cu:636-637) and k0 the
     * whole volume's index of its first slice; otherwise k0 = 0, bz_ref = bz. */
    int   k0;
    float bz_ref;                   /* boundary_voxel_z of the whole volume  */
    int   zpar_kr;                  /* the z-parallel k range of :172-178     */
                                    /* applies (not T42's, not a slab's)      */
    int   row_lo, row_hi;           /* CT_style 1/2 slab: rows of its band    */
                                    /* (multiGPU.cu:663); else 0, rows        */
    float loop_eps;                 /* Siddon loop test alpha_max - alpha_c > */
                                    /* loop_eps: 1e-6f in T42's one-device     */
                                    /* projector, 1e-16f everywhere else        */
} og_geom;

int  og_init(og_geom* g, const og_desc* d);
/* Source (X2) of the ray through detector pixel (u, v) at a view, per
 * CT_style (V63/kernel_IterativeRecon_universal.cu:21-39): one source (0);
 * the source at the row's height (1); a source per pixel, opposite it (2);
 * source v / Z_prj of the stack (3, T42/...TBCT_voxel.cu:30-33). */
void og_source(const og_geom* g, float s, float c, int u, int v, float* x2x, float* x2y, float* x2z);
/* Per-view angle.  fdk=0: SART/FP frame theta' = -(j*us+init+shift)*pi/180
 * (V63/host_IterativeRecon_CBCT.c:34-41); fdk=1: +theta (V63/host_FDK.cpp:35-40). */
void og_view_trig(const og_geom* g, int view, int fdk, float* s, float* c);
/* z of the centre of detector row v (V63/...universal.cu:40; row v % Z_prj
 * of its source's band for ct_style 3, T42/...TBCT_voxel.cu:40). */
float og_row_z(const og_geom* g, int v);

/* ---- Siddon forward projector (V63/kernel_IterativeRecon_universal.cu:7-567) ---- */
/* One ray.  Returns the ray sum; *len gets the summed chord length.  When
 * nseg/hash are non-NULL they receive the segment count and an FNV-1a hash of
 * the visited voxel index sequence.  entry64=1 computes the entry/exit alphas
 * and the first plane indices in double (the engine's optional FP64 entry). */
float og_fp_ray(const og_geom* g, const float* vol, float s, float c, int u, int v,
                int entry64, float* len, int* nseg, uint64_t* hash);
/* The alpha interval [lo, hi] the traversal of ray (u, v) covers (lo > hi when
 * it visits no voxel): the support of the engine's matched adjoint chords. */
void og_fp_window(const og_geom* g, float s, float c, int u, int v, int entry64, float* lo, float* hi);
/* ... and the voxel it starts in plus its parallel axes (start[0..2], start[3] bits x=1,y=2,z=4). */
void og_fp_start(const og_geom* g, float s, float c, int u, int v, int entry64, float* lo, float* hi, int* start);
/* command 0: out = A f ; command 1: out = (b - A f)/len (SART correction). */
void og_forward_view(const og_geom* g, const float* vol, float s, float c, int command,
                     const float* b, float* out, int entry64);
void og_forward_trace(const og_geom* g, const float* vol, float s, float c, int entry64,
                      int* nseg, uint64_t* hash, float* len);
/* The same traversal in double throughout: the FP64 oracle. */
void og_forward_view_f64(const og_geom* g, const double* vol, double s, double c, double* out);

/* ---- reference voxel-driven BP (V63/kernel_IterativeRecon_universal.cu:571-810) ----
 * ct_style 3: the TBCT backprojection and update (T42/voxel/kernel_
 * IterativeRecon_TBCT_voxel.cu:546-775), which has no command 0: the view's
 * SART update whatever command is, its per-source sums added in ascending
 * source order (one of the orders the reference's atomicAdd can take). */
void og_backproject_ref(const og_geom* g, float* vol, const float* corr, float beta,
                        float s, float c, int command);

/* ---- exact adjoint of og_fp_ray, by scattering each ray's segments ----
 * acc[idx] += seg * y[ray]; lacc (optional) += seg, for segments whose length
 * is above the reference BP's threshold vx*1e-6 when thresh=1. */
void og_adjoint_view(const og_geom* g, const float* y, float s, float c, int thresh,
                     double* acc, double* lacc);
void og_adjoint_view_f64(const og_geom* g, const double* y, double s, double c, double* acc);
/* FOV cylinder test of the reference BP (V63/...universal.cu:626-628): 1 = masked. */
int  og_fov_masked(const og_geom* g, int i, int j);

/* ---- SART pass drivers (V63/host_IterativeRecon_CBCT.c:1-67) ---- */
/* reference semantics: FP command 1, then the reference BP command 1, per view */
void og_sart_pass_ref(const og_geom* g, float* vol, const float* sino, float beta);
/* engine semantics: the BP uses the FP's own chord lengths (matched adjoint) */
void og_sart_pass_matched(const og_geom* g, float* vol, const float* sino, float beta);
void og_sart_pass_f64(const og_geom* g, double* vol, const double* sino, double beta);
/* the engine's gather SART update: reference BP semantics (candidate
 * rectangle, FOV mask, thresholds) with every alpha evaluated the Siddon
 * projector's way, float sums in the engine's pair order (detector row by
 * row, the columns of each row ascending).  The candidate
 * rows are a superset of the rows with a positive chord (the cone beam's
 * rectangle, the fan-slice / parallel beams' rows of the cell's z span, each
 * widened by a row), so they do not change the sums. */
void og_backproject_gather(const og_geom* g, float* vol, const float* corr, float beta, float s, float c);
void og_sart_pass_gather(const og_geom* g, float* vol, const float* sino, float beta);

/* ---- z-slab SART of the multi-GPU build (V63/host_IterativeRecon_CBCT_multiGPU.c:1-161,
 *      kernels V63/kernel_IterativeRecon_universal_multiGPU.cu:1-19,591-1402) ----
 * On a slab geometry: the slab's partial ray sums, Sum(len*f) -> wsum and
 * Sum(len) -> lsum, with no threshold (forward_ray_driven_3d_kernel_
 * correction_separate); og_backproject_ref on a slab geometry is
 * backprj_ray_driven_3d_kernel_multiGPU (its voxel centres, no "+= 0"). */
void og_forward_partial(const og_geom* g, const float* vol, float s, float c, float* wsum, float* lsum);
/* The host's combination (multiGPU.c:82-95): both sums start from 0 and add
 * the parts in slab order (kernel_add_proj), then kernel_divide_proj:
 * corr = 0 where Sum(len) < volumn_z*1e-6f, else (b - Sum(len*f))*1.0f/Sum(len).
 * wsum, lsum: [n_parts][rows*R]. */
void og_combine_partials(const og_geom* g, int n_parts, const float* wsum, const float* lsum, const float* b,
                         float* corr);
/* Views [v0, v0+nv) of the slab SART pass on the whole volume vol; d is the
 * whole scan with n_slabs = D (its slab field is ignored).  engine = 0: the
 * multi-GPU backprojector's arithmetic; 1: the engine's gather update
 * (og_backproject_gather) on each slab geometry.  Returns -1 if d does not
 * split into D slabs. */
int og_sart_pass_slabs(const og_desc* d, float* vol, const float* sino, float beta, int v0, int nv, int engine);

/* ---- FGP TV prox, 7-array GPU form (V63/kernel_FGP_Denoise_GPUx7.cu:2-88,
 *      driver V63/host_FGP_Denoise_GPUx7.c:1-111) ---- */
void og_fgp(int M, int N, int Z, const float* f, float lambda, int iters, float* out);
void og_fgp_f64(int M, int N, int Z, const double* f, double lambda, int iters, double* out);

/* ---- objective (V63/kernel_tool_functions.cu:30-65, V63/host_tool_functions.cu:18-101) ---- */
double og_tv_norm(int M, int N, int Z, const float* vol);
double og_l2_norm(const float* a, const float* b, long long n);

/* ---- FISTA outer step (V63/main_recon.cu:372-384) ---- */
void og_fista_momentum(long long n, float* y, float* xprev, const float* x, float t_prev, float t_k);

/* ---- FDK (V63/host_FDK.cpp, V63/FDK/kernel_FDK.cu, V63/FDK/FFT_1d_GPU.h:241-287) ---- */
void og_fdk_weight(const og_geom* g, const float* in, float* out, int nviews);
/* Spatial kernel equivalent to the reference's padded-DFT ramp: h[n+R-1], n in (-R,R). */
void og_ramp_kernel(const og_geom* g, double* h);
/* Ramp filtering of every row: direct linear convolution with og_ramp_kernel. */
void og_ramp_filter(const og_geom* g, const float* in, float* out, int nrows);
/* The reference's frequency-domain form evaluated by direct DFT (slow; small sizes). */
void og_ramp_filter_dft(const og_geom* g, const float* in, float* out, int nrows);
void og_fdk_bp_view(const og_geom* g, float* vol, const float* view, float s, float c);
void og_fdk(const og_geom* g, const float* sino, float* vol);

/* ---- seeded ellipsoid phantoms ---- */
/* params: n x 10 doubles: cx,cy,cz, ax,ay,az, phi,theta,psi (rad), mu */
void og_phantom_voxelize(const og_geom* g, const double* params, int n, float* vol);
void og_phantom_project(const og_geom* g, const double* params, int n, double s, double c,
                        float* out);

#ifdef __cplusplus
}
#endif
#endif
