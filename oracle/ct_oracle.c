/*
 * ct_oracle.c -- CPU restatement of the reference CBCT reconstruction path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product): see ct_oracle.h.
 *
 * Built with -O2 -fopenmp -ffp-contract=off and no fast-math, so every float
 * expression rounds exactly as written.  Every expression that feeds a
 * result keeps the reference's operation order; the comments give the
 * reference file:line each block restates (V63/ = CBCT/CBCT_1024V_1024P_
 * multiGPU_v6.3_20170823/).
 */
#include "ct_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OG_PI_F 3.141592653589793f   /* const float PI, V63/main_recon.cu:105 */

/* ------------------------------------------------------------------------ */
/* geometry (V63/main_recon.cu:60-111)                                      */
/* ------------------------------------------------------------------------ */
int og_init(og_geom* g, const og_desc* d)
{
    if (!g || !d || d->nx <= 0 || d->ny <= 0 || d->nz <= 0 || d->nu <= 0 || d->nv <= 0 ||
        d->vx <= 0.f || d->du <= 0.f)
        return -1;
    memset(g, 0, sizeof(*g));
    g->d = *d;
    if (g->d.vy <= 0.f) g->d.vy = d->vx;      /* volumn_y = volumn_x           */
    if (g->d.vz <= 0.f) g->d.vz = d->vx;      /* volumn_z = volumn_x (CBCT)    */
    if (g->d.dv <= 0.f) g->d.dv = d->du;      /* one pitch for both axes        */
    const og_desc* e = &g->d;
    /* Detector_Ymin = -Detector_pixel_x*(float(R)/2.0f - 0.5f) + Offset (:83) */
    g->ymin = -e->du * ((float)e->nu / 2.0f - 0.5f) + e->offset;
    /* Detector_Zmin = -Detector_pixel_x*(float(Z_prj)/2.0f - 0.5f) (:84)       */
    g->zmin = -e->dv * ((float)e->nv / 2.0f - 0.5f);
    /* inv_volumn_x = 1.0/volumn_x: a double division stored as float (:88)    */
    g->inv_vx = (float)(1.0 / (double)e->vx);
    g->inv_vy = (float)(1.0 / (double)e->vy);
    g->inv_vz = (float)(1.0 / (double)e->vz);
    /* boundary_voxel_x = -volumn_x*(float(M)/2.0f + M_Offset) (:90)           */
    g->bx = -e->vx * ((float)e->nx / 2.0f + (float)e->m_offset);
    g->by = -e->vy * ((float)e->ny / 2.0f);
    g->bz = -e->vz * ((float)e->nz / 2.0f);
    /* Source_x = DSO, Source_y = Offset, Source_z = 0 (:101-103)              */
    g->srcx = e->dso;
    g->srcy = e->offset;
    g->srcz = 0.0f;
    g->rows = e->nv;
    if (e->ct_style == 3) {
        /* the automatic source distribution of T42/main_recon.cu:76-108: the
         * first source sees the volume's bottom face from the detector's
         * bottom row, the last its top face from the top row */
        const int K = e->n_sources;
        if (K < 1 || e->dv != e->du || e->vz != e->vx) return -1;
        g->rows = e->nv * K;
        g->zmax = +e->du * ((float)e->nv / 2.0f - 0.5f);                  /* :93 */
        if (K == 1) {                                                     /* :97-100 */
            g->zsrc0 = 0.0f;
            g->zsrc_dz = 0.0f;
        } else {
            const float bzu = -e->vz * ((float)e->nz / 2.0f) + (float)e->nz * e->vz;   /* :76 */
            const float zsmax = (bzu - g->zmax) * (e->dso - e->dod) / e->dso + g->zmax; /* :105 */
            g->zsrc0 = (g->bz - g->zmin) * (e->dso - e->dod) / e->dso + g->zmin;       /* :106 */
            g->zsrc_dz = (zsmax - g->zsrc0) / (float)(K - 1);                          /* :107 */
        }
    } else if (e->ct_style < 0 || e->ct_style > 3) {
        return -1;
    }
    g->k0 = 0;
    g->bz_ref = g->bz;
    g->zpar_kr = e->ct_style != 3;
    g->row_lo = 0;
    g->row_hi = g->rows;
    /* T42's one-device projector stops at alpha_max - alpha_c > 1e-6f
     * (T42/voxel/kernel_IterativeRecon_TBCT_voxel.cu:282); V63's and T42's
     * multi-GPU projectors at 1e-16f (T42/voxel/..._multiGPU.cu:303,853) */
    g->loop_eps = e->ct_style == 3 && e->n_slabs <= 1 ? 1e-6f : 1e-16f;
    if (e->n_slabs > 1 && e->slab == -1) {
        /* the whole volume as the multi-GPU build's row-split projector
         * traverses it (V63/..._multiGPU.cu:21-590, T42/voxel/..._multiGPU.cu:22-576):
         * V63's own rules, so T42's gains the z-parallel k range */
        if (e->nz % e->n_slabs != 0 || e->nv % e->n_slabs != 0) return -1;
        g->zpar_kr = 1;
        return 0;
    }
    if (e->n_slabs > 1) {
        /* slab subVolIdx of the multi-GPU build: ZETA/D slices, its own
         * BOUNDARY_VOXEL_Z and ZETA_new in every z plane of the traversal, no
         * z-parallel k range (V63/kernel_IterativeRecon_universal_multiGPU.cu:
         * 636-637,686-687,775-800,891); fan-slice and parallel beams trace only the rows of
         * the slab's band (:663).  ZETA and Z_prj split evenly (V63/main_recon.cu:24). */
        const int D = e->n_slabs, sl = e->slab, Z = e->nz;
        if (sl < 0 || sl >= D || Z % D != 0 || e->nv % D != 0) return -1;
        g->d.nz = Z / D;
        g->k0 = Z / D * sl;
        g->bz = g->bz_ref + e->vz * (float)Z / (float)D * (float)sl;
        g->zpar_kr = 0;
        if (e->ct_style == 1 || e->ct_style == 2) {
            g->row_lo = e->nv / D * sl;
            g->row_hi = e->nv / D * (sl + 1);
        }
    }
    return 0;
}

float og_row_z(const og_geom* g, int v)
{
    const int vr = g->d.ct_style == 3 ? v % g->d.nv : v;
    return g->zmin + (float)vr * g->d.dv;
}

void og_source(const og_geom* g, float s, float c, int u, int v, float* x2x, float* x2y, float* x2z)
{
    if (g->d.ct_style == 2) {                                    /* :34-37 */
        *x2x = g->srcx * c - (g->ymin + (float)u * g->d.du) * s;
        *x2y = g->srcx * s + (g->ymin + (float)u * g->d.du) * c;
    } else {                                                     /* :23-24, :29-30 */
        *x2x = g->srcx * c - g->srcy * s;
        *x2y = g->srcx * s + g->srcy * c;
    }
    if (g->d.ct_style == 3)
        *x2z = g->zsrc0 + (float)(v / g->d.nv) * g->zsrc_dz;      /* T42/...TBCT_voxel.cu:33 */
    else
        *x2z = g->d.ct_style == 0 ? g->srcz : g->zmin + (float)v * g->d.dv;   /* :25, :31, :38 */
}

/* V63/host_IterativeRecon_CBCT.c:34-41 (SART/FP) and V63/host_FDK.cpp:35-40 (FDK) */
void og_view_trig(const og_geom* g, int view, int fdk, float* s, float* c)
{
    float t = (float)view * g->d.us_rate + g->d.initial_angle;
    t = (t + g->d.shift_angle) * OG_PI_F / 180.0f;
    if (!fdk) t = -t;
    *s = sinf(t);
    *c = cosf(t);
}

/* ------------------------------------------------------------------------ */
/* Siddon traversal (V63/kernel_IterativeRecon_universal.cu:7-567)          */
/* ------------------------------------------------------------------------ */
typedef struct {
    int mode;                 /* 0: sum, 1: scatter                        */
    const float* vol;
    float y;                  /* scatter value                              */
    int thresh;
    float thr;
    double* acc;
    double* lacc;
    int nseg;
    uint64_t hash;
    float a_lo, a_hi;         /* alpha interval the traversal covered       */
    int vi0, vj0, vk0, par;   /* start voxel and parallel axes              */
} og_visit;

#define FNV_OFFSET 1469598103934665603ULL
#define FNV_PRIME  1099511628211ULL

/* plane coordinate used by every alpha in the reference kernel:
 * (volumn_x * n + boundary_voxel_x)                                         */
static inline float og_plane(float v, int n, float b) { return v * (float)n + b; }

static inline float og_traverse(const og_geom* g, float s, float c, int u, int v, int entry64,
                                og_visit* vis, float* len_out)
{
    const int M = g->d.nx, N = g->d.ny, Z = g->d.nz;
    const float vx = g->d.vx, vy = g->d.vy, vz = g->d.vz;
    const float bx = g->bx, by = g->by, bz = g->bz;

    /* source (X2) and detector pixel centre (X1), :21-45 */
    float x2x, x2y, x2z;
    og_source(g, s, c, u, v, &x2x, &x2y, &x2z);
    const float x1x = g->d.dod * c - (g->ymin + (float)u * g->d.du) * s;
    const float x1y = g->d.dod * s + (g->ymin + (float)u * g->d.du) * c;
    const float x1z = og_row_z(g, v);
    /* T42's traversal (T42/...TBCT_voxel.cu:1-544) differs in two places:
     * no special k range for rays parallel to the z planes (:171) and the
     * loop test alpha_max - alpha_c > 1e-6f (:282) */
    const int tb = g->d.ct_style == 3;
    const int zpar_k = g->zpar_kr && fabsf(x1z - x2z) < g->d.vz * 1e-6f;

    const float ix = 1.0f / (x2x - x1x);   /* :48-50 */
    const float iy = 1.0f / (x2y - x1y);
    const float iz = 1.0f / (x2z - x1z);

    float sum = 0.0f, len = 0.0f;

    /* step 1: alpha_min / alpha_max, :77-104 */
    float a0, a1;
    a0 = (bx + vx * 0.0f - x1x) * ix;
    a1 = (bx + vx * (float)M - x1x) * ix;
    const float axmin = fminf(a0, a1), axmax = fmaxf(a0, a1);
    a0 = (by + vy * 0.0f - x1y) * iy;
    a1 = (by + vy * (float)N - x1y) * iy;
    const float aymin = fminf(a0, a1), aymax = fmaxf(a0, a1);
    a0 = (bz + vz * 0.0f - x1z) * iz;
    a1 = (bz + vz * (float)Z - x1z) * iz;
    const float azmin = fminf(a0, a1), azmax = fmaxf(a0, a1);
    float amin = fmaxf(fmaxf(axmin, aymin), fmaxf(aymin, azmin));
    float amax = fminf(fminf(axmax, aymax), fminf(aymax, azmax));

    int i_min = 0, j_min = 0, k_min = 0, i_max = 0, j_max = 0, k_max = 0;
    int hit;

    if (!entry64) {
        hit = !(amax <= amin);                                     /* :108 */
        if (hit) {
            /* steps 2,3: first/last plane index per axis, :113-209 */
            if (x1x < x2x) {
                i_min = (amin == axmin) ? 1 : (int)(floorf((amin * (x2x - x1x) + x1x - bx) * g->inv_vx) + 1.0f);
                i_max = (amax == axmax) ? M : (int)floorf((amax * (x2x - x1x) + x1x - bx) * g->inv_vx);
            } else {
                i_max = (amin == axmin) ? M - 1 : (int)floorf((amin * (x2x - x1x) + x1x - bx) * g->inv_vx);
                i_min = (amax == axmax) ? 0 : (int)(floorf((amax * (x2x - x1x) + x1x - bx) * g->inv_vx) + 1.0f);
            }
            if (x1y < x2y) {
                j_min = (amin == aymin) ? 1 : (int)(floorf((amin * (x2y - x1y) + x1y - by) * g->inv_vy) + 1.0f);
                j_max = (amax == aymax) ? N : (int)floorf((amax * (x2y - x1y) + x1y - by) * g->inv_vy);
            } else {
                j_max = (amin == aymin) ? N - 1 : (int)floorf((amin * (x2y - x1y) + x1y - by) * g->inv_vy);
                j_min = (amax == aymax) ? 0 : (int)(floorf((amax * (x2y - x1y) + x1y - by) * g->inv_vy) + 1.0f);
            }
            if (zpar_k) {
                k_min = (int)(floorf((x1z - bz) * g->inv_vz) + 1.0f);
                k_max = (int)floorf((x1z - bz) * g->inv_vz);
            } else if (x1z < x2z) {
                k_min = (amin == azmin) ? 1 : (int)(floorf((amin * (x2z - x1z) + x1z - bz) * g->inv_vz) + 1.0f);
                k_max = (amax == azmax) ? Z : (int)floorf((amax * (x2z - x1z) + x1z - bz) * g->inv_vz);
            } else {
                k_max = (amin == azmin) ? Z - 1 : (int)floorf((amin * (x2z - x1z) + x1z - bz) * g->inv_vz);
                k_min = (amax == azmax) ? 0 : (int)(floorf((amax * (x2z - x1z) + x1z - bz) * g->inv_vz) + 1.0f);
            }
        }
    } else {
        /* FP64 entry/exit: the same formulas evaluated in double on the float
         * positions; the traversal itself stays in float. */
        const double X1x = x1x, X1y = x1y, X1z = x1z;
        const double Dx = (double)x2x - X1x, Dy = (double)x2y - X1y, Dz = (double)x2z - X1z;
        const double Ix = 1.0 / Dx, Iy = 1.0 / Dy, Iz = 1.0 / Dz;
        const double Bx = bx, By = by, Bz = bz;
        const double IVx = 1.0 / (double)vx, IVy = 1.0 / (double)vy, IVz = 1.0 / (double)vz;
        double b0, b1;
        b0 = ((double)og_plane(vx, 0, bx) - X1x) * Ix; b1 = ((double)og_plane(vx, M, bx) - X1x) * Ix;
        const double Axmin = fmin(b0, b1), Axmax = fmax(b0, b1);
        b0 = ((double)og_plane(vy, 0, by) - X1y) * Iy; b1 = ((double)og_plane(vy, N, by) - X1y) * Iy;
        const double Aymin = fmin(b0, b1), Aymax = fmax(b0, b1);
        b0 = ((double)og_plane(vz, 0, bz) - X1z) * Iz; b1 = ((double)og_plane(vz, Z, bz) - X1z) * Iz;
        const double Azmin = fmin(b0, b1), Azmax = fmax(b0, b1);
        const double Amin = fmax(fmax(Axmin, Aymin), Azmin);
        const double Amax = fmin(fmin(Axmax, Aymax), Azmax);
        hit = !(Amax <= Amin);
        if (hit) {
            if (x1x < x2x) {
                i_min = (Amin == Axmin) ? 1 : (int)floor((Amin * Dx + X1x - Bx) * IVx) + 1;
                i_max = (Amax == Axmax) ? M : (int)floor((Amax * Dx + X1x - Bx) * IVx);
            } else {
                i_max = (Amin == Axmin) ? M - 1 : (int)floor((Amin * Dx + X1x - Bx) * IVx);
                i_min = (Amax == Axmax) ? 0 : (int)floor((Amax * Dx + X1x - Bx) * IVx) + 1;
            }
            if (x1y < x2y) {
                j_min = (Amin == Aymin) ? 1 : (int)floor((Amin * Dy + X1y - By) * IVy) + 1;
                j_max = (Amax == Aymax) ? N : (int)floor((Amax * Dy + X1y - By) * IVy);
            } else {
                j_max = (Amin == Aymin) ? N - 1 : (int)floor((Amin * Dy + X1y - By) * IVy);
                j_min = (Amax == Aymax) ? 0 : (int)floor((Amax * Dy + X1y - By) * IVy) + 1;
            }
            if (zpar_k) {
                k_min = (int)floor((X1z - Bz) * IVz) + 1;
                k_max = (int)floor((X1z - Bz) * IVz);
            } else if (x1z < x2z) {
                k_min = (Amin == Azmin) ? 1 : (int)floor((Amin * Dz + X1z - Bz) * IVz) + 1;
                k_max = (Amax == Azmax) ? Z : (int)floor((Amax * Dz + X1z - Bz) * IVz);
            } else {
                k_max = (Amin == Azmin) ? Z - 1 : (int)floor((Amin * Dz + X1z - Bz) * IVz);
                k_min = (Amax == Azmax) ? 0 : (int)floor((Amax * Dz + X1z - Bz) * IVz) + 1;
            }
            amin = (float)Amin;
            amax = (float)Amax;
        }
    }

    if (hit) {
        /* initial planes and next-plane alphas, :218-266 */
        float ax, ay, az;
        int i, j, k;
        if (fabsf(x1x - x2x) < vx * 1e-6f) { ax = INFINITY; i = i_min - 1; }
        else if (x1x < x2x) { ax = (vx * (float)i_min + bx - x1x) * ix; i = i_min - 1; }
        else { ax = (vx * (float)i_max + bx - x1x) * ix; i = i_max + 1; }
        if (fabsf(x1y - x2y) < vy * 1e-6f) { ay = INFINITY; j = j_min - 1; }
        else if (x1y < x2y) { ay = (vy * (float)j_min + by - x1y) * iy; j = j_min - 1; }
        else { ay = (vy * (float)j_max + by - x1y) * iy; j = j_max + 1; }
        if (fabsf(x1z - x2z) < vz * 1e-6f) { az = INFINITY; k = k_min - 1; }
        else if (x1z < x2z) { az = (vz * (float)k_min + bz - x1z) * iz; k = k_min - 1; }
        else { az = (vz * (float)k_max + bz - x1z) * iz; k = k_max + 1; }
        (void)i; (void)j; (void)k;

        /* voxel indices, :271-284 */
        int vi = (x1x < x2x) ? i_min - 1 : i_max;
        int vj = (x1y < x2y) ? j_min - 1 : j_max;
        int vk = (x1z < x2z) ? k_min - 1 : k_max;
        vis->vi0 = vi; vis->vj0 = vj; vis->vk0 = vk;
        vis->par = (ax == INFINITY ? 1 : 0) | (ay == INFINITY ? 2 : 0) | (az == INFINITY ? 4 : 0);
        /* direction per axis and the offset from the voxel index to the next
         * plane index: +1 when increasing, 0 when decreasing (the reference's
         * next_alpha_index = i+1 / i-1 with i tracking the plane). */
        const int sx = (x1x < x2x) ? 1 : ((x1x > x2x) ? -1 : 0);
        const int sy = (x1y < x2y) ? 1 : ((x1y > x2y) ? -1 : 0);
        const int sz = (x1z < x2z) ? 1 : ((x1z > x2z) ? -1 : 0);
        const int ox = sx > 0, oy = sy > 0, oz = sz > 0;

        /* :290 */
        const float d12 = sqrtf((x2x - x1x) * (x2x - x1x) + (x2y - x1y) * (x2y - x1y) +
                                (x2z - x1z) * (x2z - x1z));
        float ac = amin;
        /* :297-551.  The reference's seven branches select the smallest
         * next-plane alpha and advance every axis that attains it (ties advance
         * two or three axes at once); "advance every axis equal to the minimum"
         * is the same rule for all non-NaN alphas. */
        const int maxsteps = M + N + Z + 3;
        int steps = 0;
        const float eps = g->loop_eps;
        while (amax - ac > eps) {
            if (vi > M - 1 || vi < 0 || vj > N - 1 || vj < 0 || vk > Z - 1 || vk < 0) break;
            if (++steps > maxsteps) break;   /* unreachable for finite alphas */
            const float m = fminf(fminf(ax, ay), az);
            const float seg = d12 * (m - ac);
            const int idx = vk * M * N + vj * M + vi;
            len = len + seg;
            if (vis->mode == 0) {
                sum = sum + seg * vis->vol[idx];
            } else if (vis->mode == 1) {
                if (!vis->thresh || seg > vis->thr) {
                    vis->acc[idx] += (double)seg * (double)vis->y;
                    if (vis->lacc) vis->lacc[idx] += (double)seg;
                }
            }
            if (vis->nseg == 0) vis->a_lo = ac;
            vis->nseg++;
            vis->hash = (vis->hash ^ (uint64_t)(uint32_t)idx) * FNV_PRIME;
            ac = m;
            vis->a_hi = ac;
            if (ax == m) { vi += sx; ax = (vx * (float)(vi + ox) + bx - x1x) * ix; }
            if (ay == m) { vj += sy; ay = (vy * (float)(vj + oy) + by - x1y) * iy; }
            if (az == m) { vk += sz; az = (vz * (float)(vk + oz) + bz - x1z) * iz; }
        }
    }
    *len_out = len;
    return sum;
}

void og_fp_window(const og_geom* g, float s, float c, int u, int v, int entry64, float* lo, float* hi)
{
    int st[4];
    og_fp_start(g, s, c, u, v, entry64, lo, hi, st);
}

void og_fp_start(const og_geom* g, float s, float c, int u, int v, int entry64, float* lo, float* hi, int* start)
{
    og_visit vis;
    memset(&vis, 0, sizeof(vis));
    vis.mode = 2;
    vis.hash = FNV_OFFSET;
    vis.a_lo = 1.0f;
    vis.a_hi = 0.0f;
    vis.vi0 = vis.vj0 = vis.vk0 = -1;
    float l;
    og_traverse(g, s, c, u, v, entry64, &vis, &l);
    *lo = vis.a_lo;
    *hi = vis.a_hi;
    start[0] = vis.vi0; start[1] = vis.vj0; start[2] = vis.vk0; start[3] = vis.par;
}

float og_fp_ray(const og_geom* g, const float* vol, float s, float c, int u, int v,
                int entry64, float* len, int* nseg, uint64_t* hash)
{
    og_visit vis;
    memset(&vis, 0, sizeof(vis));
    vis.mode = 0;
    vis.vol = vol;
    vis.hash = FNV_OFFSET;
    float l;
    float sum = og_traverse(g, s, c, u, v, entry64, &vis, &l);
    if (len) *len = l;
    if (nseg) *nseg = vis.nseg;
    if (hash) *hash = vis.hash;
    return sum;
}

/* epilogue, :554-562 */
void og_forward_view(const og_geom* g, const float* vol, float s, float c, int command,
                     const float* b, float* out, int entry64)
{
    const int R = g->d.nu, ZP = g->rows;
    const float thr = g->d.vz * 1e-6f;
#pragma omp parallel for schedule(dynamic, 1)
    for (int v = 0; v < ZP; ++v) {
        for (int u = 0; u < R; ++u) {
            float len;
            const float sum = og_fp_ray(g, vol, s, c, u, v, entry64, &len, NULL, NULL);
            const int p = v * R + u;
            if (len < thr) out[p] = 0.0f;
            else if (command == 0) out[p] = sum;
            else out[p] = (b[p] - sum) / len;
        }
    }
}

void og_forward_trace(const og_geom* g, const float* vol, float s, float c, int entry64,
                      int* nseg, uint64_t* hash, float* len)
{
    const int R = g->d.nu, ZP = g->rows;
#pragma omp parallel for schedule(dynamic, 1)
    for (int v = 0; v < ZP; ++v)
        for (int u = 0; u < R; ++u) {
            const int p = v * R + u;
            og_fp_ray(g, vol, s, c, u, v, entry64, &len[p], &nseg[p], &hash[p]);
        }
}

/* ------------------------------------------------------------------------ */
/* FP64 oracle: the same Siddon traversal, every quantity in double.        */
/* ------------------------------------------------------------------------ */
typedef struct {
    int M, N, Z, ct_style, nv;
    double vx, vy, vz, bx, by, bz, ymin, zmin, du, dv, dso, dod, srcx, srcy, srcz, zsrc0, zsrc_dz;
} og_geom64;

static void og_geom_to64(const og_geom* g, og_geom64* h)
{
    const og_desc* e = &g->d;
    h->M = e->nx; h->N = e->ny; h->Z = e->nz;
    h->vx = e->vx; h->vy = e->vy; h->vz = e->vz;
    h->bx = -h->vx * ((double)e->nx / 2.0 + (double)e->m_offset);
    h->by = -h->vy * ((double)e->ny / 2.0);
    h->bz = -h->vz * ((double)e->nz / 2.0);
    h->du = e->du; h->dv = e->dv;
    h->ymin = -h->du * ((double)e->nu / 2.0 - 0.5) + (double)e->offset;
    h->zmin = -h->dv * ((double)e->nv / 2.0 - 0.5);
    h->dso = e->dso; h->dod = e->dod;
    h->srcx = e->dso; h->srcy = e->offset; h->srcz = 0.0;
    h->ct_style = e->ct_style;
    h->nv = e->nv;
    h->zsrc0 = h->zsrc_dz = 0.0;
    if (e->ct_style == 3 && e->n_sources > 1) {   /* T42/main_recon.cu:104-107 in double */
        const double zmax = h->dv * ((double)e->nv / 2.0 - 0.5), zmin = -zmax;
        const double bzu = h->bz + (double)e->nz * h->vz;
        const double zsmax = (bzu - zmax) * (h->dso - h->dod) / h->dso + zmax;
        h->zsrc0 = (h->bz - zmin) * (h->dso - h->dod) / h->dso + zmin;
        h->zsrc_dz = (zsmax - h->zsrc0) / (double)(e->n_sources - 1);
    }
}

static void og_source64(const og_geom64* h, double s, double c, int u, int v, double x2[3])
{
    const double pu = h->ymin + u * h->du;
    x2[0] = h->ct_style == 2 ? h->srcx * c - pu * s : h->srcx * c - h->srcy * s;
    x2[1] = h->ct_style == 2 ? h->srcx * s + pu * c : h->srcx * s + h->srcy * c;
    x2[2] = h->ct_style == 3 ? h->zsrc0 + (double)(v / h->nv) * h->zsrc_dz
                             : (h->ct_style == 0 ? h->srcz : h->zmin + v * h->dv);
}

typedef void (*og_visit64_fn)(void* ctx, long long idx, double seg);

static double og_traverse64(const og_geom64* h, double s, double c, int u, int v,
                            og_visit64_fn fn, void* ctx, const double* vol, double* len_out)
{
    const int M = h->M, N = h->N, Z = h->Z;
    double X2[3];
    og_source64(h, s, c, u, v, X2);
    const double x2x = X2[0], x2y = X2[1], x2z = X2[2];
    const double pu = h->ymin + u * h->du;
    const int vr = h->ct_style == 3 ? v % h->nv : v;
    const double x1x = h->dod * c - pu * s, x1y = h->dod * s + pu * c, x1z = h->zmin + vr * h->dv;
    const double dx = x2x - x1x, dy = x2y - x1y, dz = x2z - x1z;
    const double P0[3] = {h->bx, h->by, h->bz};
    const double Vv[3] = {h->vx, h->vy, h->vz};
    const int Nn[3] = {M, N, Z};
    const double X1[3] = {x1x, x1y, x1z}, D[3] = {dx, dy, dz};
    double amin = -INFINITY, amax = INFINITY;
    for (int a = 0; a < 3; ++a) {
        if (fabs(D[a]) < Vv[a] * 1e-12) {
            if (X1[a] <= P0[a] || X1[a] >= P0[a] + Vv[a] * Nn[a]) { *len_out = 0; return 0; }
            continue;
        }
        const double t0 = (P0[a] - X1[a]) / D[a], t1 = (P0[a] + Vv[a] * Nn[a] - X1[a]) / D[a];
        amin = fmax(amin, fmin(t0, t1));
        amax = fmin(amax, fmax(t0, t1));
    }
    double sum = 0, len = 0;
    if (amax > amin) {
        const double d12 = sqrt(dx * dx + dy * dy + dz * dz);
        int vox[3], dir[3];
        double an[3];
        const double amid = 0.5 * (amin + amax);
        /* start voxel from the midpoint of the first (sub-voxel) step */
        for (int a = 0; a < 3; ++a) {
            dir[a] = D[a] > 0 ? 1 : (D[a] < 0 ? -1 : 0);
            (void)amid;
        }
        /* locate the voxel containing the entry point, nudged inwards */
        double ain = amin;
        for (int a = 0; a < 3; ++a) {
            const double x = X1[a] + ain * D[a];
            int iv = (int)floor((x - P0[a]) / Vv[a]);
            if (dir[a] > 0 && fabs(x - (P0[a] + Vv[a] * (iv))) < 1e-12 * Vv[a]) { /* on plane */ }
            if (iv < 0) iv = 0;
            if (iv > Nn[a] - 1) iv = Nn[a] - 1;
            /* choose by the direction when the point sits on a plane */
            const double xin = X1[a] + (ain + 1e-9 * (amax - amin)) * D[a];
            iv = (int)floor((xin - P0[a]) / Vv[a]);
            if (iv < 0) iv = 0;
            if (iv > Nn[a] - 1) iv = Nn[a] - 1;
            vox[a] = iv;
            if (dir[a] == 0) an[a] = INFINITY;
            else an[a] = (P0[a] + Vv[a] * (iv + (dir[a] > 0)) - X1[a]) / D[a];
        }
        double ac = amin;
        int steps = 0;
        while (ac < amax && steps++ < M + N + Z + 3) {
            double m = fmin(fmin(an[0], an[1]), an[2]);
            if (m > amax) m = amax;
            const double seg = d12 * (m - ac);
            const long long idx = (long long)vox[2] * M * N + (long long)vox[1] * M + vox[0];
            len += seg;
            if (vol) sum += seg * vol[idx];
            if (fn) fn(ctx, idx, seg);
            ac = m;
            int out = 0;
            for (int a = 0; a < 3; ++a)
                if (an[a] == m) {
                    vox[a] += dir[a];
                    if (vox[a] < 0 || vox[a] >= Nn[a]) out = 1;
                    an[a] = (P0[a] + Vv[a] * (vox[a] + (dir[a] > 0)) - X1[a]) / D[a];
                }
            if (out) break;
        }
    }
    *len_out = len;
    return sum;
}

void og_forward_view_f64(const og_geom* g, const double* vol, double s, double c, double* out)
{
    og_geom64 h;
    og_geom_to64(g, &h);
    const int R = g->d.nu, ZP = g->rows;
#pragma omp parallel for schedule(dynamic, 1)
    for (int v = 0; v < ZP; ++v)
        for (int u = 0; u < R; ++u) {
            double len;
            out[v * R + u] = og_traverse64(&h, s, c, u, v, NULL, NULL, vol, &len);
        }
}

typedef struct { double* acc; double y; } og_sc64;
static void og_scatter64(void* ctx, long long idx, double seg)
{
    og_sc64* q = (og_sc64*)ctx;
    q->acc[idx] += seg * q->y;
}

void og_adjoint_view_f64(const og_geom* g, const double* y, double s, double c, double* acc)
{
    og_geom64 h;
    og_geom_to64(g, &h);
    const int R = g->d.nu, ZP = g->rows;
    for (int v = 0; v < ZP; ++v)
        for (int u = 0; u < R; ++u) {
            og_sc64 q = {acc, y[v * R + u]};
            double len;
            og_traverse64(&h, s, c, u, v, og_scatter64, &q, NULL, &len);
        }
}

/* ------------------------------------------------------------------------ */
/* reference BP (V63/kernel_IterativeRecon_universal.cu:571-810)            */
/* ------------------------------------------------------------------------ */
int og_fov_masked(const og_geom* g, int i, int j)
{
    const float vx = g->d.vx, vy = g->d.vy;
    const float hx = (float)g->d.nx * 0.5f - 0.5f, hy = (float)g->d.ny * 0.5f - 0.5f;
    const float ex = (float)i - hx - (float)g->d.m_offset;
    const float ey = (float)j - hy;
    return ex * vx * ex * vx + ey * vy * ey * vy >= hx * vx * hy * vy;   /* :626-628 */
}

/* TBCT backprojection and update, T42/voxel/kernel_IterativeRecon_TBCT_voxel.cu:
 * backprj_ray_driven_3d_kernel (:546-763) accumulates, per voxel and source,
 * the chord-weighted corrections and chord lengths of the source's rays into
 * two zeroed volumes by atomicAdd; update (:765-775) then adds
 * beta*sum/length where the summed length exceeds volumn_x*1e-3 (a double
 * comparison).  Sources are added in ascending order here. */
/* The tetrahedron-beam backprojector's voxel centre: bx + vx*(0.5f + i)
 * (T42/voxel/kernel_IterativeRecon_TBCT_voxel.cu:568-570), or in a slab of its
 * multi-GPU build bx + vx*0.5f + i*vx and boundary_voxel_z +
 * vz*(ZETA/D*s + 0.5f) + k*vz (T42/voxel/..._multiGPU.cu:1140-1142). */
static inline void og_tb_centre(const og_geom* g, int i, int j, int k, float* cx, float* cy, float* cz)
{
    const float vx = g->d.vx, vy = g->d.vy, vz = g->d.vz;
    if (g->d.n_slabs > 1) {
        *cx = g->bx + vx * 0.5f + (float)i * vx;
        *cy = g->by + vy * 0.5f + (float)j * vy;
        *cz = g->bz_ref + vz * ((float)g->k0 + 0.5f) + (float)k * vz;
    } else {
        *cx = g->bx + vx * (0.5f + (float)i);
        *cy = g->by + vy * (0.5f + (float)j);
        *cz = g->bz + vz * (0.5f + (float)k);
    }
}

static void og_backproject_ref_tbct(const og_geom* g, float* vol, const float* corr, float beta, float s, float c)
{
    const int M = g->d.nx, N = g->d.ny, Z = g->d.nz, R = g->d.nu, ZP = g->d.nv, K = g->d.n_sources;
    const float vx = g->d.vx, vy = g->d.vy, vz = g->d.vz;
    const float DSO = g->d.dso, DOD = g->d.dod, du = g->d.du;
    const float inv_dp = 1.0f / du;                                      /* :592 */
    const double thr_upd = (double)vx * 1e-3;                            /* :772 */
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < Z; ++k)
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < M; ++i) {
                const long long idx = (long long)M * N * k + (long long)M * j + i;
                float WS = 0.0f, L = 0.0f;                               /* the zeroed sums */
                if (!og_fov_masked(g, i, j)) {                           /* :600-608 */
                    float cx, cy, cz;
                    og_tb_centre(g, i, j, k, &cx, &cy, &cz);
                    const float sx = g->srcx * c - g->srcy * s;          /* :613-614 */
                    const float sy = g->srcx * s + g->srcy * c;
                    const float tc = cx * c + cy * s;                    /* :620 */
                    const float upper = (cz + vz - g->zmin) * (DSO - DOD) / (tc - DOD) + g->zmin;   /* :623 */
                    const float lower = (cz - vz - g->zmax) * (DSO - DOD) / (tc - DOD) + g->zmax;   /* :624 */
                    for (int src = 0; src < K; ++src) {
                        const float sz = g->zsrc0 + (float)src * g->zsrc_dz;                      /* :615 */
                        if (sz < lower || sz > upper) continue;                                    /* :626-627 */
                        float minY = INFINITY, minZ = INFINITY, maxY = -INFINITY, maxZ = -INFINITY;
                        for (int kk = 0; kk < 2; ++kk)                                             /* :631-655 */
                            for (int jj = 0; jj < 2; ++jj)
                                for (int ii = 0; ii < 2; ++ii) {
                                    const float px = cx + (float)ii * vx - 0.5f * vx;
                                    const float py = cy + (float)jj * vy - 0.5f * vy;
                                    const float pz = cz + (float)kk * vz - 0.5f * vz;
                                    const float t = px * c + py * s;
                                    const float ss = -px * s + py * c;
                                    const float ou = (t - DOD) / (DSO - t) * (ss - g->srcy) + ss;
                                    const float oz = (t - DOD) / (DSO - t) * (pz - sz) + pz;
                                    minY = fminf(minY, ou); maxY = fmaxf(maxY, ou);
                                    minZ = fminf(minZ, oz); maxZ = fmaxf(maxZ, oz);
                                }
                        int minYi = (int)floorf((minY - g->ymin) * inv_dp + 0.5f);               /* :659-662 */
                        int maxYi = (int)floorf((maxY - g->ymin) * inv_dp + 0.5f);
                        int minZi = (int)floorf((minZ - g->zmin) * inv_dp + 0.5f);
                        int maxZi = (int)floorf((maxZ - g->zmin) * inv_dp + 0.5f);
                        float sw = 0.0f, sl = 0.0f;
                        if (!(((minYi < 0) && (maxYi < 0)) || (minYi > R - 1 && maxYi > R - 1) ||  /* :668 */
                              ((minZi < 0) && (maxZi < 0)) || ((minZi > ZP - 1) && (maxZi > ZP - 1)))) {
                            if (minYi <= 0) minYi = 0;                                              /* :678-685 */
                            if (maxYi >= R - 1) maxYi = R - 1;
                            if (minZi <= 0) minZi = 0;
                            if (maxZi >= ZP - 1) maxZi = ZP - 1;
                            for (int jr = minZi; jr <= maxZi; ++jr)                                 /* :689-750 */
                                for (int ir = minYi; ir <= maxYi; ++ir) {
                                    const float qx = DOD * c - (g->ymin + (float)ir * du) * s;
                                    const float qy = DOD * s + (g->ymin + (float)ir * du) * c;
                                    const float qz = g->zmin + (float)jr * du;
                                    const float ax0 = ((cx - 0.5f * vx) - qx) / (sx - qx);
                                    const float ax1 = ((cx + 0.5f * vx) - qx) / (sx - qx);
                                    const float ay0 = ((cy - 0.5f * vy) - qy) / (sy - qy);
                                    const float ay1 = ((cy + 0.5f * vy) - qy) / (sy - qy);
                                    const float az0 = ((cz - 0.5f * vz) - qz) / (sz - qz);
                                    const float az1 = ((cz + 0.5f * vz) - qz) / (sz - qz);
                                    float tx = fminf(ax0, ax1), ty = fminf(ay0, ay1), tz = fminf(az0, az1);
                                    const float amin = fmaxf(fmaxf(tx, ty), fmaxf(ty, tz));
                                    tx = fmaxf(ax0, ax1); ty = fmaxf(ay0, ay1); tz = fmaxf(az0, az1);
                                    const float amax = fminf(fminf(tx, ty), fminf(ty, tz));
                                    if (amax - amin > 0) {
                                        const float d12 = sqrtf((sx - qx) * (sx - qx) + (sy - qy) * (sy - qy) +
                                                                (sz - qz) * (sz - qz));
                                        const float temp = d12 * (amax - amin);
                                        if (temp > vx * 1e-6f) {
                                            sw = sw + temp * corr[(long long)R * ZP * src + (long long)R * jr + ir];
                                            sl = sl + temp;
                                        }
                                    }
                                }
                        }
                        WS = WS + sw;                                                               /* :754-755 */
                        L = L + sl;
                    }
                }
                if ((double)L > thr_upd) vol[idx] += beta * WS / L;                                 /* :772-773 */
            }
}

void og_backproject_ref(const og_geom* g, float* vol, const float* corr, float beta,
                        float s, float c, int command)
{
    if (g->d.ct_style == 3) {
        (void)command;
        og_backproject_ref_tbct(g, vol, corr, beta, s, c);
        return;
    }
    const int M = g->d.nx, N = g->d.ny, Z = g->d.nz, R = g->d.nu, ZP = g->d.nv;
    const float vx = g->d.vx, vy = g->d.vy, vz = g->d.vz;
    const float DSO = g->d.dso, DOD = g->d.dod;
    const float inv_du = 1.0f / g->d.du, inv_dv = 1.0f / g->d.dv;   /* :615 */
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < Z; ++k)
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < M; ++i) {
                const long long idx = (long long)M * N * k + (long long)M * j + i;
                const float cx = g->bx + vx * 0.5f + (float)i * vx;     /* :592-594 */
                const float cy = g->by + vy * 0.5f + (float)j * vy;
                /* :592-594; a slab's voxel centre, multiGPU.cu:1179 (k0 = 0,
                 * bz_ref = bz otherwise: vz*(0.0f+0.5f) = vz*0.5f) */
                const float cz = g->bz_ref + vz * ((float)g->k0 + 0.5f) + (float)k * vz;
                float sw = 0.0f, sl = 0.0f;
                if (!og_fov_masked(g, i, j)) {
                    float minY = INFINITY, minZ = INFINITY, maxY = -INFINITY, maxZ = -INFINITY;
                    for (int kk = 0; kk < 2; ++kk)                       /* :639-678 */
                        for (int jj = 0; jj < 2; ++jj)
                            for (int ii = 0; ii < 2; ++ii) {
                                const float px = cx + (float)ii * vx - 0.5f * vx;
                                const float py = cy + (float)jj * vy - 0.5f * vy;
                                const float pz = cz + (float)kk * vz - 0.5f * vz;
                                const float t = px * c + py * s;
                                const float ss = -px * s + py * c;
                                float ou, oz;                                 /* :655-670 */
                                if (g->d.ct_style == 0) {
                                    ou = (t - DOD) / (DSO - t) * (ss - g->srcy) + ss;
                                    oz = (t - DOD) / (DSO - t) * (pz - g->srcz) + pz;
                                } else if (g->d.ct_style == 1) {
                                    ou = (t - DOD) / (DSO - t) * (ss - g->srcy) + ss;
                                    oz = cz;
                                } else {
                                    ou = ss;
                                    oz = cz;
                                }
                                minY = fminf(minY, ou); maxY = fmaxf(maxY, ou);
                                minZ = fminf(minZ, oz); maxZ = fmaxf(maxZ, oz);
                            }
                    int minYi = (int)floorf((minY - g->ymin) * inv_du + 0.5f);   /* :680-683 */
                    int maxYi = (int)floorf((maxY - g->ymin) * inv_du + 0.5f);
                    int minZi = (int)floorf((minZ - g->zmin) * inv_dv + 0.5f);
                    int maxZi = (int)floorf((maxZ - g->zmin) * inv_dv + 0.5f);
                    if (!(((minYi < 0) && (maxYi < 0)) || (minYi > R - 1 && maxYi > R - 1) ||
                          ((minZi < 0) && (maxZi < 0)) || ((minZi > ZP - 1) && (maxZi > ZP - 1)))) {
                        if (minYi <= 0) minYi = 0;                            /* :699-706 */
                        if (maxYi >= R - 1) maxYi = R - 1;
                        if (minZi <= 0) minZi = 0;
                        if (maxZi >= ZP - 1) maxZi = ZP - 1;
                        float sx = g->srcx * c - g->srcy * s;                 /* :711-726 */
                        float sy = g->srcx * s + g->srcy * c;
                        const float sz = g->d.ct_style == 0 ? g->srcz : cz;
                        for (int jr = minZi; jr <= maxZi; ++jr)
                            for (int ir = minYi; ir <= maxYi; ++ir) {
                                const float qx = DOD * c - (g->ymin + (float)ir * g->d.du) * s;   /* :733-735 */
                                const float qy = DOD * s + (g->ymin + (float)ir * g->d.du) * c;
                                const float qz = g->zmin + (float)jr * g->d.dv;
                                if (g->d.ct_style == 2) {                                         /* :737-742 */
                                    sx = g->srcx * c - (g->ymin + (float)ir * g->d.du) * s;
                                    sy = g->srcx * s + (g->ymin + (float)ir * g->d.du) * c;
                                }
                                const float ax0 = ((cx - 0.5f * vx) - qx) / (sx - qx);   /* :760-765 */
                                const float ax1 = ((cx + 0.5f * vx) - qx) / (sx - qx);
                                const float ay0 = ((cy - 0.5f * vy) - qy) / (sy - qy);
                                const float ay1 = ((cy + 0.5f * vy) - qy) / (sy - qy);
                                const float az0 = ((cz - 0.5f * vz) - qz) / (sz - qz);
                                const float az1 = ((cz + 0.5f * vz) - qz) / (sz - qz);
                                float tx = fminf(ax0, ax1), ty = fminf(ay0, ay1), tz = fminf(az0, az1);
                                const float amin = fmaxf(fmaxf(tx, ty), fmaxf(ty, tz));
                                tx = fmaxf(ax0, ax1); ty = fmaxf(ay0, ay1); tz = fmaxf(az0, az1);
                                const float amax = fminf(fminf(tx, ty), fminf(ty, tz));
                                if (amax - amin > 0) {                                     /* :780-792 */
                                    const float d12 = sqrtf((sx - qx) * (sx - qx) + (sy - qy) * (sy - qy) +
                                                            (sz - qz) * (sz - qz));
                                    const float temp = d12 * (amax - amin);
                                    if (temp > vx * 1e-6f) {
                                        sw = sw + temp * corr[jr * R + ir];
                                        sl = sl + temp;
                                    }
                                }
                            }
                    }
                }
                if (sl < vx * 1e-6f) {                                         /* :799-807 */
                    if (g->d.n_slabs <= 1) vol[idx] += 0.0f;                   /* none in multiGPU.cu:1388-1391 */
                }
                else if (command == 0) vol[idx] = sw;
                else vol[idx] += beta * sw / sl;
            }
}

/* ------------------------------------------------------------------------ */
/* exact adjoint of og_fp_ray (scatter)                                     */
/* ------------------------------------------------------------------------ */
void og_adjoint_view(const og_geom* g, const float* y, float s, float c, int thresh,
                     double* acc, double* lacc)
{
    const int R = g->d.nu, ZP = g->rows;
    for (int v = 0; v < ZP; ++v)
        for (int u = 0; u < R; ++u) {
            og_visit vis;
            memset(&vis, 0, sizeof(vis));
            vis.mode = 1;
            vis.y = y[v * R + u];
            vis.thresh = thresh;
            vis.thr = g->d.vx * 1e-6f;
            vis.acc = acc;
            vis.lacc = lacc;
            float len;
            og_traverse(g, s, c, u, v, 0, &vis, &len);
        }
}

/* ------------------------------------------------------------------------ */
/* SART pass drivers (V63/host_IterativeRecon_CBCT.c:1-67)                  */
/* ------------------------------------------------------------------------ */
void og_sart_pass_ref(const og_geom* g, float* vol, const float* sino, float beta)
{
    const long long P = (long long)g->d.nu * g->rows;
    float* corr = (float*)malloc(sizeof(float) * P);
    for (int j = 0; j < g->d.nviews; ++j) {
        float s, c;
        og_view_trig(g, j, 0, &s, &c);
        og_forward_view(g, vol, s, c, 1, sino + P * j, corr, 0);
        og_backproject_ref(g, vol, corr, beta, s, c, 1);
    }
    free(corr);
}

void og_sart_pass_matched(const og_geom* g, float* vol, const float* sino, float beta)
{
    const long long P = (long long)g->d.nu * g->rows;
    const long long V = (long long)g->d.nx * g->d.ny * g->d.nz;
    const int M = g->d.nx, N = g->d.ny;
    const float thr = g->d.vx * 1e-6f;
    float* corr = (float*)malloc(sizeof(float) * P);
    double* W = (double*)malloc(sizeof(double) * V);
    double* L = (double*)malloc(sizeof(double) * V);
    for (int j = 0; j < g->d.nviews; ++j) {
        float s, c;
        og_view_trig(g, j, 0, &s, &c);
        og_forward_view(g, vol, s, c, 1, sino + P * j, corr, 0);
        memset(W, 0, sizeof(double) * V);
        memset(L, 0, sizeof(double) * V);
        og_adjoint_view(g, corr, s, c, 1, W, L);
#pragma omp parallel for schedule(static)
        for (long long q = 0; q < V; ++q) {
            const int i = (int)(q % M), jj = (int)((q / M) % N);
            if (og_fov_masked(g, i, jj)) continue;
            if (L[q] < thr) continue;
            vol[q] = vol[q] + (float)((double)beta * W[q] / L[q]);
        }
    }
    free(corr); free(W); free(L);
}

typedef struct { double* W; double* L; double y; } og_sc64wl;
static void og_scatter64wl(void* ctx, long long idx, double seg)
{
    og_sc64wl* q = (og_sc64wl*)ctx;
    q->W[idx] += seg * q->y;
    q->L[idx] += seg;
}

void og_sart_pass_f64(const og_geom* g, double* vol, const double* sino, double beta)
{
    og_geom64 h;
    og_geom_to64(g, &h);
    const int R = g->d.nu, ZP = g->rows, M = g->d.nx, N = g->d.ny;
    const long long P = (long long)R * ZP;
    const long long V = (long long)g->d.nx * g->d.ny * g->d.nz;
    const double thr = (double)g->d.vx * 1e-6;
    double* corr = (double*)malloc(sizeof(double) * P);
    double* W = (double*)malloc(sizeof(double) * V);
    double* L = (double*)malloc(sizeof(double) * V);
    for (int j = 0; j < g->d.nviews; ++j) {
        const double t = -(((double)j * g->d.us_rate + g->d.initial_angle) + g->d.shift_angle) * M_PI / 180.0;
        const double s = sin(t), c = cos(t);
#pragma omp parallel for schedule(dynamic, 1)
        for (int v = 0; v < ZP; ++v)
            for (int u = 0; u < R; ++u) {
                double len;
                const double sum = og_traverse64(&h, s, c, u, v, NULL, NULL, vol, &len);
                const long long p = (long long)v * R + u;
                corr[p] = (len < thr) ? 0.0 : (sino[P * j + p] - sum) / len;
            }
        memset(W, 0, sizeof(double) * V);
        memset(L, 0, sizeof(double) * V);
        for (int v = 0; v < ZP; ++v)
            for (int u = 0; u < R; ++u) {
                og_sc64wl q = {W, L, corr[(long long)v * R + u]};
                double len;
                og_traverse64(&h, s, c, u, v, og_scatter64wl, &q, NULL, &len);
            }
#pragma omp parallel for schedule(static)
        for (long long q = 0; q < V; ++q) {
            const int i = (int)(q % M), jj = (int)((q / M) % N);
            if (og_fov_masked(g, i, jj)) continue;
            if (L[q] < thr) continue;
            vol[q] += beta * W[q] / L[q];
        }
    }
    free(corr); free(W); free(L);
}

/* ------------------------------------------------------------------------ */
/* FGP TV prox, 7-array form (V63/kernel_FGP_Denoise_GPUx7.cu:2-88,         */
/* driver V63/host_FGP_Denoise_GPUx7.c:1-111).  Duals are zero-padded:      */
/* r: Z*N*(M+1), s: Z*(N+1)*M, t: (Z+1)*N*M.                                */
/* ------------------------------------------------------------------------ */
#define OG_FGP_BODY(T, SQRT, FMAX)                                                                   \
    const long long V = (long long)M * N * Z, MN = (long long)M * N;                                 \
    const long long nr = (long long)Z * N * (M + 1), ns = (long long)Z * (N + 1) * M,                \
                    nt = (long long)(Z + 1) * N * M;                                                 \
    T* r = (T*)calloc(nr, sizeof(T)); T* o = (T*)calloc(nr, sizeof(T));                              \
    T* sd = (T*)calloc(ns, sizeof(T)); T* p = (T*)calloc(ns, sizeof(T));                             \
    T* td = (T*)calloc(nt, sizeof(T)); T* q = (T*)calloc(nt, sizeof(T));                             \
    T* L = (T*)calloc(V, sizeof(T));                                                                 \
    T t_k_1 = 1, t_k;                                                                                \
    const T alpha12 = (T)1 / (lambda * (T)12);                                                       \
    for (int it = 0; it <= iters; ++it) {                                                            \
        const int last = (it == iters);                                                              \
        const T* R_ = last ? o : r; const T* S_ = last ? p : sd; const T* T_ = last ? q : td;        \
        T* dst = last ? out : L;                                                                     \
        if (!last) t_k = ((T)1 + SQRT((T)1 + (T)4 * t_k_1 * t_k_1)) / (T)2;                           \
        _Pragma("omp parallel for collapse(2) schedule(static)")                                     \
        for (int z = 0; z < Z; ++z)                                                                  \
            for (int y = 0; y < N; ++y)                                                              \
                for (int x = 0; x < M; ++x) {                                                        \
                    const long long i = x + (long long)y * M + (long long)z * MN;                    \
                    const long long ir = (x + 1) + (long long)y * (M + 1) + (long long)z * (M + 1) * N; \
                    const long long is = x + (long long)(y + 1) * M + (long long)z * M * (N + 1);    \
                    const long long iT = x + (long long)y * M + (long long)(z + 1) * MN;             \
                    const T tl = (R_[ir] - R_[ir - 1]) + (S_[is] - S_[is - M]) + (T_[iT] - T_[iT - MN]); \
                    dst[i] = f[i] - lambda * tl;                                                     \
                }                                                                                    \
        if (last) break;                                                                             \
        _Pragma("omp parallel for collapse(2) schedule(static)")                                     \
        for (int z = 0; z < Z; ++z)                                                                  \
            for (int y = 0; y < N; ++y)                                                              \
                for (int x = 0; x < M; ++x) {                                                        \
                    const long long i = x + (long long)y * M + (long long)z * MN;                    \
                    const long long ir = (x + 1) + (long long)y * (M + 1) + (long long)z * (M + 1) * N; \
                    const long long is = x + (long long)(y + 1) * M + (long long)z * M * (N + 1);    \
                    const long long iT = x + (long long)y * M + (long long)(z + 1) * MN;             \
                    T tr = r[ir], ts = sd[is], tt = td[iT];                                          \
                    if (x < M - 1) tr = tr + alpha12 * (L[i] - L[i + 1]);                            \
                    if (y < N - 1) ts = ts + alpha12 * (L[i] - L[i + M]);                            \
                    if (z < Z - 1) tt = tt + alpha12 * (L[i] - L[i + MN]);                           \
                    const T rst = SQRT(tr * tr + ts * ts + tt * tt);                                 \
                    if (x < M - 1) {                                                                 \
                        const T on = tr / FMAX((T)1, rst);                                           \
                        r[ir] = on + (t_k_1 - (T)1) / t_k * (on - o[ir]);                            \
                        o[ir] = on;                                                                  \
                    }                                                                                \
                    if (y < N - 1) {                                                                 \
                        const T pn = ts / FMAX((T)1, rst);                                           \
                        sd[is] = pn + (t_k_1 - (T)1) / t_k * (pn - p[is]);                           \
                        p[is] = pn;                                                                  \
                    }                                                                                \
                    if (z < Z - 1) {                                                                 \
                        const T qn = tt / FMAX((T)1, rst);                                           \
                        td[iT] = qn + (t_k_1 - (T)1) / t_k * (qn - q[iT]);                           \
                        q[iT] = qn;                                                                  \
                    }                                                                                \
                }                                                                                    \
        t_k_1 = t_k;                                                                                 \
    }                                                                                                \
    free(r); free(o); free(sd); free(p); free(td); free(q); free(L);

void og_fgp(int M, int N, int Z, const float* f, float lambda, int iters, float* out)
{
    OG_FGP_BODY(float, sqrtf, fmaxf)
}

void og_fgp_f64(int M, int N, int Z, const double* f, double lambda, int iters, double* out)
{
    OG_FGP_BODY(double, sqrt, fmax)
}

/* ------------------------------------------------------------------------ */
/* objective                                                                */
/* ------------------------------------------------------------------------ */
/* TV_norm_kernel (V63/kernel_tool_functions.cu:39-65): isotropic forward
 * differences; the corner voxel (M-1,N-1,Z-1) contributes 0.  The reference
 * sums the float terms in one 1024-thread block; here the sum is in double. */
double og_tv_norm(int M, int N, int Z, const float* d)
{
    const long long MN = (long long)M * N, V = MN * Z;
    float* terms = (float*)malloc(sizeof(float) * V);
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < Z; ++z)
        for (int y = 0; y < N; ++y)
            for (int x = 0; x < M; ++x) {
                const long long i = z * MN + (long long)y * M + x;
                const long long j = i + 1, k = i + M, l = i + MN;
                float tv = 0.0f;
                if (x < M - 1 && y < N - 1 && z < Z - 1)
                    tv = sqrtf((d[i] - d[j]) * (d[i] - d[j]) + (d[i] - d[k]) * (d[i] - d[k]) + (d[i] - d[l]) * (d[i] - d[l]));
                else if (x == M - 1 && y < N - 1 && z < Z - 1)
                    tv = sqrtf((d[i] - d[k]) * (d[i] - d[k]) + (d[i] - d[l]) * (d[i] - d[l]));
                else if (x < M - 1 && y == N - 1 && z < Z - 1)
                    tv = sqrtf((d[i] - d[j]) * (d[i] - d[j]) + (d[i] - d[l]) * (d[i] - d[l]));
                else if (x < M - 1 && y < N - 1 && z == Z - 1)
                    tv = sqrtf((d[i] - d[j]) * (d[i] - d[j]) + (d[i] - d[k]) * (d[i] - d[k]));
                else if (x == M - 1 && y == N - 1 && z < Z - 1)
                    tv = fabsf(d[i] - d[l]);
                else if (x == M - 1 && y < N - 1 && z == Z - 1)
                    tv = fabsf(d[i] - d[k]);
                else if (x < M - 1 && y == N - 1 && z == Z - 1)
                    tv = fabsf(d[i] - d[j]);
                terms[i] = tv;
            }
    double total = 0.0;                 /* index order, like the reference's CPU summation */
    for (long long i = 0; i < V; ++i) total += (double)terms[i];
    free(terms);
    return total;
}

/* L2_norm_kernel + summation (V63/kernel_tool_functions.cu:30-35,
 * V63/host_tool_functions.cu:18-25): sum of float (a-b)^2 terms, in double,
 * in index order. */
double og_l2_norm(const float* a, const float* b, long long n)
{
    double total = 0.0;
    for (long long i = 0; i < n; ++i) {
        const float e = (a[i] - b[i]) * (a[i] - b[i]);
        total += (double)e;
    }
    return total;
}

/* V63/main_recon.cu:375-382 */
void og_fista_momentum(long long n, float* y, float* xprev, const float* x, float t_prev, float t_k)
{
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < n; ++i) {
        y[i] = x[i] + (t_prev - 1.0f) / t_k * (x[i] - xprev[i]);
        xprev[i] = x[i];
    }
}

/* ------------------------------------------------------------------------ */
/* FDK                                                                      */
/* ------------------------------------------------------------------------ */
/* kernel_FDK_projection_adjust (V63/FDK/kernel_FDK.cu:1-14) */
void og_fdk_weight(const og_geom* g, const float* in, float* out, int nviews)
{
    const int R = g->d.nu, ZP = g->d.nv;
    const float DSO = g->d.dso, DOD = g->d.dod;
#pragma omp parallel for collapse(2) schedule(static)
    for (int w = 0; w < nviews; ++w)
        for (int v = 0; v < ZP; ++v)
            for (int u = 0; u < R; ++u) {
                const long long p = (long long)R * ZP * w + (long long)R * v + u;
                const float x1 = DSO;
                const float x2 = (g->ymin + (float)u * g->d.du) * DSO / (DSO - DOD);
                const float x3 = (g->zmin + (float)v * g->d.dv) * DSO / (DSO - DOD);
                out[p] = in[p] * DSO / sqrtf(x1 * x1 + x2 * x2 + x3 * x3);
            }
}

/* RampFiltering_GPU (V63/FDK/FFT_1d_GPU.h:241-287): zero-pad each row to
 * 2R, C2C FFT, multiply by the float filter |k|*F_step*0.5, inverse C2C,
 * take the real part / 2R.  That is a linear convolution of the row with
 * h[n] = (1/2R) sum_i H[i] cos(2 pi i n / 2R), |n| < R. */
static void og_ramp_filter_taps(const og_geom* g, float* H, int P)
{
    const float DSO = g->d.dso, DOD = g->d.dod;
    const float F_max = (float)(1.0 / 2.0 / (double)(g->d.du * DSO / (DSO - DOD)));
    const float F_step = F_max / (float)(P / 2);
    for (int i = 0; i < P; ++i) {
        const int k = (i >= P / 2) ? i - P : i;
        float h = (float)abs(k) * F_step;
        h *= 0.5f;
        H[i] = h;
    }
}

void og_ramp_kernel(const og_geom* g, double* h)
{
    const int R = g->d.nu, P = 2 * R;
    float* H = (float*)malloc(sizeof(float) * P);
    og_ramp_filter_taps(g, H, P);
    for (int n = -(R - 1); n <= R - 1; ++n) {
        double acc = 0.0;
        for (int i = 0; i < P; ++i) {
            const long long m = ((long long)i * (n < 0 ? -n : n)) % P;
            acc += (double)H[i] * cos(2.0 * M_PI * (double)m / (double)P);
        }
        h[n + R - 1] = acc / (double)P;
    }
    free(H);
}

void og_ramp_filter(const og_geom* g, const float* in, float* out, int nrows)
{
    const int R = g->d.nu;
    double* h = (double*)malloc(sizeof(double) * (2 * R - 1));
    og_ramp_kernel(g, h);
#pragma omp parallel for schedule(static)
    for (int r = 0; r < nrows; ++r) {
        const float* gi = in + (long long)r * R;
        float* go = out + (long long)r * R;
        for (int j = 0; j < R; ++j) {
            double acc = 0.0;
            for (int m = 0; m < R; ++m) acc += (double)gi[m] * h[j - m + R - 1];
            go[j] = (float)acc;
        }
    }
    free(h);
}

void og_ramp_filter_dft(const og_geom* g, const float* in, float* out, int nrows)
{
    const int R = g->d.nu, P = 2 * R;
    float* H = (float*)malloc(sizeof(float) * P);
    og_ramp_filter_taps(g, H, P);
    double* cs = (double*)malloc(sizeof(double) * P);
    double* sn = (double*)malloc(sizeof(double) * P);
    for (int i = 0; i < P; ++i) { cs[i] = cos(2.0 * M_PI * i / P); sn[i] = sin(2.0 * M_PI * i / P); }
#pragma omp parallel for schedule(static)
    for (int r = 0; r < nrows; ++r) {
        double* Gr = (double*)malloc(sizeof(double) * P);
        double* Gi = (double*)malloc(sizeof(double) * P);
        const float* gi = in + (long long)r * R;
        for (int k = 0; k < P; ++k) {
            double ar = 0, ai = 0;
            for (int m = 0; m < R; ++m) {
                const int e = (int)(((long long)k * m) % P);
                ar += gi[m] * cs[e];
                ai -= gi[m] * sn[e];
            }
            Gr[k] = ar * H[k];
            Gi[k] = ai * H[k];
        }
        for (int j = 0; j < R; ++j) {
            double acc = 0;
            for (int k = 0; k < P; ++k) {
                const int e = (int)(((long long)k * j) % P);
                acc += Gr[k] * cs[e] - Gi[k] * sn[e];
            }
            out[(long long)r * R + j] = (float)(acc / P);
        }
        free(Gr); free(Gi);
    }
    free(H); free(cs); free(sn);
}

/* kernel_FDK_reconstruction (V63/FDK/kernel_FDK.cu:16-62) */
void og_fdk_bp_view(const og_geom* g, float* vol, const float* proj, float s_th, float c_th)
{
    const int M = g->d.nx, N = g->d.ny, Z = g->d.nz, R = g->d.nu, ZP = g->d.nv;
    const float DSO = g->d.dso, DOD = g->d.dod, vx = g->d.vx, vy = g->d.vy, vz = g->d.vz;
    const float us = g->d.us_rate;
    const int nviews = g->d.nviews;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < Z; ++k)
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < M; ++i) {
                const long long idx = (long long)M * N * k + (long long)M * j + i;
                const float x = g->bx + vx * 0.5f + (float)i * vx;
                const float y = g->by + vy * 0.5f + (float)j * vy;
                const float z = g->bz + vz * 0.5f + (float)k * vz;
                const float t = x * c_th + y * s_th;
                const float s = -x * s_th + y * c_th;
                const float temp1 = DSO * DSO / ((DSO - s) * (DSO - s));
                float ksi = DSO * z / (DSO - s);
                ksi = (ksi * (DSO - DOD) / DSO - g->zmin) / g->d.dv;
                float p = DSO * t / (DSO - s);
                p = (p * (DSO - DOD) / DSO - g->ymin) / g->d.du;
                float temp2;
                if ((0 <= ksi) && (ksi + 1 < ZP) && (0 <= p) && (p + 1 < R)) {
                    const int an = (int)floorf(ksi);
                    const float an0 = ksi - (float)an;
                    const int bn = (int)floorf(p);
                    const float bn0 = p - (float)bn;
                    temp2 = (1 - an0) * (1 - bn0) * proj[R * an + bn] + (1 - an0) * bn0 * proj[R * an + bn + 1] +
                            an0 * (1 - bn0) * proj[(an + 1) * R + bn] + an0 * bn0 * proj[(an + 1) * R + bn + 1];
                } else {
                    temp2 = 0;
                }
                vol[idx] += temp1 * temp2 * (us * OG_PI_F / 180.0f) * 360.0 / (us * nviews);
            }
}

/* Reconstruction_FDK (V63/host_FDK.cpp:4-57), with the ramp as a spatial convolution. */
void og_fdk(const og_geom* g, const float* sino, float* vol)
{
    const long long P = (long long)g->d.nu * g->d.nv;
    const int nv = g->d.nviews;
    float* w = (float*)malloc(sizeof(float) * P * nv);
    float* f = (float*)malloc(sizeof(float) * P * nv);
    og_fdk_weight(g, sino, w, nv);
    og_ramp_filter(g, w, f, nv * g->d.nv);
    for (int j = 0; j < nv; ++j) {
        float s, c;
        og_view_trig(g, j, 1, &s, &c);
        og_fdk_bp_view(g, vol, f + P * j, s, c);
    }
    free(w); free(f);
}

/* ------------------------------------------------------------------------ */
/* ellipsoid phantoms (seeded parameters come from the caller)               */
/* ------------------------------------------------------------------------ */
static void og_rot(const double* e, double Rm[9])
{
    /* z-x-z Euler rotation: R = Rz(phi) Rx(theta) Rz(psi) */
    const double cp = cos(e[0]), sp = sin(e[0]), ct = cos(e[1]), st = sin(e[1]), cs = cos(e[2]), ss = sin(e[2]);
    Rm[0] = cp * cs - sp * ct * ss; Rm[1] = -cp * ss - sp * ct * cs; Rm[2] = sp * st;
    Rm[3] = sp * cs + cp * ct * ss; Rm[4] = -sp * ss + cp * ct * cs; Rm[5] = -cp * st;
    Rm[6] = st * ss;                Rm[7] = st * cs;                 Rm[8] = ct;
}

/* Each voxel centre adds the attenuation of every ellipsoid that contains it,
 * in parameter order.  Ellipsoids whose axis-aligned bounding box (half
 * extent sqrt(sum_b (R[a][b]*axis_b)^2) along world axis a, widened by a
 * voxel) misses the voxel's slice, row or centre are skipped: they cannot
 * contain it, so the sums are those of testing every ellipsoid. */
void og_phantom_voxelize(const og_geom* g, const double* par, int n, float* vol)
{
    const int M = g->d.nx, N = g->d.ny, Z = g->d.nz;
    og_geom64 h;
    og_geom_to64(g, &h);
    double* Rm = (double*)malloc(sizeof(double) * 9 * (n > 0 ? n : 1));
    double* ext = (double*)malloc(sizeof(double) * 3 * (n > 0 ? n : 1));
    const double pad[3] = {h.vx, h.vy, h.vz};
    for (int e = 0; e < n; ++e) {
        og_rot(par + 10 * e + 6, Rm + 9 * e);
        for (int a = 0; a < 3; ++a) {
            double s2 = 0.0;
            for (int b = 0; b < 3; ++b) {
                const double t = Rm[9 * e + 3 * a + b] * par[10 * e + 3 + b];
                s2 += t * t;
            }
            ext[3 * e + a] = sqrt(s2) * (1.0 + 1e-9) + pad[a];
        }
    }
#pragma omp parallel
    {
        int* in_k = (int*)malloc(sizeof(int) * (n > 0 ? n : 1));
        int* in_kj = (int*)malloc(sizeof(int) * (n > 0 ? n : 1));
#pragma omp for schedule(dynamic, 1)
        for (int k = 0; k < Z; ++k) {
            const double pz = h.bz + h.vz * (k + 0.5);
            int nk = 0;
            for (int e = 0; e < n; ++e)
                if (fabs(pz - par[10 * e + 2]) <= ext[3 * e + 2]) in_k[nk++] = e;
            for (int j = 0; j < N; ++j) {
                const double py = h.by + h.vy * (j + 0.5);
                int nkj = 0;
                for (int t = 0; t < nk; ++t)
                    if (fabs(py - par[10 * in_k[t] + 1]) <= ext[3 * in_k[t] + 1]) in_kj[nkj++] = in_k[t];
                for (int i = 0; i < M; ++i) {
                    const double p[3] = {h.bx + h.vx * (i + 0.5), py, pz};
                    double acc = 0.0;
                    for (int t = 0; t < nkj; ++t) {
                        const int e = in_kj[t];
                        const double* q = par + 10 * e;
                        if (fabs(p[0] - q[0]) > ext[3 * e]) continue;
                        const double* R = Rm + 9 * e;
                        const double d[3] = {p[0] - q[0], p[1] - q[1], p[2] - q[2]};
                        double r2 = 0.0;
                        for (int a = 0; a < 3; ++a) {
                            const double l = (R[0 + a] * d[0] + R[3 + a] * d[1] + R[6 + a] * d[2]) / q[3 + a];
                            r2 += l * l;
                        }
                        if (r2 <= 1.0) acc += q[9];
                    }
                    vol[(long long)M * N * k + (long long)M * j + i] += (float)acc;
                }
            }
        }
        free(in_k);
        free(in_kj);
    }
    free(Rm);
    free(ext);
}

void og_phantom_project(const og_geom* g, const double* par, int n, double s, double c, float* out)
{
    og_geom64 h;
    og_geom_to64(g, &h);
    const int R = g->d.nu, ZP = g->rows;
#pragma omp parallel for schedule(static)
    for (int v = 0; v < ZP; ++v)
        for (int u = 0; u < R; ++u) {
            double x2[3];
            og_source64(&h, s, c, u, v, x2);
            const double pu = h.ymin + u * h.du;
            const int vr = h.ct_style == 3 ? v % h.nv : v;
            const double x1[3] = {h.dod * c - pu * s, h.dod * s + pu * c, h.zmin + vr * h.dv};
            const double D[3] = {x2[0] - x1[0], x2[1] - x1[1], x2[2] - x1[2]};
            const double dl = sqrt(D[0] * D[0] + D[1] * D[1] + D[2] * D[2]);
            double acc = 0.0;
            for (int e = 0; e < n; ++e) {
                const double* q = par + 10 * e;
                double Rm[9];
                og_rot(q + 6, Rm);
                double o[3], d[3];
                for (int a = 0; a < 3; ++a) {
                    const double w0 = x1[0] - q[0], w1 = x1[1] - q[1], w2 = x1[2] - q[2];
                    o[a] = (Rm[0 + a] * w0 + Rm[3 + a] * w1 + Rm[6 + a] * w2) / q[3 + a];
                    d[a] = (Rm[0 + a] * D[0] + Rm[3 + a] * D[1] + Rm[6 + a] * D[2]) / q[3 + a];
                }
                const double A = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                const double B = 2.0 * (o[0] * d[0] + o[1] * d[1] + o[2] * d[2]);
                const double C = o[0] * o[0] + o[1] * o[1] + o[2] * o[2] - 1.0;
                const double disc = B * B - 4.0 * A * C;
                if (disc <= 0.0) continue;
                const double sq = sqrt(disc);
                double t0 = (-B - sq) / (2.0 * A), t1 = (-B + sq) / (2.0 * A);
                if (t0 < 0.0) t0 = 0.0;
                if (t1 > 1.0) t1 = 1.0;
                if (t1 > t0) acc += q[9] * (t1 - t0) * dl;
            }
            out[(long long)v * R + u] = (float)acc;
        }
}

/* ------------------------------------------------------------------------ */
/* Gather SART backprojection with the projector's own alphas: the engine's  */
/* SART update (reference BP semantics: MBR candidates, FOV mask, thresholds */
/* of V63/kernel_IterativeRecon_universal.cu:626-807) with every alpha       */
/* evaluated as the Siddon projector evaluates it.  Accumulates in float in  */
/* the engine's pair order (detector column, then row).                      */
/* ------------------------------------------------------------------------ */
static void og_column_eff(const og_geom* g, float s, float c, int u, float* x1x_e, float* ix_e, float* x1y_e,
                          float* iy_e)
{
    float x2x, x2y, x2z;
    og_source(g, s, c, u, 0, &x2x, &x2y, &x2z);
    const float pu = g->ymin + (float)u * g->d.du;
    const float x1x = g->d.dod * c - pu * s, x1y = g->d.dod * s + pu * c;
    if (fabsf(x1x - x2x) < g->d.vx * 1e-6f) {
        const int iv = (int)floorf((x1x - g->bx) * g->inv_vx);
        *x1x_e = og_plane(g->d.vx, iv, g->bx) + 0.5f * g->d.vx;
        *ix_e = INFINITY;
    } else {
        *x1x_e = x1x;
        *ix_e = 1.0f / (x2x - x1x);
    }
    if (fabsf(x1y - x2y) < g->d.vy * 1e-6f) {
        const int jv = (int)floorf((x1y - g->by) * g->inv_vy);
        *x1y_e = og_plane(g->d.vy, jv, g->by) + 0.5f * g->d.vy;
        *iy_e = INFINITY;
    } else {
        *x1y_e = x1y;
        *iy_e = 1.0f / (x2y - x1y);
    }
}

static void og_row_eff(const og_geom* g, int v, float* x1z_e, float* iz_e)
{
    float x2x, x2y, x2z;
    og_source(g, 0.0f, 1.0f, 0, v, &x2x, &x2y, &x2z);
    const float x1z = og_row_z(g, v);
    if (fabsf(x1z - x2z) < g->d.vz * 1e-6f) {
        const int kv = (int)floorf((x1z - g->bz) * g->inv_vz);
        *x1z_e = og_plane(g->d.vz, kv, g->bz) + 0.5f * g->d.vz;
        *iz_e = INFINITY;
    } else {
        *x1z_e = x1z;
        *iz_e = 1.0f / (x2z - x1z);
    }
}

static float og_ray_d12(const og_geom* g, float s, float c, int u, int v)
{
    float x2x, x2y, x2z;
    og_source(g, s, c, u, v, &x2x, &x2y, &x2z);
    const float pu = g->ymin + (float)u * g->d.du;
    const float x1x = g->d.dod * c - pu * s, x1y = g->d.dod * s + pu * c, x1z = og_row_z(g, v);
    return sqrtf((x2x - x1x) * (x2x - x1x) + (x2y - x1y) * (x2y - x1y) + (x2z - x1z) * (x2z - x1z));
}

/* The engine's TBCT SART update: the TBCT semantics (FOV mask, the
 * per-voxel source exclusion of T42/...TBCT_voxel.cu:620-627 evaluated as
 * there, a source's rays summed apart and the sources added in ascending
 * order, pair threshold vx*1e-6f, update where the summed length exceeds
 * vx*1e-3 in double, :772) with the projector's own chords; a source's pairs
 * in the engine's order (detector row, then column). */
static void og_backproject_gather_tbct(const og_geom* g, float* vol, const float* corr, float beta, float s, float c)
{
    const int M = g->d.nx, N = g->d.ny, Z = g->d.nz, R = g->d.nu, ZP = g->d.nv, K = g->d.n_sources;
    const int ROWS = g->rows;
    const float vx = g->d.vx, vy = g->d.vy, vz = g->d.vz;
    const float DSO = g->d.dso, DOD = g->d.dod;
    const float inv_du = 1.0f / g->d.du, inv_dv = 1.0f / g->d.dv;
    float* col = (float*)malloc(sizeof(float) * 4 * R);
    float* row = (float*)malloc(sizeof(float) * 2 * ROWS);
    float* d12 = (float*)malloc(sizeof(float) * R * ROWS);
    for (int u = 0; u < R; ++u) og_column_eff(g, s, c, u, &col[4 * u], &col[4 * u + 1], &col[4 * u + 2], &col[4 * u + 3]);
    for (int v = 0; v < ROWS; ++v) og_row_eff(g, v, &row[2 * v], &row[2 * v + 1]);
    for (int v = 0; v < ROWS; ++v)
        for (int u = 0; u < R; ++u) d12[v * R + u] = og_ray_d12(g, s, c, u, v);
    const float thr = vx * 1e-6f;
    const double thr_upd = (double)vx * 1e-3;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < Z; ++k)
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < M; ++i) {
                if (og_fov_masked(g, i, j)) continue;
                /* source exclusion, with the reference's voxel centre */
                float cxr, cyr, czr;
                og_tb_centre(g, i, j, k, &cxr, &cyr, &czr);
                const float tc = cxr * c + cyr * s;
                const float upper = (czr + vz - g->zmin) * (DSO - DOD) / (tc - DOD) + g->zmin;
                const float lower = (czr - vz - g->zmax) * (DSO - DOD) / (tc - DOD) + g->zmax;
                /* candidate columns and, per source, rows: bounding rectangles of the corner
                 * projections, rows widened by one each side (any superset gives the same sums) */
                const float cx = g->bx + vx * 0.5f + (float)i * vx;
                const float cy = g->by + vy * 0.5f + (float)j * vy;
                const float cz = g->bz + vz * 0.5f + (float)k * vz;
                float minY = INFINITY, maxY = -INFINITY;
                for (int jj = 0; jj < 2; ++jj)
                    for (int ii = 0; ii < 2; ++ii) {
                        const float px = cx + (float)ii * vx - 0.5f * vx, py = cy + (float)jj * vy - 0.5f * vy;
                        const float t = px * c + py * s, ss = -px * s + py * c;
                        const float ou = (t - DOD) / (DSO - t) * (ss - g->srcy) + ss;
                        minY = fminf(minY, ou); maxY = fmaxf(maxY, ou);
                    }
                int u0 = (int)floorf((minY - g->ymin) * inv_du + 0.5f), u1 = (int)floorf((maxY - g->ymin) * inv_du + 0.5f);
                if ((u0 < 0 && u1 < 0) || (u0 > R - 1 && u1 > R - 1)) continue;
                u0 = u0 < 0 ? 0 : u0;
                u1 = u1 > R - 1 ? R - 1 : u1;
                const float xlo = og_plane(vx, i, g->bx), xhi = og_plane(vx, i + 1, g->bx);
                const float ylo = og_plane(vy, j, g->by), yhi = og_plane(vy, j + 1, g->by);
                const float zlo = og_plane(vz, k, g->bz), zhi = og_plane(vz, k + 1, g->bz);
                float WS = 0.0f, L = 0.0f;
                for (int src = 0; src < K; ++src) {
                    const float sz = g->zsrc0 + (float)src * g->zsrc_dz;
                    if (sz < lower || sz > upper) continue;
                    float minZ = INFINITY, maxZ = -INFINITY;
                    for (int kk = 0; kk < 2; ++kk)
                        for (int jj = 0; jj < 2; ++jj)
                            for (int ii = 0; ii < 2; ++ii) {
                                const float px = cx + (float)ii * vx - 0.5f * vx, py = cy + (float)jj * vy - 0.5f * vy;
                                const float pz = cz + (float)kk * vz - 0.5f * vz;
                                const float t = px * c + py * s;
                                const float oz = (t - DOD) / (DSO - t) * (pz - sz) + pz;
                                minZ = fminf(minZ, oz); maxZ = fmaxf(maxZ, oz);
                            }
                    int v0 = (int)floorf((minZ - g->zmin) * inv_dv + 0.5f), v1 = (int)floorf((maxZ - g->zmin) * inv_dv + 0.5f);
                    if ((v0 < 0 && v1 < 0) || (v0 > ZP - 1 && v1 > ZP - 1)) continue;
                    v0 = v0 - 1 < 0 ? 0 : v0 - 1;
                    v1 = v1 + 1 > ZP - 1 ? ZP - 1 : v1 + 1;
                    /* the band's pairs row by row (rows ascending), columns ascending within a row */
                    float ca[u1 - u0 + 1], cb[u1 - u0 + 1];
                    for (int u = u0; u <= u1; ++u) {
                        const float* ct = &col[4 * u];
                        const float ax0 = (xlo - ct[0]) * ct[1], ax1 = (xhi - ct[0]) * ct[1];
                        const float ay0 = (ylo - ct[2]) * ct[3], ay1 = (yhi - ct[2]) * ct[3];
                        ca[u - u0] = fmaxf(fminf(ax0, ax1), fminf(ay0, ay1));
                        cb[u - u0] = fminf(fmaxf(ax0, ax1), fmaxf(ay0, ay1));
                    }
                    float sw = 0.0f, sl = 0.0f;
                    for (int vr = v0; vr <= v1; ++vr) {
                        const int v = src * ZP + vr;
                        const float az0 = (zlo - row[2 * v]) * row[2 * v + 1], az1 = (zhi - row[2 * v]) * row[2 * v + 1];
                        for (int u = u0; u <= u1; ++u) {
                            const float a = ca[u - u0], b = cb[u - u0];
                            if (!(b > a)) continue;
                            const float lo = fmaxf(a, fminf(az0, az1)), hi = fminf(b, fmaxf(az0, az1));
                            const float temp = d12[v * R + u] * (hi - lo);
                            if (temp > thr) {
                                sw = sw + temp * corr[v * R + u];
                                sl = sl + temp;
                            }
                        }
                    }
                    WS = WS + sw;
                    L = L + sl;
                }
                const long long idx = (long long)M * N * k + (long long)M * j + i;
                if ((double)L > thr_upd) vol[idx] = vol[idx] + beta * WS / L;
            }
    free(col); free(row); free(d12);
}

void og_backproject_gather(const og_geom* g, float* vol, const float* corr, float beta, float s, float c)
{
    if (g->d.ct_style == 3) {
        og_backproject_gather_tbct(g, vol, corr, beta, s, c);
        return;
    }
    const int M = g->d.nx, N = g->d.ny, Z = g->d.nz, R = g->d.nu, ZP = g->rows;
    const float vx = g->d.vx, vy = g->d.vy, vz = g->d.vz;
    const float DSO = g->d.dso, DOD = g->d.dod;
    const float inv_du = 1.0f / g->d.du, inv_dv = 1.0f / g->d.dv;
    float* col = (float*)malloc(sizeof(float) * 4 * R);
    float* row = (float*)malloc(sizeof(float) * 2 * ZP);
    float* d12 = (float*)malloc(sizeof(float) * R * ZP);
    for (int u = 0; u < R; ++u) og_column_eff(g, s, c, u, &col[4 * u], &col[4 * u + 1], &col[4 * u + 2], &col[4 * u + 3]);
    for (int v = 0; v < ZP; ++v) og_row_eff(g, v, &row[2 * v], &row[2 * v + 1]);
    for (int v = 0; v < ZP; ++v)
        for (int u = 0; u < R; ++u) d12[v * R + u] = og_ray_d12(g, s, c, u, v);
    const float thr = vx * 1e-6f;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < Z; ++k)
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < M; ++i) {
                if (og_fov_masked(g, i, j)) continue;
                const float cx = g->bx + vx * 0.5f + (float)i * vx;
                const float cy = g->by + vy * 0.5f + (float)j * vy;
                const float cz = g->bz + vz * 0.5f + (float)k * vz;
                /* candidate rectangle of the reference BP (:639-706) */
                float minY = INFINITY, minZ = INFINITY, maxY = -INFINITY, maxZ = -INFINITY;
                for (int kk = 0; kk < 2; ++kk)
                    for (int jj = 0; jj < 2; ++jj)
                        for (int ii = 0; ii < 2; ++ii) {
                            const float px = cx + (float)ii * vx - 0.5f * vx;
                            const float py = cy + (float)jj * vy - 0.5f * vy;
                            const float pz = cz + (float)kk * vz - 0.5f * vz;
                            const float t = px * c + py * s, ss = -px * s + py * c;
                            const float ou = g->d.ct_style == 2 ? ss : (t - DOD) / (DSO - t) * (ss - g->srcy) + ss;
                            const float oz = g->d.ct_style == 0 ? (t - DOD) / (DSO - t) * (pz - g->srcz) + pz : cz;
                            minY = fminf(minY, ou); maxY = fmaxf(maxY, ou);
                            minZ = fminf(minZ, oz); maxZ = fmaxf(maxZ, oz);
                        }
                int u0 = (int)floorf((minY - g->ymin) * inv_du + 0.5f), u1 = (int)floorf((maxY - g->ymin) * inv_du + 0.5f);
                int v0, v1;
                if (g->d.ct_style == 0) {
                    v0 = (int)floorf((minZ - g->zmin) * inv_dv + 0.5f);
                    v1 = (int)floorf((maxZ - g->zmin) * inv_dv + 0.5f);
                } else {
                    /* rays in z planes: the rows of the cell's z span (a row on a
                     * cell plane belongs to the cell above; the centre alone can
                     * miss it when the voxel is taller than a row or the row sits
                     * on the slab's edge) */
                    v0 = (int)floorf((og_plane(vz, k, g->bz) - g->zmin) * inv_dv + 0.5f);
                    v1 = (int)floorf((og_plane(vz, k + 1, g->bz) - g->zmin) * inv_dv + 0.5f);
                }
                /* widen by one row each side before the range test: the engine's
                 * row range is any superset of the rows with a positive chord */
                v0 -= 1;
                v1 += 1;
                if ((u0 < 0 && u1 < 0) || (u0 > R - 1 && u1 > R - 1) || (v0 < 0 && v1 < 0) || (v0 > ZP - 1 && v1 > ZP - 1))
                    continue;
                v0 = v0 < 0 ? 0 : v0;
                v1 = v1 > ZP - 1 ? ZP - 1 : v1;
                u0 = u0 < 0 ? 0 : u0;
                u1 = u1 > R - 1 ? R - 1 : u1;
                const float xlo = og_plane(vx, i, g->bx), xhi = og_plane(vx, i + 1, g->bx);
                const float ylo = og_plane(vy, j, g->by), yhi = og_plane(vy, j + 1, g->by);
                const float zlo = og_plane(vz, k, g->bz), zhi = og_plane(vz, k + 1, g->bz);
                /* the pairs row by row (rows ascending), columns ascending within a row */
                float ca[u1 - u0 + 1], cb[u1 - u0 + 1];
                for (int u = u0; u <= u1; ++u) {
                    const float* ct = &col[4 * u];
                    const float ax0 = (xlo - ct[0]) * ct[1], ax1 = (xhi - ct[0]) * ct[1];
                    const float ay0 = (ylo - ct[2]) * ct[3], ay1 = (yhi - ct[2]) * ct[3];
                    ca[u - u0] = fmaxf(fminf(ax0, ax1), fminf(ay0, ay1));
                    cb[u - u0] = fminf(fmaxf(ax0, ax1), fmaxf(ay0, ay1));
                }
                float sw = 0.0f, sl = 0.0f;
                for (int v = v0; v <= v1; ++v) {
                    const float az0 = (zlo - row[2 * v]) * row[2 * v + 1], az1 = (zhi - row[2 * v]) * row[2 * v + 1];
                    for (int u = u0; u <= u1; ++u) {
                        const float a = ca[u - u0], b = cb[u - u0];
                        if (!(b > a)) continue;
                        const float lo = fmaxf(a, fminf(az0, az1)), hi = fminf(b, fmaxf(az0, az1));
                        const float temp = d12[v * R + u] * (hi - lo);
                        if (temp > thr) {
                            sw = sw + temp * corr[v * R + u];
                            sl = sl + temp;
                        }
                    }
                }
                const long long idx = (long long)M * N * k + (long long)M * j + i;
                if (!(sl < thr)) vol[idx] = vol[idx] + beta * sw / sl;
            }
    free(col); free(row); free(d12);
}

void og_sart_pass_gather(const og_geom* g, float* vol, const float* sino, float beta)
{
    const long long P = (long long)g->d.nu * g->rows;
    float* corr = (float*)malloc(sizeof(float) * P);
    for (int j = 0; j < g->d.nviews; ++j) {
        float s, c;
        og_view_trig(g, j, 0, &s, &c);
        og_forward_view(g, vol, s, c, 1, sino + P * j, corr, 0);
        og_backproject_gather(g, vol, corr, beta, s, c);
    }
    free(corr);
}

/* ------------------------------------------------------------------------ */
/* z-slab SART of the multi-GPU build                                       */
/* (V63/host_IterativeRecon_CBCT_multiGPU.c:1-161)                          */
/* ------------------------------------------------------------------------ */
void og_forward_partial(const og_geom* g, const float* vol, float s, float c, float* wsum, float* lsum)
{
    const int R = g->d.nu, ZP = g->rows;
#pragma omp parallel for schedule(dynamic, 1)
    for (int v = 0; v < ZP; ++v)
        for (int u = 0; u < R; ++u) {
            float len = 0.0f, sum = 0.0f;
            if (v >= g->row_lo && v < g->row_hi) sum = og_fp_ray(g, vol, s, c, u, v, 0, &len, NULL, NULL);
            wsum[(long long)v * R + u] = sum;                 /* multiGPU.cu:1146-1147 */
            lsum[(long long)v * R + u] = len;
        }
}

void og_combine_partials(const og_geom* g, int n_parts, const float* wsum, const float* lsum, const float* b,
                         float* corr)
{
    const long long P = (long long)g->d.nu * g->rows;
    /* V63's kernel_divide_proj zeroes below volumn_z*1e-6f, T42's below
     * volumn_z*1e-3f (T42/voxel/kernel_IterativeRecon_TBCT_voxel_multiGPU.cu:14) */
    const float thr = g->d.ct_style == 3 ? g->d.vz * 1e-3f : g->d.vz * 1e-6f;
    for (long long p = 0; p < P; ++p) {
        float w = 0.0f, l = 0.0f;                              /* memset, multiGPU.c:82-83 */
        for (int i = 0; i < n_parts; ++i) {                    /* kernel_add_proj, multiGPU.cu:1-5 */
            w = w + wsum[(long long)i * P + p];
            l = l + lsum[(long long)i * P + p];
        }
        corr[p] = l < thr ? 0.0f : (b[p] - w) * 1.0f / l;      /* kernel_divide_proj, :7-19 */
    }
}

int og_sart_pass_slabs(const og_desc* d, float* vol, const float* sino, float beta, int v0, int nv, int engine)
{
    const int D = d->n_slabs < 1 ? 1 : d->n_slabs;
    og_geom* gs = (og_geom*)calloc((size_t)D, sizeof(og_geom));
    for (int i = 0; i < D; ++i) {
        og_desc e = *d;
        e.n_slabs = D;
        e.slab = i;
        if (og_init(&gs[i], &e) != 0) {
            free(gs);
            return -1;
        }
    }
    const long long P = (long long)gs[0].d.nu * gs[0].rows;
    const long long Vs = (long long)gs[0].d.nx * gs[0].d.ny * gs[0].d.nz;
    float* w = (float*)malloc(sizeof(float) * P * D);
    float* l = (float*)malloc(sizeof(float) * P * D);
    float* corr = (float*)malloc(sizeof(float) * P);
    for (int j = v0; j < v0 + nv; ++j) {
        float s, c;
        og_view_trig(&gs[0], j, 0, &s, &c);
        for (int i = 0; i < D; ++i) og_forward_partial(&gs[i], vol + Vs * i, s, c, w + P * i, l + P * i);
        og_combine_partials(&gs[0], D, w, l, sino + P * j, corr);
        for (int i = 0; i < D; ++i) {
            if (engine) og_backproject_gather(&gs[i], vol + Vs * i, corr, beta, s, c);
            else og_backproject_ref(&gs[i], vol + Vs * i, corr, beta, s, c, 1);
        }
    }
    free(w); free(l); free(corr); free(gs);
    return 0;
}
