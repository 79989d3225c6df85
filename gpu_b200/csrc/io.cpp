// io.cpp -- the reference driver's file formats (V63/main_recon.cu:197-266,
// 434-477): per-view projection files "View_%.02f.dat", raw little-endian
// float volumes (.recon / .dat), and the objective history of doubles
// [TV, fidelity, objective] per iteration, with the reference's file names.
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ctr_internal.h"

using namespace ctr;

namespace {

// V63/main_recon.cu:203-209: the angle in the file name of view j
float file_angle(int j, float us_rate, float initial_angle, int tomo, int n_views)
{
    float a = float(j * us_rate + initial_angle);
    if (tomo == 1 && j >= n_views / 2) a = 180 + (j - n_views / 2) * us_rate + initial_angle;
    if (a < 0) a = a + 360;
    return a;
}

ctr_status fmt(char* out, size_t n, const std::string& s)
{
    if (!out || n == 0) return set_error(CTR_ERR_INVALID_ARGUMENT, "output buffer is NULL");
    if (s.size() + 1 > n) return set_error(CTR_ERR_INVALID_ARGUMENT, "output buffer of %zu bytes too small", n);
    memcpy(out, s.c_str(), s.size() + 1);
    return CTR_OK;
}

std::string join(const char* dir, const char* name)
{
    std::string p = dir ? dir : "";
    if (!p.empty() && p.back() != '/') p += '/';
    return p + name;
}

}  // namespace

extern "C" ctr_status ctr_io_view_filename(char* out, size_t n, int view, float us_rate, float initial_angle,
                                           int tomo, int n_views)
{
    clear_error();
    char buf[64];
    snprintf(buf, sizeof(buf), "View_%.02f.dat", file_angle(view, us_rate, initial_angle, tomo, n_views));
    return fmt(out, n, buf);
}

extern "C" ctr_status ctr_io_recon_filename(char* out, size_t n, const char* object, int nx, int ny, int nz,
                                            float voxel_um, int n_views, float initial_angle, float end_angle,
                                            float lambda_tv, float lambda_l1, float lip, int iteration)
{
    clear_error();
    if (!object) return set_error(CTR_ERR_INVALID_ARGUMENT, "object name is NULL");
    char buf[512];
    if (iteration < 0)   // the file rewritten every iteration, V63/main_recon.cu:438
        snprintf(buf, sizeof(buf), "%s_%d_%d_%d_%.0fum_new_view_%d_(%.0f,%.0f)_TV_%.2f_L1_%.2f_Lip_%.2f.recon", object,
                 nx, ny, nz, voxel_um, n_views, initial_angle, end_angle, lambda_tv, lambda_l1, lip);
    else                 // the numbered copy, V63/main_recon.cu:452
        snprintf(buf, sizeof(buf), "%s_%d_%d_%d_%.0fum_iterative_%d_view_%d_(%.0f,%.0f)_TV_%.2f_L1_%.2f_Lip_%.2f.recon",
                 object, nx, ny, nz, voxel_um, iteration, n_views, initial_angle, end_angle, lambda_tv, lambda_l1, lip);
    return fmt(out, n, buf);
}

extern "C" ctr_status ctr_io_objective_filename(char* out, size_t n, const char* object, int n_views,
                                                float initial_angle, float end_angle, float lambda_tv, float lip)
{
    clear_error();
    if (!object) return set_error(CTR_ERR_INVALID_ARGUMENT, "object name is NULL");
    char buf[512];
    snprintf(buf, sizeof(buf), "object_func_%s_view_%d_(%.0f,%.0f)_TV_%.2f_Lip_%.2f.bin", object, n_views,
             initial_angle, end_angle, lambda_tv, lip);   // V63/main_recon.cu:468
    return fmt(out, n, buf);
}

extern "C" ctr_status ctr_io_write_raw(const char* path, const void* data, size_t bytes)
{
    clear_error();
    if (!path || (!data && bytes)) return set_error(CTR_ERR_INVALID_ARGUMENT, "NULL argument");
    FILE* f = fopen(path, "wb");
    if (!f) return set_error(CTR_ERR_IO, "cannot open %s for writing: %s", path, strerror(errno));
    const bool ok = bytes == 0 || fwrite(data, 1, bytes, f) == bytes;
    const bool closed = fclose(f) == 0;
    if (!ok || !closed) return set_error(CTR_ERR_IO, "short write to %s", path);
    return CTR_OK;
}

extern "C" ctr_status ctr_io_read_raw(const char* path, void* data, size_t bytes, size_t offset)
{
    clear_error();
    if (!path || (!data && bytes)) return set_error(CTR_ERR_INVALID_ARGUMENT, "NULL argument");
    FILE* f = fopen(path, "rb");
    if (!f) return set_error(CTR_ERR_IO, "cannot open %s: %s", path, strerror(errno));
    bool ok = fseek(f, (long)offset, SEEK_SET) == 0;
    ok = ok && (bytes == 0 || fread(data, 1, bytes, f) == bytes);
    fclose(f);
    if (!ok) return set_error(CTR_ERR_IO, "%s holds fewer than %zu bytes after offset %zu", path, bytes, offset);
    return CTR_OK;
}

// V63/main_recon.cu:201-224: every view from dir/View_<angle>.dat, skipping
// row_offset detector rows at the start of each file (the reference's fseek).
extern "C" ctr_status ctr_io_read_views(const char* dir, int nu, int nv, int n_views, float us_rate,
                                        float initial_angle, int tomo, int row_offset, float* h_proj)
{
    clear_error();
    if (!h_proj || nu <= 0 || nv <= 0 || n_views <= 0 || row_offset < 0)
        return set_error(CTR_ERR_INVALID_ARGUMENT, "bad arguments");
    const size_t per = (size_t)nu * nv;
    for (int j = 0; j < n_views; ++j) {
        char name[64];
        CTR_TRY(ctr_io_view_filename(name, sizeof(name), j, us_rate, initial_angle, tomo, n_views));
        const std::string p = join(dir, name);
        CTR_TRY(ctr_io_read_raw(p.c_str(), h_proj + per * j, per * sizeof(float), sizeof(float) * (size_t)nu * row_offset));
    }
    return CTR_OK;
}

extern "C" ctr_status ctr_io_write_views(const char* dir, int nu, int nv, int n_views, float us_rate,
                                         float initial_angle, int tomo, const float* h_proj)
{
    clear_error();
    if (!h_proj || nu <= 0 || nv <= 0 || n_views <= 0) return set_error(CTR_ERR_INVALID_ARGUMENT, "bad arguments");
    const size_t per = (size_t)nu * nv;
    for (int j = 0; j < n_views; ++j) {
        char name[64];
        CTR_TRY(ctr_io_view_filename(name, sizeof(name), j, us_rate, initial_angle, tomo, n_views));
        const std::string p = join(dir, name);
        CTR_TRY(ctr_io_write_raw(p.c_str(), h_proj + per * j, per * sizeof(float)));
    }
    return CTR_OK;
}
