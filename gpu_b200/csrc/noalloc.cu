// noalloc.cu -- SART view updates that allocate no device memory.
//
// ctr_sart_views allocates its ray-record scratch (one float2 per detector
// pixel) with cudaMalloc the first time a geometry needs it.  Some callers
// cannot allow that: a host whose caching allocator has reserved the GPU's
// memory up front, or a real-time acquisition loop that must not stall on
// the device-wide synchronisation cudaMalloc/cudaFree can imply, or fail
// mid-scan when memory is short.  ctr_sart_views_noalloc runs the same two
// kernels per view but keeps the ray records in the file-scope device array
// below, which is part of the loaded module: every GPU that loads the library
// holds it (8 MiB) until the process exits.
#include <mutex>

#include "ctr_device.cuh"

namespace {

constexpr long long kNoAllocMaxRays = 1LL << 20;   // 1,048,576 detector pixels = 8 MiB of float2

// Ray records of the view being updated: the forward kernel writes one per
// detector pixel, the backprojector reads them.  Shared by every call.
static __device__ __align__(256) float2 g_noalloc_rays[kNoAllocMaxRays];

constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
// per device: the array's address and the context it was looked up in
struct Slot {
    void* addr;
    unsigned long long ctx_id;
};
Slot g_slot[kMaxDevices] = {};

// Identity of the current CUDA context (the driver's unique context id,
// through the runtime's driver entry points; nothing is linked against the
// driver library).  A context created after a device reset, or a
// non-primary context, has a new id, and the module -- with the array --
// is loaded afresh in it.  Returns false when the entry points are missing.
bool current_context_id(unsigned long long* id)
{
    typedef int (*GetCurrent)(void**);
    typedef int (*GetId)(void*, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
    });
    void* ctx = nullptr;
    return get_current && get_id && get_current(&ctx) == 0 && ctx && get_id(ctx, id) == 0;
}

// Device address of g_noalloc_rays on the current device.  In host code the
// array's name is only a stand-in; the address comes from
// cudaGetSymbolAddress, with the device current, once per device and
// context: a new context (after cudaDeviceReset, or another context made
// current) is looked up again.  Without the context id the lookup runs on
// every call.
ctr_status scratch_address(int dev, void** out)
{
    using namespace ctr;
    if (dev < 0 || dev >= kMaxDevices) return set_error(CTR_ERR_UNSUPPORTED, "device ordinal %d out of range", dev);
    unsigned long long id = 0;
    const bool have_id = current_context_id(&id);
    std::lock_guard<std::mutex> lk(g_addr_mu);
    Slot& s = g_slot[dev];
    if (!have_id || !s.addr || s.ctx_id != id) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_rays);
        if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(no-alloc ray records)");
        s.addr = p;
        s.ctx_id = have_id ? id : 0;
    }
    *out = s.addr;
    return CTR_OK;
}

}  // namespace

using namespace ctr;

extern "C" ctr_status ctr_sart_views_noalloc(const ctr_geometry* geom, void* vol, ctr_dtype vdt, const void* sino,
                                             ctr_dtype sdt, float beta, unsigned flags, uint32_t seed,
                                             int view_begin, int view_count, void* stream)
{
    clear_error();
    if (!geom || !vol || !sino) return set_error(CTR_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!dtype_ok(vdt) || !dtype_ok(sdt)) return set_error(CTR_ERR_INVALID_ARGUMENT, "unknown dtype");
    if (!std::isfinite(beta)) return set_error(CTR_ERR_INVALID_ARGUMENT, "beta must be finite");
    if (flags & CTR_SART_TILED)   // the tiled copy is a geometry workspace, which this entry point does not allocate
        return set_error(CTR_ERR_INVALID_ARGUMENT, "CTR_SART_TILED needs a workspace; use ctr_sart_views");
    const Geometry* g = reinterpret_cast<const Geometry*>(geom);
    if (view_begin < 0 || view_count < 0 || (long long)view_begin + view_count > g->desc.n_views)
        return set_error(CTR_ERR_INVALID_ARGUMENT, "view range [%d, %d) outside [0, %d)", view_begin,
                         view_begin + view_count, g->desc.n_views);
    const long long P = g->npix();
    if (P > kNoAllocMaxRays)
        return set_error(CTR_ERR_INVALID_ARGUMENT,
                         "detector of %lld pixels exceeds the allocation-free limit of %lld pixels (8 MiB of ray "
                         "records); use ctr_sart_views",
                         P, kNoAllocMaxRays);
    int dev = -1;
    const cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
    if (dev != g->device)
        return set_error(CTR_ERR_INVALID_ARGUMENT, "geometry lives on device %d but device %d is current", g->device, dev);
    void* rays = nullptr;
    CTR_TRY(scratch_address(dev, &rays));
    const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    for (int j = view_begin; j < view_begin + view_count; ++j) {
        FpArgs a{};
        a.vol = vol; a.vol_dtype = vdt; a.view0 = j; a.nview = 1; a.kind = FP_SART;
        a.out = rays; a.b = (const char*)sino + (size_t)j * P * dtype_size(sdt); a.b_dtype = sdt;
        CTR_TRY(launch_forward(*g, a, st, nullptr));
        BpArgs b{};
        b.vol = vol; b.vol_dtype = vdt; b.rays = rays; b.view0 = j; b.nview = 1; b.sart = 1;
        b.flags = flags; b.beta = beta; b.seed = seed * 0x9E3779B9u + (uint32_t)j;
        CTR_TRY(launch_backproject(*g, b, st));
    }
    return CTR_OK;
}
