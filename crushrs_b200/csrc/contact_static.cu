// contact_static.cu — crush_contact_apply_static, the penalty-contact call
// that allocates nothing.
//
// Its scratch is one fixed-size record in static device memory of this
// library (one copy per CUDA context, created when the module loads in that
// context). The host resolves the record's address with
// cudaGetSymbolAddress on the first call in a context and caches it per
// device together with the context's unique id; a call from another context
// on that device (a driver-API context, or the primary context recreated
// after cudaDeviceReset) resolves it again. After that a call is argument
// checks and six kernel launches on the caller's stream: no device or host
// allocation, no copy, no synchronisation.
#include <cuda.h>  // CUcontext and CUresult only: the driver calls go through cudaGetDriverEntryPoint

#include <cmath>
#include <mutex>

#include "crush.h"
#include "host/errors.hpp"
#include "kernels.cuh"

using namespace crush;

namespace {

// The scratch record, as raw bytes aligned for its f64 and FaceGeo fields.
static __device__ __align__(256) unsigned char g_contact_scratch[sizeof(StaticContactScratch)];

constexpr int MAX_DEVICES = 64;

// Per device: the id of the context whose record address is cached, and the
// address (static storage: starts empty).
struct ScratchCache {
    std::mutex lock;
    unsigned long long ctx_id[MAX_DEVICES];
    void* addr[MAX_DEVICES];
};
ScratchCache g_cache;

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

// The unique id of the current CUDA context (ids are never reused within a
// process, unlike context handles); false when no context is current or the
// driver lacks the calls. The driver entry points are looked up once.
bool current_context_id(unsigned long long* id) {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(f);
        cudaGetLastError();
    });
    if (!get_current || !get_id) return false;
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
    return get_id(ctx, id) == CUDA_SUCCESS;
}

// The scratch record's device address in the current context of device `dev`.
bool scratch_address(int dev, void** out) {
    unsigned long long id = 0;
    bool have_id = current_context_id(&id);
    std::lock_guard<std::mutex> g(g_cache.lock);
    if (have_id && dev < MAX_DEVICES && g_cache.addr[dev] && g_cache.ctx_id[dev] == id) {
        *out = g_cache.addr[dev];
        return true;
    }
    // First call in this context: resolve the address (this can load the
    // library's kernels into the context, and makes the device's primary
    // context current when none was).
    void* addr = nullptr;
    if (cudaGetSymbolAddress(&addr, g_contact_scratch) != cudaSuccess || !addr) {
        cudaGetLastError();
        return false;
    }
    if (!have_id) have_id = current_context_id(&id);
    if (have_id && dev < MAX_DEVICES) {
        g_cache.ctx_id[dev] = id;
        g_cache.addr[dev] = addr;
    }
    *out = addr;
    return true;
}

}  // namespace

extern "C" int crush_contact_apply_static(int64_t n_model_nodes, const double* positions_device, const double* u_device,
                                          const double* masses_device, int64_t n_nodes, const uint32_t* nodes_device,
                                          const double* node_scale_device, int64_t n_faces, const uint32_t* faces_device,
                                          double stiffness, double max_distance, double dt, double* f_accum_device,
                                          crush_contact_stats* stats_device, void* stream) {
    if (n_nodes < 0 || n_faces < 0) return fail_literal(CRUSH_ERR_INVALID, "crush_contact_apply_static: negative size");
    if (n_nodes > STATIC_MAX_NODES)
        return fail_literal(CRUSH_ERR_INVALID,
                            "crush_contact_apply_static: more than CRUSH_STATIC_MAX_NODES (16384) primary nodes; use crush_contact_apply");
    if (n_faces > STATIC_MAX_FACES)
        return fail_literal(CRUSH_ERR_INVALID,
                            "crush_contact_apply_static: more than CRUSH_STATIC_MAX_FACES (16384) faces; use crush_contact_apply");
    if (n_model_nodes <= 0 || n_model_nodes > 0xffffffffll)
        return fail_literal(CRUSH_ERR_INVALID, "crush_contact_apply_static: n_model_nodes must be in 1..2^32-1");
    if (!positions_device || !u_device || !masses_device || !f_accum_device || (n_nodes > 0 && !nodes_device) ||
        (n_faces > 0 && !faces_device))
        return fail_literal(CRUSH_ERR_INVALID, "crush_contact_apply_static: null device pointer");
    if (!(dt > 0.0) || !std::isfinite(dt) || !(stiffness >= 0.0) || !(max_distance >= 0.0) || !std::isfinite(max_distance))
        return fail_literal(CRUSH_ERR_INVALID,
                            "crush_contact_apply_static: needs dt > 0, stiffness >= 0 and a finite max_distance >= 0");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return fail_literal(CRUSH_ERR_CUDA, "crush_contact_apply_static: no current CUDA device");
    }
    void* addr = nullptr;
    if (!scratch_address(dev, &addr))
        return fail_literal(CRUSH_ERR_CUDA, "crush_contact_apply_static: cannot resolve the scratch address on this device");
    launch_contact_static(static_cast<cudaStream_t>(stream), static_cast<StaticContactScratch*>(addr), n_model_nodes, positions_device,
                          u_device, masses_device, n_nodes, nodes_device, node_scale_device, n_faces, faces_device, stiffness,
                          max_distance, dt, f_accum_device, stats_device ? &stats_device->penetration_count : nullptr,
                          stats_device ? &stats_device->max_penetration : nullptr, stats_device ? &stats_device->status : nullptr);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_literal(CRUSH_ERR_CUDA, "crush_contact_apply_static: kernel launch failed");
    return CRUSH_OK;
}
