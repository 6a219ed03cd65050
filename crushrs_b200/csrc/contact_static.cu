// contact_static.cu — crush_contact_apply_static, the penalty-contact call
// that allocates nothing.
//
// Its scratch is one fixed-size record in static device memory of this
// library (one copy per device, created when the module loads on that
// device). The host resolves the record's address once per device with
// cudaGetSymbolAddress and caches it; after that a call is argument checks
// and six kernel launches on the caller's stream: no device or host
// allocation, no copy, no synchronisation.
#include <atomic>
#include <cmath>

#include "crush.h"
#include "host/errors.hpp"
#include "kernels.cuh"

using namespace crush;

namespace {

// The scratch record, as raw bytes aligned for its f64 and FaceGeo fields.
static __device__ __align__(256) unsigned char g_contact_scratch[sizeof(StaticContactScratch)];

constexpr int MAX_DEVICES = 64;
std::atomic<void*> g_scratch_addr[MAX_DEVICES];  // static storage: starts null

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
    void* addr = dev < MAX_DEVICES ? g_scratch_addr[dev].load(std::memory_order_acquire) : nullptr;
    if (!addr) {
        // First call on this device: resolve the record's address (this can
        // load the library's kernels onto the device).
        if (cudaGetSymbolAddress(&addr, g_contact_scratch) != cudaSuccess || !addr) {
            cudaGetLastError();
            return fail_literal(CRUSH_ERR_CUDA, "crush_contact_apply_static: cannot resolve the scratch address on this device");
        }
        if (dev < MAX_DEVICES) g_scratch_addr[dev].store(addr, std::memory_order_release);
    }
    launch_contact_static(static_cast<cudaStream_t>(stream), static_cast<StaticContactScratch*>(addr), n_model_nodes, positions_device,
                          u_device, masses_device, n_nodes, nodes_device, node_scale_device, n_faces, faces_device, stiffness,
                          max_distance, dt, f_accum_device, stats_device ? &stats_device->penetration_count : nullptr,
                          stats_device ? &stats_device->max_penetration : nullptr, stats_device ? &stats_device->status : nullptr);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_literal(CRUSH_ERR_CUDA, "crush_contact_apply_static: kernel launch failed");
    return CRUSH_OK;
}
