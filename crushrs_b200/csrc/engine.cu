// engine.cu — the engine context and the C ABI of include/crush.h.
//
// A context holds one or many crash models ("slots") resident on one GPU.
// Host side (C++17): validates the models, concatenates them (disjoint node,
// element, face and contact ranges), builds the node incidence CSRs and the
// contact tables, owns every device buffer, and drives the explicit step
// loop (src/solver.rs:190-381) as one fixed sequence of kernels per step over
// all slots, captured into a CUDA graph one period of steps at a time. Each
// slot keeps its own control block on the device (time, step, dt, mass
// scaling, stop rules), so slots of different sizes and step sizes advance
// together and finish independently, and every slot's arithmetic is the
// arithmetic it has alone.
#include <algorithm>
#include <memory>
#include <mutex>
#include <map>
#include <unordered_map>
#include <thread>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <array>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <numeric>
#include <string>
#include <vector>
#include <new>
#include <type_traits>
#include <sys/mman.h>

#include "crush.h"
#include "host/errors.hpp"
#include "kernels.cuh"

using namespace crush;

namespace {

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t err__ = (call);                                                                \
        if (err__ != cudaSuccess) {                                                                \
            return crush::fail(err__ == cudaErrorMemoryAllocation ? CRUSH_ERR_OOM : CRUSH_ERR_CUDA, \
                               std::string(#call) + ": " + cudaGetErrorString(err__));             \
        }                                                                                          \
    } while (0)

const double INF = std::numeric_limits<double>::infinity();
constexpr int N_FORCES_SCHEDULES = 4;  // launch_forces schedules 0-3
// Step schedules the trial chooses from: (fused steps, element-kernel schedule).
struct SchedCand {
    bool fused;
    int forces;
    bool early;  // separate steps: the next step's contact forces beside this step's element forces
};
constexpr int N_CANDS = 6;
constexpr SchedCand CANDS[N_CANDS] = {{false, 2, false}, {false, 3, false}, {false, 2, true},
                                     {false, 3, true},  {true, 2, false},  {true, 1, false}};
// Without a trial (small contexts, short issues): separate passes with 8 SMs
// left to the side streams, the fastest measured on one small crash and on
// the 278k-element head-on (fused steps win only on large batches).
constexpr int DEFAULT_CAND = 0;
const unsigned long long INF_BITS = 0x7ff0000000000000ull;

// HoneycombParams::from_material with Plasticity::check (src/material.rs:116-151, :430-449).
int honeycomb_params(const crush_material& m, double knots[MAX_KNOTS][3], std::string* err) {
    const int n_curve = m.n_curve;
    const int extra = m.has_densification ? 1 : 0;
    if (m.has_densification) {
        if (m.densification[0] <= 0.0 || m.densification[1] < 0.0) { *err = "densification needs c_lock > 0 and k_lock >= 0"; return -1; }
        if (n_curve > 0 && m.curve[n_curve - 1][0] >= m.densification[0]) { *err = "densification c_lock must lie beyond the last curve knot"; return -1; }
    }
    if (n_curve != 0) {
        if (n_curve < 2 || n_curve + extra > MAX_KNOTS) { *err = "yield curve needs 2..=8 knots (one fewer with densification)"; return -1; }
        if (m.curve[0][0] != 0.0) { *err = "yield curve must start at compaction 0"; return -1; }
        for (int i = 0; i + 1 < n_curve; ++i)
            if (m.curve[i + 1][0] <= m.curve[i][0]) { *err = "yield curve compaction must be strictly increasing"; return -1; }
        for (int i = 0; i < n_curve; ++i)
            if (m.curve[i][1] <= 0.0) { *err = "yield curve stresses must be positive"; return -1; }
    }
    for (int i = 0; i < MAX_KNOTS; ++i) { knots[i][0] = INF; knots[i][1] = 0.0; knots[i][2] = 0.0; }
    int n;
    if (n_curve < 2) {
        knots[0][0] = 0.0; knots[0][1] = m.yield_stress; knots[0][2] = m.hardening;
        n = 1;
    } else {
        for (int i = 0; i < n_curve; ++i) {
            double h = (i + 1 < n_curve) ? (m.curve[i + 1][1] - m.curve[i][1]) / (m.curve[i + 1][0] - m.curve[i][0]) : knots[i - 1][2];
            knots[i][0] = m.curve[i][0]; knots[i][1] = m.curve[i][1]; knots[i][2] = h;
        }
        n = n_curve;
    }
    if (m.has_densification) {
        const double* last = knots[n - 1];
        double c_lock = m.densification[0];
        double s = last[1] + last[2] * (c_lock - last[0]);
        double h = last[2] + m.densification[1];
        knots[n][0] = c_lock; knots[n][1] = s; knots[n][2] = h;
    }
    return 0;
}

double wave_speed(const crush_material& m) {
    double e = m.youngs_modulus, v = m.poisson_ratio;
    double mm = e * (1.0 - v) / ((1.0 + v) * (1.0 - 2.0 * v));
    return std::sqrt(mm / m.density);
}

size_t next_pow2(size_t x) {
    size_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

// Contacts with fewer faces than this are searched exhaustively by a warp per
// primary node; larger ones get a hashed grid.
constexpr int64_t GRID_MIN_FACES = 256;

// Device array capacities of a context (entities of every space); the first
// add_slots call allocates them, later calls fill them further.
struct Capacity {
    long long slots = 0, nodes = 0, elems = 0, scalars = 0, parts = 0, contacts = 0, faces = 0, slaves = 0, buckets = 0, entries = 0,
              st_tabs = 0, st_ents = 0, cnodes = 0, roles = 0, vehicles = 0, vnodes = 0;
};

// The capacities a reservation asks for, or at least `need`.
Capacity capacity_for(const crush_capacity* r, const Capacity& need) {
    Capacity c = need;
    if (!r) return c;
    auto up = [](long long& x, long long y) { x = std::max(x, y); };
    up(c.slots, r->slots);
    up(c.nodes, r->nodes);
    up(c.elems, r->hexes);
    // elastic (f64) elements: a road slab or two per slot, or a tenth of the elements
    up(c.scalars, std::max<long long>(256ll * r->slots, r->hexes / 10));
    up(c.contacts, r->contacts);
    up(c.faces, r->faces);
    up(c.slaves, r->primary_nodes);
    up(c.parts, 16ll * r->slots);
    up(c.vehicles, 4ll * r->slots);
    up(c.vnodes, 2ll * r->nodes);
    // hashed grids: dynamic tables (contacts of 256+ faces: twice the
    // key-box cells rounded up to a power of two, at least 1024 buckets) and
    // their entries (faces x LEVEL_CELL_BUDGET); static tables of the fixed
    // faces (a road's: about 8 cells per face, a table of twice the cells
    // rounded up to a power of two). Models that need more than this room are
    // refused with CRUSH_ERR_BUSY.
    up(c.buckets, 16ll * r->faces + 1024ll * r->contacts);
    up(c.entries, (long long)LEVEL_CELL_BUDGET * r->faces);
    up(c.st_tabs, 8ll * r->faces + 1024ll * r->contacts);
    up(c.st_ents, 16ll * r->faces + 256ll * r->contacts);
    up(c.cnodes, r->primary_nodes + 4ll * r->faces);
    up(c.roles, r->primary_nodes + 4ll * r->faces);
    return c;
}

struct Slot {
    crush_settings settings{};
    long long node0 = 0, n_nodes = 0, elem0 = 0, n_elems = 0;
    int contact0 = 0, n_contacts = 0, vehicle0 = 0, n_vehicles = 0;
    int part0 = 0, n_parts = 0;  // the slot's parts in the concatenated part numbering
    long long hc0 = 0, n_hc = 0, sc0 = 0, n_sc = 0, face0 = 0, n_faces = 0;  // honeycomb, scalar and face ranges
    double contact_dt = INF, stable = INF, dt_floor = 0.0, dt0 = 0.0;
};

// One slot's accelerometer (crush_accelerometer), node ids local to the slot.
struct HistAccel {
    std::vector<uint32_t> nodes;
    int has_frame = 0;
    uint32_t frame[3] = {0, 0, 0};
};

// Runs fn(i) for i in [0, n) on up to `hardware_concurrency` host threads
// (dynamic scheduling), each taking at least `grain` items' worth of the
// range; serial when that leaves one thread (a thread costs tens of
// microseconds to start, more than a few small items take).
template <class F>
void parallel_for(long long n, F&& fn, long long grain = 1) {
    unsigned hw = std::thread::hardware_concurrency();
    const long long T = std::min<long long>(n / std::max<long long>(grain, 1), std::min<unsigned>(hw ? hw : 1, 64));
    if (T <= 1) {
        for (long long i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<long long> next{0};
    std::vector<std::thread> th;
    th.reserve(T);
    for (long long t = 0; t < T; ++t)
        th.emplace_back([&] {
            for (long long i = next++; i < n; i = next++) fn(i);
        });
    for (auto& x : th) x.join();
}

// Host-to-device copies through two pinned staging buffers (set-up only):
// chunks are copied into pinned memory by several threads and sent by DMA
// while the next chunk is filled. Small copies go directly.
// The pinned staging buffers are kept for the process and reused by the
// next set-up (page-locking tens of MB costs milliseconds); a set-up that
// finds them in use by another thread pins its own.
struct PinnedPool {
    std::mutex m;
    char* buf[2] = {nullptr, nullptr};
    size_t cap = 0;
    bool busy = false;
};
PinnedPool g_pinned;

// Device buffers of destroyed contexts are kept for the process, per device,
// and handed to the next context's allocations of a size they fit (at most
// twice over): set-up and teardown without cudaMalloc / cudaFree, whose
// mapping work costs tens of milliseconds per context. A cudaMalloc that
// runs out of memory frees the kept buffers and retries.
struct DeviceCache {
    std::mutex m;
    std::map<int, std::multimap<size_t, void*>> free;  // device -> (bytes, buffer)
};
DeviceCache g_device_cache;

// Pinned host buffers no longer in use, kept for the process and handed to
// the next user of a size they fit (at most twice over): cudaFreeHost waits
// for the whole device, which would stall every other context's steps (a
// serving context ends every few seconds).
struct PinnedCache {
    std::mutex m;
    std::multimap<size_t, void*> free;  // (bytes, buffer)
};
PinnedCache g_pinned_cache;
// A kept pinned buffer of at least *bytes (its size written back), else a new one; null if pinning fails.
void* pinned_take(size_t* bytes) {
    {
        std::lock_guard<std::mutex> lock(g_pinned_cache.m);
        auto it = g_pinned_cache.free.lower_bound(*bytes);
        if (it != g_pinned_cache.free.end() && it->first <= 2 * *bytes + (1u << 20)) {
            void* p = it->second;
            *bytes = it->first;
            g_pinned_cache.free.erase(it);
            return p;
        }
    }
    void* p = nullptr;
    if (cudaMallocHost(&p, *bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}
// Keeps a pinned buffer whose copies have all finished.
void pinned_give(void* p, size_t bytes) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(g_pinned_cache.m);
    g_pinned_cache.free.emplace(bytes, p);
}

// A kept buffer of at least *bytes (its size written back), or null.
void* device_take(int device, size_t* bytes) {
    std::lock_guard<std::mutex> lock(g_device_cache.m);
    auto& f = g_device_cache.free[device];
    auto it = f.lower_bound(*bytes);
    if (it == f.end() || it->first > 2 * *bytes + (1u << 20)) return nullptr;
    void* p = it->second;
    *bytes = it->first;
    f.erase(it);
    return p;
}
// Keeps a buffer whose work has finished on every stream.
void device_give(int device, void* p, size_t bytes) {
    std::lock_guard<std::mutex> lock(g_device_cache.m);
    g_device_cache.free[device].emplace(bytes, p);
}
void device_release_all(int device) {
    std::lock_guard<std::mutex> lock(g_device_cache.m);
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(device);
    for (auto& kv : g_device_cache.free[device]) cudaFree(kv.second);
    g_device_cache.free[device].clear();
    cudaSetDevice(cur);
}

struct Stager {
    cudaStream_t s = nullptr;
    char* buf[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    size_t cap = 0;
    int cur = 0;
    bool pooled = false;  // the buffers are g_pinned's
    // arena mode (slots joining an open run): every copy's source is packed
    // into a pinned arena the caller keeps, so the copies do not wait for the
    // stream; arena_done is recorded after them on release
    char* arena = nullptr;
    size_t arena_cap = 0, arena_used = 0;
    cudaEvent_t arena_done = nullptr;
    static constexpr size_t DIRECT = 1 << 20;
    int init(cudaStream_t stream, size_t total) {
        s = stream;
        if (total < 8 * DIRECT) return CRUSH_OK;  // small contexts: direct copies
        cap = std::min<size_t>(total, 64u << 20);
        for (int k = 0; k < 2; ++k)
            if (cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                release();
                return CRUSH_OK;  // fall back to direct copies
            }
        {
            std::lock_guard<std::mutex> lock(g_pinned.m);
            if (!g_pinned.busy) {
                if (g_pinned.cap < cap) {
                    for (char*& b : g_pinned.buf) {
                        pinned_give(b, g_pinned.cap);  // not in use (the pool is not busy)
                        b = nullptr;
                    }
                    g_pinned.cap = 0;
                    size_t got0 = cap, got1 = cap;
                    g_pinned.buf[0] = static_cast<char*>(pinned_take(&got0));
                    g_pinned.buf[1] = static_cast<char*>(pinned_take(&got1));
                    if (g_pinned.buf[0] && g_pinned.buf[1]) {
                        g_pinned.cap = std::min(got0, got1);
                    } else {
                        for (char*& b : g_pinned.buf) {
                            pinned_give(b, b == g_pinned.buf[0] ? got0 : got1);
                            b = nullptr;
                        }
                    }
                }
                if (g_pinned.cap >= cap) {
                    g_pinned.busy = true;
                    pooled = true;
                    buf[0] = g_pinned.buf[0];
                    buf[1] = g_pinned.buf[1];
                    return CRUSH_OK;
                }
            }
        }
        for (int k = 0; k < 2; ++k) {
            size_t got = cap;
            buf[k] = static_cast<char*>(pinned_take(&got));
            if (!buf[k]) {
                release();
                return CRUSH_OK;  // fall back to direct copies
            }
        }
        return CRUSH_OK;
    }
    void use_arena(char* base, size_t cap, cudaEvent_t done) {
        arena = base;
        arena_cap = cap;
        arena_used = 0;
        arena_done = done;
    }
    int copy(void* dst, const void* src, size_t bytes) {
        if (!bytes) return CRUSH_OK;
        if (arena && arena_used + bytes <= arena_cap) {
            char* b = arena + arena_used;
            std::memcpy(b, src, bytes);
            arena_used += (bytes + 255) / 256 * 256;
            CK(cudaMemcpyAsync(dst, b, bytes, cudaMemcpyHostToDevice, s));
            return CRUSH_OK;
        }
        if (!buf[0] || bytes < DIRECT) {
            CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
            return CRUSH_OK;
        }
        for (size_t off = 0; off < bytes; off += cap) {
            const size_t n = std::min(cap, bytes - off);
            CK(cudaEventSynchronize(ev[cur]));  // the buffer's previous DMA is done
            const size_t piece = (n + 15) / 16;
            char* b = buf[cur];
            const char* sp = static_cast<const char*>(src) + off;
            parallel_for(16, [&](long long k) {
                const size_t a = std::min(n, (size_t)k * piece), e = std::min(n, a + piece);
                if (e > a) std::memcpy(b + a, sp + a, e - a);
            });
            CK(cudaMemcpyAsync(static_cast<char*>(dst) + off, b, n, cudaMemcpyHostToDevice, s));
            CK(cudaEventRecord(ev[cur], s));
            cur ^= 1;
        }
        return CRUSH_OK;
    }
    void release() {
        if (arena && arena_used > 0 && arena_done) cudaEventRecord(arena_done, s);
        arena = nullptr;
        if (s && buf[0]) cudaStreamSynchronize(s);  // the staging buffers' DMA (direct copies are staged on return)
        for (int k = 0; k < 2; ++k) {
            if (buf[k] && !pooled) pinned_give(buf[k], cap);
            if (ev[k]) cudaEventDestroy(ev[k]);
            buf[k] = nullptr;
            ev[k] = nullptr;
        }
        if (pooled) {
            std::lock_guard<std::mutex> lock(g_pinned.m);
            g_pinned.busy = false;
            pooled = false;
        }
    }
    ~Stager() { release(); }
};

int stager_copy(Stager* st, void* dst, const void* src, size_t bytes) { return st->copy(dst, src, bytes); }

}  // namespace

struct crush_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;               // the contact search of the next step runs here, beside the forces
    cudaStream_t side2 = nullptr;              // its static-grid part, then the next step's element dt pass
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_join2 = nullptr, ev_forces = nullptr;
    cudaEvent_t ev_heavy = nullptr, ev_heavy_done = nullptr;  // the heavy-node gather beside the contact gather
    cudaEvent_t ev_gathered = nullptr;                         // the contact gather done: side2 resets the event counts
    cudaEvent_t ev_static = nullptr;                           // the static-grid entries' search done (side2)
    int* mass_flag = nullptr;                  // device: some crash scales its masses this step
    unsigned* fused_counter = nullptr;         // device: blocks of the fused pass that finished (last one ends the step)
    std::vector<void*> allocs;
    std::unordered_map<void*, size_t> alloc_bytes;  // size of every device allocation
    int64_t launches = 0;

    // sizes
    int n_slots = 0;
    std::vector<Slot> slots;
    long long n_nodes = 0, n_all = 0, n_hc = 0, stride = 0;
    std::vector<int64_t> hc_index;   // model element -> honeycomb index or -1
    std::vector<uint32_t> hc_model;  // honeycomb index -> model element
    long long n_sc = 0;              // elastic elements (the scalar f64 path)
    long long n_sc_free = 0;         // those with a node that is not fixed (listed in sc_list_d)
    long long sc_stride = 1;         // plane stride of the scalar geometry (its room)
    int n_parts = 0;                 // parts of all slots
    Capacity cap;                    // room of every entity space (device arrays)
    long long n_st_ents = 0, n_st_offs = 0, n_st_tabs = 0, n_entries = 0, n_roles = 0, n_vnodes = 0, max_vnodes = 0;
    std::vector<int> chunk_lo_h, chunk_hi_h;  // slot range of every active chunk (host copy)
    std::vector<uint32_t> sc_model;  // scalar index -> model element
    int check_steps = 5;             // common adaptive_check_steps of the slots
    bool adaptive = true;
    bool any_separation = false;

    // device arrays
    double *pos = nullptr, *u = nullptr, *v = nullptr, *v0 = nullptr, *v_half = nullptr, *f_int = nullptr, *f_ext = nullptr;
    double* f_ext_odd = nullptr;     // contact forces of odd steps (f_ext: even steps), so a step's pass can run
                                     // while the previous step's update still reads its own
    double *inv_mass = nullptr, *mass = nullptr, *added = nullptr, *lumped = nullptr, *volume = nullptr, *dt_factor = nullptr;
    double *elem_mass = nullptr, *elem_dt = nullptr, *elem_extra = nullptr;
    double *u_tmp = nullptr, *f_tmp = nullptr, *n_tmp = nullptr, *n_tmp2 = nullptr, *e_tmp = nullptr;
    uint8_t *fixed = nullptr, *eroded_all = nullptr;
    uint32_t *conn_all = nullptr, *hc_off = nullptr, *hc_slot = nullptr, *all_off = nullptr, *all_slot = nullptr;
    const uint4* hc_ell = nullptr;  // N x 8 honeycomb slots, padded rows (NodeArrays::hc_ell)
    uint32_t *node_slot = nullptr, *elem_slot = nullptr;
    int32_t* part = nullptr;
    double* mat4 = nullptr;
    int64_t* hc_index_d = nullptr;
    int64_t* sc_index_d = nullptr;
    uint32_t *sc_model_d = nullptr, *sc_off = nullptr, *sc_slot = nullptr, *sc_list_d = nullptr;
    int* setup_bad = nullptr;
    // contact, vehicle and active-table arrays at their room (ContactArrays,
    // VehicleArrays and ActiveBuild point into them)
    int *face_off_d = nullptr, *slave_off_d = nullptr, *tab_off_d = nullptr;
    long long *st_tab_off_d = nullptr, *ent_off_d = nullptr;
    uint32_t *faces_d = nullptr, *slaves_d = nullptr, *grid_faces_d = nullptr, *dyn_faces_d = nullptr, *gslaves_d = nullptr,
             *stslaves_d = nullptr, *cnode_d = nullptr, *cnode_off_d = nullptr, *slave_cn_d = nullptr, *face_cn_d = nullptr,
             *st_off_d = nullptr, *vnodes_d = nullptr;
    double *scales_d = nullptr, *stiff_d = nullptr, *md_d = nullptr, *cell_d = nullptr, *st_box_d = nullptr;
    int *brute_d = nullptr, *counts_for_stop_d = nullptr, *crole_contact_d = nullptr, *crole_slave_d = nullptr, *face_contact_d = nullptr,
        *slave_contact_d = nullptr, *contact_slot_d = nullptr, *slot_contact_off_d = nullptr, *st_entries_d = nullptr, *vslot_d = nullptr,
        *vlocal_d = nullptr, *chunk_lo_d = nullptr, *chunk_hi_d = nullptr;
    uint8_t* is_static_d = nullptr;
    long long* voff_d = nullptr;
    double *sc_geo = nullptr, *sc_mat = nullptr, *sc_corner = nullptr;
    float4 *planes = nullptr, *state = nullptr;
    float* corner = nullptr;
    MaterialF32* mats = nullptr;
    Control* ctls = nullptr;      // the run, one per slot
    Control* ctls_aux = nullptr;  // drop-in calls, one per slot
    int* slot_done = nullptr;     // per slot: done flag mirrored by the step-end kernel
    ActiveBuild ab{};             // active chunk lists of the run
    std::vector<long long> space_off_h;
    std::vector<int> done_h;

    // contact
    ContactArrays ca{};
    int n_contacts = 0;
    long long n_faces = 0, n_slaves = 0;
    std::vector<int> face_off_h, slave_off_h;
    std::vector<uint8_t> is_static_h;
    std::vector<int> tab_off_h;
    std::vector<uint8_t> is_brute_h;      // per contact: searched by one block, exhaustively
    std::vector<uint32_t> grid_slaves_h;  // entries of the other contacts (dynamic grid or none)
    std::vector<uint32_t> st_slaves_h;    // entries of the contacts with a static grid
    int slave_lanes = 32;  // lanes per primary-node contact search (autotuned)
    bool tuned = false;
    long long last_tune_step = 0;  // the open run's step of the last tuning
    double tune_ms[6] = {0, 0, 0, 0, 0, 0};

    // vehicles
    VehicleArrays va{};
    double* veh_out = nullptr;
    // crush measure: per vehicle its front nodes then its accelerometer node
    std::vector<uint32_t> crush_nodes_h;
    std::vector<size_t> crush_off_h{0};
    uint32_t* crush_nodes = nullptr;
    double* crush_ux = nullptr;
    size_t crush_cap = 0;  // room of crush_nodes / crush_ux

    // run
    bool run_open = false;
    long long host_step = 0;
    bool step_fusion = CANDS[DEFAULT_CAND].fused;  // fused full + next half step where no check or record falls between
    bool prologue_done = false;  // the last issued step was fused: the next step's contact forces and half step ran
    bool early_contact = CANDS[DEFAULT_CAND].early;  // separate steps compute the next step's contact forces beside the forces
    bool contact_done = false;   // the next step's contact forces ran beside the last issued step's element forces
    long long pen_stride = 1;    // penetration counters: two sets (even and odd steps) of this many
    int period = 20;
    int base_period = 20;            // the graph period without time histories
    // time histories (crush_history_config)
    std::vector<int> hist_steps;                 // per slot: history_steps, 0 = off
    std::vector<long long> hist_max;             // per slot: records kept
    std::vector<std::vector<HistAccel>> hist_acc;
    HistoryArrays hist{};
    bool hist_on = false;
    bool hist_ran = false;                       // a run began since the configuration
    std::vector<void*> hist_bufs;                // device buffers of `hist`
    // frames (crush_frames_config)
    std::vector<int> frame_steps;                // per slot, 0 = off
    std::vector<long long> frame_max;
    FrameArrays frames{};
    bool frames_on = false, frames_ran = false;
    std::vector<void*> frame_bufs;
    cudaGraphExec_t graph = nullptr;      // step graph of the current element-kernel schedule
    cudaGraphExec_t graphs[N_CANDS + 1] = {};  // per trial candidate (the last: schedules set by the caller)
    int cand = DEFAULT_CAND;              // the trial's choice
    int n_sms = 148;
    int forces_schedule = CANDS[DEFAULT_CAND].forces;  // launch_forces schedule (0 persistent wave, 1 block per chunk, 2/3 wave on fewer SMs)
    bool fused_contact_side = false;      // a fused step's next contact forces on the side stream (else main, after the forces)
    unsigned* forces_queue = nullptr;     // device: chunk queue of the persistent element-kernel waves
    // Slots added to an open run are set up on `setup`, beside the steps
    // issued last (the set-up writes only the new slots' ranges); the main
    // stream waits for ev_setup before its next step, and takes the
    // active-chunk table updates from pinned memory (tab_pinned, free again
    // once ev_tab has passed).
    cudaStream_t setup = nullptr;
    cudaEvent_t ev_setup = nullptr, ev_tab = nullptr;
    char* arena = nullptr;  // pinned upload arena of those set-ups (ev_arena: its last copies done)
    size_t arena_cap = 0;
    cudaEvent_t ev_arena = nullptr;
    int* tab_pinned = nullptr;
    size_t tab_pinned_cap = 0;
    int eager_periods = 0;                // graph periods launched step by step since the graphs were dropped
    bool tuning_fixed = false;            // set by crush_set_tuning / crush_set_step_fusion: no automatic re-tuning
    bool sched_trial_pending = false;     // time the schedules at the next graph launches
    double sched_ms[N_CANDS] = {};        // measured ms per step of the step graph under each candidate
    int64_t graph_launches = 0;
    bool profiling = false;
    int prof_level = 2;  // 1: events around the element-force kernel only; 2: every phase
    bool last_was_graph = false;
    std::vector<cudaEvent_t> prof_ev;
    Stager* stager = nullptr;  // set-up only: pinned staging of uploads

    ElementArrays el() const {
        ElementArrays e;
        e.n_hc = n_hc;
        e.stride = stride;
        e.planes = planes;
        e.state = state;
        e.corner = corner;
        e.mats = mats;
        e.n_all = n_all;
        e.conn_all = conn_all;
        e.dt_factor = dt_factor;
        e.elem_mass = elem_mass;
        e.eroded_all = eroded_all;
        e.elem_dt = elem_dt;
        e.elem_extra = elem_extra;
        e.elem_slot = elem_slot;
        e.act_hc = e.act_all = Active{nullptr, nullptr};
        e.n_sc = n_sc;
        e.sc_count = n_sc;
        e.sc_list = nullptr;
        e.sc_stride = sc_stride;
        e.sc_model = sc_model_d;
        e.sc_geo = sc_geo;
        e.sc_mat = sc_mat;
        e.sc_corner = sc_corner;
        e.act_sc = Active{nullptr, nullptr};
        return e;
    }
    // The run's bundles: kernels visit only the active chunks.
    ElementArrays el_run() const {
        ElementArrays e = el();
        e.act_hc = active(0);
        e.act_all = active(1);
        // A run skips the elastic elements whose nodes are all fixed (a
        // rigid road): their forces land only on fixed nodes, whose motion
        // and outputs do not depend on them. Drop-in calls compute them all.
        e.n_sc = n_sc_free;
        e.sc_list = sc_list_d;
        e.act_sc = active(8);
        return e;
    }
    NodeArrays nd_run() const {
        NodeArrays a = nd();
        a.act_node = active(2);
        return a;
    }
    ContactArrays ca_run() const {
        ContactArrays x = ca;
        x.act_slave = active(3);
        x.act_cnode = active(4);
        x.act_dynf = active(5);
        x.act_allslave = active(6);
        x.act_stslave = active(7);
        return x;
    }
    double* f_ext_of(long long step) const { return (step & 1) ? f_ext_odd : f_ext; }
    // The run's node arrays for step `step`: its contact forces and the next step's.
    NodeArrays nd_step(long long step) const {
        NodeArrays a = nd_run();
        a.f_ext = f_ext_of(step);
        a.f_ext_next = f_ext_of(step + 1);
        return a;
    }
    // The run's contact arrays for step `step`: its set of penetration counters.
    ContactArrays ca_step(long long step) const {
        ContactArrays x = ca_run();
        x.pen_count = ca.pen_count + (step & 1) * pen_stride;
        x.pen_max_bits = ca.pen_max_bits + (step & 1) * pen_stride;
        return x;
    }
    Active active(int space) const {
        if (!ab.lists) return Active{nullptr, nullptr};
        return Active{ab.lists + space_off_h[space], ab.counts + space};
    }
    NodeArrays nd() const {
        NodeArrays a;
        a.n = n_nodes;
        a.pos = pos;
        a.u = u;
        a.v = v;
        a.v_half = v_half;
        a.f_int = f_int;
        a.f_ext = f_ext;
        a.f_ext_next = f_ext_odd;
        a.inv_mass = inv_mass;
        a.mass = mass;
        a.added = added;
        a.fixed = fixed;
        a.hc_off = hc_off;
        a.hc_ell = hc_ell;
        a.hc_slot = hc_slot;
        a.all_off = all_off;
        a.all_slot = all_slot;
        a.sc_off = sc_off;
        a.sc_slot = sc_slot;
        a.node_slot = node_slot;
        a.mass_flag = mass_flag;
        a.act_node = Active{nullptr, nullptr};
        return a;
    }

    template <typename T>
    int alloc(T** p, size_t count) {
        *p = nullptr;
        if (count == 0) count = 1;
        size_t bytes = count * sizeof(T);
        void* q = device_take(device, &bytes);
        if (!q) {
            cudaError_t e = cudaMalloc(&q, bytes);
            if (e == cudaErrorMemoryAllocation) {  // memory held for reuse goes back first
                cudaGetLastError();
                device_release_all(device);
                e = cudaMalloc(&q, bytes);
            }
            if (e != cudaSuccess) {
                cudaGetLastError();
                return crush::fail(e == cudaErrorMemoryAllocation ? CRUSH_ERR_OOM : CRUSH_ERR_CUDA,
                                   std::string("cudaMalloc: ") + cudaGetErrorString(e));
            }
        }
        *p = static_cast<T*>(q);
        allocs.push_back(q);
        alloc_bytes[q] = bytes;
        return CRUSH_OK;
    }
    template <typename T>
    int upload(T** p, const T* host, size_t count) {
        int st = alloc(p, count);
        if (st != CRUSH_OK) return st;
        if (!count) return CRUSH_OK;
        if (stager) return stager_copy(stager, *p, host, count * sizeof(T));
        CK(cudaMemcpyAsync(*p, host, count * sizeof(T), cudaMemcpyHostToDevice, stream));
        return CRUSH_OK;
    }
    template <typename T>
    int upload_const(const T** p, const std::vector<T>& host) {
        T* q = nullptr;
        int st = upload(&q, host.data(), host.size());
        *p = q;
        return st;
    }
    ~crush_ctx() {
        for (cudaGraphExec_t g : graphs)
            if (g) cudaGraphExecDestroy(g);
        for (cudaEvent_t e : prof_ev) cudaEventDestroy(e);
        if (stream) cudaStreamSynchronize(stream);
        if (side) cudaStreamSynchronize(side);
        if (side2) cudaStreamSynchronize(side2);
        for (void* p : allocs) device_give(device, p, alloc_bytes[p]);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (ev_join2) cudaEventDestroy(ev_join2);
        if (ev_forces) cudaEventDestroy(ev_forces);
        if (ev_heavy) cudaEventDestroy(ev_heavy);
        if (ev_heavy_done) cudaEventDestroy(ev_heavy_done);
        if (ev_gathered) cudaEventDestroy(ev_gathered);
        if (ev_static) cudaEventDestroy(ev_static);
        if (setup) cudaStreamSynchronize(setup);
        if (ev_setup) cudaEventDestroy(ev_setup);
        if (ev_tab) cudaEventDestroy(ev_tab);
        pinned_give(tab_pinned, sizeof(int) * tab_pinned_cap);
        pinned_give(arena, arena_cap);
        if (ev_arena) cudaEventDestroy(ev_arena);
        if (setup) cudaStreamDestroy(setup);
        if (side) cudaStreamDestroy(side);
        if (side2) cudaStreamDestroy(side2);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

int check_launch(crush_ctx* c, int n = 1) {
    c->launches += n;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return crush::fail(CRUSH_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return CRUSH_OK;
}

// The step graphs (both element-kernel schedules) no longer match the
// context's launch sequence.
void drop_graphs(crush_ctx* c) {
    c->eager_periods = 0;
    for (cudaGraphExec_t& g : c->graphs) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
    c->graph = nullptr;
}

int sync(crush_ctx* c) {
    CK(cudaStreamSynchronize(c->stream));
    return CRUSH_OK;
}

// Set-up phase timing to stderr when the environment sets CRUSH_TRACE=1.
struct Trace {
    bool on = std::getenv("CRUSH_TRACE") && std::getenv("CRUSH_TRACE")[0] == '1';
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now(), t = t0;
    void mark(const char* what) {
        if (!on) return;
        auto now = std::chrono::steady_clock::now();
        std::fprintf(stderr, "[crush] %-28s %8.2f ms (total %8.2f ms)\n", what, std::chrono::duration<double, std::milli>(now - t).count(),
                     std::chrono::duration<double, std::milli>(now - t0).count());
        t = now;
    }
};

// A host array left uninitialised on allocation (large set-up arrays are
// written in full by the per-slot passes, so zeroing them first is waste,
// and their pages are first touched by those passes' threads, not by one).
// Arrays of 2 MB and more sit on 2 MB boundaries with transparent huge
// pages requested: a batched set-up writes gigabytes of them, and 4 KB page
// faults cost it more than the writes.
template <typename T>
struct Buf {
    static_assert(std::is_trivially_copyable<T>::value, "plain data only");
    static constexpr size_t HUGE_PAGE = size_t(2) << 20;
    T* p = nullptr;
    size_t n = 0;
    Buf() = default;
    explicit Buf(size_t m) { alloc(m); }
    Buf(const Buf&) = delete;
    Buf& operator=(const Buf&) = delete;
    ~Buf() { std::free(p); }
    void alloc(size_t m) {
        std::free(p);
        p = nullptr;
        size_t bytes = sizeof(T) * (m ? m : 1);
        if (bytes >= HUGE_PAGE) {
            bytes = (bytes + HUGE_PAGE - 1) / HUGE_PAGE * HUGE_PAGE;
            p = static_cast<T*>(std::aligned_alloc(HUGE_PAGE, bytes));
            if (p) madvise(p, bytes, MADV_HUGEPAGE);
        } else {
            p = static_cast<T*>(std::malloc(bytes));
        }
        if (!p) throw std::bad_alloc();
        n = m;
    }
    T* data() { return p; }
    const T* data() const { return p; }
    T& operator[](size_t i) { return p[i]; }
    const T& operator[](size_t i) const { return p[i]; }
    size_t size() const { return n; }
    bool empty() const { return n == 0; }
    T* begin() { return p; }
    T* end() { return p + n; }
    const T* begin() const { return p; }
    const T* end() const { return p + n; }
};

// Combined host arrays of the slots being added: node, element and part
// arrays start at the context's node_base, elem_base and part_base (global
// indices minus the base index them); the values stored are global.
struct Combined {
    long long node_base = 0, elem_base = 0;
    int part_base = 0;
    Buf<double> positions, v0;
    std::vector<double> mat4;
    Buf<uint32_t> hexes;
    Buf<int32_t> hex_part;
    std::vector<MaterialF32> mats;
    std::vector<crush_material> materials;
    Buf<uint8_t> fixed;
    Buf<uint32_t> node_slot, elem_slot;
};

struct SlotError {
    int code = CRUSH_OK;
    std::string msg;
    void set(int c, const std::string& m) {
        if (code == CRUSH_OK) {
            code = c;
            msg = m;
        }
    }
};

// Cheap checks of a model description (sizes and pointers).
int check_desc(const crush_model_desc* d) {
    if (!d || d->n_nodes <= 0 || !d->positions || d->n_hexes < 0 || (d->n_hexes > 0 && (!d->hexes || !d->hex_part)))
        return crush::fail(CRUSH_ERR_INVALID, "invalid model description");
    if (d->n_parts <= 0 || !d->materials) return crush::fail(CRUSH_ERR_INVALID, "model needs at least one material");
    if (d->n_fixed < 0 || (d->n_fixed > 0 && !d->fixed_nodes)) return crush::fail(CRUSH_ERR_INVALID, "invalid fixed node list");
    if (d->n_contacts < 0 || (d->n_contacts > 0 && !d->contacts)) return crush::fail(CRUSH_ERR_INVALID, "invalid contact list");
    if (d->n_vehicles < 0 || (d->n_vehicles > 0 && !d->vehicles)) return crush::fail(CRUSH_ERR_INVALID, "invalid vehicle list");
    const crush_settings& s = d->settings;
    if (!(s.dt_scale > 0.0) || s.adaptive_check_steps < 0 || !(s.hourglass >= 0.0))
        return crush::fail(CRUSH_ERR_INVALID, "invalid settings");
    return CRUSH_OK;
}

// Slot k's nodes, parts and elements into the combined arrays at its offsets.
void fill_slot(const crush_model_desc* d, int slot, const Slot& sl, int p0, Combined& cm, long long* n_hc, SlotError& err) {
    const long long N = d->n_nodes, E = d->n_hexes, n0 = sl.node0, e0 = sl.elem0;
    const long long ln0 = n0 - cm.node_base, le0 = e0 - cm.elem_base;  // positions in the combined arrays
    const int lp0 = p0 - cm.part_base;
    std::memcpy(&cm.positions[3 * ln0], d->positions, sizeof(double) * 3 * N);
    if (d->initial_velocity) std::memcpy(&cm.v0[3 * ln0], d->initial_velocity, sizeof(double) * 3 * N);
    else std::memset(&cm.v0[3 * ln0], 0, sizeof(double) * 3 * N);
    std::memset(&cm.fixed[ln0], 0, N);
    for (long long i = 0; i < N; ++i) cm.node_slot[ln0 + i] = (uint32_t)slot;
    for (int64_t i = 0; i < d->n_fixed; ++i) {
        if (d->fixed_nodes[i] >= (uint64_t)N) return err.set(CRUSH_ERR_INVALID, "fixed node out of range");
        cm.fixed[ln0 + d->fixed_nodes[i]] = 1;
    }
    for (int p = 0; p < d->n_parts; ++p) {
        const crush_material& m = d->materials[p];
        if (!(m.density > 0.0) || !(m.youngs_modulus > 0.0) || !(m.poisson_ratio >= 0.0 && m.poisson_ratio < 0.5))
            return err.set(CRUSH_ERR_INVALID, "material " + std::to_string(p) + ": needs E > 0, density > 0, 0 <= nu < 0.5");
        MaterialF32 mf;
        std::memset(&mf, 0, sizeof(mf));
        if (m.model == CRUSH_MAT_HONEYCOMB) {
            double knots[MAX_KNOTS][3];
            std::string e;
            if (honeycomb_params(m, knots, &e) != 0) return err.set(CRUSH_ERR_INVALID, "material " + std::to_string(p) + ": " + e);
            mf.youngs = (float)m.youngs_modulus;
            mf.trans = (float)m.transverse_factor;
            for (int k = 0; k < MAX_KNOTS; ++k) {
                mf.knot_c[k] = (float)knots[k][0];
                mf.knot_s[k] = (float)knots[k][1];
                mf.knot_h[k] = (float)knots[k][2];
            }
        } else if (m.model != CRUSH_MAT_ELASTIC) {
            return err.set(CRUSH_ERR_UNSUPPORTED, "unknown material model");
        }
        cm.mats[lp0 + p] = mf;
        cm.materials[lp0 + p] = m;
        const double m4[4] = {m.youngs_modulus, m.poisson_ratio, m.density, d->settings.hourglass};
        std::memcpy(&cm.mat4[4 * (size_t)(lp0 + p)], m4, sizeof(m4));
    }
    long long hc = 0;
    for (long long e = 0; e < E; ++e) {
        const int p = d->hex_part[e];
        if (p < 0 || p >= d->n_parts) return err.set(CRUSH_ERR_INVALID, "hexahedron part out of range");
        const bool honey = d->materials[p].model == CRUSH_MAT_HONEYCOMB;
        for (int i = 0; i < 8; ++i) {
            const uint64_t n = d->hexes[8 * e + i];
            if (n >= (uint64_t)N) return err.set(CRUSH_ERR_INVALID, "hexahedron node out of range");
            cm.hexes[8 * (le0 + e) + i] = (uint32_t)(n0 + n);
        }
        cm.hex_part[le0 + e] = p0 + p;
        cm.elem_slot[le0 + e] = (uint32_t)slot;
        hc += honey ? 1 : 0;
    }
    *n_hc = hc;
}

// One slot's contacts (ContactRuntime::new, src/contact.rs:48-70), with
// slot-local offsets; concatenated afterwards.
struct ContactPart {
    std::vector<int> nf, ns, tab, st;
    std::vector<uint8_t> stat, stop;
    std::vector<double> stiff, md, cell;
    std::vector<uint32_t> faces, slaves, dyn_faces, grid_faces;  // faces/slaves: global node ids; *_faces: slot-local
    std::vector<double> scales, box;  // box: 6 per contact (static key-box union, else everything)
    std::vector<uint32_t> st_off;  // per contact T+1 entries, slot-local into st_entries
    std::vector<int> st_entries;
    std::vector<uint32_t> cnode, cnode_off{0};  // contact nodes (ascending node id) and their role ranges
    std::vector<int> crole_contact, crole_slave;
    double contact_dt = INF;
};

// The geometry the broad phase needs of one face at the reference positions.
// pos holds the nodes from node_base on; q are global node ids.
void face_frame(const double* pos, long long node_base, const uint32_t* q, double x[4][3], double nr[3], double ctr[3]) {
    double e1[3], e2[3];
    for (int j = 0; j < 4; ++j)
        for (int dd = 0; dd < 3; ++dd) x[j][dd] = pos[3 * (size_t)(q[j] - node_base) + dd];
    for (int dd = 0; dd < 3; ++dd) {
        e1[dd] = x[1][dd] - x[0][dd];
        e2[dd] = x[2][dd] - x[0][dd];
    }
    nr[0] = e1[1] * e2[2] - e1[2] * e2[1];
    nr[1] = e1[2] * e2[0] - e1[0] * e2[2];
    nr[2] = e1[0] * e2[1] - e1[1] * e2[0];
    const double len = std::sqrt(nr[0] * nr[0] + nr[1] * nr[1] + nr[2] * nr[2]);
    for (int dd = 0; dd < 3; ++dd) {
        nr[dd] = len > 0.0 ? nr[dd] / len : 0.0;
        ctr[dd] = (((x[0][dd] + x[1][dd]) + x[2][dd]) + x[3][dd]) / 4.0;
    }
}

void build_contacts(const crush_model_desc* d, const Slot& sl, const Combined& cm, ContactPart& cp, SlotError& err) {
    const long long n0 = sl.node0;
    // Contact-node roles: (node, contact, sequence) sorted gives, for every
    // node, its contacts in order with its primary-node entries and the faces
    // it belongs to (the src/contact.rs:146-153 order).
    struct RoleItem {
        uint32_t node;
        int contact;
        int seq;
        int slave;  // >= 0: primary-node entry index within the contact
        int face;   // >= 0: local face index
    };
    std::vector<RoleItem> items;
    {
        size_t nf = 0, nn = 0;
        for (int k = 0; k < d->n_contacts; ++k) {
            nf += (size_t)std::max<int64_t>(d->contacts[k].n_faces, 0);
            nn += (size_t)std::max<int64_t>(d->contacts[k].n_nodes, 0);
        }
        cp.faces.reserve(4 * nf);
        cp.slaves.reserve(nn);
        cp.scales.reserve(nn);
        items.reserve(nn + 4 * nf);
    }
    int seq = 0;
    for (int k = 0; k < d->n_contacts; ++k) {
        const crush_contact& cd = d->contacts[k];
        const int kc = sl.contact0 + k;
        if (cd.n_nodes < 0 || cd.n_faces < 0 || (cd.n_nodes > 0 && !cd.nodes) || (cd.n_faces > 0 && !cd.faces))
            return err.set(CRUSH_ERR_INVALID, "invalid contact " + std::to_string(k));
        if (!(cd.max_distance >= 0.0) || !(cd.stiffness >= 0.0)) return err.set(CRUSH_ERR_INVALID, "invalid contact parameters");
        double lo[3] = {INF, INF, INF}, hi[3] = {-INF, -INF, -INF};
        bool stop = false;
        double ext = 0.0;
        const size_t face0 = cp.faces.size() / 4;
        for (int64_t f = 0; f < cd.n_faces; ++f) {
            double flo[3] = {INF, INF, INF}, fhi[3] = {-INF, -INF, -INF};
            for (int j = 0; j < 4; ++j) {
                const uint32_t nl = cd.faces[4 * f + j];
                if (nl >= (uint64_t)d->n_nodes) return err.set(CRUSH_ERR_INVALID, "contact face node out of range");
                const uint32_t n = (uint32_t)(n0 + nl);
                cp.faces.push_back(n);
                if (!cm.fixed[n - cm.node_base]) stop = true;
                for (int dd = 0; dd < 3; ++dd) {
                    const double p = cm.positions[3 * (size_t)(n - cm.node_base) + dd];
                    lo[dd] = std::fmin(lo[dd], p);
                    hi[dd] = std::fmax(hi[dd], p);
                    flo[dd] = std::fmin(flo[dd], p);
                    fhi[dd] = std::fmax(fhi[dd], p);
                }
            }
            ext = std::max(ext, std::max({fhi[0] - flo[0], fhi[1] - flo[1], fhi[2] - flo[2]}));
        }
        for (int dd = 0; dd < 3; ++dd) {
            lo[dd] += -cd.max_distance;
            hi[dd] += cd.max_distance;
        }
        int kept = 0;
        for (int64_t i = 0; i < cd.n_nodes; ++i) {
            const uint32_t nl = cd.nodes[i];
            if (nl >= (uint64_t)d->n_nodes) return err.set(CRUSH_ERR_INVALID, "contact node out of range");
            const uint32_t n = (uint32_t)(n0 + nl);
            bool inside = true;
            for (int dd = 0; dd < 3; ++dd) {
                const double p = cm.positions[3 * (size_t)(n - cm.node_base) + dd];
                if (!(p >= lo[dd] && p <= hi[dd])) inside = false;
            }
            if (!inside) continue;
            cp.slaves.push_back(n);
            cp.scales.push_back(cd.node_scale ? cd.node_scale[i] : 1.0);
            items.push_back(RoleItem{n, kc, seq++, kept, -1});
            ++kept;
        }
        for (int64_t f = 0; f < cd.n_faces; ++f)
            for (int j = 0; j < 4; ++j) items.push_back(RoleItem{(uint32_t)(n0 + cd.faces[4 * f + j]), kc, seq++, -1, (int)f});
        const double cs = ext > 0.0 ? 2.0 * ext : 1.0;  // grid cell: twice the largest face
        const bool stat = !stop && cd.n_faces > 0;
        size_t t = 0, st = 0;
        const uint32_t* fq = cp.faces.data() + 4 * face0;
        if (stat) {
            // Exact hashed grid of the fixed faces, in CSR form.
            std::vector<std::pair<uint32_t, int>> ins;  // (hash, face)
            bool ok = true;
            double box[6] = {INF, INF, INF, -INF, -INF, -INF};  // union of the key boxes
            for (int64_t f = 0; f < cd.n_faces && ok; ++f) {
                double x[4][3], nr[3], ctr[3], klo[3], khi[3];
                face_frame(cm.positions.data(), cm.node_base, fq + 4 * f, x, nr, ctr);
                face_key_box(x, nr, ctr, cd.max_distance, klo, khi);
                long long r[6];
                double cells = 1.0;
                for (int dd = 0; dd < 3; ++dd) {
                    if (!std::isfinite(klo[dd]) || !std::isfinite(khi[dd]) || std::fabs(klo[dd] / cs) > 4.0e15 ||
                        std::fabs(khi[dd] / cs) > 4.0e15) {
                        ok = false;
                        break;
                    }
                    r[2 * dd] = (long long)std::floor(klo[dd] / cs);
                    r[2 * dd + 1] = (long long)std::floor(khi[dd] / cs);
                    cells *= (double)(r[2 * dd + 1] - r[2 * dd] + 1);
                }
                if (!ok || cells > 4096.0) {
                    ok = false;
                    break;
                }
                for (int dd = 0; dd < 3; ++dd) {
                    box[dd] = std::fmin(box[dd], klo[dd]);
                    box[3 + dd] = std::fmax(box[3 + dd], khi[dd]);
                }
                for (long long kz = r[4]; kz <= r[5]; ++kz)
                    for (long long jy = r[2]; jy <= r[3]; ++jy)
                        for (long long ix = r[0]; ix <= r[1]; ++ix) ins.push_back({cell_hash(ix, jy, kz, 0), (int)f});
            }
            const uint32_t base = (uint32_t)cp.st_entries.size();
            if (ok) cp.box.insert(cp.box.end(), box, box + 6);
            if (ok) {
                st = next_pow2(std::max<size_t>(16, 2 * ins.size()));
                const size_t o0 = cp.st_off.size();
                cp.st_off.resize(o0 + st + 1, 0);
                uint32_t* off = cp.st_off.data() + o0;  // counts, then bucket starts, then the entry cursors
                for (auto& e : ins) off[(e.first & (st - 1)) + 1]++;
                for (size_t b2 = 0; b2 < st; ++b2) off[b2 + 1] += off[b2];
                cp.st_entries.resize(base + ins.size());
                for (auto& e : ins) cp.st_entries[base + off[e.first & (st - 1)]++] = e.second;  // faces ascending in a bucket
                // the cursors end at the next bucket's start: shift back, and offset by base
                for (size_t b2 = st; b2 > 0; --b2) off[b2] = base + off[b2 - 1];
                off[0] = base;
            } else {
                st = 0;
                cp.st_off.push_back(base);
            }
        } else {
            cp.st_off.push_back((uint32_t)cp.st_entries.size());
            for (int64_t f = 0; f < cd.n_faces; ++f) cp.dyn_faces.push_back((uint32_t)(face0 + f));
            if (cd.n_faces >= GRID_MIN_FACES) {
                // Hierarchical table: twice the level-0 key-box cells of the
                // faces at the reference positions, a power of two.
                size_t inserts = 0;
                for (int64_t f = 0; f < cd.n_faces; ++f) {
                    double x[4][3], nr[3], ctr[3], klo[3], khi[3];
                    face_frame(cm.positions.data(), cm.node_base, fq + 4 * f, x, nr, ctr);
                    face_key_box(x, nr, ctr, cd.max_distance, klo, khi);
                    double cells = 1.0;
                    for (int dd = 0; dd < 3; ++dd) cells *= std::floor(khi[dd] / cs) - std::floor(klo[dd] / cs) + 1.0;
                    inserts += (size_t)std::min(std::isfinite(cells) && cells > 0.0 ? cells : 0.0, (double)LEVEL_CELL_BUDGET);
                }
                t = next_pow2(std::max<size_t>(1024, 2 * inserts));
                for (int64_t f = 0; f < cd.n_faces; ++f) cp.grid_faces.push_back((uint32_t)(face0 + f));
            }
        }
        if (cp.box.size() < 6 * (cp.nf.size() + 1)) {
            const double all[6] = {-INF, -INF, -INF, INF, INF, INF};
            cp.box.insert(cp.box.end(), all, all + 6);
        }
        cp.nf.push_back((int)cd.n_faces);
        cp.ns.push_back(kept);
        cp.tab.push_back((int)t);
        cp.st.push_back((int)st);
        cp.stat.push_back(stat && st > 0 ? 1 : 0);
        cp.stop.push_back(stop ? 1 : 0);
        cp.stiff.push_back(cd.stiffness);
        cp.md.push_back(cd.max_distance);
        cp.cell.push_back(cs);
    }
    // Items were made in (contact, seq) order: a stable counting sort by node
    // gives the (node, contact, seq) order.
    {
        std::vector<uint32_t> cnt((size_t)d->n_nodes + 1, 0);
        for (const RoleItem& it : items) cnt[it.node - n0 + 1]++;
        for (size_t i = 0; i < (size_t)d->n_nodes; ++i) cnt[i + 1] += cnt[i];
        std::vector<RoleItem> sorted(items.size());
        for (const RoleItem& it : items) sorted[cnt[it.node - n0]++] = it;
        items.swap(sorted);
    }
    cp.cnode.reserve(items.size());
    cp.cnode_off.reserve(items.size() + 1);
    cp.crole_contact.reserve(items.size());
    cp.crole_slave.reserve(items.size());
    for (size_t i0 = 0; i0 < items.size();) {
        size_t i1 = i0;
        while (i1 < items.size() && items[i1].node == items[i0].node) ++i1;
        cp.cnode.push_back(items[i0].node);
        for (size_t a0 = i0; a0 < i1;) {
            size_t a1 = a0;
            while (a1 < i1 && items[a1].contact == items[a0].contact) ++a1;
            // One role per primary-node entry (or one without).
            int n_slave_roles = 0;
            for (size_t q = a0; q < a1; ++q) n_slave_roles += items[q].slave >= 0;
            int made = 0;
            for (size_t q = a0; q < a1 && made < n_slave_roles; ++q)
                if (items[q].slave >= 0) {
                    ++made;
                    cp.crole_contact.push_back(items[a0].contact);
                    cp.crole_slave.push_back(items[q].slave);
                }
            if (n_slave_roles == 0) {
                cp.crole_contact.push_back(items[a0].contact);
                cp.crole_slave.push_back(-1);
            }
            a0 = a1;
        }
        cp.cnode_off.push_back((uint32_t)cp.crole_contact.size());
        i0 = i1;
    }
}

template <typename T>
void append(std::vector<T>& dst, const std::vector<T>& src) {
    dst.insert(dst.end(), src.begin(), src.end());
}

int begin_slots(crush_ctx* c, int s0, int s1);
int search_now(crush_ctx* c);
int search_added(crush_ctx* c, int k0, long long dyn0, long long gs0, long long st0, int brute0);
static void free_bufs(crush_ctx* c, std::vector<void*>& bufs);

// Adds n_desc models as slots [c->n_slots, c->n_slots + n_desc) at the
// context's current offsets of every entity space. The first call (creating)
// allocates every device array with room for `reserve` (or exactly the
// models); a later call fails with CRUSH_ERR_BUSY, changing nothing, when
// the models do not fit that room. A slot's arrays are exactly those a
// context of the same models in the same order would hold, so its
// arithmetic is the same. A call on an open run sets the new slots up as
// run begin does (their own step 0 starts at the run's current step) and
// searches their contacts for their first step.
int add_slots(crush_ctx* c, const crush_model_desc* const* descs, int n_desc, bool creating, const crush_capacity* reserve) {
    if (n_desc <= 0 || !descs) return crush::fail(CRUSH_ERR_INVALID, "no models");
    Trace trace;
    int st;
#define TRY(x) do { st = (x); if (st != CRUSH_OK) return st; } while (0)
    const int S0 = c->n_slots;
    const long long N0 = c->n_nodes, E0 = c->n_all, H0 = c->n_hc, Q0 = c->n_sc, QF0 = c->n_sc_free;
    const int P0 = c->n_parts, K0 = c->n_contacts;
    // the contact lists' lengths before these slots (their entries follow)
    const long long dyn0 = c->ca.n_dyn_faces, gs0 = c->ca.n_grid_slaves, st0 = c->ca.n_st_slaves;
    const int brute0 = c->ca.n_brute;
    // ---- sizes and offsets of every new slot ----
    std::vector<Slot> slots(n_desc);
    long long N = 0, E = 0;
    int P = 0, K = 0;
    std::vector<int> part0(n_desc);
    for (int k = 0; k < n_desc; ++k) {
        const crush_model_desc* d = descs[k];
        TRY(check_desc(d));
        Slot& sl = slots[k];
        sl.settings = d->settings;
        sl.node0 = N0 + N;
        sl.n_nodes = d->n_nodes;
        sl.elem0 = E0 + E;
        sl.n_elems = d->n_hexes;
        sl.contact0 = K0 + K;
        sl.n_contacts = d->n_contacts;
        part0[k] = P0 + P;
        sl.part0 = P0 + P;
        sl.n_parts = d->n_parts;
        N += d->n_nodes;
        E += d->n_hexes;
        P += d->n_parts;
        K += d->n_contacts;
        if (N0 + N >= (1ll << 31) || E0 + E >= (1ll << 28)) return crush::fail(CRUSH_ERR_INVALID, "models too large for one context");
    }
    // The step schedule is shared: every slot must re-check its stable step
    // on the same cadence.
    bool adaptive = c->adaptive, any_sep = c->any_separation;
    int check_steps = c->check_steps;
    for (int k = 0; k < n_desc; ++k) {
        const crush_settings& s = descs[k]->settings;
        const bool ad = !(s.time_step > 0.0) && s.adaptive_check_steps > 0;
        const int cs = s.adaptive_check_steps > 0 ? s.adaptive_check_steps : 1;
        if (creating && k == 0) {
            adaptive = ad;
            check_steps = cs;
        } else if (ad != adaptive || (ad && cs != check_steps)) {
            return crush::fail(CRUSH_ERR_UNSUPPORTED, "models of one context must share adaptive_check_steps and time-step mode");
        }
        if (s.stop_rule == CRUSH_STOP_SEPARATION) any_sep = true;
    }
    if (!creating && (c->hist_on || c->frames_on))
        return crush::fail(CRUSH_ERR_UNSUPPORTED, "slots cannot be added to a context that records histories or frames");
    if (!creating && c->run_open && c->period > 0 && c->host_step % c->period != 0)
        return crush::fail(CRUSH_ERR_INVALID, "slots join an open run only on a step-graph boundary");
    Combined cm;
    cm.node_base = N0;
    cm.elem_base = E0;
    cm.part_base = P0;
    cm.positions.alloc(3 * N);
    cm.v0.alloc(3 * N);
    cm.fixed.alloc(N);
    cm.node_slot.alloc(N);
    cm.hexes.alloc(8 * E);
    cm.hex_part.alloc(E);
    cm.elem_slot.alloc(E);
    cm.mats.resize(P);
    cm.materials.resize(P);
    cm.mat4.resize(4 * (size_t)P);
    std::vector<SlotError> errs(n_desc);
    std::vector<long long> slot_hc(n_desc, 0);
    // per-slot passes: a thread per ~16k elements at least (a few small
    // models, as one request adds, are set up on the calling thread)
    const long long G = std::max<long long>(1, (long long)n_desc * 16384 / std::max<long long>(E, 1));
    parallel_for(n_desc, [&](long long k) { fill_slot(descs[k], S0 + (int)k, slots[k], part0[k], cm, &slot_hc[k], errs[k]); }, G);
    for (auto& e : errs)
        if (e.code != CRUSH_OK) return crush::fail(e.code, e.msg);
    trace.mark("validate + concatenate");
    auto mat_of = [&](long long e) -> const crush_material& { return cm.materials[cm.hex_part[e - E0] - P0]; };
    auto hex = [&](long long e, int i) { return cm.hexes[8 * (e - E0) + i]; };
    auto fixed_at = [&](uint32_t n) { return cm.fixed[n - N0] != 0; };
    // Honeycomb numbering (element order) and, per slot, the elastic
    // elements with a free node first, then the all-fixed ones (a run
    // lists only the first).
    std::vector<long long> slot_free(n_desc, 0);
    parallel_for(n_desc, [&](long long k) {
        const Slot& sl = slots[k];
        long long nf = 0;
        for (long long e = sl.elem0; e < sl.elem0 + sl.n_elems; ++e) {
            if (mat_of(e).model == CRUSH_MAT_HONEYCOMB) continue;
            bool all_fixed = true;
            for (int i = 0; i < 8; ++i) all_fixed = all_fixed && fixed_at(hex(e, i));
            nf += all_fixed ? 0 : 1;
        }
        slot_free[k] = nf;
    }, G);
    std::vector<long long> hc0(n_desc + 1, H0), sc0(n_desc + 1, Q0), scf0(n_desc + 1, QF0);
    for (int k = 0; k < n_desc; ++k) {
        hc0[k + 1] = hc0[k] + slot_hc[k];
        sc0[k + 1] = sc0[k] + (slots[k].n_elems - slot_hc[k]);
        scf0[k + 1] = scf0[k] + slot_free[k];
    }
    const long long H = hc0[n_desc] - H0, Q = sc0[n_desc] - Q0, QF = scf0[n_desc] - QF0;
    for (int k = 0; k < n_desc; ++k) {
        slots[k].hc0 = hc0[k];
        slots[k].n_hc = hc0[k + 1] - hc0[k];
        slots[k].sc0 = sc0[k];
        slots[k].n_sc = sc0[k + 1] - sc0[k];
    }
    if (8 * (unsigned long long)(E0 + E) >= (unsigned long long)HC_ELL_MORE)
        return crush::fail(CRUSH_ERR_INVALID, "too many hexahedra for 32-bit node incidence entries (8 x elements must stay below 2^32 - 2)");
    Buf<int64_t> hc_index(E), sc_index(E);
    Buf<uint32_t> hc_model(H), sc_model(Q), sc_list(QF);
    // Honeycomb and elastic numbering per slot (the node incidence lists are
    // built on the device from these and the connectivity).
    parallel_for(n_desc, [&](long long k) {
        const Slot& sl = slots[k];
        const long long e0 = sl.elem0;
        long long h = hc0[k], qf = sc0[k], qx = sc0[k] + slot_free[k], lf = scf0[k];
        for (long long e = e0; e < e0 + sl.n_elems; ++e)
            if (mat_of(e).model == CRUSH_MAT_HONEYCOMB) {
                hc_index[e - E0] = h;
                hc_model[h++ - H0] = (uint32_t)e;
                sc_index[e - E0] = -1;
            } else {
                hc_index[e - E0] = -1;
                bool all_fixed = true;
                for (int i = 0; i < 8; ++i) all_fixed = all_fixed && fixed_at(hex(e, i));
                const long long q = all_fixed ? qx++ : qf++;
                if (!all_fixed) sc_list[lf++ - QF0] = (uint32_t)q;
                sc_index[e - E0] = q;
                sc_model[q - Q0] = (uint32_t)e;
            }
    }, G);
    std::vector<double> sc_mat(2 * (size_t)std::max<long long>(Q, 1), 0.0);
    for (long long q = 0; q < Q; ++q) {
        const crush_material& m = mat_of(sc_model[q]);
        sc_mat[2 * q] = m.youngs_modulus;
        sc_mat[2 * q + 1] = m.poisson_ratio;
    }
    trace.mark("element numbering");

    // ---- contacts: per slot in parallel, then concatenated after the context's ----
    std::vector<ContactPart> parts(n_desc);
    parallel_for(n_desc, [&](long long k) { build_contacts(descs[k], slots[k], cm, parts[k], errs[k]); }, G);
    for (auto& e : errs)
        if (e.code != CRUSH_OK) return crush::fail(e.code, e.msg);
    trace.mark("contact runtimes per slot");
    struct Base {
        long long face, slave, ste, stoff, dyn, grid, cnode, role;
    };
    std::vector<Base> base(n_desc + 1);
    base[0] = Base{c->n_faces, c->n_slaves, c->n_st_ents, c->n_st_offs, c->ca.n_dyn_faces, c->ca.n_grid_faces, c->ca.n_cnodes, c->n_roles};
    long long tabs = 0, st_tabs = 0, ents = 0;
    for (int k = 0; k < n_desc; ++k) {
        const ContactPart& cp = parts[k];
        const Base& b0 = base[k];
        base[k + 1] = Base{b0.face + (long long)cp.faces.size() / 4, b0.slave + (long long)cp.slaves.size(),
                           b0.ste + (long long)cp.st_entries.size(), b0.stoff + (long long)cp.st_off.size(),
                           b0.dyn + (long long)cp.dyn_faces.size(), b0.grid + (long long)cp.grid_faces.size(),
                           b0.cnode + (long long)cp.cnode.size(), b0.role + (long long)cp.crole_contact.size()};
        slots[k].face0 = b0.face;
        slots[k].n_faces = (long long)cp.faces.size() / 4;
        for (size_t j = 0; j < cp.nf.size(); ++j) {
            tabs += cp.tab[j];
            st_tabs += cp.st[j];
            ents += cp.tab[j] > 0 ? (long long)cp.nf[j] * LEVEL_CELL_BUDGET : 0;
        }
    }
    const Base& tot = base[n_desc];
    if (trace.on)
        std::fprintf(stderr, "[crush] new contact tables: faces %lld, entries %lld, static-grid entries %lld, offsets %lld, contact nodes %lld, roles %lld\n",
                     tot.face - base[0].face, tot.slave - base[0].slave, tot.ste - base[0].ste, tot.stoff - base[0].stoff,
                     tot.cnode - base[0].cnode, tot.role - base[0].role);
    if (tot.face >= (1ll << 31) || tot.slave >= (1ll << 31) || tot.ste >= (1ll << 32) || tot.role >= (1ll << 32) ||
        tot.cnode >= (long long)CN_FIXED)
        return crush::fail(CRUSH_ERR_INVALID, "contacts too large for one context");
    long long n_veh = 0, n_vnodes = 0;
    for (int k = 0; k < n_desc; ++k) {
        const crush_model_desc* d = descs[k];
        const int nv = std::min(d->n_vehicles, 4);
        n_veh += nv;
        for (int v = 0; v < nv; ++v) n_vnodes += std::max<int64_t>(d->vehicles[v].n_nodes, 0);
    }
    // ---- room: allocate it (creating) or check it ----
    Capacity need;
    need.slots = S0 + n_desc;
    need.nodes = N0 + N;
    need.elems = E0 + E;
    need.scalars = Q0 + Q;
    need.parts = P0 + P;
    need.contacts = K0 + K;
    need.faces = tot.face;
    need.slaves = tot.slave;
    need.buckets = c->ca.n_buckets + tabs;
    need.entries = c->n_entries + ents;
    need.st_tabs = c->n_st_tabs + st_tabs;
    need.st_ents = tot.ste;
    need.cnodes = tot.cnode;
    need.roles = tot.role;
    need.vehicles = c->va.n_vehicles + n_veh;
    need.vnodes = c->n_vnodes + n_vnodes;
    if (creating) {
        c->cap = capacity_for(reserve, need);
    } else {
        const Capacity& cp = c->cap;
        const bool fits = need.slots <= cp.slots && need.nodes <= cp.nodes && need.elems <= cp.elems && need.scalars <= cp.scalars &&
                          need.parts <= cp.parts &&
                          need.contacts <= cp.contacts && need.faces <= cp.faces && need.slaves <= cp.slaves &&
                          need.buckets <= cp.buckets && need.entries <= cp.entries && need.st_tabs <= cp.st_tabs &&
                          need.st_ents <= cp.st_ents && need.cnodes <= cp.cnodes && need.roles <= cp.roles &&
                          need.vehicles <= cp.vehicles && need.vnodes <= cp.vnodes;
        if (!fits) return crush::fail(CRUSH_ERR_BUSY, "the models do not fit the context's reserved room");
    }
    const Capacity& cap = c->cap;
    // ---- contact arrays of the new slots (global values) ----
    std::vector<int> face_off(K + 1), slave_off(K + 1), tab_off(K + 1), counts_for_stop(K), contact_slot(K), slot_contact_off(n_desc + 1);
    std::vector<long long> st_tab_off(K + 1), ent_off(K + 1);
    // written in full by the per-slot pass below
    Buf<int> face_contact(tot.face - base[0].face), slave_contact(tot.slave - base[0].slave);
    Buf<uint32_t> faces(4 * (tot.face - base[0].face)), slaves(tot.slave - base[0].slave), dyn_faces(tot.dyn - base[0].dyn),
        grid_faces(tot.grid - base[0].grid);
    Buf<double> scales(slaves.size());
    std::vector<double> stiff(K), md(K), cell(K), st_box(6 * (size_t)std::max(K, 1));
    std::vector<uint8_t> is_static(K);
    Buf<uint32_t> st_off(tot.stoff - base[0].stoff);
    Buf<int> st_entries(tot.ste - base[0].ste);
    Buf<uint32_t> cnode(tot.cnode - base[0].cnode), cnode_off(tot.cnode - base[0].cnode + 1);
    Buf<int> crole_contact(tot.role - base[0].role), crole_slave(tot.role - base[0].role);
    Buf<uint32_t> slave_cn(slaves.size()), face_cn(faces.size());
    face_off[0] = (int)base[0].face;
    slave_off[0] = (int)base[0].slave;
    tab_off[0] = (int)c->ca.n_buckets;
    st_tab_off[0] = c->n_st_tabs;
    ent_off[0] = c->n_entries;
    for (int k = 0, q = 0; k < n_desc; ++k) {
        const ContactPart& cp = parts[k];
        slot_contact_off[k] = K0 + q;
        for (size_t j = 0; j < cp.nf.size(); ++j, ++q) {
            face_off[q + 1] = face_off[q] + cp.nf[j];
            slave_off[q + 1] = slave_off[q] + cp.ns[j];
            tab_off[q + 1] = tab_off[q] + cp.tab[j];
            st_tab_off[q + 1] = st_tab_off[q] + cp.st[j];
            ent_off[q + 1] = ent_off[q] + (cp.tab[j] > 0 ? (long long)cp.nf[j] * LEVEL_CELL_BUDGET : 0);
            is_static[q] = cp.stat[j];
            counts_for_stop[q] = cp.stop[j];
            contact_slot[q] = S0 + k;
            stiff[q] = cp.stiff[j];
            md[q] = cp.md[j];
            cell[q] = cp.cell[j];
        }
        slots[k].contact_dt = INF;
    }
    slot_contact_off[n_desc] = K0 + K;
    cnode_off[0] = (uint32_t)base[0].role;
    std::atomic<bool> cn_missing{false};
    parallel_for(n_desc, [&](long long k) {
        const ContactPart& cp = parts[k];
        const Base& b = base[k];
        const int q0 = slots[k].contact0 - K0;  // local contact index
        const long long f0 = base[0].face, s0 = base[0].slave;
        for (size_t j = 0; j < cp.nf.size(); ++j) {
            std::fill(face_contact.begin() + (face_off[q0 + j] - f0), face_contact.begin() + (face_off[q0 + j + 1] - f0), (int)(K0 + q0 + j));
            std::fill(slave_contact.begin() + (slave_off[q0 + j] - s0), slave_contact.begin() + (slave_off[q0 + j + 1] - s0),
                      (int)(K0 + q0 + j));
        }
        std::copy(cp.faces.begin(), cp.faces.end(), faces.begin() + 4 * (b.face - f0));
        std::copy(cp.slaves.begin(), cp.slaves.end(), slaves.begin() + (b.slave - s0));
        std::copy(cp.scales.begin(), cp.scales.end(), scales.begin() + (b.slave - s0));
        std::copy(cp.box.begin(), cp.box.end(), st_box.begin() + 6 * (size_t)q0);
        for (size_t j = 0; j < cp.st_off.size(); ++j) st_off[b.stoff - base[0].stoff + j] = cp.st_off[j] + (uint32_t)b.ste;
        std::copy(cp.st_entries.begin(), cp.st_entries.end(), st_entries.begin() + (b.ste - base[0].ste));
        for (size_t j = 0; j < cp.dyn_faces.size(); ++j) dyn_faces[b.dyn - base[0].dyn + j] = cp.dyn_faces[j] + (uint32_t)b.face;
        for (size_t j = 0; j < cp.grid_faces.size(); ++j) grid_faces[b.grid - base[0].grid + j] = cp.grid_faces[j] + (uint32_t)b.face;
        std::copy(cp.cnode.begin(), cp.cnode.end(), cnode.begin() + (b.cnode - base[0].cnode));
        for (size_t j = 1; j < cp.cnode_off.size(); ++j) cnode_off[b.cnode - base[0].cnode + j] = cp.cnode_off[j] + (uint32_t)b.role;
        std::copy(cp.crole_contact.begin(), cp.crole_contact.end(), crole_contact.begin() + (b.role - base[0].role));
        std::copy(cp.crole_slave.begin(), cp.crole_slave.end(), crole_slave.begin() + (b.role - base[0].role));
        // the slot's contact nodes (ascending node order): node -> their index
        const long long n0 = slots[k].node0;
        std::vector<uint32_t> at((size_t)descs[k]->n_nodes, UINT32_MAX);
        for (size_t j = 0; j < cp.cnode.size(); ++j) at[cp.cnode[j] - n0] = (uint32_t)j;
        auto cn_of = [&](uint32_t node) {
            const uint32_t j = at[node - n0];
            if (j == UINT32_MAX) {
                cn_missing = true;  // cannot happen: every primary node and face corner has a role
                return 0u;
            }
            return (uint32_t)(b.cnode + j) | (fixed_at(node) ? CN_FIXED : 0u);
        };
        for (size_t j = 0; j < cp.slaves.size(); ++j) slave_cn[b.slave - s0 + j] = cn_of(cp.slaves[j]);
        for (size_t j = 0; j < cp.faces.size(); ++j) face_cn[4 * (b.face - f0) + j] = cn_of(cp.faces[j]);
    }, G);
    if (cn_missing) return crush::fail(CRUSH_ERR_INVALID, "internal: a contact node without a role");
    trace.mark("contact tables concatenated");
    // exhaustive contacts (no grid) get a block each; the rest are listed by entry
    std::vector<int> brute;
    std::vector<uint32_t> gslaves, stslaves;
    std::vector<uint8_t> is_brute(std::max(K, 1), 0);
    int brute_max = c->ca.brute_max_faces;
    for (int q = 0; q < K; ++q) {
        const bool st_grid = st_tab_off[q + 1] > st_tab_off[q];
        const bool grid = tab_off[q + 1] > tab_off[q] || st_grid;
        if (!grid && face_off[q + 1] - face_off[q] <= 255 && slave_off[q + 1] > slave_off[q]) {
            brute.push_back(K0 + q);
            is_brute[q] = 1;
            brute_max = std::max(brute_max, face_off[q + 1] - face_off[q]);
        } else {
            for (int e = slave_off[q]; e < slave_off[q + 1]; ++e) (st_grid ? stslaves : gslaves).push_back((uint32_t)e);
        }
    }
    trace.mark("contact entry lists");
    // ---- vehicles: per slot its ranges, then the node lists filled in parallel ----
    std::vector<long long> vh_off(n_desc + 1, 0), vn_off(n_desc + 1, 0), cn_off(n_desc + 1, 0);
    long long max_vnodes = c->max_vnodes;
    for (int k = 0; k < n_desc; ++k) {
        const crush_model_desc* d = descs[k];
        const int nv = std::min(d->n_vehicles, 4);
        slots[k].vehicle0 = c->va.n_vehicles + (int)vh_off[k];
        slots[k].n_vehicles = nv;
        long long vn = 0, cn = 0;
        for (int v = 0; v < nv; ++v) {
            const crush_vehicle& vd = d->vehicles[v];
            if (vd.n_nodes < 0 || (vd.n_nodes > 0 && !vd.nodes) || vd.n_front < 0 || (vd.n_front > 0 && !vd.front_nodes))
                return crush::fail(CRUSH_ERR_INVALID, "invalid vehicle");
            if (vd.accel_node >= (uint64_t)d->n_nodes) return crush::fail(CRUSH_ERR_INVALID, "accelerometer node out of range");
            vn += vd.n_nodes;
            cn += vd.n_front + 1;
            max_vnodes = std::max<long long>(max_vnodes, vd.n_nodes);
        }
        vh_off[k + 1] = vh_off[k] + nv;
        vn_off[k + 1] = vn_off[k] + vn;
        cn_off[k + 1] = cn_off[k] + cn;
    }
    // voff: each vehicle's end in the context's vehicle-node list; crush_off_new:
    // its end in the new crush-measure node list (front nodes, then the accelerometer)
    std::vector<long long> voff(vh_off[n_desc]);
    std::vector<size_t> crush_off_new(vh_off[n_desc]);
    std::vector<int> vslot(vh_off[n_desc]), vlocal(vh_off[n_desc]);
    Buf<uint32_t> vnodes(vn_off[n_desc]), crush_nodes_new(cn_off[n_desc]);
    parallel_for(n_desc, [&](long long k) {
        const crush_model_desc* d = descs[k];
        const long long n0 = slots[k].node0;
        long long a = vn_off[k], b = cn_off[k];
        for (int v = 0; v < slots[k].n_vehicles; ++v) {
            const crush_vehicle& vd = d->vehicles[v];
            for (int64_t i = 0; i < vd.n_nodes; ++i) {
                if (vd.nodes[i] >= (uint64_t)d->n_nodes) return errs[k].set(CRUSH_ERR_INVALID, "vehicle node out of range");
                vnodes[a++] = (uint32_t)(n0 + vd.nodes[i]);
            }
            for (int64_t i = 0; i < vd.n_front; ++i) {
                if (vd.front_nodes[i] >= (uint64_t)d->n_nodes) return errs[k].set(CRUSH_ERR_INVALID, "front node out of range");
                crush_nodes_new[b++] = (uint32_t)(n0 + vd.front_nodes[i]);
            }
            crush_nodes_new[b++] = (uint32_t)(n0 + vd.accel_node);
            const long long q = vh_off[k] + v;
            voff[q] = c->n_vnodes + a;
            crush_off_new[q] = (size_t)b;
            vslot[q] = S0 + (int)k;
            vlocal[q] = v;
        }
    }, G);
    for (auto& e : errs)
        if (e.code != CRUSH_OK) return crush::fail(e.code, e.msg);
    trace.mark("contacts and vehicles built");

    // ---- device arrays: allocated with the room (creating), then the new ranges uploaded ----
    // Slots added to an open run are set up on the set-up stream (c->stream
    // names it until this function returns), beside the steps already
    // issued on the main stream: their set-up writes only their own ranges.
    const bool appending = !creating && c->run_open;
    cudaStream_t main_stream = c->stream;
    if (appending && !c->setup) {
        // high priority: its blocks go first as the steps' blocks retire
        int lo = 0, hi = 0;
        CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        CK(cudaStreamCreateWithPriority(&c->setup, cudaStreamNonBlocking, hi));
        CK(cudaEventCreateWithFlags(&c->ev_setup, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c->ev_tab, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c->ev_arena, cudaEventDisableTiming));
    }
    struct StreamRestore {
        crush_ctx* c;
        cudaStream_t s;
        bool on;
        ~StreamRestore() {
            if (on) c->stream = s;
        }
    } restore{c, main_stream, appending};
    if (appending) c->stream = c->setup;
    std::vector<std::pair<long long, long long>> tab_ranges;  // appending: chunk-table entries the main stream updates
    Stager stager;
    stager.init(c->stream, sizeof(double) * 6 * N + sizeof(uint32_t) * 27 * E);
    // A small addition (one or a few requests) packs its uploads into the
    // context's pinned arena, allocated once at ARENA_BYTES; a larger one
    // goes through the staging buffers (several threads fill them). Pinned
    // memory is never freed or grown while a run is open: freeing it waits
    // for the whole device.
    constexpr size_t ARENA_BYTES = size_t(64) << 20;
    const size_t want = 96 * (size_t)N + 64 * (size_t)E + 64 * (size_t)(tot.face - base[0].face) + 16 * (size_t)(tot.ste - base[0].ste) +
                        8 * (size_t)(tot.stoff - base[0].stoff) + 64 * (size_t)(tot.slave - base[0].slave) + (1u << 20);
    if (appending && want <= ARENA_BYTES) {
        CK(cudaEventSynchronize(c->ev_arena));  // the previous set-up's copies are done
        if (!c->arena) {
            size_t got = ARENA_BYTES;
            c->arena = static_cast<char*>(pinned_take(&got));
            if (!c->arena) return crush::fail(CRUSH_ERR_OOM, "cannot pin the upload arena");
            c->arena_cap = got;
        }
        stager.use_arena(c->arena, c->arena_cap, c->ev_arena);
    }
    c->stager = &stager;
    struct StagerRelease {
        crush_ctx* c;
        Stager* s;
        ~StagerRelease() {
            s->release();
            c->stager = nullptr;
        }
    } release_stager{c, &stager};
    ContactArrays& ca = c->ca;
    VehicleArrays& va = c->va;
    if (creating) {
        const long long NC = cap.nodes, EC = cap.elems;
        c->stride = std::max<long long>(32, (EC + 31) / 32 * 32);
        const long long QC = std::max<long long>(1, cap.scalars);
        c->sc_stride = QC;
        TRY(c->alloc(&c->pos, 3 * NC));
        TRY(c->alloc(&c->conn_all, 8 * EC));
        TRY(c->alloc(&c->part, EC));
        TRY(c->alloc(&c->mat4, 4 * cap.parts));
        TRY(c->alloc(&c->mats, cap.parts));
        TRY(c->alloc(&c->hc_index_d, EC));
        TRY(c->alloc(&c->sc_index_d, EC));
        TRY(c->alloc(&c->sc_model_d, QC));
        TRY(c->alloc(&c->sc_list_d, QC));
        TRY(c->alloc(&c->sc_mat, 2 * QC));
        TRY(c->alloc(&c->fixed, NC));
        TRY(c->alloc(&c->node_slot, NC));
        TRY(c->alloc(&c->elem_slot, EC));
        for (uint32_t** p : {&c->all_off, &c->hc_off, &c->sc_off}) TRY(c->alloc(p, NC + 1));
        for (uint32_t** p : {&c->all_slot, &c->hc_slot}) TRY(c->alloc(p, 8 * EC));
        TRY(c->alloc(&c->sc_slot, 8 * QC));
        {
            uint32_t* ell = nullptr;
            TRY(c->alloc(&ell, 8 * (size_t)NC));
            c->hc_ell = reinterpret_cast<const uint4*>(ell);
        }
        for (double** p : {&c->v0, &c->u, &c->v, &c->v_half, &c->f_int, &c->f_ext, &c->f_ext_odd, &c->u_tmp, &c->f_tmp})
            TRY(c->alloc(p, 3 * NC));
        for (double** p : {&c->inv_mass, &c->mass, &c->added, &c->n_tmp, &c->n_tmp2}) TRY(c->alloc(p, NC));
        for (double** p : {&c->volume, &c->dt_factor, &c->elem_mass, &c->elem_dt, &c->elem_extra, &c->e_tmp}) TRY(c->alloc(p, EC));
        TRY(c->alloc(&c->lumped, 8 * EC));
        TRY(c->alloc(&c->eroded_all, EC));
        TRY(c->alloc(&c->planes, (size_t)N_STATIC_PLANES * c->stride));
        TRY(c->alloc(&c->state, (size_t)N_STATE_PLANES * c->stride));
        TRY(c->alloc(&c->corner, (size_t)24 * EC));
        TRY(c->alloc(&c->sc_geo, (size_t)SC_PLANES * c->sc_stride));
        TRY(c->alloc(&c->sc_corner, (size_t)24 * QC));
        TRY(c->alloc(&c->ctls, cap.slots));
        TRY(c->alloc(&c->ctls_aux, cap.slots));
        TRY(c->alloc(&c->slot_done, cap.slots));
        TRY(c->alloc(&c->mass_flag, 1));
        TRY(c->alloc(&c->fused_counter, 1));
        TRY(c->alloc(&c->forces_queue, 2));
        TRY(c->alloc(&c->setup_bad, 1));
        CK(cudaMemsetAsync(c->mass_flag, 0, sizeof(int), c->stream));
        CK(cudaMemsetAsync(c->fused_counter, 0, sizeof(unsigned), c->stream));
        CK(cudaMemsetAsync(c->forces_queue, 0, 2 * sizeof(unsigned), c->stream));
        CK(cudaMemsetAsync(c->planes, 0, sizeof(float4) * N_STATIC_PLANES * c->stride, c->stream));
        CK(cudaMemsetAsync(c->eroded_all, 0, EC, c->stream));
        CK(cudaMemsetAsync(c->ctls, 0, sizeof(Control) * cap.slots, c->stream));
        CK(cudaMemsetAsync(c->slot_done, 0, sizeof(int) * cap.slots, c->stream));
        // contacts
        const long long KC = std::max<long long>(cap.contacts, 1), FC = std::max<long long>(cap.faces, 1),
                        SC = std::max<long long>(cap.slaves, 1), CNC = std::max<long long>(cap.cnodes, 1);
        TRY(c->alloc(&c->face_off_d, KC + 1));
        TRY(c->alloc(&c->slave_off_d, KC + 1));
        TRY(c->alloc(&c->tab_off_d, KC + 1));
        TRY(c->alloc(&c->st_tab_off_d, KC + 1));
        TRY(c->alloc(&c->ent_off_d, KC + 1));
        TRY(c->alloc(&c->faces_d, 4 * FC));
        TRY(c->alloc(&ca.geo, FC));
        TRY(c->alloc(&c->slaves_d, SC));
        TRY(c->alloc(&c->scales_d, SC));
        TRY(c->alloc(&ca.hit, SC));
        TRY(c->alloc(&ca.hit_force, 3 * SC));
        TRY(c->alloc(&ca.hit_sd, SC));
        for (double** p : {&c->stiff_d, &c->md_d, &c->cell_d}) TRY(c->alloc(p, KC));
        TRY(c->alloc(&c->st_box_d, 6 * KC));
        TRY(c->alloc(&ca.counts, std::max<long long>(cap.buckets, 1)));
        TRY(c->alloc(&ca.boff, std::max<long long>(cap.buckets, 1)));
        TRY(c->alloc(&ca.blen, std::max<long long>(cap.buckets, 1)));
        TRY(c->alloc(&ca.entries, std::max<long long>(cap.entries, 1)));
        TRY(c->alloc(&c->grid_faces_d, FC));
        TRY(c->alloc(&c->dyn_faces_d, FC));
        TRY(c->alloc(&c->brute_d, KC));
        TRY(c->alloc(&c->gslaves_d, SC));
        TRY(c->alloc(&c->stslaves_d, SC));
        TRY(c->alloc(&ca.grid_state, 2 * KC + 1));
        TRY(c->alloc(&ca.cells, FC));
        TRY(c->alloc(&ca.gather_work, CNC));
        TRY(c->alloc(&ca.ev_pool_n, 2));
        ca.big_cap = FC;
        TRY(c->alloc(&ca.big_faces, (size_t)ca.big_cap));
        TRY(c->alloc(&ca.big_box, 6 * (size_t)ca.big_cap));
        TRY(c->alloc(&ca.big_best, SC));
        TRY(c->alloc(&ca.search_stats, 3 * KC));
        c->pen_stride = KC;
        TRY(c->alloc(&ca.pen_count, 2 * (size_t)c->pen_stride));
        TRY(c->alloc(&ca.pen_max_bits, 2 * (size_t)c->pen_stride));
        TRY(c->alloc(&c->counts_for_stop_d, KC));
        TRY(c->alloc(&c->cnode_d, CNC));
        TRY(c->alloc(&c->cnode_off_d, CNC + 1));
        TRY(c->alloc(&c->crole_contact_d, std::max<long long>(cap.roles, 1)));
        TRY(c->alloc(&c->crole_slave_d, std::max<long long>(cap.roles, 1)));
        TRY(c->alloc(&c->slave_cn_d, SC));
        TRY(c->alloc(&c->face_cn_d, 4 * FC));
        TRY(c->alloc(&ca.ev_count, CNC));
        TRY(c->alloc(&ca.ev_list, EV_CAP * CNC));
        ca.ev_pool_cap = std::max<long long>(4096, SC);
        TRY(c->alloc(&ca.ev_pool, (size_t)ca.ev_pool_cap));
        TRY(c->alloc(&c->face_contact_d, FC));
        TRY(c->alloc(&c->slave_contact_d, SC));
        TRY(c->alloc(&c->contact_slot_d, KC));
        TRY(c->alloc(&c->slot_contact_off_d, cap.slots + 1));
        TRY(c->alloc(&c->is_static_d, KC));
        TRY(c->alloc(&c->st_off_d, std::max<long long>(cap.st_tabs + cap.contacts, 1)));
        TRY(c->alloc(&c->st_entries_d, std::max<long long>(cap.st_ents, 1)));
        ca.face_off = c->face_off_d;
        ca.slave_off = c->slave_off_d;
        ca.tab_off = c->tab_off_d;
        ca.st_tab_off = c->st_tab_off_d;
        ca.ent_off = c->ent_off_d;
        ca.faces = c->faces_d;
        ca.slaves = c->slaves_d;
        ca.slave_scale = c->scales_d;
        ca.stiffness = c->stiff_d;
        ca.max_distance = c->md_d;
        ca.cell = c->cell_d;
        ca.st_box = c->st_box_d;
        ca.grid_faces = c->grid_faces_d;
        ca.dyn_faces = c->dyn_faces_d;
        ca.brute_contacts = c->brute_d;
        ca.grid_slaves = c->gslaves_d;
        ca.st_slaves = c->stslaves_d;
        ca.counts_for_stop = c->counts_for_stop_d;
        ca.cnode = c->cnode_d;
        ca.cnode_off = c->cnode_off_d;
        ca.crole_contact = c->crole_contact_d;
        ca.crole_slave = c->crole_slave_d;
        ca.slave_cn = c->slave_cn_d;
        ca.face_cn = c->face_cn_d;
        ca.face_contact = c->face_contact_d;
        ca.slave_contact = c->slave_contact_d;
        ca.contact_slot = c->contact_slot_d;
        ca.slot_contact_off = c->slot_contact_off_d;
        ca.is_static = c->is_static_d;
        ca.st_off = c->st_off_d;
        ca.st_entries = c->st_entries_d;
        ca.contact_room = KC;
        ca.levels_used = ca.grid_state;
        ca.ent_cursor = ca.grid_state + KC;
        ca.big_count = ca.grid_state + 2 * KC;
        ca.gather_count = ca.ev_pool_n + 1;
        ca.exhaustive = 0;
        CK(cudaMemsetAsync(ca.counts, 0, sizeof(int) * std::max<long long>(cap.buckets, 1), c->stream));
        CK(cudaMemsetAsync(ca.blen, 0, sizeof(int) * std::max<long long>(cap.buckets, 1), c->stream));
        CK(cudaMemsetAsync(ca.big_best, 0x7F, sizeof(int) * SC, c->stream));  // BIG_NONE
        CK(cudaMemsetAsync(ca.grid_state, 0, sizeof(int) * (2 * KC + 1), c->stream));
        CK(cudaMemsetAsync(ca.search_stats, 0, sizeof(unsigned long long) * 3 * KC, c->stream));
        CK(cudaMemsetAsync(ca.pen_count, 0, sizeof(unsigned long long) * 2 * c->pen_stride, c->stream));
        CK(cudaMemsetAsync(ca.pen_max_bits, 0, sizeof(unsigned long long) * 2 * c->pen_stride, c->stream));
        CK(cudaMemsetAsync(ca.ev_count, 0, sizeof(int) * CNC, c->stream));
        CK(cudaMemsetAsync(ca.ev_pool_n, 0, 2 * sizeof(int), c->stream));
        // vehicles
        TRY(c->alloc(&c->voff_d, std::max<long long>(cap.vehicles, 1) + 1));
        TRY(c->alloc(&c->vnodes_d, std::max<long long>(cap.vnodes, 1)));
        TRY(c->alloc(&c->vslot_d, std::max<long long>(cap.vehicles, 1)));
        TRY(c->alloc(&c->vlocal_d, std::max<long long>(cap.vehicles, 1)));
        TRY(c->alloc(&c->veh_out, 7 * std::max<long long>(cap.vehicles, 1)));
        va.off = c->voff_d;
        va.nodes = c->vnodes_d;
        va.slot = c->vslot_d;
        va.local = c->vlocal_d;
        const long long zero = 0;
        CK(cudaMemcpyAsync(c->voff_d, &zero, sizeof(long long), cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));  // the zero above is a stack value
        // active chunk tables: every space's chunks at its full room
        const long long sizes[ACTIVE_SPACES] = {EC, EC, NC, SC, CNC, FC, SC, SC, QC};
        c->space_off_h.assign(ACTIVE_SPACES + 1, 0);
        for (int sp = 0; sp < ACTIVE_SPACES; ++sp) c->space_off_h[sp + 1] = c->space_off_h[sp] + (sizes[sp] + CHUNK - 1) / CHUNK;
        const long long nch = c->space_off_h[ACTIVE_SPACES];
        c->chunk_lo_h.assign(nch, INT32_MAX);
        c->chunk_hi_h.assign(nch, -1);
        TRY(c->alloc(&c->chunk_lo_d, std::max<long long>(nch, 1)));
        TRY(c->alloc(&c->chunk_hi_d, std::max<long long>(nch, 1)));
        const long long* off_d = nullptr;
        TRY(c->upload_const(&off_d, c->space_off_h));
        c->ab.n_chunks = nch;
        c->ab.chunk_lo = c->chunk_lo_d;
        c->ab.chunk_hi = c->chunk_hi_d;
        c->ab.space_off = off_d;
        TRY(c->alloc(&c->ab.lists, std::max<long long>(nch, 1)));
        TRY(c->alloc(&c->ab.counts, ACTIVE_SPACES));
        c->adaptive = adaptive;
        c->check_steps = check_steps;
        trace.mark("allocations");
    }
    c->any_separation = any_sep;
    // uploads of the new ranges
    auto put = [&](auto* dst, const auto* src, size_t count) -> int {
        if (!count) return CRUSH_OK;
        return stager_copy(&stager, dst, src, count * sizeof(*src));
    };
    TRY(put(c->pos + 3 * N0, cm.positions.data(), 3 * N));
    TRY(put(c->v0 + 3 * N0, cm.v0.data(), 3 * N));
    TRY(put(c->conn_all + 8 * E0, cm.hexes.data(), 8 * E));
    TRY(put(c->part + E0, cm.hex_part.data(), E));
    TRY(put(c->mat4 + 4 * P0, cm.mat4.data(), cm.mat4.size()));
    TRY(put(c->mats + P0, cm.mats.data(), cm.mats.size()));
    TRY(put(c->hc_index_d + E0, hc_index.data(), E));
    TRY(put(c->sc_index_d + E0, sc_index.data(), E));
    TRY(put(c->sc_model_d + Q0, sc_model.data(), Q));
    TRY(put(c->sc_list_d + QF0, sc_list.data(), QF));
    TRY(put(c->sc_mat + 2 * Q0, sc_mat.data(), 2 * Q));
    TRY(put(c->fixed + N0, cm.fixed.data(), N));
    TRY(put(c->node_slot + N0, cm.node_slot.data(), N));
    TRY(put(c->elem_slot + E0, cm.elem_slot.data(), E));
    CK(cudaMemsetAsync(c->eroded_all + E0, 0, E, c->stream));
    trace.mark("model uploads");
    const long long FB = base[0].face, SB = base[0].slave;
    TRY(put(c->face_off_d + K0, face_off.data(), K + 1));
    TRY(put(c->slave_off_d + K0, slave_off.data(), K + 1));
    TRY(put(c->tab_off_d + K0, tab_off.data(), K + 1));
    TRY(put(c->st_tab_off_d + K0, st_tab_off.data(), K + 1));
    TRY(put(c->ent_off_d + K0, ent_off.data(), K + 1));
    TRY(put(c->faces_d + 4 * FB, faces.data(), faces.size()));
    TRY(put(c->slaves_d + SB, slaves.data(), slaves.size()));
    TRY(put(c->scales_d + SB, scales.data(), scales.size()));
    TRY(put(c->stiff_d + K0, stiff.data(), K));
    TRY(put(c->md_d + K0, md.data(), K));
    TRY(put(c->cell_d + K0, cell.data(), K));
    TRY(put(c->st_box_d + 6 * K0, st_box.data(), 6 * (size_t)K));
    TRY(put(c->grid_faces_d + base[0].grid, grid_faces.data(), grid_faces.size()));
    TRY(put(c->dyn_faces_d + base[0].dyn, dyn_faces.data(), dyn_faces.size()));
    TRY(put(c->brute_d + ca.n_brute, brute.data(), brute.size()));
    TRY(put(c->gslaves_d + ca.n_grid_slaves, gslaves.data(), gslaves.size()));
    TRY(put(c->stslaves_d + ca.n_st_slaves, stslaves.data(), stslaves.size()));
    TRY(put(c->counts_for_stop_d + K0, counts_for_stop.data(), K));
    TRY(put(c->cnode_d + base[0].cnode, cnode.data(), cnode.size()));
    TRY(put(c->cnode_off_d + base[0].cnode, cnode_off.data(), cnode_off.size()));
    TRY(put(c->crole_contact_d + base[0].role, crole_contact.data(), crole_contact.size()));
    TRY(put(c->crole_slave_d + base[0].role, crole_slave.data(), crole_slave.size()));
    TRY(put(c->slave_cn_d + SB, slave_cn.data(), slave_cn.size()));
    TRY(put(c->face_cn_d + 4 * FB, face_cn.data(), face_cn.size()));
    TRY(put(c->face_contact_d + FB, face_contact.data(), face_contact.size()));
    TRY(put(c->slave_contact_d + SB, slave_contact.data(), slave_contact.size()));
    TRY(put(c->contact_slot_d + K0, contact_slot.data(), K));
    TRY(put(c->slot_contact_off_d + S0, slot_contact_off.data(), n_desc + 1));
    TRY(put(c->is_static_d + K0, is_static.data(), K));
    TRY(put(c->st_off_d + base[0].stoff, st_off.data(), st_off.size()));
    TRY(put(c->st_entries_d + base[0].ste, st_entries.data(), st_entries.size()));
    TRY(put(c->vnodes_d + c->n_vnodes, vnodes.data(), vnodes.size()));
    TRY(put(c->voff_d + 1 + va.n_vehicles, voff.data(), voff.size()));
    TRY(put(c->vslot_d + va.n_vehicles, vslot.data(), vslot.size()));
    TRY(put(c->vlocal_d + va.n_vehicles, vlocal.data(), vlocal.size()));
    trace.mark("contact uploads");

    // ---- the context's counts and host copies take the new slots ----
    c->slots.insert(c->slots.end(), slots.begin(), slots.end());
    c->n_slots = S0 + n_desc;
    c->n_nodes = N0 + N;
    c->n_all = E0 + E;
    c->n_hc = H0 + H;
    c->n_sc = Q0 + Q;
    c->n_sc_free = QF0 + QF;
    c->n_parts = P0 + P;
    c->hc_index.insert(c->hc_index.end(), hc_index.begin(), hc_index.end());
    c->hc_model.insert(c->hc_model.end(), hc_model.begin(), hc_model.end());
    c->sc_model.insert(c->sc_model.end(), sc_model.begin(), sc_model.end());
    c->n_contacts = K0 + K;
    c->n_faces = tot.face;
    c->n_slaves = tot.slave;
    c->n_st_ents = tot.ste;
    c->n_st_offs = tot.stoff;
    c->n_st_tabs = st_tab_off[K];
    c->n_entries = ent_off[K];
    c->n_roles = tot.role;
    if (creating) {
        c->face_off_h.assign(face_off.begin(), face_off.end());
        c->slave_off_h.assign(slave_off.begin(), slave_off.end());
        c->tab_off_h.assign(tab_off.begin(), tab_off.end());
    } else {
        c->face_off_h.insert(c->face_off_h.end(), face_off.begin() + 1, face_off.end());
        c->slave_off_h.insert(c->slave_off_h.end(), slave_off.begin() + 1, slave_off.end());
        c->tab_off_h.insert(c->tab_off_h.end(), tab_off.begin() + 1, tab_off.end());
    }
    c->is_static_h.insert(c->is_static_h.end(), is_static.begin(), is_static.begin() + K);
    c->is_brute_h.resize(std::max(K0 + K, 1), 0);
    for (int q = 0; q < K; ++q) c->is_brute_h[K0 + q] = is_brute[q];
    c->grid_slaves_h.insert(c->grid_slaves_h.end(), gslaves.begin(), gslaves.end());
    c->st_slaves_h.insert(c->st_slaves_h.end(), stslaves.begin(), stslaves.end());
    ca.n_contacts = c->n_contacts;
    ca.n_slots = c->n_slots;
    ca.n_buckets = tab_off[K];
    ca.n_grid_faces = tot.grid;
    ca.n_dyn_faces = tot.dyn;
    ca.n_cnodes = tot.cnode;
    ca.n_brute += (int)brute.size();
    ca.brute_max_faces = std::max(brute_max, 1);
    ca.n_grid_slaves = (long long)c->grid_slaves_h.size();
    ca.n_st_slaves = (long long)c->st_slaves_h.size();
    ca.is_brute_h = c->is_brute_h.data();
    va.n_vehicles += (int)vslot.size();
    c->n_vnodes += (long long)vnodes.size();
    c->max_vnodes = max_vnodes;
    va.vx_blocks = (int)std::min<long long>(VX_BLOCKS, std::max<long long>(1, (max_vnodes + 2047) / 2048));
    for (size_t i = 0; i < crush_off_new.size(); ++i) c->crush_off_h.push_back(c->crush_nodes_h.size() + crush_off_new[i]);
    const size_t crush_before = c->crush_nodes_h.size();
    c->crush_nodes_h.insert(c->crush_nodes_h.end(), crush_nodes_new.begin(), crush_nodes_new.end());
    trace.mark("host copies");
    // the crush-measure node list: room for the context's vehicle nodes and
    // an accelerometer per vehicle; a list beyond it moves to a new buffer
    {
        const size_t ncn = c->crush_nodes_h.size();
        if (ncn > c->crush_cap) {
            const size_t room = std::max<size_t>(std::max<size_t>(ncn, 1), (size_t)(c->cap.vnodes + c->cap.vehicles));
            TRY(c->alloc(&c->crush_nodes, room));
            TRY(c->alloc(&c->crush_ux, room));
            c->crush_cap = room;
            TRY(put(c->crush_nodes, c->crush_nodes_h.data(), ncn));
        } else {
            TRY(put(c->crush_nodes + crush_before, c->crush_nodes_h.data() + crush_before, ncn - crush_before));
        }
    }
    trace.mark("crush-measure nodes");
    // ---- active chunk tables: the slot range of every chunk the new entities touch ----
    {
        const long long ends[ACTIVE_SPACES] = {c->n_hc, c->n_all, c->n_nodes, ca.n_grid_slaves, ca.n_cnodes, ca.n_dyn_faces,
                                               c->n_slaves, ca.n_st_slaves, c->n_sc_free};
        const long long begins[ACTIVE_SPACES] = {H0, E0, N0, ca.n_grid_slaves - (long long)gslaves.size(), base[0].cnode, base[0].dyn,
                                                 SB, ca.n_st_slaves - (long long)stslaves.size(), QF0};
        auto slot_of = [&](int sp, long long i) -> int {
            switch (sp) {
                case 0: return (int)cm.elem_slot[hc_model[i - H0] - E0];
                case 1: return (int)cm.elem_slot[i - E0];
                case 2: return (int)cm.node_slot[i - N0];
                case 3: return contact_slot[slave_contact[gslaves[i - begins[3]] - SB] - K0];
                case 4: return (int)cm.node_slot[cnode[i - base[0].cnode] - N0];
                case 5: return contact_slot[face_contact[dyn_faces[i - base[0].dyn] - FB] - K0];
                case 6: return contact_slot[slave_contact[i - SB] - K0];
                case 7: return contact_slot[slave_contact[stslaves[i - begins[7]] - SB] - K0];
                default: return (int)cm.elem_slot[sc_model[sc_list[i - QF0] - Q0] - E0];
            }
        };
        for (int sp = 0; sp < ACTIVE_SPACES; ++sp) {
            if (ends[sp] <= begins[sp]) continue;
            const long long q0 = c->space_off_h[sp] + begins[sp] / CHUNK, q1 = c->space_off_h[sp] + (ends[sp] - 1) / CHUNK;
            parallel_for(q1 - q0 + 1, [&](long long j) {
                const long long q = q0 + j;
                const long long i0 = std::max(begins[sp], (q - c->space_off_h[sp]) * CHUNK);
                const long long i1 = std::min(ends[sp], (q - c->space_off_h[sp] + 1) * CHUNK);
                int a = c->chunk_lo_h[q], b = c->chunk_hi_h[q];
                for (long long i = i0; i < i1; ++i) {
                    const int sl = slot_of(sp, i);
                    a = std::min(a, sl);
                    b = std::max(b, sl);
                }
                c->chunk_lo_h[q] = a;
                c->chunk_hi_h[q] = b;
            }, 64);
            // A chunk the new entities share with running slots is read by
            // the steps in flight: an append updates the tables in the main
            // stream's order.
            if (appending) {
                tab_ranges.emplace_back(q0, q1);
            } else if (!creating) {
                TRY(put(c->chunk_lo_d + q0, c->chunk_lo_h.data() + q0, q1 - q0 + 1));
                TRY(put(c->chunk_hi_d + q0, c->chunk_hi_h.data() + q0, q1 - q0 + 1));
            }
        }
        // A new context's tables in full: chunks no slot holds yet have the
        // empty range (lo > hi), which the active-list pass never reads
        // control blocks for.
        if (creating) {
            TRY(put(c->chunk_lo_d, c->chunk_lo_h.data(), c->chunk_lo_h.size()));
            TRY(put(c->chunk_hi_d, c->chunk_hi_h.data(), c->chunk_hi_h.size()));
        }
    }
    trace.mark("active chunk tables");

    // ---- device set-up of the new elements and nodes ----
    // node incidence (CSR and padded rows), in scratch returned after the set-up's sync below
    std::vector<void*> scratch_bufs;
    {
        const size_t bytes = incidence_scratch_bytes(E, N);
        char* scratch = nullptr;
        const size_t mark = c->allocs.size();
        TRY(c->alloc(&scratch, bytes));
        scratch_bufs.assign(c->allocs.begin() + (long)mark, c->allocs.end());
        uint32_t* ell = const_cast<uint32_t*>(reinterpret_cast<const uint32_t*>(c->hc_ell)) + 8 * N0;
        if (launch_incidence(c->stream, E0, E, N0, N, c->conn_all, c->hc_index_d, c->sc_index_d, (uint32_t)(8 * E0), (uint32_t)(8 * H0),
                             (uint32_t)(8 * Q0), c->all_off + N0, c->all_slot, c->hc_off + N0, c->hc_slot, c->sc_off + N0, c->sc_slot,
                             ell, scratch) != 0)
            return crush::fail(CRUSH_ERR_CUDA, std::string("node incidence: ") + cudaGetErrorString(cudaGetLastError()));
        c->launches += 2;
    }
    trace.mark("node incidence queued");
    CK(cudaMemsetAsync(c->setup_bad, 0, sizeof(int), c->stream));
    launch_setup_geometry(c->stream, E0, E0 + E, c->pos, c->conn_all, c->part, c->mat4, c->hc_index_d, c->elem_slot, c->stride, c->planes,
                          c->volume, c->lumped, c->dt_factor, c->elem_mass, c->setup_bad, c->sc_index_d, c->sc_stride, c->sc_geo);
    TRY(check_launch(c));
    launch_node_masses(c->stream, N, c->all_off + N0, c->all_slot, c->lumped, c->mass + N0, c->inv_mass + N0);
    TRY(check_launch(c));
    launch_init_state(c->stream, H0, H0 + H, c->stride, c->state);
    TRY(check_launch(c));
    // contact_dt over every listed node of the slot's contacts (src/solver.rs:217-223)
    std::vector<double> mass_h(N);
    int bad_h = 0;
    CK(cudaMemcpyAsync(&bad_h, c->setup_bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(mass_h.data(), c->mass + N0, N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    // the stable step of every new slot at u = 0, through the drop-in control blocks
    CK(cudaMemsetAsync(c->u_tmp + 3 * N0, 0, sizeof(double) * 3 * N, c->stream));
    std::vector<Control> aux(n_desc);
    std::memset(aux.data(), 0, sizeof(Control) * aux.size());
    for (Control& a : aux) a.dt_stable_bits = INF_BITS;
    CK(cudaMemcpyAsync(c->ctls_aux + S0, aux.data(), sizeof(Control) * aux.size(), cudaMemcpyHostToDevice, c->stream));
    launch_elem_dt(c->stream, c->el(), c->nd(), c->ctls_aux, c->u_tmp, 0, E0);
    TRY(check_launch(c));
    CK(cudaMemcpyAsync(aux.data(), c->ctls_aux + S0, sizeof(Control) * aux.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    trace.mark("device set-up (sync)");
    free_bufs(c, scratch_bufs);
    if (bad_h == 1) return crush::fail(CRUSH_ERR_INVALID, "degenerate hexahedron (singular Jacobian)");
    if (bad_h == 2) return crush::fail(CRUSH_ERR_INVALID, "hourglass modes not independent");
    parallel_for(n_desc, [&](long long k) {
        const crush_model_desc* d = descs[k];
        Slot& sl = c->slots[S0 + k];
        double cdt = INF;
        for (int q = 0; q < d->n_contacts; ++q) {
            const crush_contact& cd = d->contacts[q];
            if (!(cd.stiffness > 0.0)) continue;
            for (int64_t i = 0; i < cd.n_nodes; ++i) {
                const double m = mass_h[sl.node0 - N0 + cd.nodes[i]];
                if (m > 0.0) cdt = std::fmin(cdt, 2.0 * std::sqrt(m / cd.stiffness));
            }
        }
        sl.contact_dt = cdt;
        double stable;
        std::memcpy(&stable, &aux[k].dt_stable_bits, sizeof(double));
        if (!std::isfinite(stable)) {
            static const int EDGES[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6}, {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
            double mn = INF, cmax = 0.0;
            for (long long e = sl.elem0; e < sl.elem0 + sl.n_elems; ++e) {
                cmax = std::fmax(cmax, wave_speed(mat_of(e)));
                for (auto& ed : EDGES) {
                    const double* p = &cm.positions[3 * (size_t)(hex(e, ed[0]) - N0)];
                    const double* q = &cm.positions[3 * (size_t)(hex(e, ed[1]) - N0)];
                    mn = std::fmin(mn, std::sqrt((p[0] - q[0]) * (p[0] - q[0]) + (p[1] - q[1]) * (p[1] - q[1]) + (p[2] - q[2]) * (p[2] - q[2])));
                }
            }
            stable = mn / (std::sqrt(3.0) * cmax);
        }
        sl.stable = std::fmin(stable, sl.contact_dt);
        sl.dt_floor = sl.settings.mass_scaling > 0.0 ? sl.settings.mass_scaling * sl.stable : 0.0;
        sl.dt0 = sl.settings.time_step > 0.0 ? sl.settings.time_step : sl.stable * sl.settings.dt_scale;
    }, G);
    trace.mark("initial stable step");
    if (creating) {
        c->period = std::lcm(c->check_steps, 20);
        if (c->period > 200) c->period = 0;  // no graph for odd periods
        c->base_period = c->period;
    }
    drop_graphs(c);
    if (!c->run_open) return CRUSH_OK;
    TRY(begin_slots(c, S0, c->n_slots));
    // The main stream: the set-up done, the chunk tables, then the new
    // contacts' first search (its scratch is shared with the steps').
    CK(cudaEventRecord(c->ev_setup, c->setup));
    c->stream = main_stream;
    restore.on = false;
    CK(cudaStreamWaitEvent(main_stream, c->ev_setup, 0));
    size_t n_tab = 0;
    for (auto& r : tab_ranges) n_tab += (size_t)(r.second - r.first + 1);
    if (n_tab > 0) {
        CK(cudaEventSynchronize(c->ev_tab));  // the previous append's copies are done
        if (2 * n_tab > c->tab_pinned_cap) {
            pinned_give(c->tab_pinned, sizeof(int) * c->tab_pinned_cap);  // its copies are done (ev_tab above)
            c->tab_pinned = nullptr;
            c->tab_pinned_cap = 0;
            size_t got = sizeof(int) * std::max<size_t>(2 * n_tab, 1 << 16);
            c->tab_pinned = static_cast<int*>(pinned_take(&got));
            if (!c->tab_pinned) return crush::fail(CRUSH_ERR_OOM, "cannot pin the chunk-table buffer");
            c->tab_pinned_cap = got / sizeof(int);
        }
        int* hp = c->tab_pinned;
        for (auto& r : tab_ranges) {
            const size_t n = (size_t)(r.second - r.first + 1);
            std::memcpy(hp, c->chunk_lo_h.data() + r.first, sizeof(int) * n);
            std::memcpy(hp + n, c->chunk_hi_h.data() + r.first, sizeof(int) * n);
            CK(cudaMemcpyAsync(c->chunk_lo_d + r.first, hp, sizeof(int) * n, cudaMemcpyHostToDevice, main_stream));
            CK(cudaMemcpyAsync(c->chunk_hi_d + r.first, hp + n, sizeof(int) * n, cudaMemcpyHostToDevice, main_stream));
            hp += 2 * n;
        }
        CK(cudaEventRecord(c->ev_tab, main_stream));
    }
    return search_added(c, K0, dyn0, gs0, st0, brute0);
#undef TRY
}

int create_impl(const crush_model_desc* const* descs, int n_desc, int device, crush_ctx* c, const crush_capacity* room = nullptr) {
    if (n_desc <= 0 || !descs) return crush::fail(CRUSH_ERR_INVALID, "no models");
    c->device = device;
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CK(cudaDeviceGetAttribute(&c->n_sms, cudaDevAttrMultiProcessorCount, device));

    {
        int lo = 0, hi = 0;
        CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        CK(cudaStreamCreateWithPriority(&c->side, cudaStreamNonBlocking, hi));  // search blocks first when SMs free up
        CK(cudaStreamCreateWithPriority(&c->side2, cudaStreamNonBlocking, hi));
        CK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c->ev_join2, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c->ev_forces, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c->ev_heavy, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c->ev_heavy_done, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c->ev_gathered, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c->ev_static, cudaEventDisableTiming));
    }
    return add_slots(c, descs, n_desc, true, room);
}

// Whether step `step` ends with the fused pass (its full update and the next
// step's half step in one pass over the nodes, the next step's contact forces
// computed beside its element forces): nothing falls between the two updates
// (no stable-dt check or mass scaling, active-list rebuild, non-finite or
// separation check, time-history record or frame at the next step's start),
// and the step is not the last one of this issue, so the state between calls
// is always a whole step's.
bool fuse_step(const crush_ctx* c, long long step, bool last) {
    if (!c->step_fusion || last) return false;
    const long long s1 = step + 1;
    if (s1 % 20 == 0) return false;
    if (c->adaptive && s1 % c->check_steps == 0) return false;
    if (c->any_separation && c->va.n_vehicles > 0 && s1 % 10 == 0) return false;
    if (c->hist_on && s1 % c->hist.steps == 0) return false;
    if (c->frames_on && s1 % c->frames.steps == 0) return false;
    return true;
}

// One explicit step of every slot on the stream (src/solver.rs:287-345).
// Phase boundaries of one step recorded when profiling: start, after dt,
// after contact, after half step, after element forces, after full step, end.
constexpr int N_PHASE_EVENTS = 7;

// Step `step`:
//   prologue (unless the previous step was fused, which did it): the active
//     lists, the stable-dt decision and mass scaling, the contact forces of
//     this step (its search ran beside the previous step) and the half step;
//   the next step's contact search on the side streams, reading this step's
//     X + u, beside the element forces; for a fused step the next step's
//     contact forces follow the search there, with the next step's dt;
//   the element forces;
//   fused: the fused pass (full update, the next step's half step, the
//     step's end); otherwise the full update, checks, the step's end and
//     records, with the next step's element dt pass beside the full update.
// Contact forces of even steps go to f_ext, of odd steps to f_ext_odd, and
// so do the penetration counters, so the next step's pass can run while
// this step's update still reads its own.
int enqueue_step(crush_ctx* c, long long step, cudaEvent_t* ev = nullptr, bool capturing = false, bool last = false) {
    ElementArrays el = c->el_run();
    NodeArrays nd = c->nd_step(step);
    ContactArrays cr = c->ca_step(step);
    const bool pre = c->prologue_done;
    const bool fuse = fuse_step(c, step, last);
    int n = 0;
    // Inside a stream capture an event record must be an external event node
    // for its timestamp to be readable after the graph runs.
    auto mark = [&](int i) {
        if (!ev) return;
        if (c->prof_level == 1 && i != 3 && i != 4) return;  // element-force kernel only
        if (capturing) cudaEventRecordWithFlags(ev[i], c->stream, cudaEventRecordExternal);
        else cudaEventRecord(ev[i], c->stream);
    };
    mark(0);
    if (!pre) {
        // Every 20 steps: the chunks that still hold a running crash.
        if (step % 20 == 0) {
            launch_build_active(c->stream, c->ab, c->ctls);
            ++n;
        }
        // Stable step check: the element pass ran at the end of the previous
        // step (or at run begin) on this step's X + u.
        if (c->adaptive && step % c->check_steps == 0) {
            launch_dt_finalize(c->stream, c->ctls, c->n_slots, c->mass_flag);
            launch_mass_scaling(c->stream, el, nd, c->ctls, 0);
            n += 2;
        }
    }
    mark(1);
    // Contact forces of this step from the search run beside the previous
    // step's forces (or at crush_run_begin for the first step).
    if (!pre && c->n_contacts > 0 && !c->contact_done) {
        launch_contact_finish(c->stream, cr, nd, c->ctls, 0, c->n_contacts, 0, c->n_faces, c->n_slaves, 0.0, c->mass, nd.f_ext, 1,
                              c->side2, c->ev_heavy, c->ev_heavy_done, c->ev_gathered);
        n += contact_finish_launches(c->n_slaves);
    }
    c->contact_done = false;
    // A separate step computes the next step's contact forces beside its
    // element forces when the next step has no stable-dt check (its dt is
    // then next_step_dt) and is issued with this one.
    const bool early = !fuse && c->early_contact && c->n_contacts > 0 && !last && !(c->adaptive && (step + 1) % c->check_steps == 0);
    mark(2);
    if (!pre) {
        launch_half(c->stream, nd, c->ctls);
        ++n;
    }
    mark(3);
    // The next step's contact search needs only its X + u, final now: it
    // runs on the side streams (static-grid entries on side2) beside the
    // element forces; a fused step's next contact forces follow it there.
    if (c->n_contacts > 0) {
        const ContactArrays cn = c->ca_step(step + 1);
        const NodeArrays nn = c->nd_step(step + 1);
        cudaEventRecord(c->ev_fork, c->stream);
        cudaStreamWaitEvent(c->side, c->ev_fork, 0);
        cudaStreamWaitEvent(c->side2, c->ev_fork, 0);
        launch_contact_search(c->side, cn, nn, c->ctls, 0, c->n_contacts, 0, c->n_faces, c->n_slaves, 0, c->ca.n_buckets, 1,
                              c->slave_lanes, c->side2);
        n += contact_search_launches(c->ca, true, c->n_faces, c->n_slaves, 0, c->ca.n_buckets, 0);
        if ((fuse && c->fused_contact_side) || early) {
            cudaEventRecord(c->ev_static, c->side2);
            cudaStreamWaitEvent(c->side, c->ev_static, 0);
            launch_contact_finish(c->side, cn, nn, c->ctls, 0, c->n_contacts, 0, c->n_faces, c->n_slaves, 0.0, c->mass, nn.f_ext, 1,
                                  c->side2, c->ev_heavy, c->ev_heavy_done, c->ev_gathered, 1);
            n += contact_finish_launches(c->n_slaves);
        }
        cudaEventRecord(c->ev_join, c->side);
        cudaEventRecord(c->ev_join2, c->side2);
    }
    launch_forces(c->stream, el, nd, c->ctls, 1, c->n_sms, c->forces_schedule, c->forces_queue);
    n += forces_launches(el);
    // The next step's element dt pass needs its X + u (final after the half
    // step) and this step's erosion (final after the forces): it runs on
    // side2 beside the full update.
    const bool dt_next = c->adaptive && (step + 1) % c->check_steps == 0;
    if (dt_next) {
        cudaEventRecord(c->ev_forces, c->stream);
        cudaStreamWaitEvent(c->side2, c->ev_forces, 0);
        launch_elem_dt(c->side2, el, nd, c->ctls, c->u, 1);
        ++n;
        cudaEventRecord(c->ev_join2, c->side2);
    }
    mark(4);
    if (fuse) {
        if (c->n_contacts > 0) {
            cudaStreamWaitEvent(c->stream, c->ev_join, 0);
            cudaStreamWaitEvent(c->stream, c->ev_join2, 0);
            if (!c->fused_contact_side) {
                // the next step's contact forces on the main stream, after
                // the element forces (the search ran beside them)
                const ContactArrays cn = c->ca_step(step + 1);
                const NodeArrays nn = c->nd_step(step + 1);
                launch_contact_finish(c->stream, cn, nn, c->ctls, 0, c->n_contacts, 0, c->n_faces, c->n_slaves, 0.0, c->mass, nn.f_ext,
                                      1, c->side2, c->ev_heavy, c->ev_heavy_done, c->ev_gathered, 1);
                n += contact_finish_launches(c->n_slaves);
                cudaEventRecord(c->ev_join2, c->side2);
                cudaStreamWaitEvent(c->stream, c->ev_join2, 0);
            }
        }
        launch_fused(c->stream, el, nd, c->ctls, cr, c->va, c->slot_done, c->mass_flag, c->fused_counter);
        ++n;
        mark(5);
        c->prologue_done = true;
        mark(6);
        return check_launch(c, n);
    }
    launch_full(c->stream, el, nd, c->ctls);
    ++n;
    mark(5);
    if ((step + 1) % 20 == 0) {
        launch_nonfinite(c->stream, nd, c->ctls);
        ++n;
    }
    const bool sep = c->any_separation && (step + 1) % 10 == 0 && c->va.n_vehicles > 0;
    if (sep) {
        launch_vehicle_vx(c->stream, c->va, c->mass, c->v, c->ctls);
        ++n;
    }
    if (early) {
        // the side streams' contact pass read this step's time: it ends
        // before the step's end moves it on
        cudaStreamWaitEvent(c->stream, c->ev_join, 0);
        cudaStreamWaitEvent(c->stream, c->ev_join2, 0);
    }
    launch_step_end(c->stream, c->ctls, cr, c->va, sep ? 1 : 0, c->slot_done, c->mass_flag);
    ++n;
    // Time-history records of the slots whose step is a multiple of
    // history_steps (src/solver.rs:349-351); u, v and the forces are final.
    if (c->hist_on && (step + 1) % c->hist.steps == 0) {
        launch_history(c->stream, c->hist, nd, c->ctls, nd.f_ext, HIST_STEP);
        n += (c->hist.n_pu > 0 ? 1 : 0) + 1;
    }
    // Frames at multiples of frame_steps (src/solver.rs:345-348).
    if (c->frames_on && (step + 1) % c->frames.steps == 0) {
        launch_frames(c->stream, c->frames, c->u, c->ctls, HIST_STEP);
        n += 3;
    }
    if (c->n_contacts > 0) {
        cudaStreamWaitEvent(c->stream, c->ev_join, 0);
        cudaStreamWaitEvent(c->stream, c->ev_join2, 0);
    } else if (dt_next) {
        cudaStreamWaitEvent(c->stream, c->ev_join2, 0);
    }
    c->prologue_done = false;
    c->contact_done = early;
    mark(6);
    return check_launch(c, n);
}

constexpr long long RETUNE_STEPS = 1000;
// Contexts at least this large time the element-kernel schedules on their
// own steps, once, at the run's start: which is fastest depends on how much
// of the next step's contact pass the element kernel's SMs hold back. The
// trial builds a graph per candidate (milliseconds each), which a run of a
// few hundred thousand elements does not win back (its candidates differ by
// a few percent of a 0.13 ms step); a large batch does.
constexpr long long SCHED_TRIAL_MIN_ELEMENTS = 2000000;


// The contact search at the open run's current X + u, on the main stream:
// what the next step's contact forces read (run begin, and after anything
// that reused the search buffers).
int search_now(crush_ctx* c) {
    if (c->n_contacts == 0) return CRUSH_OK;
    launch_contact_search(c->stream, c->ca, c->nd(), c->ctls, 0, c->n_contacts, 0, c->n_faces, c->n_slaves, 0, c->ca.n_buckets, 1,
                          c->slave_lanes);
    return check_launch(c, contact_search_launches(c->ca, true, c->n_faces, c->n_slaves, 0, c->ca.n_buckets, 0));
}

// The first step's contact search of contacts [k0, n_contacts) (added to the
// open run): the run's search over the tails of its lists — moving faces
// from dyn0, dynamic-grid and static-grid entries from gs0 and st0,
// exhaustive contacts from brute0 — and the new contacts' bucket range. The
// running slots' hits (found beside the last step) stay as they are; the
// search's shared bookkeeping is cleared as every search clears it.
int search_added(crush_ctx* c, int k0, long long dyn0, long long gs0, long long st0, int brute0) {
    if (c->n_contacts <= k0) return CRUSH_OK;
    if (c->ca.exhaustive) return search_now(c);
    ContactArrays v = c->ca;
    v.dyn_faces += dyn0;
    v.n_dyn_faces -= dyn0;
    v.grid_slaves += gs0;
    v.n_grid_slaves -= gs0;
    v.st_slaves += st0;
    v.n_st_slaves -= st0;
    v.brute_contacts += brute0;
    v.n_brute -= brute0;
    const long long bk0 = c->tab_off_h[k0], bk1 = c->tab_off_h[c->n_contacts];
    launch_contact_search(c->stream, v, c->nd(), c->ctls, k0, c->n_contacts, 0, c->n_faces, c->n_slaves, bk0, bk1, 1, c->slave_lanes);
    return check_launch(c, contact_search_launches(v, true, c->n_faces, c->n_slaves, bk0, bk1, 0));
}

// Launch autotuner: times the run's contact pass (at the open run's state,
// output into scratch, no state change) with 1, 2, 4, 8, 16 and 32 lanes per
// primary-node search, three passes each after a warm-up, and keeps the
// most lanes within 10 % of the fastest. Every choice finds the same hits;
// only the speed differs.
int autotune(crush_ctx* c) {
    c->tuned = true;
    for (double& x : c->tune_ms) x = 0.0;
    if (c->n_slaves == 0 || c->n_contacts == 0) return CRUSH_OK;
    cudaEvent_t t0, t1;
    CK(cudaEventCreate(&t0));
    CK(cudaEventCreate(&t1));
    const int options[6] = {1, 2, 4, 8, 16, 32};
    double best = INF;
    int best_lanes = c->slave_lanes;
    NodeArrays nd = c->nd();
    int st = CRUSH_OK;
    for (int k = 0; k < 6 && st == CRUSH_OK; ++k) {
        const int lanes = options[k];
        for (int rep = 0; rep < 4; ++rep) {
            if (rep == 1) cudaEventRecord(t0, c->stream);
            launch_contact(c->stream, c->ca, nd, c->ctls, 0, c->n_contacts, 0, c->n_faces, c->n_slaves, 0, c->ca.n_buckets, 0.0, c->mass,
                           c->f_tmp, 1, lanes);
            st = check_launch(c, contact_launches(c->ca, true, c->n_faces, c->n_slaves, 0, c->ca.n_buckets, 0));
            if (st != CRUSH_OK) break;
        }
        cudaEventRecord(t1, c->stream);
        cudaEventSynchronize(t1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t0, t1);
        c->tune_ms[k] = ms / 3.0;
        best = std::fmin(best, c->tune_ms[k]);
    }
    // The most lanes within 10 % of the fastest: a few timed passes are
    // noisy, and a slow pick costs far more than the margin (a 5000-step
    // refined run: 0.71 s with 32 lanes, 0.93 s with 1).
    for (int k = 0; k < 6; ++k)
        if (c->tune_ms[k] > 0.0 && c->tune_ms[k] <= 1.1 * best) best_lanes = options[k];
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (st != CRUSH_OK) return st;
    // The passes counted penetrations; the run starts from none.
    CK(cudaMemsetAsync(c->ca.pen_count, 0, sizeof(unsigned long long) * c->n_contacts, c->stream));
    CK(cudaMemsetAsync(c->ca.pen_max_bits, 0, sizeof(unsigned long long) * c->n_contacts, c->stream));
    if (best_lanes != c->slave_lanes) {
        c->slave_lanes = best_lanes;
        drop_graphs(c);
    }
    return CRUSH_OK;
}

// The step graph's period: the dt-check and active-list cadences and the
// recording cadences of histories and frames; no graph beyond 200 steps.
void update_period(crush_ctx* c) {
    long long p = c->base_period;
    if (p > 0 && c->hist_on) p = std::lcm(p, (long long)c->hist.steps);
    if (p > 0 && c->frames_on) p = std::lcm(p, (long long)c->frames.steps);
    c->period = p > 200 ? 0 : (int)p;
}

static void free_bufs(crush_ctx* c, std::vector<void*>& bufs) {
    if (!bufs.empty()) cudaStreamSynchronize(c->stream);
    for (void* p : bufs) {
        device_give(c->device, p, c->alloc_bytes[p]);
        c->alloc_bytes.erase(p);
        c->allocs.erase(std::remove(c->allocs.begin(), c->allocs.end(), p), c->allocs.end());
    }
    bufs.clear();
}

// Device structures of the frames from the slots' configuration.
int rebuild_frames(crush_ctx* c) {
    free_bufs(c, c->frame_bufs);
    c->frames = FrameArrays{};
    c->frames_ran = false;
    drop_graphs(c);
    int steps = 0;
    long long stride = 0, max3n = 1, maxe = 1;
    std::vector<int> on(c->n_slots);
    std::vector<long long> smax(c->n_slots), node0(c->n_slots), nn(c->n_slots), elem0(c->n_slots), ne(c->n_slots),
        dbase(c->n_slots), ebase(c->n_slots);
    long long dtot = 0, etot = 0;
    for (int k = 0; k < c->n_slots; ++k) {
        const Slot& sl = c->slots[k];
        on[k] = c->frame_steps[k] > 0;
        smax[k] = on[k] ? c->frame_max[k] : 0;
        if (on[k]) {
            steps = c->frame_steps[k];
            stride = std::max(stride, smax[k]);
            max3n = std::max(max3n, 3 * sl.n_nodes);
            maxe = std::max(maxe, sl.n_elems);
        }
        node0[k] = sl.node0;
        nn[k] = sl.n_nodes;
        elem0[k] = sl.elem0;
        ne[k] = sl.n_elems;
        dbase[k] = dtot;
        ebase[k] = etot;
        dtot += smax[k] * 3 * sl.n_nodes;
        etot += smax[k] * sl.n_elems;
    }
    c->frames_on = steps > 0;
    c->frames.steps = steps;
    update_period(c);
    if (!c->frames_on) return CRUSH_OK;
    FrameArrays& f = c->frames;
    f.n_slots = c->n_slots;
    f.steps = steps;
    f.stride = stride;
    f.hc_index = c->hc_index_d;
    f.eroded_all = c->eroded_all;
    f.state = c->state;
    f.state_stride = c->stride;
    f.sc_index = c->n_sc > 0 ? c->sc_index_d : nullptr;
    f.n_sc = c->sc_stride;  // the plane stride of the scalar geometry
    f.sc_geo = c->sc_geo;
    f.sc_mat = c->sc_mat;
    f.conn_all = c->conn_all;
    f.pos = c->pos;
    f.node_blocks = (int)std::min<long long>(1024, (max3n + 4095) / 4096);
    f.elem_blocks = (int)std::min<long long>(1024, (maxe + 2047) / 2048);
    const size_t mark = c->allocs.size();
    int st = CRUSH_OK;
    if (st == CRUSH_OK) st = c->upload_const(&f.slot_on, on);
    if (st == CRUSH_OK) st = c->upload_const(&f.slot_max, smax);
    if (st == CRUSH_OK) st = c->upload_const(&f.node0, node0);
    if (st == CRUSH_OK) st = c->upload_const(&f.n_nodes, nn);
    if (st == CRUSH_OK) st = c->upload_const(&f.elem0, elem0);
    if (st == CRUSH_OK) st = c->upload_const(&f.n_elems, ne);
    if (st == CRUSH_OK) st = c->upload_const(&f.disp_base, dbase);
    if (st == CRUSH_OK) st = c->upload_const(&f.elem_base, ebase);
    if (st == CRUSH_OK) st = c->alloc(&f.count, c->n_slots);
    if (st == CRUSH_OK) st = c->alloc(&f.last_step, c->n_slots);
    if (st == CRUSH_OK) st = c->alloc(&f.time, (size_t)c->n_slots * stride);
    if (st == CRUSH_OK) st = c->alloc(&f.step, (size_t)c->n_slots * stride);
    if (st == CRUSH_OK) st = c->alloc(&f.disp, (size_t)std::max<long long>(dtot, 1));
    if (st == CRUSH_OK) st = c->alloc(&f.pstrain, (size_t)std::max<long long>(etot, 1));
    if (st == CRUSH_OK) st = c->alloc(&f.stress, 6 * (size_t)std::max<long long>(etot, 1));
    if (st == CRUSH_OK) st = c->alloc(&f.eroded, (size_t)std::max<long long>(etot, 1));
    c->frame_bufs.assign(c->allocs.begin() + (long)mark, c->allocs.end());
    if (st != CRUSH_OK) {
        free_bufs(c, c->frame_bufs);
        c->frames = FrameArrays{};
        c->frames_on = false;
        update_period(c);
        return st;
    }
    CK(cudaMemsetAsync(f.count, 0, sizeof(long long) * c->n_slots, c->stream));
    CK(cudaMemsetAsync(f.last_step, 0xFF, sizeof(long long) * c->n_slots, c->stream));  // -1
    return sync(c);
}

// Device structures of the time histories from the slots' configuration:
// part units (each recording slot's parts and their element nodes, from the
// device connectivity), accelerometer nodes and frames, record buffers.
int rebuild_history(crush_ctx* c) {
    free_bufs(c, c->hist_bufs);
    c->hist = HistoryArrays{};
    c->hist_ran = false;
    drop_graphs(c);
    int steps = 0;
    long long stride = 0;
    for (int k = 0; k < c->n_slots; ++k)
        if (c->hist_steps[k] > 0) {
            steps = c->hist_steps[k];
            stride = std::max(stride, c->hist_max[k]);
        }
    c->hist_on = steps > 0;
    c->hist.steps = steps;
    update_period(c);
    if (!c->hist_on) return CRUSH_OK;
    std::vector<int> on(c->n_slots), pu_slot_off(c->n_slots + 1, 0), an_off(c->n_slots + 1, 0), pu_slot, an_frame;
    std::vector<long long> smax(c->n_slots, 0);
    std::vector<uint32_t> pu_off(1, 0), pu_nodes, an_node, fr_nodes;
    for (int k = 0; k < c->n_slots; ++k) {
        const Slot& sl = c->slots[k];
        on[k] = c->hist_steps[k] > 0;
        smax[k] = on[k] ? c->hist_max[k] : 0;
        if (on[k]) {
            // part_nodes (src/mesh.rs:74-82): ascending nodes of each part's elements
            std::vector<int32_t> part(sl.n_elems);
            std::vector<uint32_t> conn(8 * sl.n_elems);
            CK(cudaMemcpy(part.data(), c->part + sl.elem0, sizeof(int32_t) * sl.n_elems, cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(conn.data(), c->conn_all + 8 * sl.elem0, sizeof(uint32_t) * 8 * sl.n_elems, cudaMemcpyDeviceToHost));
            std::vector<std::vector<uint32_t>> nodes(sl.n_parts);
            for (long long e = 0; e < sl.n_elems; ++e) {
                const int p = part[e] - sl.part0;
                if (p >= 0 && p < sl.n_parts) nodes[p].insert(nodes[p].end(), conn.begin() + 8 * e, conn.begin() + 8 * e + 8);
            }
            for (auto& v : nodes) {
                std::sort(v.begin(), v.end());
                v.erase(std::unique(v.begin(), v.end()), v.end());
                pu_nodes.insert(pu_nodes.end(), v.begin(), v.end());
                pu_off.push_back((uint32_t)pu_nodes.size());
                pu_slot.push_back(k);
            }
            for (const HistAccel& a : c->hist_acc[k]) {
                int f = -1;
                if (a.has_frame) {
                    f = (int)(fr_nodes.size() / 3);
                    for (int j = 0; j < 3; ++j) fr_nodes.push_back((uint32_t)(sl.node0 + a.frame[j]));
                }
                for (uint32_t n : a.nodes) {
                    an_node.push_back((uint32_t)(sl.node0 + n));
                    an_frame.push_back(f);
                }
            }
        }
        pu_slot_off[k + 1] = (int)pu_slot.size();
        an_off[k + 1] = (int)an_node.size();
    }
    HistoryArrays& h = c->hist;
    h.n_slots = c->n_slots;
    h.steps = steps;
    h.max_rec = stride;
    h.n_pu = (int)pu_slot.size();
    h.n_an = (int)an_node.size();
    const size_t mark = c->allocs.size();
    auto up = [&](auto** dst, const auto& v) { return c->upload_const(dst, v); };
    int st = CRUSH_OK;
    if (st == CRUSH_OK) st = up(&h.slot_on, on);
    if (st == CRUSH_OK) st = up(&h.slot_max, smax);
    if (st == CRUSH_OK) st = up(&h.slot_pu_off, pu_slot_off);
    if (st == CRUSH_OK) st = up(&h.slot_an_off, an_off);
    if (st == CRUSH_OK) st = up(&h.pu_off, pu_off);
    if (st == CRUSH_OK) st = up(&h.pu_nodes, pu_nodes);
    if (st == CRUSH_OK) st = up(&h.pu_slot, pu_slot);
    if (st == CRUSH_OK) st = up(&h.an_node, an_node);
    if (st == CRUSH_OK) st = up(&h.an_frame, an_frame);
    if (st == CRUSH_OK) st = up(&h.fr_nodes, fr_nodes);
    if (st == CRUSH_OK) st = c->alloc(&h.partial, (size_t)std::max(h.n_pu, 1) * HIST_BLOCKS * HIST_PART_VALUES);
    if (st == CRUSH_OK) st = c->alloc(&h.rec_count, c->n_slots);
    if (st == CRUSH_OK) st = c->alloc(&h.last_step, c->n_slots);
    if (st == CRUSH_OK) st = c->alloc(&h.rec_time, (size_t)c->n_slots * stride);
    if (st == CRUSH_OK) st = c->alloc(&h.rec_step, (size_t)c->n_slots * stride);
    if (st == CRUSH_OK) st = c->alloc(&h.part_rec, (size_t)std::max(h.n_pu, 1) * stride * HIST_PART_VALUES);
    if (st == CRUSH_OK) st = c->alloc(&h.node_rec, (size_t)std::max(h.n_an, 1) * stride * HIST_NODE_VALUES);
    c->hist_bufs.assign(c->allocs.begin() + (long)mark, c->allocs.end());
    if (st != CRUSH_OK) return st;
    CK(cudaMemsetAsync(h.rec_count, 0, sizeof(long long) * c->n_slots, c->stream));
    CK(cudaMemsetAsync(h.last_step, 0xFF, sizeof(long long) * c->n_slots, c->stream));  // -1
    return sync(c);
}

// A slot's control block at the start of its run (src/solver.rs:214-252).
Control initial_control(const Slot& sl) {
    Control x;
    std::memset(&x, 0, sizeof(x));
    x.t = 0.0;
    x.end_time = sl.settings.end_time;
    x.dt_cfl = sl.dt0;
    x.dt_min = INF;
    x.dt_floor = sl.dt_floor;
    x.dt_scale = sl.settings.dt_scale;
    x.contact_dt = sl.contact_dt;
    x.damping = sl.settings.velocity_damping;
    x.dt_stable_bits = INF_BITS;
    x.step = 0;
    x.last_hit = -1;
    x.max_steps = sl.settings.max_steps;
    x.done = (0.0 < sl.settings.end_time) ? 0 : 1;
    x.stop_rule = sl.settings.stop_rule;
    return x;
}

int run_begin(crush_ctx* c) {
    const long long N = c->n_nodes;
    drop_graphs(c);
    CK(cudaMemsetAsync(c->u, 0, sizeof(double) * 3 * N, c->stream));
    CK(cudaMemcpyAsync(c->v, c->v0, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemsetAsync(c->v_half, 0, sizeof(double) * 3 * N, c->stream));
    CK(cudaMemsetAsync(c->f_ext, 0, sizeof(double) * 3 * N, c->stream));
    CK(cudaMemsetAsync(c->f_ext_odd, 0, sizeof(double) * 3 * N, c->stream));
    CK(cudaMemsetAsync(c->added, 0, sizeof(double) * N, c->stream));
    CK(cudaMemsetAsync(c->fused_counter, 0, sizeof(unsigned), c->stream));
    c->prologue_done = false;
    c->contact_done = false;
    if (c->n_contacts > 0) {
        CK(cudaMemsetAsync(c->ca.big_best, 0x7F, sizeof(int) * std::max<long long>(c->n_slaves, 1), c->stream));  // BIG_NONE
        CK(cudaMemsetAsync(c->ca.pen_count, 0, sizeof(unsigned long long) * 2 * c->pen_stride, c->stream));
        CK(cudaMemsetAsync(c->ca.pen_max_bits, 0, sizeof(unsigned long long) * 2 * c->pen_stride, c->stream));
    }
    CK(cudaMemsetAsync(c->eroded_all, 0, c->n_all, c->stream));
    launch_init_state(c->stream, 0, c->n_hc, c->stride, c->state);
    launch_node_masses(c->stream, N, c->all_off, c->all_slot, c->lumped, c->mass, c->inv_mass);
    int st = check_launch(c, 2);
    if (st != CRUSH_OK) return st;
    std::vector<Control> h(c->n_slots);
    for (int k = 0; k < c->n_slots; ++k) h[k] = initial_control(c->slots[k]);
    CK(cudaMemcpyAsync(c->ctls, h.data(), sizeof(Control) * h.size(), cudaMemcpyHostToDevice, c->stream));
    // Initial internal forces at u = 0 (src/solver.rs:254); the count of
    // elements it erodes is not added to the run's total (as there).
    launch_forces(c->stream, c->el(), c->nd(), c->ctls, 0);
    launch_gather(c->stream, c->el(), c->nd(), c->f_int);
    st = check_launch(c, forces_launches(c->el()) + 1);
    if (st != CRUSH_OK) return st;
    // Geometry of every contact face at u = 0; static faces keep it.
    launch_contact_geometry(c->stream, c->ca, c->nd(), 0, c->n_contacts, 0, c->n_faces);
    st = check_launch(c, c->n_faces > 0 ? 1 : 0);
    if (st != CRUSH_OK) return st;
    CK(cudaMemcpyAsync(c->ctls, h.data(), sizeof(Control) * h.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(c->mass_flag, 0, sizeof(int), c->stream));
    if (c->adaptive) {
        // Step 0's element dt pass (each step runs the next check's pass).
        launch_elem_dt(c->stream, c->el(), c->nd(), c->ctls, c->u, 1);
        st = check_launch(c);
        if (st != CRUSH_OK) return st;
    }
    c->done_h.resize(c->n_slots);
    for (int k = 0; k < c->n_slots; ++k) c->done_h[k] = h[k].done;
    CK(cudaMemcpyAsync(c->slot_done, c->done_h.data(), sizeof(int) * c->n_slots, cudaMemcpyHostToDevice, c->stream));
    c->host_step = 0;
    c->last_tune_step = 0;
    c->run_open = true;
    c->sched_trial_pending = !c->tuning_fixed && c->n_hc >= SCHED_TRIAL_MIN_ELEMENTS;
    if (!c->tuned && !c->tuning_fixed) {
        st = autotune(c);
        if (st != CRUSH_OK) return st;
    }
    st = search_now(c);
    if (st != CRUSH_OK) return st;
    if (c->hist_on) {
        // The run's first record (src/solver.rs:283-286): accelerations from
        // the step-0 forces, contact included (the contact pass at u = 0 with
        // the first dt, src/solver.rs:257-262), into scratch.
        CK(cudaMemsetAsync(c->hist.rec_count, 0, sizeof(long long) * c->n_slots, c->stream));
        CK(cudaMemsetAsync(c->hist.last_step, 0xFF, sizeof(long long) * c->n_slots, c->stream));
        CK(cudaMemsetAsync(c->f_tmp, 0, sizeof(double) * 3 * N, c->stream));
        if (c->n_contacts > 0) {
            launch_contact_finish(c->stream, c->ca, c->nd(), c->ctls, 0, c->n_contacts, 0, c->n_faces, c->n_slaves,
                                  0.0, c->mass, c->f_tmp, 1);
            st = check_launch(c, contact_finish_launches(c->n_slaves));
            if (st != CRUSH_OK) return st;
            // that pass counted penetrations; the run starts from none
            CK(cudaMemsetAsync(c->ca.pen_count, 0, sizeof(unsigned long long) * c->n_contacts, c->stream));
            CK(cudaMemsetAsync(c->ca.pen_max_bits, 0, sizeof(unsigned long long) * c->n_contacts, c->stream));
        }
        launch_history(c->stream, c->hist, c->nd(), c->ctls, c->f_tmp, HIST_INITIAL);
        st = check_launch(c, (c->hist.n_pu > 0 ? 1 : 0) + 1);
        if (st != CRUSH_OK) return st;
        c->hist_ran = true;
    }
    if (c->frames_on) {
        // the run's first frame (src/solver.rs:265-276), after the step-0 forces
        CK(cudaMemsetAsync(c->frames.count, 0, sizeof(long long) * c->n_slots, c->stream));
        CK(cudaMemsetAsync(c->frames.last_step, 0xFF, sizeof(long long) * c->n_slots, c->stream));
        launch_frames(c->stream, c->frames, c->u, c->ctls, HIST_INITIAL);
        st = check_launch(c, 3);
        if (st != CRUSH_OK) return st;
        c->frames_ran = true;
    }
    return sync(c);
}

// Slots [s0, s1) (the context's last ones, added while its run is open)
// begin their run as crush_run_begin begins every slot's: zero
// displacement, initial velocities, masses, state, the initial internal
// forces at u = 0, the static faces' geometry and the element dt pass of
// their step 0 (the caller then runs the contact search their first step's
// forces read, on the main stream: its scratch is the steps'). They join at
// the run's current step, a step-graph boundary, so their own steps fall on
// the same step-schedule positions as alone.
int begin_slots(crush_ctx* c, int s0, int s1) {
    if (s1 <= s0) return CRUSH_OK;
    const Slot& a = c->slots[s0];
    const Slot& z = c->slots[s1 - 1];
    const long long n0 = a.node0, n1 = z.node0 + z.n_nodes, e0 = a.elem0;
    const long long h0 = a.hc0, h1 = z.hc0 + z.n_hc, q0 = a.sc0, q1 = z.sc0 + z.n_sc;
    const long long nn = n1 - n0;
    CK(cudaMemsetAsync(c->u + 3 * n0, 0, sizeof(double) * 3 * nn, c->stream));
    CK(cudaMemcpyAsync(c->v + 3 * n0, c->v0 + 3 * n0, sizeof(double) * 3 * nn, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemsetAsync(c->v_half + 3 * n0, 0, sizeof(double) * 3 * nn, c->stream));
    CK(cudaMemsetAsync(c->f_ext + 3 * n0, 0, sizeof(double) * 3 * nn, c->stream));
    CK(cudaMemsetAsync(c->f_ext_odd + 3 * n0, 0, sizeof(double) * 3 * nn, c->stream));
    CK(cudaMemsetAsync(c->added + n0, 0, sizeof(double) * nn, c->stream));
    CK(cudaMemsetAsync(c->eroded_all + e0, 0, c->n_all - e0, c->stream));
    launch_init_state(c->stream, h0, h1, c->stride, c->state);
    launch_node_masses(c->stream, nn, c->all_off + n0, c->all_slot, c->lumped, c->mass + n0, c->inv_mass + n0);
    int st = check_launch(c, 2);
    if (st != CRUSH_OK) return st;
    std::vector<Control> h(s1 - s0);
    std::vector<int> done(s1 - s0);
    for (int k = s0; k < s1; ++k) {
        h[k - s0] = initial_control(c->slots[k]);
        done[k - s0] = h[k - s0].done;
    }
    CK(cudaMemcpyAsync(c->ctls + s0, h.data(), sizeof(Control) * h.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->slot_done + s0, done.data(), sizeof(int) * done.size(), cudaMemcpyHostToDevice, c->stream));
    // Initial internal forces at u = 0 of the slots' elements (src/solver.rs:254)
    // and their nodes' f_int: the element arrays and the node rows seen from
    // the slots' first entries.
    ElementArrays w = c->el();
    w.planes += h0;
    w.state += h0;
    w.corner += 24 * h0;
    w.n_hc = h1 - h0;
    w.sc_model += q0;
    w.sc_geo += q0;
    w.sc_mat += 2 * q0;
    w.sc_corner += 24 * q0;
    w.n_sc = w.sc_count = q1 - q0;
    launch_forces(c->stream, w, c->nd(), c->ctls, 0);
    NodeArrays wn = c->nd();
    wn.n = nn;
    wn.hc_ell += 2 * n0;
    wn.hc_off += n0;
    wn.sc_off += n0;
    launch_gather(c->stream, c->el(), wn, c->f_int + 3 * n0);
    st = check_launch(c, forces_launches(w) + 1);
    if (st != CRUSH_OK) return st;
    const int c0 = a.contact0, c1 = z.contact0 + z.n_contacts;
    if (c1 > c0) {
        const long long f0 = a.face0, nf = z.face0 + z.n_faces - f0;
        launch_contact_geometry(c->stream, c->ca, c->nd(), c0, c1, f0, nf);
        st = check_launch(c, nf > 0 ? 1 : 0);
        if (st != CRUSH_OK) return st;
    }
    // the element dt pass of the slots' step 0 (a step-graph boundary is a
    // stable-dt check step), and the same data's control copy
    CK(cudaMemcpyAsync(c->ctls + s0, h.data(), sizeof(Control) * h.size(), cudaMemcpyHostToDevice, c->stream));
    if (c->adaptive) {
        launch_elem_dt(c->stream, c->el(), c->nd(), c->ctls, c->u, 1, e0);
        st = check_launch(c);
        if (st != CRUSH_OK) return st;
    }
    return CRUSH_OK;
}

int ensure_prof_events(crush_ctx* c) {
    size_t want = (size_t)std::max(c->period, 1) * N_PHASE_EVENTS;
    while (c->prof_ev.size() < want) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        c->prof_ev.push_back(e);
    }
    return CRUSH_OK;
}

int build_graph(crush_ctx* c) {
    if (c->profiling) {
        int st0 = ensure_prof_events(c);
        if (st0 != CRUSH_OK) return st0;
    }
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int st = CRUSH_OK;
    for (int k = 0; k < c->period && st == CRUSH_OK; ++k)
        st = enqueue_step(c, k, c->profiling ? &c->prof_ev[(size_t)k * N_PHASE_EVENTS] : nullptr, true);
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (st != CRUSH_OK) return st;
    if (c->prologue_done || c->contact_done) {  // the period's last step has a stable-dt check next: never fused nor early
        cudaGraphDestroy(g);
        c->prologue_done = false;
        c->contact_done = false;
        return crush::fail(CRUSH_ERR_INVALID, "step graph period ends on a fused step");
    }
    if (e != cudaSuccess) return crush::fail(CRUSH_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&c->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return crush::fail(CRUSH_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    return CRUSH_OK;
}

// The step graph of element-kernel schedule `schedule`, built if missing
// (the other schedule's graph is kept for switching back).
// Whether the step graph of the schedule the next issue uses is built.
bool graph_ready(const crush_ctx* c) { return c->graphs[c->tuning_fixed ? N_CANDS : c->cand] != nullptr; }

int select_schedule(crush_ctx* c, int cand) {
    int slot = N_CANDS;  // schedules the caller set
    if (!c->tuning_fixed) {
        c->cand = cand;
        c->step_fusion = CANDS[cand].fused;
        c->forces_schedule = CANDS[cand].forces;
        c->early_contact = CANDS[cand].early;
        c->fused_contact_side = false;
        slot = cand;
    }
    c->graph = c->graphs[slot];
    if (!c->graph) {
        int64_t before = c->launches;
        int st = build_graph(c);
        if (st != CRUSH_OK) return st;
        c->graphs[slot] = c->graph;
        c->graph_launches = c->launches - before;
        c->launches = before;
    }
    return CRUSH_OK;
}

// Schedule trial: 2 x N_CANDS graph periods of the run's own steps, cycling
// through the candidate step schedules (all compute the same bits), each
// timed by events on the stream (every candidate's graph is built first, so
// no host work falls between them); the fastest is kept.
int schedule_trial(crush_ctx* c) {
    c->sched_trial_pending = false;
    const int keep = c->cand;
    int st = CRUSH_OK;
    for (int k = 0; k < N_CANDS && st == CRUSH_OK; ++k) st = select_schedule(c, k);
    if (st != CRUSH_OK) return st;
    constexpr int RUNS = 2 * N_CANDS;
    cudaEvent_t ev[RUNS + 1];
    for (auto& e : ev) CK(cudaEventCreate(&e));
    for (int k = 0; k < RUNS && st == CRUSH_OK; ++k) {
        st = select_schedule(c, k % N_CANDS);
        if (st != CRUSH_OK) break;
        CK(cudaEventRecord(ev[k], c->stream));
        CK(cudaGraphLaunch(c->graph, c->stream));
        c->launches += c->graph_launches;
        c->host_step += c->period;
    }
    if (st == CRUSH_OK) {
        CK(cudaEventRecord(ev[RUNS], c->stream));
        CK(cudaEventSynchronize(ev[RUNS]));
        double ms[N_CANDS] = {};
        for (int k = 0; k < RUNS; ++k) {
            float x = 0.f;
            cudaEventElapsedTime(&x, ev[k], ev[k + 1]);
            ms[k % N_CANDS] += x / (2.0 * c->period);
        }
        int best = keep;
        for (int k = 0; k < N_CANDS; ++k) {
            c->sched_ms[k] = ms[k];
            if (ms[k] < ms[best]) best = k;
        }
        st = select_schedule(c, best);
    }
    for (auto& e : ev) cudaEventDestroy(e);
    c->last_was_graph = true;
    return st;
}

// Issue n_steps steps (graphs where the step index is on a period boundary).
int issue_steps(crush_ctx* c, long long n_steps) {
    if (!c->run_open) return crush::fail(CRUSH_ERR_INVALID, "no open run (call crush_run_begin)");
    long long issued = 0;
    int st;
    while (issued < n_steps) {
        // Crushed faces change the contact search as a run goes on: re-tune
        // every RETUNE_STEPS steps, on a graph boundary.
        if (!c->tuning_fixed && c->host_step - c->last_tune_step >= RETUNE_STEPS && (c->period == 0 || c->host_step % c->period == 0)) {
            st = autotune(c);
            if (st != CRUSH_OK) return st;
            c->last_tune_step = c->host_step;
        }
        // A graph that is not built yet is built for an issue of two periods
        // or more, or at the second period since the graphs were dropped:
        // the first single period after slots joined is launched step by
        // step, which costs the host less than capturing and instantiating a
        // graph that the next join drops.
        const bool boundary = c->period > 0 && c->host_step % c->period == 0 && n_steps - issued >= c->period && !c->prologue_done &&
                              !c->contact_done;
        const bool use_graph = boundary && (graph_ready(c) || c->eager_periods > 0 || n_steps - issued >= 2 * (long long)c->period);
        if (boundary && !use_graph) ++c->eager_periods;
        if (use_graph && c->sched_trial_pending && !c->tuning_fixed && n_steps - issued >= 2 * N_CANDS * (long long)c->period) {
            st = schedule_trial(c);
            if (st != CRUSH_OK) return st;
            issued += 2 * N_CANDS * (long long)c->period;
        } else if (use_graph) {
            st = select_schedule(c, c->cand);
            if (st != CRUSH_OK) return st;
            CK(cudaGraphLaunch(c->graph, c->stream));
            c->launches += c->graph_launches;
            c->host_step += c->period;
            issued += c->period;
            c->last_was_graph = true;
        } else {
            if (c->profiling) {
                st = ensure_prof_events(c);
                if (st != CRUSH_OK) return st;
            }
            st = enqueue_step(c, c->host_step, c->profiling ? &c->prof_ev[0] : nullptr, false, issued + 1 == n_steps);
            if (st != CRUSH_OK) return st;
            c->host_step += 1;
            issued += 1;
            c->last_was_graph = false;
        }
    }
    return CRUSH_OK;
}

// Whether every slot has finished (device flags read back; synchronises).
int all_done(crush_ctx* c, int* done) {
    c->done_h.resize(c->n_slots);
    CK(cudaMemcpyAsync(c->done_h.data(), c->slot_done, sizeof(int) * c->n_slots, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    int d = 1;
    for (int x : c->done_h) d &= x ? 1 : 0;
    *done = d;
    return CRUSH_OK;
}

int run_steps(crush_ctx* c, long long n_steps, int* done) {
    int st = issue_steps(c, n_steps);
    if (st != CRUSH_OK) return st;
    int d = 0;
    st = all_done(c, &d);
    if (st != CRUSH_OK) return st;
    if (done) *done = d;
    return CRUSH_OK;
}

// Results of slots [s0, s1) into r[0, s1 - s0): one FP64 vehicle-sum launch
// and one gather of the u_x values the crush measure needs, then the
// per-vehicle arithmetic on the host (src/bin/crushrs.rs:237-271).
int results_range(crush_ctx* c, int s0, int s1, crush_results* r) {
    if (s0 < 0 || s1 > c->n_slots || s0 >= s1) return crush::fail(CRUSH_ERR_INVALID, "slot out of range");
    std::vector<Control> h(s1 - s0);
    CK(cudaMemcpyAsync(h.data(), c->ctls + s0, sizeof(Control) * h.size(), cudaMemcpyDeviceToHost, c->stream));
    // only the vehicles of slots [s0, s1) (consecutive, in slot order) and their crush-measure nodes
    const int v0 = c->slots[s0].vehicle0, v1 = c->slots[s1 - 1].vehicle0 + c->slots[s1 - 1].n_vehicles;
    const size_t q0 = c->crush_off_h[v0], q1 = c->crush_off_h[v1];
    std::vector<double> sums(7 * (size_t)std::max(c->va.n_vehicles, 1)), ux(std::max<size_t>(c->crush_nodes_h.size(), 1));
    if (v1 > v0) {
        VehicleArrays vr = c->va;
        vr.n_vehicles = v1 - v0;
        vr.off += v0;
        vr.slot += v0;
        vr.local += v0;
        launch_vehicle_sums(c->stream, vr, c->mass, c->v, c->v0, c->veh_out + 7 * (size_t)v0);
        launch_gather_ux(c->stream, (long long)(q1 - q0), c->crush_nodes + q0, c->u, c->crush_ux + q0);
        int st = check_launch(c, 2);
        if (st != CRUSH_OK) return st;
        CK(cudaMemcpyAsync(sums.data() + 7 * (size_t)v0, c->veh_out + 7 * (size_t)v0, sizeof(double) * 7 * (v1 - v0), cudaMemcpyDeviceToHost,
                           c->stream));
        if (q1 > q0)
            CK(cudaMemcpyAsync(ux.data() + q0, c->crush_ux + q0, sizeof(double) * (q1 - q0), cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    for (int slot = s0; slot < s1; ++slot) {
        const Control& x = h[slot - s0];
        const Slot& sl = c->slots[slot];
        crush_results* out = r + (slot - s0);
        std::memset(out, 0, sizeof(*out));
        out->time = x.t;
        out->steps = x.step;
        out->eroded_elements = x.eroded_total;
        out->dt_min = x.dt_min;
        out->added_mass_max = x.added_mass_max;
        out->status = x.status;
        out->n_vehicles = sl.n_vehicles;
        for (int k = 0; k < sl.n_vehicles; ++k) {
            const int gv = sl.vehicle0 + k;
            const double* sv = sums.data() + 7 * gv;
            crush_vehicle_result& vr = out->vehicle[k];
            vr.mass = sv[0];
            for (int dd = 0; dd < 3; ++dd) {
                double v1 = sv[0] > 0.0 ? sv[1 + dd] / sv[0] : 0.0;
                double v0 = sv[0] > 0.0 ? sv[4 + dd] / sv[0] : 0.0;
                vr.velocity[dd] = v1;
                vr.delta_v[dd] = v1 - v0;
            }
            // u_x of the front nodes in order, then of the accelerometer
            const size_t f0 = c->crush_off_h[gv], f1 = c->crush_off_h[gv + 1] - 1;
            double fu = 0.0;
            for (size_t q = f0; q < f1; ++q) fu += ux[q];
            fu = f1 > f0 ? fu / (double)(f1 - f0) : 0.0;
            vr.crush = std::fabs(ux[f1] - fu);
        }
    }
    return CRUSH_OK;
}

int results(crush_ctx* c, int slot, crush_results* r) { return results_range(c, slot, slot + 1, r); }

int reset_aux(crush_ctx* c, double dt_floor) {
    std::vector<Control> aux(c->n_slots);
    std::memset(aux.data(), 0, sizeof(Control) * aux.size());
    for (Control& a : aux) {
        a.dt_stable_bits = INF_BITS;
        a.dt_floor = dt_floor;
    }
    CK(cudaMemcpyAsync(c->ctls_aux, aux.data(), sizeof(Control) * aux.size(), cudaMemcpyHostToDevice, c->stream));
    return CRUSH_OK;
}

int read_aux(crush_ctx* c, std::vector<Control>* aux) {
    aux->resize(c->n_slots);
    CK(cudaMemcpyAsync(aux->data(), c->ctls_aux, sizeof(Control) * aux->size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return CRUSH_OK;
}

int run_to_end(crush_ctx* c) {
    int st = run_begin(c);
    if (st != CRUSH_OK) return st;
    int done = 0;
    // chunks long enough for the schedule trial (2 rounds of the candidates, a period each)
    const long long chunk = c->period > 0 ? 2 * N_CANDS * (long long)c->period : 200;
    long long total = 0;
    long long cap = 0;
    for (const Slot& sl : c->slots) cap = std::max<long long>(cap, sl.settings.max_steps > 0 ? sl.settings.max_steps : 2000000ll);
    cap += chunk;
    // A run that has not finished after this many steps is returned as a timeout.
    while (!done && total < cap) {
        st = run_steps(c, chunk, &done);
        if (st != CRUSH_OK) return st;
        total += chunk;
    }
    if (!done) return crush::fail(CRUSH_ERR_TIMEOUT, "run did not finish within " + std::to_string(cap) + " steps");
    return CRUSH_OK;
}

// Set-up of a batch pipelined with its run (crush_batch_solve): a context
// with room for every model is created from the first eighth of the
// elements and begins its run; each later eighth joins the open run at a
// step-graph boundary (crush_batch_append's path: its host set-up runs
// while the steps issued before it run, its device set-up on the set-up
// stream), so the set-up of all but the first group is hidden behind the
// run. Every model's results equal its own run
// (a slot's steps do not depend on when it joined). Models that the room
// estimate cannot take run in a further context after this one.
int solve_models(const crush_model_desc* const* descs, int n, int device, crush_results* out) {
    long long total = 0;
    crush_capacity room{};
    room.slots = n;
    for (int k = 0; k < n; ++k) {
        const crush_model_desc* d = descs[k];
        room.nodes += std::max<int64_t>(d->n_nodes, 0);
        room.hexes += std::max<int64_t>(d->n_hexes, 0);
        room.contacts += std::max(d->n_contacts, 0);
        for (int q = 0; q < d->n_contacts && d->contacts; ++q) {
            room.faces += std::max<int64_t>(d->contacts[q].n_faces, 0);
            room.primary_nodes += std::max<int64_t>(d->contacts[q].n_nodes, 0);
        }
        total += std::max<int64_t>(d->n_hexes, 1);
    }
    constexpr int GROUPS = 8;
    // group ends: model k closes group g when the running element count reaches g / GROUPS of the total
    std::vector<int> ends;
    long long acc = 0;
    for (int k = 0; k < n; ++k) {
        acc += std::max<int64_t>(descs[k]->n_hexes, 1);
        if (k == n - 1 || acc * GROUPS >= total * (long long)(ends.size() + 1)) ends.push_back(k + 1);
    }
    std::unique_ptr<crush_ctx> c(new crush_ctx());
    int st = create_impl(descs, ends[0], device, c.get(), &room);
    if (st != CRUSH_OK) return st;
    st = run_begin(c.get());
    if (st != CRUSH_OK) return st;
    int placed = ends[0];
    const long long per = c->period > 0 ? c->period : 20;
    // Periods issued before each group joins: doubled (up to 8) whenever the
    // device finished them before the group's set-up did.
    long long periods = 1;
    cudaEvent_t issued = nullptr;
    CK(cudaEventCreateWithFlags(&issued, cudaEventDisableTiming));
    struct EventGuard {
        cudaEvent_t e;
        ~EventGuard() { cudaEventDestroy(e); }
    } issued_guard{issued};
    for (size_t g = 1; g < ends.size(); ++g) {
        st = issue_steps(c.get(), periods * per);
        if (st != CRUSH_OK) return st;
        CK(cudaEventRecord(issued, c->stream));
        st = add_slots(c.get(), descs + placed, ends[g] - placed, false, nullptr);
        if (st == CRUSH_ERR_BUSY) break;  // beyond the room estimate: the rest run afterwards
        if (st != CRUSH_OK) return st;
        placed = ends[g];
        if (cudaEventQuery(issued) == cudaSuccess) periods = std::min<long long>(2 * periods, 8);
    }
    // to the end: every slot, the last joined included
    long long cap = 0;
    for (const Slot& sl : c->slots) cap = std::max<long long>(cap, sl.settings.max_steps > 0 ? sl.settings.max_steps : 2000000ll);
    cap += c->host_step + 2 * N_CANDS * per;
    int done = 0;
    while (!done && c->host_step < cap) {
        st = run_steps(c.get(), 2 * N_CANDS * per, &done);
        if (st != CRUSH_OK) return st;
    }
    if (!done) return crush::fail(CRUSH_ERR_TIMEOUT, "batch did not finish within " + std::to_string(cap) + " steps");
    st = results_range(c.get(), 0, c->n_slots, out);
    if (st != CRUSH_OK) return st;
    c.reset();
    if (placed < n) return solve_models(descs + placed, n - placed, device, out + placed);
    return CRUSH_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int crush_device_info(int device, char* name, int name_len) {
    cudaDeviceProp p;
    cudaError_t e = cudaGetDeviceProperties(&p, device);
    if (e != cudaSuccess) return crush::fail(CRUSH_ERR_CUDA, cudaGetErrorString(e));
    if (name && name_len > 0) {
        std::strncpy(name, p.name, name_len - 1);
        name[name_len - 1] = 0;
    }
    return p.multiProcessorCount;
}

int crush_batch_create(const crush_model_desc* const* descs, int n, int device, crush_ctx** out) {
    if (!out) return crush::fail(CRUSH_ERR_INVALID, "null output");
    *out = nullptr;
    crush_ctx* c = new crush_ctx();
    int st = create_impl(descs, n, device, c);
    if (st != CRUSH_OK) {
        delete c;
        return st;
    }
    *out = c;
    return CRUSH_OK;
}

int crush_batch_create_reserved(const crush_model_desc* const* descs, int n, int device, const crush_capacity* room, crush_ctx** out) {
    if (!out || !room) return crush::fail(CRUSH_ERR_INVALID, "null argument");
    if (room->slots < 0 || room->contacts < 0 || room->nodes < 0 || room->hexes < 0 || room->faces < 0 || room->primary_nodes < 0)
        return crush::fail(CRUSH_ERR_INVALID, "negative room");
    *out = nullptr;
    crush_ctx* c = new crush_ctx();
    int st = create_impl(descs, n, device, c, room);
    if (st != CRUSH_OK) {
        delete c;
        return st;
    }
    *out = c;
    return CRUSH_OK;
}

int crush_batch_append(crush_ctx* c, const crush_model_desc* const* descs, int n, int* first_slot) {
    if (!c) return crush::fail(CRUSH_ERR_INVALID, "null context");
    CK(cudaSetDevice(c->device));
    if (c->prologue_done || c->contact_done) return crush::fail(CRUSH_ERR_INVALID, "slots join an open run only between issues of steps");
    const int first = c->n_slots;
    int st = add_slots(c, descs, n, false, nullptr);
    if (st != CRUSH_OK) return st;
    if (first_slot) *first_slot = first;
    return CRUSH_OK;
}

int crush_run_issue(crush_ctx* c, int64_t n_steps) {
    if (!c || n_steps < 0) return crush::fail(CRUSH_ERR_INVALID, "invalid argument");
    CK(cudaSetDevice(c->device));
    return issue_steps(c, n_steps);
}

int crush_create(const crush_model_desc* desc, int device, crush_ctx** out) {
    const crush_model_desc* one[1] = {desc};
    return crush_batch_create(one, 1, device, out);
}

void crush_destroy(crush_ctx* ctx) { delete ctx; }

int crush_sizes(const crush_ctx* c, int64_t* n_nodes, int64_t* n_hexes, int64_t* n_active) {
    if (!c) return crush::fail(CRUSH_ERR_INVALID, "null context");
    if (n_nodes) *n_nodes = c->n_nodes;
    if (n_hexes) *n_hexes = c->n_all;
    if (n_active) *n_active = c->n_hc;
    return CRUSH_OK;
}

int crush_batch_size(const crush_ctx* c) { return c ? c->n_slots : 0; }

int64_t crush_launch_count(const crush_ctx* c) { return c ? c->launches : 0; }

int crush_compute_forces_device(crush_ctx* c, const double* u_device, double* f_device, int64_t* newly) {
    if (!c || !u_device || !f_device) return crush::fail(CRUSH_ERR_INVALID, "null argument");
    CK(cudaSetDevice(c->device));
    NodeArrays nd = c->nd();
    nd.u = const_cast<double*>(u_device);
    if (newly) {
        int st = reset_aux(c, 0.0);
        if (st != CRUSH_OK) return st;
    }
    launch_forces(c->stream, c->el(), nd, c->ctls_aux, 0);
    launch_gather(c->stream, c->el(), nd, f_device);
    int st = check_launch(c, forces_launches(c->el()) + 1);
    if (st != CRUSH_OK) return st;
    if (newly) {
        std::vector<Control> aux;
        st = read_aux(c, &aux);
        if (st != CRUSH_OK) return st;
        long long k = 0;
        for (const Control& a : aux) k += a.eroded_step;
        *newly = k;
    }
    return CRUSH_OK;
}

int crush_compute_forces(crush_ctx* c, const double* u, double* f_accum, int64_t* newly) {
    if (!c || !u || !f_accum) return crush::fail(CRUSH_ERR_INVALID, "null argument");
    CK(cudaSetDevice(c->device));
    const size_t bytes = sizeof(double) * 3 * c->n_nodes;
    CK(cudaMemcpyAsync(c->u_tmp, u, bytes, cudaMemcpyHostToDevice, c->stream));
    int64_t k = 0;
    int st = crush_compute_forces_device(c, c->u_tmp, c->f_tmp, &k);
    if (st != CRUSH_OK) return st;
    std::vector<double> f(3 * c->n_nodes);
    CK(cudaMemcpyAsync(f.data(), c->f_tmp, bytes, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (size_t i = 0; i < f.size(); ++i) f_accum[i] += f[i];
    if (newly) *newly = k;
    return CRUSH_OK;
}

int crush_contact_apply(crush_ctx* c, int id, const double* u, const double* v, const double* masses, double dt, double* f_accum,
                        int64_t* count, double* max_pen) {
    (void)v;  // the reference's contact damping ratio is the constant 0 (src/contact.rs:82)
    if (!c || !u || !f_accum) return crush::fail(CRUSH_ERR_INVALID, "null argument");
    if (id < 0 || id >= c->n_contacts) return crush::fail(CRUSH_ERR_INVALID, "contact id out of range");
    if (!(dt > 0.0)) return crush::fail(CRUSH_ERR_INVALID, "dt must be positive");
    CK(cudaSetDevice(c->device));
    const size_t bytes = sizeof(double) * 3 * c->n_nodes;
    CK(cudaMemcpyAsync(c->u_tmp, u, bytes, cudaMemcpyHostToDevice, c->stream));
    const double* m = c->mass;
    if (masses) {
        CK(cudaMemcpyAsync(c->n_tmp, masses, sizeof(double) * c->n_nodes, cudaMemcpyHostToDevice, c->stream));
        m = c->n_tmp;
    }
    CK(cudaMemsetAsync(c->f_tmp, 0, bytes, c->stream));
    CK(cudaMemsetAsync(c->ca.pen_count + id, 0, sizeof(unsigned long long), c->stream));
    CK(cudaMemsetAsync(c->ca.pen_max_bits + id, 0, sizeof(unsigned long long), c->stream));
    NodeArrays nd = c->nd();
    nd.u = c->u_tmp;
    const long long nf = c->face_off_h[id + 1] - c->face_off_h[id], ns = c->slave_off_h[id + 1] - c->slave_off_h[id];
    const long long bk0 = c->tab_off_h[id], bk1 = c->tab_off_h[id + 1];
    launch_contact(c->stream, c->ca, nd, c->ctls_aux, id, id + 1, c->face_off_h[id], nf, ns, bk0, bk1, dt, m, c->f_tmp, 0,
                   c->slave_lanes);
    int st = check_launch(c, contact_launches(c->ca, false, nf, ns, bk0, bk1, id));
    if (st != CRUSH_OK) return st;
    if (c->run_open) {
        // The call reused the run's contact buffers at its own u: restore the
        // open run's static geometry and pending search.
        if (c->is_static_h[id]) {
            launch_contact_geometry(c->stream, c->ca, c->nd(), id, id + 1, c->face_off_h[id], nf);
            st = check_launch(c);
            if (st != CRUSH_OK) return st;
        }
        st = search_now(c);
        if (st != CRUSH_OK) return st;
    }
    std::vector<double> f(3 * c->n_nodes);
    unsigned long long cnt = 0, mp = 0;
    CK(cudaMemcpyAsync(f.data(), c->f_tmp, bytes, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(&cnt, c->ca.pen_count + id, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(&mp, c->ca.pen_max_bits + id, sizeof(mp), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemsetAsync(c->ca.pen_count + id, 0, sizeof(unsigned long long), c->stream));
    CK(cudaMemsetAsync(c->ca.pen_max_bits + id, 0, sizeof(unsigned long long), c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (size_t i = 0; i < f.size(); ++i) f_accum[i] += f[i];
    if (count) *count = (int64_t)cnt;
    if (max_pen) std::memcpy(max_pen, &mp, sizeof(double));
    return CRUSH_OK;
}

int crush_stable_dt(crush_ctx* c, const double* u, double* dt) {
    if (!c || !u || !dt) return crush::fail(CRUSH_ERR_INVALID, "null argument");
    CK(cudaSetDevice(c->device));
    CK(cudaMemcpyAsync(c->u_tmp, u, sizeof(double) * 3 * c->n_nodes, cudaMemcpyHostToDevice, c->stream));
    int st = reset_aux(c, 0.0);
    if (st != CRUSH_OK) return st;
    launch_elem_dt(c->stream, c->el(), c->nd(), c->ctls_aux, c->u_tmp, 0);
    st = check_launch(c);
    if (st != CRUSH_OK) return st;
    std::vector<Control> aux;
    st = read_aux(c, &aux);
    if (st != CRUSH_OK) return st;
    double m = INF;
    for (const Control& a : aux) {
        double x;
        std::memcpy(&x, &a.dt_stable_bits, sizeof(double));
        m = std::fmin(m, x);
    }
    *dt = m;
    return std::isfinite(m) ? CRUSH_OK : CRUSH_NONE;
}

int crush_mass_scaling(crush_ctx* c, const double* u, double dt_min, const double* element_mass, double* added, double* total) {
    if (!c || !u || !added) return crush::fail(CRUSH_ERR_INVALID, "null argument");
    CK(cudaSetDevice(c->device));
    CK(cudaMemcpyAsync(c->u_tmp, u, sizeof(double) * 3 * c->n_nodes, cudaMemcpyHostToDevice, c->stream));
    ElementArrays el = c->el();
    if (element_mass) {
        CK(cudaMemcpyAsync(c->e_tmp, element_mass, sizeof(double) * c->n_all, cudaMemcpyHostToDevice, c->stream));
        el.elem_mass = c->e_tmp;
    }
    int st = reset_aux(c, dt_min);
    if (st != CRUSH_OK) return st;
    NodeArrays nd = c->nd();
    nd.added = c->n_tmp;
    nd.inv_mass = c->n_tmp2;
    launch_elem_dt(c->stream, el, nd, c->ctls_aux, c->u_tmp, 0);
    launch_mass_scaling(c->stream, el, nd, c->ctls_aux, 1);
    st = check_launch(c, 2);
    if (st != CRUSH_OK) return st;
    CK(cudaMemcpyAsync(added, c->n_tmp, sizeof(double) * c->n_nodes, cudaMemcpyDeviceToHost, c->stream));
    std::vector<Control> aux;
    st = read_aux(c, &aux);
    if (st != CRUSH_OK) return st;
    double t = 0.0;
    for (const Control& a : aux) t += a.added_total_acc;
    if (total) *total = t;
    return CRUSH_OK;
}

int crush_masses(crush_ctx* c, double* lumped, double* element_mass) {
    if (!c) return crush::fail(CRUSH_ERR_INVALID, "null context");
    if (lumped) CK(cudaMemcpyAsync(lumped, c->mass, sizeof(double) * c->n_nodes, cudaMemcpyDeviceToHost, c->stream));
    if (element_mass) CK(cudaMemcpyAsync(element_mass, c->elem_mass, sizeof(double) * c->n_all, cudaMemcpyDeviceToHost, c->stream));
    return sync(c);
}

int crush_element_data(crush_ctx* c, float* grad, float* volume, float* gamma, float* h) {
    if (!c) return crush::fail(CRUSH_ERR_INVALID, "null context");
    std::vector<float4> pl((size_t)N_STATIC_PLANES * c->stride);
    CK(cudaMemcpyAsync(pl.data(), c->planes, sizeof(float4) * pl.size(), cudaMemcpyDeviceToHost, c->stream));
    int st = sync(c);
    if (st != CRUSH_OK) return st;
    auto comp = [&](int plane, long long e, int k) {
        const float4& f = pl[(size_t)plane * c->stride + e];
        return k == 0 ? f.x : k == 1 ? f.y : k == 2 ? f.z : f.w;
    };
    for (long long e = 0; e < c->n_hc; ++e) {
        if (grad)
            for (int k = 0; k < 24; ++k) grad[24 * e + k] = comp(P_GRAD + k / 4, e, k % 4);
        if (volume) volume[e] = comp(P_META, e, 0);
        if (gamma)
            for (int k = 0; k < 32; ++k) gamma[32 * e + k] = comp(P_GAMMA + k / 4, e, k % 4);
        if (h)
            for (int col = 0; col < 12; ++col)
                for (int row = 0; row < 12; ++row) {
                    int k = h_index(row, col);
                    h[144 * e + 12 * col + row] = comp(P_H + k / 4, e, k % 4);
                }
    }
    return CRUSH_OK;
}

int crush_get_state(crush_ctx* c, float* state, uint8_t* eroded) {
    if (!c) return crush::fail(CRUSH_ERR_INVALID, "null context");
    std::vector<float4> sp((size_t)N_STATE_PLANES * c->stride);
    CK(cudaMemcpyAsync(sp.data(), c->state, sizeof(float4) * sp.size(), cudaMemcpyDeviceToHost, c->stream));
    int st = sync(c);
    if (st != CRUSH_OK) return st;
    for (long long e = 0; e < c->n_hc; ++e)
        for (int k = 0; k < 26; ++k) {
            const float4& f = sp[(size_t)(k / 4) * c->stride + e];
            float x = (k % 4) == 0 ? f.x : (k % 4) == 1 ? f.y : (k % 4) == 2 ? f.z : f.w;
            if (k < 25 && state) state[25 * e + k] = x;
            if (k == S_ERODED && eroded) {
                uint32_t b;
                std::memcpy(&b, &x, 4);
                eroded[e] = b != 0;
            }
        }
    return CRUSH_OK;
}

int crush_set_state(crush_ctx* c, const float* state, const uint8_t* eroded) {
    if (!c || !state || !eroded) return crush::fail(CRUSH_ERR_INVALID, "null argument");
    std::vector<float4> sp((size_t)N_STATE_PLANES * c->stride);
    std::vector<uint8_t> er_all(c->n_all, 0);
    CK(cudaMemcpyAsync(er_all.data(), c->eroded_all, c->n_all, cudaMemcpyDeviceToHost, c->stream));  // elastic elements keep theirs
    CK(cudaStreamSynchronize(c->stream));
    for (long long e = 0; e < c->n_hc; ++e) {
        float v[28] = {};
        for (int k = 0; k < 25; ++k) v[k] = state[25 * e + k];
        uint32_t b = eroded[e] ? 1u : 0u;
        std::memcpy(&v[S_ERODED], &b, 4);
        for (int k = 0; k < N_STATE_PLANES; ++k) sp[(size_t)k * c->stride + e] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
        er_all[c->hc_model[e]] = eroded[e] ? 1 : 0;
    }
    CK(cudaMemcpyAsync(c->state, sp.data(), sizeof(float4) * sp.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->eroded_all, er_all.data(), c->n_all, cudaMemcpyHostToDevice, c->stream));
    return sync(c);
}

int crush_run_begin(crush_ctx* c) {
    if (!c) return crush::fail(CRUSH_ERR_INVALID, "null context");
    CK(cudaSetDevice(c->device));
    return run_begin(c);
}

int crush_run_steps(crush_ctx* c, int64_t n_steps, int* done) {
    if (!c) return crush::fail(CRUSH_ERR_INVALID, "null context");
    CK(cudaSetDevice(c->device));
    return run_steps(c, n_steps, done);
}

int crush_run_results(crush_ctx* c, crush_results* r) {
    if (!c || !r) return crush::fail(CRUSH_ERR_INVALID, "null argument");
    CK(cudaSetDevice(c->device));
    return results(c, 0, r);
}

int crush_batch_done(crush_ctx* c, int* done_flags, int* all) {
    if (!c) return crush::fail(CRUSH_ERR_INVALID, "null context");
    CK(cudaSetDevice(c->device));
    int d = 0;
    int st = all_done(c, &d);
    if (st != CRUSH_OK) return st;
    if (done_flags) std::memcpy(done_flags, c->done_h.data(), sizeof(int) * c->n_slots);
    if (all) *all = d;
    return CRUSH_OK;
}

int crush_batch_results_range(crush_ctx* c, int first, int count, crush_results* r) {
    if (!c || !r) return crush::fail(CRUSH_ERR_INVALID, "null argument");
    CK(cudaSetDevice(c->device));
    return results_range(c, first, first + count, r);
}

int crush_batch_results(crush_ctx* c, int slot, crush_results* r) {
    if (!c || !r) return crush::fail(CRUSH_ERR_INVALID, "null argument");
    CK(cudaSetDevice(c->device));
    return results(c, slot, r);
}

int crush_autotune(crush_ctx* c, crush_tuning* out) {
    if (!c) return crush::fail(CRUSH_ERR_INVALID, "null context");
    if (!c->run_open) return crush::fail(CRUSH_ERR_INVALID, "no open run (call crush_run_begin)");
    CK(cudaSetDevice(c->device));
    int st = autotune(c);
    if (st != CRUSH_OK) return st;
    return crush_get_tuning(c, out);
}

int crush_history_config(crush_ctx* c, int slot, int history_steps, int64_t max_records, int n_acc, const crush_accelerometer* acc) {
    if (!c) return crush::fail(CRUSH_ERR_INVALID, "null context");
    if (slot < 0 || slot >= c->n_slots) return crush::fail(CRUSH_ERR_INVALID, "slot out of range");
    if (c->run_open) return crush::fail(CRUSH_ERR_BUSY, "history configuration while a run is open");
    if (history_steps < 0) return crush::fail(CRUSH_ERR_INVALID, "history_steps must be >= 0");
    if (history_steps > 0 && (max_records < 1 || max_records > (1ll << 31)))
        return crush::fail(CRUSH_ERR_INVALID, "max_records must be in [1, 2^31]");
    if (n_acc < 0 || (n_acc > 0 && !acc)) return crush::fail(CRUSH_ERR_INVALID, "invalid accelerometer list");
    const Slot& sl = c->slots[slot];
    std::vector<HistAccel> list;
    for (int k = 0; k < n_acc; ++k) {
        const crush_accelerometer& a = acc[k];
        if (a.n_nodes < 0 || (a.n_nodes > 0 && !a.nodes)) return crush::fail(CRUSH_ERR_INVALID, "invalid accelerometer nodes");
        HistAccel h;
        h.nodes.assign(a.nodes, a.nodes + a.n_nodes);
        h.has_frame = a.has_frame ? 1 : 0;
        h.frame[0] = a.origin;
        h.frame[1] = a.x_axis;
        h.frame[2] = a.plane;
        // out-of-range nodes: the reference panics (src/solver.rs:245-248)
        for (uint32_t n : h.nodes)
            if (n >= (uint64_t)sl.n_nodes) return crush::fail(CRUSH_ERR_INVALID, "accelerometer node out of range");
        if (h.has_frame)
            for (uint32_t n : h.frame)
                if (n >= (uint64_t)sl.n_nodes) return crush::fail(CRUSH_ERR_INVALID, "accelerometer frame node out of range");
        list.push_back(std::move(h));
    }
    c->hist_steps.resize(c->n_slots, 0);
    c->hist_max.resize(c->n_slots, 0);
    c->hist_acc.resize(c->n_slots);
    for (int k = 0; k < c->n_slots; ++k)
        if (k != slot && history_steps > 0 && c->hist_steps[k] > 0 && c->hist_steps[k] != history_steps)
            return crush::fail(CRUSH_ERR_UNSUPPORTED, "the recording slots of one context must share history_steps");
    CK(cudaSetDevice(c->device));
    c->hist_steps[slot] = history_steps;
    c->hist_max[slot] = history_steps > 0 ? max_records : 0;
    c->hist_acc[slot] = std::move(list);
    return rebuild_history(c);
}

// The last-step record of finished crashes, when due (src/solver.rs:356-358).
static int history_final(crush_ctx* c) {
    launch_history(c->stream, c->hist, c->nd(), c->ctls, c->f_ext, HIST_FINAL, c->f_ext_odd);
    return check_launch(c, (c->hist.n_pu > 0 ? 1 : 0) + 1);
}

int crush_history_counts(crush_ctx* c, int slot, int64_t* n_records, int* n_parts, int64_t* n_node_samples) {
    if (!c) return crush::fail(CRUSH_ERR_INVALID, "null context");
    if (slot < 0 || slot >= c->n_slots) return crush::fail(CRUSH_ERR_INVALID, "slot out of range");
    CK(cudaSetDevice(c->device));
    const bool on = c->hist_on && c->hist_ran && slot < (int)c->hist_steps.size() && c->hist_steps[slot] > 0;
    long long count = 0;
    if (on) {
        int st = history_final(c);
        if (st != CRUSH_OK) return st;
        CK(cudaMemcpyAsync(&count, c->hist.rec_count + slot, sizeof(count), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    long long nodes = 0;
    if (on)
        for (const HistAccel& a : c->hist_acc[slot]) nodes += (long long)a.nodes.size();
    if (n_records) *n_records = count;
    if (n_parts) *n_parts = on ? c->slots[slot].n_parts : 0;
    if (n_node_samples) *n_node_samples = nodes;
    return CRUSH_OK;
}

int crush_history_get(crush_ctx* c, int slot, double* time, int64_t* step, crush_part_state* parts, crush_node_sample* samples) {
    int64_t n_rec = 0, n_nodes = 0;
    int n_parts = 0;
    int st = crush_history_counts(c, slot, &n_rec, &n_parts, &n_nodes);
    if (st != CRUSH_OK) return st;
    if (n_rec == 0) return CRUSH_OK;
    const HistoryArrays& h = c->hist;
    const long long kept = std::min<long long>(n_rec, c->hist_max[slot]);
    const long long stride = h.max_rec;
    std::vector<long long> pu_off(c->n_slots + 1), an_off(c->n_slots + 1);
    {
        std::vector<int> a(c->n_slots + 1), b(c->n_slots + 1);
        CK(cudaMemcpy(a.data(), h.slot_pu_off, sizeof(int) * a.size(), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(b.data(), h.slot_an_off, sizeof(int) * b.size(), cudaMemcpyDeviceToHost));
        for (size_t k = 0; k < a.size(); ++k) {
            pu_off[k] = a[k];
            an_off[k] = b[k];
        }
    }
    if (time) CK(cudaMemcpy(time, h.rec_time + slot * stride, sizeof(double) * kept, cudaMemcpyDeviceToHost));
    if (step) {
        std::vector<long long> s(kept);
        CK(cudaMemcpy(s.data(), h.rec_step + slot * stride, sizeof(long long) * kept, cudaMemcpyDeviceToHost));
        for (long long k = 0; k < kept; ++k) step[k] = s[k];
    }
    if (parts && n_parts > 0) {
        std::vector<double> buf((size_t)n_parts * stride * HIST_PART_VALUES);
        CK(cudaMemcpy(buf.data(), h.part_rec + pu_off[slot] * stride * HIST_PART_VALUES, sizeof(double) * buf.size(),
                      cudaMemcpyDeviceToHost));
        for (long long r = 0; r < kept; ++r)
            for (int p = 0; p < n_parts; ++p) {
                const double* v = &buf[((size_t)p * stride + r) * HIST_PART_VALUES];
                crush_part_state& o = parts[r * n_parts + p];
                o.mass = v[0];
                for (int d = 0; d < 3; ++d) {
                    o.velocity[d] = v[1 + d];
                    o.displacement[d] = v[4 + d];
                    o.acceleration[d] = v[7 + d];
                }
                o.kinetic_energy = v[10];
            }
    }
    if (samples && n_nodes > 0) {
        std::vector<double> buf((size_t)n_nodes * stride * HIST_NODE_VALUES);
        CK(cudaMemcpy(buf.data(), h.node_rec + an_off[slot] * stride * HIST_NODE_VALUES, sizeof(double) * buf.size(),
                      cudaMemcpyDeviceToHost));
        std::vector<std::pair<int, uint32_t>> who;  // (accelerometer, node) of each sampled node
        for (size_t k = 0; k < c->hist_acc[slot].size(); ++k)
            for (uint32_t n : c->hist_acc[slot][k].nodes) who.push_back({(int)k, n});
        for (long long r = 0; r < kept; ++r)
            for (long long j = 0; j < n_nodes; ++j) {
                const double* v = &buf[((size_t)j * stride + r) * HIST_NODE_VALUES];
                crush_node_sample& o = samples[r * n_nodes + j];
                o.accelerometer = who[j].first;
                o.node = who[j].second;
                for (int d = 0; d < 3; ++d) {
                    o.position[d] = v[d];
                    o.displacement[d] = v[3 + d];
                    o.velocity[d] = v[6 + d];
                    o.acceleration[d] = v[9 + d];
                    o.local_displacement[d] = v[12 + d];
                    o.local_velocity[d] = v[15 + d];
                    o.local_acceleration[d] = v[18 + d];
                }
            }
    }
    return CRUSH_OK;
}

int crush_frames_config(crush_ctx* c, int slot, int frame_steps, int64_t max_frames) {
    if (!c) return crush::fail(CRUSH_ERR_INVALID, "null context");
    if (slot < 0 || slot >= c->n_slots) return crush::fail(CRUSH_ERR_INVALID, "slot out of range");
    if (c->run_open) return crush::fail(CRUSH_ERR_BUSY, "frame configuration while a run is open");
    if (frame_steps < 0) return crush::fail(CRUSH_ERR_INVALID, "frame_steps must be >= 0");
    if (frame_steps > 0 && (max_frames < 1 || max_frames > (1ll << 31)))
        return crush::fail(CRUSH_ERR_INVALID, "max_frames must be in [1, 2^31]");
    if (frame_steps > 0 && c->n_slots > 65535) return crush::fail(CRUSH_ERR_UNSUPPORTED, "frames need at most 65535 crashes per context");
    c->frame_steps.resize(c->n_slots, 0);
    c->frame_max.resize(c->n_slots, 0);
    for (int k = 0; k < c->n_slots; ++k)
        if (k != slot && frame_steps > 0 && c->frame_steps[k] > 0 && c->frame_steps[k] != frame_steps)
            return crush::fail(CRUSH_ERR_UNSUPPORTED, "the capturing slots of one context must share frame_steps");
    CK(cudaSetDevice(c->device));
    c->frame_steps[slot] = frame_steps;
    c->frame_max[slot] = frame_steps > 0 ? max_frames : 0;
    return rebuild_frames(c);
}

int crush_frames_count(crush_ctx* c, int slot, int64_t* n_frames) {
    if (!c || !n_frames) return crush::fail(CRUSH_ERR_INVALID, "null argument");
    if (slot < 0 || slot >= c->n_slots) return crush::fail(CRUSH_ERR_INVALID, "slot out of range");
    *n_frames = 0;
    if (!c->frames_on || !c->frames_ran || slot >= (int)c->frame_steps.size() || c->frame_steps[slot] == 0) return CRUSH_OK;
    CK(cudaSetDevice(c->device));
    launch_frames(c->stream, c->frames, c->u, c->ctls, HIST_FINAL);  // the last step's frame (src/solver.rs:353-355)
    int st = check_launch(c, 3);
    if (st != CRUSH_OK) return st;
    long long n = 0;
    CK(cudaMemcpyAsync(&n, c->frames.count + slot, sizeof(n), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *n_frames = n;
    return CRUSH_OK;
}

int crush_frame_get(crush_ctx* c, int slot, int64_t frame, double* time, int64_t* step, float* displacement, float* plastic_strain,
                    float* stress, uint8_t* eroded) {
    int64_t n = 0;
    int st = crush_frames_count(c, slot, &n);
    if (st != CRUSH_OK) return st;
    if (frame < 0 || frame >= std::min<int64_t>(n, c->frame_max.empty() ? 0 : c->frame_max[slot]))
        return crush::fail(CRUSH_ERR_INVALID, "frame not kept");
    const Slot& sl = c->slots[slot];
    const FrameArrays& f = c->frames;
    long long dbase = 0, ebase = 0;
    for (int k = 0; k < slot; ++k) {
        dbase += (c->frame_steps[k] > 0 ? c->frame_max[k] : 0) * 3 * c->slots[k].n_nodes;
        ebase += (c->frame_steps[k] > 0 ? c->frame_max[k] : 0) * c->slots[k].n_elems;
    }
    const long long e_off = ebase + frame * sl.n_elems;
    if (time) CK(cudaMemcpy(time, f.time + slot * f.stride + frame, sizeof(double), cudaMemcpyDeviceToHost));
    if (step) {
        long long s = 0;
        CK(cudaMemcpy(&s, f.step + slot * f.stride + frame, sizeof(long long), cudaMemcpyDeviceToHost));
        *step = s;
    }
    if (displacement)
        CK(cudaMemcpy(displacement, f.disp + dbase + frame * 3 * sl.n_nodes, sizeof(float) * 3 * sl.n_nodes, cudaMemcpyDeviceToHost));
    if (plastic_strain) CK(cudaMemcpy(plastic_strain, f.pstrain + e_off, sizeof(float) * sl.n_elems, cudaMemcpyDeviceToHost));
    if (stress) CK(cudaMemcpy(stress, f.stress + 6 * e_off, sizeof(float) * 6 * sl.n_elems, cudaMemcpyDeviceToHost));
    if (eroded) CK(cudaMemcpy(eroded, f.eroded + e_off, sl.n_elems, cudaMemcpyDeviceToHost));
    return CRUSH_OK;
}

int crush_get_tuning(const crush_ctx* c, crush_tuning* out) {
    if (!c || !out) return crush::fail(CRUSH_ERR_INVALID, "null argument");
    std::memset(out, 0, sizeof(*out));
    out->slave_lanes = c->slave_lanes;
    out->forces_schedule = c->forces_schedule;
    out->fused_contact_side = c->fused_contact_side ? 1 : 0;
    for (int k = 0; k < 6; ++k) out->contact_ms[k] = c->tune_ms[k];
    out->step_fusion = c->step_fusion ? 1 : 0;
    out->early_contact = c->early_contact ? 1 : 0;
    for (int k = 0; k < N_CANDS; ++k) out->step_ms[k] = c->sched_ms[k];
    return CRUSH_OK;
}

int crush_set_tuning(crush_ctx* c, const crush_tuning* t) {
    if (!c || !t) return crush::fail(CRUSH_ERR_INVALID, "null argument");
    const int lanes = t->slave_lanes;
    if (lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32)
        return crush::fail(CRUSH_ERR_INVALID, "slave_lanes must be 1, 2, 4, 8, 16 or 32");
    if (t->forces_schedule < 0 || t->forces_schedule >= N_FORCES_SCHEDULES)
        return crush::fail(CRUSH_ERR_INVALID, "forces_schedule must be 0, 1, 2 or 3");
    if (t->fused_contact_side != 0 && t->fused_contact_side != 1) return crush::fail(CRUSH_ERR_INVALID, "fused_contact_side must be 0 or 1");
    if (t->early_contact != 0 && t->early_contact != 1) return crush::fail(CRUSH_ERR_INVALID, "early_contact must be 0 or 1");
    if (lanes != c->slave_lanes || t->forces_schedule != c->forces_schedule || (t->fused_contact_side == 1) != c->fused_contact_side ||
        (t->early_contact == 1) != c->early_contact)
        drop_graphs(c);
    c->early_contact = t->early_contact == 1;
    c->slave_lanes = lanes;
    c->forces_schedule = t->forces_schedule;
    c->fused_contact_side = t->fused_contact_side == 1;
    c->tuning_fixed = true;
    c->tuned = true;
    c->sched_trial_pending = false;
    return CRUSH_OK;
}

int crush_set_contact_search(crush_ctx* c, int exhaustive) {
    if (!c || (exhaustive != 0 && exhaustive != 1)) return crush::fail(CRUSH_ERR_INVALID, "exhaustive must be 0 or 1");
    if (c->ca.exhaustive != exhaustive) {
        c->ca.exhaustive = exhaustive;
        drop_graphs(c);
    }
    return CRUSH_OK;
}

int crush_set_step_fusion(crush_ctx* c, int fused) {
    if (!c || (fused != 0 && fused != 1)) return crush::fail(CRUSH_ERR_INVALID, "fused must be 0 or 1");
    c->tuning_fixed = true;
    c->tuned = true;
    c->sched_trial_pending = false;
    if (c->step_fusion != (fused == 1)) {
        c->step_fusion = fused == 1;
        drop_graphs(c);
    }
    return CRUSH_OK;
}

int crush_contact_search_stats(crush_ctx* c, int id, uint64_t* out, int reset) {
    if (!c || !out) return crush::fail(CRUSH_ERR_INVALID, "null argument");
    if (id < 0 || id >= c->n_contacts) return crush::fail(CRUSH_ERR_INVALID, "contact id out of range");
    CK(cudaMemcpyAsync(out, c->ca.search_stats + 3 * id, 3 * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->stream));
    if (reset) CK(cudaMemsetAsync(c->ca.search_stats + 3 * id, 0, 3 * sizeof(uint64_t), c->stream));
    return sync(c);
}

int crush_run_state(crush_ctx* c, double* u, double* v) {
    if (!c) return crush::fail(CRUSH_ERR_INVALID, "null context");
    if (u) CK(cudaMemcpyAsync(u, c->u, sizeof(double) * 3 * c->n_nodes, cudaMemcpyDeviceToHost, c->stream));
    if (v) CK(cudaMemcpyAsync(v, c->v, sizeof(double) * 3 * c->n_nodes, cudaMemcpyDeviceToHost, c->stream));
    return sync(c);
}

int crush_set_profiling(crush_ctx* c, int level) {
    if (!c || level < 1 || level > 2) return crush::fail(CRUSH_ERR_INVALID, "profiling level must be 1 or 2");
    if (level != c->prof_level) {
        c->prof_level = level;
        drop_graphs(c);
    }
    return CRUSH_OK;
}

int crush_run_steps_timed(crush_ctx* c, int64_t n_steps, int* done, double* ms, double* phase_ms, int* phase_steps) {
    if (!c) return crush::fail(CRUSH_ERR_INVALID, "null context");
    CK(cudaSetDevice(c->device));
    const bool want_phases = phase_ms != nullptr;
    if (want_phases != c->profiling) {
        c->profiling = want_phases;
        drop_graphs(c);
    }
    cudaEvent_t t0, t1;
    CK(cudaEventCreate(&t0));
    CK(cudaEventCreate(&t1));
    CK(cudaEventRecord(t0, c->stream));
    int st = issue_steps(c, n_steps);
    if (st != CRUSH_OK) {
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        return st;
    }
    CK(cudaEventRecord(t1, c->stream));
    int d = 0;
    st = all_done(c, &d);
    float elapsed = 0.f;
    cudaEventElapsedTime(&elapsed, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (st != CRUSH_OK) return st;
    if (done) *done = d;
    if (ms) *ms = elapsed;
    if (want_phases) {
        int steps = c->last_was_graph ? c->period : 1;
        for (int i = 0; i < N_PHASE_EVENTS - 1; ++i) phase_ms[i] = 0.0;
        for (int k = 0; k < steps; ++k)
            for (int i = 0; i < N_PHASE_EVENTS - 1; ++i) {
                if (c->prof_level == 1 && i != 3) continue;
                float x = 0.f;
                CK(cudaEventElapsedTime(&x, c->prof_ev[(size_t)k * N_PHASE_EVENTS + i], c->prof_ev[(size_t)k * N_PHASE_EVENTS + i + 1]));
                phase_ms[i] += x;
            }
        if (phase_steps) *phase_steps = steps;
    }
    return CRUSH_OK;
}

int crush_run(crush_ctx* c, crush_results* r) {
    if (!c || !r) return crush::fail(CRUSH_ERR_INVALID, "null argument");
    CK(cudaSetDevice(c->device));
    int st = run_to_end(c);
    if (st != CRUSH_OK) return st;
    st = results(c, 0, r);
    if (st != CRUSH_OK) return st;
    return r->status;
}

int crush_batch_run(crush_ctx* c, crush_results* r) {
    if (!c || !r) return crush::fail(CRUSH_ERR_INVALID, "null argument");
    CK(cudaSetDevice(c->device));
    int st = run_to_end(c);
    if (st != CRUSH_OK) return st;
    return results_range(c, 0, c->n_slots, r);
}

int crush_batch_solve(const crush_model_desc* const* descs, int n, int device, crush_results* out) {
    if (!descs || n <= 0 || !out) return crush::fail(CRUSH_ERR_INVALID, "invalid argument");
    for (int k = 0; k < n; ++k)
        if (!descs[k]) return crush::fail(CRUSH_ERR_INVALID, "null model description");
    CK(cudaSetDevice(device));
    return solve_models(descs, n, device, out);
}

}  // extern "C"
