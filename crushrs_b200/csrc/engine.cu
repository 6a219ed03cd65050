// engine.cu — the single-model context and the C ABI of include/crush.h.
//
// Host side (C++17): validates the model, builds the node incidence CSRs and
// contact tables, owns every device buffer, and drives the explicit step loop
// (src/solver.rs:190-381) as a fixed sequence of kernels on one stream,
// captured into a CUDA graph one period of steps at a time. All per-step
// decisions (dt, mass scaling, stop rules) are taken on the device from a
// control block, so the loop never waits on the host.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <numeric>
#include <set>
#include <string>
#include <vector>

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

}  // namespace

struct crush_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<void*> allocs;
    int64_t launches = 0;

    // sizes
    long long n_nodes = 0, n_all = 0, n_hc = 0, stride = 0;
    std::vector<int64_t> hc_index;   // model element -> honeycomb index or -1
    std::vector<uint32_t> hc_model;  // honeycomb index -> model element
    crush_settings settings{};
    double contact_dt = INF, stable = INF, dt_floor = 0.0, dt0 = 0.0;

    // device arrays
    double *pos = nullptr, *u = nullptr, *v = nullptr, *v0 = nullptr, *v_half = nullptr, *f_int = nullptr, *f_ext = nullptr;
    double *inv_mass = nullptr, *mass = nullptr, *added = nullptr, *lumped = nullptr, *volume = nullptr, *dt_factor = nullptr;
    double *elem_mass = nullptr, *elem_dt = nullptr, *elem_extra = nullptr, *dt_partials = nullptr;
    double *u_tmp = nullptr, *f_tmp = nullptr, *n_tmp = nullptr, *n_tmp2 = nullptr, *e_tmp = nullptr;
    uint8_t *fixed = nullptr, *eroded_all = nullptr;
    uint32_t *conn_all = nullptr, *hc_off = nullptr, *hc_slot = nullptr, *all_off = nullptr, *all_slot = nullptr;
    int32_t* part = nullptr;
    double* mat3 = nullptr;
    int64_t* hc_index_d = nullptr;
    float4 *planes = nullptr, *state = nullptr;
    float* corner = nullptr;
    MaterialF32* mats = nullptr;
    Control* ctl = nullptr;      // the run
    Control* ctl_aux = nullptr;  // drop-in calls
    int dt_blocks = 1;

    // contact
    ContactArrays ca{};
    int n_contacts = 0;
    long long n_faces = 0, n_slaves = 0;
    int entries_cap = 0;
    std::vector<std::vector<uint32_t>> contact_nodes_all;  // unfiltered primary nodes (for contact_dt)
    std::vector<double> contact_stiffness;

    // vehicles
    int n_veh = 0;
    long long* veh_off = nullptr;
    uint32_t* veh_nodes = nullptr;
    double* veh_out = nullptr;
    std::vector<uint32_t> veh_accel;
    std::vector<std::vector<uint32_t>> veh_front;

    // run
    bool run_open = false;
    long long host_step = 0;
    int period = 20;
    cudaGraphExec_t graph = nullptr;
    int64_t graph_launches = 0;
    bool profiling = false;
    int prof_level = 2;  // 1: events around the element-force kernel only; 2: every phase
    bool last_was_graph = false;
    std::vector<cudaEvent_t> prof_ev;

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
        return e;
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
        a.inv_mass = inv_mass;
        a.mass = mass;
        a.added = added;
        a.fixed = fixed;
        a.hc_off = hc_off;
        a.hc_slot = hc_slot;
        a.all_off = all_off;
        a.all_slot = all_slot;
        return a;
    }

    template <typename T>
    int alloc(T** p, size_t count) {
        *p = nullptr;
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T));
        if (e != cudaSuccess) {
            cudaGetLastError();
            return crush::fail(e == cudaErrorMemoryAllocation ? CRUSH_ERR_OOM : CRUSH_ERR_CUDA,
                               std::string("cudaMalloc: ") + cudaGetErrorString(e));
        }
        allocs.push_back(*p);
        return CRUSH_OK;
    }
    template <typename T>
    int upload(T** p, const T* host, size_t count) {
        int st = alloc(p, count);
        if (st != CRUSH_OK) return st;
        if (count) CK(cudaMemcpyAsync(*p, host, count * sizeof(T), cudaMemcpyHostToDevice, stream));
        return CRUSH_OK;
    }
    ~crush_ctx() {
        if (graph) cudaGraphExecDestroy(graph);
        for (cudaEvent_t e : prof_ev) cudaEventDestroy(e);
        if (stream) cudaStreamSynchronize(stream);
        for (void* p : allocs) cudaFree(p);
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

int create_impl(const crush_model_desc* d, int device, crush_ctx* c) {
    if (!d || d->n_nodes <= 0 || !d->positions || d->n_hexes < 0 || (d->n_hexes > 0 && (!d->hexes || !d->hex_part)))
        return crush::fail(CRUSH_ERR_INVALID, "invalid model description");
    if (d->n_nodes >= (1ll << 31) || d->n_hexes >= (1ll << 28)) return crush::fail(CRUSH_ERR_INVALID, "model too large");
    if (d->n_parts <= 0 || !d->materials) return crush::fail(CRUSH_ERR_INVALID, "model needs at least one material");
    const crush_settings& s = d->settings;
    if (!(s.dt_scale > 0.0) || s.adaptive_check_steps < 0 || !(s.hourglass >= 0.0))
        return crush::fail(CRUSH_ERR_INVALID, "invalid settings");
    c->settings = s;
    c->device = device;
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    const long long N = d->n_nodes, E = d->n_hexes;
    c->n_nodes = N;
    c->n_all = E;

    // Fixed nodes.
    std::vector<uint8_t> fixed(N, 0);
    for (int64_t i = 0; i < d->n_fixed; ++i) {
        if (d->fixed_nodes[i] >= (uint64_t)N) return crush::fail(CRUSH_ERR_INVALID, "fixed node out of range");
        fixed[d->fixed_nodes[i]] = 1;
    }
    // Materials.
    std::vector<MaterialF32> mats(d->n_parts);
    std::vector<double> mat3(3 * d->n_parts);
    for (int p = 0; p < d->n_parts; ++p) {
        const crush_material& m = d->materials[p];
        if (!(m.density > 0.0) || !(m.youngs_modulus > 0.0) || !(m.poisson_ratio >= 0.0 && m.poisson_ratio < 0.5))
            return crush::fail(CRUSH_ERR_INVALID, "material " + std::to_string(p) + ": needs E > 0, density > 0, 0 <= nu < 0.5");
        mat3[3 * p] = m.youngs_modulus;
        mat3[3 * p + 1] = m.poisson_ratio;
        mat3[3 * p + 2] = m.density;
        std::memset(&mats[p], 0, sizeof(MaterialF32));
        if (m.model == CRUSH_MAT_HONEYCOMB) {
            double knots[MAX_KNOTS][3];
            std::string err;
            if (honeycomb_params(m, knots, &err) != 0) return crush::fail(CRUSH_ERR_INVALID, "material " + std::to_string(p) + ": " + err);
            mats[p].youngs = (float)m.youngs_modulus;
            mats[p].trans = (float)m.transverse_factor;
            for (int k = 0; k < MAX_KNOTS; ++k) {
                mats[p].knot_c[k] = (float)knots[k][0];
                mats[p].knot_s[k] = (float)knots[k][1];
                mats[p].knot_h[k] = (float)knots[k][2];
            }
        } else if (m.model != CRUSH_MAT_ELASTIC) {
            return crush::fail(CRUSH_ERR_UNSUPPORTED, "unknown material model");
        }
    }
    // Elements: honeycomb ones run the force kernel; elastic ones must be rigid.
    c->hc_index.assign(E, -1);
    c->hc_model.clear();
    for (long long e = 0; e < E; ++e) {
        int p = d->hex_part[e];
        if (p < 0 || p >= d->n_parts) return crush::fail(CRUSH_ERR_INVALID, "hexahedron part out of range");
        for (int i = 0; i < 8; ++i)
            if (d->hexes[8 * e + i] >= (uint64_t)N) return crush::fail(CRUSH_ERR_INVALID, "hexahedron node out of range");
        if (d->materials[p].model == CRUSH_MAT_HONEYCOMB) {
            c->hc_index[e] = (int64_t)c->hc_model.size();
            c->hc_model.push_back((uint32_t)e);
        } else {
            for (int i = 0; i < 8; ++i)
                if (!fixed[d->hexes[8 * e + i]])
                    return crush::fail(CRUSH_ERR_UNSUPPORTED, "elastic elements are supported only as rigid slabs (every node fixed)");
        }
    }
    c->n_hc = (long long)c->hc_model.size();
    c->stride = std::max<long long>(32, (c->n_hc + 31) / 32 * 32);
    // Node incidence CSRs, slots in increasing element order.
    std::vector<uint32_t> all_off(N + 1, 0), hc_off(N + 1, 0);
    for (long long e = 0; e < E; ++e)
        for (int i = 0; i < 8; ++i) {
            all_off[d->hexes[8 * e + i] + 1]++;
            if (c->hc_index[e] >= 0) hc_off[d->hexes[8 * e + i] + 1]++;
        }
    for (long long n = 0; n < N; ++n) {
        all_off[n + 1] += all_off[n];
        hc_off[n + 1] += hc_off[n];
    }
    std::vector<uint32_t> all_slot(all_off[N]), hc_slot(hc_off[N]);
    {
        std::vector<uint32_t> ca(all_off.begin(), all_off.end() - 1), ch(hc_off.begin(), hc_off.end() - 1);
        for (long long e = 0; e < E; ++e)
            for (int i = 0; i < 8; ++i) {
                uint32_t n = d->hexes[8 * e + i];
                all_slot[ca[n]++] = (uint32_t)(8 * e + i);
                if (c->hc_index[e] >= 0) hc_slot[ch[n]++] = (uint32_t)(8 * c->hc_index[e] + i);
            }
    }

    int st;
#define TRY(x) do { st = (x); if (st != CRUSH_OK) return st; } while (0)
    TRY(c->upload(&c->pos, d->positions, 3 * N));
    TRY(c->upload(&c->conn_all, d->hexes, 8 * E));
    TRY(c->upload(&c->part, d->hex_part, E));
    TRY(c->upload(&c->mat3, mat3.data(), mat3.size()));
    TRY(c->upload(&c->mats, mats.data(), mats.size()));
    TRY(c->upload(&c->hc_index_d, c->hc_index.data(), E));
    TRY(c->upload(&c->fixed, fixed.data(), N));
    TRY(c->upload(&c->all_off, all_off.data(), N + 1));
    TRY(c->upload(&c->all_slot, all_slot.data(), all_slot.size()));
    TRY(c->upload(&c->hc_off, hc_off.data(), N + 1));
    TRY(c->upload(&c->hc_slot, hc_slot.data(), hc_slot.size()));
    std::vector<double> v0(3 * N, 0.0);
    if (d->initial_velocity) std::copy(d->initial_velocity, d->initial_velocity + 3 * N, v0.begin());
    TRY(c->upload(&c->v0, v0.data(), 3 * N));
    for (double** p : {&c->u, &c->v, &c->v_half, &c->f_int, &c->f_ext, &c->u_tmp, &c->f_tmp}) TRY(c->alloc(p, 3 * N));
    for (double** p : {&c->inv_mass, &c->mass, &c->added, &c->n_tmp, &c->n_tmp2}) TRY(c->alloc(p, N));
    for (double** p : {&c->volume, &c->dt_factor, &c->elem_mass, &c->elem_dt, &c->elem_extra, &c->e_tmp}) TRY(c->alloc(p, E));
    TRY(c->alloc(&c->lumped, 8 * E));
    TRY(c->alloc(&c->eroded_all, E));
    c->dt_blocks = elem_dt_blocks(E);
    TRY(c->alloc(&c->dt_partials, c->dt_blocks));
    TRY(c->alloc(&c->planes, (size_t)N_STATIC_PLANES * c->stride));
    TRY(c->alloc(&c->state, (size_t)N_STATE_PLANES * c->stride));
    TRY(c->alloc(&c->corner, (size_t)24 * std::max<long long>(c->n_hc, 1)));
    TRY(c->alloc(&c->ctl, 1));
    TRY(c->alloc(&c->ctl_aux, 1));
    CK(cudaMemsetAsync(c->planes, 0, sizeof(float4) * N_STATIC_PLANES * c->stride, c->stream));
    CK(cudaMemsetAsync(c->eroded_all, 0, E, c->stream));

    // Device set-up geometry (HexGeometry::new for every element).
    int* bad = nullptr;
    TRY(c->alloc(&bad, 1));
    CK(cudaMemsetAsync(bad, 0, sizeof(int), c->stream));
    launch_setup_geometry(c->stream, E, c->pos, c->conn_all, c->part, c->mat3, s.hourglass, c->hc_index_d, c->stride, c->planes,
                          c->volume, c->lumped, c->dt_factor, c->elem_mass, bad);
    TRY(check_launch(c));
    launch_node_masses(c->stream, N, c->all_off, c->all_slot, c->lumped, c->mass, c->inv_mass);
    TRY(check_launch(c));
    int bad_h = 0;
    CK(cudaMemcpyAsync(&bad_h, bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    std::vector<double> mass_h(N);
    CK(cudaMemcpyAsync(mass_h.data(), c->mass, N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (bad_h == 1) return crush::fail(CRUSH_ERR_INVALID, "degenerate hexahedron (singular Jacobian)");
    if (bad_h == 2) return crush::fail(CRUSH_ERR_INVALID, "hourglass modes not independent");

    // ---- contacts (ContactRuntime::new, src/contact.rs:48-70) ----
    c->n_contacts = d->n_contacts;
    std::vector<int> face_off(1, 0), slave_off(1, 0), tab_off(1, 0), counts_for_stop;
    std::vector<uint32_t> faces, slaves;
    std::vector<double> scales, stiff, md, cell;
    // roles per node: contact, position among the contact's primary nodes
    // (-1: none), and the contact's faces that contain the node
    struct Role {
        int c;
        int slave;
        std::vector<int> faces;
    };
    std::map<uint32_t, std::vector<Role>> roles;
    for (int k = 0; k < d->n_contacts; ++k) {
        const crush_contact& cd = d->contacts[k];
        if (cd.n_nodes < 0 || cd.n_faces < 0 || (cd.n_nodes > 0 && !cd.nodes) || (cd.n_faces > 0 && !cd.faces))
            return crush::fail(CRUSH_ERR_INVALID, "invalid contact " + std::to_string(k));
        if (!(cd.max_distance >= 0.0) || !(cd.stiffness >= 0.0)) return crush::fail(CRUSH_ERR_INVALID, "invalid contact parameters");
        double lo[3] = {INF, INF, INF}, hi[3] = {-INF, -INF, -INF};
        bool stop = false;
        double ext = 0.0;
        std::vector<std::array<double, 6>> keys;  // grid key box of each face at the reference positions
        for (int64_t f = 0; f < cd.n_faces; ++f) {
            double flo[3] = {INF, INF, INF}, fhi[3] = {-INF, -INF, -INF};
            double xs[4][3];
            for (int j = 0; j < 4; ++j) {
                uint32_t n = cd.faces[4 * f + j];
                if (n >= (uint64_t)N) return crush::fail(CRUSH_ERR_INVALID, "contact face node out of range");
                faces.push_back(n);
                if (!fixed[n]) stop = true;
                for (int dd = 0; dd < 3; ++dd) {
                    double p = d->positions[3 * n + dd];
                    xs[j][dd] = p;
                    lo[dd] = std::fmin(lo[dd], p);
                    hi[dd] = std::fmax(hi[dd], p);
                    flo[dd] = std::fmin(flo[dd], p);
                    fhi[dd] = std::fmax(fhi[dd], p);
                }
            }
            double fext = std::max({fhi[0] - flo[0], fhi[1] - flo[1], fhi[2] - flo[2]});
            ext = std::max(ext, fext);
            double e1[3], e2[3], nrm[3];
            for (int dd = 0; dd < 3; ++dd) { e1[dd] = xs[1][dd] - xs[0][dd]; e2[dd] = xs[2][dd] - xs[0][dd]; }
            nrm[0] = e1[1] * e2[2] - e1[2] * e2[1];
            nrm[1] = e1[2] * e2[0] - e1[0] * e2[2];
            nrm[2] = e1[0] * e2[1] - e1[1] * e2[0];
            double len = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
            std::array<double, 6> kb;
            for (int dd = 0; dd < 3; ++dd) {
                double nd = len > 0.0 ? nrm[dd] / len : 0.0;
                kb[dd] = flo[dd] - 0.25 * fext - cd.max_distance * std::max(nd, 0.0);
                kb[3 + dd] = fhi[dd] + 0.25 * fext + cd.max_distance * std::max(-nd, 0.0);
            }
            keys.push_back(kb);
        }
        for (int dd = 0; dd < 3; ++dd) { lo[dd] += -cd.max_distance; hi[dd] += cd.max_distance; }
        std::vector<uint32_t> all_nodes;
        int kept = 0;
        for (int64_t i = 0; i < cd.n_nodes; ++i) {
            uint32_t n = cd.nodes[i];
            if (n >= (uint64_t)N) return crush::fail(CRUSH_ERR_INVALID, "contact node out of range");
            all_nodes.push_back(n);
            bool inside = true;
            for (int dd = 0; dd < 3; ++dd) {
                double p = d->positions[3 * n + dd];
                if (!(p >= lo[dd] && p <= hi[dd])) inside = false;
            }
            if (!inside) continue;
            slaves.push_back(n);
            scales.push_back(cd.node_scale ? cd.node_scale[i] : 1.0);
            roles[n].push_back(Role{k, kept, {}});
            ++kept;
        }
        for (int64_t f = 0; f < cd.n_faces; ++f)
            for (int j = 0; j < 4; ++j) {
                uint32_t n = cd.faces[4 * f + j];
                auto& r = roles[n];
                if (r.empty() || r.back().c != k) r.push_back(Role{k, -1, {}});
                if (r.back().faces.empty() || r.back().faces.back() != (int)f) r.back().faces.push_back((int)f);
            }
        c->contact_nodes_all.push_back(all_nodes);
        c->contact_stiffness.push_back(cd.stiffness);
        face_off.push_back(face_off.back() + (int)cd.n_faces);
        slave_off.push_back(slave_off.back() + kept);
        // Grid cell: twice the largest face; table: twice the initial key-box
        // cell count, a power of two.
        const double cs = ext > 0.0 ? 2.0 * ext : 1.0;
        size_t inserts = 0;
        for (const auto& kb : keys) {
            size_t cells = 1;
            for (int dd = 0; dd < 3; ++dd) cells *= (size_t)(std::floor(kb[3 + dd] / cs) - std::floor(kb[dd] / cs) + 1.0);
            inserts += std::min<size_t>(cells, 128);
        }
        size_t t = next_pow2(std::max<size_t>(1024, 2 * inserts));
        tab_off.push_back(tab_off.back() + (int)t);
        stiff.push_back(cd.stiffness);
        md.push_back(cd.max_distance);
        cell.push_back(cs);
        counts_for_stop.push_back(stop ? 1 : 0);
    }
    c->n_faces = face_off.back();
    c->n_slaves = slave_off.back();
    c->entries_cap = 0;
    std::vector<uint32_t> cnode, cnode_off(1, 0);
    std::vector<int> crole_contact, crole_slave, crole_faces;
    std::vector<uint8_t> crole_face;
    std::vector<uint32_t> crole_faces_off(1, 0);
    for (auto& kv : roles) {
        cnode.push_back(kv.first);
        for (auto& r : kv.second) {
            crole_contact.push_back(r.c);
            crole_slave.push_back(r.slave);
            crole_face.push_back(r.faces.empty() ? 0 : 1);
            crole_faces.insert(crole_faces.end(), r.faces.begin(), r.faces.end());
            crole_faces_off.push_back((uint32_t)crole_faces.size());
        }
        cnode_off.push_back((uint32_t)crole_contact.size());
    }
    ContactArrays& ca = c->ca;
    ca.n_contacts = c->n_contacts;
    int nc1 = c->n_contacts + 1;
    TRY(c->upload(const_cast<int**>(&ca.face_off), face_off.data(), nc1));
    TRY(c->upload(const_cast<uint32_t**>(&ca.faces), faces.data(), faces.size()));
    TRY(c->alloc(&ca.geo, std::max<long long>(c->n_faces, 1)));
    TRY(c->upload(const_cast<int**>(&ca.slave_off), slave_off.data(), nc1));
    TRY(c->upload(const_cast<uint32_t**>(&ca.slaves), slaves.data(), slaves.size()));
    TRY(c->upload(const_cast<double**>(&ca.slave_scale), scales.data(), scales.size()));
    TRY(c->alloc(&ca.hit, std::max<long long>(c->n_slaves, 1)));
    TRY(c->alloc(&ca.hit_force, 3 * std::max<long long>(c->n_slaves, 1)));
    TRY(c->upload(const_cast<double**>(&ca.stiffness), stiff.data(), stiff.size()));
    TRY(c->upload(const_cast<double**>(&ca.max_distance), md.data(), md.size()));
    TRY(c->upload(const_cast<double**>(&ca.cell), cell.data(), cell.size()));
    TRY(c->upload(const_cast<int**>(&ca.tab_off), tab_off.data(), nc1));
    TRY(c->alloc(&ca.counts, std::max(tab_off.back(), 1)));
    TRY(c->alloc(&ca.entries, (size_t)std::max(tab_off.back(), 1) * BUCKET_CAP));
    ca.overflow_cap = (int)std::max<long long>(1, face_off.empty() ? 1 : *std::max_element(face_off.begin(), face_off.end()));
    {
        int cap = 1;
        for (int k = 0; k < c->n_contacts; ++k) cap = std::max(cap, face_off[k + 1] - face_off[k]);
        ca.overflow_cap = cap;
    }
    TRY(c->alloc(&ca.overflow, (size_t)std::max(c->n_contacts, 1) * ca.overflow_cap));
    TRY(c->alloc(&ca.n_overflow, std::max(c->n_contacts, 1)));
    TRY(c->alloc(&ca.entry_overrun, std::max(c->n_contacts, 1)));
    TRY(c->alloc(&ca.pen_count, std::max(c->n_contacts, 1)));
    TRY(c->alloc(&ca.pen_max_bits, std::max(c->n_contacts, 1)));
    TRY(c->upload(const_cast<int**>(&ca.counts_for_stop), counts_for_stop.data(), counts_for_stop.size()));
    ca.n_cnodes = (long long)cnode.size();
    TRY(c->upload(const_cast<uint32_t**>(&ca.cnode), cnode.data(), cnode.size()));
    TRY(c->upload(const_cast<uint32_t**>(&ca.cnode_off), cnode_off.data(), cnode_off.size()));
    TRY(c->upload(const_cast<int**>(&ca.crole_contact), crole_contact.data(), crole_contact.size()));
    TRY(c->upload(const_cast<int**>(&ca.crole_slave), crole_slave.data(), crole_slave.size()));
    TRY(c->upload(const_cast<uint8_t**>(&ca.crole_face), crole_face.data(), crole_face.size()));
    TRY(c->upload(const_cast<uint32_t**>(&ca.crole_faces_off), crole_faces_off.data(), crole_faces_off.size()));
    TRY(c->upload(const_cast<int**>(&ca.crole_faces), crole_faces.data(), crole_faces.size()));
    TRY(c->alloc(&ca.face_hits, std::max<long long>(c->n_faces, 1)));
    TRY(c->alloc(&ca.face_list, (size_t)std::max<long long>(c->n_faces, 1) * FACE_HIT_CAP));
    CK(cudaMemsetAsync(ca.face_hits, 0, sizeof(int) * std::max<long long>(c->n_faces, 1), c->stream));
    CK(cudaMemsetAsync(ca.counts, 0, sizeof(int) * std::max(tab_off.back(), 1), c->stream));
    CK(cudaMemsetAsync(ca.n_overflow, 0, sizeof(int) * std::max(c->n_contacts, 1), c->stream));
    CK(cudaMemsetAsync(ca.entry_overrun, 0, sizeof(int) * std::max(c->n_contacts, 1), c->stream));
    CK(cudaMemsetAsync(ca.pen_count, 0, sizeof(unsigned long long) * std::max(c->n_contacts, 1), c->stream));
    CK(cudaMemsetAsync(ca.pen_max_bits, 0, sizeof(unsigned long long) * std::max(c->n_contacts, 1), c->stream));

    // ---- vehicles ----
    c->n_veh = std::min(d->n_vehicles, 4);
    std::vector<long long> voff(1, 0);
    std::vector<uint32_t> vnodes;
    for (int k = 0; k < c->n_veh; ++k) {
        const crush_vehicle& vd = d->vehicles[k];
        for (int64_t i = 0; i < vd.n_nodes; ++i) {
            if (vd.nodes[i] >= (uint64_t)N) return crush::fail(CRUSH_ERR_INVALID, "vehicle node out of range");
            vnodes.push_back(vd.nodes[i]);
        }
        voff.push_back((long long)vnodes.size());
        if (vd.accel_node >= (uint64_t)N) return crush::fail(CRUSH_ERR_INVALID, "accelerometer node out of range");
        c->veh_accel.push_back(vd.accel_node);
        std::vector<uint32_t> fr(vd.front_nodes, vd.front_nodes + vd.n_front);
        for (uint32_t n : fr)
            if (n >= (uint64_t)N) return crush::fail(CRUSH_ERR_INVALID, "front node out of range");
        c->veh_front.push_back(fr);
    }
    TRY(c->upload(&c->veh_off, voff.data(), voff.size()));
    TRY(c->upload(&c->veh_nodes, vnodes.data(), vnodes.size()));
    TRY(c->alloc(&c->veh_out, 7 * 4));

    // ---- time step (src/solver.rs:214-228) ----
    for (size_t k = 0; k < c->contact_nodes_all.size(); ++k)
        for (uint32_t n : c->contact_nodes_all[k])
            if (mass_h[n] > 0.0 && c->contact_stiffness[k] > 0.0)
                c->contact_dt = std::fmin(c->contact_dt, 2.0 * std::sqrt(mass_h[n] / c->contact_stiffness[k]));
    launch_init_state(c->stream, c->n_hc, c->stride, c->state);
    TRY(check_launch(c));
    CK(cudaMemsetAsync(c->u_tmp, 0, sizeof(double) * 3 * N, c->stream));
    Control aux{};
    aux.dt_stable_bits = 0x7ff0000000000000ull;
    aux.dt_floor = 0.0;
    CK(cudaMemcpyAsync(c->ctl_aux, &aux, sizeof(Control), cudaMemcpyHostToDevice, c->stream));
    launch_elem_dt(c->stream, c->el(), c->nd(), c->ctl_aux, c->u_tmp, c->dt_partials, 0);
    TRY(check_launch(c));
    CK(cudaMemcpyAsync(&aux, c->ctl_aux, sizeof(Control), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    double stable;
    std::memcpy(&stable, &aux.dt_stable_bits, sizeof(double));
    if (!std::isfinite(stable)) {
        static const int EDGES[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6}, {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
        double mn = INF, cmax = 0.0;
        for (long long e = 0; e < E; ++e) {
            cmax = std::fmax(cmax, wave_speed(d->materials[d->hex_part[e]]));
            for (auto& ed : EDGES) {
                const double* p = d->positions + 3 * d->hexes[8 * e + ed[0]];
                const double* q = d->positions + 3 * d->hexes[8 * e + ed[1]];
                mn = std::fmin(mn, std::sqrt((p[0] - q[0]) * (p[0] - q[0]) + (p[1] - q[1]) * (p[1] - q[1]) + (p[2] - q[2]) * (p[2] - q[2])));
            }
        }
        stable = mn / (std::sqrt(3.0) * cmax);
    }
    c->stable = std::fmin(stable, c->contact_dt);
    c->dt_floor = s.mass_scaling > 0.0 ? s.mass_scaling * c->stable : 0.0;
    c->dt0 = s.time_step > 0.0 ? s.time_step : c->stable * s.dt_scale;
    int chk = s.adaptive_check_steps > 0 ? s.adaptive_check_steps : 1;
    c->period = std::lcm(chk, 20);
    if (c->period > 200) c->period = 0;  // no graph for odd periods
    return CRUSH_OK;
#undef TRY
}

int sync(crush_ctx* c) {
    CK(cudaStreamSynchronize(c->stream));
    return CRUSH_OK;
}

// One explicit step on the stream (src/solver.rs:287-345).
// Phase boundaries of one step recorded when profiling: start, after dt,
// after contact, after half step, after element forces, after full step, end.
constexpr int N_PHASE_EVENTS = 7;

int enqueue_step(crush_ctx* c, long long step, cudaEvent_t* ev = nullptr, bool capturing = false) {
    const crush_settings& s = c->settings;
    ElementArrays el = c->el();
    NodeArrays nd = c->nd();
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
    const bool adaptive = !(s.time_step > 0.0) && s.adaptive_check_steps > 0;
    if (adaptive && step % s.adaptive_check_steps == 0) {
        launch_elem_dt(c->stream, el, nd, c->ctl, c->u, c->dt_partials, 1);
        launch_dt_finalize(c->stream, c->ctl, c->dt_partials, c->dt_blocks);
        launch_mass_scaling(c->stream, el, nd, c->ctl, 0);
        n += 3;
    }
    mark(1);
    if (c->n_contacts > 0) {
        launch_contact(c->stream, c->ca, nd, c->ctl, 0, c->n_contacts, c->n_faces, c->n_slaves, c->entries_cap, 0.0, c->mass, c->f_ext, 1);
        n += (c->n_faces > 0 ? 1 : 0) + (c->n_slaves > 0 ? 1 : 0) + 1;
    }
    mark(2);
    launch_half(c->stream, nd, c->ctl);
    mark(3);
    launch_forces(c->stream, el, nd, c->ctl, 1);
    mark(4);
    launch_full(c->stream, el, nd, c->ctl);
    mark(5);
    n += 2 + (c->n_hc > 0 ? 1 : 0);
    if ((step + 1) % 20 == 0) {
        launch_nonfinite(c->stream, nd, c->ctl);
        ++n;
    }
    const bool sep = s.stop_rule == CRUSH_STOP_SEPARATION && (step + 1) % 10 == 0 && c->n_veh >= 2;
    if (sep) {
        launch_vehicle_vx(c->stream, c->n_veh, c->veh_off, c->veh_nodes, c->mass, c->v, c->ctl);
        ++n;
    }
    launch_step_end(c->stream, c->ctl, c->ca, sep ? 1 : 0);
    ++n;
    mark(6);
    return check_launch(c, n);
}

int run_begin(crush_ctx* c) {
    const long long N = c->n_nodes;
    if (c->graph) {
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
    CK(cudaMemsetAsync(c->u, 0, sizeof(double) * 3 * N, c->stream));
    CK(cudaMemcpyAsync(c->v, c->v0, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemsetAsync(c->v_half, 0, sizeof(double) * 3 * N, c->stream));
    CK(cudaMemsetAsync(c->f_ext, 0, sizeof(double) * 3 * N, c->stream));
    CK(cudaMemsetAsync(c->added, 0, sizeof(double) * N, c->stream));
    CK(cudaMemsetAsync(c->eroded_all, 0, c->n_all, c->stream));
    launch_init_state(c->stream, c->n_hc, c->stride, c->state);
    launch_node_masses(c->stream, N, c->all_off, c->all_slot, c->lumped, c->mass, c->inv_mass);
    int st = check_launch(c, 2);
    if (st != CRUSH_OK) return st;
    Control h{};
    h.t = 0.0;
    h.end_time = c->settings.end_time;
    h.dt_cfl = c->dt0;
    h.dt_min = INF;
    h.dt_floor = c->dt_floor;
    h.dt_scale = c->settings.dt_scale;
    h.contact_dt = c->contact_dt;
    h.damping = c->settings.velocity_damping;
    h.dt_stable_bits = 0x7ff0000000000000ull;
    h.step = 0;
    h.last_hit = -1;
    h.max_steps = c->settings.max_steps;
    h.done = (0.0 < c->settings.end_time) ? 0 : 1;
    h.stop_rule = c->settings.stop_rule;
    CK(cudaMemcpyAsync(c->ctl, &h, sizeof(Control), cudaMemcpyHostToDevice, c->stream));
    // Initial internal forces at u = 0 (src/solver.rs:254); the count of
    // elements it erodes is not added to the run's total (as there).
    launch_forces(c->stream, c->el(), c->nd(), c->ctl, 0);
    launch_gather(c->stream, c->el(), c->nd(), c->f_int);
    st = check_launch(c, 2);
    if (st != CRUSH_OK) return st;
    long long zero = 0;
    CK(cudaMemcpyAsync(&c->ctl->eroded_step, &zero, sizeof(long long), cudaMemcpyHostToDevice, c->stream));
    c->host_step = 0;
    c->run_open = true;
    return sync(c);
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
    if (e != cudaSuccess) return crush::fail(CRUSH_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&c->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return crush::fail(CRUSH_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    return CRUSH_OK;
}

int run_steps(crush_ctx* c, long long n_steps, int* done) {
    if (!c->run_open) return crush::fail(CRUSH_ERR_INVALID, "no open run (call crush_run_begin)");
    long long issued = 0;
    int st;
    while (issued < n_steps) {
        if (c->period > 0 && c->host_step % c->period == 0 && n_steps - issued >= c->period) {
            if (!c->graph) {
                int64_t before = c->launches;
                st = build_graph(c);
                if (st != CRUSH_OK) return st;
                c->graph_launches = c->launches - before;
                c->launches = before;
            }
            CK(cudaGraphLaunch(c->graph, c->stream));
            c->launches += c->graph_launches;
            c->host_step += c->period;
            issued += c->period;
        } else {
            if (c->profiling) {
                st = ensure_prof_events(c);
                if (st != CRUSH_OK) return st;
            }
            st = enqueue_step(c, c->host_step, c->profiling ? &c->prof_ev[0] : nullptr);
            if (st != CRUSH_OK) return st;
            c->host_step += 1;
            issued += 1;
            c->last_was_graph = false;
            continue;
        }
        c->last_was_graph = true;
    }
    int d = 0;
    CK(cudaMemcpyAsync(&d, &c->ctl->done, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (done) *done = d;
    return CRUSH_OK;
}

int results(crush_ctx* c, crush_results* r) {
    Control h;
    CK(cudaMemcpyAsync(&h, c->ctl, sizeof(Control), cudaMemcpyDeviceToHost, c->stream));
    launch_vehicle_sums(c->stream, c->n_veh, c->veh_off, c->veh_nodes, c->mass, c->v, c->v0, c->veh_out);
    int st = check_launch(c, c->n_veh > 0 ? 1 : 0);
    if (st != CRUSH_OK) return st;
    double sums[28];
    if (c->n_veh > 0) CK(cudaMemcpyAsync(sums, c->veh_out, sizeof(double) * 7 * c->n_veh, cudaMemcpyDeviceToHost, c->stream));
    // Crush needs u_x of the accelerometer and front nodes only.
    std::vector<double> u(3 * c->n_nodes);
    CK(cudaMemcpyAsync(u.data(), c->u, sizeof(double) * 3 * c->n_nodes, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::memset(r, 0, sizeof(*r));
    r->time = h.t;
    r->steps = h.step;
    r->eroded_elements = h.eroded_total;
    r->dt_min = h.dt_min;
    r->added_mass_max = h.added_mass_max;
    r->status = h.status;
    r->n_vehicles = c->n_veh;
    for (int k = 0; k < c->n_veh; ++k) {
        const double* s = sums + 7 * k;
        crush_vehicle_result& vr = r->vehicle[k];
        vr.mass = s[0];
        for (int dd = 0; dd < 3; ++dd) {
            double v1 = s[0] > 0.0 ? s[1 + dd] / s[0] : 0.0;
            double v0 = s[0] > 0.0 ? s[4 + dd] / s[0] : 0.0;
            vr.velocity[dd] = v1;
            vr.delta_v[dd] = v1 - v0;
        }
        double fu = 0.0;
        for (uint32_t n : c->veh_front[k]) fu += u[3 * (size_t)n];
        fu = c->veh_front[k].empty() ? 0.0 : fu / (double)c->veh_front[k].size();
        vr.crush = std::fabs(u[3 * (size_t)c->veh_accel[k]] - fu);
    }
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

int crush_create(const crush_model_desc* desc, int device, crush_ctx** out) {
    if (!out) return crush::fail(CRUSH_ERR_INVALID, "null output");
    *out = nullptr;
    crush_ctx* c = new crush_ctx();
    int st = create_impl(desc, device, c);
    if (st != CRUSH_OK) {
        delete c;
        return st;
    }
    *out = c;
    return CRUSH_OK;
}

void crush_destroy(crush_ctx* ctx) { delete ctx; }

int crush_sizes(const crush_ctx* c, int64_t* n_nodes, int64_t* n_hexes, int64_t* n_active) {
    if (!c) return crush::fail(CRUSH_ERR_INVALID, "null context");
    if (n_nodes) *n_nodes = c->n_nodes;
    if (n_hexes) *n_hexes = c->n_all;
    if (n_active) *n_active = c->n_hc;
    return CRUSH_OK;
}

int64_t crush_launch_count(const crush_ctx* c) { return c ? c->launches : 0; }

int crush_compute_forces_device(crush_ctx* c, const double* u_device, double* f_device, int64_t* newly) {
    if (!c || !u_device || !f_device) return crush::fail(CRUSH_ERR_INVALID, "null argument");
    CK(cudaSetDevice(c->device));
    NodeArrays nd = c->nd();
    nd.u = const_cast<double*>(u_device);
    if (newly) {
        CK(cudaMemsetAsync(&c->ctl_aux->eroded_step, 0, sizeof(long long), c->stream));
        CK(cudaMemsetAsync(&c->ctl_aux->copy_timeout, 0, sizeof(int), c->stream));
    }
    launch_forces(c->stream, c->el(), nd, c->ctl_aux, 0);
    launch_gather(c->stream, c->el(), nd, f_device);
    int st = check_launch(c, (c->n_hc > 0 ? 1 : 0) + 1);
    if (st != CRUSH_OK) return st;
    if (newly) {
        long long k = 0;
        int timeout = 0;
        CK(cudaMemcpyAsync(&k, &c->ctl_aux->eroded_step, sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(&timeout, &c->ctl_aux->copy_timeout, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        if (timeout) return crush::fail(CRUSH_ERR_TIMEOUT, "element tile copy did not complete");
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
    // host mirror of this contact's face / slave ranges
    int fo[2], so[2];
    CK(cudaMemcpyAsync(fo, c->ca.face_off + id, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(so, c->ca.slave_off + id, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    launch_contact(c->stream, c->ca, nd, nullptr, id, id + 1, fo[1] - fo[0], so[1] - so[0], c->entries_cap, dt, m, c->f_tmp, 0);
    int st = check_launch(c, (fo[1] > fo[0] ? 1 : 0) + (so[1] > so[0] ? 1 : 0) + 1);
    if (st != CRUSH_OK) return st;
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
    Control aux{};
    aux.dt_stable_bits = 0x7ff0000000000000ull;
    CK(cudaMemcpyAsync(c->ctl_aux, &aux, sizeof(Control), cudaMemcpyHostToDevice, c->stream));
    launch_elem_dt(c->stream, c->el(), c->nd(), c->ctl_aux, c->u_tmp, c->dt_partials, 0);
    int st = check_launch(c);
    if (st != CRUSH_OK) return st;
    unsigned long long bits = 0;
    CK(cudaMemcpyAsync(&bits, &c->ctl_aux->dt_stable_bits, sizeof(bits), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::memcpy(dt, &bits, sizeof(double));
    return std::isfinite(*dt) ? CRUSH_OK : CRUSH_NONE;
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
    Control aux{};
    aux.dt_stable_bits = 0x7ff0000000000000ull;
    aux.dt_floor = dt_min;
    CK(cudaMemcpyAsync(c->ctl_aux, &aux, sizeof(Control), cudaMemcpyHostToDevice, c->stream));
    NodeArrays nd = c->nd();
    nd.added = c->n_tmp;
    nd.inv_mass = c->n_tmp2;
    launch_elem_dt(c->stream, el, nd, c->ctl_aux, c->u_tmp, c->dt_partials, 0);
    launch_mass_scaling(c->stream, el, nd, c->ctl_aux, 1);
    int st = check_launch(c, 2);
    if (st != CRUSH_OK) return st;
    std::vector<double> parts(c->dt_blocks);
    CK(cudaMemcpyAsync(added, c->n_tmp, sizeof(double) * c->n_nodes, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(parts.data(), c->dt_partials, sizeof(double) * c->dt_blocks, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    double t = 0.0;
    for (double p : parts) t += p;
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
    return results(c, r);
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
        if (c->graph) {
            cudaGraphExecDestroy(c->graph);
            c->graph = nullptr;
        }
    }
    return CRUSH_OK;
}

int crush_run_steps_timed(crush_ctx* c, int64_t n_steps, int* done, double* ms, double* phase_ms, int* phase_steps) {
    if (!c) return crush::fail(CRUSH_ERR_INVALID, "null context");
    CK(cudaSetDevice(c->device));
    const bool want_phases = phase_ms != nullptr;
    if (want_phases != c->profiling) {
        c->profiling = want_phases;
        if (c->graph) {
            cudaGraphExecDestroy(c->graph);
            c->graph = nullptr;
        }
    }
    cudaEvent_t t0, t1;
    CK(cudaEventCreate(&t0));
    CK(cudaEventCreate(&t1));
    CK(cudaEventRecord(t0, c->stream));
    // run_steps ends with a sync after reading the done flag; record t1 first.
    int st = CRUSH_OK;
    {
        long long issued = 0;
        while (issued < n_steps && st == CRUSH_OK) {
            const bool use_graph = c->period > 0 && c->host_step % c->period == 0 && n_steps - issued >= c->period;
            const long long chunk = use_graph ? c->period : 1;
            // enqueue without the trailing sync of run_steps
            if (use_graph) {
                if (!c->graph) {
                    int64_t before = c->launches;
                    st = build_graph(c);
                    if (st != CRUSH_OK) break;
                    c->graph_launches = c->launches - before;
                    c->launches = before;
                }
                cudaError_t e = cudaGraphLaunch(c->graph, c->stream);
                if (e != cudaSuccess) { st = crush::fail(CRUSH_ERR_CUDA, cudaGetErrorString(e)); break; }
                c->launches += c->graph_launches;
                c->host_step += c->period;
                c->last_was_graph = true;
            } else {
                if (c->profiling) {
                    st = ensure_prof_events(c);
                    if (st != CRUSH_OK) break;
                }
                st = enqueue_step(c, c->host_step, c->profiling ? &c->prof_ev[0] : nullptr);
                c->host_step += 1;
                c->last_was_graph = false;
            }
            issued += chunk;
        }
    }
    CK(cudaEventRecord(t1, c->stream));
    int d = 0;
    CK(cudaMemcpyAsync(&d, &c->ctl->done, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    float elapsed = 0.f;
    CK(cudaEventElapsedTime(&elapsed, t0, t1));
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
    int st = crush_run_begin(c);
    if (st != CRUSH_OK) return st;
    int done = 0;
    const long long chunk = c->period > 0 ? 10 * (long long)c->period : 200;
    long long total = 0;
    // A run that has not finished after this many steps is returned as a timeout.
    const long long cap = c->settings.max_steps > 0 ? (long long)c->settings.max_steps + chunk : 2000000ll;
    while (!done && total < cap) {
        st = run_steps(c, chunk, &done);
        if (st != CRUSH_OK) return st;
        total += chunk;
    }
    st = results(c, r);
    if (st != CRUSH_OK) return st;
    if (!done && r->status == CRUSH_OK) {
        r->status = CRUSH_ERR_TIMEOUT;
        return crush::fail(CRUSH_ERR_TIMEOUT, "run did not finish within " + std::to_string(cap) + " steps");
    }
    return r->status;
}

}  // extern "C"
