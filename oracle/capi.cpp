// capi.cpp — TEST INFRASTRUCTURE ONLY (see oracle.hpp).
// extern "C" entry points of the oracle, loaded by the tests and by the CPU
// baseline leg of bench.py through ctypes.
#include <algorithm>
#include "oracle.hpp"
#include <cstring>
#include <memory>
#include <string>
#include <thread>

using namespace oracle;

namespace {
thread_local std::string g_err;
int fail(const std::string& e) { g_err = e; return CRUSH_ERR_INVALID; }

struct Session {
    Model model;
    Elements el;
    std::vector<ContactRuntime> contacts;
};
}  // namespace

extern "C" {

const char* oracle_last_error(void) { return g_err.c_str(); }

int oracle_hardware_threads(void) { return (int)std::thread::hardware_concurrency(); }

int oracle_geometry(const double* x24, double youngs, double poisson, double density, double hourglass,
                    double* grad24, double* volume, double* lumped8, double* gamma32, double* h144) {
    double x[8][3];
    for (int i = 0; i < 8; ++i)
        for (int d = 0; d < 3; ++d) x[i][d] = x24[3 * i + d];
    HexGeometry g;
    if (!hex_geometry(x, youngs, poisson, density, hourglass, &g)) return fail("degenerate hexahedron");
    for (int i = 0; i < 8; ++i) {
        for (int d = 0; d < 3; ++d) grad24[3 * i + d] = g.center_grad[i][d];
        lumped8[i] = g.lumped_mass[i];
        for (int a = 0; a < 4; ++a) gamma32[4 * i + a] = g.gamma[i][a];
    }
    *volume = g.volume;
    for (int r = 0; r < 12; ++r)
        for (int c = 0; c < 12; ++c) h144[12 * r + c] = g.h[r][c];
    return 0;
}

int oracle_char_length(const double* p24, double* l, double* vol) {
    double p[8][3];
    for (int i = 0; i < 8; ++i)
        for (int d = 0; d < 3; ++d) p[i][d] = p24[3 * i + d];
    characteristic_length_and_volume(p, l, vol);
    return 0;
}

// state25: f_prev_inv 9, rotation 9, stress 6, compaction (all row-major).
int oracle_honeycomb_update(const crush_material* mat, const double* f9, const double* state25, double* tau9, double* out25) {
    HoneycombParams p;
    std::string e = honeycomb_params(*mat, &p);
    if (!e.empty()) return fail(e);
    RateState s;
    for (int k = 0; k < 9; ++k) { s.f_prev_inv.m[k] = state25[k]; s.rotation.m[k] = state25[9 + k]; }
    for (int k = 0; k < 6; ++k) s.stress[k] = state25[18 + k];
    s.compaction = state25[24];
    M3 f, tau;
    for (int k = 0; k < 9; ++k) f.m[k] = f9[k];
    RateState ns;
    honeycomb_rate_update(p, f, s, &tau, &ns);
    for (int k = 0; k < 9; ++k) { tau9[k] = tau.m[k]; out25[k] = ns.f_prev_inv.m[k]; out25[9 + k] = ns.rotation.m[k]; }
    for (int k = 0; k < 6; ++k) out25[18 + k] = ns.stress[k];
    out25[24] = ns.compaction;
    return 0;
}

// knots (8x3) of HoneycombParams and both yield_at forms.
int oracle_honeycomb_params(const crush_material* mat, double* knots24) {
    HoneycombParams p;
    std::string e = honeycomb_params(*mat, &p);
    if (!e.empty()) return fail(e);
    for (int i = 0; i < MAX_KNOTS; ++i)
        for (int j = 0; j < 3; ++j) knots24[3 * i + j] = p.knots[i][j];
    return 0;
}
int oracle_yield_at(const crush_material* mat, double c, double* sy, double* h, double* sy_curve, double* h_curve) {
    HoneycombParams p;
    std::string e = honeycomb_params(*mat, &p);
    if (!e.empty()) return fail(e);
    p.yield_at(c, sy, h);
    plasticity_yield_at(*mat, c, sy_curve, h_curve);
    return 0;
}

// ---- element sessions: the drop-in calls on a whole model ----
void* oracle_session_new(const crush_model_desc* d, int simd, int threads) {
    auto s = std::make_unique<Session>();
    std::string e = model_from_desc(d, &s->model);
    if (e.empty()) e = elements_build(s->model, simd != 0, threads, &s->el);
    if (!e.empty()) { g_err = e; return nullptr; }
    for (const Contact& c : s->model.contacts) s->contacts.push_back(contact_new(c, s->model.positions.data()));
    return s.release();
}
void oracle_session_free(void* h) { delete static_cast<Session*>(h); }

int oracle_session_forces(void* h, const double* u, double* global, int64_t* newly) {
    Session* s = static_cast<Session*>(h);
    size_t k = compute_forces(s->el, u, global);
    if (newly) *newly = (int64_t)k;
    return 0;
}
int oracle_session_stable_dt(void* h, const double* u, double* dt) {
    Session* s = static_cast<Session*>(h);
    return stable_time_step(s->el, u, dt) ? 0 : CRUSH_NONE;
}
int oracle_session_element_dts(void* h, const double* u, double* out) {
    Session* s = static_cast<Session*>(h);
    std::vector<double> t;
    element_time_steps(s->el, u, &t);
    std::memcpy(out, t.data(), t.size() * sizeof(double));
    return 0;
}
int oracle_session_mass_scaling(void* h, const double* u, double dt_min, const double* element_mass, double* added, double* total) {
    Session* s = static_cast<Session*>(h);
    std::vector<double> em;
    if (!element_mass) {
        em.resize(s->model.hexes.size());
        for (size_t e = 0; e < em.size(); ++e) em[e] = s->el.volume[e] * s->model.materials[s->model.hex_part[e]].density;
        element_mass = em.data();
    }
    *total = mass_scaling(s->el, u, dt_min, element_mass, added);
    return 0;
}
int oracle_session_masses(void* h, double* lumped, double* element_mass) {
    Session* s = static_cast<Session*>(h);
    if (lumped) {
        std::vector<double> m = lumped_masses(s->el, s->model.n_nodes());
        std::memcpy(lumped, m.data(), m.size() * sizeof(double));
    }
    if (element_mass)
        for (size_t e = 0; e < s->model.hexes.size(); ++e) element_mass[e] = s->el.volume[e] * s->model.materials[s->model.hex_part[e]].density;
    return 0;
}
// f64 geometry: grad (24), volume, gamma (32, [i][a]), h (144, row-major).
int oracle_session_geometry(void* h, double* grad, double* volume, double* gamma, double* hh) {
    Session* s = static_cast<Session*>(h);
    for (size_t e = 0; e < s->model.hexes.size(); ++e) {
        if (grad) std::memcpy(grad + 24 * e, s->el.center_grad[e].data(), 24 * sizeof(double));
        if (volume) volume[e] = s->el.volume[e];
        if (gamma) std::memcpy(gamma + 32 * e, s->el.gamma[e].data(), 32 * sizeof(double));
        if (hh) std::memcpy(hh + 144 * e, s->el.h[e].data(), 144 * sizeof(double));
    }
    return 0;
}
// Replace the f32 lane geometry by externally supplied f32 data (grad 24,
// volume, gamma 32 [i][a], h 144 column-major), for identical-state checks.
int oracle_session_set_lane_geometry(void* h, const float* grad, const float* volume, const float* gamma, const float* hh) {
    Session* s = static_cast<Session*>(h);
    size_t k = 0;
    for (Block& b : s->el.blocks)
        for (int l = 0; l < b.count; ++l) {
            size_t e = s->el.simd_ids[k++];
            for (int j = 0; j < 24; ++j) b.grad[j][l] = grad[24 * e + j];
            b.volume[l] = volume[e];
            for (int j = 0; j < 32; ++j) b.gamma[j][l] = gamma[32 * e + j];
            for (int j = 0; j < 144; ++j) b.h[j][l] = hh[144 * e + j];
        }
    return 0;
}
// Lane state per element: 25 f32 (f_prev_inv 9, rotation 9, stress 6, compaction) + eroded.
int oracle_session_get_state(void* h, float* state, uint8_t* eroded) {
    Session* s = static_cast<Session*>(h);
    if (s->el.blocks.empty()) {
        for (size_t e = 0; e < s->model.hexes.size(); ++e) {
            const RateState& r = s->el.state[e];
            for (int j = 0; j < 9; ++j) { state[25 * e + j] = (float)r.f_prev_inv.m[j]; state[25 * e + 9 + j] = (float)r.rotation.m[j]; }
            for (int j = 0; j < 6; ++j) state[25 * e + 18 + j] = (float)r.stress[j];
            state[25 * e + 24] = (float)r.compaction;
            eroded[e] = s->el.eroded[e];
        }
        return 0;
    }
    size_t k = 0;
    for (Block& b : s->el.blocks)
        for (int l = 0; l < b.count; ++l) {
            size_t e = s->el.simd_ids[k++];
            for (int j = 0; j < 9; ++j) { state[25 * e + j] = b.f_prev_inv[j][l]; state[25 * e + 9 + j] = b.rotation[j][l]; }
            for (int j = 0; j < 6; ++j) state[25 * e + 18 + j] = b.stress[j][l];
            state[25 * e + 24] = b.compaction[l];
            eroded[e] = b.eroded[l];
        }
    return 0;
}
int oracle_session_set_state(void* h, const float* state, const uint8_t* eroded) {
    Session* s = static_cast<Session*>(h);
    size_t k = 0;
    for (Block& b : s->el.blocks)
        for (int l = 0; l < b.count; ++l) {
            size_t e = s->el.simd_ids[k++];
            for (int j = 0; j < 9; ++j) { b.f_prev_inv[j][l] = state[25 * e + j]; b.rotation[j][l] = state[25 * e + 9 + j]; }
            for (int j = 0; j < 6; ++j) b.stress[j][l] = state[25 * e + 18 + j];
            b.compaction[l] = state[25 * e + 24];
            b.eroded[l] = eroded[e] != 0;
            s->el.eroded[e] = eroded[e];
        }
    return 0;
}
int oracle_session_contact_apply(void* h, int c, const double* u, const double* v, const double* masses, double dt,
                                 double* force, int64_t* count, double* max_pen) {
    Session* s = static_cast<Session*>(h);
    if (c < 0 || c >= (int)s->contacts.size()) return fail("contact id out of range");
    contact_apply(s->contacts[c], s->model.positions.data(), u, v, masses, dt, force);
    if (count) *count = (int64_t)s->contacts[c].penetration_count;
    if (max_pen) *max_pen = s->contacts[c].max_penetration;
    return 0;
}
int oracle_session_contact_nodes(void* h, int c, uint32_t* nodes, int64_t* n) {
    Session* s = static_cast<Session*>(h);
    if (c < 0 || c >= (int)s->contacts.size()) return fail("contact id out of range");
    *n = (int64_t)s->contacts[c].nodes.size();
    if (nodes) std::memcpy(nodes, s->contacts[c].nodes.data(), s->contacts[c].nodes.size() * sizeof(uint32_t));
    return 0;
}

// Whole run (solver.rs:190). u_out / v_out (3N) and dt_log (cap entries) may be NULL.
int oracle_run(const crush_model_desc* d, int simd, int threads, crush_results* out, double* u_out, double* v_out,
               double* dt_log, int64_t dt_log_cap, double* seconds3) {
    Model m;
    std::string e = model_from_desc(d, &m);
    if (!e.empty()) return fail(e);
    RunOptions opt;
    opt.simd = simd != 0;
    opt.threads = threads;
    opt.log_steps = dt_log != nullptr;
    RunResults r;
    e = run(m, opt, &r);
    if (!e.empty()) return fail(e);
    std::memset(out, 0, sizeof(*out));
    out->time = r.time;
    out->steps = r.steps;
    out->eroded_elements = r.eroded;
    out->dt_min = r.dt_min;
    out->added_mass_max = r.added_mass_max;
    out->status = r.status;
    out->n_vehicles = (int)m.vehicles.size();
    for (int vi = 0; vi < (int)m.vehicles.size() && vi < 4; ++vi) vehicle_result(m, r, vi, &out->vehicle[vi]);
    if (u_out) std::memcpy(u_out, r.u.data(), r.u.size() * sizeof(double));
    if (v_out) std::memcpy(v_out, r.v.data(), r.v.size() * sizeof(double));
    if (dt_log)
        for (int64_t k = 0; k < dt_log_cap && k < (int64_t)r.dt_log.size(); ++k) dt_log[k] = r.dt_log[k];
    if (seconds3) {  // wall, forces, contact, step loop
        seconds3[0] = r.wall_seconds;
        seconds3[1] = r.force_seconds;
        seconds3[2] = r.contact_seconds;
        seconds3[3] = r.loop_seconds;
    }
    return r.status;
}

// Whole run (src/solver.rs:190-381) with the loop time of the steps from
// `time_from_step` to the end in seconds5[4] (seconds5: wall, forces,
// contact, step loop, window) and the end state: u, v (3N each) and the
// per-element erosion flags (E), each optional.
int oracle_run_window(const crush_model_desc* d, int simd, int threads, int64_t time_from_step, crush_results* out, double* u_out,
                      double* v_out, uint8_t* eroded_out, double* seconds5) {
    Model m;
    std::string e = model_from_desc(d, &m);
    if (!e.empty()) return fail(e);
    RunOptions opt;
    opt.simd = simd != 0;
    opt.threads = threads;
    opt.time_from_step = time_from_step;
    RunResults r;
    e = run(m, opt, &r);
    if (!e.empty()) return fail(e);
    std::memset(out, 0, sizeof(*out));
    out->time = r.time;
    out->steps = r.steps;
    out->eroded_elements = r.eroded;
    out->dt_min = r.dt_min;
    out->added_mass_max = r.added_mass_max;
    out->status = r.status;
    out->n_vehicles = (int)m.vehicles.size();
    for (int vi = 0; vi < (int)m.vehicles.size() && vi < 4; ++vi) vehicle_result(m, r, vi, &out->vehicle[vi]);
    if (u_out) std::memcpy(u_out, r.u.data(), r.u.size() * sizeof(double));
    if (v_out) std::memcpy(v_out, r.v.data(), r.v.size() * sizeof(double));
    if (eroded_out) std::memcpy(eroded_out, r.eroded_flags.data(), r.eroded_flags.size());
    if (seconds5) {
        seconds5[0] = r.wall_seconds;
        seconds5[1] = r.force_seconds;
        seconds5[2] = r.contact_seconds;
        seconds5[3] = r.loop_seconds;
        seconds5[4] = r.window_seconds;
    }
    return r.status;
}

// Whole run with time histories (solver.rs:114-187, :283-286, :349-358):
// the records' times and steps (cap_records each), parts (cap x n_parts x 11)
// and accelerometer node values (cap x n_acc_nodes x 21); *n_records = taken.
int oracle_run_history(const crush_model_desc* d, int simd, int threads, int history_steps, int n_acc, const crush_accelerometer* acc,
                       int64_t cap_records, double* time, int64_t* step, double* parts, double* nodes, int64_t* n_records,
                       crush_results* out) {
    Model m;
    std::string e = model_from_desc(d, &m);
    if (!e.empty()) return fail(e);
    RunOptions opt;
    opt.simd = simd != 0;
    opt.threads = threads;
    opt.history_steps = history_steps;
    for (int k = 0; k < n_acc; ++k) {
        HistoryAccel a;
        a.nodes.assign(acc[k].nodes, acc[k].nodes + acc[k].n_nodes);
        a.has_frame = acc[k].has_frame != 0;
        a.origin = acc[k].origin;
        a.x_axis = acc[k].x_axis;
        a.plane = acc[k].plane;
        opt.accelerometers.push_back(a);
    }
    RunResults r;
    e = run(m, opt, &r);
    if (!e.empty()) return fail(e);
    const int64_t nr = (int64_t)r.hist_time.size();
    *n_records = nr;
    const size_t per_p = r.hist_parts.size() / std::max<int64_t>(nr, 1), per_n = r.hist_nodes.size() / std::max<int64_t>(nr, 1);
    for (int64_t k = 0; k < nr && k < cap_records; ++k) {
        time[k] = r.hist_time[k];
        step[k] = r.hist_step[k];
        std::memcpy(parts + k * per_p, r.hist_parts.data() + k * per_p, per_p * sizeof(double));
        std::memcpy(nodes + k * per_n, r.hist_nodes.data() + k * per_n, per_n * sizeof(double));
    }
    if (out) {
        std::memset(out, 0, sizeof(*out));
        out->time = r.time;
        out->steps = r.steps;
        out->status = r.status;
    }
    return r.status;
}

// Whole run with frames every frame_steps (src/solver.rs:265-281): frame k's
// time, step, displacement (3N), plastic strain (E), stress (6E), eroded (E)
// into cap-frame arrays; returns the frames taken in *n_frames.
int oracle_run_frames(const crush_model_desc* d, int simd, int threads, int frame_steps, int64_t cap, double* time, int64_t* step,
                      float* disp, float* pstrain, float* stress, uint8_t* eroded, int64_t* n_frames) {
    Model m;
    std::string e = model_from_desc(d, &m);
    if (!e.empty()) return fail(e);
    RunOptions opt;
    opt.simd = simd != 0;
    opt.threads = threads;
    opt.frame_steps = frame_steps;
    RunResults r;
    e = run(m, opt, &r);
    if (!e.empty()) return fail(e);
    const int64_t nf = (int64_t)r.frame_time.size();
    *n_frames = nf;
    const size_t n3 = 3 * m.n_nodes(), ne = m.hexes.size();
    for (int64_t k = 0; k < nf && k < cap; ++k) {
        time[k] = r.frame_time[k];
        step[k] = r.frame_step[k];
        std::memcpy(disp + k * n3, r.frame_disp.data() + k * n3, n3 * sizeof(float));
        std::memcpy(pstrain + k * ne, r.frame_pstrain.data() + k * ne, ne * sizeof(float));
        std::memcpy(stress + 6 * k * ne, r.frame_stress.data() + 6 * k * ne, 6 * ne * sizeof(float));
        std::memcpy(eroded + k * ne, r.frame_eroded.data() + k * ne, ne);
    }
    return r.status;
}

// src/signal.rs:9-40 and :42-66.
int oracle_cfc_filter(const double* x, int64_t n, double dt, double cfc, double* y) {
    std::vector<double> in(x, x + n), outv = cfc_filter(in, dt, cfc);
    std::memcpy(y, outv.data(), outv.size() * sizeof(double));
    return 0;
}
int64_t oracle_resample(const double* t, const double* y, int64_t n, double t0, double dt, double t_end, double* tu, double* yu,
                        int64_t cap) {
    std::vector<double> tv(t, t + n), yv(y, y + n), a, b;
    resample(tv, yv, t0, dt, t_end, &a, &b);
    for (size_t k = 0; k < a.size() && (int64_t)k < cap; ++k) {
        tu[k] = a[k];
        yu[k] = b[k];
    }
    return (int64_t)a.size();
}

// symmetric_eigen3 (material.rs:570) on a row-major 3x3; eigenvectors as
// the columns of the row-major evec.
int oracle_symmetric_eigen3(const double* a, double* eval, double* evec) {
    M3 m, v;
    for (int k = 0; k < 9; ++k) m.m[k] = a[k];
    symmetric_eigen3(m, eval, &v);
    for (int k = 0; k < 9; ++k) evec[k] = v.m[k];
    return 0;
}
// Hencky elastic Kirchhoff stress (material.rs:708-771), row-major F and tau.
int oracle_hencky_elastic(double youngs, double poisson, const double* f, double* tau) {
    M3 m, t;
    for (int k = 0; k < 9; ++k) m.m[k] = f[k];
    hencky_elastic(youngs, poisson, m, &t);
    for (int k = 0; k < 9; ++k) tau[k] = t.m[k];
    return 0;
}

}  // extern "C"
