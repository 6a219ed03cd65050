// solver.cpp — TEST INFRASTRUCTURE ONLY (see oracle.hpp).
// Restates crushrs::run (src/solver.rs:190-381) without frames,
// plus the delta-v / crush outputs of src/bin/crushrs.rs:237-271 and the
// separation stop rule of include/crush.h (CRUSH_STOP_SEPARATION), which the
// reference does not have.
#include "oracle.hpp"
#include <chrono>
#include <cmath>
#include <limits>
#include <set>

namespace oracle {

static const double INF = std::numeric_limits<double>::infinity();

static double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static double min_edge_length(const Model& m) {
    static const int EDGES[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6}, {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
    double mn = INF;
    for (const auto& h : m.hexes)
        for (const auto& e : EDGES) {
            const double* p = &m.positions[3 * h[e[0]]];
            const double* q = &m.positions[3 * h[e[1]]];
            double d = std::sqrt((p[0] - q[0]) * (p[0] - q[0]) + (p[1] - q[1]) * (p[1] - q[1]) + (p[2] - q[2]) * (p[2] - q[2]));
            mn = std::fmin(mn, d);
        }
    return mn;
}

// Model::mean_velocity, model.rs:281 (x component only is needed by the stop rule).
static double mean_vx(const std::vector<double>& masses, const double* v, const std::vector<uint32_t>& nodes) {
    double m = 0.0, p = 0.0;
    for (uint32_t n : nodes) { m += masses[n]; p += masses[n] * v[3 * n]; }
    return m > 0.0 ? p / m : 0.0;
}

// LocalFrame::axes, src/model.rs:45-61 (nalgebra's norm, normalize and
// cross written out: sqrt of the ordered sum of squares, division by it).
static void frame_axes(const double o[3], const double xa[3], const double pl[3], double ax[3][3]) {
    auto norm = [](const double* a) { return std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); };
    auto cross = [](const double* a, const double* b, double* c) {
        c[0] = a[1] * b[2] - a[2] * b[1];
        c[1] = a[2] * b[0] - a[0] * b[2];
        c[2] = a[0] * b[1] - a[1] * b[0];
    };
    double e1[3], p[3], c[3], e2[3], e3[3];
    for (int d = 0; d < 3; ++d) {
        e1[d] = xa[d] - o[d];
        p[d] = pl[d] - o[d];
    }
    if (norm(e1) < 1e-300) { e1[0] = 1.0; e1[1] = 0.0; e1[2] = 0.0; }
    const double n1 = norm(e1);
    for (double& x : e1) x /= n1;
    cross(p, e1, c);
    if (norm(c) < 1e-12 * std::fmax(norm(p), 1e-300)) {
        const bool ux = std::fabs(e1[0]) < 0.9;
        p[0] = ux ? 1.0 : 0.0; p[1] = ux ? 0.0 : 1.0; p[2] = 0.0;
    }
    cross(e1, p, e3);
    const double n3 = norm(e3);
    for (double& x : e3) x /= n3;
    cross(e3, e1, e2);
    for (int d = 0; d < 3; ++d) { ax[0][d] = e1[d]; ax[1][d] = e2[d]; ax[2][d] = e3[d]; }
}

std::string run(const Model& model, const RunOptions& opt, RunResults* res) {
    double wall0 = now_s();
    const crush_settings& s = model.settings;
    size_t n_nodes = model.n_nodes();
    size_t n = 3 * n_nodes;
    Elements elements;
    std::string err = elements_build(model, opt.simd, opt.threads, &elements);
    if (!err.empty()) return err;
    std::vector<double> masses = lumped_masses(elements, n_nodes);
    std::vector<double> element_mass(model.hexes.size());
    for (size_t e = 0; e < model.hexes.size(); ++e) element_mass[e] = elements.volume[e] * model.materials[model.hex_part[e]].density;
    std::vector<double> added_mass(n_nodes, 0.0), inv_mass(n, 0.0);
    auto set_inv_mass = [&]() {
        for (size_t i = 0; i < n_nodes; ++i) {
            double m = masses[i] + added_mass[i];
            for (int d = 0; d < 3; ++d) inv_mass[3 * i + d] = m > 0.0 ? 1.0 / m : 0.0;
        }
    };
    set_inv_mass();
    std::vector<ContactRuntime> contacts;
    for (const Contact& c : model.contacts) contacts.push_back(contact_new(c, model.positions.data()));
    std::vector<size_t> fixed;
    for (uint32_t nd : model.fixed_nodes) for (int d = 0; d < 3; ++d) fixed.push_back(3 * (size_t)nd + d);

    std::vector<double> u(n, 0.0);
    double contact_dt = INF;
    for (const Contact& c : model.contacts)
        for (uint32_t nd : c.nodes)
            if (masses[nd] > 0.0 && c.stiffness > 0.0) contact_dt = std::fmin(contact_dt, 2.0 * std::sqrt(masses[nd] / c.stiffness));
    double stable;
    if (!stable_time_step(elements, u.data(), &stable)) {
        double cmax = 0.0;
        for (int32_t p : model.hex_part) cmax = std::fmax(cmax, dilatational_wave_speed(model.materials[p]));
        stable = min_edge_length(model) / (std::sqrt(3.0) * cmax);
    }
    stable = std::fmin(stable, contact_dt);
    double dt_floor = s.mass_scaling > 0.0 ? s.mass_scaling * stable : 0.0;
    double added_mass_total = 0.0;
    double dt = s.time_step > 0.0 ? s.time_step : stable * s.dt_scale;
    bool adaptive = !(s.time_step > 0.0) && s.adaptive_check_steps > 0;

    std::vector<double> v = model.initial_velocity;
    std::vector<double> v_half(n, 0.0), f_int(n, 0.0), f_ext(n, 0.0), acc(n, 0.0);
    double tf = now_s();
    compute_forces(elements, u.data(), f_int.data());
    res->force_seconds = now_s() - tf;
    for (ContactRuntime& c : contacts) contact_apply(c, model.positions.data(), u.data(), v.data(), masses.data(), dt, f_ext.data());
    for (size_t k = 0; k < n; ++k) acc[k] = (f_ext[k] - f_int[k]) * inv_mass[k];

    // Time histories: part_states and sample_accelerometers, src/solver.rs:114-187.
    std::vector<std::vector<uint32_t>> part_nodes(model.materials.size());  // Mesh::part_nodes, src/mesh.rs:74-82
    for (size_t p = 0; p < part_nodes.size(); ++p) {
        std::set<uint32_t> set;
        for (size_t e = 0; e < model.hexes.size(); ++e)
            if (model.hex_part[e] == (int32_t)p) set.insert(model.hexes[e].begin(), model.hexes[e].end());
        part_nodes[p].assign(set.begin(), set.end());
    }
    res->hist_time.clear();
    res->hist_step.clear();
    res->hist_parts.clear();
    res->hist_nodes.clear();
    auto record = [&](double tr, int64_t sr) {
        res->hist_time.push_back(tr);
        res->hist_step.push_back(sr);
        for (const auto& nodes : part_nodes) {
            double m = 0.0, mv[3] = {0, 0, 0}, mu[3] = {0, 0, 0}, ma[3] = {0, 0, 0}, ke = 0.0;
            for (uint32_t nd : nodes) {
                m += masses[nd];
                for (int d = 0; d < 3; ++d) {
                    mv[d] += masses[nd] * v[3 * nd + d];
                    mu[d] += masses[nd] * u[3 * nd + d];
                    ma[d] += masses[nd] * acc[3 * nd + d];
                    ke += 0.5 * masses[nd] * v[3 * nd + d] * v[3 * nd + d];
                }
            }
            const double inv = m > 0.0 ? 1.0 / m : 0.0;
            res->hist_parts.push_back(m);
            for (int d = 0; d < 3; ++d) res->hist_parts.push_back(mv[d] * inv);
            for (int d = 0; d < 3; ++d) res->hist_parts.push_back(mu[d] * inv);
            for (int d = 0; d < 3; ++d) res->hist_parts.push_back(ma[d] * inv);
            res->hist_parts.push_back(ke);
        }
        auto x = [&](uint32_t nd, int d) { return model.positions[3 * nd + d] + u[3 * nd + d]; };
        for (const HistoryAccel& a : opt.accelerometers) {
            double ax[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
            if (a.has_frame) {
                double o[3], xa[3], pl[3];
                for (int d = 0; d < 3; ++d) { o[d] = x(a.origin, d); xa[d] = x(a.x_axis, d); pl[d] = x(a.plane, d); }
                frame_axes(o, xa, pl, ax);
            }
            for (uint32_t nd : a.nodes) {
                double un[3], vn[3], an[3];
                for (int d = 0; d < 3; ++d) { un[d] = u[3 * nd + d]; vn[d] = v[3 * nd + d]; an[d] = acc[3 * nd + d]; }
                for (int d = 0; d < 3; ++d) res->hist_nodes.push_back(x(nd, d));
                for (const double* w : {un, vn, an})
                    for (int d = 0; d < 3; ++d) res->hist_nodes.push_back(w[d]);
                for (const double* w : {un, vn, an})
                    for (int i = 0; i < 3; ++i)  // rotate, src/solver.rs:143-145
                        res->hist_nodes.push_back(a.has_frame ? ax[i][0] * w[0] + ax[i][1] * w[1] + ax[i][2] * w[2] : w[i]);
            }
        }
    };
    if (opt.history_steps > 0) record(0.0, 0);

    // Frames: the capture closure of crushrs::run (src/solver.rs:265-275)
    // with plastic_strain and cauchy_stress (src/kernel.rs:269-321). Elastic
    // elements have no plastic strain; their Cauchy stress is the Hencky
    // tau / J at the current u (zero when inverted).
    res->frame_time.clear();
    res->frame_step.clear();
    res->frame_disp.clear();
    res->frame_pstrain.clear();
    res->frame_stress.clear();
    res->frame_eroded.clear();
    auto capture = [&](double tr, int64_t sr) {
        sync_states(elements);
        res->frame_time.push_back(tr);
        res->frame_step.push_back(sr);
        for (double x : u) res->frame_disp.push_back((float)x);
        for (size_t e = 0; e < model.hexes.size(); ++e) {
            const bool honey = elements.honeycomb[e] != 0;
            const RateState& st = elements.state[e];
            res->frame_pstrain.push_back(honey ? (float)st.compaction : 0.0f);
            res->frame_eroded.push_back(elements.eroded[e] ? 1 : 0);
            double c6[6] = {0, 0, 0, 0, 0, 0};
            if (honey && !elements.eroded[e]) {
                const double* s6 = st.stress;
                M3 sh;
                sh(0, 0) = s6[0]; sh(0, 1) = s6[3]; sh(0, 2) = s6[5];
                sh(1, 0) = s6[3]; sh(1, 1) = s6[1]; sh(1, 2) = s6[4];
                sh(2, 0) = s6[5]; sh(2, 1) = s6[4]; sh(2, 2) = s6[2];
                const M3 c = m3_mul(m3_mul(st.rotation, sh), m3_transpose(st.rotation));
                c6[0] = c(0, 0); c6[1] = c(1, 1); c6[2] = c(2, 2); c6[3] = c(0, 1); c6[4] = c(1, 2); c6[5] = c(0, 2);
            } else if (!honey && !elements.eroded[e]) {
                const double* grad = elements.center_grad[e].data();
                M3 f = m3_zero();
                for (int i = 0; i < 8; ++i) {
                    const size_t nd = elements.conn[e][i];
                    for (int a = 0; a < 3; ++a) {
                        const double xa = model.positions[3 * nd + a] + u[3 * nd + a];
                        for (int b = 0; b < 3; ++b) f(a, b) += xa * grad[3 * i + b];
                    }
                }
                const double j = m3_det(f);
                if (j > 0.0) {
                    const crush_material& mat = model.materials[model.hex_part[e]];
                    M3 tau;
                    hencky_elastic(mat.youngs_modulus, mat.poisson_ratio, f, &tau);
                    c6[0] = tau(0, 0) / j; c6[1] = tau(1, 1) / j; c6[2] = tau(2, 2) / j;
                    c6[3] = tau(0, 1) / j; c6[4] = tau(1, 2) / j; c6[5] = tau(0, 2) / j;
                }
            }
            for (double x : c6) res->frame_stress.push_back((float)x);
        }
    };
    if (opt.frame_steps > 0) capture(0.0, 0);

    // Separation rule bookkeeping: contacts whose faces are not all fixed.
    std::set<uint32_t> fixed_set(model.fixed_nodes.begin(), model.fixed_nodes.end());
    std::vector<char> counts(contacts.size(), 0);
    for (size_t c = 0; c < contacts.size(); ++c)
        for (const auto& f : model.contacts[c].faces)
            for (uint32_t nd : f) if (!fixed_set.count(nd)) counts[c] = 1;
    int64_t last_hit = -1;

    double loop0 = now_s();
    double t = 0.0;
    int64_t step = 0;
    int64_t eroded_total = 0;
    double dt_cfl = dt, dt_min = INF;
    res->status = 0;
    res->dt_log.clear();
    double win0 = -1.0;
    while (t < s.end_time) {
        if (step == opt.time_from_step) win0 = now_s();
        if (adaptive && step % s.adaptive_check_steps == 0) {
            double dt_stable;
            if (stable_time_step(elements, u.data(), &dt_stable)) {
                double dt_use = dt_stable;
                if (dt_floor > 0.0 && dt_stable < dt_floor) {
                    double total = mass_scaling(elements, u.data(), dt_floor, element_mass.data(), added_mass.data());
                    set_inv_mass();
                    added_mass_total = std::fmax(added_mass_total, total);
                    dt_use = dt_floor;
                }
                dt_cfl = s.dt_scale * std::fmin(dt_use, contact_dt);
            }
        }
        dt = std::fmax(std::fmin(dt_cfl, s.end_time - t), 1e-15);
        if (step % 20 == 0) {
            bool bad = false;
            for (double x : u) if (!std::isfinite(x)) { bad = true; break; }
            if (bad) { res->status = CRUSH_ERR_NONFINITE; break; }
        }
        double tc = now_s();
        std::fill(f_ext.begin(), f_ext.end(), 0.0);
        bool hit = false;
        for (size_t c = 0; c < contacts.size(); ++c) {
            contact_apply(contacts[c], model.positions.data(), u.data(), v.data(), masses.data(), dt, f_ext.data());
            if (counts[c] && contacts[c].penetration_count > 0) hit = true;
        }
        if (hit) last_hit = step;
        res->contact_seconds += now_s() - tc;
        for (size_t k = 0; k < n; ++k) {
            double a = (f_ext[k] - f_int[k]) * inv_mass[k];
            v_half[k] = v[k] + 0.5 * dt * a;
            u[k] += dt * v_half[k];
        }
        for (size_t k : fixed) { u[k] = 0.0; v[k] = 0.0; v_half[k] = 0.0; }
        tf = now_s();
        std::fill(f_int.begin(), f_int.end(), 0.0);
        eroded_total += (int64_t)compute_forces(elements, u.data(), f_int.data());
        res->force_seconds += now_s() - tf;
        for (size_t k = 0; k < n; ++k) {
            double a = (f_ext[k] - f_int[k]) * inv_mass[k];
            v[k] = (v_half[k] + 0.5 * dt * a) * s.velocity_damping;
            acc[k] = a;
        }
        for (size_t k : fixed) { v[k] = 0.0; acc[k] = 0.0; }
        step += 1;
        t += dt;
        dt_min = std::fmin(dt_min, dt);
        if (opt.log_steps) res->dt_log.push_back(dt);
        if (opt.frame_steps > 0 && step % opt.frame_steps == 0) capture(t, step);
        if (opt.history_steps > 0 && step % opt.history_steps == 0) record(t, step);
        if (s.max_steps > 0 && step >= s.max_steps) break;
        if (s.stop_rule == CRUSH_STOP_SEPARATION && step % 10 == 0 && last_hit >= 0 && step - 1 - last_hit >= 100 &&
            model.vehicles.size() >= 2) {
            double va = mean_vx(masses, v.data(), model.vehicles[0].nodes);
            double vb = mean_vx(masses, v.data(), model.vehicles[1].nodes);
            if (vb - va >= 0.0) break;
        }
    }
    if (opt.frame_steps > 0 && step % opt.frame_steps != 0) capture(t, step);
    if (opt.history_steps > 0 && step % opt.history_steps != 0) record(t, step);
    res->time = t;
    res->steps = step;
    res->eroded = eroded_total;
    res->dt_min = dt_min;
    res->added_mass_max = added_mass_total;
    res->u = u;
    res->v = v;
    res->masses = masses;
    res->loop_seconds = now_s() - loop0;
    res->window_seconds = win0 >= 0.0 ? now_s() - win0 : 0.0;
    res->eroded_flags.assign(elements.eroded.begin(), elements.eroded.end());
    res->wall_seconds = now_s() - wall0;
    return "";
}

void vehicle_result(const Model& m, const RunResults& r, int vi, crush_vehicle_result* out) {
    const Vehicle& veh = m.vehicles[vi];
    double mass = 0.0, p1[3] = {0, 0, 0}, p0[3] = {0, 0, 0};
    for (uint32_t nd : veh.nodes) {
        mass += r.masses[nd];
        for (int d = 0; d < 3; ++d) {
            p1[d] += r.masses[nd] * r.v[3 * nd + d];
            p0[d] += r.masses[nd] * m.initial_velocity[3 * nd + d];
        }
    }
    out->mass = mass;
    for (int d = 0; d < 3; ++d) {
        double v1 = mass > 0.0 ? p1[d] / mass : 0.0;
        double v0 = mass > 0.0 ? p0[d] / mass : 0.0;
        out->velocity[d] = v1;
        out->delta_v[d] = v1 - v0;
    }
    double fu = 0.0;
    for (uint32_t nd : veh.front) fu += r.u[3 * nd];
    fu = veh.front.empty() ? 0.0 : fu / (double)veh.front.size();
    out->crush = std::fabs(r.u[3 * veh.accel_node] - fu);
}

}  // namespace oracle
