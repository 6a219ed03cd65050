// kernel.cpp — TEST INFRASTRUCTURE ONLY (see oracle.hpp).
// Restates src/kernel.rs (Elements: build, scalar f64 element force,
// compute_forces, stable dt, mass scaling), Blocks::build / scatter of
// src/kernel_simd.rs:534-596 and Model::lumped_masses (src/model.rs:268).
#include "oracle.hpp"
#include <cmath>
#include <cstring>
#include <limits>
#include <set>
#include "pool.hpp"

namespace oracle {

static const double INF = std::numeric_limits<double>::infinity();

std::string model_from_desc(const crush_model_desc* d, Model* m) {
    if (!d || d->n_nodes <= 0 || !d->positions || d->n_hexes < 0 || (d->n_hexes > 0 && (!d->hexes || !d->hex_part)))
        return "invalid model description";
    if (d->n_parts <= 0 || !d->materials) return "model needs at least one material";
    m->positions.assign(d->positions, d->positions + 3 * d->n_nodes);
    m->hexes.resize(d->n_hexes);
    m->hex_part.assign(d->hex_part, d->hex_part + d->n_hexes);
    for (int64_t e = 0; e < d->n_hexes; ++e) {
        for (int i = 0; i < 8; ++i) {
            uint32_t n = d->hexes[8 * e + i];
            if (n >= (uint64_t)d->n_nodes) return "hexahedron node out of range";
            m->hexes[e][i] = n;
        }
        if (d->hex_part[e] < 0 || d->hex_part[e] >= d->n_parts) return "hexahedron part out of range";
    }
    m->materials.assign(d->materials, d->materials + d->n_parts);
    if (d->initial_velocity) m->initial_velocity.assign(d->initial_velocity, d->initial_velocity + 3 * d->n_nodes);
    else m->initial_velocity.assign(3 * d->n_nodes, 0.0);
    m->fixed_nodes.clear();
    for (int64_t i = 0; i < d->n_fixed; ++i) {
        if (d->fixed_nodes[i] >= (uint64_t)d->n_nodes) return "fixed node out of range";
        m->fixed_nodes.push_back(d->fixed_nodes[i]);
    }
    m->contacts.clear();
    for (int c = 0; c < d->n_contacts; ++c) {
        const crush_contact& cd = d->contacts[c];
        Contact k;
        for (int64_t i = 0; i < cd.n_nodes; ++i) {
            if (cd.nodes[i] >= (uint64_t)d->n_nodes) return "contact node out of range";
            k.nodes.push_back(cd.nodes[i]);
            if (cd.node_scale) k.node_scale.push_back(cd.node_scale[i]);
        }
        for (int64_t f = 0; f < cd.n_faces; ++f) {
            std::array<uint32_t, 4> q;
            for (int i = 0; i < 4; ++i) {
                q[i] = cd.faces[4 * f + i];
                if (q[i] >= (uint64_t)d->n_nodes) return "contact face node out of range";
            }
            k.faces.push_back(q);
        }
        k.stiffness = cd.stiffness;
        k.max_distance = cd.max_distance;
        m->contacts.push_back(k);
    }
    m->vehicles.clear();
    for (int v = 0; v < d->n_vehicles; ++v) {
        const crush_vehicle& vd = d->vehicles[v];
        Vehicle w;
        w.nodes.assign(vd.nodes, vd.nodes + vd.n_nodes);
        w.accel_node = vd.accel_node;
        w.front.assign(vd.front_nodes, vd.front_nodes + vd.n_front);
        m->vehicles.push_back(w);
    }
    m->settings = d->settings;
    return "";
}

static void set_lane(Block* b, int l, const Elements& el, size_t e) {
    for (int i = 0; i < 8; ++i) b->conn[l][i] = el.conn[e][i];
    for (int k = 0; k < 24; ++k) b->grad[k][l] = (float)el.center_grad[e][k];
    b->volume[l] = (float)el.volume[e];
    for (int i = 0; i < 8; ++i)
        for (int a = 0; a < 4; ++a) b->gamma[4 * i + a][l] = (float)el.gamma[e][4 * i + a];
    for (int c = 0; c < 12; ++c)
        for (int r = 0; r < 12; ++r) b->h[12 * c + r][l] = (float)el.h[e][12 * r + c];
    const crush_material& mat = el.model->materials[el.part[e]];
    HoneycombParams p;
    honeycomb_params(mat, &p);
    b->youngs[l] = (float)p.youngs_modulus;
    b->trans[l] = (float)p.cap_factor[1];
    b->yield0[l] = (float)p.yield_stress;
    b->hard[l] = (float)p.hardening;
    for (int i = 0; i < MAX_KNOTS; ++i) {
        b->knot_c[i][l] = (float)p.knots[i][0];
        b->knot_s[i][l] = (float)p.knots[i][1];
        b->knot_h[i][l] = (float)p.knots[i][2];
    }
    const RateState& s = el.state[e];
    for (int k = 0; k < 9; ++k) {
        b->f_prev_inv[k][l] = (float)s.f_prev_inv.m[k];
        b->rotation[k][l] = (float)s.rotation.m[k];
    }
    for (int k = 0; k < 6; ++k) b->stress[k][l] = (float)s.stress[k];
    b->compaction[l] = (float)s.compaction;
    b->eroded[l] = el.eroded[e] != 0;
    if (l + 1 > b->count) b->count = l + 1;
}

std::string elements_build(const Model& m, bool simd, int threads, Elements* el) {
    el->model = &m;
    el->simd = simd;
    el->threads = threads < 1 ? 1 : threads;
    size_t ne = m.hexes.size();
    el->conn = m.hexes;
    el->center_grad.resize(ne);
    el->volume.resize(ne);
    el->gamma.resize(ne);
    el->h.resize(ne);
    el->part = m.hex_part;
    el->dt_factor.resize(ne);
    el->state.assign(ne, rate_state_default());
    el->eroded.assign(ne, 0);
    el->honeycomb.resize(ne);
    el->lumped.resize(8 * ne);
    el->simd_ids.clear();
    el->scalar_ids.clear();
    for (const crush_material& mat : m.materials) {
        if (mat.model == CRUSH_MAT_HONEYCOMB) {
            HoneycombParams p;
            std::string err = honeycomb_params(mat, &p);
            if (!err.empty()) return err;
        }
    }
    std::vector<uint8_t> bad(ne, 0);
    parallel_for(el->threads, (long)ne, 64, [&](long el_index) {
        size_t e = (size_t)el_index;
        const crush_material& mat = m.materials[m.hex_part[e]];
        double x[8][3];
        for (int i = 0; i < 8; ++i)
            for (int d = 0; d < 3; ++d) x[i][d] = m.positions[3 * m.hexes[e][i] + d];
        HexGeometry g;
        if (!hex_geometry(x, mat.youngs_modulus, mat.poisson_ratio, mat.density, m.settings.hourglass, &g)) {
            bad[e] = 1;
            return;
        }
        for (int i = 0; i < 8; ++i)
            for (int d = 0; d < 3; ++d) el->center_grad[e][3 * i + d] = g.center_grad[i][d];
        el->volume[e] = g.volume;
        for (int i = 0; i < 8; ++i)
            for (int a = 0; a < 4; ++a) el->gamma[e][4 * i + a] = g.gamma[i][a];
        for (int r = 0; r < 12; ++r)
            for (int c = 0; c < 12; ++c) el->h[e][12 * r + c] = g.h[r][c];
        for (int i = 0; i < 8; ++i) el->lumped[8 * e + i] = g.lumped_mass[i];
        el->dt_factor[e] = (1.0 - 0.36 * mat.poisson_ratio) / dilatational_wave_speed(mat);
    });
    for (uint8_t b : bad)
        if (b) return "degenerate hexahedron (singular Jacobian)";
    for (size_t e = 0; e < ne; ++e) {
        const crush_material& mat = m.materials[m.hex_part[e]];
        el->honeycomb[e] = mat.model == CRUSH_MAT_HONEYCOMB;
        if (simd && el->honeycomb[e]) el->simd_ids.push_back(e);
        else el->scalar_ids.push_back(e);
    }
    el->blocks.clear();
    Block cur;
    block_empty(&cur);
    for (size_t e : el->simd_ids) {
        if (cur.count == L) {
            el->blocks.push_back(cur);
            block_empty(&cur);
        }
        set_lane(&cur, cur.count, *el, e);
    }
    if (cur.count > 0) el->blocks.push_back(cur);
    el->block_out.assign(el->blocks.size(), {});
    return "";
}

// kernel.rs:116-156, the scalar f64 element (honeycomb rate form or Hencky elastic).
static bool element_force(const Elements& el, size_t e, const double* u, double* out, RateState* st) {
    const double* pos = el.model->positions.data();
    double x[8][3], ul[24];
    for (int i = 0; i < 8; ++i) {
        size_t n = el.conn[e][i];
        for (int d = 0; d < 3; ++d) {
            x[i][d] = pos[3 * n + d] + u[3 * n + d];
            ul[3 * i + d] = u[3 * n + d];
        }
    }
    const double* grad = el.center_grad[e].data();
    M3 f = m3_zero();
    for (int i = 0; i < 8; ++i)
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) f(a, b) += x[i][a] * grad[3 * i + b];
    if (m3_det(f) <= 0.0) {
        for (int k = 0; k < 24; ++k) out[k] = 0.0;
        return false;
    }
    // Elements::stress_update (kernel.rs:100-114): the honeycomb rate form
    // commits its state; an elastic material is Hencky with no state.
    const crush_material& mat = el.model->materials[el.part[e]];
    M3 tau;
    if (el.honeycomb[e]) {
        HoneycombParams p;
        honeycomb_params(mat, &p);
        RateState ns;
        honeycomb_rate_update(p, f, *st, &tau, &ns);
        *st = ns;
    } else {
        hencky_elastic(mat.youngs_modulus, mat.poisson_ratio, f, &tau);
    }
    M3 finv;
    m3_inverse(f, &finv);
    M3 m = m3_mul(tau, m3_transpose(finv));
    for (int k = 0; k < 9; ++k) m.m[k] = m.m[k] * el.volume[e];
    for (int i = 0; i < 8; ++i)
        for (int a = 0; a < 3; ++a) {
            double s = m(a, 0) * grad[3 * i];
            s = s + m(a, 1) * grad[3 * i + 1];
            s = s + m(a, 2) * grad[3 * i + 2];
            out[3 * i + a] = s;
        }
    // q (3x4) = U (3x8) Γ (8x4), r = H q, f_hg = R Γᵀ.
    const double* gam = el.gamma[e].data();
    double q[12];
    for (int a = 0; a < 4; ++a)
        for (int d = 0; d < 3; ++d) {
            double s = ul[d] * gam[a];
            for (int i = 1; i < 8; ++i) s = s + ul[3 * i + d] * gam[4 * i + a];
            q[3 * a + d] = s;
        }
    const double* h = el.h[e].data();
    double r[12];
    for (int row = 0; row < 12; ++row) {
        double s = h[12 * row] * q[0];
        for (int c = 1; c < 12; ++c) s = s + h[12 * row + c] * q[c];
        r[row] = s;
    }
    for (int i = 0; i < 8; ++i)
        for (int d = 0; d < 3; ++d) {
            double s = r[d] * gam[4 * i];
            for (int a = 1; a < 4; ++a) s = s + r[3 * a + d] * gam[4 * i + a];
            out[3 * i + d] += s;
        }
    return true;
}

size_t compute_forces(Elements& el, const double* u, double* global) {
    size_t newly = 0;
    const double* pos = el.model->positions.data();
    if (!el.blocks.empty()) {
        size_t before = 0, after = 0;
        for (const Block& b : el.blocks)
            for (int l = 0; l < b.count; ++l) before += b.eroded[l];
        long nb = (long)el.blocks.size();
        if (el.threads > 1) {
            parallel_for(el.threads, nb, 4, [&](long k) {
                block_forces(&el.blocks[k], u, pos, reinterpret_cast<float(*)[24]>(el.block_out[k].data()));
            });
        } else {
            for (long k = 0; k < nb; ++k)
                block_forces(&el.blocks[k], u, pos, reinterpret_cast<float(*)[24]>(el.block_out[k].data()));
        }
        for (const Block& b : el.blocks)
            for (int l = 0; l < b.count; ++l) after += b.eroded[l];
        newly += after - before;
        // Blocks::scatter, kernel_simd.rs:573
        for (size_t k = 0; k < el.blocks.size(); ++k) {
            const Block& b = el.blocks[k];
            for (int l = 0; l < b.count; ++l) {
                const float* f = el.block_out[k][l].data();
                for (int i = 0; i < 8; ++i) {
                    size_t n = b.conn[l][i];
                    global[3 * n] += (double)f[3 * i];
                    global[3 * n + 1] += (double)f[3 * i + 1];
                    global[3 * n + 2] += (double)f[3 * i + 2];
                }
            }
        }
        // mirror_erosion, kernel_simd.rs:588
        size_t k = 0;
        for (const Block& b : el.blocks)
            for (int l = 0; l < b.count; ++l) el.eroded[el.simd_ids[k++]] = b.eroded[l];
    }
    if (!el.scalar_ids.empty()) {
        const std::vector<size_t>& ids = el.scalar_ids;
        long ns = (long)ids.size();
        std::vector<std::array<double, 24>> outs(ns);
        std::vector<RateState> states(ns);
        std::vector<uint8_t> er(ns), newly_flag(ns, 0);
        for (long k = 0; k < ns; ++k) { states[k] = el.state[ids[k]]; er[k] = el.eroded[ids[k]]; }
        parallel_for(el.threads, ns, 32, [&](long k) {
            size_t e = ids[k];
            outs[k].fill(0.0);
            if (er[k]) return;
            if (!element_force(el, e, u, outs[k].data(), &states[k])) { er[k] = 1; newly_flag[k] = 1; }
        });
        for (long k = 0; k < ns; ++k) {
            size_t e = ids[k];
            el.state[e] = states[k];
            el.eroded[e] = er[k];
            newly += newly_flag[k];
            for (int i = 0; i < 8; ++i) {
                size_t n = el.conn[e][i];
                for (int d = 0; d < 3; ++d) global[3 * n + d] += outs[k][3 * i + d];
            }
        }
    }
    return newly;
}

void element_time_steps(const Elements& el, const double* u, std::vector<double>* out) {
    const double* pos = el.model->positions.data();
    size_t ne = el.conn.size();
    out->resize(ne);
    for (size_t e = 0; e < ne; ++e) {
        if (el.eroded[e]) { (*out)[e] = INF; continue; }
        double p[8][3];
        for (int i = 0; i < 8; ++i) {
            size_t n = el.conn[e][i];
            for (int d = 0; d < 3; ++d) p[i][d] = pos[3 * n + d] + u[3 * n + d];
        }
        double l, vol;
        characteristic_length_and_volume(p, &l, &vol);
        (*out)[e] = (std::isfinite(l) && vol > 0.0) ? l * el.dt_factor[e] : INF;
    }
}

bool stable_time_step(const Elements& el, const double* u, double* dt) {
    std::vector<double> t;
    element_time_steps(el, u, &t);
    double m = INF;
    for (double x : t) m = std::fmin(m, x);
    *dt = m;
    return std::isfinite(m);
}

double mass_scaling(const Elements& el, const double* u, double dt_min, const double* element_mass, double* added) {
    size_t nn = el.model->n_nodes();
    for (size_t i = 0; i < nn; ++i) added[i] = 0.0;
    std::vector<double> t;
    element_time_steps(el, u, &t);
    double total = 0.0;
    for (size_t e = 0; e < t.size(); ++e) {
        double dt = t[e];
        if (dt < dt_min) {
            double r = dt_min / dt;
            double extra = (std::fmin(r * r, 100.0) - 1.0) * element_mass[e];
            for (int i = 0; i < 8; ++i) added[el.conn[e][i]] += extra / 8.0;
            total += extra;
        }
    }
    return total;
}

std::vector<double> lumped_masses(const Elements& el, size_t n_nodes) {
    std::vector<double> m(n_nodes, 0.0);
    for (size_t e = 0; e < el.conn.size(); ++e)
        for (int i = 0; i < 8; ++i) m[el.conn[e][i]] += el.lumped[8 * e + i];
    return m;
}

void sync_states(Elements& el) {
    size_t k = 0;
    for (const Block& b : el.blocks)
        for (int l = 0; l < b.count; ++l) {
            RateState& s = el.state[el.simd_ids[k++]];
            for (int j = 0; j < 9; ++j) {
                s.f_prev_inv.m[j] = b.f_prev_inv[j][l];
                s.rotation.m[j] = b.rotation[j][l];
            }
            for (int j = 0; j < 6; ++j) s.stress[j] = b.stress[j][l];
            s.compaction = b.compaction[l];
        }
}

}  // namespace oracle
