// material.cpp — TEST INFRASTRUCTURE ONLY (see oracle.hpp).
// Restates the honeycomb part of src/material.rs.
#include "oracle.hpp"
#include <cmath>
#include <limits>

namespace oracle {

static const double INF = std::numeric_limits<double>::infinity();

// Plasticity::check, material.rs:116-151 (honeycomb only).
static std::string check(const crush_material& m) {
    int n = m.n_curve;
    int extra = m.has_densification ? 1 : 0;
    if (m.has_densification) {
        double c_lock = m.densification[0], k_lock = m.densification[1];
        if (c_lock <= 0.0 || k_lock < 0.0) return "densification needs c_lock > 0 and k_lock >= 0";
        if (n > 0 && m.curve[n - 1][0] >= c_lock) return "densification c_lock must lie beyond the last curve knot";
    }
    if (n == 0) return "";
    if (n < 2 || n + extra > MAX_KNOTS) return "yield curve needs 2..=8 knots (one fewer with densification)";
    if (m.curve[0][0] != 0.0) return "yield curve must start at compaction 0";
    for (int i = 0; i + 1 < n; ++i)
        if (m.curve[i + 1][0] <= m.curve[i][0]) return "yield curve compaction must be strictly increasing";
    for (int i = 0; i < n; ++i)
        if (m.curve[i][1] <= 0.0) return "yield curve stresses must be positive";
    return "";
}

// HoneycombParams::from_material, material.rs:430-449.
std::string honeycomb_params(const crush_material& m, HoneycombParams* p) {
    std::string err = check(m);
    if (!err.empty()) return err;
    for (int i = 0; i < MAX_KNOTS; ++i) { p->knots[i][0] = INF; p->knots[i][1] = 0.0; p->knots[i][2] = 0.0; }
    int n;
    if (m.n_curve < 2) {
        p->knots[0][0] = 0.0; p->knots[0][1] = m.yield_stress; p->knots[0][2] = m.hardening;
        n = 1;
    } else {
        for (int i = 0; i < m.n_curve; ++i) {
            double h = (i + 1 < m.n_curve) ? (m.curve[i + 1][1] - m.curve[i][1]) / (m.curve[i + 1][0] - m.curve[i][0])
                                           : p->knots[i - 1][2];
            p->knots[i][0] = m.curve[i][0]; p->knots[i][1] = m.curve[i][1]; p->knots[i][2] = h;
        }
        n = m.n_curve;
    }
    if (m.has_densification) {
        double c_lock = m.densification[0], k_lock = m.densification[1];
        const double* last = p->knots[n - 1];
        double s = last[1] + last[2] * (c_lock - last[0]);
        double h = last[2] + k_lock;
        p->knots[n][0] = c_lock; p->knots[n][1] = s; p->knots[n][2] = h;
    }
    p->youngs_modulus = m.youngs_modulus;
    p->yield_stress = m.yield_stress;
    p->hardening = m.hardening;
    p->cap_factor[0] = 1.0;
    p->cap_factor[1] = m.transverse_factor;
    p->cap_factor[2] = m.transverse_factor;
    return "";
}

// material.rs:459-467
void HoneycombParams::yield_at(double c, double* sy, double* h) const {
    const double* k = knots[0];
    for (int i = 1; i < MAX_KNOTS; ++i)
        if (c >= knots[i][0]) k = knots[i];
    *sy = k[1] + k[2] * (c - k[0]);
    *h = k[2];
}

// Plasticity::yield_at, material.rs:83-102.
void plasticity_yield_at(const crush_material& m, double c, double* sy_out, double* h_out) {
    double sy, h;
    if (m.n_curve < 2) {
        sy = m.yield_stress + m.hardening * c;
        h = m.hardening;
    } else {
        int i = 0;
        while (i + 2 < m.n_curve && c >= m.curve[i + 1][0]) ++i;
        h = (m.curve[i + 1][1] - m.curve[i][1]) / (m.curve[i + 1][0] - m.curve[i][0]);
        sy = m.curve[i][1] + h * (c - m.curve[i][0]);
    }
    if (m.has_densification && c > m.densification[0]) {
        sy += m.densification[1] * (c - m.densification[0]);
        h += m.densification[1];
    }
    *sy_out = sy;
    *h_out = h;
}

// material.rs:226
double dilatational_wave_speed(const crush_material& m) {
    double e = m.youngs_modulus, v = m.poisson_ratio;
    double mm = e * (1.0 - v) / ((1.0 + v) * (1.0 - 2.0 * v));
    return std::sqrt(mm / m.density);
}

RateState rate_state_default() {
    RateState s;
    s.f_prev_inv = m3_identity();
    s.rotation = m3_identity();
    for (double& x : s.stress) x = 0.0;
    s.compaction = 0.0;
    return s;
}

// honeycomb_rate_update, material.rs:472-535.
void honeycomb_rate_update(const HoneycombParams& p, const M3& f, const RateState& state, M3* tau_out, RateState* ns) {
    const double e = p.youngs_modulus;
    const M3 i3 = m3_identity();
    M3 f_inc = m3_mul(f, state.f_prev_inv);
    M3 mid;
    for (int k = 0; k < 9; ++k) mid.m[k] = 0.5 * (f_inc.m[k] + i3.m[k]);
    M3 mid_inv;
    if (!m3_inverse(mid, &mid_inv)) mid_inv = i3;
    M3 dm;
    for (int k = 0; k < 9; ++k) dm.m[k] = f_inc.m[k] - i3.m[k];
    M3 g = m3_mul(dm, mid_inv);
    M3 d, w;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            d(i, j) = 0.5 * (g(i, j) + g(j, i));
            w(i, j) = 0.5 * (g(i, j) - g(j, i));
        }
    double omega2 = w(0, 1) * w(0, 1) + w(0, 2) * w(0, 2) + w(1, 2) * w(1, 2);
    M3 hw;
    for (int k = 0; k < 9; ++k) hw.m[k] = 0.5 * w.m[k];
    M3 ww = m3_mul(hw, w);
    double den = 1.0 + 0.25 * omega2;
    M3 delta_r;
    for (int k = 0; k < 9; ++k) delta_r.m[k] = i3.m[k] + (w.m[k] + ww.m[k]) / den;
    M3 r = m3_mul(delta_r, state.rotation);
    M3 de = m3_mul(m3_mul(m3_transpose(r), d), r);
    double s[6];
    for (int k = 0; k < 6; ++k) s[k] = state.stress[k];
    s[0] += e * de(0, 0);
    s[1] += e * de(1, 1);
    s[2] += e * de(2, 2);
    s[3] += e * de(0, 1);
    s[4] += e * de(1, 2);
    s[5] += e * de(0, 2);

    double sigma_yc, hard;
    p.yield_at(state.compaction, &sigma_yc, &hard);
    const double* t = p.cap_factor;
    double dc = 0.0;
    for (int it = 0; it < 3; ++it) {
        double sigma_y = sigma_yc + hard * dc;
        double sum = 0.0, t_active = 0.0;
        for (int k = 0; k < 3; ++k) {
            if (-s[k] > t[k] * sigma_y) {
                sum += -s[k] - t[k] * sigma_yc;
                t_active += t[k];
            }
        }
        double dc_new = (t_active == 0.0) ? 0.0 : sum / (e + t_active * hard);
        if (std::fabs(dc_new - dc) <= 1e-14 * std::fmax(dc_new, 1e-300)) {
            dc = dc_new;
            break;
        }
        dc = dc_new;
    }
    double sigma_y = std::fmax(sigma_yc + hard * dc, 0.0);
    auto clamp = [](double x, double lo, double hi) { return x < lo ? lo : (x > hi ? hi : x); };
    for (int k = 0; k < 3; ++k) s[k] = clamp(s[k], -t[k] * sigma_y, t[k] * sigma_y);
    double tau_y = 0.5 * sigma_y;
    for (int k = 3; k < 6; ++k) s[k] = clamp(s[k], -tau_y, tau_y);

    M3 sh;
    sh(0, 0) = s[0]; sh(0, 1) = s[3]; sh(0, 2) = s[5];
    sh(1, 0) = s[3]; sh(1, 1) = s[1]; sh(1, 2) = s[4];
    sh(2, 0) = s[5]; sh(2, 1) = s[4]; sh(2, 2) = s[2];
    M3 rs = m3_mul(m3_mul(r, sh), m3_transpose(r));
    double j = m3_det(f);
    for (int k = 0; k < 9; ++k) tau_out->m[k] = j * rs.m[k];
    M3 finv;
    if (!m3_inverse(f, &finv)) finv = i3;
    ns->f_prev_inv = finv;
    ns->rotation = r;
    for (int k = 0; k < 6; ++k) ns->stress[k] = s[k];
    ns->compaction = state.compaction + dc;
}

}  // namespace oracle
