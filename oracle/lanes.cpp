// lanes.cpp — TEST INFRASTRUCTURE ONLY (see oracle.hpp).
// Restates the f32 8-lane honeycomb kernel of src/kernel_simd.rs:300-491
// (block_forces_impl) operation for operation. Every lane helper below is a
// loop over the 8 lanes, which GCC vectorises into one AVX2 instruction,
// as rustc does for the reference. Compiled with -ffp-contract=off: the
// reference's `fma(a, b, c)` helper is a*b + c with two roundings.
#include "oracle.hpp"
#include <cmath>
#include <cstring>
#include <limits>

namespace oracle {

namespace {

struct V { float v[L]; };

inline V splat(float x) { V r; for (int l = 0; l < L; ++l) r.v[l] = x; return r; }
inline V zero() { return splat(0.0f); }
inline V add(V a, V b) { V r; for (int l = 0; l < L; ++l) r.v[l] = a.v[l] + b.v[l]; return r; }
inline V sub(V a, V b) { V r; for (int l = 0; l < L; ++l) r.v[l] = a.v[l] - b.v[l]; return r; }
inline V mul(V a, V b) { V r; for (int l = 0; l < L; ++l) r.v[l] = a.v[l] * b.v[l]; return r; }
inline V fma_(V a, V b, V c) { V r; for (int l = 0; l < L; ++l) r.v[l] = a.v[l] * b.v[l] + c.v[l]; return r; }
inline V scale(V a, float s) { V r; for (int l = 0; l < L; ++l) r.v[l] = a.v[l] * s; return r; }
inline V div_(V a, V b) { V r; for (int l = 0; l < L; ++l) r.v[l] = a.v[l] / b.v[l]; return r; }
inline V select(const bool m[L], V a, V b) { V r; for (int l = 0; l < L; ++l) r.v[l] = m[l] ? a.v[l] : b.v[l]; return r; }
// f32::max / f32::min: the non-NaN operand wins.
inline float fmax_(float a, float b) { return (a > b || b != b) ? a : b; }
inline float fmin_(float a, float b) { return (a < b || b != b) ? a : b; }
inline V vmax(V a, V b) { V r; for (int l = 0; l < L; ++l) r.v[l] = fmax_(a.v[l], b.v[l]); return r; }
inline V clamp(V a, V lo, V hi) { V r; for (int l = 0; l < L; ++l) r.v[l] = fmin_(fmax_(a.v[l], lo.v[l]), hi.v[l]); return r; }

struct M { V m[9]; };

inline M mat_mul(const M& a, const M& b) {
    M r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            V acc = mul(a.m[3 * i], b.m[j]);
            acc = fma_(a.m[3 * i + 1], b.m[3 + j], acc);
            acc = fma_(a.m[3 * i + 2], b.m[6 + j], acc);
            r.m[3 * i + j] = acc;
        }
    return r;
}
inline M mat_mul_t(const M& a, const M& b) {  // a · bᵀ
    M r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            V acc = mul(a.m[3 * i], b.m[3 * j]);
            acc = fma_(a.m[3 * i + 1], b.m[3 * j + 1], acc);
            acc = fma_(a.m[3 * i + 2], b.m[3 * j + 2], acc);
            r.m[3 * i + j] = acc;
        }
    return r;
}
inline M mat_t_mul(const M& a, const M& b) {  // aᵀ · b
    M r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            V acc = mul(a.m[i], b.m[j]);
            acc = fma_(a.m[3 + i], b.m[3 + j], acc);
            acc = fma_(a.m[6 + i], b.m[6 + j], acc);
            r.m[3 * i + j] = acc;
        }
    return r;
}
inline V det3(const M& m) {
    V c0 = sub(mul(m.m[4], m.m[8]), mul(m.m[5], m.m[7]));
    V c1 = sub(mul(m.m[5], m.m[6]), mul(m.m[3], m.m[8]));
    V c2 = sub(mul(m.m[3], m.m[7]), mul(m.m[4], m.m[6]));
    return fma_(m.m[0], c0, fma_(m.m[1], c1, mul(m.m[2], c2)));
}
inline M inv3(const M& m, V det) {
    V inv_det = div_(splat(1.0f), det);
    M r;
    r.m[0] = sub(mul(m.m[4], m.m[8]), mul(m.m[5], m.m[7]));
    r.m[1] = sub(mul(m.m[2], m.m[7]), mul(m.m[1], m.m[8]));
    r.m[2] = sub(mul(m.m[1], m.m[5]), mul(m.m[2], m.m[4]));
    r.m[3] = sub(mul(m.m[5], m.m[6]), mul(m.m[3], m.m[8]));
    r.m[4] = sub(mul(m.m[0], m.m[8]), mul(m.m[2], m.m[6]));
    r.m[5] = sub(mul(m.m[2], m.m[3]), mul(m.m[0], m.m[5]));
    r.m[6] = sub(mul(m.m[3], m.m[7]), mul(m.m[4], m.m[6]));
    r.m[7] = sub(mul(m.m[1], m.m[6]), mul(m.m[0], m.m[7]));
    r.m[8] = sub(mul(m.m[0], m.m[4]), mul(m.m[1], m.m[3]));
    for (int k = 0; k < 9; ++k) r.m[k] = mul(r.m[k], inv_det);
    return r;
}
inline M identity() {
    M r;
    for (int k = 0; k < 9; ++k) r.m[k] = zero();
    r.m[0] = r.m[4] = r.m[8] = splat(1.0f);
    return r;
}
inline V load(const float* p) { V r; std::memcpy(r.v, p, sizeof(r.v)); return r; }
inline void store(float* p, V a) { std::memcpy(p, a.v, sizeof(a.v)); }

}  // namespace

void block_empty(Block* b) {
    std::memset(b, 0, sizeof(Block));
    const float inf = std::numeric_limits<float>::infinity();
    for (int l = 0; l < L; ++l) {
        b->youngs[l] = 1.0f;
        b->yield0[l] = 1.0f;
        b->trans[l] = 1.0f;
        for (int k = 0; k < MAX_KNOTS; ++k) b->knot_c[k][l] = inf;
        b->f_prev_inv[0][l] = b->f_prev_inv[4][l] = b->f_prev_inv[8][l] = 1.0f;
        b->rotation[0][l] = b->rotation[4][l] = b->rotation[8][l] = 1.0f;
        b->eroded[l] = true;
    }
    b->count = 0;
}

void block_forces(Block* b, const double* u, const double* positions, float out[L][24]) {
    // Gather x = (X + u) as f32 and u as f32 (kernel_simd.rs:301-314).
    V x[24], ul[24];
    for (int k = 0; k < 24; ++k) { x[k] = zero(); ul[k] = zero(); }
    for (int l = 0; l < b->count; ++l)
        for (int i = 0; i < 8; ++i) {
            size_t n = b->conn[l][i];
            for (int c = 0; c < 3; ++c) {
                double p = positions[3 * n + c], d = u[3 * n + c];
                x[3 * i + c].v[l] = (float)(p + d);
                ul[3 * i + c].v[l] = (float)d;
            }
        }
    V grad[24];
    for (int k = 0; k < 24; ++k) grad[k] = load(b->grad[k]);
    // F = Σ x_i ⊗ ∇N_i
    M f;
    for (int k = 0; k < 9; ++k) f.m[k] = zero();
    for (int i = 0; i < 8; ++i)
        for (int a = 0; a < 3; ++a)
            for (int c = 0; c < 3; ++c) f.m[3 * a + c] = fma_(x[3 * i + a], grad[3 * i + c], f.m[3 * a + c]);
    V det = det3(f);
    bool active[L];
    for (int l = 0; l < L; ++l) active[l] = false;
    for (int l = 0; l < b->count; ++l) {
        if (!b->eroded[l] && det.v[l] <= 0.0f) b->eroded[l] = true;
        active[l] = !b->eroded[l];
    }
    V det_safe = select(active, det, splat(1.0f));
    M id = identity();
    M f_safe;
    for (int k = 0; k < 9; ++k) f_safe.m[k] = select(active, f.m[k], id.m[k]);

    M f_prev_inv, rot;
    for (int k = 0; k < 9; ++k) { f_prev_inv.m[k] = load(b->f_prev_inv[k]); rot.m[k] = load(b->rotation[k]); }
    // ---- honeycomb rate update ----
    M f_inc = mat_mul(f_safe, f_prev_inv);
    M d_inc, mid;
    for (int k = 0; k < 9; ++k) {
        d_inc.m[k] = sub(f_inc.m[k], id.m[k]);
        mid.m[k] = fma_(d_inc.m[k], splat(0.5f), id.m[k]);
    }
    M mid_inv = inv3(mid, det3(mid));
    M g = mat_mul(d_inc, mid_inv);
    M d, w;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            d.m[3 * i + j] = scale(add(g.m[3 * i + j], g.m[3 * j + i]), 0.5f);
            w.m[3 * i + j] = scale(sub(g.m[3 * i + j], g.m[3 * j + i]), 0.5f);
        }
    V omega2 = fma_(w.m[1], w.m[1], fma_(w.m[2], w.m[2], mul(w.m[5], w.m[5])));
    V inv_den = div_(splat(1.0f), fma_(omega2, splat(0.25f), splat(1.0f)));
    M ww = mat_mul(w, w);
    M delta_r;
    for (int k = 0; k < 9; ++k) delta_r.m[k] = fma_(fma_(ww.m[k], splat(0.5f), w.m[k]), inv_den, id.m[k]);
    M r = mat_mul(delta_r, rot);
    M de = mat_mul(mat_t_mul(r, d), r);
    V e = load(b->youngs);
    V s[6];
    for (int k = 0; k < 6; ++k) s[k] = load(b->stress[k]);
    s[0] = fma_(e, de.m[0], s[0]);
    s[1] = fma_(e, de.m[4], s[1]);
    s[2] = fma_(e, de.m[8], s[2]);
    s[3] = fma_(e, de.m[1], s[3]);
    s[4] = fma_(e, de.m[5], s[4]);
    s[5] = fma_(e, de.m[2], s[5]);
    V comp = load(b->compaction);
    V kc = load(b->knot_c[0]), ks = load(b->knot_s[0]), kh = load(b->knot_h[0]);
    for (int i = 1; i < MAX_KNOTS; ++i) {
        bool m[L];
        for (int l = 0; l < L; ++l) m[l] = b->compaction[l] >= b->knot_c[i][l];
        kc = select(m, load(b->knot_c[i]), kc);
        ks = select(m, load(b->knot_s[i]), ks);
        kh = select(m, load(b->knot_h[i]), kh);
    }
    V hard = kh;
    V sigma_yc = fma_(hard, sub(comp, kc), ks);
    V trans = load(b->trans);
    V tk[3] = {splat(1.0f), trans, trans};
    V dc = zero();
    for (int it = 0; it < 3; ++it) {
        V sigma_y = fma_(hard, dc, sigma_yc);
        V sum = zero(), t_active = zero();
        for (int k = 0; k < 3; ++k) {
            V a = scale(s[k], -1.0f);
            V cap = mul(tk[k], sigma_y);
            bool over[L];
            for (int l = 0; l < L; ++l) over[l] = a.v[l] > cap.v[l];
            sum = add(sum, select(over, sub(a, mul(tk[k], sigma_yc)), zero()));
            t_active = add(t_active, select(over, tk[k], zero()));
        }
        V den = fma_(t_active, hard, e);
        V dc_new = div_(sum, den);
        bool any[L];
        for (int l = 0; l < L; ++l) any[l] = t_active.v[l] > 0.0f;
        dc = select(any, dc_new, zero());
    }
    V sigma_y = vmax(fma_(hard, dc, sigma_yc), zero());
    for (int k = 0; k < 3; ++k) {
        V cap = mul(tk[k], sigma_y);
        s[k] = clamp(s[k], scale(cap, -1.0f), cap);
    }
    V tau_y = scale(sigma_y, 0.5f);
    V neg_tau_y = scale(tau_y, -1.0f);
    for (int k = 3; k < 6; ++k) s[k] = clamp(s[k], neg_tau_y, tau_y);
    M sigma_hat;
    sigma_hat.m[0] = s[0]; sigma_hat.m[1] = s[3]; sigma_hat.m[2] = s[5];
    sigma_hat.m[3] = s[3]; sigma_hat.m[4] = s[1]; sigma_hat.m[5] = s[4];
    sigma_hat.m[6] = s[5]; sigma_hat.m[7] = s[4]; sigma_hat.m[8] = s[2];
    M tau = mat_mul_t(mat_mul(r, sigma_hat), r);
    for (int k = 0; k < 9; ++k) tau.m[k] = mul(tau.m[k], det_safe);
    // Commit state in active lanes.
    M f_inv = inv3(f_safe, det_safe);
    for (int k = 0; k < 9; ++k) {
        store(b->f_prev_inv[k], select(active, f_inv.m[k], f_prev_inv.m[k]));
        store(b->rotation[k], select(active, r.m[k], rot.m[k]));
    }
    for (int k = 0; k < 6; ++k) store(b->stress[k], select(active, s[k], load(b->stress[k])));
    store(b->compaction, select(active, add(comp, dc), comp));

    // ---- nodal forces: f_i = τ F⁻ᵀ ∇N_i V₀ ----
    M m = mat_mul_t(tau, f_inv);
    V vol = load(b->volume);
    for (int k = 0; k < 9; ++k) m.m[k] = mul(m.m[k], vol);
    V fo[24];
    for (int i = 0; i < 8; ++i)
        for (int a = 0; a < 3; ++a) {
            V acc = mul(m.m[3 * a], grad[3 * i]);
            acc = fma_(m.m[3 * a + 1], grad[3 * i + 1], acc);
            acc = fma_(m.m[3 * a + 2], grad[3 * i + 2], acc);
            fo[3 * i + a] = acc;
        }
    // ---- hourglass: q = U Γ, rr = H q, f += rr Γᵀ ----
    V q[12];
    for (int mode = 0; mode < 4; ++mode)
        for (int dir = 0; dir < 3; ++dir) {
            V acc = zero();
            for (int i = 0; i < 8; ++i) acc = fma_(ul[3 * i + dir], load(b->gamma[4 * i + mode]), acc);
            q[3 * mode + dir] = acc;
        }
    V rr[12];
    for (int k = 0; k < 12; ++k) rr[k] = zero();
    for (int col = 0; col < 12; ++col)
        for (int row = 0; row < 12; ++row) rr[row] = fma_(load(b->h[12 * col + row]), q[col], rr[row]);
    for (int i = 0; i < 8; ++i)
        for (int dir = 0; dir < 3; ++dir) {
            V acc = fo[3 * i + dir];
            for (int mode = 0; mode < 4; ++mode) acc = fma_(rr[3 * mode + dir], load(b->gamma[4 * i + mode]), acc);
            fo[3 * i + dir] = acc;
        }
    for (int l = 0; l < L; ++l)
        for (int k = 0; k < 24; ++k) out[l][k] = active[l] ? fo[k].v[l] : 0.0f;
}

}  // namespace oracle
