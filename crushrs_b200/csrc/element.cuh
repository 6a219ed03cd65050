// element.cuh — the one-point honeycomb hexahedron on one CUDA thread.
//
// The arithmetic is the reference's f32 lane kernel (crushrs
// src/kernel_simd.rs:300-491) for one lane: the same operations in the same
// order, each rounded once (the file is compiled with --fmad=false), so the
// corner forces and committed state equal the reference's bit for bit on the
// same inputs. Only the data movement is B200-specific: the element record is
// read as 16-byte planes, node positions and displacements as f64 gathers.
#pragma once
#include "common.cuh"

namespace crush {

struct M3f {
    float m[9];
};

__device__ __forceinline__ void mat_mul(const M3f& a, const M3f& b, M3f& r) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float acc = a.m[3 * i] * b.m[j];
            acc = a.m[3 * i + 1] * b.m[3 + j] + acc;
            acc = a.m[3 * i + 2] * b.m[6 + j] + acc;
            r.m[3 * i + j] = acc;
        }
}
// a · bᵀ
__device__ __forceinline__ void mat_mul_t(const M3f& a, const M3f& b, M3f& r) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float acc = a.m[3 * i] * b.m[3 * j];
            acc = a.m[3 * i + 1] * b.m[3 * j + 1] + acc;
            acc = a.m[3 * i + 2] * b.m[3 * j + 2] + acc;
            r.m[3 * i + j] = acc;
        }
}
// aᵀ · b
__device__ __forceinline__ void mat_t_mul(const M3f& a, const M3f& b, M3f& r) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float acc = a.m[i] * b.m[j];
            acc = a.m[3 + i] * b.m[3 + j] + acc;
            acc = a.m[6 + i] * b.m[6 + j] + acc;
            r.m[3 * i + j] = acc;
        }
}
__device__ __forceinline__ float det3(const M3f& m) {
    float c0 = m.m[4] * m.m[8] - m.m[5] * m.m[7];
    float c1 = m.m[5] * m.m[6] - m.m[3] * m.m[8];
    float c2 = m.m[3] * m.m[7] - m.m[4] * m.m[6];
    return m.m[0] * c0 + (m.m[1] * c1 + m.m[2] * c2);
}
__device__ __forceinline__ void inv3(const M3f& m, float det, M3f& r) {
    float inv_det = 1.0f / det;
    r.m[0] = (m.m[4] * m.m[8] - m.m[5] * m.m[7]) * inv_det;
    r.m[1] = (m.m[2] * m.m[7] - m.m[1] * m.m[8]) * inv_det;
    r.m[2] = (m.m[1] * m.m[5] - m.m[2] * m.m[4]) * inv_det;
    r.m[3] = (m.m[5] * m.m[6] - m.m[3] * m.m[8]) * inv_det;
    r.m[4] = (m.m[0] * m.m[8] - m.m[2] * m.m[6]) * inv_det;
    r.m[5] = (m.m[2] * m.m[3] - m.m[0] * m.m[5]) * inv_det;
    r.m[6] = (m.m[3] * m.m[7] - m.m[4] * m.m[6]) * inv_det;
    r.m[7] = (m.m[1] * m.m[6] - m.m[0] * m.m[7]) * inv_det;
    r.m[8] = (m.m[0] * m.m[4] - m.m[1] * m.m[3]) * inv_det;
}
// f32::max / f32::min: the non-NaN operand wins (fmaxf / fminf semantics).
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

// Material update of one element (src/kernel_simd.rs:336-443 for one lane).
// In: deformation gradient f (det > 0), state st[25]. Out: Kirchhoff stress
// tau, the new state written back into st, f_inv = f⁻¹.
__device__ __forceinline__ void honeycomb_update(const M3f& f, float det, float* st, const MaterialF32& mat, M3f& tau,
                                                 M3f& f_inv) {
    M3f f_prev_inv, rot;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        f_prev_inv.m[k] = st[k];
        rot.m[k] = st[9 + k];
    }
    const float id[9] = {1.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 1.f};
    M3f f_inc, d_inc, mid, mid_inv, g;
    mat_mul(f, f_prev_inv, f_inc);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        d_inc.m[k] = f_inc.m[k] - id[k];
        mid.m[k] = d_inc.m[k] * 0.5f + id[k];
    }
    inv3(mid, det3(mid), mid_inv);
    mat_mul(d_inc, mid_inv, g);
    M3f d, w;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            d.m[3 * i + j] = (g.m[3 * i + j] + g.m[3 * j + i]) * 0.5f;
            w.m[3 * i + j] = (g.m[3 * i + j] - g.m[3 * j + i]) * 0.5f;
        }
    float omega2 = w.m[1] * w.m[1] + (w.m[2] * w.m[2] + w.m[5] * w.m[5]);
    float inv_den = 1.0f / (omega2 * 0.25f + 1.0f);
    M3f ww, delta_r, r, rtd, de;
    mat_mul(w, w, ww);
#pragma unroll
    for (int k = 0; k < 9; ++k) delta_r.m[k] = (ww.m[k] * 0.5f + w.m[k]) * inv_den + id[k];
    mat_mul(delta_r, rot, r);
    mat_t_mul(r, d, rtd);
    mat_mul(rtd, r, de);
    const float e = mat.youngs;
    float s[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) s[k] = st[18 + k];
    s[0] = e * de.m[0] + s[0];
    s[1] = e * de.m[4] + s[1];
    s[2] = e * de.m[8] + s[2];
    s[3] = e * de.m[1] + s[3];
    s[4] = e * de.m[5] + s[4];
    s[5] = e * de.m[2] + s[5];
    const float comp = st[S_COMPACTION];
    float kc = mat.knot_c[0], ks = mat.knot_s[0], kh = mat.knot_h[0];
#pragma unroll
    for (int i = 1; i < MAX_KNOTS; ++i) {
        bool m = comp >= mat.knot_c[i];
        kc = m ? mat.knot_c[i] : kc;
        ks = m ? mat.knot_s[i] : ks;
        kh = m ? mat.knot_h[i] : kh;
    }
    const float hard = kh;
    const float sigma_yc = hard * (comp - kc) + ks;
    const float tk[3] = {1.0f, mat.trans, mat.trans};
    float dc = 0.0f;
#pragma unroll
    for (int it = 0; it < 3; ++it) {
        float sigma_y = hard * dc + sigma_yc;
        float sum = 0.0f, t_active = 0.0f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            float a = s[k] * -1.0f;
            float cap = tk[k] * sigma_y;
            bool over = a > cap;
            sum = sum + (over ? a - tk[k] * sigma_yc : 0.0f);
            t_active = t_active + (over ? tk[k] : 0.0f);
        }
        float den = t_active * hard + e;
        float dc_new = sum / den;
        dc = t_active > 0.0f ? dc_new : 0.0f;
    }
    float sigma_y = fmaxf(hard * dc + sigma_yc, 0.0f);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float cap = tk[k] * sigma_y;
        s[k] = clampf(s[k], cap * -1.0f, cap);
    }
    float tau_y = sigma_y * 0.5f;
    float neg_tau_y = tau_y * -1.0f;
#pragma unroll
    for (int k = 3; k < 6; ++k) s[k] = clampf(s[k], neg_tau_y, tau_y);
    M3f sigma_hat, rs;
    sigma_hat.m[0] = s[0]; sigma_hat.m[1] = s[3]; sigma_hat.m[2] = s[5];
    sigma_hat.m[3] = s[3]; sigma_hat.m[4] = s[1]; sigma_hat.m[5] = s[4];
    sigma_hat.m[6] = s[5]; sigma_hat.m[7] = s[4]; sigma_hat.m[8] = s[2];
    mat_mul(r, sigma_hat, rs);
    mat_mul_t(rs, r, tau);
#pragma unroll
    for (int k = 0; k < 9; ++k) tau.m[k] = tau.m[k] * det;
    inv3(f, det, f_inv);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        st[k] = f_inv.m[k];
        st[9 + k] = r.m[k];
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) st[18 + k] = s[k];
    st[S_COMPACTION] = comp + dc;
}

}  // namespace crush
