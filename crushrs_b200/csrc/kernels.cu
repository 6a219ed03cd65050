// kernels.cu — CUDA kernels of the explicit time step (sm_100a).
//
// Data layout and roofline notes:
//  * The element kernel streams each honeycomb element's static record
//    (37 x 16 B planes: connectivity, dN/dX, hourglass base vectors, the
//    symmetric 12x12 hourglass stiffness, volume/material) and its state
//    (7 planes, read + written), gathers its 8 nodes' f64 position and
//    displacement through L2, and writes 24 f32 corner forces. All loads of
//    per-element data are 128-bit and coalesced (one plane = 512 B per warp).
//  * Force assembly is a gather, not an atomic scatter: each node sums its
//    incident (element, corner) forces in increasing element order over a
//    CSR built at set-up, in f64 — the order and precision of the reference's
//    serial scatter (src/kernel_simd.rs:573-586), so results are reproducible
//    run to run and identical to the reference's summation.
//  * Nothing here waits on another block or another GPU; every kernel is a
//    plain data-parallel pass whose only cross-block interaction is an
//    atomic integer count or an atomicMin on a bit pattern.
#include <cmath>
#include <cfloat>
#include <climits>
#include <math_constants.h>

#include "element.cuh"
#include "kernels.cuh"

namespace crush {

namespace {

constexpr int TPB = 256;

__host__ __device__ inline long long blocks_for(long long n, int tpb) { return (n + tpb - 1) / tpb; }

// ---------------------------------------------------------------------------
// Set-up geometry (f64), restating src/element.rs:141-162 (HexGeometry::new)
// with the hourglass stiffness reduced directly to its rank-12 form.
// ---------------------------------------------------------------------------
__constant__ double c_xi[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                  {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
__constant__ double c_modes[4][8] = {{1, 1, -1, -1, -1, -1, 1, 1},
                                     {1, -1, -1, 1, -1, 1, 1, -1},
                                     {1, -1, 1, -1, 1, -1, 1, -1},
                                     {-1, 1, -1, 1, 1, -1, 1, -1}};

__device__ void shape_derivatives(double xi, double eta, double zeta, double dn[8][3]) {
    for (int i = 0; i < 8; ++i) {
        const double s0 = c_xi[i][0], s1 = c_xi[i][1], s2 = c_xi[i][2];
        dn[i][0] = 0.125 * s0 * (1.0 + s1 * eta) * (1.0 + s2 * zeta);
        dn[i][1] = 0.125 * s1 * (1.0 + s0 * xi) * (1.0 + s2 * zeta);
        dn[i][2] = 0.125 * s2 * (1.0 + s0 * xi) * (1.0 + s1 * eta);
    }
}

// First-row cofactor determinant and inverse of a row-major 3x3.
__device__ double det3d(const double* a) {
    double m11 = a[4] * a[8] - a[7] * a[5];
    double m12 = a[3] * a[8] - a[6] * a[5];
    double m13 = a[3] * a[7] - a[6] * a[4];
    return a[0] * m11 - a[1] * m12 + a[2] * m13;
}
__device__ bool inv3d(const double* a, double* r) {
    double m11 = a[4] * a[8] - a[7] * a[5];
    double m12 = a[3] * a[8] - a[6] * a[5];
    double m13 = a[3] * a[7] - a[6] * a[4];
    double det = a[0] * m11 - a[1] * m12 + a[2] * m13;
    if (det == 0.0) return false;
    r[0] = m11 / det;
    r[1] = -(a[1] * a[8] - a[7] * a[2]) / det;
    r[2] = (a[1] * a[5] - a[4] * a[2]) / det;
    r[3] = -m12 / det;
    r[4] = (a[0] * a[8] - a[6] * a[2]) / det;
    r[5] = -(a[0] * a[5] - a[3] * a[2]) / det;
    r[6] = m13 / det;
    r[7] = -(a[0] * a[7] - a[6] * a[1]) / det;
    r[8] = (a[0] * a[4] - a[3] * a[1]) / det;
    return true;
}

// J = dNᵀ x, grad = dN J⁻ᵀ (src/element.rs:43).
__device__ bool reference_gradients(const double x[8][3], const double dn[8][3], double g[8][3], double* det) {
    double j[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double s = dn[0][r] * x[0][c];
            for (int k = 1; k < 8; ++k) s = s + dn[k][r] * x[k][c];
            j[3 * r + c] = s;
        }
    double ji[9];
    if (!inv3d(j, ji)) return false;
    for (int i = 0; i < 8; ++i)
        for (int c = 0; c < 3; ++c) {
            double s = dn[i][0] * ji[3 * c];
            s = s + dn[i][1] * ji[3 * c + 1];
            s = s + dn[i][2] * ji[3 * c + 2];
            g[i][c] = s;
        }
    *det = det3d(j);
    return true;
}

__global__ void __launch_bounds__(128) k_setup_geometry(long long n_all, const double* __restrict__ pos,
                                                        const uint32_t* __restrict__ conn, const int32_t* __restrict__ part,
                                                        const double* __restrict__ mat, double hourglass,
                                                        const int64_t* __restrict__ hc_index, long long stride,
                                                        float4* __restrict__ planes, double* __restrict__ volume_out,
                                                        double* __restrict__ lumped_out, double* __restrict__ dt_factor,
                                                        double* __restrict__ elem_mass, int* __restrict__ bad) {
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_all) return;
    double x[8][3];
    uint32_t nid[8];
    for (int i = 0; i < 8; ++i) {
        nid[i] = conn[8 * e + i];
        for (int d = 0; d < 3; ++d) x[i][d] = pos[3 * (long long)nid[i] + d];
    }
    const int p = part[e];
    const double youngs = mat[3 * p], nu = mat[3 * p + 1], rho = mat[3 * p + 2];
    double dnc[8][3], gc[8][3], detc;
    shape_derivatives(0.0, 0.0, 0.0, dnc);
    if (!reference_gradients(x, dnc, gc, &detc)) {
        atomicExch(bad, 1);
        return;
    }
    // Hourglass base vectors (src/element.rs:93-102).
    double gam[8][4];
    for (int a = 0; a < 4; ++a) {
        double hx[3] = {0.0, 0.0, 0.0};
        for (int j = 0; j < 8; ++j)
            for (int d = 0; d < 3; ++d) hx[d] += c_modes[a][j] * x[j][d];
        for (int i = 0; i < 8; ++i) {
            double dot = hx[0] * gc[i][0] + hx[1] * gc[i][1] + hx[2] * gc[i][2];
            gam[i][a] = c_modes[a][i] - dot;
        }
    }
    // Isotropic stabilisation matrix with E_hg = hourglass * E (material.rs:662).
    const double ehg = hourglass * youngs;
    const double lam = ehg * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double mu = ehg / (2.0 * (1.0 + nu));
    // G K Gᵀ accumulated per Gauss point as Mᵀ C M with M = (B_gp - B_c) Gᵀ (6 x 12).
    double gkg[12][12];
    for (int r = 0; r < 12; ++r)
        for (int c = 0; c < 12; ++c) gkg[r][c] = 0.0;
    double mass[8][8];
    for (int i = 0; i < 8; ++i)
        for (int j = 0; j < 8; ++j) mass[i][j] = 0.0;
    double volume = 0.0;
    const double GAUSS = 0.5773502691896258;
    for (int q = 0; q < 8; ++q) {
        double xi = c_xi[q][0] * GAUSS, eta = c_xi[q][1] * GAUSS, zeta = c_xi[q][2] * GAUSS;
        double dn[8][3], gq[8][3], detj;
        shape_derivatives(xi, eta, zeta, dn);
        if (!reference_gradients(x, dn, gq, &detj)) {
            atomicExch(bad, 1);
            return;
        }
        // P[b][d] = Σ_j γ_jb (g_q - g_c)_jd
        double pm[4][3];
        for (int b = 0; b < 4; ++b)
            for (int d = 0; d < 3; ++d) {
                double s = 0.0;
                for (int j = 0; j < 8; ++j) s += gam[j][b] * (gq[j][d] - gc[j][d]);
                pm[b][d] = s;
            }
        // M rows (Voigt xx, yy, zz, xy, yz, xz; engineering shear) over columns 3b + e.
        double m[6][12];
        for (int s = 0; s < 6; ++s)
            for (int c = 0; c < 12; ++c) m[s][c] = 0.0;
        for (int b = 0; b < 4; ++b) {
            m[0][3 * b + 0] = pm[b][0];
            m[1][3 * b + 1] = pm[b][1];
            m[2][3 * b + 2] = pm[b][2];
            m[3][3 * b + 0] = pm[b][1];
            m[3][3 * b + 1] = pm[b][0];
            m[4][3 * b + 1] = pm[b][2];
            m[4][3 * b + 2] = pm[b][1];
            m[5][3 * b + 0] = pm[b][2];
            m[5][3 * b + 2] = pm[b][0];
        }
        // C M (normal block lam/lam+2mu, shear block mu).
        double cm[6][12];
        for (int c = 0; c < 12; ++c) {
            double t0 = m[0][c], t1 = m[1][c], t2 = m[2][c];
            cm[0][c] = (lam + 2.0 * mu) * t0 + lam * t1 + lam * t2;
            cm[1][c] = lam * t0 + (lam + 2.0 * mu) * t1 + lam * t2;
            cm[2][c] = lam * t0 + lam * t1 + (lam + 2.0 * mu) * t2;
            cm[3][c] = mu * m[3][c];
            cm[4][c] = mu * m[4][c];
            cm[5][c] = mu * m[5][c];
        }
        for (int r = 0; r < 12; ++r)
            for (int c = r; c < 12; ++c) {
                double s = 0.0;
                for (int t = 0; t < 6; ++t) s += m[t][r] * cm[t][c];
                gkg[r][c] += s * detj;
            }
        volume += detj;
        // Consistent mass rows, as src/element.rs:156-157 accumulates them.
        double nq[8];
        for (int i = 0; i < 8; ++i)
            nq[i] = 0.125 * (1.0 + c_xi[i][0] * xi) * (1.0 + c_xi[i][1] * eta) * (1.0 + c_xi[i][2] * zeta);
        for (int i = 0; i < 8; ++i)
            for (int j = 0; j < 8; ++j) mass[i][j] += rho * nq[i] * nq[j] * detj;
    }
    volume_out[e] = volume;
    elem_mass[e] = volume * rho;
    for (int i = 0; i < 8; ++i) {
        double s = 0.0;
        for (int j = 0; j < 8; ++j) s += mass[i][j];
        lumped_out[8 * e + i] = s;
    }
    {
        // Material::dilatational_wave_speed, src/material.rs:226; kernel.rs:73.
        double mm = youngs * (1.0 - nu) / ((1.0 + nu) * (1.0 - 2.0 * nu));
        dt_factor[e] = (1.0 - 0.36 * nu) / sqrt(mm / rho);
    }
    const long long h = hc_index[e];
    if (h < 0) return;
    // A = (ΓᵀΓ)⁻¹ (GGᵀ = A⁻¹ ⊗ I3), by Gauss-Jordan with partial pivoting on 4x4.
    double a[4][8];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            double s = 0.0;
            for (int i = 0; i < 8; ++i) s += gam[i][r] * gam[i][c];
            a[r][c] = s;
            a[r][4 + c] = (r == c) ? 1.0 : 0.0;
        }
    for (int k = 0; k < 4; ++k) {
        int pv = k;
        for (int r = k + 1; r < 4; ++r)
            if (fabs(a[r][k]) > fabs(a[pv][k])) pv = r;
        if (a[pv][k] == 0.0) {
            atomicExch(bad, 2);
            return;
        }
        if (pv != k)
            for (int c = 0; c < 8; ++c) {
                double t = a[k][c];
                a[k][c] = a[pv][c];
                a[pv][c] = t;
            }
        double piv = a[k][k];
        for (int c = 0; c < 8; ++c) a[k][c] /= piv;
        for (int r = 0; r < 4; ++r)
            if (r != k) {
                double f = a[r][k];
                for (int c = 0; c < 8; ++c) a[r][c] -= f * a[k][c];
            }
    }
    // H[(a,d),(b,e)] = Σ A[a][a'] GKG[(a',d),(b',e)] A[b'][b] (upper triangle).
    float hs[80];
    for (int k = 78; k < 80; ++k) hs[k] = 0.0f;
    for (int r = 0; r < 12; ++r)
        for (int c = r; c < 12; ++c) {
            const int ar = r / 3, dr = r % 3, bc = c / 3, ec = c % 3;
            double s = 0.0;
            for (int a1 = 0; a1 < 4; ++a1)
                for (int b1 = 0; b1 < 4; ++b1) {
                    int rr = 3 * a1 + dr, cc = 3 * b1 + ec;
                    double g = rr <= cc ? gkg[rr][cc] : gkg[cc][rr];
                    s += a[ar][4 + a1] * g * a[b1][4 + bc];
                }
            hs[h_index(r, c)] = (float)s;
        }
    float4* pl = planes;
    pl[(P_CONN + 0) * stride + h] = make_float4(__uint_as_float(nid[0]), __uint_as_float(nid[1]), __uint_as_float(nid[2]), __uint_as_float(nid[3]));
    pl[(P_CONN + 1) * stride + h] = make_float4(__uint_as_float(nid[4]), __uint_as_float(nid[5]), __uint_as_float(nid[6]), __uint_as_float(nid[7]));
    float gf[24];
    for (int i = 0; i < 8; ++i)
        for (int d = 0; d < 3; ++d) gf[3 * i + d] = (float)gc[i][d];
    for (int k = 0; k < 6; ++k) pl[(P_GRAD + k) * stride + h] = make_float4(gf[4 * k], gf[4 * k + 1], gf[4 * k + 2], gf[4 * k + 3]);
    float gm[32];
    for (int i = 0; i < 8; ++i)
        for (int aa = 0; aa < 4; ++aa) gm[4 * i + aa] = (float)gam[i][aa];
    for (int k = 0; k < 8; ++k) pl[(P_GAMMA + k) * stride + h] = make_float4(gm[4 * k], gm[4 * k + 1], gm[4 * k + 2], gm[4 * k + 3]);
    for (int k = 0; k < 20; ++k) pl[(P_H + k) * stride + h] = make_float4(hs[4 * k], hs[4 * k + 1], hs[4 * k + 2], hs[4 * k + 3]);
    pl[P_META * stride + h] = make_float4((float)volume, __uint_as_float((uint32_t)p), __uint_as_float((uint32_t)e), 0.0f);
}

// Lumped nodal masses: Σ over incident (element, corner) in element order
// (src/model.rs:268-278), and 1/m.
__global__ void k_node_masses(long long n, const uint32_t* __restrict__ off, const uint32_t* __restrict__ slot,
                              const double* __restrict__ lumped, double* __restrict__ mass, double* __restrict__ inv_mass) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double m = 0.0;
    for (uint32_t k = off[i]; k < off[i + 1]; ++k) m += lumped[slot[k]];
    mass[i] = m;
    inv_mass[i] = m > 0.0 ? 1.0 / m : 0.0;
}

__global__ void k_init_state(long long n_hc, long long stride, float4* __restrict__ st) {
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_hc) return;
    // identity F_prev⁻¹ (0-8), identity R (9-17), zero stress, compaction, not eroded.
    const float v[28] = {1, 0, 0, 0, 1, 0, 0, 0, 1, 1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = 0; k < N_STATE_PLANES; ++k) st[k * stride + e] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
}

// ---------------------------------------------------------------------------
// Element forces (src/kernel_simd.rs:300-491, one element per thread).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(TPB) k_forces(ElementArrays el, NodeArrays nd, Control* ctl, int respect_done) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (respect_done && ctl->done) return;
    if (e >= el.n_hc) return;
    const long long S = el.stride;
    float4* out = reinterpret_cast<float4*>(el.corner + 24 * e);
    const float4 st6 = el.state[6 * S + e];
    if (__float_as_uint(st6.y) != 0u) {  // already eroded: no force
        for (int k = 0; k < 6; ++k) out[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    const float4 c0 = ld_plane(el.planes, S, P_CONN, e), c1 = ld_plane(el.planes, S, P_CONN + 1, e);
    const uint32_t nid[8] = {__float_as_uint(c0.x), __float_as_uint(c0.y), __float_as_uint(c0.z), __float_as_uint(c0.w),
                             __float_as_uint(c1.x), __float_as_uint(c1.y), __float_as_uint(c1.z), __float_as_uint(c1.w)};
    float grad[24];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        float4 g = ld_plane(el.planes, S, P_GRAD + k, e);
        grad[4 * k] = g.x; grad[4 * k + 1] = g.y; grad[4 * k + 2] = g.z; grad[4 * k + 3] = g.w;
    }
    float gam[32];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float4 g = ld_plane(el.planes, S, P_GAMMA + k, e);
        gam[4 * k] = g.x; gam[4 * k + 1] = g.y; gam[4 * k + 2] = g.z; gam[4 * k + 3] = g.w;
    }
    // F = Σ x_i ⊗ ∇N_i with x = (X + u) as f32; q = U Γ with u as f32.
    M3f f;
#pragma unroll
    for (int k = 0; k < 9; ++k) f.m[k] = 0.0f;
    float q[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) q[k] = 0.0f;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const long long n = nid[i];
        const double* P = nd.pos + 3 * n;
        const double* U = nd.u + 3 * n;
        const double u0 = U[0], u1 = U[1], u2 = U[2];
        const float x[3] = {(float)(__ldg(P) + u0), (float)(__ldg(P + 1) + u1), (float)(__ldg(P + 2) + u2)};
        const float ul[3] = {(float)u0, (float)u1, (float)u2};
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int c = 0; c < 3; ++c) f.m[3 * a + c] = x[a] * grad[3 * i + c] + f.m[3 * a + c];
#pragma unroll
        for (int mode = 0; mode < 4; ++mode)
#pragma unroll
            for (int dir = 0; dir < 3; ++dir) q[3 * mode + dir] = ul[dir] * gam[4 * i + mode] + q[3 * mode + dir];
    }
    const float det = det3(f);
    if (det <= 0.0f) {  // inverted: erode (src/kernel_simd.rs:324-331)
        el.state[6 * S + e] = make_float4(st6.x, __uint_as_float(1u), st6.z, st6.w);
        const uint32_t model_e = __float_as_uint(ld_plane(el.planes, S, P_META, e).z);
        el.eroded_all[model_e] = 1;
        atomicAdd(reinterpret_cast<unsigned long long*>(&ctl->eroded_step), 1ull);
        for (int k = 0; k < 6; ++k) out[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    float st[28];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        float4 s4 = el.state[k * S + e];
        st[4 * k] = s4.x; st[4 * k + 1] = s4.y; st[4 * k + 2] = s4.z; st[4 * k + 3] = s4.w;
    }
    st[24] = st6.x; st[25] = st6.y; st[26] = st6.z; st[27] = st6.w;
    const float4 meta = ld_plane(el.planes, S, P_META, e);
    const MaterialF32& mat = el.mats[__float_as_uint(meta.y)];
    M3f tau, f_inv;
    honeycomb_update(f, det, st, mat, tau, f_inv);
#pragma unroll
    for (int k = 0; k < 7; ++k) el.state[k * S + e] = make_float4(st[4 * k], st[4 * k + 1], st[4 * k + 2], st[4 * k + 3]);
    // f_i = τ F⁻ᵀ ∇N_i V₀
    M3f m;
    mat_mul_t(tau, f_inv, m);
    const float vol = meta.x;
#pragma unroll
    for (int k = 0; k < 9; ++k) m.m[k] = m.m[k] * vol;
    float fo[24];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            float acc = m.m[3 * a] * grad[3 * i];
            acc = m.m[3 * a + 1] * grad[3 * i + 1] + acc;
            acc = m.m[3 * a + 2] * grad[3 * i + 2] + acc;
            fo[3 * i + a] = acc;
        }
    // Hourglass: rr = H q (column order), f += rr Γᵀ.
    float hsym[80];
#pragma unroll
    for (int k = 0; k < 20; ++k) {
        float4 h4 = ld_plane(el.planes, S, P_H + k, e);
        hsym[4 * k] = h4.x; hsym[4 * k + 1] = h4.y; hsym[4 * k + 2] = h4.z; hsym[4 * k + 3] = h4.w;
    }
    float rr[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) rr[k] = 0.0f;
#pragma unroll
    for (int col = 0; col < 12; ++col)
#pragma unroll
        for (int row = 0; row < 12; ++row) rr[row] = hsym[h_index(row, col)] * q[col] + rr[row];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int dir = 0; dir < 3; ++dir) {
            float acc = fo[3 * i + dir];
#pragma unroll
            for (int mode = 0; mode < 4; ++mode) acc = rr[3 * mode + dir] * gam[4 * i + mode] + acc;
            fo[3 * i + dir] = acc;
        }
#pragma unroll
    for (int k = 0; k < 6; ++k) out[k] = make_float4(fo[4 * k], fo[4 * k + 1], fo[4 * k + 2], fo[4 * k + 3]);
}

// Nodal internal force: ordered f64 sum of incident corner forces.
__device__ __forceinline__ void gather_node(const NodeArrays& nd, const float* __restrict__ corner, long long n,
                                            double& fx, double& fy, double& fz) {
    fx = 0.0; fy = 0.0; fz = 0.0;
    const uint32_t b = nd.hc_off[n], en = nd.hc_off[n + 1];
    for (uint32_t k = b; k < en; ++k) {
        const uint32_t s = __ldg(nd.hc_slot + k);
        const float* c = corner + 3ull * s;  // slot = 8 e + corner -> 24 e + 3 corner
        fx += (double)__ldg(c);
        fy += (double)__ldg(c + 1);
        fz += (double)__ldg(c + 2);
    }
}

__global__ void k_gather(ElementArrays el, NodeArrays nd, double* __restrict__ f_out) {
    long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nd.n) return;
    double fx, fy, fz;
    gather_node(nd, el.corner, n, fx, fy, fz);
    f_out[3 * n] = fx;
    f_out[3 * n + 1] = fy;
    f_out[3 * n + 2] = fz;
}

// Half step: v½ = v + ½dt (f_ext - f_int)/m ; u += dt v½ ; fixed -> 0 (src/solver.rs:314-323).
__global__ void k_half(NodeArrays nd, Control* ctl) {
    long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nd.n || ctl->done) return;
    const double dt = step_dt(ctl);
    const double im = nd.inv_mass[n];
    const bool fixed = nd.fixed[n] != 0;
    for (int d = 0; d < 3; ++d) {
        const long long k = 3 * n + d;
        const double a = (nd.f_ext[k] - nd.f_int[k]) * im;
        double vh = nd.v[k] + 0.5 * dt * a;
        double u = nd.u[k] + dt * vh;
        if (fixed) {
            u = 0.0;
            vh = 0.0;
            nd.v[k] = 0.0;
        }
        nd.v_half[k] = vh;
        nd.u[k] = u;
    }
}

// Full step with the fused force gather: v = (v½ + ½dt a) damping (src/solver.rs:334-342).
__global__ void k_full(ElementArrays el, NodeArrays nd, Control* ctl) {
    long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nd.n || ctl->done) return;
    const double dt = step_dt(ctl);
    double f[3];
    gather_node(nd, el.corner, n, f[0], f[1], f[2]);
    const double im = nd.inv_mass[n];
    const bool fixed = nd.fixed[n] != 0;
    const double damping = ctl->damping;
    for (int d = 0; d < 3; ++d) {
        const long long k = 3 * n + d;
        const double a = (nd.f_ext[k] - f[d]) * im;
        double v = (nd.v_half[k] + 0.5 * dt * a) * damping;
        nd.v[k] = fixed ? 0.0 : v;
        nd.f_int[k] = f[d];
    }
}

// ---------------------------------------------------------------------------
// Stable time step (src/kernel.rs:207-237, src/element.rs:176-186) and the
// per-element added mass of selective mass scaling (src/kernel.rs:243-258).
// ---------------------------------------------------------------------------
__device__ void char_length_and_volume(const double p[8][3], double* l, double* vol_out) {
    const int TETS[6][4] = {{0, 1, 2, 6}, {0, 2, 3, 6}, {0, 3, 7, 6}, {0, 7, 4, 6}, {0, 4, 5, 6}, {0, 5, 1, 6}};
    const int FACES[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}};
    double vol = 0.0;
#pragma unroll
    for (int t = 0; t < 6; ++t) {
        const double* a = p[TETS[t][0]];
        double e1[3], e2[3], e3[3];
        for (int d = 0; d < 3; ++d) {
            e1[d] = p[TETS[t][1]][d] - a[d];
            e2[d] = p[TETS[t][2]][d] - a[d];
            e3[d] = p[TETS[t][3]][d] - a[d];
        }
        double cx = e1[1] * e2[2] - e1[2] * e2[1];
        double cy = e1[2] * e2[0] - e1[0] * e2[2];
        double cz = e1[0] * e2[1] - e1[1] * e2[0];
        vol = vol + (cx * e3[0] + cy * e3[1] + cz * e3[2]) / 6.0;
    }
    double a_max = 0.0;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        double d1[3], d2[3];
        for (int d = 0; d < 3; ++d) {
            d1[d] = p[FACES[f][2]][d] - p[FACES[f][0]][d];
            d2[d] = p[FACES[f][3]][d] - p[FACES[f][1]][d];
        }
        double cx = d1[1] * d2[2] - d1[2] * d2[1];
        double cy = d1[2] * d2[0] - d1[0] * d2[2];
        double cz = d1[0] * d2[1] - d1[1] * d2[0];
        double a = 0.5 * sqrt(cx * cx + cy * cy + cz * cz);
        a_max = fmax(a_max, a);
    }
    *vol_out = vol;
    *l = (vol <= 0.0 || a_max <= 0.0) ? CUDART_INF : vol / a_max;
}

constexpr int DT_TPB = 256;

__global__ void __launch_bounds__(DT_TPB) k_elem_dt(ElementArrays el, NodeArrays nd, Control* ctl, const double* __restrict__ u,
                                                    double* __restrict__ partials, int respect_done) {
    __shared__ double s_min[DT_TPB];
    __shared__ double s_sum[DT_TPB];
    if (respect_done && ctl->done) return;
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double dt = CUDART_INF, extra = 0.0;
    if (e < el.n_all) {
        if (!el.eroded_all[e]) {
            double p[8][3];
            for (int i = 0; i < 8; ++i) {
                long long n = el.conn_all[8 * e + i];
                for (int d = 0; d < 3; ++d) p[i][d] = nd.pos[3 * n + d] + u[3 * n + d];
            }
            double l, vol;
            char_length_and_volume(p, &l, &vol);
            if (isfinite(l) && vol > 0.0) dt = l * el.dt_factor[e];
        }
        const double floor = ctl->dt_floor;
        if (dt < floor) {
            double r = floor / dt;
            extra = (fmin(r * r, 100.0) - 1.0) * el.elem_mass[e];
        }
        el.elem_dt[e] = dt;
        el.elem_extra[e] = extra;
    }
    s_min[threadIdx.x] = dt;
    s_sum[threadIdx.x] = extra;
    __syncthreads();
    for (int w = DT_TPB / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            s_min[threadIdx.x] = fmin(s_min[threadIdx.x], s_min[threadIdx.x + w]);
            s_sum[threadIdx.x] = s_sum[threadIdx.x] + s_sum[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        atomicMin(&ctl->dt_stable_bits, (unsigned long long)__double_as_longlong(s_min[0]));
        partials[blockIdx.x] = s_sum[0];
    }
}

// The adaptive step decision of src/solver.rs:288-299 (one thread).
__global__ void k_dt_finalize(Control* ctl, const double* __restrict__ partials, int n_blocks) {
    if (ctl->done) return;
    const double dt_stable = __longlong_as_double((long long)ctl->dt_stable_bits);
    ctl->dt_stable_bits = (unsigned long long)__double_as_longlong(CUDART_INF);
    if (!isfinite(dt_stable)) return;
    double dt_use = dt_stable;
    if (ctl->dt_floor > 0.0 && dt_stable < ctl->dt_floor) {
        double total = 0.0;
        for (int b = 0; b < n_blocks; ++b) total += partials[b];
        ctl->mass_scale_now = 1;
        ctl->added_total = total;
        ctl->added_mass_max = fmax(ctl->added_mass_max, total);
        dt_use = ctl->dt_floor;
    }
    ctl->dt_cfl = ctl->dt_scale * fmin(dt_use, ctl->contact_dt);
}

// Added nodal mass (element order, src/kernel.rs:246-255) and 1/(m + added).
__global__ void k_mass_scaling(ElementArrays el, NodeArrays nd, Control* ctl, int force_apply) {
    long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nd.n) return;
    if (!force_apply && (ctl->done || !ctl->mass_scale_now)) return;
    const double floor = ctl->dt_floor;
    double add = 0.0;
    for (uint32_t k = nd.all_off[n]; k < nd.all_off[n + 1]; ++k) {
        uint32_t e = nd.all_slot[k] >> 3;
        if (el.elem_dt[e] < floor) add += el.elem_extra[e] / 8.0;
    }
    nd.added[n] = add;
    const double m = nd.mass[n] + add;
    nd.inv_mass[n] = m > 0.0 ? 1.0 / m : 0.0;
}

__global__ void k_nonfinite(NodeArrays nd, Control* ctl) {
    long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 3 * nd.n || ctl->done) return;
    if (!isfinite(nd.u[k])) ctl->nonfinite = 1;
}

// End of a step (src/solver.rs:344-345 plus the stop rules).
__global__ void k_step_end(Control* ctl, ContactArrays ca, int check_separation) {
    if (ctl->done) return;
    const double dt = step_dt(ctl);
    ctl->step += 1;
    ctl->t = ctl->t + dt;
    ctl->dt_min = fmin(ctl->dt_min, dt);
    ctl->eroded_total += ctl->eroded_step;
    ctl->eroded_step = 0;
    ctl->mass_scale_now = 0;
    int hit = 0;
    for (int c = 0; c < ca.n_contacts; ++c) {
        if (ca.counts_for_stop[c] && ca.pen_count[c] > 0) hit = 1;
        ca.pen_count[c] = 0;
        ca.pen_max_bits[c] = 0;
    }
    if (hit) ctl->last_hit = ctl->step - 1;
    if (ctl->nonfinite) {
        ctl->done = 1;
        ctl->status = -2;  // CRUSH_ERR_NONFINITE
        return;
    }
    if (ctl->max_steps > 0 && ctl->step >= ctl->max_steps) ctl->done = 1;
    if (!(ctl->t < ctl->end_time)) ctl->done = 1;
    if (check_separation && ctl->stop_rule == 1 && ctl->step % 10 == 0 && ctl->last_hit >= 0 &&
        ctl->step - 1 - ctl->last_hit >= 100 && ctl->vx[1] - ctl->vx[0] >= 0.0)
        ctl->done = 1;
}

// ---------------------------------------------------------------------------
// Node-to-face penalty contact (src/contact.rs:92-160): face geometry and a
// hashed uniform grid rebuilt every step, first-hit (minimum face index)
// search per primary node, and an ordered gather of the reactions.
// ---------------------------------------------------------------------------
constexpr int MAX_CELLS_PER_FACE = 64;

__device__ __forceinline__ int contact_of(const int* off, int n_contacts, long long i) {
    int c = 0;
    while (c + 1 < n_contacts && i >= off[c + 1]) ++c;
    return c;
}
__device__ __forceinline__ unsigned cell_hash(long long i, long long j, long long k) {
    unsigned long long h = (unsigned long long)i * 73856093ull ^ (unsigned long long)j * 19349663ull ^
                           (unsigned long long)k * 83492791ull;
    return (unsigned)(h ^ (h >> 29));
}

// Grid cells covered by a face's expanded box. False (the face goes to the
// contact's overflow list) when the box is not finite or spans more than
// MAX_CELLS_PER_FACE cells; each axis range is checked before any product,
// so a loop over the returned range is always short.
__device__ __forceinline__ bool face_cells(const FaceGeo& g, double cs, long long* i0, long long* i1, long long* j0,
                                           long long* j1, long long* k0, long long* k1) {
    for (int d = 0; d < 3; ++d)
        if (!isfinite(g.lo[d]) || !isfinite(g.hi[d]) || !(g.lo[d] <= g.hi[d])) return false;
    const double lim = 4.0e15;  // cell coordinates stay exact in f64 and far from long long overflow
    double a0 = floor(g.lo[0] / cs), a1 = floor(g.hi[0] / cs);
    double b0 = floor(g.lo[1] / cs), b1 = floor(g.hi[1] / cs);
    double c0 = floor(g.lo[2] / cs), c1 = floor(g.hi[2] / cs);
    if (fabs(a0) > lim || fabs(a1) > lim || fabs(b0) > lim || fabs(b1) > lim || fabs(c0) > lim || fabs(c1) > lim) return false;
    const double da = a1 - a0, db = b1 - b0, dc = c1 - c0;
    if (da < 0.0 || db < 0.0 || dc < 0.0 || da >= MAX_CELLS_PER_FACE || db >= MAX_CELLS_PER_FACE || dc >= MAX_CELLS_PER_FACE) return false;
    if ((da + 1.0) * (db + 1.0) * (dc + 1.0) > MAX_CELLS_PER_FACE) return false;
    *i0 = (long long)a0; *i1 = (long long)a1;
    *j0 = (long long)b0; *j1 = (long long)b1;
    *k0 = (long long)c0; *k1 = (long long)c1;
    return true;
}

// Cell of a point (any finite coordinates; non-finite points map to cell 0).
__device__ __forceinline__ unsigned point_cell_hash(const double* p, double cs) {
    long long q[3];
    for (int d = 0; d < 3; ++d) {
        double a = floor(p[d] / cs);
        q[d] = (isfinite(a) && fabs(a) <= 4.0e15) ? (long long)a : 0;
    }
    return cell_hash(q[0], q[1], q[2]);
}

__global__ void k_contact_faces(ContactArrays ca, NodeArrays nd, Control* ctl, int c0, int c1, int run_mode) {
    long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (run_mode && ctl->done) return;
    const long long f_begin = ca.face_off[c0], f_end = ca.face_off[c1];
    f += f_begin;
    if (f >= f_end) return;
    const int c = contact_of(ca.face_off, ca.n_contacts, f);
    FaceGeo g;
    for (int k = 0; k < 4; ++k) {
        long long n = ca.faces[4 * f + k];
        for (int d = 0; d < 3; ++d) g.x[k][d] = nd.pos[3 * n + d] + nd.u[3 * n + d];
    }
    double e1[3], e2[3];
    for (int d = 0; d < 3; ++d) {
        e1[d] = g.x[1][d] - g.x[0][d];
        e2[d] = g.x[2][d] - g.x[0][d];
    }
    double nx = e1[1] * e2[2] - e1[2] * e2[1];
    double ny = e1[2] * e2[0] - e1[0] * e2[2];
    double nz = e1[0] * e2[1] - e1[1] * e2[0];
    double len = sqrt(nx * nx + ny * ny + nz * nz);
    g.n[0] = nx / len; g.n[1] = ny / len; g.n[2] = nz / len;
    const double md = ca.max_distance[c];
    for (int d = 0; d < 3; ++d) {
        g.c[d] = (((g.x[0][d] + g.x[1][d]) + g.x[2][d]) + g.x[3][d]) / 4.0;
        double lo = g.x[0][d], hi = g.x[0][d];
        for (int k = 1; k < 4; ++k) {
            lo = fmin(lo, g.x[k][d]);
            hi = fmax(hi, g.x[k][d]);
        }
        g.lo[d] = lo + -md;
        g.hi[d] = hi + md;
    }
    ca.geo[f] = g;
    const double cs = ca.cell[c];
    long long i0, i1, j0, j1, k0, k1;
    const int local = (int)(f - ca.face_off[c]);
    if (!face_cells(g, cs, &i0, &i1, &j0, &j1, &k0, &k1)) {
        int slot = atomicAdd(&ca.n_overflow[c], 1);
        if (slot < ca.overflow_cap) ca.overflow[(long long)c * ca.overflow_cap + slot] = local;
        return;
    }
    const int tab = ca.tab_off[c];
    const unsigned mask = (unsigned)(ca.tab_off[c + 1] - tab - 1);
    for (long long i = i0; i <= i1; ++i)
        for (long long j = j0; j <= j1; ++j)
            for (long long k = k0; k <= k1; ++k) atomicAdd(&ca.counts[tab + (cell_hash(i, j, k) & mask)], 1);
}

// Exclusive scan of the grid counts of contacts [c0, c1) (one block).
__global__ void __launch_bounds__(1024) k_contact_scan(ContactArrays ca, Control* ctl, int c0, int c1, int run_mode) {
    __shared__ int s_part[1024];
    if (run_mode && ctl->done) return;
    const int begin = ca.tab_off[c0], end = ca.tab_off[c1];
    const int n = end - begin;
    const int per = (n + blockDim.x - 1) / blockDim.x;
    const int lo = begin + threadIdx.x * per;
    const int hi = min(lo + per, end);
    int sum = 0;
    for (int i = lo; i < hi; ++i) sum += ca.counts[i];
    s_part[threadIdx.x] = sum;
    __syncthreads();
    for (int w = 1; w < (int)blockDim.x; w <<= 1) {
        int v = threadIdx.x >= (unsigned)w ? s_part[threadIdx.x - w] : 0;
        __syncthreads();
        s_part[threadIdx.x] += v;
        __syncthreads();
    }
    int run = s_part[threadIdx.x] - sum;
    for (int i = lo; i < hi; ++i) {
        int cnt = ca.counts[i];
        ca.starts[i] = run;
        ca.counts[i] = 0;
        run += cnt;
    }
}

__global__ void k_contact_fill(ContactArrays ca, Control* ctl, int c0, int c1, int run_mode, int entries_cap) {
    long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (run_mode && ctl->done) return;
    const long long f_begin = ca.face_off[c0], f_end = ca.face_off[c1];
    f += f_begin;
    if (f >= f_end) return;
    const int c = contact_of(ca.face_off, ca.n_contacts, f);
    const FaceGeo& g = ca.geo[f];
    const double cs = ca.cell[c];
    long long i0, i1, j0, j1, k0, k1;
    if (!face_cells(g, cs, &i0, &i1, &j0, &j1, &k0, &k1)) return;
    const int local = (int)(f - ca.face_off[c]);
    const int tab = ca.tab_off[c];
    const unsigned mask = (unsigned)(ca.tab_off[c + 1] - tab - 1);
    for (long long i = i0; i <= i1; ++i)
        for (long long j = j0; j <= j1; ++j)
            for (long long k = k0; k <= k1; ++k) {
                const int b = tab + (int)(cell_hash(i, j, k) & mask);
                const int pos = ca.starts[b] + atomicAdd(&ca.counts[b], 1);
                if (pos < entries_cap) ca.entries[pos] = local;
                else ca.entry_overrun[c] = 1;
            }
}

// src/contact.rs:29-43
__device__ __forceinline__ bool point_in_triangle(const double* p, const double* a, const double* b, const double* c) {
    const double tol = 0.1;
    double v0[3], v1[3], v2[3];
    for (int d = 0; d < 3; ++d) {
        v0[d] = c[d] - a[d];
        v1[d] = b[d] - a[d];
        v2[d] = p[d] - a[d];
    }
    double d00 = v0[0] * v0[0] + v0[1] * v0[1] + v0[2] * v0[2];
    double d01 = v0[0] * v1[0] + v0[1] * v1[1] + v0[2] * v1[2];
    double d02 = v0[0] * v2[0] + v0[1] * v2[1] + v0[2] * v2[2];
    double d11 = v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2];
    double d12 = v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2];
    double inv = 1.0 / (d00 * d11 - d01 * d01);
    double uu = (d11 * d02 - d01 * d12) * inv;
    double vv = (d00 * d12 - d01 * d02) * inv;
    return uu >= -tol && vv >= -tol && uu + vv <= 1.0 + tol;
}

// The narrow test of one face for one point; returns the signed distance in *sd.
__device__ __forceinline__ bool face_hit(const FaceGeo& g, const double* p, double md, double* sd) {
    if (p[0] < g.lo[0] || p[0] > g.hi[0] || p[1] < g.lo[1] || p[1] > g.hi[1] || p[2] < g.lo[2] || p[2] > g.hi[2])
        return false;
    double dc0 = g.c[0] - p[0], dc1 = g.c[1] - p[1], dc2 = g.c[2] - p[2];
    double signed_d = -(g.n[0] * dc0 + g.n[1] * dc1 + g.n[2] * dc2);
    if (signed_d > 0.0 || signed_d < -md) return false;
    double proj[3] = {p[0] - g.n[0] * signed_d, p[1] - g.n[1] * signed_d, p[2] - g.n[2] * signed_d};
    bool inside = point_in_triangle(proj, g.x[0], g.x[1], g.x[2]) || point_in_triangle(proj, g.x[0], g.x[2], g.x[3]) ||
                  point_in_triangle(proj, g.x[1], g.x[2], g.x[3]) || point_in_triangle(proj, g.x[1], g.x[3], g.x[0]);
    *sd = signed_d;
    return inside;
}

__global__ void k_contact_slaves(ContactArrays ca, NodeArrays nd, Control* ctl, int c0, int c1, int run_mode, double dt_override,
                                 const double* __restrict__ masses, int entries_cap) {
    long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (run_mode && ctl->done) return;
    const long long s_begin = ca.slave_off[c0], s_end = ca.slave_off[c1];
    s += s_begin;
    if (s >= s_end) return;
    const int c = contact_of(ca.slave_off, ca.n_contacts, s);
    const long long n = ca.slaves[s];
    const double p[3] = {nd.pos[3 * n] + nd.u[3 * n], nd.pos[3 * n + 1] + nd.u[3 * n + 1], nd.pos[3 * n + 2] + nd.u[3 * n + 2]};
    const double md = ca.max_distance[c];
    const long long fb = ca.face_off[c];
    const FaceGeo* geo = ca.geo + fb;
    int best = INT_MAX;
    double best_sd = 0.0, sd;
    if (ca.entry_overrun[c]) {
        const int nf = (int)(ca.face_off[c + 1] - fb);
        for (int f = 0; f < nf; ++f)
            if (face_hit(geo[f], p, md, &sd)) { best = f; best_sd = sd; break; }
    } else {
        const double cs = ca.cell[c];
        const int tab = ca.tab_off[c];
        const unsigned mask = (unsigned)(ca.tab_off[c + 1] - tab - 1);
        const int b = tab + (int)(point_cell_hash(p, cs) & mask);
        const int e0 = ca.starts[b], e1 = e0 + ca.counts[b];
        for (int k = e0; k < e1 && k < entries_cap; ++k) {
            const int f = ca.entries[k];
            if (f < best && face_hit(geo[f], p, md, &sd)) { best = f; best_sd = sd; }
        }
        const int no = min(ca.n_overflow[c], ca.overflow_cap);
        for (int k = 0; k < no; ++k) {
            const int f = ca.overflow[(long long)c * ca.overflow_cap + k];
            if (f < best && face_hit(geo[f], p, md, &sd)) { best = f; best_sd = sd; }
        }
    }
    if (best == INT_MAX) {
        ca.hit[s] = -1;
        return;
    }
    const double dt = dt_override > 0.0 ? dt_override : step_dt(ctl);
    const double m = masses[n];
    const double depth = fmin(-best_sd, 0.1 * md);
    const double k_pen = fmin(ca.stiffness[c] * ca.slave_scale[s], 0.1 * m / (dt * dt));
    const double mag = fmin(k_pen * depth, m * 1.0e5);
    const FaceGeo& g = geo[best];
    ca.hit[s] = best;
    ca.hit_force[3 * s] = mag * g.n[0];
    ca.hit_force[3 * s + 1] = mag * g.n[1];
    ca.hit_force[3 * s + 2] = mag * g.n[2];
    atomicAdd(&ca.pen_count[c], 1ull);
    atomicMax(&ca.pen_max_bits[c], (unsigned long long)__double_as_longlong(-best_sd));
}

// Ordered reaction gather: one warp per contact node walks its contacts in
// order and, within each, the primary nodes in order, adding +F for its own
// hit and -F/4 for every hit on a face it belongs to — the sequence in which
// src/contact.rs:146-153 adds them. Also clears the grid counts.
__global__ void k_contact_gather(ContactArrays ca, NodeArrays nd, Control* ctl, int c0, int c1, int run_mode,
                                 double* __restrict__ f_out, int skip_fixed) {
    if (run_mode && ctl->done) return;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp < ca.n_cnodes) {
        const long long n = ca.cnode[warp];
        if (!(skip_fixed && nd.fixed[n])) {
            double sx = 0.0, sy = 0.0, sz = 0.0;
            bool touched = false;
            for (uint32_t r = ca.cnode_off[warp]; r < ca.cnode_off[warp + 1]; ++r) {
                const int c = ca.crole_contact[r];
                if (c < c0 || c >= c1) continue;
                touched = true;
                const long long sb = ca.slave_off[c], se = ca.slave_off[c + 1];
                const int own = ca.crole_slave[r];
                if (!ca.crole_face[r]) {
                    if (own >= 0 && ca.hit[sb + own] >= 0) {
                        sx += ca.hit_force[3 * (sb + own)];
                        sy += ca.hit_force[3 * (sb + own) + 1];
                        sz += ca.hit_force[3 * (sb + own) + 2];
                    }
                    continue;
                }
                const uint32_t* faces = ca.faces + 4 * ca.face_off[c];
                for (long long base = sb; base < se; base += 32) {
                    const long long s = base + lane;
                    int flags = 0;
                    if (s < se) {
                        const int h = ca.hit[s];
                        if (h >= 0) {
                            if (s - sb == own) flags |= 1;
                            const uint32_t* q = faces + 4 * (long long)h;
                            if (q[0] == n || q[1] == n || q[2] == n || q[3] == n) flags |= 2;
                        }
                    }
                    unsigned mask = __ballot_sync(0xffffffffu, flags != 0);
                    while (mask) {
                        const int l = __ffs(mask) - 1;
                        mask &= mask - 1;
                        const int fl = __shfl_sync(0xffffffffu, flags, l);
                        const long long ss = base + l;
                        if (lane == 0) {
                            const double fx = ca.hit_force[3 * ss], fy = ca.hit_force[3 * ss + 1], fz = ca.hit_force[3 * ss + 2];
                            if (fl & 1) { sx += fx; sy += fy; sz += fz; }
                            if (fl & 2) { sx -= 0.25 * fx; sy -= 0.25 * fy; sz -= 0.25 * fz; }
                        }
                    }
                }
            }
            if (lane == 0 && touched) {
                f_out[3 * n] = sx;
                f_out[3 * n + 1] = sy;
                f_out[3 * n + 2] = sz;
            }
        }
    }
    // Clear the grid for the next build.
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nthreads = (long long)gridDim.x * blockDim.x;
    for (long long i = ca.tab_off[c0] + tid; i < ca.tab_off[c1]; i += nthreads) ca.counts[i] = 0;
    for (long long c = c0 + tid; c < c1; c += nthreads) ca.n_overflow[c] = 0;
}

// ---------------------------------------------------------------------------
// FP64 vehicle reductions (delta-v, crush, separation rule), one block per
// vehicle, fixed summation order.
// ---------------------------------------------------------------------------
constexpr int VEH_TPB = 256;

__global__ void __launch_bounds__(VEH_TPB) k_vehicle_sums(const long long* __restrict__ off, const uint32_t* __restrict__ nodes,
                                                          const double* __restrict__ mass, const double* __restrict__ v,
                                                          const double* __restrict__ v0, double* __restrict__ out) {
    __shared__ double s[7][VEH_TPB];
    const int veh = blockIdx.x;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    for (long long i = off[veh] + threadIdx.x; i < off[veh + 1]; i += VEH_TPB) {
        const long long n = nodes[i];
        const double m = mass[n];
        acc[0] += m;
        for (int d = 0; d < 3; ++d) {
            acc[1 + d] += m * v[3 * n + d];
            acc[4 + d] += m * v0[3 * n + d];
        }
    }
    for (int k = 0; k < 7; ++k) s[k][threadIdx.x] = acc[k];
    __syncthreads();
    for (int w = VEH_TPB / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int k = 0; k < 7; ++k) s[k][threadIdx.x] += s[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 7; ++k) out[7 * veh + k] = s[k][0];
}

__global__ void __launch_bounds__(VEH_TPB) k_vehicle_vx(const long long* __restrict__ off, const uint32_t* __restrict__ nodes,
                                                        const double* __restrict__ mass, const double* __restrict__ v, Control* ctl) {
    __shared__ double sm[VEH_TPB], sp[VEH_TPB];
    if (ctl->done) return;
    const int veh = blockIdx.x;
    double m_acc = 0.0, p_acc = 0.0;
    for (long long i = off[veh] + threadIdx.x; i < off[veh + 1]; i += VEH_TPB) {
        const long long n = nodes[i];
        m_acc += mass[n];
        p_acc += mass[n] * v[3 * n];
    }
    sm[threadIdx.x] = m_acc;
    sp[threadIdx.x] = p_acc;
    __syncthreads();
    for (int w = VEH_TPB / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            sm[threadIdx.x] += sm[threadIdx.x + w];
            sp[threadIdx.x] += sp[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && veh < 4) ctl->vx[veh] = sm[0] > 0.0 ? sp[0] / sm[0] : 0.0;
}

}  // namespace

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
void launch_setup_geometry(cudaStream_t s, long long n_all, const double* pos, const uint32_t* conn_all, const int32_t* part,
                           const double* mat, double hourglass, const int64_t* hc_index, long long stride, float4* planes,
                           double* volume, double* lumped, double* dt_factor, double* elem_mass, int* bad) {
    if (n_all <= 0) return;
    k_setup_geometry<<<(unsigned)blocks_for(n_all, 128), 128, 0, s>>>(n_all, pos, conn_all, part, mat, hourglass, hc_index, stride,
                                                                       planes, volume, lumped, dt_factor, elem_mass, bad);
}
void launch_node_masses(cudaStream_t s, long long n, const uint32_t* off, const uint32_t* slot, const double* lumped,
                        double* mass, double* inv_mass) {
    k_node_masses<<<(unsigned)blocks_for(n, TPB), TPB, 0, s>>>(n, off, slot, lumped, mass, inv_mass);
}
void launch_init_state(cudaStream_t s, long long n_hc, long long stride, float4* state) {
    if (n_hc <= 0) return;
    k_init_state<<<(unsigned)blocks_for(n_hc, TPB), TPB, 0, s>>>(n_hc, stride, state);
}
void launch_forces(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, Control* ctl, int respect_done) {
    if (el.n_hc <= 0) return;
    k_forces<<<(unsigned)blocks_for(el.n_hc, TPB), TPB, 0, s>>>(el, nd, ctl, respect_done);
}
void launch_gather(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, double* f_out) {
    k_gather<<<(unsigned)blocks_for(nd.n, TPB), TPB, 0, s>>>(el, nd, f_out);
}
void launch_half(cudaStream_t s, const NodeArrays& nd, Control* ctl) {
    k_half<<<(unsigned)blocks_for(nd.n, TPB), TPB, 0, s>>>(nd, ctl);
}
void launch_full(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, Control* ctl) {
    k_full<<<(unsigned)blocks_for(nd.n, TPB), TPB, 0, s>>>(el, nd, ctl);
}
int elem_dt_blocks(long long n_all) { return (int)blocks_for(n_all > 0 ? n_all : 1, DT_TPB); }
void launch_elem_dt(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, Control* ctl, const double* u, double* partials,
                    int respect_done) {
    k_elem_dt<<<elem_dt_blocks(el.n_all), DT_TPB, 0, s>>>(el, nd, ctl, u, partials, respect_done);
}
void launch_dt_finalize(cudaStream_t s, Control* ctl, const double* partials, int n_blocks) {
    k_dt_finalize<<<1, 1, 0, s>>>(ctl, partials, n_blocks);
}
void launch_mass_scaling(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, Control* ctl, int force_apply) {
    k_mass_scaling<<<(unsigned)blocks_for(nd.n, TPB), TPB, 0, s>>>(el, nd, ctl, force_apply);
}
void launch_nonfinite(cudaStream_t s, const NodeArrays& nd, Control* ctl) {
    k_nonfinite<<<(unsigned)blocks_for(3 * nd.n, TPB), TPB, 0, s>>>(nd, ctl);
}
void launch_step_end(cudaStream_t s, Control* ctl, const ContactArrays& ca, int check_separation) {
    k_step_end<<<1, 1, 0, s>>>(ctl, ca, check_separation);
}
void launch_vehicle_sums(cudaStream_t s, int n_veh, const long long* veh_off, const uint32_t* veh_nodes, const double* mass,
                         const double* v, const double* v0, double* out) {
    if (n_veh <= 0) return;
    k_vehicle_sums<<<n_veh, VEH_TPB, 0, s>>>(veh_off, veh_nodes, mass, v, v0, out);
}
void launch_vehicle_vx(cudaStream_t s, int n_veh, const long long* veh_off, const uint32_t* veh_nodes, const double* mass,
                       const double* v, Control* ctl) {
    if (n_veh <= 0) return;
    k_vehicle_vx<<<n_veh, VEH_TPB, 0, s>>>(veh_off, veh_nodes, mass, v, ctl);
}

// Contact pass over contacts [c0, c1): faces + grid, first-hit search, ordered
// reaction gather into f_out. n_faces / n_slaves are the host-known totals of
// that range. dt_override > 0 is the drop-in call (no run control block).
void launch_contact(cudaStream_t s, const ContactArrays& ca, const NodeArrays& nd, Control* ctl, int c0, int c1,
                          long long n_faces, long long n_slaves, int entries_cap, double dt_override, const double* masses,
                          double* f_out, int skip_fixed) {
    if (c1 <= c0) return;
    const int run_mode = dt_override > 0.0 ? 0 : 1;
    if (n_faces > 0) {
        k_contact_faces<<<(unsigned)blocks_for(n_faces, TPB), TPB, 0, s>>>(ca, nd, ctl, c0, c1, run_mode);
        k_contact_scan<<<1, 1024, 0, s>>>(ca, ctl, c0, c1, run_mode);
        k_contact_fill<<<(unsigned)blocks_for(n_faces, TPB), TPB, 0, s>>>(ca, ctl, c0, c1, run_mode, entries_cap);
    }
    if (n_slaves > 0)
        k_contact_slaves<<<(unsigned)blocks_for(n_slaves, TPB), TPB, 0, s>>>(ca, nd, ctl, c0, c1, run_mode, dt_override, masses,
                                                                           entries_cap);
    long long warps = ca.n_cnodes > 0 ? ca.n_cnodes : 1;
    k_contact_gather<<<(unsigned)blocks_for(warps * 32, TPB), TPB, 0, s>>>(ca, nd, ctl, c0, c1, run_mode, f_out, skip_fixed);
}

}  // namespace crush
