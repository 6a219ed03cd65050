// geometry.cpp — TEST INFRASTRUCTURE ONLY (see oracle.hpp).
// Restates src/element.rs (hexahedron set-up) and the small dense linear
// algebra nalgebra provides to it.
#include "oracle.hpp"
#include <cmath>
#include <cstring>
#include <limits>

namespace oracle {

M3 m3_zero() { M3 r; for (double& x : r.m) x = 0.0; return r; }
M3 m3_identity() { M3 r = m3_zero(); r.m[0] = r.m[4] = r.m[8] = 1.0; return r; }

// Column-by-column accumulation, k ascending: r_ij = (a_i0 b_0j + a_i1 b_1j) + a_i2 b_2j.
M3 m3_mul(const M3& a, const M3& b) {
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = a(i, 0) * b(0, j);
            s = s + a(i, 1) * b(1, j);
            s = s + a(i, 2) * b(2, j);
            r(i, j) = s;
        }
    return r;
}

M3 m3_transpose(const M3& a) {
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r(i, j) = a(j, i);
    return r;
}

// First-row cofactor expansion.
double m3_det(const M3& a) {
    double m11 = a(1, 1) * a(2, 2) - a(2, 1) * a(1, 2);
    double m12 = a(1, 0) * a(2, 2) - a(2, 0) * a(1, 2);
    double m13 = a(1, 0) * a(2, 1) - a(2, 0) * a(1, 1);
    return a(0, 0) * m11 - a(0, 1) * m12 + a(0, 2) * m13;
}

bool m3_inverse(const M3& a, M3* out) {
    double m11 = a(1, 1) * a(2, 2) - a(2, 1) * a(1, 2);
    double m12 = a(1, 0) * a(2, 2) - a(2, 0) * a(1, 2);
    double m13 = a(1, 0) * a(2, 1) - a(2, 0) * a(1, 1);
    double det = a(0, 0) * m11 - a(0, 1) * m12 + a(0, 2) * m13;
    if (det == 0.0) return false;
    M3 r;
    r(0, 0) = m11 / det;
    r(0, 1) = -(a(0, 1) * a(2, 2) - a(2, 1) * a(0, 2)) / det;
    r(0, 2) = (a(0, 1) * a(1, 2) - a(1, 1) * a(0, 2)) / det;
    r(1, 0) = -m12 / det;
    r(1, 1) = (a(0, 0) * a(2, 2) - a(2, 0) * a(0, 2)) / det;
    r(1, 2) = -(a(0, 0) * a(1, 2) - a(1, 0) * a(0, 2)) / det;
    r(2, 0) = m13 / det;
    r(2, 1) = -(a(0, 0) * a(2, 1) - a(2, 0) * a(0, 1)) / det;
    r(2, 2) = (a(0, 0) * a(1, 1) - a(1, 0) * a(0, 1)) / det;
    *out = r;
    return true;
}

// Dense n x n inverse by LU with partial pivoting (nalgebra's try_inverse
// for sizes above 4 goes through an LU decomposition).
static bool dense_inverse(int n, const double* a_in, double* inv) {
    std::vector<double> a(a_in, a_in + n * n);
    std::vector<int> perm(n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int k = 0; k < n; ++k) {
        int p = k;
        double best = std::fabs(a[k * n + k]);
        for (int i = k + 1; i < n; ++i)
            if (std::fabs(a[i * n + k]) > best) { best = std::fabs(a[i * n + k]); p = i; }
        if (best == 0.0) return false;
        if (p != k) {
            for (int j = 0; j < n; ++j) std::swap(a[k * n + j], a[p * n + j]);
            std::swap(perm[k], perm[p]);
        }
        for (int i = k + 1; i < n; ++i) {
            double f = a[i * n + k] / a[k * n + k];
            a[i * n + k] = f;
            for (int j = k + 1; j < n; ++j) a[i * n + j] -= f * a[k * n + j];
        }
    }
    for (int c = 0; c < n; ++c) {
        std::vector<double> y(n);
        for (int i = 0; i < n; ++i) {
            double s = (perm[i] == c) ? 1.0 : 0.0;
            for (int j = 0; j < i; ++j) s -= a[i * n + j] * y[j];
            y[i] = s;
        }
        for (int i = n - 1; i >= 0; --i) {
            double s = y[i];
            for (int j = i + 1; j < n; ++j) s -= a[i * n + j] * inv[j * n + c];
            inv[i * n + c] = s / a[i * n + i];
        }
    }
    return true;
}

// C3D8 parametric corners, element.rs:9.
static const double XI[8][3] = {
    {-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
    {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
static const double GAUSS = 0.5773502691896258;  // element.rs:20
// Flanagan–Belytschko hourglass base vectors, element.rs:83.
static const double MODES[4][8] = {
    {1, 1, -1, -1, -1, -1, 1, 1},
    {1, -1, -1, 1, -1, 1, 1, -1},
    {1, -1, 1, -1, 1, -1, 1, -1},
    {-1, 1, -1, 1, 1, -1, 1, -1}};

// element.rs:23
static void shape_derivatives(double xi, double eta, double zeta, double dn[8][3]) {
    for (int i = 0; i < 8; ++i) {
        const double* s = XI[i];
        dn[i][0] = 0.125 * s[0] * (1.0 + s[1] * eta) * (1.0 + s[2] * zeta);
        dn[i][1] = 0.125 * s[1] * (1.0 + s[0] * xi) * (1.0 + s[2] * zeta);
        dn[i][2] = 0.125 * s[2] * (1.0 + s[0] * xi) * (1.0 + s[1] * eta);
    }
}

// element.rs:35
static void shape_functions(double xi, double eta, double zeta, double n[8]) {
    for (int i = 0; i < 8; ++i) {
        const double* s = XI[i];
        n[i] = 0.125 * (1.0 + s[0] * xi) * (1.0 + s[1] * eta) * (1.0 + s[2] * zeta);
    }
}

// element.rs:43: J = dNᵀ x, grad = dN J⁻ᵀ.
static bool reference_gradients(const double x[8][3], const double dn[8][3], double g[8][3], double* det) {
    M3 j;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double s = dn[0][r] * x[0][c];
            for (int k = 1; k < 8; ++k) s = s + dn[k][r] * x[k][c];
            j(r, c) = s;
        }
    M3 ji;
    if (!m3_inverse(j, &ji)) return false;
    for (int i = 0; i < 8; ++i)
        for (int c = 0; c < 3; ++c) {
            // (dN * J⁻ᵀ)_ic = Σ_k dN_ik (J⁻¹)_ck
            double s = dn[i][0] * ji(c, 0);
            s = s + dn[i][1] * ji(c, 1);
            s = s + dn[i][2] * ji(c, 2);
            g[i][c] = s;
        }
    *det = m3_det(j);
    return true;
}

// element.rs:50, engineering shear.
static void b_matrix(const double g[8][3], double b[6][24]) {
    std::memset(b, 0, sizeof(double) * 6 * 24);
    for (int i = 0; i < 8; ++i) {
        const double n0 = g[i][0], n1 = g[i][1], n2 = g[i][2];
        b[0][3 * i] = n0;
        b[1][3 * i + 1] = n1;
        b[2][3 * i + 2] = n2;
        b[3][3 * i] = n1;
        b[3][3 * i + 1] = n0;
        b[4][3 * i + 1] = n2;
        b[4][3 * i + 2] = n1;
        b[5][3 * i] = n2;
        b[5][3 * i + 2] = n0;
    }
}

// material.rs:662
static void elastic_matrix(double e, double nu, double c[6][6]) {
    double lam = e * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    double mu = e / (2.0 * (1.0 + nu));
    std::memset(c, 0, sizeof(double) * 36);
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) c[i][j] = (i == j) ? lam + 2.0 * mu : lam;
        c[i + 3][i + 3] = mu;
    }
}

bool hex_geometry(const double x[8][3], double youngs, double poisson, double density, double hourglass, HexGeometry* g) {
    double dnc[8][3];
    shape_derivatives(0.0, 0.0, 0.0, dnc);
    double detc;
    if (!reference_gradients(x, dnc, g->center_grad, &detc)) return false;
    double cs[6][6];
    elastic_matrix(hourglass * youngs, poisson, cs);
    double bc[6][24];
    b_matrix(g->center_grad, bc);
    static thread_local double k[24][24];
    std::memset(k, 0, sizeof(k));
    double mass[8][8] = {};
    double volume = 0.0;
    for (int q = 0; q < 8; ++q) {
        double xi = XI[q][0] * GAUSS, eta = XI[q][1] * GAUSS, zeta = XI[q][2] * GAUSS;
        double dn[8][3], gq[8][3], detj;
        shape_derivatives(xi, eta, zeta, dn);
        if (!reference_gradients(x, dn, gq, &detj)) return false;
        double b[6][24];
        b_matrix(gq, b);
        double db[6][24];
        for (int s = 0; s < 6; ++s)
            for (int j = 0; j < 24; ++j) db[s][j] = b[s][j] - bc[s][j];
        // k += dbᵀ C db det_j
        double cdb[6][24];
        for (int s = 0; s < 6; ++s)
            for (int j = 0; j < 24; ++j) {
                double acc = 0.0;
                for (int t = 0; t < 6; ++t) acc += cs[s][t] * db[t][j];
                cdb[s][j] = acc;
            }
        for (int i = 0; i < 24; ++i)
            for (int j = 0; j < 24; ++j) {
                double acc = 0.0;
                for (int s = 0; s < 6; ++s) acc += db[s][i] * cdb[s][j];
                k[i][j] += acc * detj;
            }
        volume += detj;
        double n[8];
        shape_functions(xi, eta, zeta, n);
        for (int i = 0; i < 8; ++i)
            for (int j = 0; j < 8; ++j) mass[i][j] += density * n[i] * n[j] * detj;
    }
    g->volume = volume;
    for (int i = 0; i < 8; ++i) {
        double s = 0.0;
        for (int j = 0; j < 8; ++j) s += mass[i][j];
        g->lumped_mass[i] = s;
    }
    // Hourglass::from_dense, element.rs:91-114.
    for (int a = 0; a < 4; ++a) {
        double hx[3] = {0.0, 0.0, 0.0};
        for (int j = 0; j < 8; ++j)
            for (int d = 0; d < 3; ++d) hx[d] += MODES[a][j] * x[j][d];
        for (int i = 0; i < 8; ++i) {
            const double* b = g->center_grad[i];
            double dot = hx[0] * b[0] + hx[1] * b[1] + hx[2] * b[2];
            g->gamma[i][a] = MODES[a][i] - dot;
        }
    }
    double G[12][24] = {};
    for (int a = 0; a < 4; ++a)
        for (int i = 0; i < 8; ++i)
            for (int d = 0; d < 3; ++d) G[3 * a + d][3 * i + d] = g->gamma[i][a];
    double ggt[12 * 12], ggt_inv[12 * 12];
    for (int r = 0; r < 12; ++r)
        for (int c = 0; c < 12; ++c) {
            double s = 0.0;
            for (int j = 0; j < 24; ++j) s += G[r][j] * G[c][j];
            ggt[r * 12 + c] = s;
        }
    if (!dense_inverse(12, ggt, ggt_inv)) return false;
    // h = ggt_inv * g * k * gᵀ * ggt_inv, left to right.
    double ig[12][24];
    for (int r = 0; r < 12; ++r)
        for (int j = 0; j < 24; ++j) {
            double s = 0.0;
            for (int t = 0; t < 12; ++t) s += ggt_inv[r * 12 + t] * G[t][j];
            ig[r][j] = s;
        }
    double igk[12][24];
    for (int r = 0; r < 12; ++r)
        for (int j = 0; j < 24; ++j) {
            double s = 0.0;
            for (int t = 0; t < 24; ++t) s += ig[r][t] * k[t][j];
            igk[r][j] = s;
        }
    double igkg[12][12];
    for (int r = 0; r < 12; ++r)
        for (int c = 0; c < 12; ++c) {
            double s = 0.0;
            for (int t = 0; t < 24; ++t) s += igk[r][t] * G[c][t];
            igkg[r][c] = s;
        }
    for (int r = 0; r < 12; ++r)
        for (int c = 0; c < 12; ++c) {
            double s = 0.0;
            for (int t = 0; t < 12; ++t) s += igkg[r][t] * ggt_inv[t * 12 + c];
            g->h[r][c] = s;
        }
    return true;
}

// element.rs:176-186
void characteristic_length_and_volume(const double p[8][3], double* l, double* vol_out) {
    static const int TETS[6][4] = {{0, 1, 2, 6}, {0, 2, 3, 6}, {0, 3, 7, 6}, {0, 7, 4, 6}, {0, 4, 5, 6}, {0, 5, 1, 6}};
    static const int FACES[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}};
    auto sub = [](const double* a, const double* b, double* r) { r[0] = a[0] - b[0]; r[1] = a[1] - b[1]; r[2] = a[2] - b[2]; };
    auto cross = [](const double* a, const double* b, double* r) {
        r[0] = a[1] * b[2] - a[2] * b[1];
        r[1] = a[2] * b[0] - a[0] * b[2];
        r[2] = a[0] * b[1] - a[1] * b[0];
    };
    auto dot = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
    double vol = 0.0;
    for (int t = 0; t < 6; ++t) {
        double e1[3], e2[3], e3[3], c[3];
        sub(p[TETS[t][1]], p[TETS[t][0]], e1);
        sub(p[TETS[t][2]], p[TETS[t][0]], e2);
        sub(p[TETS[t][3]], p[TETS[t][0]], e3);
        cross(e1, e2, c);
        vol = vol + dot(c, e3) / 6.0;
    }
    double a_max = 0.0;
    for (int f = 0; f < 6; ++f) {
        double d1[3], d2[3], c[3];
        sub(p[FACES[f][2]], p[FACES[f][0]], d1);
        sub(p[FACES[f][3]], p[FACES[f][1]], d2);
        cross(d1, d2, c);
        double a = 0.5 * std::sqrt(dot(c, c));
        a_max = std::fmax(a_max, a);
    }
    *vol_out = vol;
    if (vol <= 0.0 || a_max <= 0.0) *l = std::numeric_limits<double>::infinity();
    else *l = vol / a_max;
}

}  // namespace oracle
