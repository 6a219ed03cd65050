// hencky.cpp — TEST INFRASTRUCTURE ONLY (part of the oracle; see oracle.hpp).
//
// Hencky (logarithmic) hyperelasticity of the reference's elastic
// materials: finite_strain_return (src/material.rs:708-771) for a material
// without plasticity, whose plastic state stays the identity, and the
// closed-form symmetric 3x3 eigensolver it uses, symmetric_eigen3
// (src/material.rs:570-659; the reference cites D. Eberly, "A Robust
// Eigensolver for 3x3 Symmetric Matrices", 2014). Written over plain
// doubles, operation for operation in the reference's order, compiled with
// -ffp-contract=off like the rest of the oracle.
#include <cmath>

#include "oracle.hpp"

namespace oracle {

namespace {

struct V3 {
    double x, y, z;
};
V3 v3(double x, double y, double z) { return V3{x, y, z}; }
V3 cross(const V3& a, const V3& b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
double dot(const V3& a, const V3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 scale(const V3& a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
V3 divide(const V3& a, double s) { return v3(a.x / s, a.y / s, a.z / s); }
V3 add(const V3& a, const V3& b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
V3 sub(const V3& a, const V3& b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
V3 mat_vec(const double m[3][3], const V3& u) {
    return v3(m[0][0] * u.x + m[0][1] * u.y + m[0][2] * u.z, m[1][0] * u.x + m[1][1] * u.y + m[1][2] * u.z,
              m[2][0] * u.x + m[2][1] * u.y + m[2][2] * u.z);
}

// Stable ascending order of three (value, payload) pairs.
template <class T>
void sort3(double val[3], T pay[3]) {
    for (int i = 1; i < 3; ++i)
        for (int j = i; j > 0 && val[j] < val[j - 1]; --j) {
            std::swap(val[j], val[j - 1]);
            std::swap(pay[j], pay[j - 1]);
        }
}

}  // namespace

void symmetric_eigen3(const M3& a, double eval[3], M3* evec) {
    double a00 = a(0, 0), a01 = a(0, 1), a02 = a(0, 2), a11 = a(1, 1), a12 = a(1, 2), a22 = a(2, 2);
    double max_abs = std::fmax(std::fmax(std::fmax(std::fmax(std::fmax(std::fabs(a00), std::fabs(a01)), std::fabs(a02)), std::fabs(a11)),
                                         std::fabs(a12)),
                               std::fabs(a22));
    if (max_abs == 0.0) {
        eval[0] = eval[1] = eval[2] = 0.0;
        *evec = m3_identity();
        return;
    }
    const double inv = 1.0 / max_abs;
    a00 = a00 * inv;
    a01 = a01 * inv;
    a02 = a02 * inv;
    a11 = a11 * inv;
    a12 = a12 * inv;
    a22 = a22 * inv;
    const double norm = a01 * a01 + a02 * a02 + a12 * a12;
    if (norm == 0.0) {
        // already diagonal: the diagonal sorted, unit axes as vectors
        double val[3] = {a00, a11, a22};
        int axis[3] = {0, 1, 2};
        sort3(val, axis);
        *evec = m3_zero();
        for (int c = 0; c < 3; ++c) {
            (*evec)(axis[c], c) = 1.0;
            eval[c] = val[c] * max_abs;
        }
        return;
    }
    // trigonometric eigenvalues of the shifted, scaled matrix
    const double q = (a00 + a11 + a22) / 3.0;
    const double b00 = a00 - q, b11 = a11 - q, b22 = a22 - q;
    const double p = std::sqrt((b00 * b00 + b11 * b11 + b22 * b22 + 2.0 * norm) / 6.0);
    const double c00 = b11 * b22 - a12 * a12;
    const double c01 = a01 * b22 - a12 * a02;
    const double c02 = a01 * a12 - b11 * a02;
    const double det = (b00 * c00 - a01 * c01 + a02 * c02) / (p * p * p);
    const double half_det = std::fmin(std::fmax(0.5 * det, -1.0), 1.0);
    const double angle = std::acos(half_det) / 3.0;
    const double two_thirds_pi = 2.0943951023931955;
    const double beta2 = 2.0 * std::cos(angle);
    const double beta0 = 2.0 * std::cos(angle + two_thirds_pi);
    const double beta1 = -(beta0 + beta2);
    const double ev[3] = {q + p * beta0, q + p * beta1, q + p * beta2};
    const double am[3][3] = {{a00, a01, a02}, {a01, a11, a12}, {a02, a12, a22}};

    // eigenvector of the well-separated eigenvalue: the longest cross
    // product of two rows of (A - e I)
    auto vector0 = [&](double e) {
        const V3 r0 = v3(a00 - e, a01, a02), r1 = v3(a01, a11 - e, a12), r2 = v3(a02, a12, a22 - e);
        const V3 x01 = cross(r0, r1), x02 = cross(r0, r2), x12 = cross(r1, r2);
        const double d0 = dot(x01, x01), d1 = dot(x02, x02), d2 = dot(x12, x12);
        if (d0 >= d1 && d0 >= d2) return divide(x01, std::sqrt(d0));
        if (d1 >= d2) return divide(x02, std::sqrt(d1));
        return divide(x12, std::sqrt(d2));
    };
    const V3 w = half_det >= 0.0 ? vector0(ev[2]) : vector0(ev[0]);
    // the other two: one exact Jacobi rotation of A restricted to the plane
    // orthogonal to w
    V3 u;
    if (std::fabs(w.x) > std::fabs(w.y)) u = divide(v3(-w.z, 0.0, w.x), std::sqrt(w.x * w.x + w.z * w.z));
    else u = divide(v3(0.0, w.z, -w.y), std::sqrt(w.y * w.y + w.z * w.z));
    const V3 v = cross(w, u);
    const V3 au = mat_vec(am, u), av = mat_vec(am, v);
    const double m00 = dot(u, au), m01 = dot(u, av), m11 = dot(v, av);
    const double theta = 0.5 * std::atan2(2.0 * m01, m00 - m11);
    const double sn = std::sin(theta), cs = std::cos(theta);
    const V3 p1 = add(scale(u, cs), scale(v, sn));
    const V3 p2 = sub(scale(v, cs), scale(u, sn));
    // eigenvalues again as Rayleigh quotients, ascending
    V3 vec[3] = {w, p1, p2};
    double val[3];
    for (int k = 0; k < 3; ++k) val[k] = dot(vec[k], mat_vec(am, vec[k]));
    sort3(val, vec);
    for (int c = 0; c < 3; ++c) {
        eval[c] = val[c] * max_abs;
        (*evec)(0, c) = vec[c].x;
        (*evec)(1, c) = vec[c].y;
        (*evec)(2, c) = vec[c].z;
    }
}

void hencky_elastic(double youngs, double poisson, const M3& f, M3* tau) {
    const double g = youngs / (2.0 * (1.0 + poisson));
    const double k = youngs / (3.0 * (1.0 - 2.0 * poisson));
    // trial elastic left Cauchy-Green tensor F C_p^-1 F^T with C_p^-1 = I
    M3 be;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) be(i, j) = f(i, 0) * f(j, 0) + f(i, 1) * f(j, 1) + f(i, 2) * f(j, 2);
    M3 bs;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) bs(i, j) = 0.5 * (be(i, j) + be(j, i));
    double lam[3];
    M3 n;
    symmetric_eigen3(bs, lam, &n);
    double eps[3];
    for (int a = 0; a < 3; ++a) eps[a] = 0.5 * std::log(std::fmax(lam[a], 1e-300));
    const double vol = eps[0] + eps[1] + eps[2];
    const double pressure = k * vol;
    *tau = m3_zero();
    for (int a = 0; a < 3; ++a) {
        const double dev = eps[a] - vol / 3.0;
        const double s = pressure + 2.0 * g * dev;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) (*tau)(i, j) = (*tau)(i, j) + s * (n(i, a) * n(j, a));
    }
}

}  // namespace oracle
