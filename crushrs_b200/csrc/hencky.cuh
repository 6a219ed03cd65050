// hencky.cuh — Hencky (logarithmic) hyperelasticity of the elastic
// materials, the stress of the reference's scalar element path for a
// material without plasticity: finite_strain_return (src/material.rs:708-771)
// with the plastic state at identity, and the closed-form symmetric 3x3
// eigensolver it uses, symmetric_eigen3 (src/material.rs:570-659; trigonometric
// eigenvalues after D. Eberly, "A Robust Eigensolver for 3x3 Symmetric
// Matrices", 2014, the separated eigenvector from row cross products, the
// other two from one exact Jacobi rotation, eigenvalues as Rayleigh
// quotients). f64 throughout, the reference's order of operations; built
// without FMA contraction, so only the library transcendentals (acos, cos,
// sin, atan2, log) can differ from a host evaluation, in the last place.
#pragma once

namespace crush {

struct Vec3d {
    double x, y, z;
};
__device__ __forceinline__ Vec3d vd(double x, double y, double z) { return Vec3d{x, y, z}; }
__device__ __forceinline__ Vec3d vcross(const Vec3d& a, const Vec3d& b) {
    return vd(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double vdot(const Vec3d& a, const Vec3d& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ Vec3d vdiv(const Vec3d& a, double s) { return vd(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ Vec3d vmat(const double m[9], const Vec3d& u) {
    return vd(m[0] * u.x + m[1] * u.y + m[2] * u.z, m[3] * u.x + m[4] * u.y + m[5] * u.z, m[6] * u.x + m[7] * u.y + m[8] * u.z);
}

// Eigenvalues ascending in ev, unit eigenvectors in vec (row-major 3x3 input
// a, symmetric).
__device__ inline void symmetric_eigen3(const double a[9], double ev[3], Vec3d vec[3]) {
    double a00 = a[0], a01 = a[1], a02 = a[2], a11 = a[4], a12 = a[5], a22 = a[8];
    const double max_abs = fmax(fmax(fmax(fmax(fmax(fabs(a00), fabs(a01)), fabs(a02)), fabs(a11)), fabs(a12)), fabs(a22));
    if (max_abs == 0.0) {
        ev[0] = ev[1] = ev[2] = 0.0;
        vec[0] = vd(1.0, 0.0, 0.0);
        vec[1] = vd(0.0, 1.0, 0.0);
        vec[2] = vd(0.0, 0.0, 1.0);
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
    double val[3];
    if (norm == 0.0) {
        val[0] = a00;
        val[1] = a11;
        val[2] = a22;
        vec[0] = vd(1.0, 0.0, 0.0);
        vec[1] = vd(0.0, 1.0, 0.0);
        vec[2] = vd(0.0, 0.0, 1.0);
    } else {
        const double q = (a00 + a11 + a22) / 3.0;
        const double b00 = a00 - q, b11 = a11 - q, b22 = a22 - q;
        const double p = sqrt((b00 * b00 + b11 * b11 + b22 * b22 + 2.0 * norm) / 6.0);
        const double c00 = b11 * b22 - a12 * a12;
        const double c01 = a01 * b22 - a12 * a02;
        const double c02 = a01 * a12 - b11 * a02;
        const double det = (b00 * c00 - a01 * c01 + a02 * c02) / (p * p * p);
        const double half_det = fmin(fmax(0.5 * det, -1.0), 1.0);
        const double angle = acos(half_det) / 3.0;
        const double beta2 = 2.0 * cos(angle);
        const double beta0 = 2.0 * cos(angle + 2.0943951023931955);
        // the separated root: the largest when half_det >= 0, else the smallest
        const double e = half_det >= 0.0 ? q + p * beta2 : q + p * beta0;
        const Vec3d r0 = vd(a00 - e, a01, a02), r1 = vd(a01, a11 - e, a12), r2 = vd(a02, a12, a22 - e);
        const Vec3d x01 = vcross(r0, r1), x02 = vcross(r0, r2), x12 = vcross(r1, r2);
        const double d0 = vdot(x01, x01), d1 = vdot(x02, x02), d2 = vdot(x12, x12);
        Vec3d w;
        if (d0 >= d1 && d0 >= d2) w = vdiv(x01, sqrt(d0));
        else if (d1 >= d2) w = vdiv(x02, sqrt(d1));
        else w = vdiv(x12, sqrt(d2));
        Vec3d u;
        if (fabs(w.x) > fabs(w.y)) u = vdiv(vd(-w.z, 0.0, w.x), sqrt(w.x * w.x + w.z * w.z));
        else u = vdiv(vd(0.0, w.z, -w.y), sqrt(w.y * w.y + w.z * w.z));
        const Vec3d v = vcross(w, u);
        const double am[9] = {a00, a01, a02, a01, a11, a12, a02, a12, a22};
        const Vec3d au = vmat(am, u), av = vmat(am, v);
        const double m00 = vdot(u, au), m01 = vdot(u, av), m11 = vdot(v, av);
        const double theta = 0.5 * atan2(2.0 * m01, m00 - m11);
        const double sn = sin(theta), cs = cos(theta);
        vec[0] = w;
        vec[1] = vd(u.x * cs + v.x * sn, u.y * cs + v.y * sn, u.z * cs + v.z * sn);
        vec[2] = vd(v.x * cs - u.x * sn, v.y * cs - u.y * sn, v.z * cs - u.z * sn);
        for (int k = 0; k < 3; ++k) val[k] = vdot(vec[k], vmat(am, vec[k]));
    }
    // stable ascending order (insertion sort of three)
    for (int i = 1; i < 3; ++i)
        for (int j = i; j > 0 && val[j] < val[j - 1]; --j) {
            const double t = val[j];
            val[j] = val[j - 1];
            val[j - 1] = t;
            const Vec3d tv = vec[j];
            vec[j] = vec[j - 1];
            vec[j - 1] = tv;
        }
    for (int k = 0; k < 3; ++k) ev[k] = val[k] * max_abs;
}

// Kirchhoff stress tau (row-major) of an elastic material (Young's modulus,
// Poisson ratio) at deformation gradient f (row-major).
__device__ inline void hencky_elastic(double youngs, double poisson, const double f[9], double tau[9]) {
    const double g = youngs / (2.0 * (1.0 + poisson));
    const double k = youngs / (3.0 * (1.0 - 2.0 * poisson));
    double be[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) be[3 * i + j] = f[3 * i] * f[3 * j] + f[3 * i + 1] * f[3 * j + 1] + f[3 * i + 2] * f[3 * j + 2];
    double bs[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) bs[3 * i + j] = 0.5 * (be[3 * i + j] + be[3 * j + i]);
    double lam[3];
    Vec3d n[3];
    symmetric_eigen3(bs, lam, n);
    double eps[3];
    for (int a = 0; a < 3; ++a) eps[a] = 0.5 * log(fmax(lam[a], 1e-300));
    const double vol = eps[0] + eps[1] + eps[2];
    const double pressure = k * vol;
    for (int i = 0; i < 9; ++i) tau[i] = 0.0;
    for (int a = 0; a < 3; ++a) {
        const double dev = eps[a] - vol / 3.0;
        const double s = pressure + 2.0 * g * dev;
        const double nv[3] = {n[a].x, n[a].y, n[a].z};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) tau[3 * i + j] = tau[3 * i + j] + s * (nv[i] * nv[j]);
    }
}

}  // namespace crush
