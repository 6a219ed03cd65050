// contact.cpp — TEST INFRASTRUCTURE ONLY (see oracle.hpp).
// Restates src/contact.rs: the static broad phase of ContactRuntime::new
// (:48-70) and the serial O(nodes x faces) first-hit penalty loop of
// ContactRuntime::apply (:92-160).
#include "oracle.hpp"
#include <cmath>
#include <limits>

namespace oracle {

namespace {
struct Vec3 { double x, y, z; };
inline Vec3 operator+(Vec3 a, Vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Vec3 operator-(Vec3 a, Vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vec3 operator*(Vec3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(Vec3 a, Vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline Vec3 cross(Vec3 a, Vec3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

const double MAX_ACCEL = 1.0e5;  // contact.rs:75
const double DAMPING = 0.0;      // contact.rs:82
const double SOFT = 0.1;         // contact.rs:87

// contact.rs:29-43
bool point_in_triangle(Vec3 p, Vec3 a, Vec3 b, Vec3 c) {
    const double tol = 0.1;
    Vec3 v0 = c - a, v1 = b - a, v2 = p - a;
    double d00 = dot(v0, v0), d01 = dot(v0, v1), d02 = dot(v0, v2), d11 = dot(v1, v1), d12 = dot(v1, v2);
    double inv = 1.0 / (d00 * d11 - d01 * d01);
    double u = (d11 * d02 - d01 * d12) * inv;
    double v = (d00 * d12 - d01 * d02) * inv;
    return u >= -tol && v >= -tol && u + v <= 1.0 + tol;
}
}  // namespace

ContactRuntime contact_new(const Contact& c, const double* positions) {
    const double inf = std::numeric_limits<double>::infinity();
    double lo[3] = {inf, inf, inf}, hi[3] = {-inf, -inf, -inf};
    for (const auto& f : c.faces)
        for (uint32_t n : f)
            for (int d = 0; d < 3; ++d) {
                lo[d] = std::fmin(lo[d], positions[3 * n + d]);
                hi[d] = std::fmax(hi[d], positions[3 * n + d]);
            }
    for (int d = 0; d < 3; ++d) { lo[d] += -c.max_distance; hi[d] += c.max_distance; }
    ContactRuntime r;
    for (size_t i = 0; i < c.nodes.size(); ++i) {
        uint32_t n = c.nodes[i];
        bool inside = true;
        for (int d = 0; d < 3; ++d) {
            double p = positions[3 * n + d];
            if (!(p >= lo[d] && p <= hi[d])) inside = false;
        }
        if (inside) {
            r.nodes.push_back(n);
            r.scales.push_back(i < c.node_scale.size() ? c.node_scale[i] : 1.0);
        }
    }
    r.faces = c.faces;
    r.stiffness = c.stiffness;
    r.max_distance = c.max_distance;
    r.depth_cap = 0.1 * c.max_distance;
    return r;
}

void contact_apply(ContactRuntime& c, const double* positions, const double* u, const double* v,
                   const double* masses, double dt, double* force) {
    auto cur = [&](uint32_t n) {
        return Vec3{positions[3 * n] + u[3 * n], positions[3 * n + 1] + u[3 * n + 1], positions[3 * n + 2] + u[3 * n + 2]};
    };
    auto vel = [&](uint32_t n) { return v ? Vec3{v[3 * n], v[3 * n + 1], v[3 * n + 2]} : Vec3{0, 0, 0}; };
    struct Face { Vec3 x[4], normal, center, lo, hi; };
    std::vector<Face> faces(c.faces.size());
    for (size_t fi = 0; fi < c.faces.size(); ++fi) {
        Face& f = faces[fi];
        for (int k = 0; k < 4; ++k) f.x[k] = cur(c.faces[fi][k]);
        Vec3 nrm = cross(f.x[1] - f.x[0], f.x[2] - f.x[0]);
        double len = std::sqrt(dot(nrm, nrm));
        f.normal = {nrm.x / len, nrm.y / len, nrm.z / len};
        Vec3 s = ((f.x[0] + f.x[1]) + f.x[2]) + f.x[3];
        f.center = {s.x / 4.0, s.y / 4.0, s.z / 4.0};
        Vec3 lo = f.x[0], hi = f.x[0];
        for (int k = 1; k < 4; ++k) {
            lo = {std::fmin(lo.x, f.x[k].x), std::fmin(lo.y, f.x[k].y), std::fmin(lo.z, f.x[k].z)};
            hi = {std::fmax(hi.x, f.x[k].x), std::fmax(hi.y, f.x[k].y), std::fmax(hi.z, f.x[k].z)};
        }
        f.lo = {lo.x + -c.max_distance, lo.y + -c.max_distance, lo.z + -c.max_distance};
        f.hi = {hi.x + c.max_distance, hi.y + c.max_distance, hi.z + c.max_distance};
    }
    c.penetration_count = 0;
    c.max_penetration = 0.0;
    for (size_t k = 0; k < c.nodes.size(); ++k) {
        uint32_t n = c.nodes[k];
        double scale = c.scales[k];
        Vec3 point = cur(n);
        for (size_t fi = 0; fi < faces.size(); ++fi) {
            const Face& face = faces[fi];
            if (point.x < face.lo.x || point.x > face.hi.x || point.y < face.lo.y || point.y > face.hi.y ||
                point.z < face.lo.z || point.z > face.hi.z)
                continue;
            double signed_d = -dot(face.normal, face.center - point);
            if (signed_d > 0.0 || signed_d < -c.max_distance) continue;
            Vec3 projected = point - face.normal * signed_d;
            bool inside = point_in_triangle(projected, face.x[0], face.x[1], face.x[2]) ||
                          point_in_triangle(projected, face.x[0], face.x[2], face.x[3]) ||
                          point_in_triangle(projected, face.x[1], face.x[2], face.x[3]) ||
                          point_in_triangle(projected, face.x[1], face.x[3], face.x[0]);
            if (!inside) continue;
            double depth = std::fmin(-signed_d, c.depth_cap);
            double k_pen = std::fmin(c.stiffness * scale, SOFT * masses[n] / (dt * dt));
            const auto& fn = c.faces[fi];
            Vec3 v_face = (((vel(fn[0]) + vel(fn[1])) + vel(fn[2])) + vel(fn[3]));
            v_face = {v_face.x / 4.0, v_face.y / 4.0, v_face.z / 4.0};
            double v_rel = dot(face.normal, vel(n) - v_face);
            double damping = 2.0 * DAMPING * std::sqrt(k_pen * masses[n]) * std::fmax(-v_rel, 0.0);
            double magnitude = std::fmin(k_pen * depth + damping, masses[n] * MAX_ACCEL);
            Vec3 f = {magnitude * face.normal.x, magnitude * face.normal.y, magnitude * face.normal.z};
            force[3 * n] += f.x;
            force[3 * n + 1] += f.y;
            force[3 * n + 2] += f.z;
            for (int j = 0; j < 4; ++j) {
                uint32_t m = fn[j];
                force[3 * m] -= 0.25 * f.x;
                force[3 * m + 1] -= 0.25 * f.y;
                force[3 * m + 2] -= 0.25 * f.z;
            }
            c.penetration_count += 1;
            c.max_penetration = std::fmax(c.max_penetration, -signed_d);
            break;
        }
    }
}

}  // namespace oracle
