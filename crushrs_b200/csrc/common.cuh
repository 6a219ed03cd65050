// common.cuh — shared device definitions of the B200 crash engine.
//
// Everything here is compiled with --fmad=false: no multiply-add is fused,
// so every f32 and f64 expression rounds exactly as the reference's Rust code
// (which never contracts a*b+c) and the element results can be bit-identical
// to the reference's f32 lane kernel on the same inputs.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace crush {

constexpr int MAX_KNOTS = 8;

// ---------------- element record layout (SoA of 16-byte planes) ----------------
// Plane p of element e lives at planes[p * stride + e]; a warp reading one
// plane reads 512 contiguous bytes. Static planes are written once at set-up;
// state planes are read and written every step.
constexpr int P_CONN = 0;    // 2 planes: node ids 0-3, 4-7 (uint32 bits)
constexpr int P_GRAD = 2;    // 6 planes: dN/dX at the centre, grad[3 i + c]
constexpr int P_GAMMA = 8;   // 8 planes: gamma[4 i + a]
constexpr int P_H = 16;      // 20 planes: upper triangle of H, row-major (78 used)
constexpr int P_META = 36;   // 1 plane: volume (f32), material index, model element index, crash slot
constexpr int N_STATIC_PLANES = 37;
// State: F_prev^-1 (9), R (9), stress (6), compaction, eroded flag (as bits), 2 pad.
constexpr int N_STATE_PLANES = 7;
constexpr int S_COMPACTION = 24;
constexpr int S_ERODED = 25;

// Index of H(row, col) in the packed upper triangle (row <= col).
__host__ __device__ constexpr int h_index(int r, int c) {
    return r <= c ? r * 12 - (r * (r - 1)) / 2 + (c - r) : c * 12 - (c * (c - 1)) / 2 + (r - c);
}

// Material of a part, as the f32 lane kernel sees it (src/kernel_simd.rs:263-271).
struct MaterialF32 {
    float youngs;
    float trans;
    float knot_c[MAX_KNOTS];
    float knot_s[MAX_KNOTS];
    float knot_h[MAX_KNOTS];
    float pad[6];
};
static_assert(sizeof(MaterialF32) == 128, "material record is two 64-byte lines");

// Per-run scalars kept on the device, so the step loop needs no host sync.
struct Control {
    double t;             // simulated time
    double end_time;
    double dt_cfl;        // dt before the end-time clip
    double dt_min;        // smallest step taken
    double dt_floor;      // mass-scaling floor
    double dt_scale;
    double contact_dt;
    double damping;       // velocity damping factor
    double added_mass_max;
    double added_total;   // total of the last mass scaling
    double added_total_acc;  // accumulating total of the current stable-dt pass
    unsigned long long dt_stable_bits;  // atomicMin target (bit pattern of a non-negative double)
    long long step;
    long long eroded_total;
    long long last_hit;   // last step with a penetration in a vehicle-vehicle contact
    long long max_steps;
    int done;
    int status;
    int nonfinite;
    int copy_timeout;     // an element tile's bulk copy did not complete within the wait bound
    int mass_scale_now;
    int hit_this_step;
    int adaptive;
    int stop_rule;
    int pad0;
    long long eroded_step;
    double vx[4];         // mean x-velocities for the separation rule
    double vx_part[4][64][2];  // per-block (mass, x-momentum) partial sums of the vehicles
};

constexpr int VX_BLOCKS = 64;

// The step's dt from the control block: dt_cfl clipped to the end time,
// never below 1e-15 (src/solver.rs:300).
__device__ __forceinline__ double step_dt(const Control* c) {
    double rem = c->end_time - c->t;
    double d = c->dt_cfl < rem ? c->dt_cfl : rem;
    return d > 1e-15 ? d : 1e-15;
}

// The dt of the step after the current one when no stable-dt check falls
// between them: step_dt once the step's end has added this step's dt to t
// (the same arithmetic, so it is the value the next step will use).
__device__ __forceinline__ double next_step_dt(const Control* c) {
    const double t1 = c->t + step_dt(c);
    double rem = c->end_time - t1;
    double d = c->dt_cfl < rem ? c->dt_cfl : rem;
    return d > 1e-15 ? d : 1e-15;
}

// Whether the current step is the crash's last by the step count or the end
// time (the stop rules that need no reduction), as the step's end decides it.
__device__ __forceinline__ bool last_step_by_count_or_time(const Control* c) {
    const double t1 = c->t + step_dt(c);
    return (c->max_steps > 0 && c->step + 1 >= c->max_steps) || !(t1 < c->end_time);
}

// Static planes are read once per step: streamed past L1 (evict-first), so
// L1 keeps the node positions that neighbouring elements share.
__device__ __forceinline__ float4 ld_plane(const float4* __restrict__ planes, long long stride, int p, long long e) {
    return __ldcs(planes + p * stride + e);
}

// ---------------- contact broad phase, shared by the kernels and the host ----------------
// Hash of grid cell (i, j, k) of grid level `level` (cell size cell * 4^level).
__host__ __device__ __forceinline__ unsigned cell_hash(long long i, long long j, long long k, int level) {
    unsigned long long h = (unsigned long long)i * 73856093ull ^ (unsigned long long)j * 19349663ull ^
                           (unsigned long long)k * 83492791ull ^ (unsigned long long)level * 2654435761ull;
    return (unsigned)(h ^ (h >> 29));
}

// Grid key box of a face at corners x (unit normal n, centre c): a box that
// contains every point the narrow test (src/contact.rs:113-128) can accept.
// A hit needs the point p inside the face box +- md, signed = n.(p - c) in
// [-md, 0], and proj = p - n signed (on the face plane) passing
// point_in_triangle for one of the triangles 012, 023, 123, 130. That test
// takes the barycentric coordinates of proj's orthogonal projection onto the
// triangle's plane, with tolerance 0.1: the projection lies in the triangle
// scaled 1.3x about its centroid. The face-plane points that project into
// that scaled triangle form the triangle whose corners are the scaled
// corners moved along the triangle normal onto the face plane (unbounded
// when the two planes are perpendicular). So the key box is the box of those
// corners over the four triangles, extended by md along -n, grown by a
// rounding margin and clipped to the face box +- md (which alone bounds it).
// Degenerate triangles accept nothing and are skipped. The margin (1e-7
// relative) and the 1.3001 scale dwarf the rounding of the reciprocals used
// here, so the box stays a superset of the narrow test's region.
constexpr int KEY_TRI_NONE = 0;   // degenerate triangle: accepts nothing
constexpr int KEY_TRI_PERP = 1;   // plane nearly perpendicular to the face: keep the whole face box +- md
constexpr int KEY_TRI_ADDED = 2;  // its corners were added to rlo/rhi

// Triangle t's part of the key box: its three moved corners added to
// (rlo, rhi), or one of the other outcomes above.
__host__ __device__ inline int key_box_triangle(const double x[4][3], const double n[3], const double c[3], int t, double* rlo,
                                                double* rhi) {
    // corners of triangles 012, 023, 123, 130, picked by value (no indexing
    // by t, which would put x in local memory on the device)
    double a[3], b[3], e[3];
    for (int d = 0; d < 3; ++d) {
        a[d] = t < 2 ? x[0][d] : x[1][d];
        b[d] = t == 0 ? x[1][d] : (t == 3 ? x[3][d] : x[2][d]);
        e[d] = t == 0 ? x[2][d] : (t == 3 ? x[0][d] : x[3][d]);
    }
    double u[3], v[3];
    for (int d = 0; d < 3; ++d) {
        u[d] = b[d] - a[d];
        v[d] = e[d] - a[d];
    }
    double m[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
    const double len = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
    if (!(len > 0.0)) return KEY_TRI_NONE;  // degenerate (or non-finite)
    const double il = 1.0 / len;
    for (int d = 0; d < 3; ++d) m[d] *= il;
    const double dn = n[0] * m[0] + n[1] * m[1] + n[2] * m[2];
    if (!(fabs(dn) > 1e-6)) return KEY_TRI_PERP;
    const double idn = 1.0 / dn;
    double cen[3];
    for (int d = 0; d < 3; ++d) cen[d] = (a[d] + b[d] + e[d]) * (1.0 / 3.0);
    for (int k = 0; k < 3; ++k) {
        double w[3];
        for (int d = 0; d < 3; ++d) w[d] = cen[d] + 1.3001 * ((k == 0 ? a[d] : (k == 1 ? b[d] : e[d])) - cen[d]);
        const double tt = (n[0] * (c[0] - w[0]) + n[1] * (c[1] - w[1]) + n[2] * (c[2] - w[2])) * idn;
        for (int d = 0; d < 3; ++d) {
            const double q = w[d] + tt * m[d];
            rlo[d] = fmin(rlo[d], q);
            rhi[d] = fmax(rhi[d], q);
        }
    }
    return KEY_TRI_ADDED;
}

// The key box from the triangles' parts: the face box +- md when a triangle
// was perpendicular, empty (klo > khi) when none added corners, else their
// box extended by md along -n, grown by the margin and clipped.
__host__ __device__ inline void key_box_finish(const double x[4][3], const double n[3], double md, bool any_perp, const double* rlo,
                                               const double* rhi, double* klo, double* khi) {
    double flo[3], fhi[3];
    for (int d = 0; d < 3; ++d) {
        double lo = x[0][d], hi = x[0][d];
        for (int k = 1; k < 4; ++k) {
            lo = fmin(lo, x[k][d]);
            hi = fmax(hi, x[k][d]);
        }
        flo[d] = lo;
        fhi[d] = hi;
        klo[d] = lo + -md;  // the narrow test's face box
        khi[d] = hi + md;
    }
    if (any_perp) return;
    if (!(rlo[0] <= rhi[0])) {  // every triangle degenerate: no point can hit
        for (int d = 0; d < 3; ++d) {
            klo[d] = 1.0;
            khi[d] = -1.0;
        }
        return;
    }
    const double ext = fmax(fmax(fhi[0] - flo[0], fhi[1] - flo[1]), fhi[2] - flo[2]);
    for (int d = 0; d < 3; ++d) {
        const double margin = 1e-7 * (1.0 + ext + md + fabs(rlo[d]) + fabs(rhi[d]));
        klo[d] = fmax(klo[d], rlo[d] - md * fmax(n[d], 0.0) - margin);
        khi[d] = fmin(khi[d], rhi[d] + md * fmax(-n[d], 0.0) + margin);
    }
}

__host__ __device__ inline void face_key_box(const double x[4][3], const double n[3], const double c[3], double md, double* klo,
                                             double* khi) {
    double rlo[3] = {1e300, 1e300, 1e300}, rhi[3] = {-1e300, -1e300, -1e300};
    bool perp = false;
    for (int t = 0; t < 4 && !perp; ++t) perp = key_box_triangle(x, n, c, t, rlo, rhi) == KEY_TRI_PERP;
    key_box_finish(x, n, md, perp, rlo, rhi, klo, khi);
}

}  // namespace crush
