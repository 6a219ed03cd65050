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

__device__ __forceinline__ float4 ld_plane(const float4* __restrict__ planes, long long stride, int p, long long e) {
    return __ldg(planes + p * stride + e);
}

}  // namespace crush
