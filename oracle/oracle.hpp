// oracle.hpp — TEST INFRASTRUCTURE ONLY.
//
// A CPU restatement of the crushrs explicit time-step hot path, used as the
// checker for the CUDA engine (tests/, __graft_entry__.smoke() and the CPU
// baseline leg of bench.py are its only callers). It is never linked into,
// loaded by or called from the product library.
//
// Two element paths are restated, each following the reference line by line:
//   * the scalar f64 path: src/kernel.rs:116-156 with
//     honeycomb_rate_update, src/material.rs:472-535;
//   * the f32 8-lane path: src/kernel_simd.rs:300-491 (block_forces_impl),
//     written over float[8] lane arrays so the compiler vectorises it the way
//     rustc/LLVM does. Rust never fuses a*b+c into an FMA, so neither does
//     this file (it is compiled with -ffp-contract=off); the lane helper the
//     reference names `fma` is a multiply followed by an add.
// Plus geometry (src/element.rs), stable dt and mass scaling
// (src/kernel.rs:207-258), contact (src/contact.rs), the solver loop
// (src/solver.rs:190-381) and the delta-v / crush outputs
// (src/bin/crushrs.rs:237-271).
//
// Third-party arithmetic: nalgebra 0.33.3 (not vendored with the reference)
// supplies 3x3 determinant/inverse, matrix products and the 12x12 inverse in
// src/element.rs:111. They are restated here with first-row cofactor
// expansion and LU with partial pivoting; results agree with nalgebra to
// round-off, not bitwise. Parity of this restatement with the reference is
// pinned by the reference's own unit tests (restated in tests/) and by the
// README's `crash 30 30` known answers (README.md:34-37).
#pragma once
#include <cstdint>
#include <cstddef>
#include <vector>
#include <string>
#include <array>
#include "../include/crush.h"

namespace oracle {

constexpr int MAX_KNOTS = 8;
constexpr int L = 8;  // lanes per block, src/kernel_simd.rs:18

// ---------------- small f64 linear algebra ----------------
struct M3 {
    double m[9];  // row-major
    double& operator()(int i, int j) { return m[3 * i + j]; }
    double operator()(int i, int j) const { return m[3 * i + j]; }
};
M3 m3_zero();
M3 m3_identity();
M3 m3_mul(const M3& a, const M3& b);
M3 m3_transpose(const M3& a);
double m3_det(const M3& a);
bool m3_inverse(const M3& a, M3* out);

// ---------------- materials (src/material.rs) ----------------
struct HoneycombParams {
    double youngs_modulus, yield_stress, hardening;
    double knots[MAX_KNOTS][3];  // compaction, stress, slope
    double cap_factor[3];
    void yield_at(double c, double* sy, double* h) const;  // material.rs:459
};
// material.rs:116 (check) + :430 (from_material); returns "" or an error.
std::string honeycomb_params(const crush_material& m, HoneycombParams* out);
// Plasticity::yield_at (material.rs:83), the curve-based form.
void plasticity_yield_at(const crush_material& m, double c, double* sy, double* h);
double dilatational_wave_speed(const crush_material& m);  // material.rs:226
// Closed-form eigen-decomposition of a symmetric 3x3 (material.rs:570):
// eigenvalues ascending, unit eigenvectors as the columns of *evec.
void symmetric_eigen3(const M3& a, double eval[3], M3* evec);
// Kirchhoff stress of an elastic (Hencky) material at F: finite_strain_return
// (material.rs:708-771) without plasticity.
void hencky_elastic(double youngs, double poisson, const M3& f, M3* tau);

struct RateState {  // material.rs:383
    M3 f_prev_inv, rotation;
    double stress[6];
    double compaction;
};
RateState rate_state_default();
// material.rs:472
void honeycomb_rate_update(const HoneycombParams& p, const M3& f, const RateState& s, M3* tau, RateState* ns);

// ---------------- geometry (src/element.rs) ----------------
struct HexGeometry {
    double center_grad[8][3];
    double volume;
    double lumped_mass[8];
    double gamma[8][4];
    double h[12][12];
};
// element.rs:141; returns false on a singular Jacobian / dependent modes.
bool hex_geometry(const double x[8][3], double youngs, double poisson, double density, double hourglass, HexGeometry* g);
// element.rs:176
void characteristic_length_and_volume(const double p[8][3], double* l, double* vol);

// ---------------- f32 lane blocks (src/kernel_simd.rs) ----------------
struct Block {
    uint32_t conn[L][8];
    float grad[24][L];
    float volume[L];
    float gamma[32][L];
    float h[144][L];  // column-major h[12*col + row]
    float youngs[L], yield0[L], hard[L], trans[L];
    float knot_c[MAX_KNOTS][L], knot_s[MAX_KNOTS][L], knot_h[MAX_KNOTS][L];
    float f_prev_inv[9][L], rotation[9][L], stress[6][L], compaction[L];
    bool eroded[L];
    int count;
};
void block_empty(Block* b);
// kernel_simd.rs:300-491
void block_forces(Block* b, const double* u, const double* positions, float out[L][24]);

// ---------------- model + elements (src/kernel.rs, src/model.rs) ----------------
struct Contact {
    std::vector<uint32_t> nodes;
    std::vector<double> node_scale;
    std::vector<std::array<uint32_t, 4>> faces;
    double stiffness, max_distance;
};
struct Vehicle {
    std::vector<uint32_t> nodes;
    uint32_t accel_node;
    std::vector<uint32_t> front;
};
struct Model {
    std::vector<double> positions;  // 3N
    std::vector<std::array<uint32_t, 8>> hexes;
    std::vector<int32_t> hex_part;
    std::vector<crush_material> materials;
    std::vector<double> initial_velocity;  // 3N
    std::vector<uint32_t> fixed_nodes;
    std::vector<Contact> contacts;
    std::vector<Vehicle> vehicles;
    crush_settings settings;
    size_t n_nodes() const { return positions.size() / 3; }
};
std::string model_from_desc(const crush_model_desc* d, Model* m);

struct Elements {
    std::vector<std::array<uint32_t, 8>> conn;
    std::vector<std::array<double, 24>> center_grad;
    std::vector<double> volume;
    std::vector<std::array<double, 32>> gamma;   // gamma[i*4 + a]
    std::vector<std::array<double, 144>> h;      // h[row*12 + col]
    std::vector<int32_t> part;
    std::vector<double> dt_factor;
    std::vector<RateState> state;
    std::vector<uint8_t> eroded;
    std::vector<uint8_t> honeycomb;
    std::vector<double> lumped;  // 8 per element
    std::vector<size_t> simd_ids, scalar_ids;
    std::vector<Block> blocks;
    std::vector<std::array<std::array<float, 24>, L>> block_out;
    const Model* model = nullptr;
    bool simd = true;
    int threads = 1;
};
std::string elements_build(const Model& m, bool simd, int threads, Elements* el);
// kernel.rs:160; returns newly eroded count, adds into global.
size_t compute_forces(Elements& el, const double* u, double* global);
// kernel.rs:207
bool stable_time_step(const Elements& el, const double* u, double* dt);
void element_time_steps(const Elements& el, const double* u, std::vector<double>* out);
// kernel.rs:243
double mass_scaling(const Elements& el, const double* u, double dt_min, const double* element_mass, double* added);
// model.rs:268
std::vector<double> lumped_masses(const Elements& el, size_t n_nodes);
// Lane-state sync into el.state (kernel.rs:261).
void sync_states(Elements& el);

// ---------------- contact (src/contact.rs) ----------------
struct ContactRuntime {
    std::vector<uint32_t> nodes;
    std::vector<double> scales;
    std::vector<std::array<uint32_t, 4>> faces;
    double stiffness, max_distance, depth_cap;
    size_t penetration_count = 0;
    double max_penetration = 0.0;
};
ContactRuntime contact_new(const Contact& c, const double* positions);
void contact_apply(ContactRuntime& c, const double* positions, const double* u, const double* v,
                   const double* masses, double dt, double* force);

// ---------------- solver (src/solver.rs) ----------------
struct HistoryAccel {  // Accelerometer, src/model.rs:64-73
    std::vector<uint32_t> nodes;
    bool has_frame = false;
    uint32_t origin = 0, x_axis = 0, plane = 0;
};
struct RunOptions {
    bool simd = true;
    int threads = 1;
    bool log_steps = false;  // record dt per step
    int history_steps = 0;   // Settings::history_steps
    std::vector<HistoryAccel> accelerometers;
    int frame_steps = 0;     // Settings::frame_steps
    int64_t time_from_step = -1;  // window_seconds covers the steps from this one to the end
};
struct RunResults {
    double time = 0.0;
    int64_t steps = 0;
    int64_t eroded = 0;
    double dt_min = 0.0;
    double added_mass_max = 0.0;
    int status = 0;
    std::vector<double> u, v, masses;
    std::vector<double> dt_log;
    // history records (src/solver.rs:114-187): per record its time and step,
    // n_parts x 11 part values (mass, v 3, u 3, a 3, ke) and per accelerometer
    // node 21 values (x, u, v, a, local u, v, a)
    std::vector<double> hist_time;
    std::vector<int64_t> hist_step;
    std::vector<double> hist_parts, hist_nodes;
    // frames (src/solver.rs:265-281): per frame time, step, displacement (3N
    // f32), plastic strain (E f32), Cauchy stress (6E f32), eroded (E)
    std::vector<double> frame_time;
    std::vector<int64_t> frame_step;
    std::vector<float> frame_disp, frame_pstrain, frame_stress;
    std::vector<uint8_t> frame_eroded;
    double force_seconds = 0.0, contact_seconds = 0.0, wall_seconds = 0.0, loop_seconds = 0.0, window_seconds = 0.0;
    std::vector<uint8_t> eroded_flags;  // per element at the end of the run
};
std::string run(const Model& m, const RunOptions& opt, RunResults* r);
// SAE J211 filter and resampling (src/signal.rs:9-66).
std::vector<double> cfc_filter(const std::vector<double>& x, double dt, double cfc);
void resample(const std::vector<double>& t, const std::vector<double>& y, double t0, double dt, double t_end, std::vector<double>* tu,
              std::vector<double>* yu);
// Delta-v / crush outputs (bin/crushrs.rs:237, :265).
void vehicle_result(const Model& m, const RunResults& r, int vehicle, crush_vehicle_result* out);

}  // namespace oracle
