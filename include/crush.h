/*
 * crush.h — C ABI of the B200 explicit time-step engine for crushrs-style
 * crash models (one-point honeycomb hexahedra, node-to-face penalty contact,
 * central-difference integration with selective mass scaling).
 *
 * The entry points replace the Rust-internal calls the reference solver makes
 * on its hot path (paths are relative to the crushrs source tree):
 *
 *   crush_compute_forces   <- Elements::compute_forces      src/kernel.rs:160
 *                             (Blocks::compute_forces + scatter,
 *                              src/kernel_simd.rs:558, :573)
 *   crush_contact_apply    <- ContactRuntime::apply         src/contact.rs:92
 *   crush_stable_dt        <- Elements::stable_time_step    src/kernel.rs:207
 *   crush_mass_scaling     <- Elements::mass_scaling        src/kernel.rs:243
 *   crush_create           <- Elements::build               src/kernel.rs:53
 *                             + Model::lumped_masses        src/model.rs:268
 *                             + ContactRuntime::new         src/contact.rs:48
 *   crush_run              <- crushrs::run                  src/solver.rs:190
 *   crush_vehicle_result   <- part_delta_v / crush_rear     src/bin/crushrs.rs:237, :265
 *
 * Conventions
 *   - Every function returns an int status: CRUSH_OK (0) or a negative
 *     CRUSH_ERR_* code; crush_stable_dt may also return CRUSH_NONE (1) for the
 *     reference's `None`. Nothing aborts the process; crush_last_error()
 *     gives a message for the calling thread's last failure.
 *   - Buffers passed in are caller-owned host memory unless the name says
 *     `_device`, in which case they are device pointers on the context's GPU.
 *     "accum" outputs are ADDED into, like the reference's `global: &mut [f64]`
 *     (callers zero them first, as solver.rs:307,327 does).
 *   - Vectors of nodal quantities are flat f64 arrays of length 3*n_nodes
 *     (x,y,z interleaved), exactly the reference's `u`, `v`, `f_int`, `f_ext`.
 *   - One context per thread, or an external mutex. Work is ordered on the
 *     context's CUDA stream; host-buffer entry points synchronise before
 *     returning.
 */
#ifndef CRUSH_H
#define CRUSH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CRUSH_OK 0
#define CRUSH_NONE 1
#define CRUSH_ERR_INVALID (-1)
#define CRUSH_ERR_NONFINITE (-2)
#define CRUSH_ERR_OOM (-3)
#define CRUSH_ERR_TIMEOUT (-4)
#define CRUSH_ERR_CUDA (-5)
#define CRUSH_ERR_UNSUPPORTED (-6)
#define CRUSH_ERR_BUSY (-7)

/* Material models (src/material.rs:20). Honeycomb runs on the device kernels.
 * Elastic parts are accepted only when every node of every element of the
 * part is fixed (a rigid road or wall slab): their deformation gradient stays
 * the identity, so they carry no force and contribute only a constant
 * element stability limit. */
#define CRUSH_MAT_HONEYCOMB 0
#define CRUSH_MAT_ELASTIC 1

#define CRUSH_MAX_KNOTS 8

/* One part's material, mirroring Material + Plasticity (src/material.rs:42,155). */
typedef struct crush_material {
    int32_t model;             /* CRUSH_MAT_* */
    double youngs_modulus;     /* Pa */
    double poisson_ratio;      /* honeycomb: 0 */
    double density;            /* kg/m^3 */
    double yield_stress;       /* Pa, bilinear curve when n_curve == 0 */
    double hardening;          /* Pa per unit compaction */
    int32_t n_curve;           /* 0, or 2..8 tabulated knots (one fewer with densification) */
    double curve[CRUSH_MAX_KNOTS][2]; /* [compaction, yield stress] ascending from c = 0 */
    int32_t has_densification; /* 1: lock-up knot [c_lock, k_lock] appended */
    double densification[2];
    double transverse_factor;  /* cap factor of local y, z normal stresses (1 = isotropic) */
} crush_material;

/* One-way node-to-face penalty contact (src/model.rs:13). A two-way pair is
 * two of these at half stiffness each (src/model.rs:257). */
typedef struct crush_contact {
    int64_t n_nodes;
    const uint32_t* nodes;     /* primary (slave) nodes, sorted unique */
    const double* node_scale;  /* per-node stiffness factor aligned with nodes, or NULL (= 1) */
    int64_t n_faces;
    const uint32_t* faces;     /* 4 node ids per quad, counter-clockwise about the outward normal */
    double stiffness;          /* N/m per node */
    double max_distance;       /* m */
} crush_contact;

/* Stop rules for crush_run. */
#define CRUSH_STOP_END_TIME 0
/* Run until the two vehicles separate: every 10 steps after the first contact
 * hit, stop when vehicle[1]'s mass-weighted mean x-velocity minus vehicle[0]'s
 * is >= 0 and no contact node has penetrated for the last 100 steps. The
 * settings' max_steps caps the run. Not in the reference (which only runs to
 * end_time); defined identically in the oracle. */
#define CRUSH_STOP_SEPARATION 1

/* Solver settings (src/model.rs:76-150). */
typedef struct crush_settings {
    double end_time;           /* s */
    double dt_scale;           /* safety factor on the stable step (0.85) */
    double time_step;          /* fixed step if > 0, else adaptive */
    int32_t adaptive_check_steps; /* re-evaluate the stable step every N steps (5) */
    double hourglass;          /* stabilisation stiffness as a fraction of E (0.1) */
    double velocity_damping;   /* per-step velocity factor (1.0) */
    double mass_scaling;       /* dt floor as a fraction of the initial stable step (0.25) */
    int32_t stop_rule;         /* CRUSH_STOP_* */
    int32_t max_steps;         /* 0 = unlimited */
} crush_settings;

/* Outputs wanted per vehicle: delta-v over `nodes` (src/bin/crushrs.rs:237)
 * and crush = |u_x(accel_node) - mean u_x(front_nodes)| (src/bin/crushrs.rs:265). */
typedef struct crush_vehicle {
    int64_t n_nodes;
    const uint32_t* nodes;
    uint32_t accel_node;
    int64_t n_front;
    const uint32_t* front_nodes;
} crush_vehicle;

/* Whole model (src/model.rs:153), as flat arrays. */
typedef struct crush_model_desc {
    int64_t n_nodes;
    const double* positions;        /* 3*n_nodes reference coordinates */
    int64_t n_hexes;
    const uint32_t* hexes;          /* 8 node ids per hexahedron, C3D8 order */
    const int32_t* hex_part;        /* part index per hexahedron */
    int32_t n_parts;
    const crush_material* materials;/* one per part */
    const double* initial_velocity; /* 3*n_nodes */
    int64_t n_fixed;
    const uint32_t* fixed_nodes;
    int32_t n_contacts;
    const crush_contact* contacts;
    int32_t n_vehicles;
    const crush_vehicle* vehicles;
    crush_settings settings;
} crush_model_desc;

/* Per-vehicle result of a run. */
typedef struct crush_vehicle_result {
    double mass;          /* kg, lumped masses without added mass */
    double delta_v[3];    /* m/s, FP64 mass-weighted mean velocity change */
    double velocity[3];   /* m/s, final mass-weighted mean velocity */
    double crush;         /* m */
} crush_vehicle_result;

typedef struct crush_results {
    double time;          /* simulated time reached (s) */
    int64_t steps;
    int64_t eroded_elements;
    double dt_min;        /* smallest step taken */
    double added_mass_max;/* kg, largest total added by mass scaling */
    int32_t status;       /* CRUSH_OK or CRUSH_ERR_NONFINITE */
    int32_t n_vehicles;
    crush_vehicle_result vehicle[4];
} crush_results;

typedef struct crush_ctx crush_ctx;

/* Last error message of the calling thread ("" if none). */
const char* crush_last_error(void);

/* Library and device information: fills name (>= 64 bytes), returns SM count
 * or a negative status. */
int crush_device_info(int device, char* name, int name_len);

/* ---- single-model context: drop-in for the reference's hot-path calls ---- */

/* Upload a model to `device`, run the device geometry precompute
 * (HexGeometry::new, src/element.rs:141), build the node incidence used by the
 * deterministic force gather, lumped masses, contact runtimes and the initial
 * stable step. The desc's arrays may be freed after return. */
int crush_create(const crush_model_desc* desc, int device, crush_ctx** out);
void crush_destroy(crush_ctx* ctx);

/* Sizes of the uploaded model. */
int crush_sizes(const crush_ctx* ctx, int64_t* n_nodes, int64_t* n_hexes, int64_t* n_active_hexes);

/* Element forces at displacement u (host, 3N), committing material states;
 * the nodal sum is ADDED into f_int_accum (host, 3N). `newly_eroded` gets the
 * number of elements that inverted in this call (may be NULL).
 * Replaces Elements::compute_forces (src/kernel.rs:160). */
int crush_compute_forces(crush_ctx* ctx, const double* u, double* f_int_accum, int64_t* newly_eroded);
/* The same with device buffers (3N f64 each); f_int_device is overwritten. */
int crush_compute_forces_device(crush_ctx* ctx, const double* u_device, double* f_int_device, int64_t* newly_eroded);

/* Penalty forces of contact `contact_id` for the configuration X + u, ADDED
 * into f_ext_accum (host, 3N). `masses` are the lumped nodal masses (N) the
 * soft-constraint limit uses; NULL = the context's own. `v` feeds the
 * reference's damping term, whose ratio is the constant 0, so it may be NULL.
 * Replaces ContactRuntime::apply (src/contact.rs:92). */
int crush_contact_apply(crush_ctx* ctx, int contact_id, const double* u, const double* v,
                        const double* masses, double dt, double* f_ext_accum,
                        int64_t* penetration_count, double* max_penetration);

/* Smallest element stability limit f(nu) L / c_d at X + u (host, 3N).
 * Returns CRUSH_NONE (and *dt = +inf) when no element gives a finite limit.
 * Replaces Elements::stable_time_step (src/kernel.rs:207). */
int crush_stable_dt(crush_ctx* ctx, const double* u, double* dt);

/* Selective mass scaling: nodal mass `added` (host, N; overwritten) so that no
 * element's limit falls below dt_min; returns the total in *total.
 * element_mass (host, n_hexes) may be NULL for the context's rho*V.
 * Replaces Elements::mass_scaling (src/kernel.rs:243). */
int crush_mass_scaling(crush_ctx* ctx, const double* u, double dt_min, const double* element_mass,
                       double* added, double* total);

/* Lumped nodal masses (N) and element masses rho*V (n_hexes), host outputs. */
int crush_masses(crush_ctx* ctx, double* lumped, double* element_mass);

/* Per-element f32 data the device derived in set-up, for parity checks:
 * grad (24/hex), volume (1), gamma (32), h (144, column-major as in
 * src/kernel_simd.rs:189), all f32; any pointer may be NULL. */
int crush_element_data(crush_ctx* ctx, float* grad, float* volume, float* gamma, float* h);
/* Material state per element: 25 f32 (F_prev^-1 9, R 9, stress 6, compaction)
 * and eroded flags; set_ writes them back (both host arrays, n_hexes long). */
int crush_get_state(crush_ctx* ctx, float* state, uint8_t* eroded);
int crush_set_state(crush_ctx* ctx, const float* state, const uint8_t* eroded);

/* ---- device-resident run (solver::run, src/solver.rs:190) ---- */
int crush_run(crush_ctx* ctx, crush_results* results);
/* Begin a run (set-up of solver.rs:197-286) without stepping. */
int crush_run_begin(crush_ctx* ctx);
/* Advance an open run by n_steps (fewer if it stops); *done = 1 when finished. */
int crush_run_steps(crush_ctx* ctx, int64_t n_steps, int* done);
/* crush_run_steps with the device time of the steps measured by CUDA events
 * on the context's stream (*ms). With phase_ms (6 doubles) non-NULL the step
 * graph also records events between phases and phase_ms gets the summed
 * device time of each phase (stable dt + mass scaling, contact, half step,
 * element forces, force gather + full step, checks) over the last
 * *phase_steps steps of the call. */
int crush_run_steps_timed(crush_ctx* ctx, int64_t n_steps, int* done, double* ms, double* phase_ms, int* phase_steps);
/* What crush_run_steps_timed's phase events cover: 1 = only the element-force
 * kernel (two events per step, little overhead; phase_ms[3] is filled),
 * 2 = every phase (default). */
int crush_set_profiling(crush_ctx* ctx, int level);
/* Results of the open run so far (final after *done). */
int crush_run_results(crush_ctx* ctx, crush_results* results);
/* Nodal displacement and velocity (host, 3N each; either may be NULL). */
int crush_run_state(crush_ctx* ctx, double* u, double* v);
/* Kernel launches issued by this context since creation. */
int64_t crush_launch_count(const crush_ctx* ctx);
/* Broad-phase statistics of contact `contact_id` accumulated since creation
 * (or the last reset): out[0] primary-node searches of a contact with a grid
 * that tested every face (its overflow list overran), out[1] faces put on the
 * overflow list (key box not finite or beyond the coarsest grid level),
 * out[2] contact-node roles whose reaction sum walked the contact's primary
 * nodes (a per-face hit list overflowed). No counterpart in the reference
 * (whose search is exhaustive). reset != 0 zeroes them after reading. */
int crush_contact_search_stats(crush_ctx* ctx, int contact_id, uint64_t* out, int reset);
/* exhaustive = 1 makes every contact search test every face of its contact,
 * as the reference does (src/contact.rs:115); 0 (default) uses the grids.
 * Both give the same hits: the grids only skip faces that cannot pass the
 * narrow test. For checking that equality; takes effect at the next step. */
int crush_set_contact_search(crush_ctx* ctx, int exhaustive);
/* fused = 1 runs a step whose next step starts with no stable-dt
 * check, record or reduction stop rule as one pass over the nodes (the
 * step's full update and the next step's half step), with the next step's
 * contact forces computed beside this step's element forces; 0 runs every
 * step's half and full updates as separate passes. Both give bit-identical
 * results (for checking that, and for timing the schedules); takes effect
 * at the next step and turns the automatic schedule choice off (see
 * crush_autotune). No counterpart in the reference. */
int crush_set_step_fusion(crush_ctx* ctx, int fused);

/* ---- Time histories: part states and accelerometer samples ----
 * A sampled node set (Accelerometer, src/model.rs:64-73): `nodes` (model
 * node ids) are recorded; with has_frame, also in the body-fixed frame of
 * nodes origin / x_axis / plane (LocalFrame::axes, src/model.rs:45-61). */
typedef struct crush_accelerometer {
    int64_t n_nodes;
    const uint32_t* nodes;
    int32_t has_frame;
    uint32_t origin, x_axis, plane;
} crush_accelerometer;
/* One part's state in one record (PartState, src/solver.rs:23-31): mass
 * (lumped, no added mass) and the mass-weighted means of velocity,
 * displacement and acceleration (net force / mass), and kinetic energy. */
typedef struct crush_part_state {
    double mass;
    double velocity[3];
    double displacement[3];
    double acceleration[3];
    double kinetic_energy;
} crush_part_state;
/* One accelerometer node in one record (a NodeHistory row,
 * src/solver.rs:37-50); local_* repeat the global values without a frame. */
typedef struct crush_node_sample {
    int32_t accelerometer;
    uint32_t node;
    double position[3], displacement[3], velocity[3], acceleration[3];
    double local_displacement[3], local_velocity[3], local_acceleration[3];
} crush_node_sample;
/* Records crash `slot` (0 for crush_create) every history_steps steps, on the
 * device (Settings::history_steps and the record calls of
 * src/solver.rs:283-286, :349-358): one record at step 0, one each step that
 * is a multiple of history_steps, and one at the run's last step when that is
 * not. A record holds time, step, every part's state (parts of the model, in
 * order) and every accelerometer node's sample. Keeps up to max_records per
 * run (later ones are counted, not kept). All configured slots of a context
 * share history_steps; 0 turns a slot's recording off. Call between runs
 * (not while a run is open); the accelerometer arrays are copied. Fixed
 * nodes record zero acceleration (the reference's step-0 record keeps their
 * contact reaction). */
int crush_history_config(crush_ctx* ctx, int slot, int history_steps, int64_t max_records, int n_accelerometers,
                         const crush_accelerometer* accelerometers);
/* Sizes of slot's history of the last (or open) run: records taken
 * (*n_records may exceed the kept ones, min(n_records, max_records)), parts
 * per record and accelerometer nodes per record. Takes the last-step record
 * of a finished crash first if it is due. */
int crush_history_counts(crush_ctx* ctx, int slot, int64_t* n_records, int* n_parts, int64_t* n_node_samples);
/* The kept records: time[k], step[k], parts[k * n_parts + p],
 * samples[k * n_node_samples + j] (any pointer may be NULL). */
int crush_history_get(crush_ctx* ctx, int slot, double* time, int64_t* step, crush_part_state* parts,
                      crush_node_sample* samples);
/* Frames of crash `slot` (Frame and its capture in crushrs::run,
 * src/solver.rs:52-60, :265-281, :345-355; Settings::frame_steps): at step
 * 0, every frame_steps steps and at the last step when that is not a
 * multiple, the device copies the nodal displacement (f32, 3 per node) and
 * per element the plastic strain (honeycomb compaction; 0 for elastic
 * elements), the Cauchy stress R sigma_hat R^T (Voigt xx yy zz xy yz xz,
 * f32; zero when eroded, src/kernel.rs:269-321) and the erosion flag into
 * buffers of max_frames frames (later frames are counted, not kept).
 * Capturing slots of a context share frame_steps; 0 turns a slot off. Call
 * between runs. Node and element indices are the slot's model's. */
int crush_frames_config(crush_ctx* ctx, int slot, int frame_steps, int64_t max_frames);
/* Frames of the last (or open) run taken so far (kept: min with max_frames);
 * takes the last-step frame of a finished crash first if it is due. */
int crush_frames_count(crush_ctx* ctx, int slot, int64_t* n_frames);
/* Kept frame `frame`: time, step, displacement (3 n_nodes), plastic_strain,
 * stress (6 per element), eroded (n_hexes each); any pointer may be NULL. */
int crush_frame_get(crush_ctx* ctx, int slot, int64_t frame, double* time, int64_t* step, float* displacement,
                    float* plastic_strain, float* stress, uint8_t* eroded);
/* SAE J211 channel-frequency-class filter (cfc_filter, src/signal.rs:9-40):
 * a 2-pole Butterworth run forward and backward with reflection padding;
 * y may alias x. n < 4 copies x. */
int crush_cfc_filter(const double* x, int64_t n, double dt, double cfc, double* y);
/* Linear resampling of (t, y) (t ascending) onto t0 + k dt up to t_end
 * (resample, src/signal.rs:42-66): writes min(cap, count) points and the
 * count to *n_out. */
int crush_resample(const double* t, const double* y, int64_t n, double t0, double dt, double t_end, double* tu, double* yu,
                   int64_t cap, int64_t* n_out);

/* Launch schedule of a context, chosen by the engine's autotuner (no
 * counterpart in the reference). The first crush_run_begin of a context times
 * the run's contact pass with 1, 2, 4, 8, 16 and 32 lanes per primary-node search
 * on the context's own models and keeps the fastest; all choices find the
 * same hits. */
typedef struct crush_tuning {
    int32_t slave_lanes;         /* lanes per primary-node search */
    int32_t forces_schedule;     /* element kernel: 0 one persistent wave of blocks taking chunks from a queue,
                                    1 a block per 256 elements, 2 (3) the persistent wave on all but 8 (16) SMs */
    int32_t fused_contact_side;  /* a fused step computes the next step's contact forces 1: on a side stream
                                    beside its element forces, 0: on the main stream after them */
    int32_t step_fusion;         /* fused steps (read only; crush_set_step_fusion sets it) */
    int32_t early_contact;       /* separate steps compute the next step's contact forces beside their element
                                    forces when the next step has no stable-dt check */
    double contact_ms[6];        /* measured contact pass with 1, 2, 4, 8, 16, 32 lanes (0 = not measured) */
    double step_ms[6];           /* measured ms per step of the step graph under the trial's candidates: separate
                                    steps with forces_schedule 2 / 3, the same with early contact forces, fused
                                    steps with 2 / 1; 0 = not measured */
} crush_tuning;
/* Re-tune now, at the open run's current state (e.g. late in a crash, when
 * crushed faces change the search); the next step uses the new schedule.
 * The step schedule is tuned on the run's own steps: a run of a context of
 * 2,000,000+ hexahedra times six candidates (separate steps leaving 8 or 16
 * SMs of the element kernel's wave to the side streams, with or without the
 * next step's contact forces computed there; fused steps with the wave or a
 * block per 256 elements) over its first twelve step graphs, once, and keeps
 * the fastest; smaller contexts take separate steps with 8 SMs left free.
 * The contact lanes are re-tuned every 1000 steps. */
int crush_autotune(crush_ctx* ctx, crush_tuning* out);
int crush_get_tuning(const crush_ctx* ctx, crush_tuning* out);
/* Fixes the schedule to t's slave_lanes, forces_schedule,
 * fused_contact_side and early_contact (measured fields ignored) and turns automatic tuning off for this context. Every
 * schedule gives the same results. */
int crush_set_tuning(crush_ctx* ctx, const crush_tuning* t);

/* ---- batched contexts: many crash models in one context ----
 *
 * No counterpart in the reference, whose unit of work is one model per
 * process (src/bin/crushrs.rs:30). A batch context holds n models ("slots")
 * resident on one GPU; every step is one launch sequence over the nodes and
 * elements of all slots, and each slot carries its own device control block
 * (time, step, stable dt, mass scaling, stop rule), so slots of different
 * sizes and step sizes advance together and each stops on its own rule. The
 * arithmetic of every slot is the arithmetic of the same model run alone:
 * its results are bit-identical to crush_create + crush_run of that model.
 * All models of a batch must share adaptive_check_steps and the time-step
 * mode (fixed time_step or adaptive). The drop-in calls above act on all
 * slots at once (nodes and elements in slot order; contact ids run over the
 * slots' contacts in order); crush_stable_dt then returns the minimum over
 * the slots. crush_create is crush_batch_create with n = 1. */
int crush_batch_create(const crush_model_desc* const* descs, int n, int device, crush_ctx** out);
/* Number of slots of a context (1 for crush_create). */
int crush_batch_size(const crush_ctx* ctx);
/* Run every slot to its stop; results[n] receives each slot's results. */
int crush_batch_run(crush_ctx* ctx, crush_results* results);
/* Results of one slot of the open run (crush_run_begin / crush_run_steps
 * drive all slots; *done = 1 once every slot has stopped). */
int crush_batch_results(crush_ctx* ctx, int slot, crush_results* results);
/* Results of slots [first, first + count) in one pass (one device read). */
int crush_batch_results_range(crush_ctx* ctx, int first, int count, crush_results* results);
/* Which slots of the open run have stopped: done_flags[n] (may be NULL) and
 * *all = 1 when every slot has (may be NULL). Reads a compact flag array the
 * step kernels keep; synchronises the context's stream. */
int crush_batch_done(crush_ctx* ctx, int* done_flags, int* all);

/* ---- continuous batching: slots added to a running context ----
 * No counterpart in the reference. A context created with room to spare
 * (crush_batch_create_reserved) takes more models later
 * (crush_batch_append), also while its run is open: the new slots join the
 * run at its current step and advance with the others from then on, each
 * with its own step 0 (so a slot's results are bit-identical to the same
 * model run alone). The room is fixed at creation: `room` gives the
 * slots, contacts, nodes, hexahedra, contact faces and listed contact nodes
 * (primary nodes) the context must hold in total (at least the initial
 * models' needs; the grid tables, entries and contact-node lists get room in
 * proportion to the faces). */
typedef struct crush_capacity {
    int32_t slots;
    int32_t contacts;
    int64_t nodes;
    int64_t hexes;
    int64_t faces;
    int64_t primary_nodes;
} crush_capacity;
int crush_batch_create_reserved(const crush_model_desc* const* descs, int n, int device, const crush_capacity* room, crush_ctx** out);
/* Runs n models as one batch and writes each one's results to out[k]: the
 * one-call form of crush_batch_create + crush_batch_run, with the set-up
 * pipelined with the run (the first eighth of the elements starts the
 * run; the other models join it group by group at step-graph boundaries,
 * their set-up overlapping the steps in flight). Results are those of each
 * model run alone. The descriptions must stay valid for the call. */
int crush_batch_solve(const crush_model_desc* const* descs, int n, int device, crush_results* out);
/* Adds n models as slots [*first_slot, *first_slot + n). With a run open,
 * only on a step-graph boundary (a multiple of 20 steps: between
 * crush_run_steps calls of multiples of 20 steps, the default issue of
 * crush_run); the call sets the new slots up as crush_run_begin does and
 * searches their contacts for their first step. CRUSH_ERR_BUSY, with
 * nothing added, when the models do not fit the room; CRUSH_ERR_UNSUPPORTED
 * for models with another stable-dt cadence or time-step mode than the
 * context's, or a context recording histories or frames. Synchronises the
 * context's stream. */
int crush_batch_append(crush_ctx* ctx, const crush_model_desc* const* descs, int n, int* first_slot);
/* Issues n_steps steps of the open run on the context's stream and returns
 * without waiting for them (crush_run_steps is this plus the wait and the
 * done flags). Host work done after it, a crush_batch_append's set-up of new
 * slots included, overlaps the steps on the device. */
int crush_run_issue(crush_ctx* ctx, int64_t n_steps);

/* ---- allocation-free contact call ----
 *
 * No counterpart in the reference (its ContactRuntime::new + ::apply,
 * src/contact.rs:48, :92, allocate their face list on every call). For
 * callers that cannot allocate device memory at the point of the call: a
 * solver step loop running inside another framework's memory pool (a
 * cudaMalloc there fails or fragments the pool), or a serving loop
 * overlapping many crashes on streams, where cudaMalloc / cudaFree would
 * synchronise the device. It needs no context either.
 *
 * One ContactRuntime::new filter + ContactRuntime::apply for one contact on
 * device buffers: primary nodes nodes_device[n_nodes] (model node ids) with
 * optional penalty scales node_scale_device[n_nodes] (NULL = 1), quads
 * faces_device[4 * n_faces], reference positions positions_device and
 * displacements u_device (3 * n_model_nodes f64 each), lumped masses
 * masses_device (n_model_nodes). The penalty forces are ADDED into
 * f_accum_device (3 * n_model_nodes f64), each node's contributions in the
 * reference's order starting from the value already there (zero it first for
 * the contact's forces alone). With f_accum zero the result is bit-identical
 * to crush_contact_apply of the same contact.
 *
 * Limits: n_nodes <= CRUSH_STATIC_MAX_NODES and n_faces <=
 * CRUSH_STATIC_MAX_FACES; larger contacts are rejected with
 * CRUSH_ERR_INVALID and a message (use crush_contact_apply). The primary-node
 * search is exhaustive (cost n_nodes x n_faces), and the reaction pass scans
 * the hits once per node occurrence (cost (n_nodes + 4 n_faces) x hits): at
 * the limits one call is of the order of a billion comparisons, so the call
 * suits small and mid-size contacts.
 *
 * Memory: the call allocates nothing, host or device. Its scratch is one
 * fixed-size record (about 5.4 MB) in this library's static device memory,
 * one copy per device. The call clears what it uses at its start, so nothing
 * needs zeroing by the caller. The FIRST call in each CUDA context resolves
 * the record's address (cudaGetSymbolAddress, which may load the library's
 * kernels into the context) and caches it per device with the context's
 * unique id: make that first call with the device current and before any
 * stream capture. A new context on the device (a driver-API context, or the
 * primary context after cudaDeviceReset, which also discards the record)
 * makes the next call resolve the address again, so it counts as a first
 * call. Every call on a device shares the one record, so
 * calls that can overlap in time (other streams or threads without ordering
 * between them) race and corrupt each other's results: serialise them.
 *
 * Asynchronous: six kernel launches on `stream` (a cudaStream_t; NULL = the
 * legacy default stream) of the current device, no copy, no synchronisation.
 * The host checks only sizes and arguments; node ids are checked on the
 * device: an id >= n_model_nodes writes nothing and sets stats->status to
 * CRUSH_ERR_INVALID. stats_device (device memory, may be NULL) receives the
 * penetration count, the largest penetration and that status when the
 * stream reaches the end of the call. */
#define CRUSH_STATIC_MAX_NODES 16384
#define CRUSH_STATIC_MAX_FACES 16384
typedef struct crush_contact_stats {
    int64_t penetration_count;
    double max_penetration;
    int32_t status;
    int32_t reserved;
} crush_contact_stats;
int crush_contact_apply_static(int64_t n_model_nodes, const double* positions_device, const double* u_device,
                               const double* masses_device, int64_t n_nodes, const uint32_t* nodes_device,
                               const double* node_scale_device, int64_t n_faces, const uint32_t* faces_device,
                               double stiffness, double max_distance, double dt, double* f_accum_device,
                               crush_contact_stats* stats_device, void* stream);

#ifdef __cplusplus
}
#endif
#endif
