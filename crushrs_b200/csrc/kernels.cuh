// kernels.cuh — declarations of the engine's CUDA kernels and their
// argument bundles (definitions in kernels.cu).
#pragma once
#include "common.cuh"

namespace crush {

// Work lists of active 256-entity chunks: a kernel given a list visits only
// the chunks on it (the chunks that hold an entity of a crash slot still
// running, rebuilt every 20 steps); a null list means every chunk.
constexpr int CHUNK = 256;
struct Active {
    const int* list;   // chunk indices
    const int* count;  // their number (device)
};

// Element-side device arrays of one model (honeycomb elements only in the
// planes; all model elements in the f64 arrays used by dt / mass scaling).
struct ElementArrays {
    long long n_hc;          // honeycomb elements
    long long stride;        // plane stride (n_hc rounded up)
    const float4* planes;    // N_STATIC_PLANES * stride
    float4* state;           // N_STATE_PLANES * stride
    float* corner;           // 24 floats per honeycomb element (corner forces)
    const MaterialF32* mats;
    long long n_all;         // all model elements
    const uint32_t* conn_all;  // 8 per model element
    const double* dt_factor; // per model element
    const double* elem_mass; // per model element
    uint8_t* eroded_all;     // per model element
    double* elem_dt;         // per model element (written by the dt kernel)
    double* elem_extra;      // per model element added mass (mass scaling)
    const uint32_t* elem_slot;  // crash slot per model element
    Active act_hc, act_all;     // active chunks of honeycomb / all elements
    // Elastic (Hencky) elements: the reference's scalar f64 path
    // (src/kernel.rs:116-156), element order.
    long long n_sc;              // scalar elements visited (a run: those with a free node, numbered first)
    long long sc_stride;         // all scalar elements (the plane stride of sc_geo)
    const uint32_t* sc_model;    // scalar index -> model element
    long long sc_count;          // scalar elements (n_sc: those processed, the length of sc_list when given)
    const uint32_t* sc_list;     // a run: the scalar indices of elastic elements with a free node (null: 0..n_sc)
    const double* sc_geo;        // SC_PLANES x sc_stride (SoA): grad 24, volume, gamma 32, H upper triangle 78
    const double* sc_mat;        // 2 per scalar element: Young's modulus, Poisson ratio
    double* sc_corner;           // 24 per scalar element: corner forces (f64)
    Active act_sc;               // active chunks of scalar elements
};
constexpr int SC_GRAD = 0, SC_VOL = 24, SC_GAMMA = 25, SC_H = 57, SC_PLANES = 135;
constexpr uint32_t HC_ELL_NONE = 0xFFFFFFFFu, HC_ELL_MORE = 0xFFFFFFFEu;

struct NodeArrays {
    long long n;
    const double* pos;       // 3N reference positions
    double* u;
    double* v;
    double* v_half;
    double* f_int;
    double* f_ext;           // the step's external (contact) forces
    double* f_ext_next;      // the next step's, when the step's full update also makes the next step's half step
    double* inv_mass;        // N
    const double* mass;      // N lumped
    double* added;           // N
    const uint8_t* fixed;    // N
    const uint32_t* hc_off;  // N+1 CSR over honeycomb (element, corner) slots, element order
    const uint4* hc_ell;     // N x 2 uint4: the node's first 8 of those slots, HC_ELL_NONE padding,
                             // HC_ELL_MORE first when it has more (then the CSR)
    const uint32_t* hc_slot;
    const uint32_t* all_off; // N+1 CSR over all model (element, corner) slots
    const uint32_t* all_slot;
    const uint32_t* sc_off;  // N+1 CSR over scalar (element, corner) slots, element order
    const uint32_t* sc_slot;
    const uint32_t* node_slot;  // crash slot per node
    const int* mass_flag;       // set when some crash scales its masses this step
    Active act_node;            // active chunks of nodes
};

// A face's key-box cells at its grid level (level -1: no inserts,
// GRID_LEVELS: a big face), written by the face pass for the fill pass.
struct FaceCells {
    long long lo[3];
    int span[3];
    int level;
};

// Contact runtime arrays (all contacts concatenated).
struct FaceGeo {
    double x[4][3];
    double n[3];
    double c[3];
    double lo[3];
    double hi[3];
};

// Reaction events per contact node: EV_CAP keys in the node's own list, the
// rest in a shared pool; CN_FIXED marks a fixed node in slave_cn / face_cn.
constexpr int EV_CAP = 16;
constexpr uint32_t CN_FIXED = 0x80000000u;
// Dynamic grids are hashed and hierarchical: level l has cells of size
// cell * 4^l, and a face goes into the finest level where its key box covers
// at most LEVEL_CELL_BUDGET cells. Buckets are exact CSR ranges rebuilt every
// step (count, allocate, fill), so a contact needs at most faces x
// LEVEL_CELL_BUDGET entries and no bucket ever overflows. A face whose key
// box fits no level (a stretched face: one of its nodes flew off with
// eroded elements) is a big face: one pass per big face tests it against
// every primary node of its contact, and the primary-node search starts
// from the smallest big face that hit (big_best).
constexpr int GRID_LEVELS = 2;
constexpr int LEVEL_CELL_BUDGET = 64;
constexpr int BIG_NONE = 0x7F7F7F7F;  // big_best of a primary node no big face hit (memset byte 0x7F)

struct ContactArrays {
    int n_contacts;
    const int* face_off;        // n_contacts+1
    const uint32_t* faces;      // 4 per face (global face index)
    FaceGeo* geo;               // per face
    const int* slave_off;       // n_contacts+1
    const uint32_t* slaves;     // node id per primary node
    const double* slave_scale;
    int* hit;                   // per primary node: local face index or -1 (written by the search)
    double* hit_sd;             // per primary node: signed distance to that face
    double* hit_force;          // 3 per primary node
    const double* stiffness;    // per contact
    const double* max_distance; // per contact
    const double* cell;         // per contact grid cell size
    const int* tab_off;         // n_contacts+1, hash tables concatenated (each a power of two, >= 1024)
    int* counts;                // per bucket: faces to insert this step (zero again after the fill)
    unsigned* boff;             // per bucket: start of its range in entries
    int* blen;                  // per bucket: length of its range
    const long long* ent_off;   // n_contacts+1: entry capacity ranges (faces x LEVEL_CELL_BUDGET)
    int* ent_cursor;            // per contact: entries allocated this step
    int* grid_state;            // levels_used (contact_room), ent_cursor (contact_room), big_count (1): cleared per search
    long long contact_room;     // contacts the per-contact arrays have room for (>= n_contacts)
    FaceCells* cells;           // per face: its cells this search (faces of contacts with a dynamic grid)
    int* entries;               // local face indices
    uint32_t* big_faces;        // this search's big faces (global index), capacity big_cap
    double* big_box;            // 6 per big face: its key box (lo xyz, hi xyz)
    int* big_count;             // big faces listed this search
    long long big_cap;          // faces of the contacts with a dynamic grid
    int* big_best;              // per primary node: smallest local big face that hit, or BIG_NONE
    unsigned long long* search_stats;  // 3 per contact, accumulated: (unused: 0), big faces
                                       // searched face by face, contact-node roles gathered by
                                       // walking the primary nodes (per-face hit lists overflowed)
    unsigned long long* pen_count;  // per contact, per step
    unsigned long long* pen_max_bits;
    const int* counts_for_stop; // per contact: faces not all fixed
    // contact-node gather: nodes with roles in contacts, and the reaction
    // events the force pass appends to per-node lists
    long long n_cnodes;
    const uint32_t* cnode;      // node id
    const uint32_t* cnode_off;  // n_cnodes+1: range of the node's roles
    const int* crole_contact;   // per role: contact id
    const int* crole_slave;     // per role: position among the contact's primary nodes (-1 none)
    const uint32_t* slave_cn;   // per primary-node entry: contact node of its node (| CN_FIXED if fixed)
    const uint32_t* face_cn;    // 4 per face: contact node of each corner (| CN_FIXED if fixed)
    int* ev_count;              // per contact node: events this pass (zeroed again by the gather)
    uint32_t* ev_list;          // EV_CAP event keys per contact node
    uint2* ev_pool;             // (contact node, key) of the events past a full list
    int* ev_pool_n;             // [0] pool entries, [1] heavy contact nodes (= gather_count)
    long long ev_pool_cap;
    const int* face_contact;    // contact of each face
    const int* slave_contact;   // contact of each primary node entry
    const int* contact_slot;    // crash slot of each contact
    const int* slot_contact_off;// n_slots+1: contacts of each crash slot
    int n_slots;
    int* levels_used;           // per contact: bit l set when a face went to grid level l this step
    // Static contacts (every face node fixed): geometry computed once per run
    // and an exact hashed grid built at set-up, in CSR form.
    const uint8_t* is_static;   // per contact
    const long long* st_tab_off;// n_contacts+1: bucket ranges of the static tables (power of two each, or 0)
    const uint32_t* st_off;     // per bucket + 1 per table: CSR offsets into st_entries
    const int* st_entries;      // local face indices, ascending within a bucket
    const uint32_t* dyn_faces;  // global indices of the faces of non-static contacts
    long long n_dyn_faces;
    const uint32_t* grid_faces; // global indices of the faces of contacts with a dynamic grid
    long long n_grid_faces;
    long long n_buckets;        // total dynamic buckets (tab_off[n_contacts])
    int exhaustive;             // 1: every search tests every face of its contact (no broad phase)
    int* gather_work;           // contact nodes with over EV_CAP events this pass (n_cnodes capacity)
    int* gather_count;          // their number (ev_pool_n + 1)
    Active act_slave, act_cnode, act_dynf;  // active chunks of grid-searched entries, contact nodes, moving faces
    Active act_allslave;        // active chunks of all primary-node entries (the force pass)
    Active act_stslave;         // active chunks of st_slaves
    // Contacts without a grid are searched by one block each; the entries of
    // the others are listed for the lane-parallel search.
    const int* brute_contacts;
    int n_brute;
    int brute_max_faces;        // most faces of a listed contact (its shared-memory stage)
    const double* st_box;       // 6 per contact: union of a static contact's key boxes (lo xyz, hi xyz)
    const uint32_t* grid_slaves;  // entries searched with the tuned lane count (dynamic grids, no usable grid)
    long long n_grid_slaves;
    const uint32_t* st_slaves;    // entries of contacts with a static grid (searched with ST_LANES lanes)
    long long n_st_slaves;
    const uint8_t* is_brute_h;  // host copy, per contact (launchers only)
};

// Chunks of every entity space with the crash-slot range each covers, and
// the active lists built from them.
struct ActiveBuild {
    long long n_chunks;          // all spaces together
    const int* chunk_lo;         // first and last slot of each chunk
    const int* chunk_hi;
    const long long* space_off;  // ACTIVE_SPACES + 1 chunk offsets
    int* lists;                  // same layout as the chunks
    int* counts;                 // ACTIVE_SPACES
};
constexpr int ACTIVE_SPACES = 9;  // honeycomb elements, all elements, nodes, searched entries (dynamic grids and the
                                  // rest), contact nodes, moving faces, all primary-node entries, static-grid entries,
                                  // scalar elements

// Vehicles of all crash slots: node lists and the reduction layout.
struct VehicleArrays {
    int n_vehicles;
    const long long* off;       // n_vehicles+1 into nodes
    const uint32_t* nodes;
    const int* slot;            // crash slot of each vehicle
    const int* local;           // index of the vehicle within its slot (0..3)
    int vx_blocks;              // blocks per vehicle for the separation-rule reduction (<= 64)
};

// Every launcher takes the array of per-crash control blocks (`ctls`, one
// per crash slot); entities find their slot through the *_slot arrays.
// Elements [e_begin, n_all).
void launch_setup_geometry(cudaStream_t s, long long e_begin, long long n_all, const double* pos, const uint32_t* conn_all,
                           const int32_t* part, const double* mat_e_nu_rho_hg, const int64_t* hc_index,
                           const uint32_t* elem_slot, long long stride, float4* planes, double* volume, double* lumped,
                           double* dt_factor, double* elem_mass, int* bad, const int64_t* sc_index, long long n_sc,
                           double* sc_geo);
void launch_node_masses(cudaStream_t s, long long n, const uint32_t* off, const uint32_t* slot, const double* lumped,
                        double* mass, double* inv_mass);
void launch_init_state(cudaStream_t s, long long h_begin, long long n_hc, long long stride, float4* state);
// Node incidence of new elements [e0, e0 + ne) over their nodes [n0, n0 + nn)
// on the device: per node its (element, corner) slots in element order (a
// stable radix sort by node), in all elements (all_off / all_slot), split
// into honeycomb and elastic lists, and the padded honeycomb rows. The
// offset arrays and hc_ell point at the new nodes' first entries, the slot
// arrays at their context-wide start (base_* = the new entries' first global
// position). scratch holds incidence_scratch_bytes(ne, nn). Returns 0, or -1
// on a CUDA error.
size_t incidence_scratch_bytes(long long ne, long long nn);
int launch_incidence(cudaStream_t s, long long e0, long long ne, long long n0, long long nn, const uint32_t* conn_all,
                     const int64_t* hc_index, const int64_t* sc_index, uint32_t base_all, uint32_t base_hc, uint32_t base_sc,
                     uint32_t* all_off, uint32_t* all_slot, uint32_t* hc_off, uint32_t* hc_slot, uint32_t* sc_off, uint32_t* sc_slot,
                     uint32_t* hc_ell, void* scratch);
// Element forces: the honeycomb lane kernel and, when the model has
// elastic elements, the scalar f64 kernel (forces_launches of them).
// schedule: 0 = one persistent wave of blocks on the n_sms SMs, 1 = a block
// per chunk of 256 elements, 2 (3) = the persistent wave on all but 8 (16)
// SMs; all compute the same bits. queue (two zeroed unsigned, left zero): the
// persistent waves take chunks from it (null: they stride).
void launch_forces(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, Control* ctls, int respect_done, int n_sms = 148,
                   int schedule = 0, unsigned* queue = nullptr);
int forces_launches(const ElementArrays& el);
void launch_gather(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, double* f_out);
void launch_half(cudaStream_t s, const NodeArrays& nd, Control* ctls);
void launch_full(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, Control* ctls);
// Elements [e_begin, el.n_all) (e_begin > 0: no active list).
void launch_elem_dt(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, Control* ctls, const double* u, int respect_done,
                    long long e_begin = 0);
// mass_flag: set when a crash scales its masses this step (k_mass_scaling
// does nothing otherwise), cleared by the step's end.
void launch_dt_finalize(cudaStream_t s, Control* ctls, int n_slots, int* mass_flag);
void launch_mass_scaling(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, Control* ctls, int force_apply);
void launch_nonfinite(cudaStream_t s, const NodeArrays& nd, Control* ctls);
void launch_build_active(cudaStream_t s, const ActiveBuild& b, const Control* ctls);
void launch_step_end(cudaStream_t s, Control* ctls, const ContactArrays& ca, const VehicleArrays& va, int check_separation,
                     int* done_out, int* mass_flag);
// A step's full update fused with the next step's half step, for steps
// after which no stable-dt check, record or reduction stop rule comes: one
// pass over the nodes (the ordered corner-force gather, v, then v_half and u
// of the next step from nd.f_ext_next), and the step's end for every slot
// in the last block to finish (block_counter: one zeroed int, left zero).
void launch_fused(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, Control* ctls, const ContactArrays& ca,
                  const VehicleArrays& va, int* done_out, int* mass_flag, unsigned* block_counter);
// Contact pass over contacts [c0, c1) (faces [f0, f0 + n_faces), n_slaves
// primary-node entries, dynamic grid buckets [bk0, bk1)); `lanes` lanes per
// primary-node search (4, 8, 16 or 32). dt_override > 0 is a drop-in call: every face's
// geometry is rebuilt and static contacts are searched exhaustively; the run
// (dt_override = 0) rebuilds only the dynamic faces and uses the static grids.
void launch_contact(cudaStream_t s, const ContactArrays& ca, const NodeArrays& nd, Control* ctls, int c0, int c1, long long f0,
                    long long n_faces, long long n_slaves, long long bk0, long long bk1, double dt_override, const double* masses,
                    double* f_out, int skip_fixed, int lanes);
// Kernel launches one launch_contact call issues.
int contact_launches(const ContactArrays& ca, bool run_mode, long long n_faces, long long n_slaves, long long bk0, long long bk1,
                     int c0);
// The two halves of a contact pass. The search (face geometry, grids, first
// hits) needs only X + u and may run while other work of the step runs; the
// finish (forces of the hits with the step's dt, hit lists, counters, the
// ordered gather into f_out) follows it. A run's finish with next_step = 1
// is the next step's pass, run beside this step's element forces: it takes
// the next step's dt (next_step_dt).
// s_static (optional): the stream for the static-grid entries' search,
// which needs nothing else the search builds.
void launch_contact_search(cudaStream_t s, const ContactArrays& ca, const NodeArrays& nd, Control* ctls, int c0, int c1, long long f0,
                           long long n_faces, long long n_slaves, long long bk0, long long bk1, int run_mode, int lanes,
                           cudaStream_t s_static = nullptr);
void launch_contact_finish(cudaStream_t s, const ContactArrays& ca, const NodeArrays& nd, Control* ctls, int c0, int c1, long long f0,
                           long long n_faces, long long n_slaves, double dt_override, const double* masses, double* f_out,
                           int skip_fixed, cudaStream_t s_heavy = nullptr, cudaEvent_t ev_a = nullptr,
                           cudaEvent_t ev_b = nullptr, cudaEvent_t ev_c = nullptr, int next_step = 0);
int contact_search_launches(const ContactArrays& ca, bool run_mode, long long n_faces, long long n_slaves, long long bk0, long long bk1,
                            int c0);
int contact_finish_launches(long long n_slaves);
// Geometry of every face of contacts [c0, c1) at X + u (no grid insertion):
// the static contacts' geometry for a run.
void launch_contact_geometry(cudaStream_t s, const ContactArrays& ca, const NodeArrays& nd, int c0, int c1, long long f0,
                             long long n_faces);
void launch_vehicle_sums(cudaStream_t s, const VehicleArrays& va, const double* mass, const double* v, const double* v0,
                         double* out7);
void launch_vehicle_vx(cudaStream_t s, const VehicleArrays& va, const double* mass, const double* v, Control* ctls);
void launch_gather_ux(cudaStream_t s, long long n, const uint32_t* nodes, const double* u, double* out);

// Fixed-size scratch of the allocation-free contact call
// (crush_contact_apply_static): one record in a static device array, so the
// call needs no allocation. Limits: STATIC_MAX_NODES primary nodes (before
// the bounding-box filter) and STATIC_MAX_FACES faces per call.
constexpr int STATIC_MAX_NODES = 16384;
constexpr int STATIC_MAX_FACES = 16384;
constexpr int STATIC_MAX_OCC = STATIC_MAX_NODES + 4 * STATIC_MAX_FACES;  // node occurrences
struct StaticContactScratch {
    FaceGeo geo[STATIC_MAX_FACES];
    double hit_force[3 * STATIC_MAX_NODES];
    double occ[3 * STATIC_MAX_OCC];    // new force value of the node of each occurrence
    int hit[STATIC_MAX_NODES];         // face hit by each primary node entry, or -1
    int hit_list[STATIC_MAX_NODES];    // entries that hit, in entry order
    double box_lo[3], box_hi[3];       // primary-node filter box (reference positions)
    unsigned long long pen_count, pen_max_bits;
    int n_hits;
    int error;                         // 1: a node id was out of range (nothing is written)
};

// ---- Time histories (part states and accelerometer samples) ----
// A part unit is one (crash slot, part) pair of a slot that records; its
// nodes (the part's element nodes, ascending, src/mesh.rs:74-82) are reduced
// by HIST_BLOCKS blocks into fixed-order partial sums, which the finishing
// kernel adds in block order. Records are kept per slot in arrays of
// max_rec entries.
constexpr int HIST_BLOCKS = 32;
constexpr int HIST_PART_VALUES = 11;  // mass, velocity 3, displacement 3, acceleration 3, kinetic energy
constexpr int HIST_NODE_VALUES = 21;  // position, displacement, velocity, acceleration, local u, v, a (3 each)
enum HistMode { HIST_INITIAL = 0, HIST_STEP = 1, HIST_FINAL = 2 };
struct HistoryArrays {
    int n_slots;
    int steps;                  // history_steps shared by the recording slots
    long long max_rec;          // record capacity per slot (the stride of the record arrays)
    const int* slot_on;         // per slot: records
    const long long* slot_max;  // per slot: records kept
    const int* slot_pu_off;     // n_slots+1: the slot's part units
    const int* slot_an_off;     // n_slots+1: the slot's accelerometer nodes
    int n_pu;
    const uint32_t* pu_off;     // n_pu+1 into pu_nodes
    const uint32_t* pu_nodes;   // global node ids
    const int* pu_slot;
    double* partial;            // n_pu x HIST_BLOCKS x HIST_PART_VALUES
    int n_an;
    const uint32_t* an_node;    // global node id of each accelerometer node
    const int* an_frame;        // frame of its accelerometer (-1: none)
    const uint32_t* fr_nodes;   // 3 global node ids (origin, x axis, plane) per frame
    long long* rec_count;       // per slot: records taken this run
    long long* last_step;       // per slot: step of the last record (-1: none)
    double* rec_time;           // n_slots x max_rec
    long long* rec_step;        // n_slots x max_rec
    double* part_rec;           // n_pu x max_rec x HIST_PART_VALUES
    double* node_rec;           // n_an x max_rec x HIST_NODE_VALUES
};
// One record of every slot that is due (mode: the run's first record, a
// step record every `steps` steps, or the last-step record of a finished
// crash). f_ext is the external force the accelerations use.
// HIST_FINAL records take each slot's last step's forces: f_ext when that
// step (ctl->step - 1) is even, f_ext_odd when it is odd.
void launch_history(cudaStream_t s, const HistoryArrays& h, const NodeArrays& nd, const Control* ctls, const double* f_ext, int mode,
                    const double* f_ext_odd = nullptr);

// ---- Frames: nodal displacement and element plastic strain, Cauchy
// stress and erosion every frame_steps steps (Frame, src/solver.rs) ----
struct FrameArrays {
    int n_slots;
    int steps;                  // frame_steps shared by the capturing slots
    long long stride;           // frame capacity per slot (stride of time / step)
    const int* slot_on;
    const long long* slot_max;  // frames kept per slot
    const long long* node0;     // per slot: first node, node count
    const long long* n_nodes;
    const long long* elem0;     // per slot: first model element, element count
    const long long* n_elems;
    const long long* disp_base; // per slot: float offset of its frames' displacements (max x 3 n_nodes)
    const long long* elem_base; // per slot: offset of its frames' element records (max x n_elems)
    long long* count;           // per slot: frames taken this run
    long long* last_step;       // per slot: step of the last frame (-1: none)
    double* time;               // n_slots x stride
    long long* step;
    float* disp;                // displacement (f32 of u)
    float* pstrain;             // plastic strain (compaction; 0 for elastic elements)
    float* stress;              // Cauchy stress, Voigt xx yy zz xy yz xz (0 when eroded)
    uint8_t* eroded;
    const int64_t* hc_index;    // model element -> honeycomb index or -1
    const uint8_t* eroded_all;  // per model element
    const float4* state;        // honeycomb state planes
    long long state_stride;
    int node_blocks, elem_blocks;  // blocks per slot of the two copy kernels
    // elastic elements: Hencky stress at the current u
    const int64_t* sc_index;    // model element -> scalar index or -1 (null: none)
    long long n_sc;
    const double* sc_geo;
    const double* sc_mat;
    const uint32_t* conn_all;
    const double* pos;
};
// One frame of every slot that is due (modes as for the histories).
void launch_frames(cudaStream_t s, const FrameArrays& f, const double* u, const Control* ctls, int mode);

// The call's kernels on `s`; every count is within the limits above.
void launch_contact_static(cudaStream_t s, StaticContactScratch* sc, long long n_model_nodes, const double* pos, const double* u,
                           const double* masses, long long n_nodes, const uint32_t* nodes, const double* node_scale,
                           long long n_faces, const uint32_t* faces, double stiffness, double max_distance, double dt,
                           double* f_accum, int64_t* stats_count, double* stats_max, int* stats_status);

}  // namespace crush
