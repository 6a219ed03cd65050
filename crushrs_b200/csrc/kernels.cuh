// kernels.cuh — declarations of the engine's CUDA kernels and their
// argument bundles (definitions in kernels.cu).
#pragma once
#include "common.cuh"

namespace crush {

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
};

struct NodeArrays {
    long long n;
    const double* pos;       // 3N reference positions
    double* u;
    double* v;
    double* v_half;
    double* f_int;
    double* f_ext;
    double* inv_mass;        // N
    const double* mass;      // N lumped
    double* added;           // N
    const uint8_t* fixed;    // N
    const uint32_t* hc_off;  // N+1 CSR over honeycomb (element, corner) slots, element order
    const uint32_t* hc_slot;
    const uint32_t* all_off; // N+1 CSR over all model (element, corner) slots
    const uint32_t* all_slot;
};

// Contact runtime arrays (all contacts concatenated).
struct FaceGeo {
    double x[4][3];
    double n[3];
    double c[3];
    double lo[3];
    double hi[3];
};

// Grid buckets hold up to BUCKET_CAP faces (a fuller bucket makes its
// primary nodes test every face of the contact); per-face hit lists hold
// FACE_HIT_CAP primary nodes (fuller lists make the gather walk the contact's
// primary nodes in order).
constexpr int BUCKET_CAP = 64;
constexpr int FACE_HIT_CAP = 8;

struct ContactArrays {
    int n_contacts;
    const int* face_off;        // n_contacts+1
    const uint32_t* faces;      // 4 per face (global face index)
    FaceGeo* geo;               // per face
    const int* slave_off;       // n_contacts+1
    const uint32_t* slaves;     // node id per primary node
    const double* slave_scale;
    int* hit;                   // per primary node: local face index or -1
    double* hit_force;          // 3 per primary node
    const double* stiffness;    // per contact
    const double* max_distance; // per contact
    const double* cell;         // per contact grid cell size
    const int* tab_off;         // n_contacts+1, hash tables concatenated (each a power of two)
    int* counts;                // per bucket: faces inserted this step
    int* entries;               // BUCKET_CAP local face indices per bucket
    int* overflow;              // per contact: faces whose key box spans too many cells
    int* n_overflow;            // per contact
    int* entry_overrun;         // per contact flag: overflow list full (search every face)
    int overflow_cap;           // per contact capacity of overflow
    unsigned long long* pen_count;  // per contact, per step
    unsigned long long* pen_max_bits;
    const int* counts_for_stop; // per contact: faces not all fixed
    // contact-node gather: nodes with roles in contacts
    long long n_cnodes;
    const uint32_t* cnode;      // node id
    const uint32_t* cnode_off;  // n_cnodes+1
    const int* crole_contact;   // per role: contact id
    const int* crole_slave;     // per role: position among the contact's primary nodes (-1 none)
    const uint8_t* crole_face;  // per role: node belongs to a face of the contact
    const uint32_t* crole_faces_off;  // per role + 1: range in crole_faces
    const int* crole_faces;     // local indices of the contact's faces that contain the node
    int* face_hits;             // per face: primary nodes hitting it this step
    int* face_list;             // FACE_HIT_CAP primary nodes (global index) per face
};

void launch_setup_geometry(cudaStream_t s, long long n_all, const double* pos, const uint32_t* conn_all,
                           const int32_t* part, const double* mat_e_nu_rho, double hourglass, const int64_t* hc_index,
                           long long stride, float4* planes, double* volume, double* lumped, double* dt_factor,
                           double* elem_mass, int* bad);
void launch_node_masses(cudaStream_t s, long long n, const uint32_t* off, const uint32_t* slot, const double* lumped,
                        double* mass, double* inv_mass);
void launch_init_state(cudaStream_t s, long long n_hc, long long stride, float4* state);
void launch_forces(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, Control* ctl, int respect_done);
void launch_gather(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, double* f_out);
void launch_half(cudaStream_t s, const NodeArrays& nd, Control* ctl);
void launch_full(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, Control* ctl);
void launch_elem_dt(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, Control* ctl, const double* u,
                    double* block_partials, int respect_done);
int elem_dt_blocks(long long n_all);
void launch_dt_finalize(cudaStream_t s, Control* ctl, const double* block_partials, int n_blocks);
void launch_mass_scaling(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, Control* ctl, int force_apply);
void launch_nonfinite(cudaStream_t s, const NodeArrays& nd, Control* ctl);
void launch_step_end(cudaStream_t s, Control* ctl, const ContactArrays& ca, int check_separation);
void launch_contact(cudaStream_t s, const ContactArrays& ca, const NodeArrays& nd, Control* ctl, int c0, int c1,
                    long long n_faces, long long n_slaves, int entries_cap, double dt_override, const double* masses,
                    double* f_out, int skip_fixed);
void launch_vehicle_sums(cudaStream_t s, int n_veh, const long long* veh_off, const uint32_t* veh_nodes,
                         const double* mass, const double* v, const double* v0, double* out5);
void launch_vehicle_vx(cudaStream_t s, int n_veh, const long long* veh_off, const uint32_t* veh_nodes,
                       const double* mass, const double* v, Control* ctl);

}  // namespace crush
