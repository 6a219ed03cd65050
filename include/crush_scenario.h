/*
 * crush_scenario.h — host-side model builders of the B200 crash engine.
 *
 * They restate the reference's block-vehicle scenario construction so a model
 * built here is the model crushrs would build (paths relative to the crushrs
 * source tree):
 *   structured hexahedral blocks      Mesh::add_hex_block(_n)   src/mesh.rs:111-171
 *   vehicle block + materials         add_vehicle / assign_vehicle src/vehicle.rs:663, :750
 *   road slab + road contact          add_ground / add_ground_contact src/vehicle.rs:829, :838
 *   penalty stiffness per node        contact_stiffness_per_node src/vehicle.rs:384
 *   two-way front contact             Model::add_contact_pair_scaled src/model.rs:257
 *   head-on / rear-end layout         HeadOn::build src/headon.rs:40 (rear-end: src/bin/crushrs.rs:522)
 *   T-bone layout                     src/bin/crushrs.rs:550-576
 *   rail box                          rail_box_factors / front_contact_scales src/vehicle.rs:367, :397
 *   rear-seat accelerometer node      add_vehicle_accelerometer src/vehicle.rs:792
 * The result is a crush_model whose crush_model_desc feeds crush_create (and
 * the test oracle).
 */
#ifndef CRUSH_SCENARIO_H
#define CRUSH_SCENARIO_H

#include "crush.h"

#ifdef __cplusplus
extern "C" {
#endif

/* A crushable vehicle (the reference's Vehicle, src/vehicle.rs:107-196):
 * a homogeneous honeycomb block, or with crush_zone_length in (0, length)
 * the two-part vehicle of add_vehicle / assign_vehicle (src/vehicle.rs:663-790):
 * an elastic body (part <name>), a honeycomb crush zone in front of it
 * (<name>_crush), an optional elastic bumper layer at the very front
 * (<name>_bumper), and an optional rail box carved out of the crush zone
 * (<name>_rails) and the bumper (<name>_bumper_rails). */
typedef struct crush_vehicle_spec {
    double mass;             /* kg */
    double size[3];          /* length (x), width (y), height (z), m */
    crush_material material; /* crush material; density <= 0 means the crush zone's mass / volume */
    double contact_modulus;  /* modulus for the penalty stiffness (Pa); <= 0: material E */
    int32_t has_rail_box;    /* carve a rail box (a homogeneous block: out of the whole block) */
    double rail_box_width;   /* m, centred on the block */
    double rail_box_z[2];    /* m above the block bottom */
    double rail_box_force_fraction;
    double crush_zone_length;  /* m, bumper included; <= 0 or >= length: the whole block is the crush zone */
    double body_modulus;       /* Pa, the elastic body's modulus (Poisson ratio 0.3, Vehicle::body_material) */
    double crush_zone_mass;    /* kg of the crush zone with its bumper; <= 0: uniform density */
    double bumper[3];          /* thickness m, mass kg, modulus Pa of the bumper layer; thickness <= 0: none */
    double crush_element_size; /* m along x inside the crush zone; <= 0: the block element size */
} crush_vehicle_spec;

#define CRUSH_LAYOUT_HEADON 0 /* A heads +x, B heads -x, noses 2*5 mm apart (rear-end: negative speed_b) */
#define CRUSH_LAYOUT_TBONE 1  /* A heads +x into the -x side of B; B is given as its side profile */
#define CRUSH_LAYOUT_BARRIER 2 /* A heads +x into a fixed rigid wall at x = 0 (barrier_model, src/vehicle.rs:951); B unused */

typedef struct crush_scenario {
    int32_t layout;
    crush_vehicle_spec a, b;
    double speed_a;       /* m/s along +x */
    double speed_b;       /* head-on: m/s along -x; T-bone: m/s along +y */
    double offset;        /* head-on: lateral offset of B (m); T-bone: B's centre at y = -offset */
    double clearance;     /* road this far below the underbodies (m); < 0: no road */
    double element_size;  /* m */
    crush_settings settings;
} crush_scenario;

typedef struct crush_model crush_model;

/* Defaults of Settings::default (src/model.rs:134) with the given end time. */
crush_settings crush_settings_default(double end_time);

/* Build a scenario; *out is freed with crush_model_free. */
int crush_scenario_build(const crush_scenario* s, crush_model** out);
void crush_model_free(crush_model* m);
/* A view of the model's arrays (valid until crush_model_free). */
int crush_model_desc_get(const crush_model* m, crush_model_desc* out);
/* Mutable settings of a built model. */
crush_settings* crush_model_settings(crush_model* m);
/* The body-fixed frame of vehicle `vehicle`'s accelerometer (origin, x-axis
 * and plane nodes, Model::add_accelerometer_at, src/model.rs:185-214), for
 * crush_history_config: the rear-seat pulse of src/vehicle.rs:792-822. */
int crush_model_vehicle_frame(const crush_model* m, int32_t vehicle, uint32_t frame[3]);

/* Generic block builder (Mesh::add_hex_block_n, src/mesh.rs:117) on an empty
 * model, for tests: adds one block as part `part`; `surfaces` is a bit mask of
 * block faces (1 XMin, 2 XMax, 4 YMin, 8 YMax, 16 ZMin, 32 ZMax) whose quads
 * are appended as a face set. */
int crush_model_new(crush_model** out);
int crush_model_add_block(crush_model* m, const double origin[3], const double size[3], const int32_t n[3],
                          int32_t surfaces, int32_t* part_out);
/* Face set `k` of the model (quads as 4 node ids): count and copy-out. */
int crush_model_face_set(const crush_model* m, int32_t k, int64_t* n_faces, uint32_t* faces);
/* Replace the materials / add fixed nodes / set initial velocities of a generic model. */
int crush_model_set_materials(crush_model* m, int32_t n, const crush_material* mats);
int crush_model_set_velocity(crush_model* m, const double* v3n);

#ifdef __cplusplus
}
#endif
#endif
