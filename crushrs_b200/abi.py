"""ctypes mirror of include/crush.h and include/crush_scenario.h.

The structures here are field-for-field the C structs of the engine's C ABI,
so Python callers (the tests, bench.py) pass the same descriptors a C, C++ or
Rust caller would.
"""
import ctypes as C

MAX_KNOTS = 8

CRUSH_OK = 0
CRUSH_NONE = 1
CRUSH_ERR_INVALID = -1
CRUSH_ERR_NONFINITE = -2
CRUSH_ERR_OOM = -3
CRUSH_ERR_TIMEOUT = -4
CRUSH_ERR_CUDA = -5
CRUSH_ERR_UNSUPPORTED = -6
CRUSH_ERR_BUSY = -7

MAT_HONEYCOMB = 0
MAT_ELASTIC = 1
STOP_END_TIME = 0
STOP_SEPARATION = 1
LAYOUT_HEADON = 0
LAYOUT_TBONE = 1
LAYOUT_BARRIER = 2

STATUS_NAMES = {
    CRUSH_OK: "OK", CRUSH_NONE: "NONE", CRUSH_ERR_INVALID: "INVALID", CRUSH_ERR_NONFINITE: "NONFINITE",
    CRUSH_ERR_OOM: "OOM", CRUSH_ERR_TIMEOUT: "TIMEOUT", CRUSH_ERR_CUDA: "CUDA",
    CRUSH_ERR_UNSUPPORTED: "UNSUPPORTED", CRUSH_ERR_BUSY: "BUSY",
}


class Material(C.Structure):
    _fields_ = [
        ("model", C.c_int32),
        ("youngs_modulus", C.c_double),
        ("poisson_ratio", C.c_double),
        ("density", C.c_double),
        ("yield_stress", C.c_double),
        ("hardening", C.c_double),
        ("n_curve", C.c_int32),
        ("curve", (C.c_double * 2) * MAX_KNOTS),
        ("has_densification", C.c_int32),
        ("densification", C.c_double * 2),
        ("transverse_factor", C.c_double),
    ]


class Contact(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int64),
        ("nodes", C.POINTER(C.c_uint32)),
        ("node_scale", C.POINTER(C.c_double)),
        ("n_faces", C.c_int64),
        ("faces", C.POINTER(C.c_uint32)),
        ("stiffness", C.c_double),
        ("max_distance", C.c_double),
    ]


class Settings(C.Structure):
    _fields_ = [
        ("end_time", C.c_double),
        ("dt_scale", C.c_double),
        ("time_step", C.c_double),
        ("adaptive_check_steps", C.c_int32),
        ("hourglass", C.c_double),
        ("velocity_damping", C.c_double),
        ("mass_scaling", C.c_double),
        ("stop_rule", C.c_int32),
        ("max_steps", C.c_int32),
    ]


class Vehicle(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int64),
        ("nodes", C.POINTER(C.c_uint32)),
        ("accel_node", C.c_uint32),
        ("n_front", C.c_int64),
        ("front_nodes", C.POINTER(C.c_uint32)),
    ]


class ModelDesc(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int64),
        ("positions", C.POINTER(C.c_double)),
        ("n_hexes", C.c_int64),
        ("hexes", C.POINTER(C.c_uint32)),
        ("hex_part", C.POINTER(C.c_int32)),
        ("n_parts", C.c_int32),
        ("materials", C.POINTER(Material)),
        ("initial_velocity", C.POINTER(C.c_double)),
        ("n_fixed", C.c_int64),
        ("fixed_nodes", C.POINTER(C.c_uint32)),
        ("n_contacts", C.c_int32),
        ("contacts", C.POINTER(Contact)),
        ("n_vehicles", C.c_int32),
        ("vehicles", C.POINTER(Vehicle)),
        ("settings", Settings),
    ]


class VehicleResult(C.Structure):
    _fields_ = [
        ("mass", C.c_double),
        ("delta_v", C.c_double * 3),
        ("velocity", C.c_double * 3),
        ("crush", C.c_double),
    ]


class Results(C.Structure):
    _fields_ = [
        ("time", C.c_double),
        ("steps", C.c_int64),
        ("eroded_elements", C.c_int64),
        ("dt_min", C.c_double),
        ("added_mass_max", C.c_double),
        ("status", C.c_int32),
        ("n_vehicles", C.c_int32),
        ("vehicle", VehicleResult * 4),
    ]


class VehicleSpec(C.Structure):
    _fields_ = [
        ("mass", C.c_double),
        ("size", C.c_double * 3),
        ("material", Material),
        ("contact_modulus", C.c_double),
        ("has_rail_box", C.c_int32),
        ("rail_box_width", C.c_double),
        ("rail_box_z", C.c_double * 2),
        ("rail_box_force_fraction", C.c_double),
        ("crush_zone_length", C.c_double),
        ("body_modulus", C.c_double),
        ("crush_zone_mass", C.c_double),
        ("bumper", C.c_double * 3),
        ("crush_element_size", C.c_double),
    ]


class Scenario(C.Structure):
    _fields_ = [
        ("layout", C.c_int32),
        ("a", VehicleSpec),
        ("b", VehicleSpec),
        ("speed_a", C.c_double),
        ("speed_b", C.c_double),
        ("offset", C.c_double),
        ("clearance", C.c_double),
        ("element_size", C.c_double),
        ("settings", Settings),
    ]


def declare_scenario_api(lib):
    """Argument/return types of the crush_scenario.h entry points."""
    P = C.POINTER
    lib.crush_settings_default.restype = Settings
    lib.crush_settings_default.argtypes = [C.c_double]
    lib.crush_scenario_build.argtypes = [P(Scenario), P(C.c_void_p)]
    lib.crush_model_free.argtypes = [C.c_void_p]
    lib.crush_model_free.restype = None
    lib.crush_model_desc_get.argtypes = [C.c_void_p, P(ModelDesc)]
    lib.crush_model_settings.argtypes = [C.c_void_p]
    lib.crush_model_settings.restype = P(Settings)
    lib.crush_model_vehicle_frame.argtypes = [C.c_void_p, C.c_int32, P(C.c_uint32)]
    lib.crush_model_new.argtypes = [P(C.c_void_p)]
    lib.crush_model_add_block.argtypes = [C.c_void_p, P(C.c_double), P(C.c_double), P(C.c_int32), C.c_int32, P(C.c_int32)]
    lib.crush_model_face_set.argtypes = [C.c_void_p, C.c_int32, P(C.c_int64), P(C.c_uint32)]
    lib.crush_model_set_materials.argtypes = [C.c_void_p, C.c_int32, P(Material)]
    lib.crush_model_set_velocity.argtypes = [C.c_void_p, P(C.c_double)]
    lib.crush_last_error.restype = C.c_char_p
    lib.crush_last_error.argtypes = []


def declare_engine_api(lib):
    """Argument/return types of the crush.h device entry points."""
    P = C.POINTER
    vp = C.c_void_p
    dp = P(C.c_double)
    lib.crush_device_info.argtypes = [C.c_int, C.c_char_p, C.c_int]
    lib.crush_create.argtypes = [P(ModelDesc), C.c_int, P(vp)]
    lib.crush_destroy.argtypes = [vp]
    lib.crush_destroy.restype = None
    lib.crush_sizes.argtypes = [vp, P(C.c_int64), P(C.c_int64), P(C.c_int64)]
    lib.crush_compute_forces.argtypes = [vp, dp, dp, P(C.c_int64)]
    lib.crush_compute_forces_device.argtypes = [vp, vp, vp, P(C.c_int64)]
    lib.crush_contact_apply.argtypes = [vp, C.c_int, dp, dp, dp, C.c_double, dp, P(C.c_int64), dp]
    lib.crush_stable_dt.argtypes = [vp, dp, dp]
    lib.crush_mass_scaling.argtypes = [vp, dp, C.c_double, dp, dp, dp]
    lib.crush_masses.argtypes = [vp, dp, dp]
    fp = P(C.c_float)
    lib.crush_element_data.argtypes = [vp, fp, fp, fp, fp]
    lib.crush_get_state.argtypes = [vp, fp, P(C.c_uint8)]
    lib.crush_set_state.argtypes = [vp, fp, P(C.c_uint8)]
    lib.crush_run.argtypes = [vp, P(Results)]
    lib.crush_run_begin.argtypes = [vp]
    lib.crush_run_steps.argtypes = [vp, C.c_int64, P(C.c_int)]
    lib.crush_run_results.argtypes = [vp, P(Results)]
    lib.crush_run_state.argtypes = [vp, dp, dp]
    lib.crush_launch_count.argtypes = [vp]
    lib.crush_launch_count.restype = C.c_int64
    lib.crush_run_steps_timed.argtypes = [vp, C.c_int64, P(C.c_int), dp, dp, P(C.c_int)]
    lib.crush_set_profiling.argtypes = [vp, C.c_int]
    lib.crush_contact_search_stats.argtypes = [vp, C.c_int, P(C.c_uint64), C.c_int]
    lib.crush_set_contact_search.argtypes = [vp, C.c_int]
    lib.crush_set_step_fusion.argtypes = [vp, C.c_int]
    lib.crush_autotune.argtypes = [vp, P(Tuning)]
    lib.crush_get_tuning.argtypes = [vp, P(Tuning)]
    lib.crush_set_tuning.argtypes = [vp, P(Tuning)]
    lib.crush_batch_create.argtypes = [P(P(ModelDesc)), C.c_int, C.c_int, P(vp)]
    lib.crush_batch_create_reserved.argtypes = [P(P(ModelDesc)), C.c_int, C.c_int, P(Capacity), P(vp)]
    lib.crush_batch_solve.argtypes = [P(P(ModelDesc)), C.c_int, C.c_int, P(Results)]
    lib.crush_batch_append.argtypes = [vp, P(P(ModelDesc)), C.c_int, P(C.c_int)]
    lib.crush_run_issue.argtypes = [vp, C.c_int64]
    lib.crush_batch_size.argtypes = [vp]
    lib.crush_batch_run.argtypes = [vp, P(Results)]
    lib.crush_batch_results.argtypes = [vp, C.c_int, P(Results)]
    lib.crush_batch_results_range.argtypes = [vp, C.c_int, C.c_int, P(Results)]
    lib.crush_batch_done.argtypes = [vp, P(C.c_int), P(C.c_int)]
    lib.crush_server_create.argtypes = [P(ServerConfig), P(vp)]
    lib.crush_server_submit.argtypes = [vp, P(ModelDesc), P(C.c_uint64)]
    lib.crush_server_poll.argtypes = [vp, P(ServerResult), C.c_int, P(C.c_int), C.c_int]
    lib.crush_server_stats_get.argtypes = [vp, P(ServerStats)]
    lib.crush_server_destroy.argtypes = [vp]
    lib.crush_server_destroy.restype = None
    lib.crush_model_footprint.argtypes = [P(ModelDesc)]
    lib.crush_model_footprint.restype = C.c_double
    lib.crush_history_config.argtypes = [vp, C.c_int, C.c_int, C.c_int64, C.c_int, P(Accelerometer)]
    lib.crush_history_counts.argtypes = [vp, C.c_int, P(C.c_int64), P(C.c_int), P(C.c_int64)]
    lib.crush_history_get.argtypes = [vp, C.c_int, dp, P(C.c_int64), P(PartState), P(NodeSample)]
    lib.crush_frames_config.argtypes = [vp, C.c_int, C.c_int, C.c_int64]
    lib.crush_frames_count.argtypes = [vp, C.c_int, P(C.c_int64)]
    lib.crush_frame_get.argtypes = [vp, C.c_int, C.c_int64, dp, P(C.c_int64), P(C.c_float), P(C.c_float), P(C.c_float),
                                    P(C.c_uint8)]
    lib.crush_cfc_filter.argtypes = [dp, C.c_int64, C.c_double, C.c_double, dp]
    lib.crush_resample.argtypes = [dp, dp, C.c_int64, C.c_double, C.c_double, C.c_double, dp, dp, C.c_int64, P(C.c_int64)]
    lib.crush_contact_apply_static.argtypes = [C.c_int64, vp, vp, vp, C.c_int64, vp, vp, C.c_int64, vp,
                                               C.c_double, C.c_double, C.c_double, vp, vp, vp]


class ServerConfig(C.Structure):
    """crush_server_config (include/crush_server.h)."""
    _fields_ = [
        ("device", C.c_int32),
        ("max_waves", C.c_int32),
        ("max_wave_slots", C.c_int32),
        ("chunk_steps", C.c_int32),
        ("max_wave_elements", C.c_int64),
        ("hbm_budget_bytes", C.c_double),
        ("gather_ms", C.c_double),
        ("idle_ms", C.c_double),
        ("max_queue", C.c_int32),
        ("max_running", C.c_int32),
    ]


class ServerResult(C.Structure):
    _fields_ = [
        ("ticket", C.c_uint64),
        ("status", C.c_int32),
        ("wave", C.c_int32),
        ("submit_s", C.c_double),
        ("start_s", C.c_double),
        ("finish_s", C.c_double),
        ("results", Results),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_int64),
        ("completed", C.c_int64),
        ("waves", C.c_int64),
        ("queued", C.c_int64),
        ("running", C.c_int64),
        ("bytes_in_use", C.c_double),
        ("peak_bytes_in_use", C.c_double),
        ("budget_bytes", C.c_double),
    ]


class Capacity(C.Structure):
    """crush_capacity: the room of a context that takes more models later."""
    _fields_ = [
        ("slots", C.c_int32),
        ("contacts", C.c_int32),
        ("nodes", C.c_int64),
        ("hexes", C.c_int64),
        ("faces", C.c_int64),
        ("primary_nodes", C.c_int64),
    ]


class Tuning(C.Structure):
    """crush_tuning: the launch schedule the autotuner chose."""
    _fields_ = [
        ("slave_lanes", C.c_int32),
        ("forces_schedule", C.c_int32),
        ("fused_contact_side", C.c_int32),
        ("step_fusion", C.c_int32),
        ("early_contact", C.c_int32),
        ("contact_ms", C.c_double * 6),
        ("step_ms", C.c_double * 6),
    ]


class Accelerometer(C.Structure):
    """crush_accelerometer (include/crush.h)."""
    _fields_ = [
        ("n_nodes", C.c_int64),
        ("nodes", C.POINTER(C.c_uint32)),
        ("has_frame", C.c_int32),
        ("origin", C.c_uint32),
        ("x_axis", C.c_uint32),
        ("plane", C.c_uint32),
    ]


class PartState(C.Structure):
    _fields_ = [
        ("mass", C.c_double),
        ("velocity", C.c_double * 3),
        ("displacement", C.c_double * 3),
        ("acceleration", C.c_double * 3),
        ("kinetic_energy", C.c_double),
    ]


class NodeSample(C.Structure):
    _fields_ = [
        ("accelerometer", C.c_int32),
        ("node", C.c_uint32),
        ("position", C.c_double * 3),
        ("displacement", C.c_double * 3),
        ("velocity", C.c_double * 3),
        ("acceleration", C.c_double * 3),
        ("local_displacement", C.c_double * 3),
        ("local_velocity", C.c_double * 3),
        ("local_acceleration", C.c_double * 3),
    ]


class ContactStats(C.Structure):
    """crush_contact_stats (device-side output of crush_contact_apply_static)."""
    _fields_ = [
        ("penetration_count", C.c_int64),
        ("max_penetration", C.c_double),
        ("status", C.c_int32),
        ("reserved", C.c_int32),
    ]


STATIC_MAX_NODES = 16384
STATIC_MAX_FACES = 16384
