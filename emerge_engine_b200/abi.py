"""ctypes mirror of include/emerge_cuda.h and the loader of the CUDA library.

The struct layouts are byte-identical to the reference's `#[repr(C)]` types
(`Particle`, matter/particle.rs:13-138; `MaterialParams`, matter/materials/params.rs:10-101)
and to the C structs of include/emerge_cuda.h.  The CPU oracle (oracle/) uses the same
layouts, so these classes serve both libraries.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import (POINTER, Structure, c_char_p, c_float, c_int, c_int32, c_int64, c_uint32,
                    c_uint64, c_void_p)

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libemerge_cuda.so")

# emerge_status
OK = 0
ERR_INVALID_ARG = 1
ERR_UNSUPPORTED = 2
ERR_CUDA = 3
ERR_TIMEOUT = 4
ERR_NONFINITE = 5
ERR_OOM = 6
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "UNSUPPORTED", 3: "CUDA", 4: "TIMEOUT",
                5: "NONFINITE", 6: "OOM"}

OPT_USE_GRAPH = 1
OPT_SORT_INTERVAL = 2
OPT_P2G_AGGREGATE = 3
OPT_DETERMINISTIC = 4
OPT_PRECISE_MATH = 5
OPT_TILE_SHAPE = 7
OPT_CHUNKS_PER_CTA = 8
TUNE_MAX_TRIALS = 16


class Particle(Structure):
    """`Particle` (matter/particle.rs:13-138), 128 bytes."""
    _fields_ = [
        ("x", c_float * 2), ("v", c_float * 2), ("c", c_float * 4), ("f", c_float * 4),
        ("mass", c_float), ("initial_volume", c_float), ("volume", c_float), ("density", c_float),
        ("material_id", c_uint32), ("plastic_volume_ratio", c_float), ("hardening_scale", c_float),
        ("friction_hardening", c_float), ("log_volume_strain", c_float), ("temperature", c_float),
        ("user_tag", c_uint32), ("activation", c_float), ("activation_dir", c_float * 2),
        ("muscle_group_id", c_uint32), ("contact_group", c_uint32), ("sleeping", c_uint32),
        ("pinned", c_uint32), ("scalar_field", c_float), ("pad_", c_uint32),
    ]


assert ctypes.sizeof(Particle) == 128

# numpy view of an array of Particle
PARTICLE_DTYPE = np.dtype([
    ("x", np.float32, (2,)), ("v", np.float32, (2,)), ("c", np.float32, (4,)),
    ("f", np.float32, (4,)), ("mass", np.float32), ("initial_volume", np.float32),
    ("volume", np.float32), ("density", np.float32), ("material_id", np.uint32),
    ("plastic_volume_ratio", np.float32), ("hardening_scale", np.float32),
    ("friction_hardening", np.float32), ("log_volume_strain", np.float32),
    ("temperature", np.float32), ("user_tag", np.uint32), ("activation", np.float32),
    ("activation_dir", np.float32, (2,)), ("muscle_group_id", np.uint32),
    ("contact_group", np.uint32), ("sleeping", np.uint32), ("pinned", np.uint32),
    ("scalar_field", np.float32), ("pad_", np.uint32),
])
assert PARTICLE_DTYPE.itemsize == 128


class SimConfigC(Structure):
    """`SimConfig` (spacetime/solver/config.rs:26-121)."""
    _fields_ = [
        ("grid_res", c_uint64), ("grid_cell_size", c_float), ("dt", c_float),
        ("adaptive_timestep", c_uint32), ("cfl_include_affine_speed", c_uint32),
        ("cfl_coefficient", c_float), ("material_cfl_coefficient", c_float),
        ("viscous_timestep_coefficient", c_float), ("min_dt", c_float),
        ("project_invalid_state", c_uint32), ("projection_min_density", c_float),
        ("projection_min_volume", c_float), ("projection_min_deformation_j", c_float),
        ("gravity", c_float * 2), ("boundary_thickness", c_uint64),
        ("default_initial_volume", c_float), ("recompute_density_each_step", c_uint32),
        ("particle_mass", c_float), ("pad0_", c_uint32), ("max_substeps_per_step", c_uint64),
        ("apic_blend", c_float), ("j_max", c_float), ("sleep_threshold", c_float),
        ("contact_friction", c_float), ("asflip_blend", c_float),
        ("mixture_drag_coefficient", c_float), ("mixture_pressure_iterations", c_uint32),
        ("dx_meters", c_float), ("dt_seconds", c_float), ("pad1_", c_uint32),
    ]


assert ctypes.sizeof(SimConfigC) == 136


class ForceFieldC(Structure):
    """`emerge_force_field` (include/emerge_cuda.h), 48 bytes."""
    _fields_ = [("kind", c_uint32), ("material_mask", c_uint32), ("material_filter", c_uint32),
                ("count", c_uint32), ("data_offset", c_uint32), ("n_charges", c_uint32),
                ("params", c_float * 6)]


class MaterialParamsC(Structure):
    """`MaterialParams` (matter/materials/params.rs:10-101), 96 bytes."""
    _fields_ = [(name, c_uint32 if name == "model" else c_float) for name in (
        "model", "lambda_", "mu", "hardening_exponent", "compression_limit", "stretch_limit",
        "rest_density", "eos_stiffness", "eos_power", "dynamic_viscosity", "volume_ratio_min",
        "volume_ratio_max", "dp_h0", "dp_h1", "dp_h2", "dp_h3", "active_stress_coeff",
        "hardening_modulus", "thermal_viscosity_coeff", "thermal_expansion", "pressure_floor",
        "bulk_viscosity", "surface_tension_coeff", "cohesion_coeff")]


assert ctypes.sizeof(MaterialParamsC) == 96


class SpawnRegionC(Structure):
    """`SpawnRegion` (spacetime/solver/config.rs:317-346)."""
    _fields_ = [
        ("spacing", c_float), ("box_size", c_int32 * 2), ("box_center", c_float * 2),
        ("shape", c_uint32), ("disk_radius", c_float),
        ("initial_deformation_gradient", c_float * 4), ("precompute_initial_volumes", c_uint32),
        ("initial_velocity_scale", c_float), ("position_jitter", c_float),
        ("rng_seed", c_uint32), ("material_id", c_uint32), ("has_mass_override", c_uint32),
        ("mass_override", c_float),
    ]


assert ctypes.sizeof(SpawnRegionC) == 72


class BodyStateC(Structure):
    """`BodyState` (spacetime/solver/query.rs:17-32)."""
    _fields_ = [
        ("count", c_uint64), ("avg_volume_ratio", c_float), ("max_volume_ratio", c_float),
        ("avg_speed", c_float), ("avg_det_f", c_float), ("avg_density", c_float),
        ("centroid", c_float * 2), ("pad_", c_uint32),
    ]


assert ctypes.sizeof(BodyStateC) == 40


class StepTimingC(Structure):
    """`StepTiming` (systems/diagnostics/snapshot.rs:82-105)."""
    _fields_ = [(name, c_uint64) for name in (
        "p2g_us", "grid_update_us", "g2p_us", "fields_us", "thermal_us", "cfl_us",
        "spatial_hash_us", "phase_sleep_us", "project_us", "density_us", "total_us")]


class StatsC(Structure):
    """`emerge_stats` (include/emerge_cuda.h)."""
    _fields_ = [(name, c_uint64) for name in (
        "steps", "substeps", "kernel_launches", "p2g_blocks", "p2g_fallback_blocks", "sorts")]


class ClosureStatsC(Structure):
    """`emerge_closure_stats` (include/emerge_cuda.h)."""
    _fields_ = [("smooth", c_uint64), ("net", c_uint64), ("hull_fallback", c_uint64),
                ("judged", c_uint64), ("logged", c_uint64 * 2), ("err_mean", ctypes.c_double),
                ("err_max", c_float), ("pad_", c_uint32), ("judge_replaced", c_uint64),
                ("err_p50", c_float), ("err_p99", c_float)]


class ClosureTrainConfigC(Structure):
    """`emerge_closure_train_config` (include/emerge_cuda.h)."""
    _fields_ = [("epochs", c_uint32), ("batch", c_uint32), ("lr", c_float), ("lr_decay", c_float),
                ("beta1", c_float), ("beta2", c_float), ("eps", c_float), ("val_fraction", c_float),
                ("seed", c_uint64), ("max_samples", c_uint64)]


class ClosureTrainReportC(Structure):
    """`emerge_closure_train_report` (include/emerge_cuda.h)."""
    _fields_ = [("n_train", c_uint64), ("n_val", c_uint64), ("train_loss", c_float),
                ("val_loss", c_float), ("val_err_mean", c_float), ("val_err_p50", c_float),
                ("val_err_p99", c_float), ("val_err_max", c_float), ("val_err_trial_mean", c_float),
                ("seconds", c_float),
                ("steps", c_uint32)]


class BatchTuneReportC(Structure):
    """`emerge_batch_tune_report` (include/emerge_cuda.h)."""
    _fields_ = [("sort_interval", c_int32), ("aggregate", c_int32), ("tile_shape", c_int32),
                ("chunks_per_cta", c_int32), ("n_trials", c_uint32), ("from_cache", c_uint32),
                ("best_ms", c_float), ("trial_sort_interval", c_int32 * TUNE_MAX_TRIALS),
                ("trial_aggregate", c_int32 * TUNE_MAX_TRIALS),
                ("trial_tile_shape", c_int32 * TUNE_MAX_TRIALS),
                ("trial_chunks", c_int32 * TUNE_MAX_TRIALS), ("trial_ms", c_float * TUNE_MAX_TRIALS)]


CLOSURE_NPARAMS = 8963  # W1[6][64] b1 W2[64][64] b2 W3[64][64] b3 W4[64][3] b4
CLOSURE_NNORM = 18      # in_shift[6] in_scale[6] out_shift[3] out_scale[3]

# Entry points declared in include/emerge_cuda.h: (name, restype, argtypes)
SIM = c_void_p
ABI_FUNCTIONS = [
    ("emerge_cuda_create", c_int, [POINTER(SimConfigC), c_int, POINTER(c_void_p)]),
    ("emerge_cuda_destroy", c_int, [SIM]),
    ("emerge_cuda_last_error", c_char_p, [SIM]),
    ("emerge_cuda_last_global_error", c_char_p, []),
    ("emerge_cuda_set_materials", c_int, [SIM, POINTER(MaterialParamsC), c_uint32]),
    ("emerge_cuda_set_slip_boundaries", c_int, [SIM, POINTER(c_uint64), c_uint32]),
    ("emerge_cuda_set_force_fields", c_int, [SIM, POINTER(ForceFieldC), c_uint32, POINTER(c_float),
                                             c_uint64]),
    ("emerge_cuda_field_accelerations", c_int, [SIM, POINTER(c_float), c_uint64]),
    ("emerge_cuda_set_contact_grip", c_int, [SIM, c_int, c_float, c_float, c_float, c_float]),
    ("emerge_cuda_set_mixture_phases", c_int, [SIM, POINTER(c_uint32), c_uint32]),
    ("emerge_cuda_active_count", c_int, [SIM, POINTER(c_uint64)]),
    ("emerge_cuda_replace_particles", c_int, [SIM, c_void_p, c_uint64, c_uint64]),
    ("emerge_cuda_add_body", c_int, [SIM, POINTER(SpawnRegionC), POINTER(c_uint32)]),
    ("emerge_cuda_init_with_spawn", c_int, [SIM, POINTER(SpawnRegionC)]),
    ("emerge_cuda_add_particles", c_int, [SIM, c_void_p, c_uint64, c_int]),
    ("emerge_cuda_particle_count", c_int, [SIM, POINTER(c_uint64)]),
    ("emerge_cuda_read_particles", c_int, [SIM, c_void_p, c_uint64]),
    ("emerge_cuda_read_particles_async", c_int, [SIM, c_void_p, c_uint64]),
    ("emerge_cuda_write_particles", c_int, [SIM, c_void_p, c_uint64]),
    ("emerge_cuda_step", c_int, [SIM, c_uint32, POINTER(StepTimingC)]),
    ("emerge_cuda_last_substeps", c_int, [SIM, POINTER(c_uint64)]),
    ("emerge_cuda_effective_dt", c_int, [SIM, POINTER(c_float)]),
    ("emerge_cuda_last_counters", c_int, [SIM, POINTER(c_uint64), POINTER(c_uint64),
                                          POINTER(c_float)]),
    ("emerge_cuda_synchronize", c_int, [SIM]),
    ("emerge_cuda_region_state", c_int, [SIM, c_float, c_float, c_float, POINTER(BodyStateC)]),
    ("emerge_cuda_set_option", c_int, [SIM, c_int, c_int64]),
    ("emerge_cuda_sort_now", c_int, [SIM, c_int]),
    ("emerge_cuda_sort_keys", c_int, [c_void_p, c_uint64, c_uint32, c_int, c_void_p, c_void_p]),
    ("emerge_cuda_sort_keys_noalloc", c_int, [c_void_p, c_uint32, c_uint32, c_int, c_void_p,
                                              c_void_p, c_void_p]),
    ("emerge_cuda_stream", c_void_p, [SIM]),
    ("emerge_cuda_kernel_launches", c_int, [SIM, POINTER(c_uint64)]),
    ("emerge_cuda_event_record", c_int, [SIM, c_int]),
    ("emerge_cuda_event_elapsed", c_int, [SIM, c_int, c_int, POINTER(c_float)]),
    ("emerge_cuda_flush_l2", c_int, [SIM]),
    ("emerge_cuda_host_alloc", c_int, [ctypes.c_size_t, POINTER(c_void_p)]),
    ("emerge_cuda_host_free", c_int, [c_void_p]),
    ("emerge_cuda_stats", c_int, [SIM, POINTER(StatsC)]),
    ("emerge_cuda_closure_log", c_int, [SIM, c_uint64, c_uint32]),
    ("emerge_cuda_closure_train", c_int, [SIM, c_int, POINTER(ClosureTrainConfigC),
                                          POINTER(ClosureTrainReportC)]),
    ("emerge_cuda_closure_enable", c_int, [SIM, c_int, c_uint32]),
    ("emerge_cuda_closure_stats", c_int, [SIM, POINTER(ClosureStatsC), c_int]),
    ("emerge_cuda_closure_set_mode", c_int, [SIM, c_int, c_float]),
    ("emerge_cuda_closure_get_params", c_int, [SIM, c_int, c_void_p, c_void_p]),
    ("emerge_cuda_closure_get_log", c_int, [SIM, c_int, c_void_p, c_void_p, c_uint64, POINTER(c_uint64)]),
    ("emerge_cuda_closure_set_params", c_int, [SIM, c_int, c_void_p, c_void_p, c_void_p]),
    ("emerge_cuda_mlp_loss_grad", c_int, [c_void_p, c_void_p, c_void_p, c_uint32, c_void_p, c_void_p]),
    ("emerge_cuda_mlp_adam", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_uint32, c_uint32,
                                     c_float, c_float, c_float, c_float]),
    ("emerge_cuda_mlp_infer_bf16", c_int, [c_void_p, c_void_p, c_uint32, c_void_p]),
    ("emerge_cuda_mlp_infer_tc", c_int, [c_void_p, c_void_p, c_uint32, c_void_p]),
    ("emerge_cuda_silu_fast", c_int, [c_void_p, c_uint32, c_void_p]),
    ("emerge_cuda_batch_create", c_int, [POINTER(c_void_p), c_uint32, POINTER(c_void_p)]),
    ("emerge_cuda_batch_destroy", c_int, [c_void_p]),
    ("emerge_cuda_batch_last_error", c_char_p, [c_void_p]),
    ("emerge_cuda_batch_step", c_int, [c_void_p, c_uint32]),
    ("emerge_cuda_batch_time_steps", c_int, [c_void_p, c_uint32, c_int, POINTER(c_float)]),
    ("emerge_cuda_batch_scene_count", c_int, [c_void_p, POINTER(c_uint32)]),
    ("emerge_cuda_batch_particle_count", c_int, [c_void_p, c_uint32, POINTER(c_uint64)]),
    ("emerge_cuda_batch_read_particles", c_int, [c_void_p, c_uint32, c_void_p, c_uint64]),
    ("emerge_cuda_batch_region_state", c_int, [c_void_p, c_uint32, c_float, c_float, c_float,
                                               POINTER(BodyStateC)]),
    ("emerge_cuda_batch_substeps", c_int, [c_void_p, c_void_p, c_void_p]),
    ("emerge_cuda_batch_set_option", c_int, [c_void_p, c_int, c_int64]),
    ("emerge_cuda_batch_autotune", c_int, [c_void_p, c_uint32, c_char_p, POINTER(BatchTuneReportC)]),
]

_lib = None


class EmergeError(RuntimeError):
    """A non-OK emerge_status; `.status` holds the code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def load_library(path: str | None = None) -> ctypes.CDLL:
    """Loads libemerge_cuda.so.  Raises if it is missing: there is no CPU fallback."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or os.environ.get("EMERGE_CUDA_LIB") or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"CUDA backend library not found at {p}; build it with "
            "`python -m emerge_engine_b200.build` (there is no CPU fallback)")
    lib = ctypes.CDLL(p)
    for name, res, args in ABI_FUNCTIONS:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(lib, status: int, sim=None) -> None:
    if status == OK:
        return
    if sim is not None:
        msg = lib.emerge_cuda_last_error(sim)
    else:
        msg = lib.emerge_cuda_last_global_error()
    raise EmergeError(status, (msg or b"").decode(errors="replace"))
