"""ctypes wrapper of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: used by tests/, the smoke check and bench.py's CPU-baseline leg
as the parity checker / timed CPU baseline.  `OracleSimulation` has the same methods as
`emerge_engine_b200.Simulation`, so a scene script can drive both.
"""
from __future__ import annotations

import contextlib
import ctypes
import os
import subprocess
from ctypes import POINTER, Structure, byref, c_double, c_float, c_int, c_uint32, c_uint64, c_void_p

import numpy as np

from emerge_engine_b200.abi import (PARTICLE_DTYPE, BodyStateC, ForceFieldC, Particle,
                                    SimConfigC, SpawnRegionC)
from emerge_engine_b200 import lifecycle
from emerge_engine_b200.fields import pack_fields
from emerge_engine_b200.config import BodyState, SimConfig, SlipBoundary, SpawnRegion
from emerge_engine_b200.materials import FallbackMaterial, Material
from emerge_engine_b200.simulation import MaterialRegistry

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(ORACLE_DIR, "liboracle.so")

_MAT_FIELDS = (
    "lambda_ mu min_density thermal_expansion active_stress_coeff damage_softening_rate "
    "viscosity rest_density dynamic_viscosity eos_stiffness eos_power pressure_floor "
    "fluid_min_density fluid_min_volume thermal_viscosity_coeff bulk_viscosity "
    "surface_tension_coeff settling_damping friction_angle hardening_peak hardening_decay "
    "friction_residual volume_correction dilatancy_angle cohesion min_volume_jacobian "
    "hardening_exponent compression_limit stretch_limit min_plastic_jacobian "
    "max_plastic_jacobian cohesion_coeff kappa friction nacc_cohesion hardening_factor").split()


class OracleMaterialC(Structure):
    """`oracle_material` (oracle/emerge_oracle.h)."""
    _fields_ = ([("model", c_uint32)] + [(n, c_float) for n in _MAT_FIELDS]
                + [("hardening_enabled", c_uint32), ("nacc_min_density", c_float)]
                + [(n, c_float) for n in ("yield_stress", "hardening_modulus", "tensile_strength",
                                          "softening_rate", "mu_static", "mu_dynamic",
                                          "inertial_q", "j_min", "bingham_yield_stress",
                                          "critical_shear_rate")]
                + [("bingham", c_uint32), ("mixture_phase", c_uint32)])


def oracle_material(m: Material) -> OracleMaterialC:
    c = OracleMaterialC()
    for k, v in m.oracle_fields().items():
        setattr(c, k, v)
    return c


def build_oracle(force: bool = False) -> str:
    """Builds liboracle.so with the Makefile beside this file."""
    if force or not os.path.exists(ORACLE_LIB) or (
            os.path.getmtime(ORACLE_LIB) < os.path.getmtime(os.path.join(ORACLE_DIR, "emerge_oracle.cpp"))):
        subprocess.run(["make", "-C", ORACLE_DIR, "-s", "liboracle.so"], check=True)
    return ORACLE_LIB


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build_oracle()
        L = ctypes.CDLL(ORACLE_LIB)
        P = POINTER
        sig = {
            "oracle_create": (c_void_p, [P(SimConfigC)]),
            "oracle_destroy": (None, [c_void_p]),
            "oracle_set_material": (c_int, [c_void_p, c_uint32, P(OracleMaterialC)]),
            "oracle_add_slip_boundary": (c_int, [c_void_p, c_uint64, c_int]),
            "oracle_add_body": (c_int, [c_void_p, P(SpawnRegionC), P(c_uint32)]),
            "oracle_init_with_spawn": (c_int, [c_void_p, P(SpawnRegionC)]),
            "oracle_push_particles": (c_int, [c_void_p, c_void_p, c_uint64]),
            "oracle_step": (None, [c_void_p, c_uint32]),
            "oracle_particle_count": (c_uint64, [c_void_p]),
            "oracle_read_particles": (None, [c_void_p, c_void_p]),
            "oracle_write_particles": (None, [c_void_p, c_void_p]),
            "oracle_region_state": (None, [c_void_p, c_float, c_float, c_float, P(BodyStateC)]),
            "oracle_effective_dt": (c_float, [c_void_p]),
            "oracle_last_substeps": (c_uint64, [c_void_p]),
            "oracle_last_vel_clamp_count": (c_uint64, [c_void_p]),
            "oracle_last_j_projection_count": (c_uint64, [c_void_p]),
            "oracle_last_timing_us": (None, [c_void_p, P(c_double)]),
            "oracle_set_threads": (c_int, [c_int]),
            "oracle_svd2": (None, [P(c_float), P(c_float), P(c_float), P(c_float)]),
            "oracle_set_correctly_rounded": (None, [c_int]),
            "oracle_set_force_fields": (c_int, [c_void_p, P(ForceFieldC), c_uint32, P(c_float),
                                                c_uint64]),
            "oracle_field_acceleration": (None, [P(ForceFieldC), P(c_float), P(Particle), P(c_float)]),
            "oracle_field_accelerations": (None, [c_void_p, P(c_float)]),
            "oracle_active_count": (c_uint64, [c_void_p]),
            "oracle_replace_particles": (c_int, [c_void_p, c_void_p, c_uint64, c_uint64]),
            "oracle_wake_tag": (None, [c_void_p, c_uint32]),
            "oracle_set_contact_grip": (None, [c_void_p, c_int, c_float, c_float, c_float, c_float]),
            "oracle_fit_contact_normal": (c_int, [P(c_float), c_uint32, c_float, c_float, c_float,
                                                  P(c_float)]),
            "oracle_sleep_tag": (None, [c_void_p, c_uint32]),
            "oracle_polar": (None, [P(c_float), P(c_float)]),
            "oracle_axis_weights": (None, [c_float, P(c_float)]),
            "oracle_kirchhoff": (None, [P(OracleMaterialC), P(Particle), P(c_float)]),
            "oracle_update_particle": (None, [P(OracleMaterialC), P(Particle), c_float]),
            "oracle_init_particle": (None, [P(OracleMaterialC), P(Particle)]),
            "oracle_timestep_bound": (c_float, [P(OracleMaterialC), c_float, c_float, c_float,
                                                c_float, c_float]),
            "oracle_nacc_project": (None, [P(OracleMaterialC), P(c_float), c_float, P(c_float),
                                           P(c_float)]),
            "oracle_dp_project": (c_int, [P(OracleMaterialC), P(c_float), c_float, c_float,
                                          P(c_float), P(c_float)]),
            "oracle_slip_velocity": (None, [c_uint64, c_uint64, c_uint64, P(c_float)]),
            "oracle_block_index": (c_uint32, [c_float, c_float, c_uint32]),
            "oracle_stable_argsort_u32": (None, [c_void_p, c_uint64, c_void_p]),
            "oracle_project_particle": (c_int, [P(SimConfigC), P(Particle)]),
            "oracle_choose_substep_dt": (c_float, [c_void_p, c_float]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def farr(vals, n=None):
    vals = list(vals)
    return (c_float * (n or len(vals)))(*vals)


class OracleSimulation:
    """Reference CPU step (restated), same surface as emerge_engine_b200.Simulation."""

    def __init__(self, config: SimConfig):
        config.validate()
        self._lib = lib()
        self.config = config.copy()
        cfg = config.to_c()
        self._sim = self._lib.oracle_create(byref(cfg))
        if not self._sim:
            raise ValueError("invalid SimConfig")
        self.registry = MaterialRegistry(FallbackMaterial())
        self.boundaries = [SlipBoundary(config.boundary_thickness)]
        self.force_fields: list = []

    @classmethod
    def empty(cls, config: SimConfig) -> "OracleSimulation":
        return cls(config)

    @classmethod
    def new(cls, config: SimConfig, spawn: SpawnRegion) -> "OracleSimulation":
        s = cls(config)
        sp = spawn.to_c()
        if s._lib.oracle_init_with_spawn(s._sim, byref(sp)) != 0:
            raise ValueError("spawn region must stay inside the simulation domain")
        return s

    def close(self):
        if getattr(self, "_sim", None):
            self._lib.oracle_destroy(self._sim)
            self._sim = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _set(self, mid, m):
        om = oracle_material(m)
        if self._lib.oracle_set_material(self._sim, mid, byref(om)) != 0:
            raise ValueError("material registry rejected id")

    def with_default_material(self, material):
        self.registry.set_default(material)
        self._set(0, material)
        return self

    def set_material(self, material_id, material):
        self.registry.insert(material_id, material)
        self._set(material_id, material)

    def with_material(self, material_id, material):
        self.set_material(material_id, material)
        return self

    def register_material(self, material):
        mid = self.registry.next_id()
        self.set_material(mid, material)
        return mid

    def _upload_fields(self):
        table, data = pack_fields([f for _, f in self.force_fields])
        arr = (ForceFieldC * max(len(table), 1))(*table)
        d = np.asarray(data if data else [0.0], dtype=np.float32)
        rc = self._lib.oracle_set_force_fields(self._sim, arr, len(table),
                                               d.ctypes.data_as(POINTER(c_float)), len(data))
        if rc != 0:
            raise ValueError("invalid force field")

    def add_named_force_field(self, name, field):
        self.force_fields.append((str(name), field))
        self._upload_fields()

    def add_force_field(self, field):
        self.add_named_force_field(f"force_field_{len(self.force_fields)}", field)

    def with_force_field(self, field):
        self.add_force_field(field)
        return self

    def with_named_force_field(self, name, field):
        self.add_named_force_field(name, field)
        return self

    def remove_force_field(self, name):
        for k, (n, _) in enumerate(self.force_fields):
            if n == name:
                del self.force_fields[k]
                self._upload_fields()
                return True
        return False

    def clear_force_fields(self):
        self.force_fields = []
        self._upload_fields()

    def force_field_names(self):
        return [n for n, _ in self.force_fields]

    def field_accelerations(self) -> np.ndarray:
        """(n, 2) float32: the fields' summed Field::acceleration per particle at the current
        state (n-body trees built from the current positions, n_body.rs:332-360)."""
        n = self.particle_count()
        out = np.zeros((max(n, 1), 2), dtype=np.float32)
        self._lib.oracle_field_accelerations(self._sim, out.ctypes.data_as(POINTER(c_float)))
        return out[:n]

    def add_boundary_condition(self, b):
        self.boundaries.append(b)
        self._lib.oracle_add_slip_boundary(self._sim, b.thickness, 0)

    def with_boundary(self, b):
        self.add_boundary_condition(b)
        return self

    def set_boundary_condition(self, b):
        self.boundaries = [b]
        self._lib.oracle_add_slip_boundary(self._sim, b.thickness, 1)

    def add_body(self, spawn: SpawnRegion) -> int:
        sp = spawn.to_c()
        tag = c_uint32()
        if self._lib.oracle_add_body(self._sim, byref(sp), byref(tag)) != 0:
            raise ValueError("spawn region must stay inside the simulation domain")
        return int(tag.value)

    def add_particles(self, particles: np.ndarray) -> None:
        arr = np.ascontiguousarray(particles, dtype=PARTICLE_DTYPE)
        self._lib.oracle_push_particles(self._sim, arr.ctypes.data_as(c_void_p), len(arr))

    def particle_count(self) -> int:
        return int(self._lib.oracle_particle_count(self._sim))

    def particles(self) -> np.ndarray:
        out = np.zeros(self.particle_count(), dtype=PARTICLE_DTYPE)
        if len(out):
            self._lib.oracle_read_particles(self._sim, out.ctypes.data_as(c_void_p))
        return out

    def set_particles(self, particles: np.ndarray) -> None:
        arr = np.ascontiguousarray(particles, dtype=PARTICLE_DTYPE)
        assert len(arr) == self.particle_count()
        self._lib.oracle_write_particles(self._sim, arr.ctypes.data_as(c_void_p))

    # ---------------------------------------------------------------- sleep partition
    def active_count(self) -> int:
        return int(self._lib.oracle_active_count(self._sim))

    def _replace(self, particles, active: int) -> None:
        arr = np.ascontiguousarray(particles, dtype=PARTICLE_DTYPE)
        if self._lib.oracle_replace_particles(self._sim, arr.ctypes.data_as(c_void_p), len(arr),
                                              int(active)) != 0:
            raise ValueError("active count above particle count")

    def with_contact_grip(self, grip):
        self.set_contact_grip(grip)
        return self

    def set_contact_grip(self, grip):
        if grip is None:
            self._lib.oracle_set_contact_grip(self._sim, 0, 0.0, 0.0, 0.0, 0.0)
        else:
            self._lib.oracle_set_contact_grip(self._sim, 1, grip.mu_easy, grip.mu_resist,
                                              grip.easy_direction[0], grip.easy_direction[1])

    def wake_tag(self, tag: int) -> None:
        self._lib.oracle_wake_tag(self._sim, int(tag))

    def sleep_tag(self, tag: int) -> None:
        self._lib.oracle_sleep_tag(self._sim, int(tag))

    def remove_particles(self, predicate) -> int:
        p, active, removed = lifecycle.remove_particles(self.particles(), self.active_count(), predicate)
        if removed:
            self._replace(p, active)
        return removed

    def retain_particles(self, predicate) -> None:
        p, active = lifecycle.retain_particles(self.particles(), self.active_count(), predicate)
        self._replace(p, active)

    def split_particles(self, should_split, jitter: float) -> None:
        p, active = lifecycle.split_particles(self.particles(), self.active_count(), should_split, jitter)
        self._replace(p, active)

    def step(self):
        self._lib.oracle_step(self._sim, 1)

    def step_n(self, n: int):
        self._lib.oracle_step(self._sim, int(n))

    def last_substeps(self) -> int:
        return int(self._lib.oracle_last_substeps(self._sim))

    def effective_dt(self) -> float:
        return float(self._lib.oracle_effective_dt(self._sim))

    def last_counters(self):
        return (int(self._lib.oracle_last_vel_clamp_count(self._sim)),
                int(self._lib.oracle_last_j_projection_count(self._sim)), None)

    def last_timing_us(self) -> dict:
        buf = (c_double * 7)()
        self._lib.oracle_last_timing_us(self._sim, buf)
        keys = ("cfl", "project", "density", "p2g", "grid_update", "g2p", "total")
        return dict(zip(keys, list(buf)))

    def region_state(self, center, radius: float) -> BodyState:
        out = BodyStateC()
        self._lib.oracle_region_state(self._sim, float(center[0]), float(center[1]),
                                      float(radius), byref(out))
        return BodyState.from_c(out)

    def choose_substep_dt(self, max_dt: float) -> float:
        return float(self._lib.oracle_choose_substep_dt(self._sim, float(max_dt)))


def set_threads(n: int) -> int:
    return int(lib().oracle_set_threads(int(n)))


@contextlib.contextmanager
def correctly_rounded_math():
    """Within the block the oracle evaluates exp/log/pow/sin/sinh in double and rounds once
    (oracle_set_correctly_rounded); outside it, the C library's f32 functions."""
    lib().oracle_set_correctly_rounded(1)
    try:
        yield
    finally:
        lib().oracle_set_correctly_rounded(0)
