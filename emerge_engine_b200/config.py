"""`SimConfig` and `SpawnRegion` with the reference's defaults and builders.

Mirrors spacetime/solver/config.rs: `SimConfig` (:26-121), its `Default` (:127-158),
`standard` (:165-172), `unsafe_defaults` (:179-185), `earth` (:207-216), `validate`
(:247-299); `SpawnRegion` (:317-346), `Default` (:348-364), `for_sim` (:370-375), the
fluent builders (:380-458) and `fits_in_sim` (:472-482).  Violations raise ValueError
where the reference panics.
"""
from __future__ import annotations

import copy
from dataclasses import dataclass, field

import numpy as np

from .abi import SimConfigC, SpawnRegionC

f32 = np.float32


@dataclass
class SimConfig:
    grid_res: int = 64
    grid_cell_size: float = 1.0
    dt: float = 1.0
    adaptive_timestep: bool = True
    cfl_include_affine_speed: bool = True
    cfl_coefficient: float = 0.9
    material_cfl_coefficient: float = 0.5
    viscous_timestep_coefficient: float = 0.5
    min_dt: float = 1.0e-3
    project_invalid_state: bool = True
    projection_min_density: float = 1.0e-6
    projection_min_volume: float = 1.0e-6
    projection_min_deformation_j: float = 1.0e-6
    gravity: tuple = (0.0, -0.05)
    boundary_thickness: int = 2
    default_initial_volume: float = 1.0
    recompute_density_each_step: bool = False
    particle_mass: float = 1.0
    max_substeps_per_step: int = 64
    apic_blend: float = 1.0
    j_max: float = 50.0
    sleep_threshold: float = 0.0
    contact_friction: float = 0.5
    asflip_blend: float = 0.0
    mixture_drag_coefficient: float = 0.0
    mixture_pressure_iterations: int = 0
    dx_meters: float = 1.0
    dt_seconds: float = 1.0

    @classmethod
    def standard(cls, grid_res: int, dt: float, gravity) -> "SimConfig":
        return cls(grid_res=grid_res, dt=dt, gravity=(float(gravity[0]), float(gravity[1])))

    @classmethod
    def unsafe_defaults(cls) -> "SimConfig":
        return cls(adaptive_timestep=False, project_invalid_state=False)

    @classmethod
    def earth(cls, grid_res: int, cell_m: float, dt: float) -> "SimConfig":
        g = float(f32(9.81) / f32(cell_m))
        c = cls.standard(grid_res, dt, (0.0, -g))
        c.dx_meters, c.dt_seconds = cell_m, dt
        return c

    def copy(self) -> "SimConfig":
        return copy.deepcopy(self)

    def validate(self) -> None:
        checks = [
            (self.grid_res >= 4, "grid_res must be >= 4"),
            (self.grid_cell_size > 0.0, "grid_cell_size must be positive"),
            (self.dt > 0.0, "dt must be positive"),
            (self.cfl_coefficient > 0.0, "cfl_coefficient must be positive"),
            (self.material_cfl_coefficient > 0.0, "material_cfl_coefficient must be positive"),
            (self.viscous_timestep_coefficient > 0.0,
             "viscous_timestep_coefficient must be positive"),
            (self.min_dt > 0.0, "min_dt must be positive"),
            (self.min_dt <= self.dt, "min_dt must be <= dt"),
            (self.projection_min_density > 0.0, "projection_min_density must be positive"),
            (self.projection_min_volume > 0.0, "projection_min_volume must be positive"),
            (self.projection_min_deformation_j > 0.0,
             "projection_min_deformation_j must be positive"),
            (self.particle_mass > 0.0, "particle_mass must be positive"),
            (self.contact_friction >= 0.0, "contact_friction must be non-negative"),
            (self.max_substeps_per_step > 0, "max_substeps_per_step must be > 0"),
            (self.default_initial_volume > 0.0, "default_initial_volume must be positive"),
            (self.j_max > 1.0, "j_max must be > 1.0"),
            (0.0 <= self.apic_blend <= 1.0, "apic_blend must be in [0, 1]"),
            (0 < self.boundary_thickness < self.grid_res - 1,
             "boundary_thickness must be in [1, grid_res-2]"),
        ]
        for ok, msg in checks:
            if not ok:
                raise ValueError(msg)

    def to_c(self) -> SimConfigC:
        c = SimConfigC()
        for name, _ in SimConfigC._fields_:
            if name.startswith("pad"):
                continue
            val = getattr(self, name)
            if name == "gravity":
                c.gravity[0], c.gravity[1] = float(val[0]), float(val[1])
            elif isinstance(val, bool):
                setattr(c, name, 1 if val else 0)
            else:
                setattr(c, name, val)
        return c


BOX, DISK = 0, 1


@dataclass
class SpawnRegion:
    spacing: float = 1.0
    box_size: tuple = (16, 16)
    box_center: tuple = (32.0, 32.0)
    shape: int = BOX
    disk_radius: float = 0.0
    initial_deformation_gradient: tuple = (1.0, 0.0, 0.0, 1.0)
    precompute_initial_volumes: bool = False
    initial_velocity_scale: float = 0.0
    position_jitter: float = 0.0
    rng_seed: int = 1
    material_id: int = 0
    mass_override: float | None = None

    @classmethod
    def for_sim(cls, config: SimConfig) -> "SpawnRegion":
        c = float(f32(config.grid_res) * f32(0.5))
        return cls(box_center=(c, c))

    # fluent builders (config.rs:380-458)
    def at(self, center):
        self.box_center = (float(center[0]), float(center[1]))
        return self

    def box_of(self, size):
        self.box_size = (int(size[0]), int(size[1]))
        return self

    def disk(self, r: float):
        self.shape, self.disk_radius = DISK, float(r)
        side = int(np.ceil(f32(2.0) * f32(r))) + 1
        self.box_size = (side, side)
        return self

    def with_spacing(self, s: float):
        self.spacing = float(s)
        return self

    def material(self, mid: int):
        self.material_id = int(mid)
        return self

    def mass(self, m: float):
        self.mass_override = float(m)
        return self

    def precompute_volumes(self):
        self.precompute_initial_volumes = True
        return self

    def velocity_scale(self, s: float):
        self.initial_velocity_scale = float(s)
        return self

    def jitter(self, s: float):
        self.position_jitter = float(s)
        return self

    def seed(self, seed: int):
        self.rng_seed = int(seed) & 0xFFFFFFFF
        return self

    def fits_in_sim(self, config: SimConfig) -> bool:
        if not (self.spacing > 0.0 and self.box_size[0] > 0 and self.box_size[1] > 0):
            return False
        hx = f32(f32(self.box_size[0]) * f32(0.5))
        hy = f32(f32(self.box_size[1]) * f32(0.5))
        mnx, mny = f32(self.box_center[0]) - hx, f32(self.box_center[1]) - hy
        mxx, mxy = f32(self.box_center[0]) + hx, f32(self.box_center[1]) + hy
        dmin = f32(config.boundary_thickness)
        dmax = f32(max(config.grid_res - config.boundary_thickness, 0))
        return bool(mnx >= dmin and mny >= dmin and mxx <= dmax and mxy <= dmax)

    def to_c(self) -> SpawnRegionC:
        s = SpawnRegionC()
        s.spacing = self.spacing
        s.box_size[0], s.box_size[1] = self.box_size
        s.box_center[0], s.box_center[1] = self.box_center
        s.shape = self.shape
        s.disk_radius = self.disk_radius
        for k in range(4):
            s.initial_deformation_gradient[k] = self.initial_deformation_gradient[k]
        s.precompute_initial_volumes = 1 if self.precompute_initial_volumes else 0
        s.initial_velocity_scale = self.initial_velocity_scale
        s.position_jitter = self.position_jitter
        s.rng_seed = self.rng_seed & 0xFFFFFFFF
        s.material_id = self.material_id
        s.has_mass_override = 0 if self.mass_override is None else 1
        s.mass_override = 0.0 if self.mass_override is None else self.mass_override
        return s


@dataclass
class SlipBoundary:
    """`SlipBoundary` (forces/boundary/slip.rs:1-24)."""
    thickness: int


@dataclass
class BodyState:
    """`BodyState` (spacetime/solver/query.rs:17-32)."""
    count: int = 0
    avg_volume_ratio: float = 0.0
    max_volume_ratio: float = 0.0
    avg_speed: float = 0.0
    avg_det_f: float = 0.0
    avg_density: float = 0.0
    centroid: tuple = field(default=(0.0, 0.0))

    @classmethod
    def from_c(cls, b) -> "BodyState":
        return cls(int(b.count), float(b.avg_volume_ratio), float(b.max_volume_ratio),
                   float(b.avg_speed), float(b.avg_det_f), float(b.avg_density),
                   (float(b.centroid[0]), float(b.centroid[1])))
