"""Built-in force fields with the reference's constructors (forces/fields/), in f32.

Each class mirrors one reference field struct and packs itself into the flat
`emerge_force_field` table plus a shared float data array (`pack(data)` appends its sources,
charge table or potential to `data` and returns the table entry).  The fields apply after
G2P: v += sub_dt * (sum of the fields' accelerations), then the G2P speed clamp
(spacetime/solver/step.rs:212-259).

`NBodyGravityField` is the particles' own gravity through a Barnes-Hut quadtree, rebuilt on
the device every substep between the G2P half and the fields half of the particle pass.
Not on the device: `SpatialDragField` (a host function pointer).
"""
from __future__ import annotations

import numpy as np

from .abi import ForceFieldC

f32 = np.float32
INF = float("inf")
ALL_MATERIALS = 0xFFFFFFFF
FADE_ONSET_RATIO = f32(0.85)  # forces/fields/mod.rs:10

GRAVITY_WELL, BUOYANCY, LINEAR_DRAG, RADIAL_CONFINEMENT, AABB_CONFINEMENT = 1, 2, 3, 4, 5
COULOMB, UNIFORM_ELECTRIC, CHEMOTAXIS, NBODY_GRAVITY = 6, 7, 8, 9
NBODY_MAX_DEPTH = 10  # the device tree's limit (the reference takes any usize)


def _entry(kind, params=(), **kw) -> ForceFieldC:
    e = ForceFieldC()
    e.kind = kind
    e.material_mask = ALL_MATERIALS
    e.material_filter = ALL_MATERIALS
    for k, v in kw.items():
        setattr(e, k, v)
    for k, v in enumerate(params):
        e.params[k] = float(f32(v))
    return e


def _charge_table(charges: dict) -> list:
    """HashMap<u32, f32> as a table by material id (missing ids carry no charge)."""
    if not charges:
        return []
    n = max(int(k) for k in charges) + 1
    table = [0.0] * n
    for k, q in charges.items():
        table[int(k)] = float(f32(q))
    return table


class Field:
    """`Field` trait (forces/fields/force_field.rs): the device-supported built-ins."""

    def pack(self, data: list) -> ForceFieldC:
        raise NotImplementedError


class GravityWellField(Field):
    """`GravityWellField` (forces/fields/gravity.rs): Plummer-softened point masses with an
    optional smooth cutoff."""

    def __init__(self, sources, gravitational_constant, softening):
        self.sources = [((float(f32(p[0])), float(f32(p[1]))), float(f32(m))) for p, m in sources]
        self.gravitational_constant = f32(gravitational_constant)
        self.softening = f32(softening)
        self.cutoff = f32(INF)
        self.switch_on = f32(INF)

    @classmethod
    def new(cls, sources, gravitational_constant, softening):
        return cls(sources, gravitational_constant, softening)

    @classmethod
    def point(cls, position, mass, gravitational_constant, softening):
        return cls([(position, mass)], gravitational_constant, softening)

    def with_cutoff(self, cutoff):
        self.cutoff = f32(cutoff)
        self.switch_on = f32(FADE_ONSET_RATIO * self.cutoff)
        return self

    def pack(self, data):
        e = _entry(GRAVITY_WELL, (self.gravitational_constant, self.softening, self.cutoff,
                                  self.switch_on), count=len(self.sources), data_offset=len(data))
        for (x, y), m in self.sources:
            data += [x, y, m]
        return e


class BuoyancyField(Field):
    """`BuoyancyField` (forces/fields/buoyancy.rs): a = -g * fluid_density / density."""

    def __init__(self, fluid_density, gravity, min_density=1.0e-4):
        self.fluid_density = f32(fluid_density)
        self.gravity = (float(f32(gravity[0])), float(f32(gravity[1])))
        self.min_density = f32(min_density)

    @classmethod
    def new(cls, fluid_density, gravity):
        return cls(fluid_density, gravity)

    @classmethod
    def for_fluid(cls, fluid_density, gravity):
        return cls(fluid_density, gravity)

    def pack(self, data):
        return _entry(BUOYANCY, (self.fluid_density, self.gravity[0], self.gravity[1],
                                 self.min_density))


class LinearDragField(Field):
    """`LinearDragField` (forces/fields/drag.rs): a = c (target - v) for the masked materials."""
    ALL_MATERIALS = ALL_MATERIALS

    def __init__(self, target_velocity, drag_coefficient, material_mask=ALL_MATERIALS):
        self.target_velocity = (float(f32(target_velocity[0])), float(f32(target_velocity[1])))
        self.drag_coefficient = f32(drag_coefficient)
        self.material_mask = int(material_mask) & 0xFFFFFFFF

    @classmethod
    def new(cls, target_velocity, drag_coefficient, material_mask):
        return cls(target_velocity, drag_coefficient, material_mask)

    def pack(self, data):
        return _entry(LINEAR_DRAG, (self.target_velocity[0], self.target_velocity[1],
                                    self.drag_coefficient), material_mask=self.material_mask)


class RadialConfinementField(Field):
    """`RadialConfinementField` (forces/fields/confinement.rs): spring back inside a circle."""

    def __init__(self, center, radius, stiffness):
        self.center = (float(f32(center[0])), float(f32(center[1])))
        self.radius = f32(radius)
        self.stiffness = f32(stiffness)

    @classmethod
    def new(cls, center, radius, stiffness):
        return cls(center, radius, stiffness)

    def pack(self, data):
        return _entry(RADIAL_CONFINEMENT, (self.center[0], self.center[1], self.radius,
                                           self.stiffness))


class AabbConfinementField(Field):
    """`AabbConfinementField` (forces/fields/confinement.rs): spring back inside a box."""

    def __init__(self, lo, hi, stiffness):
        self.min = (float(f32(lo[0])), float(f32(lo[1])))
        self.max = (float(f32(hi[0])), float(f32(hi[1])))
        self.stiffness = f32(stiffness)

    @classmethod
    def new(cls, lo, hi, stiffness):
        return cls(lo, hi, stiffness)

    def pack(self, data):
        return _entry(AABB_CONFINEMENT, (self.min[0], self.min[1], self.max[0], self.max[1],
                                         self.stiffness))


class CoulombField(Field):
    """`CoulombField` (forces/fields/coulomb.rs): softened point charges acting on charged
    materials, a = k q_src q_p r / (r^2 + eps^2)^(3/2) / m."""

    def __init__(self, sources, material_charges, coulomb_constant, softening):
        self.sources = [((float(f32(p[0])), float(f32(p[1]))), float(f32(q))) for p, q in sources]
        self.material_charges = {int(k): float(f32(v)) for k, v in material_charges.items()}
        self.coulomb_constant = f32(coulomb_constant)
        self.softening = f32(softening)
        self.cutoff = f32(INF)
        self.switch_on = f32(INF)

    @classmethod
    def new(cls, sources, material_charges, coulomb_constant, softening):
        return cls(sources, material_charges, coulomb_constant, softening)

    def with_cutoff(self, cutoff):
        self.cutoff = f32(cutoff)
        self.switch_on = f32(FADE_ONSET_RATIO * self.cutoff)
        return self

    def pack(self, data):
        table = _charge_table(self.material_charges)
        e = _entry(COULOMB, (self.coulomb_constant, self.softening, self.cutoff, self.switch_on),
                   count=len(self.sources), data_offset=len(data), n_charges=len(table))
        for (x, y), q in self.sources:
            data += [x, y, q]
        data += table
        return e


class UniformElectricField(Field):
    """`UniformElectricField` (forces/fields/em.rs): a = E q / m for charged materials."""

    def __init__(self, field, material_charges):
        self.field = (float(f32(field[0])), float(f32(field[1])))
        self.material_charges = {int(k): float(f32(v)) for k, v in material_charges.items()}

    @classmethod
    def new(cls, field, material_charges):
        return cls(field, material_charges)

    @classmethod
    def for_material(cls, field, material_id, charge):
        return cls(field, {material_id: charge})

    def pack(self, data):
        table = _charge_table(self.material_charges)
        e = _entry(UNIFORM_ELECTRIC, self.field, data_offset=len(data), n_charges=len(table))
        data += table
        return e


class ChemotaxisField(Field):
    """`ChemotaxisField` (forces/fields/chemotaxis.rs): a = sensitivity * grad(phi) by central
    differences at the particle's cell; phi is a grid_res^2 potential indexed x * res + y."""

    def __init__(self, grid_res, sensitivity):
        self.grid_res = int(grid_res)
        self.phi = np.zeros(self.grid_res * self.grid_res, dtype=np.float32)
        self.sensitivity = f32(sensitivity)
        self.material_filter = None

    @classmethod
    def new(cls, grid_res, sensitivity):
        return cls(grid_res, sensitivity)

    def with_material_filter(self, material_id):
        self.material_filter = int(material_id)
        return self

    def sync_from(self, phi):
        """Copies a potential (the reference copies ScalarDiffusionField::current_phi)."""
        phi = np.asarray(phi, dtype=np.float32).ravel()
        if phi.size != self.phi.size:
            raise ValueError("ChemotaxisField grid_res mismatch")
        self.phi[:] = phi

    def pack(self, data):
        e = _entry(CHEMOTAXIS, (self.sensitivity,), count=self.grid_res, data_offset=len(data),
                   material_filter=ALL_MATERIALS if self.material_filter is None else self.material_filter)
        data += self.phi.tolist()
        return e


class NBodyGravityField(Field):
    """`NBodyGravityField` (forces/fields/n_body.rs:287-361): Plummer-softened gravity of every
    particle of positive mass on every particle, a = G M r / (|r|^2 + eps^2)^(3/2), through a
    Barnes-Hut quadtree rebuilt each substep from the post-G2P positions; a node whose width
    over its distance is below theta pulls with its center of mass.  max_depth (default 8)
    and max_bodies_per_node (default 4) shape the tree; the device takes max_depth up to 10,
    and all NBody fields of one simulation share both."""

    def __init__(self, gravitational_constant, softening, theta):
        theta = f32(theta)
        if not (theta > 0.0 and theta <= 1.0):  # NBodyGravityField::new's assertion
            raise ValueError(f"theta must be in (0, 1]; got {float(theta)}. "
                             "0.5 is a common Barnes-Hut trade-off value in practice.")
        self.gravitational_constant = f32(gravitational_constant)
        self.softening = f32(softening)
        self.theta = theta
        self.max_depth = 8
        self.max_bodies_per_node = 4

    @classmethod
    def new(cls, gravitational_constant, softening, theta):
        return cls(gravitational_constant, softening, theta)

    def pack(self, data):
        depth, maxb = int(self.max_depth), int(self.max_bodies_per_node)
        if depth < 0 or maxb < 0:
            raise ValueError("max_depth and max_bodies_per_node must be non-negative")
        return _entry(NBODY_GRAVITY, (self.gravitational_constant, self.softening, self.theta,
                                      depth, maxb))


class orbit:
    """Orbit helpers for bodies under NBodyGravityField (n_body.rs:366-429), f32 like the
    reference; units are grid cells and cells/s, g the field's gravitational_constant."""
    _EPS = float(np.finfo(np.float32).eps)

    @staticmethod
    def circular_velocity(g, central_mass, orbit_radius):
        if f32(orbit_radius) <= orbit._EPS:
            return f32(0.0)
        return f32(np.sqrt(f32(g) * f32(central_mass) / f32(orbit_radius)))

    @staticmethod
    def circular_velocity_softened(g, central_mass, orbit_radius, softening):
        r, e = f32(orbit_radius), f32(softening)
        norm_s = r * r + e * e
        if norm_s <= orbit._EPS:
            return f32(0.0)
        return f32(r * np.sqrt(f32(g) * f32(central_mass) / (norm_s * np.sqrt(norm_s))))

    @staticmethod
    def escape_velocity(g, central_mass, distance):
        if f32(distance) <= orbit._EPS:
            return f32(0.0)
        return f32(np.sqrt(f32(2.0) * f32(g) * f32(central_mass) / f32(distance)))

    @staticmethod
    def elliptical_velocity(g, central_mass, distance, eccentricity, at_periapsis):
        d = f32(distance)
        if d <= orbit._EPS:
            return f32(0.0)
        mu = f32(g) * f32(central_mass)
        sign = f32(1.0) if at_periapsis else f32(-1.0)
        semimajor = d / (f32(1.0) - f32(eccentricity) * sign)
        return f32(np.sqrt(max(mu * (f32(2.0) / d - f32(1.0) / semimajor), f32(0.0))))


def pack_fields(fields) -> tuple:
    """(table, data) for a list of fields in application order."""
    data: list = []
    table = [f.pack(data) for f in fields]
    return table, data
