"""Pins the oracle's force fields and ASFLIP to the reference's own tests for them
(forces/fields/*.rs unit tests, solver/cutoff.rs, tests/accuracy.rs ASFLIP tests), plus the
field pass's invariants on whole scenes.
"""
from ctypes import POINTER, byref, c_float

import numpy as np
import pytest

from emerge_engine_b200 import (AabbConfinementField, BuoyancyField, ChemotaxisField,
                                CoulombField, GravityWellField, LinearDragField,
                                NeoHookeanMaterial, RadialConfinementField, SimConfig,
                                SpawnRegion, UniformElectricField)
from emerge_engine_b200.abi import Particle
from emerge_engine_b200.fields import pack_fields
from oracle.oracle import OracleSimulation, lib
from tests import scenes

f32 = np.float32


def accel(field, x=(0.0, 0.0), v=(0.0, 0.0), mass=1.0, density=1.0, material_id=0):
    table, data = pack_fields([field])
    d = np.asarray(data if data else [0.0], dtype=np.float32)
    p = Particle()
    p.x[:] = x
    p.v[:] = v
    p.mass, p.density, p.material_id = mass, density, material_id
    out = (c_float * 2)()
    lib().oracle_field_acceleration(byref(table[0]), d.ctypes.data_as(POINTER(c_float)), byref(p), out)
    return np.array([out[0], out[1]], dtype=np.float64)


# ---------------------------------------------------------------- solver/cutoff.rs:33-44
def test_smooth_cutoff_through_a_gravity_well():
    """cutoff 10 gives switch_on 8.5: full force inside, none at or past the cutoff, a
    fraction in between."""
    well = GravityWellField.point((0.0, 0.0), 1.0, 1.0, 0.0).with_cutoff(10.0)
    free = GravityWellField.point((0.0, 0.0), 1.0, 1.0, 0.0)
    for r in (7.0, 8.0):
        np.testing.assert_array_equal(accel(well, (r, 0.0)), accel(free, (r, 0.0)))
    assert np.all(accel(well, (10.0, 0.0)) == 0.0) and np.all(accel(well, (11.0, 0.0)) == 0.0)
    ratio = accel(well, (9.0, 0.0))[0] / accel(free, (9.0, 0.0))[0]
    assert 0.0 < ratio < 1.0


def test_gravity_well_points_at_the_source_with_plummer_magnitude():
    g, m, eps = 0.5, 40.0, 2.0
    well = GravityWellField.point((10.0, 10.0), m, g, eps)
    a = accel(well, (13.0, 14.0))
    r = np.array([-3.0, -4.0])
    expect = r * g * m / (25.0 + eps * eps) ** 1.5
    np.testing.assert_allclose(a, expect, rtol=1e-6)
    assert np.all(accel(well, (10.0, 10.0)) == 0.0)  # r < EPSILON: skipped


# ---------------------------------------------------------------- buoyancy.rs:76-108
@pytest.mark.parametrize("rho,sign", [(600.0, 1), (7800.0, -1)])
def test_buoyancy_floats_light_and_slows_heavy(rho, sign):
    g = np.array([0.0, -9.8])
    net = g + accel(BuoyancyField.new(1000.0, tuple(g)), density=rho)
    assert np.sign(net[1]) == sign
    if sign < 0:
        assert net[1] > g[1]


def test_buoyancy_matching_density_hovers():
    g = np.array([0.0, -9.8])
    assert np.linalg.norm(g + accel(BuoyancyField.new(1000.0, tuple(g)), density=1000.0)) < 1e-4


# ---------------------------------------------------------------- drag.rs:150-177
def test_linear_drag():
    drag = LinearDragField.new((2.0, 0.0), 3.0, LinearDragField.ALL_MATERIALS)
    assert np.all(accel(drag, v=(2.0, 0.0)) == 0.0)
    np.testing.assert_allclose(accel(drag), [6.0, 0.0], atol=1e-6)
    only2 = LinearDragField.new((5.0, 0.0), 1.0, 1 << 2)
    assert np.all(accel(only2, material_id=0) == 0.0)
    assert np.any(accel(only2, material_id=2) != 0.0)


# ---------------------------------------------------------------- confinement.rs
def test_confinement_springs_back_only_outside():
    radial = RadialConfinementField.new((0.0, 0.0), 5.0, 2.0)
    assert np.all(accel(radial, (3.0, 0.0)) == 0.0)
    np.testing.assert_allclose(accel(radial, (8.0, 0.0)), [-6.0, 0.0], atol=1e-6)
    box = AabbConfinementField.new((0.0, 0.0), (10.0, 10.0), 2.0)
    assert np.all(accel(box, (5.0, 5.0)) == 0.0)
    np.testing.assert_allclose(accel(box, (-1.0, 12.0)), [2.0, -4.0], atol=1e-6)


# ---------------------------------------------------------------- em.rs:87-180
def test_uniform_electric_field():
    e = (3.0, -2.0)
    assert np.all(accel(UniformElectricField.for_material(e, 1, 5.0), material_id=0) == 0.0)
    assert np.all(accel(UniformElectricField.for_material(e, 0, 0.0)) == 0.0)
    a = accel(UniformElectricField.for_material(e, 0, 2.0), mass=4.0)
    np.testing.assert_array_equal(a, np.array(e, dtype=np.float32) * f32(2.0 * f32(1.0 / 4.0)))
    a2 = accel(UniformElectricField.for_material(e, 0, 4.0), mass=4.0)
    np.testing.assert_allclose(a2, 2 * a, rtol=1e-6)
    a3 = accel(UniformElectricField.for_material(e, 0, 2.0), mass=8.0)
    np.testing.assert_allclose(a3, a / 2, rtol=1e-6)
    np.testing.assert_allclose(accel(UniformElectricField.for_material(e, 0, -2.0), mass=4.0), -a)
    assert np.all(accel(UniformElectricField.for_material(e, 0, 2.0), mass=0.0) == 0.0)


def test_coulomb_like_charges_repel():
    c = CoulombField.new([((0.0, 0.0), 1.0)], {0: 1.0, 1: -1.0}, 1.0, 0.5)
    assert accel(c, (4.0, 0.0), material_id=0)[0] > 0.0
    assert accel(c, (4.0, 0.0), material_id=1)[0] < 0.0
    assert np.all(accel(c, (4.0, 0.0), material_id=2) == 0.0)


# ---------------------------------------------------------------- chemotaxis.rs:138-190
def ramp(res=8):
    f = ChemotaxisField.new(res, 1.0)
    f.sync_from(np.repeat(np.arange(res, dtype=np.float32), res))  # phi[x * res + y] = x
    return f


def test_chemotaxis_follows_the_gradient():
    a = accel(ramp(), (3.0, 4.0))
    assert a[0] > 0.0 and abs(a[1]) < 1e-5
    neg = ramp()
    neg.sensitivity = f32(-1.0)
    assert accel(neg, (3.0, 4.0))[0] < 0.0
    filt = ramp().with_material_filter(7)
    assert accel(filt, (3.0, 4.0), material_id=7)[0] > 0.0
    assert np.all(accel(filt, (3.0, 4.0), material_id=0) == 0.0)


# ---------------------------------------------------------------- tests/accuracy.rs:471-600
def asflip_split_block(blend):
    cfg = SimConfig.standard(64, 0.1, (0.0, 0.0))
    cfg.max_substeps_per_step, cfg.asflip_blend = 4, blend
    spawn = SpawnRegion(spacing=0.5, box_size=(6, 6), box_center=(32.0, 32.0),
                        precompute_initial_volumes=True)
    sim = OracleSimulation.new(cfg, spawn).with_default_material(NeoHookeanMaterial.new(1.0, 1.0))
    p = sim.particles()
    p["v"][:, 0] = np.where(p["x"][:, 0] - 32.0 < 0.0, -2.0, 2.0)
    p["v"][:, 1] = 0.0
    sim.set_particles(p)
    return sim


def test_asflip_keeps_more_relative_velocity_than_apic():
    apic, asflip = asflip_split_block(0.0), asflip_split_block(0.97)
    apic.step()
    asflip.step()
    keep_apic = np.abs(apic.particles()["v"][:, 0]).mean()
    keep_asflip = np.abs(asflip.particles()["v"][:, 0]).mean()
    assert np.isfinite(keep_apic) and np.isfinite(keep_asflip)
    assert keep_asflip > keep_apic


def test_asflip_conserves_momentum_in_free_fall():
    cfg = SimConfig.standard(64, 0.1, (0.0, -0.3))
    cfg.max_substeps_per_step, cfg.asflip_blend = 32, 0.9
    spawn = SpawnRegion(spacing=0.5, box_size=(6, 6), box_center=(32.0, 48.0),
                        precompute_initial_volumes=True)
    from emerge_engine_b200 import NeoHookeanMaterial as NH
    sim = OracleSimulation.new(cfg, spawn).with_default_material(NH.from_young_modulus(1.0e3, 0.3))
    mass = sim.particles()["mass"].sum(dtype=np.float32)
    sim.step_n(40)
    p = sim.particles()
    py = float((p["mass"] * p["v"][:, 1]).sum())
    expect = float(mass) * -0.3 * 40 * 0.1
    assert abs(py - expect) / max(abs(expect), 1.0) < 0.05


# ---------------------------------------------------------------- the field pass
def test_uniform_field_impulse_and_pinned_particles():
    """v += dt * a on every unpinned particle: with no gravity and only a uniform electric
    field on material 0, total momentum after one step is the field impulse q E t summed
    over the unpinned particles; pinned particles never move."""
    cfg = SimConfig.standard(64, 0.05, (0.0, 0.0))
    sim = OracleSimulation.new(cfg, SpawnRegion(spacing=0.5, box_size=(8, 8), box_center=(32.0, 32.0)))
    sim = sim.with_default_material(NeoHookeanMaterial.new(10.0, 20.0))
    p = sim.particles()
    p["pinned"][::5] = 1
    sim.set_particles(p)
    q, e = 0.2, (1.0, 0.5)
    sim.add_force_field(UniformElectricField.for_material(e, 0, q))
    x0 = sim.particles()["x"].copy()
    sim.step()
    p = sim.particles()
    free = p["pinned"] == 0
    mom = (p["mass"][:, None] * p["v"]).sum(0)
    np.testing.assert_allclose(mom, np.array(e) * q * 0.05 * free.sum(), rtol=1e-3)
    np.testing.assert_array_equal(p["x"][~free], x0[~free])
    assert np.all(p["v"][~free] == 0.0)


def test_field_list_api():
    sim = scenes.field_scene(OracleSimulation, fields=False)
    sim.add_force_field(BuoyancyField.new(2.0, (0.0, -1.0)))
    sim.add_named_force_field("wind", LinearDragField.new((1.0, 0.0), 0.5, LinearDragField.ALL_MATERIALS))
    assert sim.force_field_names() == ["force_field_0", "wind"]
    assert sim.remove_force_field("wind") and not sim.remove_force_field("wind")
    sim.clear_force_fields()
    assert sim.force_field_names() == []


@pytest.mark.parametrize("asflip", [0.0, 0.9])
def test_field_scene_invariants(asflip):
    sim = scenes.field_scene(OracleSimulation, asflip=asflip)
    p0 = sim.particles()
    sim.step_n(5)
    p = sim.particles()
    assert p["mass"].sum(dtype=np.float64) == p0["mass"].sum(dtype=np.float64)
    assert np.isfinite(p["x"]).all() and np.isfinite(p["v"]).all()
    pinned = p0["pinned"] == 1
    np.testing.assert_array_equal(p["x"][pinned], p0["x"][pinned])
