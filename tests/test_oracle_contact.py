"""Pins the oracle's multi-field contact and two-phase mixture coupling to the reference's own
tests for them (grid/contact_normal.rs LR fits, tests/physics_correctness.rs Coulomb slip /
stick, tests/solver.rs mixture drag), plus invariants of the contact and mixture scenes.
"""
from ctypes import c_float

import numpy as np
import pytest

from emerge_engine_b200 import (CorotatedMaterial, DirectionalContactGrip, DruckerPragerMaterial,
                                FLUID_PHASE, NewtonianFluidMaterial, SOLID_PHASE, SimConfig,
                                SlipBoundary, SpawnRegion, WithMixturePhase)
from oracle.oracle import OracleSimulation, lib
from tests import scenes


def fit(points, node, cell=1.0):
    arr = (c_float * (3 * len(points)))(*[v for p in points for v in (p[0], p[1], p[2])])
    out = (c_float * 2)()
    ok = lib().oracle_fit_contact_normal(arr, len(points), node[0], node[1], cell, out)
    return (out[0], out[1]) if ok else None


# ---------------------------------------------------------------- grid/contact_normal.rs tests
def test_lr_fit_recovers_the_corner_case_normal():
    pts = [(28.0 + i * 0.5, 8.25 + j * 0.3, -1.0) for i in range(8) for j in range(4)]
    pts += [(28.0 + i * 0.5, 10.25 + j * 0.3, 1.0) for i in range(4) for j in range(4)]
    n = fit(pts, (30.0, 10.0))
    assert n is not None and abs(n[0]) < 0.1


def test_lr_fit_clean_horizontal_interface():
    pts = []
    for i in range(6):
        for j in range(6):
            pts.append((30.0 + i * 0.5, 10.25 + j * 0.3, 1.0))
            pts.append((30.0 + i * 0.5, 8.25 + j * 0.3, -1.0))
    n = fit(pts, (32.0, 10.0))
    assert n is not None and abs(n[0]) < 0.1


def test_lr_fit_needs_both_labels():
    assert fit([(1.0, 1.0, 1.0), (2.0, 1.0, 1.0)], (1.0, 1.0)) is None


# ---------------------------------------------------------------- physics_correctness.rs:2015-2100
def coulomb_run(friction):
    cfg = SimConfig.standard(64, 0.02, (0.0, -0.3))
    cfg.contact_friction, cfg.min_dt, cfg.max_substeps_per_step = friction, 0.001, 128
    cfg.project_invalid_state = True
    sim = OracleSimulation.new(cfg, SpawnRegion(spacing=0.5, box_size=(6, 6), box_center=(32.0, 11.6),
                                                precompute_initial_volumes=True))
    sim = sim.with_default_material(CorotatedMaterial.new(200.0, 400.0)).with_boundary(SlipBoundary(2))
    p = sim.particles()
    block = len(p)
    p["contact_group"] = 1
    sim.set_particles(p)
    sim = sim.with_material(1, CorotatedMaterial.new(200.0, 400.0))
    sim.add_body(SpawnRegion(spacing=0.5, box_size=(48, 8), box_center=(32.0, 8.0), material_id=1,
                             precompute_initial_volumes=True))
    sim.step_n(300)
    p = sim.particles()
    p["v"][:block, 0] = 3.0
    sim.set_particles(p)
    sim.step_n(150)
    return float(sim.particles()["v"][:block, 0].mean())


def test_contact_coulomb_slip_and_stick():
    assert coulomb_run(0.0) > 1.0
    assert coulomb_run(3.0) < 0.5


# ---------------------------------------------------------------- tests/solver.rs:1888-1990
def mixture_pair(drag):
    cfg = SimConfig(grid_res=32, dt=0.1, adaptive_timestep=True, gravity=(0.0, 0.0))
    cfg.mixture_drag_coefficient = drag
    solid = WithMixturePhase(DruckerPragerMaterial.from_young_modulus(1.0e6, 0.2), SOLID_PHASE)
    fluid = WithMixturePhase(NewtonianFluidMaterial.low_viscosity(4.0, 10.0), FLUID_PHASE)
    sim = OracleSimulation.new(cfg, SpawnRegion(spacing=0.5, box_size=(10, 10), box_center=(16.0, 16.0),
                                                precompute_initial_volumes=True))
    sim = sim.with_default_material(solid).with_material(1, fluid)
    sim.add_body(SpawnRegion(spacing=0.5, box_size=(10, 10), box_center=(16.0, 16.0), material_id=1,
                             precompute_initial_volumes=True))
    p = sim.particles()
    p["v"][p["material_id"] == 1] = (0.0, -3.0)
    sim.set_particles(p)
    return sim


def relative_speed(sim):
    p = sim.particles()
    a = p["v"][p["material_id"] == 0].mean(0)
    b = p["v"][p["material_id"] == 1].mean(0)
    return float(np.linalg.norm(a - b))


def test_higher_drag_relaxes_the_phases_faster():
    low, high = mixture_pair(1.0), mixture_pair(50.0)
    start = relative_speed(low)
    low.step_n(1)
    high.step_n(1)
    assert relative_speed(low) < start
    assert relative_speed(high) < relative_speed(low)


# ---------------------------------------------------------------- scene invariants
@pytest.mark.parametrize("grip", [None, DirectionalContactGrip(0.1, 0.9, (1.0, 0.0))])
def test_contact_scene_conserves_mass(grip):
    sim = scenes.contact_scene(OracleSimulation, grip=grip)
    m0 = sim.particles()["mass"].sum(dtype=np.float64)
    sim.step_n(6)
    p = sim.particles()
    assert p["mass"].sum(dtype=np.float64) == m0 and np.isfinite(p["v"]).all()


def test_directional_grip_changes_the_outcome():
    a = scenes.contact_scene(OracleSimulation)
    b = scenes.contact_scene(OracleSimulation, grip=DirectionalContactGrip(0.0, 1.0, (-1.0, 0.0)))
    a.step_n(20)
    b.step_n(20)
    assert np.abs(a.particles()["v"] - b.particles()["v"]).max() > 1e-4


@pytest.mark.parametrize("iterations", [0, 2])
def test_mixture_scene_conserves_mass(iterations):
    sim = scenes.mixture_scene(OracleSimulation, iterations=iterations)
    m0 = sim.particles()["mass"].sum(dtype=np.float64)
    sim.step_n(3)
    p = sim.particles()
    assert p["mass"].sum(dtype=np.float64) == m0 and np.isfinite(p["v"]).all()
