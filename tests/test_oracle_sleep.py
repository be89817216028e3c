"""Sleep partition and particle-set edits on the oracle: the reference's own tests for them
(tests/solver.rs retain / split, tests/gpu.rs sleep freeze / wake properties restated for the
CPU step) and the partition invariant, plus agreement of the host-side edit helpers
(emerge_engine_b200/lifecycle.py) with the oracle's C restatement of wake_tag / sleep_tag.
"""
import numpy as np
import pytest

from emerge_engine_b200 import NeoHookeanMaterial, SimConfig, SlipBoundary, SpawnRegion
from emerge_engine_b200 import lifecycle
from oracle.oracle import OracleSimulation
from tests import scenes


def zone_ok(sim):
    p, a = sim.particles(), sim.active_count()
    return bool(np.all(p["sleeping"][:a] == 0) and np.all(p["sleeping"][a:] == 1))


def test_settled_particles_sleep_and_stay_frozen():
    sim = scenes.sleep_scene(OracleSimulation)
    sim.step()
    p0 = sim.particles()
    asleep = p0["sleeping"] == 1
    assert asleep.sum() == (p0["user_tag"] == 1).sum()  # the resting block, all of it
    assert zone_ok(sim)
    sim.step()
    p1 = sim.particles()
    tags = p0["user_tag"][asleep]
    # a sleeping particle keeps its state bit for bit (matched by position in its tag group)
    still = p1[(p1["sleeping"] == 1)]
    assert len(still) == asleep.sum()
    np.testing.assert_array_equal(np.sort(still["x"][:, 0]), np.sort(p0["x"][asleep][:, 0]))
    assert set(np.unique(tags)) == {1}


def test_activity_wakes_neighbours_and_activation_keeps_awake():
    sim = scenes.sleep_scene(OracleSimulation)
    awake_block = []
    for _ in range(10):
        sim.step()
        p = sim.particles()
        awake_block.append(int(((p["user_tag"] == 1) & (p["sleeping"] == 0)).sum()))
        assert ((p["user_tag"] == 3) & (p["sleeping"] == 1)).sum() == 0
        assert zone_ok(sim)
    assert awake_block[0] == 0 and awake_block[-1] > 0


def test_tag_sleep_and_wake_match_the_host_helpers():
    sim = scenes.sleep_scene(OracleSimulation, threshold=0.0)
    sim.step()
    p, a = sim.particles(), sim.active_count()
    sim.sleep_tag(3)
    q, b = lifecycle.sleep_tag(p, a, 3)
    np.testing.assert_array_equal(sim.particles(), q)
    assert sim.active_count() == b and zone_ok(sim)
    sim.wake_tag(3)
    r, c = lifecycle.wake_tag(q, b, 3)
    np.testing.assert_array_equal(sim.particles(), r)
    assert sim.active_count() == c == len(r)


def test_add_body_goes_before_the_sleeping_zone():
    sim = scenes.sleep_scene(OracleSimulation)
    sim.step()
    a0, n0 = sim.active_count(), sim.particle_count()
    sleeping_before = sim.particles()[a0:]
    s = SpawnRegion(spacing=0.5, box_size=(6, 6), box_center=(70.0, 60.0))
    tag = sim.add_body(s)
    p = sim.particles()
    k = sim.particle_count() - n0
    assert sim.active_count() == a0 + k
    assert np.all(p["user_tag"][a0:a0 + k] == tag)
    np.testing.assert_array_equal(p[a0 + k:], sleeping_before)


# ---------------------------------------------------------------- tests/solver.rs:1690-1720
def test_retain_syncs_active_count_and_steps_cleanly():
    cfg = SimConfig.standard(32, 0.1, (0.0, -0.1))
    sim = (OracleSimulation.empty(cfg).with_default_material(NeoHookeanMaterial.new(100.0, 50.0))
           .with_boundary(SlipBoundary(cfg.boundary_thickness)))
    sim.add_body(SpawnRegion(spacing=0.5, box_size=(16, 16), box_center=(16.0, 16.0)))
    before = sim.particle_count()
    sim.retain_particles(lambda p: p.x[0] < 16.0)
    assert sim.particle_count() < before and sim.active_count() == sim.particle_count()
    sim.step_n(5)
    assert np.isfinite(sim.particles()["x"]).all()


# ---------------------------------------------------------------- tests/solver.rs:1724-1790
def test_split_conserves_mass_and_jitters_apart():
    cfg = SimConfig(grid_res=32, dt=0.1)
    sim = (OracleSimulation.empty(cfg).with_default_material(NeoHookeanMaterial.new(100.0, 50.0))
           .with_boundary(SlipBoundary(cfg.boundary_thickness)))
    sim.add_body(SpawnRegion(spacing=0.5, box_size=(8, 8), box_center=(16.0, 16.0)))
    p = sim.particles()
    p["friction_hardening"][::2] = 10.0
    sim.set_particles(p)
    n0, m0 = sim.particle_count(), p["mass"].sum(dtype=np.float32)
    damaged = int((p["friction_hardening"] > 5.0).sum())
    sim.split_particles(lambda q: q.friction_hardening > 5.0, 0.1)
    q = sim.particles()
    assert sim.particle_count() == n0 + damaged
    assert abs(q["mass"].sum(dtype=np.float32) - m0) < 1e-4
    kids = q[np.abs(q["mass"] - p["mass"][0] * 0.5) < 1e-4]
    assert len(kids) >= 2 and np.any(np.linalg.norm(kids["x"][0] - kids["x"][1:], axis=1) > 0)
    assert sim.active_count() == sim.particle_count()


def test_remove_particles_repartitions_the_sleeping_zone():
    sim = scenes.sleep_scene(OracleSimulation)
    for _ in range(8):
        sim.step()
    before = sim.particle_count()
    removed = sim.remove_particles(lambda q: q.user_tag == 2)
    assert removed > 0 and sim.particle_count() == before - removed
    assert zone_ok(sim)
    sim.step_n(2)
    assert zone_ok(sim) and np.isfinite(sim.particles()["v"]).all()
