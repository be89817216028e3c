"""Edge cases of the step on the device against the CPU oracle (through the C ABI), in
reference order and bit for bit with the oracle rounding exp/log/pow correctly:

* an empty simulation still takes its frame as one substep (step.rs:34-49), and a body
  added to it afterwards steps like the oracle's;
* particle counts that leave partial warps and CTAs (12, 49, 260, 1133 particles);
* grids whose side is not a multiple of the 8-cell tile (37, 61, 100 cells);
* particles on the domain boundary pushed outward, with stencils reaching past the grid;
* a frame that hits the substep cap (max_substeps_per_step);
* a simulation whose particles all leave the active zone of a sleep partition.
"""
import numpy as np
import pytest

from emerge_engine_b200 import (DeterministicSimulation, NeoHookeanMaterial, NewtonianFluidMaterial,
                                SimConfig, Simulation, SlipBoundary, SpawnRegion)
from oracle.oracle import OracleSimulation, correctly_rounded_math

pytestmark = pytest.mark.gpu


def same(g, c, what):
    assert g.last_substeps() == c.last_substeps(), what
    assert g.effective_dt() == c.effective_dt(), what
    pg, pc = g.particles(), c.particles()
    assert len(pg) == len(pc), what
    np.testing.assert_array_equal(pg["x"], pc["x"], err_msg=what)
    np.testing.assert_array_equal(pg["v"], pc["v"], err_msg=what)
    np.testing.assert_array_equal(pg["f"], pc["f"], err_msg=what)


def blocks_scene(cls, res, boxes, seed=3, dt=0.05, **cfg_kw):
    cfg = SimConfig.standard(res, dt, (0.0, -1.0))
    for k, v in cfg_kw.items():
        setattr(cfg, k, v)
    sim = (cls.empty(cfg).with_default_material(NeoHookeanMaterial.new(400.0, 200.0))
           .with_material(1, NewtonianFluidMaterial.low_viscosity(1000.0, 1e4)))
    for i, (size, center, mat, shape) in enumerate(boxes):
        s = SpawnRegion.for_sim(cfg)
        s.spacing, s.box_size, s.box_center, s.material_id = 0.5, size, center, mat
        s.position_jitter, s.rng_seed = 0.3, seed + i
        if shape is not None:
            s = s.disk(shape)
        sim.add_body(s)
    return sim


def test_empty_simulation_steps_like_the_reference(cuda_lib):
    cfg = SimConfig.standard(64, 0.05, (0.0, -1.0))
    g = DeterministicSimulation.empty(cfg)
    c = OracleSimulation.empty(cfg)
    for sim in (g, c):
        sim.step()
    assert g.particle_count() == 0 and len(g.particles()) == 0
    assert g.last_substeps() == c.last_substeps() == 1
    assert g.effective_dt() == c.effective_dt()
    assert g.region_state((32.0, 32.0), 10.0).count == 0
    with correctly_rounded_math():
        for sim in (g, c):
            sim.with_default_material(NeoHookeanMaterial.new(400.0, 200.0))
            sim.add_body(SpawnRegion(spacing=0.5, box_size=(6, 5), box_center=(32.0, 40.0)))
            sim.step_n(3)
        same(g, c, "after add_body")
    f = Simulation.empty(cfg)
    f.step_n(2)
    assert f.last_substeps() == 1


@pytest.mark.parametrize("boxes", [
    [((3, 1), (20.0, 30.0), 0, None)],                                   # 12 particles
    [((4, 4), (20.0, 30.0), 0, 2.0)],                                    # a small disk
    [((8, 8), (20.0, 30.0), 0, None), ((1, 1), (40.0, 20.0), 1, None)],  # 256 + 4
    [((15, 17), (30.0, 28.0), 1, None), ((5, 5), (12.0, 40.0), 0, 3.0)],
], ids=["12", "disk", "260", "mixed"])
def test_ragged_particle_counts(cuda_lib, boxes):
    g = blocks_scene(DeterministicSimulation, 64, boxes)
    with correctly_rounded_math():
        c = blocks_scene(OracleSimulation, 64, boxes)
        assert g.particle_count() == c.particle_count()
        for k in range(3):
            g.step()
            c.step()
            same(g, c, f"frame {k}, {g.particle_count()} particles")


@pytest.mark.parametrize("res", [37, 61, 100])
def test_grid_sides_off_the_tile(cuda_lib, res):
    boxes = [((res // 3, res // 4), (res / 2.0, res / 3.0), 0, None),
             ((res // 5, res // 5), (res / 3.0, 2.0 * res / 3.0), 1, None)]
    g = blocks_scene(DeterministicSimulation, res, boxes)
    with correctly_rounded_math():
        c = blocks_scene(OracleSimulation, res, boxes)
        for k in range(3):
            g.step()
            c.step()
            same(g, c, f"grid {res} frame {k}")


def test_boundary_particles_pushed_outward(cuda_lib):
    """Particles against every wall with velocities into it: the slip walls, the position
    clamp and stencils that reach past the grid's edge."""
    res = 48
    boxes = [((4, 40), (3.0 + 2.0, 24.0), 0, None), ((4, 40), (res - 5.0, 24.0), 1, None),
             ((36, 3), (24.0, 3.0 + 1.5), 0, None)]

    def build(cls):
        sim = blocks_scene(cls, res, boxes)
        p = sim.particles()
        x = p["x"]
        p["v"][:, 0] = np.where(x[:, 0] < res / 2, -40.0, 40.0).astype(np.float32)
        p["v"][:, 1] = np.where(x[:, 1] < 8.0, -40.0, 5.0).astype(np.float32)
        sim.set_particles(p)
        return sim
    g = build(DeterministicSimulation)
    with correctly_rounded_math():
        c = build(OracleSimulation)
        for k in range(3):
            g.step()
            c.step()
            same(g, c, f"frame {k}")
    x = g.particles()["x"]
    assert x.min() >= 1.0 and x.max() <= res - 2.0


def test_frame_that_hits_the_substep_cap(cuda_lib):
    boxes = [((16, 8), (32.0, 20.0), 0, None)]
    g = blocks_scene(DeterministicSimulation, 64, boxes, dt=2.0, max_substeps_per_step=3)
    with correctly_rounded_math():
        c = blocks_scene(OracleSimulation, 64, boxes, dt=2.0, max_substeps_per_step=3)
        for k in range(2):
            g.step()
            c.step()
            same(g, c, f"frame {k}")
            assert g.last_substeps() == 3
            assert g.last_counters()[:2] == c.last_counters()[:2]
            assert g.last_counters()[2] > 0.0  # the frame's time left over (solver/mod.rs:65)


def test_every_particle_asleep(cuda_lib):
    """A resting block that falls asleep whole: the passes run over an empty active zone."""
    boxes = [((16, 6), (32.0, 2.0 + 1.0 + 3.0), 0, None)]
    g = blocks_scene(DeterministicSimulation, 64, boxes, sleep_threshold=10.0)
    with correctly_rounded_math():
        c = blocks_scene(OracleSimulation, 64, boxes, sleep_threshold=10.0)
        for k in range(3):
            g.step()
            c.step()
            same(g, c, f"frame {k}")
            assert g.active_count() == c.active_count()
    assert g.active_count() == 0
