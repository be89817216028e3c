"""Force fields and ASFLIP on the device vs the CPU oracle (through the C ABI), on the
field scene (tests/scenes.py::field_scene: a NeoHookean block and a fluid block, every 7th
particle pinned, one field of each device kind, ASFLIP off and at 0.9).

Reference order: per particle 1e-5 after one frame against the oracle with correctly
rounded math (the C library's last-bit behaviour is isolated by test_gpu_models), and
after one substep against the C library's math.  Fast path: per particle after one substep
(fast bars of test_gpu_parity), and mass, momentum and region statistics after ten frames.
"""
import numpy as np
import pytest

from emerge_engine_b200 import Batch, DeterministicSimulation, Simulation
from oracle.oracle import OracleSimulation, correctly_rounded_math
from tests import scenes
from tests.test_gpu_parity import compare_particles, tol

pytestmark = pytest.mark.gpu

CASES = [(0.0, True), (0.9, False), (0.9, True)]


@pytest.mark.parametrize("asflip,fields", CASES)
def test_fields_one_frame_reference_order(cuda_lib, asflip, fields):
    g = scenes.field_scene(DeterministicSimulation, asflip=asflip, fields=fields)
    g.step()
    with correctly_rounded_math():
        c = scenes.field_scene(OracleSimulation, asflip=asflip, fields=fields)
        c.step()
    assert g.last_substeps() == c.last_substeps()
    pg, pc = g.particles(), c.particles()
    stats = compare_particles(pg, pc, **tol("reference_order"))
    pinned = pc["pinned"] == 1
    np.testing.assert_array_equal(pg["x"][pinned], pc["x"][pinned])
    print("asflip", asflip, "fields", fields, "reference order 1 frame", stats)


@pytest.mark.parametrize("asflip,fields", CASES)
def test_fields_one_substep_reference_order_libm(cuda_lib, asflip, fields):
    g = scenes.field_scene(DeterministicSimulation, asflip=asflip, fields=fields, dt=1e-3)
    c = scenes.field_scene(OracleSimulation, asflip=asflip, fields=fields, dt=1e-3)
    g.step()
    c.step()
    assert g.last_substeps() == c.last_substeps() == 1
    compare_particles(g.particles(), c.particles(), **tol("reference_order"))


@pytest.mark.parametrize("asflip,fields", CASES)
def test_fields_fast(cuda_lib, asflip, fields):
    g = scenes.field_scene(Simulation, asflip=asflip, fields=fields, dt=1e-3)
    c = scenes.field_scene(OracleSimulation, asflip=asflip, fields=fields, dt=1e-3)
    g.step()
    c.step()
    assert g.last_substeps() == c.last_substeps() == 1
    print("asflip", asflip, "fields", fields, "fast 1 substep",
          compare_particles(g.particles(), c.particles(), **tol("fast")))
    g = scenes.field_scene(Simulation, asflip=asflip, fields=fields)
    c = scenes.field_scene(OracleSimulation, asflip=asflip, fields=fields)
    g.step_n(10)
    c.step_n(10)
    pg, pc = g.particles(), c.particles()
    assert pg["mass"].sum(dtype=np.float64) == pc["mass"].sum(dtype=np.float64)
    m = pc["mass"].astype(np.float64)
    p_abs = (m * np.linalg.norm(pc["v"].astype(np.float64), axis=1)).sum()
    dp = (m[:, None] * pg["v"]).sum(0) - (m[:, None] * pc["v"]).sum(0)
    assert np.linalg.norm(dp) <= 1e-3 * p_abs
    for center, r in (((48.0, 48.0), 96.0), ((30.0, 20.0), 12.0), ((62.0, 30.0), 12.0)):
        sg, sc = g.region_state(center, r), c.region_state(center, r)
        assert sg.count == sc.count
        for k in ("avg_speed", "avg_det_f", "avg_density"):
            assert getattr(sg, k) == pytest.approx(getattr(sc, k), rel=1e-3, abs=1e-6), (k, center)


def test_field_api_on_the_device(cuda_lib):
    from emerge_engine_b200 import BuoyancyField, LinearDragField
    sim = scenes.field_scene(Simulation, fields=False)
    sim.add_force_field(BuoyancyField.new(2.0, (0.0, -1.0)))
    sim.add_named_force_field("wind", LinearDragField.new((1.0, 0.0), 0.5, LinearDragField.ALL_MATERIALS))
    assert sim.force_field_names() == ["force_field_0", "wind"]
    sim.step()
    assert sim.remove_force_field("wind")
    sim.clear_force_fields()
    sim.step()
    assert np.isfinite(sim.particles()["v"]).all()
    with pytest.raises(Exception):
        Batch([scenes.field_scene(Simulation)])  # fields run as single simulations


# ---------------------------------------------------------------- NBodyGravityField
NBODY_CASES = [  # layout, particles, G, softening, theta, max_depth, max_bodies_per_node
    ("blobs", 20_000, 20.0, 1.0, 0.5, 8, 4),
    ("uniform", 50_000, 5.0, 0.5, 1.0, 8, 4),
    ("blobs", 30_000, 20.0, 2.0, 0.3, 10, 1),
    ("clustered", 40_000, 10.0, 0.01, 0.7, 6, 2),
    ("duplicates", 25_000, 1.0, 1.0, 0.5, 8, 0),
    ("uniform", 3_000, 3.0, 0.5, 0.5, 0, 4),
    ("blobs", 1, 3.0, 0.5, 0.5, 8, 4),
]


def _with_points(cls, p, field):
    from emerge_engine_b200 import SimConfig
    sim = cls.empty(SimConfig.standard(128, 0.05, (0.0, 0.0)))
    sim.add_particles(p)
    sim.add_force_field(field)
    return sim


def assert_fast_nbody_close(got, want):
    """The fast pipeline's centers of mass are lane sums (sum m x / sum m), not the
    reference's body-by-body fold: the same tree, the same open/far decisions (they depend on
    box centers only), centers of mass that differ by the two summations' rounding (a
    node's fold over ~10^4 bodies rounds by ~1e-4 of a cell itself).  Far pulls largely
    cancel in an even distribution, so the bar is on the field's scale: every particle within
    2e-4 of the RMS |a| (the Barnes-Hut approximation itself is ~4e-3 at the median)."""
    got, want = got.astype(np.float64), want.astype(np.float64)
    mag = np.linalg.norm(want, axis=1)
    rms = np.sqrt((mag ** 2).mean()) if mag.size else 0.0
    err = np.linalg.norm(got - want, axis=1)
    assert np.all(err <= 2e-4 * rms), (err.max(), rms)
    return float(err.max() / rms) if rms > 0 else 0.0


@pytest.mark.parametrize("cls", [Simulation, DeterministicSimulation])
@pytest.mark.parametrize("layout,n,g,soft,theta,depth,maxb", NBODY_CASES)
def test_nbody_accelerations_match_the_oracle(cuda_lib, cls, layout, n, g, soft, theta, depth, maxb):
    """The device tree (built from sorted quadrant paths) and its traversal against the
    oracle's one-at-a-time insertion and recursion, for any tree shape: in the reference-order
    mode (centers of mass folded in insertion order) identical bits; on the fast pipeline
    within its bar."""
    p = scenes.nbody_points(n, seed=n + depth, layout=layout)
    field = scenes.nbody_field(g, soft, theta, depth, maxb)
    got = _with_points(cls, p, field).field_accelerations()
    want = _with_points(OracleSimulation, p, field).field_accelerations()
    if cls is DeterministicSimulation:
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
    else:
        print("nbody fast accelerations", layout, n, "max error / RMS |a|", assert_fast_nbody_close(got, want))


def test_nbody_with_other_fields_in_order(cuda_lib):
    from emerge_engine_b200 import LinearDragField, RadialConfinementField
    p = scenes.nbody_points(10_000, seed=2, layout="blobs")
    p["v"] = np.float32(0.5)
    out = []
    for cls in (DeterministicSimulation, Simulation, OracleSimulation):
        sim = _with_points(cls, p, RadialConfinementField.new((64.0, 64.0), 30.0, 0.3))
        sim.add_force_field(scenes.nbody_field(G=8.0))
        sim.add_force_field(LinearDragField.new((1.0, 0.0), 0.4, LinearDragField.ALL_MATERIALS))
        out.append(sim.field_accelerations())
    np.testing.assert_array_equal(out[0].view(np.uint32), out[2].view(np.uint32))
    assert_fast_nbody_close(out[1], out[2])


def test_two_nbody_fields_share_one_tree(cuda_lib):
    """Two NBody fields of one tree shape with their own G, softening and theta, a drag field
    between them: each field's walk has its own result block and the sum keeps the
    application order -- identical bits in the reference-order mode, the fast bar otherwise."""
    from emerge_engine_b200 import LinearDragField
    p = scenes.nbody_points(20_000, seed=9, layout="blobs")
    p["v"] = np.float32(0.25)
    out = []
    for cls in (DeterministicSimulation, Simulation, OracleSimulation):
        sim = _with_points(cls, p, scenes.nbody_field(G=6.0, softening=0.8, theta=0.4, max_depth=7, max_bodies=3))
        sim.add_force_field(LinearDragField.new((0.5, 0.0), 0.3, LinearDragField.ALL_MATERIALS))
        sim.add_force_field(scenes.nbody_field(G=2.0, softening=1.5, theta=0.9, max_depth=7, max_bodies=3))
        out.append(sim.field_accelerations())
    np.testing.assert_array_equal(out[0].view(np.uint32), out[2].view(np.uint32))
    assert_fast_nbody_close(out[1], out[2])


def test_nbody_parameters_are_checked(cuda_lib):
    from emerge_engine_b200.abi import EmergeError
    sim = scenes.nbody_scene(Simulation)
    with pytest.raises(EmergeError):  # above the device tree's depth limit
        sim.add_force_field(scenes.nbody_field(max_depth=11))
    sim.clear_force_fields()
    sim.add_force_field(scenes.nbody_field(max_depth=6))
    with pytest.raises(EmergeError):  # two trees of different shape
        sim.add_force_field(scenes.nbody_field(max_depth=7))
    sim.clear_force_fields()
    sim.add_force_field(scenes.nbody_field(max_depth=6, theta=0.4))
    sim.add_force_field(scenes.nbody_field(max_depth=6, theta=0.9, G=2.0))  # one tree, two fields
    sim.step()
    assert np.all(np.isfinite(sim.particles()["x"]))


@pytest.mark.parametrize("pinned_every", [0, 5])
def test_nbody_scene_one_frame_reference_order(cuda_lib, pinned_every):
    g = scenes.nbody_scene(DeterministicSimulation, pinned_every=pinned_every)
    g.step()
    with correctly_rounded_math():
        c = scenes.nbody_scene(OracleSimulation, pinned_every=pinned_every)
        c.step()
    assert g.last_substeps() == c.last_substeps()
    print("nbody reference order 1 frame", compare_particles(g.particles(), c.particles(), **tol("reference_order")))


def test_nbody_scene_fast(cuda_lib):
    g = scenes.nbody_scene(Simulation, dt=1e-3)
    c = scenes.nbody_scene(OracleSimulation, dt=1e-3)
    g.step()
    c.step()
    assert g.last_substeps() == c.last_substeps() == 1
    print("nbody fast 1 substep", compare_particles(g.particles(), c.particles(), **tol("fast")))
    g = scenes.nbody_scene(Simulation)
    c = scenes.nbody_scene(OracleSimulation)
    g.step_n(5)
    c.step_n(5)
    pg, pc = g.particles(), c.particles()
    assert pg["mass"].sum(dtype=np.float64) == pc["mass"].sum(dtype=np.float64)
    m = pc["mass"].astype(np.float64)
    p_abs = (m * np.linalg.norm(pc["v"].astype(np.float64), axis=1)).sum()
    dp = (m[:, None] * pg["v"]).sum(0) - (m[:, None] * pc["v"]).sum(0)
    assert np.linalg.norm(dp) <= 1e-3 * p_abs
    for center, r in (((64.0, 64.0), 128.0), ((38.0, 51.0), 14.0), ((87.0, 70.0), 12.0)):
        sg, sc = g.region_state(center, r), c.region_state(center, r)
        assert sg.count == sc.count
        for k in ("avg_speed", "avg_det_f"):
            assert getattr(sg, k) == pytest.approx(getattr(sc, k), rel=1e-3, abs=1e-6), (k, center)


def test_nbody_with_the_sleep_partition_reference_order(cuda_lib):
    """The tree inserts the bodies in reference index order, which the sleep partition
    changes every substep (a sleeping particle swaps with the last awake one): with sleep on,
    the reference-order mode stays within the reference-order bar of the oracle frame by
    frame, with the same partition size."""
    def build_cfg(cls):
        from emerge_engine_b200 import NeoHookeanMaterial, SimConfig, SpawnRegion
        cfg = SimConfig.standard(128, 0.05, (0.0, 0.0))
        cfg.sleep_threshold = 0.05
        sim = cls.empty(cfg).with_default_material(NeoHookeanMaterial.new(400.0, 200.0))
        for k, (cx, cy, side, v) in enumerate(((0.3, 0.4, 18, 0.0), (0.68, 0.55, 14, 1.0))):
            sp = SpawnRegion.for_sim(cfg)
            sp.spacing, sp.box_size, sp.box_center = 0.5, (side, side), (128 * cx, 128 * cy)
            sp.position_jitter, sp.rng_seed, sp.initial_velocity_scale = 0.3, 30 + k, v
            sim.add_body(sp)
        sim.add_force_field(scenes.nbody_field(G=0.5))
        return sim

    g = build_cfg(DeterministicSimulation)
    fewest_awake = None
    with correctly_rounded_math():
        c = build_cfg(OracleSimulation)
        for k in range(4):
            g.step()
            c.step()
            assert g.last_substeps() == c.last_substeps(), k
            assert g.active_count() == c.active_count(), k
            compare_particles(g.particles(), c.particles(), **tol("reference_order"))
            fewest_awake = min(fewest_awake or c.active_count(), c.active_count())
    assert fewest_awake < c.particle_count()  # part of the scene slept: the partition was in use

