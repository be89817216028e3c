"""CUDA step vs the CPU oracle on the same seeded scenes (through the C ABI).

Tolerances (f32; the device sums P2G contributions with float atomics, so the
per-cell summation order differs from the reference's particle-index order):
  * positions: |dx| <= 1e-5 * max(|x_ref|, 1) per particle after one step,
  * velocities: |dv| <= 1e-5 * max(|v_ref|, V_FLOOR) with V_FLOOR = 1e-2 * max|v_ref|
    (the relative bound is taken against a floor so particles at rest, whose v is
    a cancellation of large stress terms, are judged on the scene's velocity scale),
  * total mass: exact (masses are never changed by the step),
  * region_state statistics after many steps: 1e-3 relative.
"""
import numpy as np
import pytest

from emerge_engine_b200 import Simulation, SimConfig, SpawnRegion, NeoHookeanMaterial
from oracle.oracle import OracleSimulation
from tests import scenes

pytestmark = pytest.mark.gpu

X_TOL = 1e-5
V_TOL = 1e-5


def compare_particles(pg, pc, x_tol=X_TOL, v_tol=V_TOL):
    assert len(pg) == len(pc)
    dx = np.linalg.norm(pg["x"].astype(np.float64) - pc["x"], axis=1)
    x_rel = dx / np.maximum(np.linalg.norm(pc["x"], axis=1), 1.0)
    vn = np.linalg.norm(pc["v"].astype(np.float64), axis=1)
    floor = max(1e-2 * vn.max(), 1e-12)
    dv = np.linalg.norm(pg["v"].astype(np.float64) - pc["v"], axis=1)
    v_rel = dv / np.maximum(vn, floor)
    stats = dict(x_rel_max=float(x_rel.max()), v_rel_max=float(v_rel.max()),
                 v_rel_p99=float(np.quantile(v_rel, 0.99)))
    assert x_rel.max() <= x_tol, stats
    assert v_rel.max() <= v_tol, stats
    return stats


def both(builder, *args, **kw):
    return builder(Simulation, *args, **kw), builder(OracleSimulation, *args, **kw)


def test_spawn_state_matches(cuda_lib):
    g, c = both(scenes.quickstart)
    pg, pc = g.particles(), c.particles()
    # spawn lattice, tags and init are integer/exact work on the host side
    np.testing.assert_array_equal(pg["x"], pc["x"])
    np.testing.assert_array_equal(pg["user_tag"], pc["user_tag"])
    np.testing.assert_array_equal(pg["material_id"], pc["material_id"])
    # add_body's local volume estimate ran on the device (float atomics)
    for k in ("initial_volume", "volume", "density"):
        np.testing.assert_allclose(pg[k], pc[k], rtol=1e-6, atol=0)


def test_quickstart_one_step(cuda_lib):
    g, c = both(scenes.quickstart)
    g.step()
    c.step()
    assert g.last_substeps() == c.last_substeps()
    assert g.effective_dt() == pytest.approx(c.effective_dt(), rel=1e-6)
    stats = compare_particles(g.particles(), c.particles())
    print("quickstart 1 step", stats)


def test_quickstart_region_state_60_steps(cuda_lib):
    g, c = both(scenes.quickstart)
    g.step_n(60)
    c.step_n(60)
    pg, pc = g.particles(), c.particles()
    assert pg["mass"].sum(dtype=np.float64) == pc["mass"].sum(dtype=np.float64)
    for center, r in (((40.0, 36.0), 10.0), ((24.0, 40.0), 8.0), ((32.0, 32.0), 100.0)):
        sg, sc = g.region_state(center, r), c.region_state(center, r)
        assert sg.count == sc.count
        for k in ("avg_volume_ratio", "max_volume_ratio", "avg_speed", "avg_det_f", "avg_density"):
            a, b = getattr(sg, k), getattr(sc, k)
            assert a == pytest.approx(b, rel=1e-3, abs=1e-6), (k, a, b)
        assert sg.centroid == pytest.approx(sc.centroid, rel=1e-3)


def test_dam_break_small_one_step(cuda_lib):
    g, c = both(scenes.dam_break, grid_res=128, column=64)
    g.step()
    c.step()
    assert g.last_substeps() == c.last_substeps()
    stats = compare_particles(g.particles(), c.particles())
    print("dam break 1 step", stats)


def test_granular_small_one_step(cuda_lib):
    g, c = both(scenes.mixed_granular, grid_res=256, target_particles=120_000)
    g.step()
    c.step()
    assert g.last_substeps() == c.last_substeps()
    pg, pc = g.particles(), c.particles()
    stats = compare_particles(pg, pc)
    # plastic state (Drucker-Prager q, NACC alpha, snow Jp/h)
    for k in ("friction_hardening", "log_volume_strain", "plastic_volume_ratio", "hardening_scale"):
        np.testing.assert_allclose(pg[k], pc[k], rtol=1e-4, atol=1e-5, err_msg=k)
    print("granular 1 step", stats)


def test_projection_recovers_guarded_fields(cuda_lib):
    """physics_correctness.rs:2237 NaN-injection recovery, GPU vs oracle."""
    def build(cls):
        cfg = SimConfig.standard(32, 0.02, (0.0, 0.0))
        sp = SpawnRegion.for_sim(cfg)
        sp.spacing, sp.box_size, sp.box_center = 0.5, (4, 4), (16.0, 16.0)
        sim = cls.new(cfg, sp).with_default_material(NeoHookeanMaterial.new(100.0, 200.0))
        p = sim.particles()
        nan = np.float32(np.nan)
        p["x"][0] = nan
        p["x"][1] = 1.0e9
        p["v"][2] = nan
        p["c"][3][:2] = nan
        p["f"][4][:2] = nan
        p["f"][5] = 0.0
        p["f"][6] = (1.0e6, 0.0, 0.0, 1.0e6)
        p["plastic_volume_ratio"][7] = -1.0
        p["hardening_scale"][8] = nan
        p["friction_hardening"][9] = nan
        p["log_volume_strain"][9] = nan
        p["mass"][10] = -1.0
        p["volume"][11] = 0.0
        p["initial_volume"][12] = nan
        p["density"][13] = -1.0
        sim.set_particles(p)
        return sim
    g, c = build(Simulation), build(OracleSimulation)
    g.step()
    c.step()
    pg, pc = g.particles(), c.particles()
    for k in ("x", "v", "c", "f", "mass", "initial_volume", "volume", "density",
              "plastic_volume_ratio", "hardening_scale", "friction_hardening", "log_volume_strain"):
        assert np.isfinite(pg[k]).all(), k
    compare_particles(pg, pc)
    assert g.last_counters()[1] == c.last_counters()[1]


def test_sort_preserves_results(cuda_lib):
    """Sorting permutes device storage only: reference-order readback is unchanged and a
    step after a sort agrees with the oracle."""
    g, c = both(scenes.quickstart)
    before = g.particles()
    g.sort_now(0)
    np.testing.assert_array_equal(before, g.particles())
    g.sort_now(1)
    np.testing.assert_array_equal(before, g.particles())
    g.step()
    c.step()
    compare_particles(g.particles(), c.particles())
