"""CUDA step vs the CPU oracle on the same seeded scenes (through the C ABI).

Two device modes are checked:
  * reference order (`DeterministicSimulation`): every grid cell sums its contributions in
    the reference's particle index order, so device and oracle differ only by the last-ulp
    behaviour of expf/logf/sinf/powf.  Bar: per-particle relative error <= 1e-5 on x and v
    after one step (v judged against max(|v_ref|, 1e-2 * max|v_ref|) so particles at rest
    are measured on the scene's velocity scale).
  * fast (`Simulation`): P2G adds contributions with float reductions in L2, so the per-cell
    summation order changes from run to run.  Where stress impulses cancel, the resulting
    velocity is ill-conditioned; the bar is x <= 1e-5 per particle, v <= 1e-4 at the 99th
    percentile and <= 5e-3 at the maximum (same floor), total momentum within 1e-6 of the
    total absolute momentum, total mass exact.  Where one frame is tens of substeps of
    plastic yield decisions (granular scene), the per-particle bar applies to one substep and
    the frame is judged on invariants and region statistics.
region_state statistics after many steps: 1e-3 relative in both modes.
"""
import numpy as np
import pytest

from emerge_engine_b200 import (DeterministicSimulation, NeoHookeanMaterial, SimConfig,
                                Simulation, SpawnRegion)
from oracle.oracle import OracleSimulation
from tests import scenes

pytestmark = pytest.mark.gpu

class PairsSimulation(Simulation):
    """The fast path with lane-pair / quad aggregation of the P2G reductions
    (EMERGE_OPT_P2G_AGGREGATE = 2)."""

    def __init__(self, *a, **kw):
        super().__init__(*a, **kw)
        from emerge_engine_b200.abi import OPT_P2G_AGGREGATE
        self.set_option(OPT_P2G_AGGREGATE, 2)


MODES = {
    "reference_order": dict(cls=DeterministicSimulation, x_tol=1e-5, v_tol=1e-5, v_p99=1e-5),
    "fast": dict(cls=Simulation, x_tol=1e-5, v_tol=5e-3, v_p99=1e-4),
    "fast_pairs": dict(cls=PairsSimulation, x_tol=1e-5, v_tol=5e-3, v_p99=1e-4),
}


def compare_particles(pg, pc, x_tol, v_tol, v_p99):
    assert len(pg) == len(pc)
    dx = np.linalg.norm(pg["x"].astype(np.float64) - pc["x"], axis=1)
    x_rel = dx / np.maximum(np.linalg.norm(pc["x"], axis=1), 1.0)
    vn = np.linalg.norm(pc["v"].astype(np.float64), axis=1)
    floor = max(1e-2 * vn.max(), 1e-12)
    dv = np.linalg.norm(pg["v"].astype(np.float64) - pc["v"], axis=1)
    v_rel = dv / np.maximum(vn, floor)
    m = pc["mass"].astype(np.float64)
    p_g = (m[:, None] * pg["v"]).sum(0)
    p_c = (m[:, None] * pc["v"]).sum(0)
    p_abs = (m * vn).sum()
    stats = dict(x_rel_max=float(x_rel.max()), v_rel_max=float(v_rel.max()),
                 v_rel_p99=float(np.quantile(v_rel, 0.99)),
                 momentum_rel=float(np.linalg.norm(p_g - p_c) / max(p_abs, 1e-30)))
    assert pg["mass"].sum(dtype=np.float64) == pc["mass"].sum(dtype=np.float64)
    assert x_rel.max() <= x_tol, stats
    assert np.quantile(v_rel, 0.99) <= v_p99, stats
    assert v_rel.max() <= v_tol, stats
    assert stats["momentum_rel"] <= 1e-6, stats
    return stats


def both(mode, builder, *args, **kw):
    return builder(MODES[mode]["cls"], *args, **kw), builder(OracleSimulation, *args, **kw)


def tol(mode):
    t = MODES[mode]
    return dict(x_tol=t["x_tol"], v_tol=t["v_tol"], v_p99=t["v_p99"])


@pytest.mark.parametrize("mode", sorted(MODES))
def test_spawn_state_matches(cuda_lib, mode):
    g, c = both(mode, scenes.quickstart)
    pg, pc = g.particles(), c.particles()
    # spawn lattice, tags and init_particle are exact host-side work
    np.testing.assert_array_equal(pg["x"], pc["x"])
    np.testing.assert_array_equal(pg["user_tag"], pc["user_tag"])
    np.testing.assert_array_equal(pg["material_id"], pc["material_id"])
    # add_body's local volume estimate ran on the device
    rtol = 0 if mode == "reference_order" else 1e-6
    for k in ("initial_volume", "volume", "density"):
        np.testing.assert_allclose(pg[k], pc[k], rtol=rtol, atol=0, err_msg=k)


@pytest.mark.parametrize("mode", sorted(MODES))
def test_quickstart_one_step(cuda_lib, mode):
    g, c = both(mode, scenes.quickstart)
    g.step()
    c.step()
    assert g.last_substeps() == c.last_substeps()
    assert g.effective_dt() == pytest.approx(c.effective_dt(), rel=1e-6)
    print(mode, "quickstart 1 step", compare_particles(g.particles(), c.particles(), **tol(mode)))


@pytest.mark.parametrize("mode", sorted(MODES))
def test_quickstart_region_state_60_steps(cuda_lib, mode):
    g, c = both(mode, scenes.quickstart)
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


@pytest.mark.parametrize("mode", sorted(MODES))
def test_dam_break_small_one_step(cuda_lib, mode):
    g, c = both(mode, scenes.dam_break, grid_res=128, column=64)
    g.step()
    c.step()
    assert g.last_substeps() == c.last_substeps()
    print(mode, "dam break 1 step", compare_particles(g.particles(), c.particles(), **tol(mode)))


def test_granular_small_one_step_reference_order(cuda_lib):
    """One frame (~35 substeps of DP / snow / NACC plasticity) in reference order."""
    g, c = both("reference_order", scenes.mixed_granular, grid_res=256, target_particles=120_000)
    g.step()
    c.step()
    assert g.last_substeps() == c.last_substeps()
    pg, pc = g.particles(), c.particles()
    stats = compare_particles(pg, pc, **tol("reference_order"))
    for k in ("friction_hardening", "log_volume_strain", "plastic_volume_ratio", "hardening_scale"):
        np.testing.assert_allclose(pg[k], pc[k], rtol=1e-5, atol=1e-6, err_msg=k)
    print("reference_order granular 1 step", stats)


def test_granular_small_fast(cuda_lib):
    """Fast path on the granular scene.  Per particle after one substep (frame dt =
    min_dt = 1e-3 < the CFL bound, so one step is one substep); after one full frame of
    ~35 substeps the atomic summation order is amplified by yield decisions, so the frame is
    judged on mass, momentum and region statistics."""
    def sub(cls):
        return scenes.mixed_granular(cls, grid_res=256, target_particles=120_000)
    g = scenes.mixed_granular(Simulation, grid_res=256, target_particles=120_000, dt=1e-3)
    c = scenes.mixed_granular(OracleSimulation, grid_res=256, target_particles=120_000, dt=1e-3)
    g.step()
    c.step()
    assert g.last_substeps() == c.last_substeps() == 1
    stats = compare_particles(g.particles(), c.particles(), **tol("fast"))
    print("fast granular 1 substep", stats)
    g, c = sub(Simulation), sub(OracleSimulation)
    g.step()
    c.step()
    assert g.last_substeps() == c.last_substeps()
    pg, pc = g.particles(), c.particles()
    assert pg["mass"].sum(dtype=np.float64) == pc["mass"].sum(dtype=np.float64)
    m = pc["mass"].astype(np.float64)
    p_g, p_c = (m[:, None] * pg["v"]).sum(0), (m[:, None] * pc["v"]).sum(0)
    p_abs = (m * np.linalg.norm(pc["v"].astype(np.float64), axis=1)).sum()
    assert np.linalg.norm(p_g - p_c) <= 1e-4 * p_abs
    for center, r in (((128.0, 128.0), 200.0), ((64.0, 64.0), 40.0), ((180.0, 90.0), 30.0)):
        sg, sc = g.region_state(center, r), c.region_state(center, r)
        assert abs(sg.count - sc.count) <= max(2, 1e-3 * sc.count)
        # 5e-3: one frame is ~35 substeps of yield decisions, each fed by atomically
        # reordered sums; the reference-order mode matches this frame bit for bit.
        for k in ("avg_volume_ratio", "avg_speed", "avg_det_f", "avg_density"):
            assert getattr(sg, k) == pytest.approx(getattr(sc, k), rel=5e-3, abs=1e-6), k


@pytest.mark.parametrize("mode", sorted(MODES))
def test_projection_recovers_guarded_fields(cuda_lib, mode):
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
    g, c = build(MODES[mode]["cls"]), build(OracleSimulation)
    g.step()
    c.step()
    pg, pc = g.particles(), c.particles()
    for k in ("x", "v", "c", "f", "mass", "initial_volume", "volume", "density",
              "plastic_volume_ratio", "hardening_scale", "friction_hardening", "log_volume_strain"):
        assert np.isfinite(pg[k]).all(), k
        np.testing.assert_allclose(pg[k], pc[k], rtol=1e-5, atol=1e-6, err_msg=k)
    compare_particles(pg, pc, **tol(mode))
    assert g.last_counters()[1] == c.last_counters()[1]


def test_sort_preserves_results(cuda_lib):
    """Sorting permutes device storage only: reference-order readback is unchanged and a
    step after a sort agrees with the oracle."""
    g, c = both("reference_order", scenes.quickstart)
    before = g.particles()
    g.sort_now(0)
    np.testing.assert_array_equal(before, g.particles())
    g.sort_now(1)
    np.testing.assert_array_equal(before, g.particles())
    g.step()
    c.step()
    compare_particles(g.particles(), c.particles(), **tol("reference_order"))


def test_reference_order_is_run_to_run_deterministic(cuda_lib):
    a = scenes.dam_break(DeterministicSimulation, grid_res=128, column=64)
    b = scenes.dam_break(DeterministicSimulation, grid_res=128, column=64)
    a.step_n(3)
    b.step_n(3)
    np.testing.assert_array_equal(a.particles(), b.particles())


def test_graph_and_host_loop_agree(cuda_lib):
    """The device-side substep loop (CUDA graph while node) and the host-driven loop run
    the same kernels; results agree to float-reduction order."""
    from emerge_engine_b200.abi import OPT_USE_GRAPH
    a = scenes.dam_break(Simulation, grid_res=128, column=64)
    b = scenes.dam_break(Simulation, grid_res=128, column=64)
    b.set_option(OPT_USE_GRAPH, 0)
    a.step_n(3)
    b.step_n(3, timing=True)
    assert a.last_substeps() == b.last_substeps()
    compare_particles(a.particles(), b.particles(), **tol("fast"))
    assert b.last_timing["total_us"] > 0 and b.last_timing["g2p_us"] > 0
