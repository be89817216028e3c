"""Corotated, VonMises, Rankine, mu(I), Viscoelastic, GranularFluid and Bingham on the
device vs the CPU oracle (through the C ABI), on the material-zoo scenes: a pre-strained
block on the floor and a disk with random velocities, each scene one model.

The reference order mode evaluates exp/log/pow in double and rounds once; the C library's
f32 functions the reference calls differ from that in the last bit for a few percent of
arguments (logf near 1), and these scenes' return mappings amplify a last-bit difference
over a frame's substeps.  So the reference order mode is checked
  * against the oracle with correctly rounded math over one full frame: per particle
    1e-5 on x and v, and the models' state fields 1e-5;
  * against the oracle with the C library's math after one substep: per particle 1e-5.
The fast path: per particle after one substep (fast bars of test_gpu_parity), and mass,
momentum and region statistics after five frames.
"""
import numpy as np
import pytest

from emerge_engine_b200 import Batch, DeterministicSimulation, Simulation
from oracle.oracle import OracleSimulation, correctly_rounded_math
from tests import scenes
from tests.test_gpu_parity import compare_particles, tol

pytestmark = pytest.mark.gpu

KINDS = sorted(scenes.ZOO)
STATE = ("friction_hardening", "plastic_volume_ratio", "hardening_scale", "volume", "density")


def compare_state(pg, pc, rtol, loose=()):
    """State fields per particle; fields in `loose` get 2e-3 relative."""
    for k in STATE:
        np.testing.assert_allclose(pg[k], pc[k], rtol=2e-3 if k in loose else rtol, atol=1e-6,
                                   err_msg=k)
    # F per particle relative to its largest entry (off-diagonal entries can be ~0)
    df = np.abs(pg["f"].astype(np.float64) - pc["f"]).max(axis=1)
    scale = np.maximum(np.abs(pc["f"].astype(np.float64)).max(axis=1), 1e-6)
    assert (df / scale).max() <= rtol, ("f", float((df / scale).max()))


@pytest.mark.parametrize("kind", KINDS)
def test_zoo_one_frame_reference_order(cuda_lib, kind):
    g = scenes.material_zoo(DeterministicSimulation, kind)
    g.step()
    with correctly_rounded_math():
        c = scenes.material_zoo(OracleSimulation, kind)
        c.step()
    assert g.last_substeps() == c.last_substeps()
    pg, pc = g.particles(), c.particles()
    stats = compare_particles(pg, pc, **tol("reference_order"))
    compare_state(pg, pc, 1e-5)
    same = float(np.mean(np.all(pg["v"] == pc["v"], axis=1)))
    print(kind, "reference order 1 frame", g.last_substeps(), "substeps, bit-identical v",
          same, stats)


@pytest.mark.parametrize("kind", KINDS)
def test_zoo_one_substep_reference_order_libm(cuda_lib, kind):
    g = scenes.material_zoo(DeterministicSimulation, kind, dt=1e-3)
    c = scenes.material_zoo(OracleSimulation, kind, dt=1e-3)
    g.step()
    c.step()
    assert g.last_substeps() == c.last_substeps() == 1
    pg, pc = g.particles(), c.particles()
    stats = compare_particles(pg, pc, **tol("reference_order"))
    compare_state(pg, pc, 1e-5)
    print(kind, "reference order 1 substep (C library math)", stats)


@pytest.mark.parametrize("kind", KINDS)
def test_zoo_fast(cuda_lib, kind):
    # one substep: frame dt 1e-3 is below every zoo scene's CFL bound
    g = scenes.material_zoo(Simulation, kind, dt=1e-3)
    c = scenes.material_zoo(OracleSimulation, kind, dt=1e-3)
    g.step()
    c.step()
    assert g.last_substeps() == c.last_substeps() == 1
    pg, pc = g.particles(), c.particles()
    stats = compare_particles(pg, pc, **tol("fast"))
    # mu(I)'s rate root (-b + sqrt(b^2 - 4ac)) / 2a cancels when b^2 >> |4ac|, so the
    # fast path's other rounding of b^2 - 4ac and of the square root (FMA, approximate
    # sqrt) moves mu_i by up to ~1e-3 relative; the reference-order tests hold it to 1e-5
    compare_state(pg, pc, 1e-4, loose=("friction_hardening",) if kind == "mu_i" else ())
    print(kind, "fast 1 substep", stats)
    # five frames: the atomically ordered sums feed yield decisions, so judge invariants
    g, c = scenes.material_zoo(Simulation, kind), scenes.material_zoo(OracleSimulation, kind)
    g.step_n(5)
    c.step_n(5)
    pg, pc = g.particles(), c.particles()
    assert pg["mass"].sum(dtype=np.float64) == pc["mass"].sum(dtype=np.float64)
    m = pc["mass"].astype(np.float64)
    p_abs = (m * np.linalg.norm(pc["v"].astype(np.float64), axis=1)).sum()
    dp = (m[:, None] * pg["v"]).sum(0) - (m[:, None] * pc["v"]).sum(0)
    assert np.linalg.norm(dp) <= 1e-3 * p_abs
    res = g.config.grid_res
    for center, r in (((res / 2, res / 2), float(res)), ((30.0, 16.0), 14.0),
                      ((res * 0.62, res * 0.5), 14.0)):
        sg, sc = g.region_state(center, r), c.region_state(center, r)
        assert abs(sg.count - sc.count) <= max(2, 1e-2 * sc.count)
        for k in ("avg_volume_ratio", "avg_speed", "avg_det_f", "avg_density"):
            assert getattr(sg, k) == pytest.approx(getattr(sc, k), rel=1e-2, abs=1e-4), (k, center)


def test_zoo_batch_matches_single_scenes(cuda_lib):
    """All seven models in one batch (the all-models kernel instantiation)."""
    sources = [scenes.material_zoo(Simulation, k, grid_res=64 + 16 * i) for i, k in enumerate(KINDS)]
    start = [s.particles() for s in sources]
    batch = Batch(sources)
    singles = [scenes.material_zoo(Simulation, k, grid_res=64 + 16 * i) for i, k in enumerate(KINDS)]
    for s, p in zip(singles, start):
        s.set_particles(p)
    batch.step(2)
    for s in singles:
        s.step_n(2)
    last, _ = batch.substeps()
    for k, s in enumerate(singles):
        assert last[k] == s.last_substeps(), KINDS[k]
        pb, ps = batch.particles(k), s.particles()
        assert pb["mass"].sum(dtype=np.float64) == ps["mass"].sum(dtype=np.float64)
        g = s.config.grid_res
        rb, rs = batch.region_state(k, (g / 2, g / 2), g), s.region_state((g / 2, g / 2), g)
        assert rb.count == rs.count
        assert rb.avg_speed == pytest.approx(rs.avg_speed, rel=1e-2, abs=1e-4), KINDS[k]
        assert rb.avg_det_f == pytest.approx(rs.avg_det_f, rel=1e-3), KINDS[k]


def test_bingham_without_yield_stress_is_rejected(cuda_lib):
    from emerge_engine_b200 import BinghamFluidMaterial, SimConfig
    sim = Simulation.empty(SimConfig.standard(32, 0.05, (0.0, -1.0)))
    with pytest.raises(ValueError):
        sim.with_default_material(BinghamFluidMaterial.new(1000.0, 0.5, 1e4, 7.0, 0.0))
