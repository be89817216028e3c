"""Multi-field contact and two-phase mixture coupling on the device vs the CPU oracle
(through the C ABI).

Scenes (tests/scenes.py): contact_scene, a grip block (contact_group 1) thrown onto a slab,
with SimConfig.contact_friction or a DirectionalContactGrip; mixture_scene, water (fluid
phase) resting on sand (solid phase) with mixture drag, with and without the Jacobi pressure
projection.

Reference order: after every frame the whole particle array against the oracle with
correctly rounded math, bit for bit (x and v identical every frame); the contact scene is
followed for 20 frames (contact starts after about 8), the mixture scene for 4 (its
resolved phase velocities carry no boundary conditions in the reference, so the scene is
not meant to run long).  Simulation (the default class) runs the fused pipeline (field sums
reduced with the total, point clouds from per-base-cell lists): the same scenes within the
fast bar.
"""
import contextlib
import ctypes

import numpy as np
import pytest

from emerge_engine_b200 import Batch, DeterministicSimulation, DirectionalContactGrip, Simulation
from emerge_engine_b200.abi import ERR_INVALID_ARG
from oracle.oracle import OracleSimulation, correctly_rounded_math
from tests import scenes
from tests.test_gpu_parity import compare_particles, tol

pytestmark = pytest.mark.gpu

GRIPS = {"friction": None, "grip": DirectionalContactGrip(0.1, 0.9, (1.0, 0.0))}


def run_frames(g, c, frames, mode="reference_order"):
    exact_until = None
    stats = None
    for k in range(frames):
        g.step()
        c.step()
        assert g.last_substeps() == c.last_substeps(), k
        pg, pc = g.particles(), c.particles()
        same = np.array_equal(pg["x"], pc["x"]) and np.array_equal(pg["v"], pc["v"])
        if not same and exact_until is None:
            exact_until = k
        stats = compare_particles(pg, pc, **tol(mode))
    return exact_until, stats


@pytest.mark.parametrize("which", sorted(GRIPS))
def test_contact_frames_reference_order(cuda_lib, which):
    grip = GRIPS[which]
    g = scenes.contact_scene(DeterministicSimulation, grip=grip)
    with correctly_rounded_math():
        c = scenes.contact_scene(OracleSimulation, grip=grip)
        exact_until, stats = run_frames(g, c, 20)
    assert exact_until is None, (exact_until, stats)


@pytest.mark.parametrize("iterations", [0, 2])
def test_mixture_frames_reference_order(cuda_lib, iterations):
    g = scenes.mixture_scene(DeterministicSimulation, iterations=iterations)
    with correctly_rounded_math():
        c = scenes.mixture_scene(OracleSimulation, iterations=iterations)
        exact_until, stats = run_frames(g, c, 4)
    assert exact_until is None, (exact_until, stats)


def run_frames_fast(g, c, frames, strict):
    """The fast bar per particle for the first `strict` frames; after them the contact
    decisions (directional friction, overlap correction) may differ with the summation
    order, and the frames are judged on mass, momentum and region statistics."""
    for k in range(frames):
        g.step()
        c.step()
        assert g.last_substeps() == c.last_substeps(), k
        pg, pc = g.particles(), c.particles()
        if k < strict:
            compare_particles(pg, pc, **tol("fast"))
            continue
        assert pg["mass"].sum(dtype=np.float64) == pc["mass"].sum(dtype=np.float64)
        m = pc["mass"].astype(np.float64)
        p_abs = (m * np.linalg.norm(pc["v"].astype(np.float64), axis=1)).sum()
        dp = (m[:, None] * pg["v"]).sum(0) - (m[:, None] * pc["v"]).sum(0)
        assert np.linalg.norm(dp) <= 1e-4 * p_abs, k
    for center, r in (((48.0, 48.0), 96.0), ((42.0, 20.0), 12.0)):  # the 96-cell scene, its contact zone
        sg, sc = g.region_state(center, r), c.region_state(center, r)
        assert sg.count == sc.count
        for key in ("avg_speed", "avg_det_f", "avg_density"):
            assert getattr(sg, key) == pytest.approx(getattr(sc, key), rel=1e-3, abs=1e-6), key


@pytest.mark.parametrize("which", sorted(GRIPS))
def test_contact_fast_pipeline(cuda_lib, which):
    """Simulation (the default class) runs multi-field scenes on the fused pipeline: field
    sums reduced with the total, point clouds from per-base-cell lists."""
    g = scenes.contact_scene(Simulation, grip=GRIPS[which])
    c = scenes.contact_scene(OracleSimulation, grip=GRIPS[which])
    run_frames_fast(g, c, 12, strict=9)


@pytest.mark.parametrize("iterations", [0, 2])
def test_mixture_fast_pipeline(cuda_lib, iterations):
    g = scenes.mixture_scene(Simulation, iterations=iterations)
    c = scenes.mixture_scene(OracleSimulation, iterations=iterations)
    print("mixture, fast pipeline 3 frames", run_frames(g, c, 3, "fast"))


def combined_scene(sim_cls):
    """The contact scene with ASFLIP, a linear drag field and the sleep partition on."""
    from emerge_engine_b200 import LinearDragField
    sim = scenes.contact_scene(sim_cls, grip=GRIPS["grip"], asflip=0.3, sleep=0.02)
    sim.add_force_field(LinearDragField.new((0.5, 0.0), 0.05, LinearDragField.ALL_MATERIALS))
    return sim


def test_contact_with_fields_asflip_and_sleep(cuda_lib):
    """Contact together with the other extras: bit for bit in reference order.  On the fused
    pipeline (which steps it with the host-driven substep loop, as every scene with a sleep
    partition) ASFLIP's position gate, gamma = [trace B >= 0] (g2p.rs:291-296), is a sign
    decision on rounding noise for the rigidly translating block: with any other summation
    order a few dozen particles take the other branch from the first frame (about 3e-3 cells
    apart), and the sleep partition may differ by a particle or two (a particle asleep in one
    run moves on in the other), so the frames are judged on substep counts, the partition
    size, mass, momentum and displacement statistics instead of the per-particle bar."""
    g = combined_scene(DeterministicSimulation)
    with correctly_rounded_math():
        c = combined_scene(OracleSimulation)
        exact_until, stats = run_frames(g, c, 10)
    assert exact_until is None, (exact_until, stats)
    assert g.active_count() == c.active_count()
    g = combined_scene(Simulation)
    c = combined_scene(OracleSimulation)
    for k in range(8):
        g.step()
        c.step()
        assert g.last_substeps() == c.last_substeps(), k
        assert abs(g.active_count() - c.active_count()) <= 2, k
    pg, pc = g.particles(), c.particles()
    assert pg["mass"].sum(dtype=np.float64) == pc["mass"].sum(dtype=np.float64)
    m = pc["mass"].astype(np.float64)
    p_abs = (m * np.linalg.norm(pc["v"].astype(np.float64), axis=1)).sum()
    dp = np.linalg.norm((m[:, None] * pg["v"]).sum(0) - (m[:, None] * pc["v"]).sum(0))
    dx = np.linalg.norm(pg["x"].astype(np.float64) - pc["x"], axis=1)
    far = int((dx > 0.25).sum())
    print("combined scene, fused pipeline: |dp| / sum |p| %.2e, dx p99 %.2e cells, %d particles "
          "over 0.25 cells (max %.2e)" % (dp / p_abs, np.percentile(dx, 99), far, dx.max()))
    assert dp <= 1e-3 * p_abs
    assert np.percentile(dx, 99) <= 0.05
    # a particle that took the other sleep or contact branch (the partition may differ by two
    # particles per frame) is followed by its stencil neighbours, not by the whole block
    assert far <= 16


def test_contact_with_fields_and_sleep_per_particle(cuda_lib):
    """The combined scene without ASFLIP (whose position gate is the sign decision above), on
    the fused pipeline: every particle within the fast bar for 3 frames, with the same
    partition size as the oracle's, so a field-sum routing error cannot hide under the
    aggregate statistics."""
    from emerge_engine_b200 import LinearDragField

    def build(sim_cls):
        sim = scenes.contact_scene(sim_cls, grip=GRIPS["grip"], asflip=0.0, sleep=0.02)
        sim.add_force_field(LinearDragField.new((0.5, 0.0), 0.05, LinearDragField.ALL_MATERIALS))
        return sim

    g, c = build(Simulation), build(OracleSimulation)
    for k in range(3):
        g.step()
        c.step()
        assert g.last_substeps() == c.last_substeps(), k
        assert g.active_count() == c.active_count(), k
        compare_particles(g.particles(), c.particles(), **tol("fast"))


class _AggregatedSimulation(Simulation):
    """The fused pipeline with warp-aggregated P2G (EMERGE_OPT_P2G_AGGREGATE = 1): with one
    kind of field a warp whose lanes all target one array (the total, or one field's sums)
    aggregates, and a warp mixing field and non-field particles scatters lane by lane."""

    def __init__(self, *a, **kw):
        super().__init__(*a, **kw)
        from emerge_engine_b200.abi import OPT_P2G_AGGREGATE
        self.set_option(OPT_P2G_AGGREGATE, 1)


@pytest.mark.parametrize("scene", ["contact", "mixture"])
def test_aggregated_field_scatter(cuda_lib, scene):
    """Per-warp target selection on single-kind field scenes: the contact block lands on the
    slab (warps along the interface mix grip and slab particles), the water sits on the sand
    (warps along the interface mix the phases), against the oracle at the fast bar."""
    if scene == "contact":
        g, c = scenes.contact_scene(_AggregatedSimulation), scenes.contact_scene(OracleSimulation)
        frames = 10
    else:
        g, c = scenes.mixture_scene(_AggregatedSimulation), scenes.mixture_scene(OracleSimulation)
        frames = 3
    print(scene, "aggregated, fast pipeline", run_frames(g, c, frames, "fast"))


@pytest.mark.parametrize("mode", ["reference_order", "fast"])
def test_contact_groups_follow_each_upload(cuda_lib, mode):
    """A write-back that sets contact groups switches the contact fields on; one that clears
    them switches them off again (particles_mut() edits, lifecycle.rs:233)."""
    exact = mode == "reference_order"
    g = scenes.quickstart(DeterministicSimulation if exact else Simulation)
    with correctly_rounded_math() if exact else contextlib.nullcontext():
        c = scenes.quickstart(OracleSimulation)
        p = g.particles()
        p["contact_group"][p["x"][:, 1] > np.median(p["x"][:, 1])] = 2
        for sim in (g, c):
            sim.set_particles(p)
        first_inexact, _ = run_frames(g, c, 2, mode)
        assert first_inexact is None or not exact
        q = g.particles()
        q["contact_group"][:] = 0
        for sim in (g, c):
            sim.set_particles(q)
        first_inexact, _ = run_frames(g, c, 2, mode)
        assert first_inexact is None or not exact


def test_grip_and_phase_arguments_are_checked(cuda_lib):
    sim = scenes.contact_scene(Simulation)
    lib, h = sim._lib, sim._sim
    assert lib.emerge_cuda_set_contact_grip(h, 1, 1.5, 0.5, 1.0, 0.0) == ERR_INVALID_ARG
    assert lib.emerge_cuda_set_contact_grip(h, 1, 0.5, 0.5, float("nan"), 0.0) == ERR_INVALID_ARG
    bad = (ctypes.c_uint32 * 2)(0, 3)
    assert lib.emerge_cuda_set_mixture_phases(h, bad, 2) == ERR_INVALID_ARG
    with pytest.raises(Exception):
        Batch([scenes.contact_scene(Simulation)])  # multi-field scenes run as single simulations
    sim.set_contact_grip(None)
    sim.step()
    assert np.isfinite(sim.particles()["v"]).all()


@pytest.mark.parametrize("mode", ["reference_order", "fast"])
def test_single_field_scenes(cuda_lib, mode):
    """Contact with every particle in the grip field (no interface anywhere) and a mixture
    with one phase only (drag never engages): the resolves must fall back to the total
    velocity exactly as the reference's do."""
    exact = mode == "reference_order"
    cls = DeterministicSimulation if exact else Simulation

    def all_grip(sim_cls):
        sim = scenes.contact_scene(sim_cls)
        p = sim.particles()
        p["contact_group"][:] = 3
        sim.set_particles(p)
        return sim

    def one_phase(sim_cls):
        sim = scenes.mixture_scene(sim_cls)
        p = sim.particles()
        p["material_id"][:] = 0  # every particle in the solid phase
        sim.set_particles(p)
        return sim

    for build in (all_grip, one_phase):
        g = build(cls)
        with correctly_rounded_math() if exact else contextlib.nullcontext():
            c = build(OracleSimulation)
            first_inexact, _ = run_frames(g, c, 3, mode)
        assert first_inexact is None or not exact, build.__name__
