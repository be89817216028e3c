"""Sleep partition on the device vs the CPU oracle (through the C ABI), on the sleep scene
(tests/scenes.py::sleep_scene: a resting block that falls asleep, a disk that wakes it,
an activated block that never sleeps).

Reference order: after every one of 12 frames the whole particle array in reference order
(x, v per particle at 1e-5, sleeping flags and the active count exactly) against the oracle
with correctly rounded math.  The particle-set edits (sleep_tag, wake_tag, add_body into a
sleeping scene, remove / retain / split) are compared the same way, edit by edit.  Fast
path: the partition invariant every frame and the active count and region statistics
against the oracle.
"""
import numpy as np
import pytest

from emerge_engine_b200 import DeterministicSimulation, Simulation, SpawnRegion
from oracle.oracle import OracleSimulation, correctly_rounded_math
from tests import scenes
from tests.test_gpu_parity import compare_particles, tol

pytestmark = pytest.mark.gpu


def zone_ok(sim):
    p, a = sim.particles(), sim.active_count()
    return bool(np.all(p["sleeping"][:a] == 0) and np.all(p["sleeping"][a:] == 1))


def same(g, c, what):
    assert g.active_count() == c.active_count(), what
    pg, pc = g.particles(), c.particles()
    np.testing.assert_array_equal(pg["sleeping"], pc["sleeping"], err_msg=what)
    np.testing.assert_array_equal(pg["user_tag"], pc["user_tag"], err_msg=what)
    return compare_particles(pg, pc, **tol("reference_order"))


def test_sleep_wake_frames_reference_order(cuda_lib):
    g = scenes.sleep_scene(DeterministicSimulation)
    with correctly_rounded_math():
        c = scenes.sleep_scene(OracleSimulation)
        for k in range(12):
            g.step()
            c.step()
            assert g.last_substeps() == c.last_substeps()
            stats = same(g, c, f"frame {k}")
    p = g.particles()
    assert ((p["user_tag"] == 1) & (p["sleeping"] == 0)).sum() > 0  # the disk woke the block
    print("sleep scene 12 frames", g.active_count(), "active", stats)


def test_partition_edits_reference_order(cuda_lib):
    g = scenes.sleep_scene(DeterministicSimulation)
    with correctly_rounded_math():
        c = scenes.sleep_scene(OracleSimulation)
        for sim in (g, c):
            sim.step_n(8)
        same(g, c, "before edits")
        edits = [
            ("sleep_tag 3", lambda s: s.sleep_tag(3)),
            ("add_body", lambda s: s.add_body(SpawnRegion(spacing=0.5, box_size=(6, 6),
                                                          box_center=(70.0, 60.0)))),
            ("wake_tag 3", lambda s: s.wake_tag(3)),
            ("remove tag 2", lambda s: s.remove_particles(lambda q: q.user_tag == 2)),
            ("split", lambda s: s.split_particles(lambda q: q.x[0] > 60.0, 0.1)),
            ("retain", lambda s: s.retain_particles(lambda q: q.x[1] < 40.0)),
        ]
        for name, edit in edits:
            edit(g)
            edit(c)
            same(g, c, name)
            g.step_n(2)
            c.step_n(2)
            same(g, c, name + " + 2 frames")


def test_sleep_fast_path(cuda_lib):
    g = scenes.sleep_scene(Simulation)
    c = scenes.sleep_scene(OracleSimulation)
    for k in range(12):
        g.step()
        c.step()
        assert zone_ok(g), k
        # a sleep decision at the threshold can differ by the fast path's rounding
        assert abs(g.active_count() - c.active_count()) <= max(2, c.active_count() // 200), k
    for center, r in (((48.0, 48.0), 96.0), ((56.0, 8.0), 12.0)):
        sg, sc = g.region_state(center, r), c.region_state(center, r)
        assert abs(sg.count - sc.count) <= max(2, sc.count // 200)
        for key in ("avg_speed", "avg_det_f", "avg_density"):
            assert getattr(sg, key) == pytest.approx(getattr(sc, key), rel=1e-2, abs=1e-4), key
