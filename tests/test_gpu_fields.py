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
