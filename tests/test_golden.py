"""Golden fixtures (tests/golden/, generated by tests/golden/make_golden.py from the oracle):
the oracle reproduces them exactly; on a GPU the reference-order mode reproduces them to the
parity bar."""
import json
import os

import numpy as np
import pytest

from emerge_engine_b200.abi import PARTICLE_DTYPE
from oracle.oracle import OracleSimulation
from tests import scenes

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    raw = np.load(os.path.join(HERE, name))["particles"]
    return raw.view(PARTICLE_DTYPE)


def test_oracle_reproduces_quickstart_fixtures():
    sim = scenes.quickstart(OracleSimulation)
    sim.step()
    np.testing.assert_array_equal(sim.particles(), load("quickstart_step1.npz"))
    sim.step_n(59)
    np.testing.assert_array_equal(sim.particles(), load("quickstart_step60.npz"))


def test_oracle_reproduces_dam_break_fixture():
    sim = scenes.dam_break(OracleSimulation, grid_res=128, column=64)
    sim.step()
    np.testing.assert_array_equal(sim.particles()[::16], load("dam_break_128_step1.npz"))


@pytest.mark.gpu
def test_reference_order_device_matches_fixtures(cuda_lib):
    from emerge_engine_b200 import DeterministicSimulation
    sim = scenes.quickstart(DeterministicSimulation)
    sim.step()
    g = sim.particles()
    ref = load("quickstart_step1.npz")
    for k in ("x", "v", "c", "f", "volume", "density"):
        np.testing.assert_array_equal(g[k], ref[k], err_msg=k)
    sim = scenes.dam_break(DeterministicSimulation, grid_res=128, column=64)
    sim.step()
    g, ref = sim.particles()[::16], load("dam_break_128_step1.npz")
    np.testing.assert_array_equal(g["x"], ref["x"])
    np.testing.assert_allclose(g["v"], ref["v"], rtol=1e-5, atol=1e-6)


def test_oracle_reproduces_granular_substep_fixture():
    sim = scenes.mixed_granular(OracleSimulation, grid_res=256, target_particles=120_000, dt=1e-3)
    sim.step()
    assert sim.last_substeps() == 1
    np.testing.assert_array_equal(sim.particles()[::32], load("granular_256_substep1.npz"))


@pytest.mark.gpu
def test_granular_substep_fixture(cuda_lib):
    """One substep of DP / snow / NACC (return mappings included) in reference order."""
    from emerge_engine_b200 import DeterministicSimulation
    sim = scenes.mixed_granular(DeterministicSimulation, grid_res=256, target_particles=120_000,
                                dt=1e-3)
    sim.step()
    assert sim.last_substeps() == 1
    g, ref = sim.particles()[::32], load("granular_256_substep1.npz")
    np.testing.assert_array_equal(g["x"], ref["x"])
    for k in ("v", "c", "f", "volume", "density", "plastic_volume_ratio", "hardening_scale",
              "friction_hardening", "log_volume_strain"):
        np.testing.assert_allclose(g[k], ref[k], rtol=1e-5, atol=1e-6, err_msg=k)


@pytest.mark.gpu
def test_granular_region_fixture(cuda_lib):
    """A full frame (34 substeps) against the fixture.  Transcendentals in the return
    mappings differ in the last bit between hosts' libm builds (and from the device's
    correctly rounded precise path) in rare cases; 34 substeps of yield decisions amplify
    that, so the frame is judged at 5e-3 (the live-oracle parity test on the same host is
    the tight check)."""
    from emerge_engine_b200 import DeterministicSimulation
    with open(os.path.join(HERE, "granular_256_region.json")) as f:
        ref = json.load(f)
    sim = scenes.mixed_granular(DeterministicSimulation, grid_res=256, target_particles=120_000)
    sim.step()
    assert sim.last_substeps() == ref["center"]["substeps"]
    for key, r in ref.items():
        b = sim.region_state(r["center"], r["radius"])
        assert abs(b.count - r["count"]) <= max(2, 1e-3 * r["count"])
        for k in ("avg_volume_ratio", "max_volume_ratio", "avg_speed", "avg_det_f", "avg_density"):
            assert getattr(b, k) == pytest.approx(r[k], rel=5e-3, abs=1e-6), k
