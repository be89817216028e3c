"""Particle write-back (`particles_mut()` edits, lifecycle.rs:233) through the C ABI: the
upload is checked on the device, and pinned particles follow the uploaded flags (G2P zeroes
their velocity and affine matrix, transfer/g2p.rs).  Uploaded contact groups are covered by
test_gpu_contact."""
import numpy as np
import pytest

from emerge_engine_b200 import DeterministicSimulation, Simulation
from oracle.oracle import OracleSimulation
from tests import scenes

pytestmark = pytest.mark.gpu


def test_pinned_flags_follow_each_upload(cuda_lib):
    g = scenes.quickstart(DeterministicSimulation)
    c = scenes.quickstart(OracleSimulation)
    p = g.particles()
    p["pinned"][::7] = 1
    g.set_particles(p)
    c.set_particles(p)
    g.step()
    c.step()
    pg, pc = g.particles(), c.particles()
    np.testing.assert_array_equal(pg["x"], pc["x"])
    np.testing.assert_array_equal(pg["v"], pc["v"])
    assert not pg["v"][::7].any() and not pg["c"][::7].any()
    assert pg["v"].any()
    # an upload without pinned particles switches the pinned path off again
    q = pg.copy()
    q["pinned"][:] = 0
    g.set_particles(q)
    c.set_particles(q)
    g.step()
    c.step()
    pg, pc = g.particles(), c.particles()
    np.testing.assert_array_equal(pg["x"], pc["x"])
    np.testing.assert_array_equal(pg["v"], pc["v"])
    assert pg["v"][::7].any()


def test_repeated_uploads_in_the_fast_path(cuda_lib):
    """Upload, step, read back in a loop (the end-to-end pattern) keeps agreeing with the
    same loop on the oracle within the fast path's bar."""
    g = scenes.dam_break(Simulation, grid_res=128, column=64)
    c = scenes.dam_break(OracleSimulation, grid_res=128, column=64)
    host = g.particles()
    for _ in range(3):
        g.set_particles(host)
        c.set_particles(host)
        g.step()
        c.step()
        host = g.particles()
        pc = c.particles()
        dx = np.abs(host["x"].astype(np.float64) - pc["x"]).max()
        assert dx <= 1e-3, dx
        assert g.last_substeps() == c.last_substeps()
