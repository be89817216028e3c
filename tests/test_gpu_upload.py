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


def test_async_readback_returns_the_state_it_was_queued_after(cuda_lib):
    """emerge_cuda_read_particles_async copies the state left by the work queued before it:
    a step queued after it does not leak into the copy, and the copy equals a synchronous
    read of the same state bit for bit (also with an upload and a readback in flight at
    once, the end-to-end loop's pattern)."""
    from emerge_engine_b200.simulation import PinnedBuffer
    g = scenes.dam_break(Simulation, grid_res=128, column=64)
    g.step()
    n = g.particle_count()
    state_k = g.particles()
    bufs = [PinnedBuffer(n * 128), PinnedBuffer(n * 128)]
    try:
        g.read_particles_raw_async(bufs[0].ptr, n)
        g.step()
        g.read_particles_raw_async(bufs[1].ptr, n)
        g.set_particles(state_k)  # upload while the second readback may still be copying
        g.synchronize()
        np.testing.assert_array_equal(bufs[0].as_particles(n), state_k)
        state_k1 = bufs[1].as_particles(n).copy()
        assert not np.array_equal(state_k1["x"], state_k["x"])
        np.testing.assert_array_equal(g.particles(), state_k)
    finally:
        for b in bufs:
            b.free()


@pytest.mark.parametrize("scene", ["quickstart", "dam_break"])
def test_async_readback_into_pinned_and_pageable_memory(cuda_lib, scene):
    """Two readbacks in flight at once, one into pinned and one into pageable memory: both
    give particles() bit for bit (240 particles, and 60,001 particles of a dam break)."""
    from emerge_engine_b200.abi import PARTICLE_DTYPE
    from emerge_engine_b200.simulation import PinnedBuffer
    g = scenes.quickstart(Simulation) if scene == "quickstart" else scenes.dam_break(
        Simulation, grid_res=512, column=128)
    if scene == "dam_break":
        p = g.particles()
        g._replace(p[:60_001], min(g.active_count(), 60_001))
    g.step()
    n = g.particle_count()
    want = g.particles()
    pinned = PinnedBuffer(n * 128)
    pageable = np.zeros(n, dtype=PARTICLE_DTYPE)
    try:
        g.read_particles_raw_async(pinned.ptr, n)
        g.read_particles_raw_async(pageable.ctypes.data, n)
        g.synchronize()
        np.testing.assert_array_equal(pinned.as_particles(n), want)
        np.testing.assert_array_equal(pageable, want)
    finally:
        pinned.free()

