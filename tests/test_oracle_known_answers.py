"""Pins the CPU oracle to the reference's own known-answer tests for this path.

The reference ships no golden trajectories; these are its unit and integration tests
restated against the oracle (each test names the reference test it ports).
"""
import ctypes
from ctypes import byref, c_float

import numpy as np
import pytest

from emerge_engine_b200 import (DruckerPragerMaterial, NaccMaterial, NeoHookeanMaterial,
                                NewtonianFluidMaterial, SimConfig, SlipBoundary, SpawnRegion,
                                StomakhinMaterial)
from emerge_engine_b200.abi import PARTICLE_DTYPE, Particle
from oracle.oracle import OracleSimulation, farr, lib, oracle_material

f32 = np.float32


def mat2(x_axis, y_axis):
    return [x_axis[0], x_axis[1], y_axis[0], y_axis[1]]


def mmul(a, b):  # column-major 2x2
    A = np.array([[a[0], a[2]], [a[1], a[3]]], dtype=np.float64)
    B = np.array([[b[0], b[2]], [b[1], b[3]]], dtype=np.float64)
    C = A @ B
    return [C[0, 0], C[1, 0], C[0, 1], C[1, 1]]


def det(m):
    return m[0] * m[3] - m[2] * m[1]


def svd(f):
    u, s, vt = (c_float * 4)(), (c_float * 2)(), (c_float * 4)()
    lib().oracle_svd2(farr(f), u, s, vt)
    return list(u), list(s), list(vt)


def particle(f=(1, 0, 0, 1), **kw):
    p = Particle()
    p.f[:] = f
    p.plastic_volume_ratio = 1.0
    p.hardening_scale = 1.0
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def kirchhoff(m, p):
    tau = (c_float * 4)()
    lib().oracle_kirchhoff(byref(oracle_material(m)), byref(p), tau)
    return list(tau)


def update(m, p, dt):
    lib().oracle_update_particle(byref(oracle_material(m)), byref(p), dt)
    return p


# ---------------------------------------------------------------- grid/kernel.rs:59-66
@pytest.mark.parametrize("d", [0.0, 0.1, 0.35, -0.2])
def test_quadratic_weights_sum_to_one(d):
    w = (c_float * 3)()
    lib().oracle_axis_weights(d, w)
    assert abs(sum(w) - 1.0) < 1e-5


# ---------------------------------------------------------------- materials/svd.rs:87-183
SVD_CASES = {
    "identity": mat2((1, 0), (0, 1)),
    "diagonal": mat2((3, 0), (0, 1.5)),
    "shear": mat2((1, 0.5), (0.5, 1)),
    "generic": mat2((1.2, 0.3), (-0.1, 0.9)),
    "rank_deficient": mat2((1, 2), (2, 4)),
    "negative_det": mat2((1, 0), (0, -1)),
    "near_identity": mat2((0.99, 0.01), (-0.01, 1.01)),
    "pure_rotation": mat2((np.cos(f32(0.7)), np.sin(f32(0.7))), (-np.sin(f32(0.7)), np.cos(f32(0.7)))),
}


@pytest.mark.parametrize("name", sorted(SVD_CASES))
def test_svd2_check(name):
    f = SVD_CASES[name]
    u, s, vt = svd(f)
    r = mmul(mmul(u, [s[0], 0, 0, s[1]]), vt)
    np.testing.assert_allclose(r, f, atol=1e-5)
    assert abs(det(u) - 1.0) < 1e-5
    assert abs(det(vt) - 1.0) < 1e-5
    assert s[0] >= 0.0
    assert s[0] >= abs(s[1]) - 1e-6
    utu = mmul([u[0], u[2], u[1], u[3]], u)
    assert abs(utu[0] - 1) < 1e-5 and abs(utu[3] - 1) < 1e-5 and abs(utu[1]) < 1e-5


def test_svd2_negative_det_uses_signed_sigma():
    u, s, vt = svd(mat2((1, 0), (0, -1)))
    assert abs(det(u) - 1.0) < 1e-5 and abs(det(vt) - 1.0) < 1e-5
    assert s[1] <= 0.0


# ---------------------------------------------------------------- sand.rs:365-449
def marginal_state(ratio, trace, phi_deg):
    phi = f32(phi_deg) * f32(f32(np.pi) / f32(180))
    dev_norm = f32(-trace) * f32(ratio) * np.sin(phi) / np.sqrt(f32(2))
    diff = dev_norm * np.sqrt(f32(2))
    e1, e2 = (trace + diff) * 0.5, (trace - diff) * 0.5
    return (float(np.exp(f32(e1))), float(np.exp(f32(e2))))


def test_dp_marginal_yield_25_vs_40_degrees():
    sand = DruckerPragerMaterial.new(2000.0, 3000.0)
    q_init = float(sand.friction_residual / sand.hardening_peak)
    ratio = float((sand.lambda_ + sand.mu) / sand.mu)

    def run(sig):
        p = particle(f=(sig[0], 0, 0, sig[1]), mass=1.0, initial_volume=1.0,
                     friction_hardening=q_init)
        update(sand, p, 1.0)
        return (p.f[0], p.f[3]), p.friction_hardening

    s_in = marginal_state(ratio, -0.01, 25.0)
    after, q_after = run(s_in)
    assert np.linalg.norm(np.subtract(after, s_in)) < 1e-6
    assert abs(q_after - q_init) < 1e-6
    s_out = marginal_state(ratio, -0.01, 40.0)
    after2, q_after2 = run(s_out)
    assert np.linalg.norm(np.subtract(after2, s_out)) > 1e-6
    assert q_after2 > q_init


# ---------------------------------------------------------------- snow.rs:214-316
def frob(m):
    return float(np.sqrt(sum(v * v for v in m)))


def test_snow_small_strain_matches_hooke():
    lam, mu = 1000.0, 800.0
    mat = StomakhinMaterial.new(lam, mu, 10.0, 0.025, 0.0075, 0.6, 20.0)
    delta = f32(1e-4)
    e = (1.0, 0.0, 0.0, -0.4)
    f = [1 + delta * e[0], delta * e[1], delta * e[2], 1 + delta * e[3]]
    tau = kirchhoff(mat, particle(f=f, mass=1.0, initial_volume=1.0))
    eps = [delta * v for v in e]
    tr = eps[0] + eps[3]
    pred = [lam * tr + 2 * mu * eps[0], 2 * mu * eps[1], 2 * mu * eps[2], lam * tr + 2 * mu * eps[3]]
    assert frob(np.subtract(tau, pred)) / frob(pred) < 1e-3


def test_snow_marginally_inside_compression_limit_unclamped():
    mat = StomakhinMaterial.new(1000.0, 800.0, 10.0, 0.025, 0.0075, 0.6, 20.0)
    sx = float(f32(1.0) - f32(0.99) * mat.compression_limit)
    p = update(mat, particle(f=(sx, 0, 0, 1), mass=1.0, initial_volume=1.0), 1.0)
    assert abs(p.f[0] - sx) < 1e-5
    assert p.plastic_volume_ratio == 1.0


def test_snow_beyond_compression_limit_clamps_exactly():
    mat = StomakhinMaterial.new(1000.0, 800.0, 10.0, 0.025, 0.0075, 0.6, 20.0)
    sx = float(f32(1.0) - f32(1.5) * mat.compression_limit)
    p = update(mat, particle(f=(sx, 0, 0, 1), mass=1.0, initial_volume=1.0), 1.0)
    expected = float(f32(1.0) - mat.compression_limit)
    assert abs(p.f[0] - expected) < 1e-5
    assert abs(p.plastic_volume_ratio - sx / expected) < 1e-5


# ---------------------------------------------------------------- nacc.rs:317-401
def nacc_project(mat, f, alpha):
    fo, ao = (c_float * 4)(), c_float()
    lib().oracle_nacc_project(byref(oracle_material(mat)), farr(f), alpha, fo, byref(ao))
    return list(fo), ao.value


def pressure_from_j(kappa, j):
    return -(kappa * 0.5 * (j - 1.0 / j)) * j


def test_nacc_compression_cap_projects_exactly_to_p0():
    mat = NaccMaterial.new(3000.0, 2000.0, 1.2, 0.0, 0.0)
    p0 = float(mat.kappa) * 1e-5
    j_trial = 0.5
    f = [np.sqrt(j_trial), 0, 0, np.sqrt(j_trial)]
    assert pressure_from_j(float(mat.kappa), j_trial) > p0
    fa, _ = nacc_project(mat, f, 0.0)
    assert abs(pressure_from_j(float(mat.kappa), det(fa)) - p0) < 1e-2


def test_nacc_small_elastic_strain_not_projected():
    mat = NaccMaterial.new(3000.0, 2000.0, 1.2, 0.0, 2.0)
    f = [0.99895, 0, 0, 0.99905]
    fa, aa = nacc_project(mat, f, -1.0)
    assert np.linalg.norm(np.subtract(fa, np.array(f, dtype=np.float32))) < 1e-6 * 2
    assert aa == -1.0


# ---------------------------------------------------------------- elastic_tests.rs:66-132
@pytest.mark.parametrize("lam,mu,e", [(1000.0, 800.0, (1, 0, 0, 0)), (500.0, 1200.0, (0, 1, 1, 0))])
def test_neohookean_small_strain_matches_hooke(lam, mu, e):
    mat = NeoHookeanMaterial.new(lam, mu)
    delta = f32(1e-4)
    f = [1 + delta * e[0], delta * e[1], delta * e[2], 1 + delta * e[3]]
    tau = kirchhoff(mat, particle(f=f, mass=1.0, initial_volume=1.0))
    eps = [delta * v for v in e]
    tr = eps[0] + eps[3]
    pred = [lam * tr + 2 * mu * eps[0], 2 * mu * eps[1], 2 * mu * eps[2], lam * tr + 2 * mu * eps[3]]
    assert frob(np.subtract(tau, pred)) / frob(pred) < 1e-3


# ---------------------------------------------------------------- boundary/mod.rs:122-152
def slip(t, idx, res, v):
    arr = farr(v)
    lib().oracle_slip_velocity(t, idx, res, arr)
    return list(arr)


def test_slip_wall_preserves_tangential_velocity_exactly():
    v = slip(2, 32, 64, (-3.0, 7.5))
    assert v[1] == 7.5 and v[0] >= 0.0


def test_slip_wall_does_not_touch_outward_velocity():
    assert slip(2, 32, 64, (4.0, -2.0)) == [4.0, -2.0]


# ---------------------------------------------------------------- config.rs:508-571
def test_spawn_fit_rules():
    c = SimConfig.standard(64, 0.05, (0.0, -1.0))
    r = SpawnRegion.for_sim(c)
    r.spacing, r.box_size, r.box_center = 0.5, (6, 6), (32.0, 32.0)
    assert r.fits_in_sim(c)
    r.box_center = (59.5, 19.8)
    assert not r.fits_in_sim(c)
    edge = 64 - 2 - 3.0
    r.box_center = (edge, edge)
    assert r.fits_in_sim(c)
    sim = OracleSimulation.empty(c)
    r.box_center = (59.5, 19.8)
    with pytest.raises(ValueError):
        sim.add_body(r)


# ---------------------------------------------------------------- physics_correctness.rs
def zero_gravity(res):
    c = SimConfig(grid_res=res, dt=0.05, gravity=(0.0, 0.0))
    return c


def center_spawn(res, side):
    return SpawnRegion(spacing=0.5, box_size=(side, side), box_center=(res * 0.5, res * 0.5))


@pytest.mark.parametrize("material", [
    NeoHookeanMaterial.new(10.0, 20.0),
    StomakhinMaterial.from_young_modulus(1.4e5, 0.2),
])
def test_mass_is_conserved(material):  # :91-162
    sim = OracleSimulation.new(zero_gravity(32), center_spawn(32, 6)).with_default_material(material)
    m0 = sim.particles()["mass"].sum(dtype=np.float32)
    sim.step_n(100)
    assert abs(sim.particles()["mass"].sum(dtype=np.float32) - m0) < 1e-6


def test_mass_is_conserved_fluid():
    c = zero_gravity(32)
    c.recompute_density_each_step = True
    sim = OracleSimulation.new(c, center_spawn(32, 6)).with_default_material(
        NewtonianFluidMaterial.new(4.0, 0.1, 10.0, 4.0))
    m0 = sim.particles()["mass"].sum(dtype=np.float32)
    sim.step_n(100)
    assert abs(sim.particles()["mass"].sum(dtype=np.float32) - m0) < 1e-6


def test_zero_velocity_spawn_has_near_zero_momentum():  # :166-182
    sim = OracleSimulation.new(zero_gravity(32), center_spawn(32, 8)).with_default_material(
        NeoHookeanMaterial.new(20.0, 40.0))
    p = sim.particles()
    p0 = (p["mass"][:, None] * p["v"]).sum(0)
    sim.step_n(50)
    p = sim.particles()
    p1 = (p["mass"][:, None] * p["v"]).sum(0)
    assert np.linalg.norm(p1 - p0) / len(p) < 1e-3


def test_gravity_grows_momentum_linearly():  # :185-218
    c = SimConfig(gravity=(0.0, -9.81), dt=0.01, adaptive_timestep=False)
    sim = OracleSimulation.new(c, center_spawn(64, 4)).with_default_material(
        NeoHookeanMaterial.new(100.0, 200.0))
    p = sim.particles()
    m = p["mass"].sum()
    pb = (p["mass"][:, None] * p["v"]).sum(0)
    sim.step_n(10)
    p = sim.particles()
    pa = (p["mass"][:, None] * p["v"]).sum(0)
    expected = np.array([0.0, -9.81]) * m * 0.1
    assert np.linalg.norm((pa - pb) - expected) / np.linalg.norm(expected) < 0.05


@pytest.mark.parametrize("material", [
    NeoHookeanMaterial.new(10.0, 20.0),
    DruckerPragerMaterial.cohesionless(1e5, 0.2),
    StomakhinMaterial.from_young_modulus(1.4e5, 0.2),
    NaccMaterial.soft_clay(5e4, 0.3),
])
def test_j_stays_positive(material):  # :221-280
    c = SimConfig.standard(64, 0.05, (0.0, -9.81))
    sim = OracleSimulation.new(c, center_spawn(64, 8)).with_default_material(material)
    sim.step_n(60)
    f = sim.particles()["f"]
    j = f[:, 0] * f[:, 3] - f[:, 2] * f[:, 1]
    assert j.min() > 0.0


def test_region_state_returns_subset_in_radius():  # solver.rs:1391-1416
    c = SimConfig.standard(32, 0.05, (0.0, -1.0))
    sim = OracleSimulation.new(c, center_spawn(32, 8)).with_default_material(
        NeoHookeanMaterial.new(10.0, 20.0))
    small = sim.region_state((16.0, 16.0), 2.0)
    large = sim.region_state((16.0, 16.0), 100.0)
    assert small.count > 0 and large.count >= small.count
    assert large.count == sim.particle_count()


def test_project_invalid_state_recovers_every_guarded_field():  # physics_correctness.rs:2237
    c = SimConfig.standard(32, 0.02, (0.0, 0.0))
    sp = SpawnRegion(spacing=0.5, box_size=(4, 4), box_center=(16.0, 16.0))
    sim = OracleSimulation.new(c, sp).with_default_material(NeoHookeanMaterial.new(100.0, 200.0))
    p = sim.particles()
    assert len(p) >= 14
    nan = np.float32(np.nan)
    p["x"][0] = nan
    p["x"][1] = 1e9
    p["v"][2] = nan
    p["c"][3][:2] = nan
    p["f"][4][:2] = nan
    p["f"][5] = 0.0
    p["f"][6] = (1e6, 0, 0, 1e6)
    p["plastic_volume_ratio"][7] = -1.0
    p["hardening_scale"][8] = nan
    p["friction_hardening"][9] = nan
    p["log_volume_strain"][9] = nan
    p["mass"][10] = -1.0
    p["volume"][11] = 0.0
    p["initial_volume"][12] = nan
    p["density"][13] = -1.0
    sim.set_particles(p)
    sim.step()
    q = sim.particles()
    for k in ("x", "v", "c", "f", "mass", "initial_volume", "volume", "density",
              "plastic_volume_ratio", "hardening_scale", "friction_hardening",
              "log_volume_strain"):
        assert np.isfinite(q[k]).all(), k
    assert (q["mass"] > 0).all() and (q["volume"] > 0).all() and (q["density"] > 0).all()
    j = q["f"][:, 0] * q["f"][:, 3] - q["f"][:, 2] * q["f"][:, 1]
    assert (j > 0).all()


def test_block_index_key():  # particle_sort.wgsl:94-102
    L = lib()
    assert L.oracle_block_index(0.0, 0.0, 64) == 0
    assert L.oracle_block_index(63.9, 0.0, 64) == 15
    assert L.oracle_block_index(0.0, 63.9, 64) == 15 * 16
    assert L.oracle_block_index(-5.0, 100.0, 64) == 15 * 16
    assert L.oracle_block_index(8.0, 4.0, 100) == 1  # block size ceil(100/16) = 7
