"""Pins the oracle's Corotated, VonMises, Rankine, mu(I), Viscoelastic, GranularFluid and
Bingham models to the reference's own unit tests for them (each test names the reference
test it restates), plus whole-scene invariants on the oracle.
"""
from ctypes import byref

import numpy as np
import pytest

from emerge_engine_b200 import (BinghamFluidMaterial, CorotatedMaterial, GranularFluidMaterial,
                                MuIRheologyMaterial, RankineMaterial, SimConfig, SpawnRegion,
                                ViscoelasticMaterial, VonMisesMaterial)
from oracle.oracle import OracleSimulation, lib, oracle_material
from tests import scenes
from tests.test_oracle_known_answers import frob, kirchhoff, particle, update

f32 = np.float32
SQRT_2 = f32(np.sqrt(2.0))


def hooke(lam, mu, eps):
    """lambda tr(eps) I + 2 mu eps, column-major 2x2."""
    tr = eps[0] + eps[3]
    return [lam * tr + 2 * mu * eps[0], 2 * mu * eps[1], 2 * mu * eps[2], lam * tr + 2 * mu * eps[3]]


def strained(delta, e):
    return [1 + delta * e[0], delta * e[1], delta * e[2], 1 + delta * e[3]]


def diag_step(mat, sigma, q, dt=1.0, init=False):
    """One update_particle from F = diag(sigma), zero velocity gradient."""
    p = particle(f=(sigma[0], 0, 0, sigma[1]), mass=1.0, initial_volume=1.0, friction_hardening=q)
    if init:
        lib().oracle_init_particle(byref(oracle_material(mat)), byref(p))
    update(mat, p, dt)
    return np.array([p.f[0], p.f[3]], dtype=np.float64), float(p.friction_hardening)


def hencky(sigma):
    return np.log(np.maximum(np.abs(np.asarray(sigma, dtype=np.float64)), 1e-10))


# ---------------------------------------------------------------- corotated.rs:183-249
@pytest.mark.parametrize("lam,mu,e", [(1000.0, 800.0, (1, 0, 0, 0)), (500.0, 1200.0, (0, 1, 1, 0))])
def test_corotated_small_strain_matches_hooke(lam, mu, e):
    delta = f32(1e-4)
    tau = kirchhoff(CorotatedMaterial.new(lam, mu), particle(f=strained(delta, e)))
    pred = hooke(lam, mu, [delta * v for v in e])
    assert frob(np.subtract(tau, pred)) / frob(pred) < 1e-3


def test_corotated_symmetric_f_has_identity_rotation():
    """For symmetric F the polar rotation is exactly I, so the stress is
    2 mu (F - I) F^T + lambda (J - 1) J I at any strain."""
    lam, mu = 1000.0, 800.0
    f = [1.3, -0.15, -0.15, 1.6]
    tau = kirchhoff(CorotatedMaterial.new(lam, mu), particle(f=f))
    F = np.array([[f[0], f[2]], [f[1], f[3]]], dtype=np.float64)
    j = np.linalg.det(F)
    ref = 2 * mu * (F - np.eye(2)) @ F.T + lam * (j - 1) * j * np.eye(2)
    np.testing.assert_allclose(tau, [ref[0, 0], ref[1, 0], ref[0, 1], ref[1, 1]], rtol=1e-5)


def test_corotated_hardening_and_thermal_scale_moduli():
    """mu and lambda scale by hardening_scale * (1 + thermal_expansion * T)."""
    f = strained(f32(1e-3), (1, 0.5, 0.5, -0.4))
    base = kirchhoff(CorotatedMaterial.new(1000.0, 800.0), particle(f=f))
    warm = CorotatedMaterial(1000.0, 800.0, thermal_expansion=0.1)
    tau = kirchhoff(warm, particle(f=f, hardening_scale=2.0, temperature=3.0))
    np.testing.assert_allclose(tau, np.multiply(base, 2.0 * 1.3), rtol=1e-5)


# ---------------------------------------------------------------- von_mises.rs:212-300
def test_von_mises_inside_yield_is_elastic():
    mat = VonMisesMaterial.new(2000.0, 3000.0, 100.0)
    d = f32(0.99 * mat.yield_stress / (2.0 * mat.mu)) / SQRT_2
    sigma = (np.exp(f32(d)), np.exp(f32(-d)))
    after, kappa = diag_step(mat, sigma, 0.0)
    assert np.linalg.norm(after - sigma) < 1e-4
    assert kappa == 0.0


def test_von_mises_beyond_yield_projects_to_the_surface():
    mat = VonMisesMaterial.new(2000.0, 3000.0, 100.0)
    d = f32(1.5 * mat.yield_stress / (2.0 * mat.mu)) / SQRT_2
    trace = 0.4
    sigma = (np.exp(f32(trace * 0.5 + d)), np.exp(f32(trace * 0.5 - d)))
    after, kappa = diag_step(mat, sigma, 0.0)
    eps = hencky(after)
    tr = eps.sum()
    dev = np.linalg.norm(eps - tr * 0.5)
    assert abs(dev - mat.yield_stress / (2.0 * mat.mu)) < 1e-4
    assert abs(tr - trace) < 1e-4  # volumetric strain preserved
    assert kappa > 0.0


def test_von_mises_hardening_shrinks_the_increment():
    mat = VonMisesMaterial.with_hardening(2000.0, 3000.0, 100.0, 500.0)
    d = f32(1.5 * mat.yield_stress / (2.0 * mat.mu)) / SQRT_2
    sigma = (np.exp(f32(d)), np.exp(f32(-d)))
    _, k0 = diag_step(mat, sigma, 0.0)
    _, k1 = diag_step(mat, sigma, 1.0)
    assert (k1 - 1.0) < (k0 - 0.0)
    with pytest.raises(ValueError):
        VonMisesMaterial.with_hardening(2000.0, 3000.0, 100.0, -1.0)


# ---------------------------------------------------------------- rankine.rs:271-370
def rankine_tau(mat, sigma):
    e = hencky(sigma)
    a = 2.0 * mat.mu + mat.lambda_
    return np.array([a * e[0] + mat.lambda_ * e[1], mat.lambda_ * e[0] + a * e[1]])


def test_rankine_inside_tensile_strength_is_elastic():
    mat = RankineMaterial.new(2000.0, 3000.0, 100.0, 1.0)
    ex = f32(0.99 * mat.tensile_strength) / f32(2.0 * mat.mu + mat.lambda_)
    sigma = (np.exp(ex), 1.0)
    after, damage = diag_step(mat, sigma, 0.0)
    assert np.linalg.norm(after - sigma) < 1e-4
    assert damage == 0.0


def test_rankine_uniaxial_tension_projects_to_the_cutoff():
    mat = RankineMaterial.new(2000.0, 3000.0, 100.0, 1.0)
    ex = f32(1.5 * mat.tensile_strength) / f32(2.0 * mat.mu + mat.lambda_)
    sigma = (np.exp(ex), 1.0)
    after, damage = diag_step(mat, sigma, 0.0)
    tau = rankine_tau(mat, after)
    assert abs(tau[0] - mat.tensile_strength) < 1e-3
    assert abs(tau[1] - mat.lambda_ * ex) < 1e-3  # the other principal stress is untouched
    assert damage > 0.0


def test_rankine_biaxial_tension_returns_to_the_corner():
    mat = RankineMaterial.new(2000.0, 3000.0, 100.0, 1.0)
    a = 2.0 * mat.mu + mat.lambda_
    e = f32(1.5 * mat.tensile_strength) / f32(a + mat.lambda_)
    after, damage = diag_step(mat, (np.exp(e), np.exp(e)), 0.0)
    tau = rankine_tau(mat, after)
    assert np.all(np.abs(tau - mat.tensile_strength) < 1e-3)
    assert damage > 0.0


def test_rankine_damage_saturates():
    """Damage stops at -ln(0.05) / softening_rate (utils.rs:43-49)."""
    mat = RankineMaterial.new(2000.0, 3000.0, 100.0, 1.0)
    ex = f32(50.0 * mat.tensile_strength) / f32(2.0 * mat.mu + mat.lambda_)
    _, damage = diag_step(mat, (np.exp(ex), 1.0), 2.99)
    assert damage == pytest.approx(-np.log(0.05), rel=1e-6)


# ---------------------------------------------------------------- sand_mui.rs:282-380
def test_mui_defaults_are_the_reference_angles():
    m = MuIRheologyMaterial.new(2000.0, 3000.0)
    assert m.mu_static == pytest.approx(np.tan(np.radians(20.9)), rel=1e-6)
    assert m.mu_dynamic == pytest.approx(np.tan(np.radians(32.8)), rel=1e-6)
    assert m.inertial_q == f32(5.58)


def test_mui_tension_projects_to_identity():
    mat = MuIRheologyMaterial.new(2000.0, 3000.0)
    after, mu_after = diag_step(mat, (1.05, 1.02), 0.0, dt=0.1, init=True)
    assert np.linalg.norm(after - 1.0) < 1e-5
    assert mu_after == mat.mu_static


def test_mui_inside_quasistatic_yield_does_not_flow():
    mat = MuIRheologyMaterial.new(2000.0, 3000.0)
    ex = f32(-0.01)
    p_trial = -(mat.lambda_ + mat.mu) * ex
    dev_needed = f32(0.99) * mat.mu_static * p_trial / (SQRT_2 * mat.mu)
    ey = ex - dev_needed * SQRT_2
    sigma = (np.exp(ex), np.exp(f32(ey)))
    after, mu_after = diag_step(mat, sigma, 0.0, dt=0.1, init=True)
    assert np.linalg.norm(after - sigma) < 1e-4
    assert mu_after == mat.mu_static


def test_mui_gamma_dot_solves_its_quadratic():
    mat = MuIRheologyMaterial.new(2000.0, 3000.0)
    dt = 0.1
    sigma = (np.exp(f32(-0.08)), np.exp(f32(0.02)))
    _, mu_i = diag_step(mat, sigma, 0.0, dt=dt, init=True)
    assert mu_i > mat.mu_static
    eps = hencky(sigma)
    tr = eps.sum()
    p_trial = -(mat.lambda_ + mat.mu) * tr
    dev_norm = np.linalg.norm(eps - tr * 0.5)
    dq = np.sqrt(2.0) * mat.mu * dev_norm - mat.mu_static * p_trial
    sp = np.sqrt(p_trial)
    a = mat.mu * dt
    b = p_trial * (mat.mu_dynamic - mat.mu_static) + a * mat.inertial_q * sp - dq
    c = -dq * mat.inertial_q * sp
    g = mat.inertial_q * sp / ((mat.mu_dynamic - mat.mu_static) / (mu_i - mat.mu_static) - 1.0)
    scale = max(abs(a * g * g), abs(b * g), abs(c))
    assert abs(a * g * g + b * g + c) / scale < 1e-3


# ---------------------------------------------------------------- viscoelastic.rs:220-310
def test_viscoelastic_small_strain_matches_hooke():
    lam, mu = 1000.0, 800.0
    delta = f32(1e-4)
    e = (1, 0, 0, -0.4)
    tau = kirchhoff(ViscoelasticMaterial.new(lam, mu, 50.0), particle(f=strained(delta, e)))
    pred = hooke(lam, mu, [delta * v for v in e])
    assert frob(np.subtract(tau, pred)) / frob(pred) < 1e-3


def test_viscoelastic_dashpot_is_eta_times_deviatoric_rate():
    eta, g = 50.0, 3.0
    tau = kirchhoff(ViscoelasticMaterial.new(1000.0, 800.0, eta), particle(c=(0, g, g, 0)))
    assert frob(np.subtract(tau, [0, eta * g, eta * g, 0])) < 1e-4


def test_viscoelastic_spring_and_dashpot_add():
    mat = ViscoelasticMaterial.new(1000.0, 800.0, 50.0)
    f = strained(f32(0.02), (1, 0, 0, -0.3))
    c = (0, 4.0, 4.0, 0)
    both = kirchhoff(mat, particle(f=f, c=c))
    spring = kirchhoff(mat, particle(f=f))
    dashpot = kirchhoff(mat, particle(c=c))
    assert frob(np.subtract(both, np.add(spring, dashpot))) < 1e-3


def test_viscoelastic_active_stress_is_isotropic():
    """transfer.rs:77-104: Viscoelastic's active stress is activation * coeff * I whatever
    the fibre direction; Corotated's follows F (n0 x n0) F^T."""
    f = [1.1, 0.0, 0.0, 1.0]
    ve = ViscoelasticMaterial.new(1000.0, 800.0, 0.0)
    ve.active_stress_coeff = f32(10.0)
    base = kirchhoff(ve, particle(f=f))
    act = kirchhoff(ve, particle(f=f, activation=0.5, activation_dir=(1.0, 0.0)))
    np.testing.assert_allclose(np.subtract(act, base), [5.0, 0, 0, 5.0], atol=1e-4)
    co = CorotatedMaterial(1000.0, 800.0, active_stress_coeff=10.0)
    base = kirchhoff(co, particle(f=f))
    act = kirchhoff(co, particle(f=f, activation=0.5, activation_dir=(1.0, 0.0)))
    np.testing.assert_allclose(np.subtract(act, base), [5.0 * 1.21, 0, 0, 0], atol=1e-3)


# ---------------------------------------------------------------- bingham.rs:261-320
def bingham_dev(mat, g):
    """Deviatoric stress alone: density at rest (zero Tait pressure), F = I."""
    return kirchhoff(mat, particle(c=(0, g, g, 0), density=float(mat.rest_density)))


def test_bingham_below_critical_rate_is_a_rigid_plug():
    mat = BinghamFluidMaterial.new(1000.0, 0.5, 5000.0, 7.0, 100.0)
    assert all(v == 0.0 for v in bingham_dev(mat, 1e-6))


def test_bingham_above_yield_matches_formula():
    mat = BinghamFluidMaterial.new(1000.0, 0.5, 5000.0, 7.0, 100.0)
    g = 5.0
    eta_app = mat.yield_stress / (2.0 * g) + mat.dynamic_viscosity
    assert frob(np.subtract(bingham_dev(mat, g), [0, g * eta_app, g * eta_app, 0])) < 1e-3


def test_bingham_shear_thins():
    mat = BinghamFluidMaterial.new(1000.0, 0.5, 5000.0, 7.0, 100.0)
    assert bingham_dev(mat, 10.0)[1] / 20.0 < bingham_dev(mat, 1.0)[1] / 2.0


def test_bingham_cuda_packing():
    """MaterialParams marks a Bingham fluid by compression_limit = yield_stress; fields
    params() cannot carry must keep the constructor's values on the CUDA backend."""
    mat = BinghamFluidMaterial.high_yield(1000.0, 1e4)
    p = mat.abi_params()
    assert p.model == 1 and p.compression_limit == 100.0 and p.dynamic_viscosity == f32(0.5)
    with pytest.raises(ValueError):
        BinghamFluidMaterial.new(1000.0, 0.5, 1e4, 7.0, 0.0).abi_params()
    odd = BinghamFluidMaterial.new(1000.0, 0.5, 1e4, 7.0, 10.0)
    odd.critical_shear_rate = f32(1e-3)
    with pytest.raises(ValueError):
        odd.abi_params()


# ---------------------------------------------------------------- granular_fluid.rs
def test_granular_fluid_rest_state_is_stress_free():
    mat = GranularFluidMaterial.saturated_loam(2e4, 0.3)
    assert frob(kirchhoff(mat, particle())) == 0.0


def test_granular_fluid_compression_clamps_and_hardens():
    """Singular values below 1 - compression_limit are clamped, the excess goes into
    plastic_volume_ratio, and hardening_scale = clamp(exp(xi (1 - Jp)), 0.1, 7)."""
    mat = GranularFluidMaterial.saturated_loam(2e4, 0.3)
    p = particle(f=(0.5, 0, 0, 1.0), mass=1.0, initial_volume=1.0)
    update(mat, p, 1.0)
    lo = float(f32(1.0) - mat.compression_limit)
    assert p.f[0] == pytest.approx(lo, rel=1e-6) and p.f[3] == pytest.approx(1.0, rel=1e-6)
    assert p.plastic_volume_ratio == pytest.approx(0.5 / lo, rel=1e-5)
    h = np.clip(np.exp(mat.hardening_exponent * (1.0 - p.plastic_volume_ratio)), 0.1, 7.0)
    assert p.hardening_scale == pytest.approx(h, rel=1e-5)
    assert p.volume == pytest.approx(lo, rel=1e-5)


def test_timestep_bounds_use_the_right_hardening():
    """Corotated and GranularFluid scale the wave speed with hardening_scale; VonMises,
    Rankine and mu(I) use 1."""
    def bound(mat, h):
        return lib().oracle_timestep_bound(byref(oracle_material(mat)), 4.0, h, 1.0, 0.5, 0.5)
    for mat in (CorotatedMaterial.new(1000.0, 800.0), GranularFluidMaterial.saturated_loam(2e4, 0.3)):
        assert bound(mat, 4.0) == pytest.approx(bound(mat, 1.0) / 2.0, rel=1e-6)
    for mat in (VonMisesMaterial.new(1000.0, 800.0, 10.0), RankineMaterial.new(1000.0, 800.0, 10.0, 1.0),
                MuIRheologyMaterial.new(1000.0, 800.0)):
        assert bound(mat, 4.0) == bound(mat, 1.0)


# ---------------------------------------------------------------- whole scenes
@pytest.mark.parametrize("kind", sorted(scenes.ZOO))
def test_zoo_scene_conserves_mass_and_keeps_j_positive(kind):
    sim = scenes.material_zoo(OracleSimulation, kind)
    m0 = sim.particles()["mass"].sum(dtype=np.float64)
    sim.step_n(5)
    p = sim.particles()
    assert p["mass"].sum(dtype=np.float64) == m0
    assert np.isfinite(p["x"]).all() and np.isfinite(p["v"]).all()
    f = p["f"]
    assert (f[:, 0] * f[:, 3] - f[:, 2] * f[:, 1]).min() > 0.0


def test_zoo_scenes_reach_their_plastic_branches():
    """The parity scenes exercise each model's return mapping, not only its elastic branch."""
    def run(kind):
        sim = scenes.material_zoo(OracleSimulation, kind)
        sim.step_n(2)
        return sim.particles()
    assert run("von_mises")["friction_hardening"].max() > 0.0
    assert run("rankine")["friction_hardening"].max() > 0.0
    q = run("mu_i")["friction_hardening"]
    assert q.max() > MuIRheologyMaterial.new(1.0, 1.0).mu_static
    jp = run("granular_fluid")["plastic_volume_ratio"]
    assert np.abs(jp - 1.0).max() > 1e-3
