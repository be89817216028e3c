"""Host-side mirror of the reference API: config validation, spawn builders, material
registry and the MaterialParams packing of each constitutive model."""
import numpy as np
import pytest

from emerge_engine_b200 import (DruckerPragerMaterial, MaterialRegistry, NaccMaterial,
                                NeoHookeanMaterial, NewtonianFluidMaterial, SimConfig,
                                SpawnRegion, StomakhinMaterial, lame_from_young, to_radians)
from emerge_engine_b200.materials import FallbackMaterial

f32 = np.float32


def test_standard_config_defaults():  # config.rs:127-172
    c = SimConfig.standard(64, 0.05, (0.0, -1.0))
    assert (c.grid_res, c.dt, c.gravity) == (64, 0.05, (0.0, -1.0))
    assert c.cfl_coefficient == 0.9 and c.material_cfl_coefficient == 0.5
    assert c.max_substeps_per_step == 64 and c.boundary_thickness == 2
    assert c.adaptive_timestep and c.project_invalid_state
    c.validate()


@pytest.mark.parametrize("field,value", [
    ("grid_res", 3), ("grid_cell_size", 0.0), ("dt", 0.0), ("cfl_coefficient", 0.0),
    ("min_dt", 0.0), ("min_dt", 1.0), ("particle_mass", 0.0), ("max_substeps_per_step", 0),
    ("j_max", 1.0), ("apic_blend", 1.5), ("boundary_thickness", 0), ("boundary_thickness", 63),
])
def test_config_validate_rejects(field, value):  # config.rs:247-299
    c = SimConfig.standard(64, 0.05, (0.0, -1.0))
    setattr(c, field, value)
    with pytest.raises(ValueError):
        c.validate()


def test_spawn_builders():  # config.rs:370-458
    c = SimConfig.standard(64, 0.05, (0.0, -1.0))
    s = SpawnRegion.for_sim(c)
    assert s.box_center == (32.0, 32.0)
    s.disk(12.0)
    assert s.box_size == (25, 25)  # ceil(2r) + 1
    s.with_spacing(0.5).material(3).mass(2.5).jitter(0.2).seed(7).velocity_scale(0.1)
    cs = s.to_c()
    assert cs.shape == 1 and cs.material_id == 3 and cs.has_mass_override == 1
    assert cs.mass_override == f32(2.5) and cs.rng_seed == 7


def test_registry_contiguous_ids():  # registry.rs:29-49
    r = MaterialRegistry(FallbackMaterial())
    r.insert(1, NeoHookeanMaterial.new(1.0, 1.0))
    with pytest.raises(ValueError):
        r.insert(3, NeoHookeanMaterial.new(1.0, 1.0))
    with pytest.raises(ValueError):
        r.insert(64, NeoHookeanMaterial.new(1.0, 1.0))
    assert r.next_id() == 2
    assert r.get(17) is r.materials[0]  # unknown ids fall back to slot 0


def test_lame_from_young_is_f32():  # utils.rs:183-194
    lam, mu = lame_from_young(1e5, 0.2)
    e, nu = f32(1e5), f32(0.2)
    assert lam == f32(e * nu) / f32((f32(1) + nu) * (f32(1) - f32(2) * nu))
    assert mu == e / (f32(2) * (f32(1) + nu))
    assert to_radians(35.0) == f32(35.0) * f32(f32(np.pi) / f32(180.0))


def test_params_packing_matches_reference_layouts():
    nh = NeoHookeanMaterial.new(400.0, 200.0)  # elastic.rs:275-288
    p = nh.params()
    assert (p.model, p.lambda_, p.mu) == (2, 400.0, 200.0)

    fl = NewtonianFluidMaterial.low_viscosity(1000.0, 1e4)  # fluid.rs:209-226
    p = fl.params()
    assert (p.model, p.rest_density, p.eos_stiffness, p.eos_power) == (1, 1000.0, 1e4, 7.0)
    assert p.dynamic_viscosity == f32(1e-3) and p.volume_ratio_max == 2.0
    assert p.pressure_floor == f32(-0.1)

    dp = DruckerPragerMaterial.cohesionless(1e5, 0.2)  # sand.rs:321-343
    p = dp.params()
    assert p.model == 5 and p.dp_h0 == to_radians(35.0) and p.dp_h1 == to_radians(9.0)
    assert p.dp_h2 == f32(0.2) and p.dp_h3 == to_radians(10.0)
    assert p.volume_ratio_min == f32(0.6) and p.compression_limit == 0.0

    sn = StomakhinMaterial.from_young_modulus(1.4e5, 0.2)  # snow.rs:178-191
    p = sn.params()
    assert (p.model, p.hardening_exponent) == (4, 10.0)
    assert p.compression_limit == f32(0.025) and p.stretch_limit == f32(0.0075)
    assert (p.volume_ratio_min, p.volume_ratio_max) == (f32(0.6), 20.0)

    nc = NaccMaterial.soft_clay(5e4, 0.3)  # nacc.rs:93-100, 300-314
    p = nc.params()
    assert p.model == 2  # NaccMaterial::params reports NeoHookean
    assert nc.abi_params().model == 10  # the ABI carries constitutive_model()
    assert p.lambda_ == f32(nc.kappa - nc.mu) and p.stretch_limit == f32(1.2)
    assert p.hardening_exponent == 2.0 and p.compression_limit == 0.0


def test_dp_init_particle_neutral_hardening():  # sand.rs:237-246
    dp = DruckerPragerMaterial.new(1.0, 1.0)
    assert dp.friction_residual / dp.hardening_peak == pytest.approx(10.0 / 9.0, rel=1e-6)
