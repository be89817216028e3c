"""Constitutive models with the reference's constructors, in f32.

Each class mirrors one reference material struct (field names and defaults from the cited
constructor) and produces
  * `params()`        -- the reference's flat `MaterialParams` (materials/params.rs:10-101),
  * `abi_params()`    -- the same with `model` = `constitutive_model()`, which is what the
                         CUDA backend takes (NaccMaterial::params() reports NeoHookean,
                         nacc.rs:300-314, so the model id must travel separately),
  * `oracle_fields()` -- every struct field, for the CPU oracle.
All arithmetic is numpy float32, which rounds like Rust's f32 operators.
"""
from __future__ import annotations

from dataclasses import dataclass, fields

import numpy as np

from .abi import MaterialParamsC

f32 = np.float32

# ConstitutiveModel discriminants (matter/materials/mod.rs:53-66)
FALLBACK, FLUID, NEOHOOKEAN, COROTATED, SNOW, DRUCKER_PRAGER = 0, 1, 2, 3, 4, 5
VON_MISES, RANKINE, DP_MUI, VISCOELASTIC, NACC, GRANULAR_FLUID = 6, 7, 8, 9, 10, 11
DEVICE_MODELS = set(range(12))  # every ConstitutiveModel runs on the device

_RADS_PER_DEG = f32(f32(np.pi) / f32(180.0))  # f32::to_radians constant


def to_radians(deg) -> np.float32:
    return f32(f32(deg) * _RADS_PER_DEG)


def lame_from_young(young_modulus, poisson_ratio):
    """`lame_from_young` (matter/materials/utils.rs:183-194)."""
    e, nu = f32(young_modulus), f32(poisson_ratio)
    lam = f32(f32(e * nu) / f32(f32(f32(1.0) + nu) * f32(f32(1.0) - f32(f32(2.0) * nu))))
    mu = f32(e / f32(f32(2.0) * f32(f32(1.0) + nu)))
    return lam, mu


def _params(**kw) -> MaterialParamsC:
    p = MaterialParamsC()
    for k, v in kw.items():
        setattr(p, "lambda_" if k == "lambda" else k, v)
    return p


class Material:
    """Base: `MaterialModel` trait defaults (matter/materials/mod.rs:105-208)."""

    model = FALLBACK

    def constitutive_model(self) -> int:
        return self.model

    def params(self) -> MaterialParamsC:
        return _params(model=FALLBACK)

    def abi_params(self) -> MaterialParamsC:
        p = self.params()
        p.model = self.constitutive_model()
        return p

    def needs_density_recompute(self) -> bool:
        return False

    def oracle_fields(self) -> dict:
        return {"model": self.model}


class FallbackMaterial(Material):
    """`FallbackMaterial` (matter/materials/mod.rs:362-366): zero stress, no update."""


@dataclass
class NeoHookeanMaterial(Material):
    """`NeoHookeanMaterial` (matter/materials/elastic.rs:20-61)."""
    lambda_: float
    mu: float
    min_density: float = 1.0e-6
    thermal_expansion: float = 0.0
    active_stress_coeff: float = 0.0
    damage_softening_rate: float = 0.0
    viscosity: float = 0.0
    model = NEOHOOKEAN

    def __post_init__(self):
        for fl in fields(self):
            setattr(self, fl.name, f32(getattr(self, fl.name)))

    @classmethod
    def new(cls, lam, mu):
        return cls(lam, mu)

    @classmethod
    def from_young_modulus(cls, young_modulus, poisson_ratio):
        return cls(*lame_from_young(young_modulus, poisson_ratio))

    def params(self):  # elastic.rs:275-288
        return _params(model=NEOHOOKEAN, **{"lambda": self.lambda_}, mu=self.mu,
                       thermal_expansion=self.thermal_expansion,
                       active_stress_coeff=self.active_stress_coeff,
                       cohesion_coeff=self.damage_softening_rate,
                       dynamic_viscosity=self.viscosity)

    def oracle_fields(self):
        return dict(model=NEOHOOKEAN, lambda_=self.lambda_, mu=self.mu,
                    min_density=self.min_density, thermal_expansion=self.thermal_expansion,
                    active_stress_coeff=self.active_stress_coeff,
                    damage_softening_rate=self.damage_softening_rate, viscosity=self.viscosity)


@dataclass
class NewtonianFluidMaterial(Material):
    """`NewtonianFluidMaterial` (matter/materials/fluid.rs:10-75)."""
    rest_density: float
    dynamic_viscosity: float
    eos_stiffness: float
    eos_power: float
    pressure_floor: float = -0.1
    min_density: float = 1.0e-6
    min_volume: float = 1.0e-6
    thermal_viscosity_coeff: float = 0.0
    bulk_viscosity: float = 0.0
    surface_tension_coeff: float = 0.0
    settling_damping: float = 0.0
    model = FLUID

    def __post_init__(self):
        for fl in fields(self):
            setattr(self, fl.name, f32(getattr(self, fl.name)))

    @classmethod
    def new(cls, rest_density, dynamic_viscosity, eos_stiffness, eos_power):
        return cls(rest_density, dynamic_viscosity, eos_stiffness, eos_power)

    @classmethod
    def low_viscosity(cls, rest_density, eos_stiffness):  # fluid.rs:73-75
        return cls(rest_density, 1.0e-3, eos_stiffness, 7.0)

    def needs_density_recompute(self):  # fluid.rs:261-263
        return True

    def params(self):  # fluid.rs:209-226
        return _params(model=FLUID, rest_density=self.rest_density,
                       eos_stiffness=self.eos_stiffness, eos_power=self.eos_power,
                       dynamic_viscosity=self.dynamic_viscosity,
                       thermal_viscosity_coeff=self.thermal_viscosity_coeff,
                       volume_ratio_max=2.0, pressure_floor=self.pressure_floor,
                       bulk_viscosity=self.bulk_viscosity,
                       surface_tension_coeff=self.surface_tension_coeff,
                       dp_h0=self.settling_damping)

    def oracle_fields(self):
        return dict(model=FLUID, rest_density=self.rest_density,
                    dynamic_viscosity=self.dynamic_viscosity, eos_stiffness=self.eos_stiffness,
                    eos_power=self.eos_power, pressure_floor=self.pressure_floor,
                    fluid_min_density=self.min_density, fluid_min_volume=self.min_volume,
                    thermal_viscosity_coeff=self.thermal_viscosity_coeff,
                    bulk_viscosity=self.bulk_viscosity,
                    surface_tension_coeff=self.surface_tension_coeff,
                    settling_damping=self.settling_damping)


@dataclass
class DruckerPragerMaterial(Material):
    """`DruckerPragerMaterial` (matter/materials/sand.rs:11-130)."""
    lambda_: float
    mu: float
    friction_angle: float = None
    hardening_peak: float = None
    hardening_decay: float = 0.2
    friction_residual: float = None
    volume_correction: float = 1.0
    dilatancy_angle: float = 0.0
    cohesion: float = 0.0
    min_volume_jacobian: float = 0.6
    model = DRUCKER_PRAGER

    def __post_init__(self):
        if self.friction_angle is None:
            self.friction_angle = to_radians(35.0)
        if self.hardening_peak is None:
            self.hardening_peak = to_radians(9.0)
        if self.friction_residual is None:
            self.friction_residual = to_radians(10.0)
        for fl in fields(self):
            setattr(self, fl.name, f32(getattr(self, fl.name)))

    @classmethod
    def new(cls, lam, mu):  # sand.rs:81-94
        return cls(lam, mu)

    @classmethod
    def from_young_modulus(cls, young_modulus, poisson_ratio):  # sand.rs:100-103
        return cls(*lame_from_young(young_modulus, poisson_ratio))

    @classmethod
    def cohesionless(cls, young_modulus, poisson_ratio):  # sand.rs:106-108
        return cls.from_young_modulus(young_modulus, poisson_ratio)

    @classmethod
    def low_friction(cls, young_modulus, poisson_ratio):  # sand.rs:111-120
        lam, mu = lame_from_young(young_modulus, poisson_ratio)
        return cls(lam, mu, friction_angle=to_radians(25.0), hardening_peak=to_radians(4.0),
                   hardening_decay=0.1, friction_residual=to_radians(5.0))

    @classmethod
    def dilatant(cls, young_modulus, poisson_ratio):  # sand.rs:123-130
        lam, mu = lame_from_young(young_modulus, poisson_ratio)
        return cls(lam, mu, friction_angle=to_radians(38.0), dilatancy_angle=to_radians(12.0))

    def params(self):  # sand.rs:321-343
        return _params(model=DRUCKER_PRAGER, **{"lambda": self.lambda_}, mu=self.mu,
                       dp_h0=self.friction_angle, dp_h1=self.hardening_peak,
                       dp_h2=self.hardening_decay, dp_h3=self.friction_residual,
                       compression_limit=self.dilatancy_angle, stretch_limit=self.cohesion,
                       volume_ratio_min=self.min_volume_jacobian)

    def oracle_fields(self):
        return dict(model=DRUCKER_PRAGER, lambda_=self.lambda_, mu=self.mu,
                    friction_angle=self.friction_angle, hardening_peak=self.hardening_peak,
                    hardening_decay=self.hardening_decay,
                    friction_residual=self.friction_residual,
                    volume_correction=self.volume_correction,
                    dilatancy_angle=self.dilatancy_angle, cohesion=self.cohesion,
                    min_volume_jacobian=self.min_volume_jacobian)


@dataclass
class StomakhinMaterial(Material):
    """`StomakhinMaterial` snow (matter/materials/snow.rs:19-84)."""
    lambda_: float
    mu: float
    hardening_exponent: float
    compression_limit: float
    stretch_limit: float
    min_plastic_jacobian: float
    max_plastic_jacobian: float
    cohesion_coeff: float = 0.0
    model = SNOW

    def __post_init__(self):
        for fl in fields(self):
            setattr(self, fl.name, f32(getattr(self, fl.name)))

    @classmethod
    def new(cls, lam, mu, xi, theta_c, theta_s, min_jp, max_jp):
        return cls(lam, mu, xi, theta_c, theta_s, min_jp, max_jp)

    def with_cohesion(self, coeff):
        self.cohesion_coeff = f32(coeff)
        return self

    @classmethod
    def from_young_modulus(cls, young_modulus, poisson_ratio):  # snow.rs:68-71
        lam, mu = lame_from_young(young_modulus, poisson_ratio)
        return cls(lam, mu, 10.0, 0.025, 0.0075, 0.6, 20.0)

    @classmethod
    def low_cohesion(cls, young_modulus, poisson_ratio):  # snow.rs:74-77
        lam, mu = lame_from_young(young_modulus, poisson_ratio)
        return cls(lam, mu, 5.0, 0.01, 0.003, 0.5, 20.0)

    @classmethod
    def high_cohesion(cls, young_modulus, poisson_ratio):  # snow.rs:80-83
        lam, mu = lame_from_young(young_modulus, poisson_ratio)
        return cls(lam, mu, 15.0, 0.04, 0.005, 0.6, 20.0).with_cohesion(800.0)

    def params(self):  # snow.rs:178-191
        return _params(model=SNOW, **{"lambda": self.lambda_}, mu=self.mu,
                       hardening_exponent=self.hardening_exponent,
                       compression_limit=self.compression_limit,
                       stretch_limit=self.stretch_limit,
                       volume_ratio_min=self.min_plastic_jacobian,
                       volume_ratio_max=self.max_plastic_jacobian,
                       cohesion_coeff=self.cohesion_coeff)

    def oracle_fields(self):
        return dict(model=SNOW, lambda_=self.lambda_, mu=self.mu,
                    hardening_exponent=self.hardening_exponent,
                    compression_limit=self.compression_limit, stretch_limit=self.stretch_limit,
                    min_plastic_jacobian=self.min_plastic_jacobian,
                    max_plastic_jacobian=self.max_plastic_jacobian,
                    cohesion_coeff=self.cohesion_coeff)


@dataclass
class NaccMaterial(Material):
    """`NaccMaterial` Cam-clay (matter/materials/nacc.rs:34-120)."""
    mu: float
    kappa: float
    friction: float
    cohesion: float
    hardening_factor: float
    hardening_enabled: bool = None
    min_density: float = 1.0e-6
    model = NACC

    def __post_init__(self):
        self.mu, self.kappa = f32(self.mu), f32(self.kappa)
        self.friction, self.cohesion = f32(self.friction), f32(self.cohesion)
        self.hardening_factor = f32(self.hardening_factor)
        if self.hardening_enabled is None:
            self.hardening_enabled = bool(self.hardening_factor > 0.0)
        self.min_density = f32(self.min_density)

    @classmethod
    def new(cls, mu, kappa, friction, cohesion, hardening_factor):  # nacc.rs:63-73
        return cls(mu, kappa, friction, cohesion, hardening_factor)

    @classmethod
    def from_young_modulus(cls, young_modulus, poisson_ratio, friction, cohesion,
                           hardening_factor):  # nacc.rs:77-90
        lam, mu = lame_from_young(young_modulus, poisson_ratio)
        return cls(mu, f32(lam + mu), friction, cohesion, hardening_factor)

    @classmethod
    def soft_clay(cls, young_modulus, poisson_ratio):  # nacc.rs:93-100
        lam, mu = lame_from_young(young_modulus, poisson_ratio)
        return cls(mu, f32(lam + mu), 1.2, 0.0, 2.0)

    @classmethod
    def wet_soil(cls, young_modulus, poisson_ratio):  # nacc.rs:103-110
        lam, mu = lame_from_young(young_modulus, poisson_ratio)
        return cls(mu, f32(lam + mu), 1.0, 0.0, 3.0)

    @classmethod
    def low_hardening(cls, young_modulus, poisson_ratio):  # nacc.rs:113-120
        lam, mu = lame_from_young(young_modulus, poisson_ratio)
        return cls(mu, f32(lam + mu), 1.5, 0.0, 1.0)

    def params(self):  # nacc.rs:300-314 (reports the NeoHookean model id)
        return _params(model=NEOHOOKEAN, **{"lambda": f32(self.kappa - self.mu)}, mu=self.mu,
                       hardening_exponent=self.hardening_factor,
                       compression_limit=self.cohesion, stretch_limit=self.friction)

    def oracle_fields(self):
        return dict(model=NACC, mu=self.mu, kappa=self.kappa, friction=self.friction,
                    nacc_cohesion=self.cohesion, hardening_factor=self.hardening_factor,
                    hardening_enabled=int(self.hardening_enabled),
                    nacc_min_density=self.min_density)


def _tan_deg(deg) -> np.float32:
    """`deg.to_radians().tan()` in f32."""
    return f32(np.tan(to_radians(deg)))


@dataclass
class CorotatedMaterial(Material):
    """`CorotatedMaterial` (matter/materials/corotated.rs): corotated linear elasticity with
    snow-style hardening scale, thermal modulus scaling and fibre active stress."""
    lambda_: float
    mu: float
    thermal_expansion: float = 0.0
    active_stress_coeff: float = 0.0
    model = COROTATED

    def __post_init__(self):
        for fl in fields(self):
            setattr(self, fl.name, f32(getattr(self, fl.name)))

    @classmethod
    def new(cls, lam, mu):
        return cls(lam, mu)

    @classmethod
    def from_young_modulus(cls, young_modulus, poisson_ratio):
        return cls(*lame_from_young(young_modulus, poisson_ratio))

    def params(self):  # corotated.rs params()
        return _params(model=COROTATED, **{"lambda": self.lambda_}, mu=self.mu,
                       thermal_expansion=self.thermal_expansion,
                       active_stress_coeff=self.active_stress_coeff)

    def oracle_fields(self):
        return dict(model=COROTATED, lambda_=self.lambda_, mu=self.mu,
                    thermal_expansion=self.thermal_expansion,
                    active_stress_coeff=self.active_stress_coeff)


@dataclass
class VonMisesMaterial(Material):
    """`VonMisesMaterial` (matter/materials/von_mises.rs:27-74): J2 plasticity on the Hencky
    strain with linear isotropic hardening."""
    lambda_: float
    mu: float
    yield_stress: float
    hardening_modulus: float = 0.0
    model = VON_MISES

    def __post_init__(self):
        for fl in fields(self):
            setattr(self, fl.name, f32(getattr(self, fl.name)))

    @classmethod
    def new(cls, lam, mu, yield_stress):  # von_mises.rs:49-56
        return cls(lam, mu, yield_stress)

    @classmethod
    def with_hardening(cls, lam, mu, yield_stress, hardening_modulus):  # von_mises.rs:60-68
        if not hardening_modulus >= 0.0:
            raise ValueError("hardening_modulus must be >= 0")
        return cls(lam, mu, yield_stress, hardening_modulus)

    @classmethod
    def from_young_modulus(cls, young_modulus, poisson_ratio, yield_stress):  # von_mises.rs:43-46
        return cls(*lame_from_young(young_modulus, poisson_ratio), yield_stress)

    @classmethod
    def soft_ductile(cls, young_modulus, poisson_ratio):  # von_mises.rs:71-73
        return cls.from_young_modulus(young_modulus, poisson_ratio,
                                      f32(f32(young_modulus) * f32(0.005)))

    def params(self):  # von_mises.rs:143-152
        return _params(model=VON_MISES, **{"lambda": self.lambda_}, mu=self.mu,
                       hardening_exponent=self.yield_stress,
                       hardening_modulus=self.hardening_modulus)

    def oracle_fields(self):
        return dict(model=VON_MISES, lambda_=self.lambda_, mu=self.mu,
                    yield_stress=self.yield_stress, hardening_modulus=self.hardening_modulus)


@dataclass
class RankineMaterial(Material):
    """`RankineMaterial` (matter/materials/rankine.rs): maximum principal stress tensile
    failure with exponential softening, damage in `friction_hardening`."""
    lambda_: float
    mu: float
    tensile_strength: float
    softening_rate: float
    model = RANKINE

    def __post_init__(self):
        for fl in fields(self):
            setattr(self, fl.name, f32(getattr(self, fl.name)))

    @classmethod
    def new(cls, lam, mu, tensile_strength, softening_rate):
        return cls(lam, mu, tensile_strength, softening_rate)

    @classmethod
    def from_young_modulus(cls, young_modulus, poisson_ratio, tensile_strength, softening_rate):
        return cls(*lame_from_young(young_modulus, poisson_ratio), tensile_strength,
                   softening_rate)

    @classmethod
    def stiff_brittle(cls, young_modulus, poisson_ratio):  # rock: tensile 2.5e-4 E, rate 2
        return cls.from_young_modulus(young_modulus, poisson_ratio,
                                      f32(f32(young_modulus) * f32(2.5e-4)), 2.0)

    @classmethod
    def high_tensile(cls, young_modulus, poisson_ratio):  # bone: tensile 7e-3 E, rate 1
        return cls.from_young_modulus(young_modulus, poisson_ratio,
                                      f32(f32(young_modulus) * f32(7.0e-3)), 1.0)

    def params(self):  # rankine.rs params()
        return _params(model=RANKINE, **{"lambda": self.lambda_}, mu=self.mu,
                       hardening_exponent=self.tensile_strength,
                       hardening_modulus=self.softening_rate)

    def oracle_fields(self):
        return dict(model=RANKINE, lambda_=self.lambda_, mu=self.mu,
                    tensile_strength=self.tensile_strength, softening_rate=self.softening_rate)


@dataclass
class MuIRheologyMaterial(Material):
    """`MuIRheologyMaterial` (matter/materials/sand_mui.rs): rate-dependent granular
    friction mu(I) = mu_s + (mu_d - mu_s) / (I0 / I + 1), current mu in
    `friction_hardening`."""
    lambda_: float
    mu: float
    mu_static: float = None
    mu_dynamic: float = None
    inertial_q: float = 5.58
    model = DP_MUI

    def __post_init__(self):
        if self.mu_static is None:
            self.mu_static = _tan_deg(20.9)
        if self.mu_dynamic is None:
            self.mu_dynamic = _tan_deg(32.8)
        for fl in fields(self):
            setattr(self, fl.name, f32(getattr(self, fl.name)))

    @classmethod
    def new(cls, lam, mu):
        return cls(lam, mu)

    @classmethod
    def from_young_modulus(cls, young_modulus, poisson_ratio):
        return cls(*lame_from_young(young_modulus, poisson_ratio))

    @classmethod
    def large_grain(cls, young_modulus, poisson_ratio):
        return cls(*lame_from_young(young_modulus, poisson_ratio), inertial_q=1.12)

    @classmethod
    def small_grain(cls, young_modulus, poisson_ratio):
        return cls.from_young_modulus(young_modulus, poisson_ratio)

    @classmethod
    def dense_packed(cls, young_modulus, poisson_ratio):
        return cls(*lame_from_young(young_modulus, poisson_ratio), mu_static=_tan_deg(30.0),
                   mu_dynamic=_tan_deg(40.0))

    def params(self):  # sand_mui.rs params()
        return _params(model=DP_MUI, **{"lambda": self.lambda_}, mu=self.mu,
                       dp_h0=self.mu_static, dp_h1=self.mu_dynamic, dp_h2=self.inertial_q)

    def oracle_fields(self):
        return dict(model=DP_MUI, lambda_=self.lambda_, mu=self.mu, mu_static=self.mu_static,
                    mu_dynamic=self.mu_dynamic, inertial_q=self.inertial_q)


@dataclass
class ViscoelasticMaterial(Material):
    """`ViscoelasticMaterial` (matter/materials/viscoelastic.rs): Neo-Hookean spring with a
    Kelvin-Voigt deviatoric dashpot and isotropic active stress."""
    lambda_: float
    mu: float
    viscosity: float
    j_min: float = 0.01
    active_stress_coeff: float = 0.0
    thermal_expansion: float = 0.0
    model = VISCOELASTIC

    def __post_init__(self):
        for fl in fields(self):
            setattr(self, fl.name, f32(getattr(self, fl.name)))

    @classmethod
    def new(cls, lam, mu, viscosity):
        return cls(lam, mu, viscosity)

    @classmethod
    def from_young_modulus(cls, young_modulus, poisson_ratio, viscosity):
        return cls(*lame_from_young(young_modulus, poisson_ratio), viscosity)

    @classmethod
    def near_incompressible(cls, young_modulus, viscosity):
        return cls.from_young_modulus(young_modulus, 0.45, viscosity)

    @classmethod
    def moderately_compressible(cls, young_modulus, viscosity):
        return cls.from_young_modulus(young_modulus, 0.40, viscosity)

    @classmethod
    def rubber_damper(cls, young_modulus, viscosity):
        return cls.from_young_modulus(young_modulus, 0.45, viscosity)

    def params(self):  # viscoelastic.rs params()
        return _params(model=VISCOELASTIC, **{"lambda": self.lambda_}, mu=self.mu,
                       dynamic_viscosity=self.viscosity,
                       active_stress_coeff=self.active_stress_coeff,
                       volume_ratio_min=self.j_min)

    def abi_params(self):
        # params() leaves thermal_expansion out; the CPU stress uses it, so the CUDA
        # backend receives it in the same slot NeoHookean and Corotated use.
        p = super().abi_params()
        p.thermal_expansion = self.thermal_expansion
        return p

    def oracle_fields(self):
        return dict(model=VISCOELASTIC, lambda_=self.lambda_, mu=self.mu,
                    viscosity=self.viscosity, j_min=self.j_min,
                    active_stress_coeff=self.active_stress_coeff,
                    thermal_expansion=self.thermal_expansion)


@dataclass
class GranularFluidMaterial(Material):
    """`GranularFluidMaterial` (matter/materials/granular_fluid.rs): Tait pressure plus
    deviatoric corotated elasticity with snow-style plastic volume hardening."""
    lambda_: float
    mu: float
    rest_density: float
    eos_stiffness: float
    hardening_exponent: float
    compression_limit: float
    eos_power: float = 7.0
    stretch_limit: float = 0.01
    min_plastic_jacobian: float = 0.2
    max_plastic_jacobian: float = 3.0
    pressure_floor: float = 0.0
    model = GRANULAR_FLUID

    def __post_init__(self):
        for fl in fields(self):
            setattr(self, fl.name, f32(getattr(self, fl.name)))

    @classmethod
    def new(cls, lam, mu, rest_density, eos_stiffness, hardening_exponent, compression_limit):
        return cls(lam, mu, rest_density, eos_stiffness, hardening_exponent, compression_limit)

    @classmethod
    def saturated_loam(cls, young_modulus, poisson_ratio):
        return cls(*lame_from_young(young_modulus, poisson_ratio), 1.0, 200.0, 5.0, 0.4)

    @classmethod
    def consolidated_clay(cls, young_modulus, poisson_ratio):
        return cls(*lame_from_young(young_modulus, poisson_ratio), 1.2, 500.0, 3.0, 0.3,
                   min_plastic_jacobian=0.3, max_plastic_jacobian=2.5)

    @classmethod
    def cytoplasmic(cls, young_modulus, poisson_ratio):
        return cls(*lame_from_young(young_modulus, poisson_ratio), 1.0, 50.0, 1.0, 0.6,
                   stretch_limit=0.05, min_plastic_jacobian=0.1, max_plastic_jacobian=5.0)

    def params(self):  # granular_fluid.rs params()
        return _params(model=GRANULAR_FLUID, mu=self.mu, **{"lambda": self.lambda_},
                       rest_density=self.rest_density, eos_stiffness=self.eos_stiffness,
                       eos_power=self.eos_power, hardening_exponent=self.hardening_exponent,
                       compression_limit=self.compression_limit,
                       stretch_limit=self.stretch_limit,
                       volume_ratio_min=self.min_plastic_jacobian,
                       volume_ratio_max=self.max_plastic_jacobian,
                       pressure_floor=self.pressure_floor)

    def oracle_fields(self):
        return dict(model=GRANULAR_FLUID, lambda_=self.lambda_, mu=self.mu,
                    rest_density=self.rest_density, eos_stiffness=self.eos_stiffness,
                    eos_power=self.eos_power, hardening_exponent=self.hardening_exponent,
                    compression_limit=self.compression_limit,
                    stretch_limit=self.stretch_limit,
                    min_plastic_jacobian=self.min_plastic_jacobian,
                    max_plastic_jacobian=self.max_plastic_jacobian,
                    pressure_floor=self.pressure_floor)


@dataclass
class BinghamFluidMaterial(Material):
    """`BinghamFluidMaterial` (matter/materials/bingham.rs): Tait pressure plus the Bingham
    deviatoric stress (yield / shear_rate + viscosity) D_dev above the critical shear rate.
    Its constitutive model is Fluid; MaterialParams carries the yield stress in
    `compression_limit`, which is how the CUDA backend tells it from a Newtonian fluid."""
    rest_density: float
    dynamic_viscosity: float
    eos_stiffness: float
    eos_power: float
    yield_stress: float
    critical_shear_rate: float = 1.0e-4
    pressure_floor: float = 0.0
    min_density: float = 1.0e-6
    min_volume: float = 1.0e-6
    surface_tension_coeff: float = 0.0
    settling_damping: float = 0.0
    model = FLUID

    def __post_init__(self):
        for fl in fields(self):
            setattr(self, fl.name, f32(getattr(self, fl.name)))

    @classmethod
    def new(cls, rest_density, dynamic_viscosity, eos_stiffness, eos_power, yield_stress):
        return cls(rest_density, dynamic_viscosity, eos_stiffness, eos_power, yield_stress)

    @classmethod
    def high_yield(cls, rest_density, eos_stiffness):
        return cls(rest_density, 0.5, eos_stiffness, 7.0, 100.0)

    @classmethod
    def viscous_high_yield(cls, rest_density, eos_stiffness):
        return cls(rest_density, 500.0, eos_stiffness, 7.0, 1000.0)

    @classmethod
    def low_yield(cls, rest_density, eos_stiffness):
        return cls(rest_density, 0.01, eos_stiffness, 7.0, 1.0)

    @classmethod
    def medium_yield(cls, rest_density, eos_stiffness):
        return cls(rest_density, 0.1, eos_stiffness, 7.0, 10.0)

    def needs_density_recompute(self):  # bingham.rs
        return True

    def params(self):  # bingham.rs params()
        return _params(model=FLUID, rest_density=self.rest_density,
                       eos_stiffness=self.eos_stiffness, eos_power=self.eos_power,
                       dynamic_viscosity=self.dynamic_viscosity,
                       compression_limit=self.yield_stress, volume_ratio_max=2.0,
                       pressure_floor=self.pressure_floor,
                       surface_tension_coeff=self.surface_tension_coeff,
                       dp_h0=self.settling_damping)

    def abi_params(self):
        # Fields params() cannot carry are fixed on the device at the constructor's values.
        if not self.yield_stress > 0.0:
            raise ValueError("BinghamFluidMaterial needs yield_stress > 0 on the CUDA backend "
                             "(MaterialParams marks a Bingham fluid by compression_limit > 0)")
        fixed = dict(critical_shear_rate=1.0e-4, min_density=1.0e-6, min_volume=1.0e-6)
        for k, v in fixed.items():
            if getattr(self, k) != f32(v):
                raise ValueError(f"BinghamFluidMaterial.{k} must be {v} on the CUDA backend")
        return super().abi_params()

    def oracle_fields(self):
        return dict(model=FLUID, bingham=1, rest_density=self.rest_density,
                    dynamic_viscosity=self.dynamic_viscosity, eos_stiffness=self.eos_stiffness,
                    eos_power=self.eos_power, bingham_yield_stress=self.yield_stress,
                    critical_shear_rate=self.critical_shear_rate,
                    pressure_floor=self.pressure_floor, fluid_min_density=self.min_density,
                    fluid_min_volume=self.min_volume,
                    surface_tension_coeff=self.surface_tension_coeff,
                    settling_damping=self.settling_damping)


SOLID_PHASE, FLUID_PHASE = 1, 2  # MixturePhase (materials/mod.rs:96-103)


class WithMixturePhase(Material):
    """`WithMixturePhase` (matter/materials/mod.rs:296-357): any material tagged as the solid
    or fluid phase of a two-phase mixture; every other behaviour is the inner material's."""

    def __init__(self, inner: Material, phase: int):
        if phase not in (SOLID_PHASE, FLUID_PHASE):
            raise ValueError("phase must be SOLID_PHASE or FLUID_PHASE")
        self.inner = inner
        self.phase = phase
        self.model = inner.model

    @classmethod
    def new(cls, inner: Material, phase: int):
        return cls(inner, phase)

    def mixture_phase(self) -> int:
        return self.phase

    def constitutive_model(self) -> int:
        return self.inner.constitutive_model()

    def params(self):
        return self.inner.params()

    def abi_params(self):
        return self.inner.abi_params()

    def needs_density_recompute(self) -> bool:
        return self.inner.needs_density_recompute()

    def oracle_fields(self):
        return dict(self.inner.oracle_fields(), mixture_phase=self.phase)


def mixture_phase_of(m: Material) -> int:
    """MaterialModel::mixture_phase (materials/mod.rs:170-172): 0 for none."""
    return m.mixture_phase() if hasattr(m, "mixture_phase") else 0


class DirectionalContactGrip:
    """`DirectionalContactGrip` (spacetime/grid/directional_grip.rs): contact friction that
    depends on the slip direction; Simulation.with_contact_grip installs it.  Changes made
    with set_easy_direction / set_friction apply when the simulation is given it again."""

    def __init__(self, mu_easy, mu_resist, easy_direction):
        self.set_friction(mu_easy, mu_resist)
        self.set_easy_direction(easy_direction)

    @classmethod
    def new(cls, mu_easy, mu_resist, easy_direction):
        return cls(mu_easy, mu_resist, easy_direction)

    def set_friction(self, mu_easy, mu_resist):
        if not (0.0 <= mu_easy <= 1.0 and 0.0 <= mu_resist <= 1.0):
            raise ValueError("mu_easy and mu_resist must be in [0.0, 1.0]")
        self.mu_easy, self.mu_resist = f32(mu_easy), f32(mu_resist)

    def set_easy_direction(self, direction):
        """glam Vec2::normalize_or_zero in f32 (directional_grip.rs:55-58)."""
        d = np.array([direction[0], direction[1]], dtype=np.float32)
        with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
            rcp = np.float32(1.0) / np.sqrt(d[0] * d[0] + d[1] * d[1], dtype=np.float32)
        d = d * rcp if np.isfinite(rcp) and rcp > 0.0 else np.zeros(2, dtype=np.float32)
        self.easy_direction = (float(d[0]), float(d[1]))
