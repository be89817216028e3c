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
DEVICE_MODELS = {FALLBACK, FLUID, NEOHOOKEAN, SNOW, DRUCKER_PRAGER, NACC}

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
