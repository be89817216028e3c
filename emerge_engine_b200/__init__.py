"""B200-native (sm_100a) MLS-MPM step for emerge-engine, behind the reference's API.

`Simulation`, `SimConfig`, `SpawnRegion`, the constitutive models and `SlipBoundary` keep the
reference crate's names and semantics; the step runs in libemerge_cuda.so (include/emerge_cuda.h).
"""
from .config import BodyState, SimConfig, SlipBoundary, SpawnRegion  # noqa: F401
from .materials import (BinghamFluidMaterial, CorotatedMaterial,  # noqa: F401
                        DruckerPragerMaterial, FallbackMaterial, GranularFluidMaterial,
                        MuIRheologyMaterial, NaccMaterial, NeoHookeanMaterial,
                        NewtonianFluidMaterial, RankineMaterial, StomakhinMaterial,
                        ViscoelasticMaterial, VonMisesMaterial, lame_from_young, to_radians,
                        WithMixturePhase, SOLID_PHASE, FLUID_PHASE, DirectionalContactGrip)
from .fields import (AabbConfinementField, BuoyancyField, ChemotaxisField,  # noqa: F401
                     CoulombField, GravityWellField, LinearDragField, NBodyGravityField,
                     RadialConfinementField, UniformElectricField, orbit)
from .simulation import Batch, DeterministicSimulation, MaterialRegistry, Simulation  # noqa: F401
