"""Scene builders shared by the parity tests, the smoke check and bench.py.

Each builder takes the simulation class (the CUDA `Simulation` or the oracle's
`OracleSimulation`) so both backends see identical construction calls.
"""
from __future__ import annotations

import numpy as np

from emerge_engine_b200 import (BinghamFluidMaterial, CorotatedMaterial, DruckerPragerMaterial,
                                GranularFluidMaterial, MuIRheologyMaterial, NaccMaterial,
                                NeoHookeanMaterial, NewtonianFluidMaterial, RankineMaterial,
                                SimConfig, SlipBoundary, SpawnRegion, StomakhinMaterial,
                                ViscoelasticMaterial, VonMisesMaterial, lame_from_young)


def quickstart(sim_cls, **sim_kw):
    """README quick start (README.md:20-49): NeoHookean 12x12 block + fluid 12x8 block."""
    cfg = SimConfig.standard(64, 0.05, (0.0, -1.0))
    sim = (sim_cls.empty(cfg, **sim_kw)
           .with_default_material(NeoHookeanMaterial.new(400.0, 200.0))
           .with_material(1, NewtonianFluidMaterial.low_viscosity(1000.0, 1e4))
           .with_boundary(SlipBoundary(2)))
    a = SpawnRegion.for_sim(cfg)
    a.box_size, a.box_center, a.precompute_initial_volumes = (12, 12), (24.0, 40.0), True
    b = SpawnRegion.for_sim(cfg)
    b.box_size, b.box_center, b.material_id, b.precompute_initial_volumes = (12, 8), (40.0, 36.0), 1, True
    sim.add_body(a)
    sim.add_body(b)
    return sim


def dam_break(sim_cls, grid_res=512, column=256, seed=1, gravity=-1.0, **sim_kw):
    """Dam break: a `column` x `column` water column at 4 particles per cell (spacing 0.5,
    seeded jitter of +-0.25 cell) in the lower-left corner of a grid_res^2 grid.
    NewtonianFluid Tait EOS rho0 = 1000, stiffness 1e4, gamma 7; particle mass
    rho0 * spacing^2 = 250 so the rest density matches rho0."""
    cfg = SimConfig.standard(grid_res, 0.05, (0.0, gravity))
    sim = sim_cls.empty(cfg, **sim_kw).with_default_material(
        NewtonianFluidMaterial.low_viscosity(1000.0, 1e4))
    s = SpawnRegion.for_sim(cfg)
    t = cfg.boundary_thickness
    s.spacing = 0.5
    s.box_size = (column, column)
    s.box_center = (t + column / 2.0, t + column / 2.0)
    s.position_jitter = 0.5
    s.rng_seed = seed
    s.mass_override = 1000.0 * 0.25
    sim.add_body(s)
    return sim


def granular_blocks(grid_res, target_particles, seed=42, side_range=(16, 128), spacing=0.5):
    """Seeded axis-aligned blocks with sides in side_range cells: a guillotine partition of
    [t, grid_res - t)^2 (split each rectangle at a random position until both sides are at
    most side_range[1], never below side_range[0]), then blocks are kept in seeded random
    order until the particle target is reached; the dropped blocks leave voids.  Each block
    gets a material index uniform over {0, 1, 2}.  Returns [(x0, y0, w, h, mat)]."""
    rng = np.random.default_rng(seed)
    t = 2
    lo, hi = side_range
    stack = [(t, t, grid_res - 2 * t, grid_res - 2 * t)]
    leaves = []
    while stack:
        x0, y0, w, h = stack.pop()
        axis = None
        if w > hi and (h <= hi or w >= h):
            axis = 0
        elif h > hi:
            axis = 1
        if axis is None:
            leaves.append((x0, y0, w, h))
            continue
        side = w if axis == 0 else h
        cut = int(rng.integers(lo, side - lo + 1))
        if axis == 0:
            stack += [(x0, y0, cut, h), (x0 + cut, y0, w - cut, h)]
        else:
            stack += [(x0, y0, w, cut), (x0, y0 + cut, w, h - cut)]
    per_cell = int(round(1.0 / spacing)) ** 2
    order = rng.permutation(len(leaves))
    blocks, count = [], 0
    for k in order:
        if count >= target_particles:
            break
        x0, y0, w, h = leaves[k]
        blocks.append((x0, y0, w, h, int(rng.integers(0, 3))))
        count += w * h * per_cell
    blocks.sort()
    return blocks


def mixed_granular(sim_cls, grid_res=1024, target_particles=4_000_000, seed=42, gravity=-1.0,
                   dt=0.05, **sim_kw):
    """Mixed granular: seeded random blocks (16-128 cells a side), each block uniformly
    DruckerPrager sand, Stomakhin snow or NACC soil with the reference's canonical
    constructors (sand.rs:106, snow.rs:68, nacc.rs:93), 4 particles per cell."""
    cfg = SimConfig.standard(grid_res, dt, (0.0, gravity))
    sim = (sim_cls.empty(cfg, **sim_kw)
           .with_default_material(DruckerPragerMaterial.cohesionless(1e5, 0.2))
           .with_material(1, StomakhinMaterial.from_young_modulus(1.4e5, 0.2))
           .with_material(2, NaccMaterial.soft_clay(5e4, 0.3)))
    for (x0, y0, w, h, mat) in granular_blocks(grid_res, target_particles, seed):
        s = SpawnRegion.for_sim(cfg)
        s.spacing = 0.5
        s.box_size = (w, h)
        s.box_center = (x0 + w / 2.0, y0 + h / 2.0)
        s.material_id = mat
        s.position_jitter = 0.2
        s.rng_seed = (seed * 7919 + x0 * 131 + y0) & 0xFFFFFFFF
        sim.add_body(s)
    return sim


def batched_scene_draws(n_scenes=256, seed=7, grid_range=(64, 256), n_range=(4_000, 200_000),
                        pair_sizes=False):
    """The seeded per-scene draws of batched_scenes: (grid size G, particle target, material
    kind) per scene.  With pair_sizes, the drawn grid sizes and particle counts are paired by
    rank (the largest count with the largest grid), which keeps both distributions as drawn
    and lets every block fit at 4 particles per cell: 256 scenes then hold the ~12.8M
    particles the two distributions give (mean N ~ 50k)."""
    rng = np.random.default_rng(seed)
    draws = []
    for k in range(n_scenes):
        g = int(rng.integers(grid_range[0], grid_range[1] + 1))
        target = float(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1]))))
        kind = int(rng.integers(4))
        draws.append((g, target, kind))
    if pair_sizes:
        gs = sorted(d[0] for d in draws)
        ns = sorted(d[1] for d in draws)
        order = np.argsort([d[0] for d in draws], kind="stable")
        paired = list(draws)
        for rank, k in enumerate(order):
            paired[k] = (gs[rank], ns[rank], draws[k][2])
        draws = paired
    return draws


def _block_side(g, target, thickness=2):
    return int(min(np.sqrt(target / 4.0), g - 2 * thickness - 6))


def batched_scene_particles(draws):
    """Particles each drawn scene spawns (4 per cell of its side x side block)."""
    return [4 * _block_side(g, t) ** 2 for g, t, _ in draws]


def batched_scenes(sim_cls, n_scenes=256, seed=7, grid_range=(64, 256), n_range=(4_000, 200_000),
                   pair_sizes=False, only=None, **sim_kw):
    """Independent scenes for the batched path: per scene a seeded grid size G ~ U{64..256},
    a particle target N ~ logU[4k, 200k] and a material uniform over {NewtonianFluid,
    DruckerPrager sand, Stomakhin snow, NeoHookean}; one square block at 4 particles per cell
    (seeded jitter) resting on the floor of a G^2 grid, clipped to fit inside the walls (so
    small grids hold fewer particles than their target).  pair_sizes: see
    batched_scene_draws.  only: the indices of the scenes to build (a rank's share of one
    fixed list; each scene's seeds depend on its index only).  Returns the simulations."""
    draws = batched_scene_draws(n_scenes, seed, grid_range, n_range, pair_sizes)
    keep = range(n_scenes) if only is None else only
    sims = []
    for k in keep:
        g, target, kind = draws[k]
        cfg = SimConfig.standard(g, 0.05, (0.0, -1.0))
        t = cfg.boundary_thickness
        if kind == 0:
            mat = NewtonianFluidMaterial.low_viscosity(1000.0, 1e4)
        elif kind == 1:
            mat = DruckerPragerMaterial.cohesionless(1e5, 0.2)
        elif kind == 2:
            mat = StomakhinMaterial.from_young_modulus(1.4e5, 0.2)
        else:
            mat = NeoHookeanMaterial.new(400.0, 200.0)
        sim = sim_cls.empty(cfg, **sim_kw).with_default_material(mat)
        side = _block_side(g, target, t)
        s = SpawnRegion.for_sim(cfg)
        s.spacing = 0.5
        s.box_size = (side, side)
        s.box_center = (g / 2.0, t + 2 + side / 2.0)
        s.position_jitter = 0.4
        s.rng_seed = (seed * 1000003 + k) & 0xFFFFFFFF
        if kind == 0:
            s.mass_override = 1000.0 * 0.25
        sim.add_body(s)
        sims.append(sim)
    return sims


def nacc_ellipse(sim_cls, grid_res=256, n_blocks=40, side=24, seed=11, **sim_kw):
    """NACC soil (NaccMaterial.soft_clay(5e4, 0.3), nacc.rs:93-100) whose particles start on
    the smooth plastic branch of the projection, the ellipse (nacc.rs:171-223).  The
    reference's CPU update never advances a NACC particle's F (nacc.rs:255-269), so soil
    spawned with F = I stays elastic; here each of n_blocks side x side-cell blocks (4
    particles per cell) gets a seeded pre-deformation F0 = [[1 + e1, g], [0, 1 + e2]] (shear
    g in [-0.3, 0.3], compressive strains e in [-0.03, 0]) and a seeded hardened state
    (log_volume_strain alpha in [-0.2, -0.01]: p0 = kappa (1e-5 + sinh(2 |alpha|))), so that
    about two thirds of the blocks' trial states lie outside the ellipse at moderate
    pressure.  No gravity; blocks on a lattice."""
    rng = np.random.default_rng(seed)
    cfg = SimConfig.standard(grid_res, 0.05, (0.0, 0.0))
    sim = sim_cls.empty(cfg, **sim_kw).with_default_material(NaccMaterial.soft_clay(5e4, 0.3))
    per_row = int((grid_res - 8) // (side + 4))
    alphas = {}
    for k in range(n_blocks):
        r, c = divmod(k, per_row)
        cx = 6 + c * (side + 4) + side / 2.0
        cy = 6 + r * (side + 4) + side / 2.0
        if cy + side / 2.0 > grid_res - 6:
            break
        s = SpawnRegion.for_sim(cfg)
        s.spacing = 0.5
        s.box_size = (side, side)
        s.box_center = (cx, cy)
        g, e1, e2 = rng.uniform(-0.3, 0.3), rng.uniform(-0.03, 0.0), rng.uniform(-0.03, 0.0)
        s.initial_deformation_gradient = (1.0 + e1, 0.0, g, 1.0 + e2)  # x_axis, y_axis columns
        s.position_jitter = 0.2
        s.rng_seed = (seed * 7919 + k) & 0xFFFFFFFF
        tag = sim.add_body(s)
        alphas[tag] = rng.uniform(-0.2, -0.01)
    p = sim.particles()
    for tag, a in alphas.items():
        p["log_volume_strain"][p["user_tag"] == tag] = a
    sim.set_particles(p)
    return sim


# One material per constitutive model beyond the core set, with parameters that put it in
# its plastic / viscous / yield regime within the first frame: (constructor, mass override
# for 0.5-cell spacing or None, whether particles carry temperature and activation).
ZOO = {
    "corotated": (lambda: CorotatedMaterial(*lame_from_young(2e4, 0.3), thermal_expansion=0.02,
                                            active_stress_coeff=40.0), None, True),
    "von_mises": (lambda: VonMisesMaterial.with_hardening(*lame_from_young(2e4, 0.3), 60.0, 400.0),
                  None, False),
    "rankine": (lambda: RankineMaterial.from_young_modulus(2e4, 0.3, 30.0, 2.0), None, False),
    "mu_i": (lambda: MuIRheologyMaterial.from_young_modulus(2e4, 0.3), None, False),
    "viscoelastic": (lambda: ViscoelasticMaterial(*lame_from_young(2e4, 0.3), 4.0,
                                                  active_stress_coeff=40.0, thermal_expansion=0.02),
                     None, True),
    "granular_fluid": (lambda: GranularFluidMaterial.saturated_loam(2e4, 0.3), 1.0 * 0.25, False),
    "bingham": (lambda: BinghamFluidMaterial.medium_yield(1000.0, 1e4), 1000.0 * 0.25, False),
}


def material_zoo(sim_cls, kind, grid_res=96, seed=3, dt=0.05, gravity=-1.0, **sim_kw):
    """One model of ZOO in a grid_res^2 grid: a pre-strained 40x24 block (F0 = [[1.04, 0],
    [0.01, 0.95]], column-major x_axis (1.04, 0.01)) resting on the floor and a disk of
    radius 10 with seeded random velocities in [-4, 4)^2, both at 4 particles per cell with
    seeded jitter.  Where the model reads them, every particle gets temperature 1 and every
    other particle activation 0.5 along (1, 0.3)."""
    make, mass, active = ZOO[kind]
    cfg = SimConfig.standard(grid_res, dt, (0.0, gravity))
    t = cfg.boundary_thickness
    sim = sim_cls.empty(cfg, **sim_kw).with_default_material(make())
    a = SpawnRegion.for_sim(cfg)
    a.spacing, a.box_size = 0.5, (40, 24)
    a.box_center = (t + 4 + 20.0, t + 1 + 12.0)
    a.initial_deformation_gradient = (1.04, 0.01, 0.0, 0.95)
    a.position_jitter, a.rng_seed = 0.3, seed
    b = SpawnRegion.for_sim(cfg).disk(10.0)
    b.spacing, b.box_center = 0.5, (grid_res * 0.62, grid_res * 0.6)
    b.initial_velocity_scale = 8.0
    b.position_jitter, b.rng_seed = 0.3, seed + 1
    for s in (a, b):
        if mass is not None:
            s.mass_override = mass
        sim.add_body(s)
    if active:
        p = sim.particles()
        p["temperature"] = 1.0
        p["activation"][::2] = 0.5
        p["activation_dir"][::2] = (1.0, 0.3)
        sim.set_particles(p)
    return sim


def field_scene(sim_cls, asflip=0.0, fields=True, grid_res=96, seed=5, dt=0.05, **sim_kw):
    """Force fields and ASFLIP: a NeoHookean block (material 0) and a fluid block (material 1,
    rho0 = 1000 at 4 ppc) in a grid_res^2 grid with gravity (0, -1), every 7th particle
    pinned, and (fields=True) one field of each device kind in this order: a gravity well
    with a cutoff, buoyancy, linear drag on material 1, radial and box confinement, a
    Coulomb source charging material 0, a uniform electric field on material 1 and a
    chemotaxis ramp phi = x / grid_res.  asflip: SimConfig.asflip_blend."""
    from emerge_engine_b200 import (AabbConfinementField, BuoyancyField, ChemotaxisField,
                                    CoulombField, GravityWellField, LinearDragField,
                                    RadialConfinementField, UniformElectricField)
    cfg = SimConfig.standard(grid_res, dt, (0.0, -1.0))
    cfg.asflip_blend = asflip
    sim = (sim_cls.empty(cfg, **sim_kw)
           .with_default_material(NeoHookeanMaterial.new(400.0, 200.0))
           .with_material(1, NewtonianFluidMaterial.low_viscosity(1000.0, 1e4)))
    a = SpawnRegion.for_sim(cfg)
    a.spacing, a.box_size, a.box_center = 0.5, (24, 16), (30.0, 20.0)
    a.position_jitter, a.rng_seed, a.initial_velocity_scale = 0.3, seed, 2.0
    b = SpawnRegion.for_sim(cfg)
    b.spacing, b.box_size, b.box_center, b.material_id = 0.5, (20, 20), (grid_res * 0.65, 30.0), 1
    b.position_jitter, b.rng_seed, b.mass_override = 0.3, seed + 1, 1000.0 * 0.25
    sim.add_body(a)
    sim.add_body(b)
    p = sim.particles()
    p["pinned"][::7] = 1
    sim.set_particles(p)
    if fields:
        c = grid_res * 0.5
        chem = ChemotaxisField.new(grid_res, 0.5)
        chem.sync_from(np.repeat(np.arange(grid_res, dtype=np.float32) / grid_res, grid_res))
        for f in (GravityWellField.new([((c, c), 40.0), ((c * 0.5, c * 1.5), 15.0)], 0.5, 2.0)
                  .with_cutoff(grid_res * 0.6),
                  BuoyancyField.new(2.0, (0.0, -1.0)),
                  LinearDragField.new((0.5, 0.0), 0.8, 1 << 1),
                  RadialConfinementField.new((c, c), grid_res * 0.4, 0.3),
                  AabbConfinementField.new((8.0, 8.0), (grid_res - 8.0, grid_res * 0.6), 0.3),
                  CoulombField.new([((c, 10.0), 3.0)], {0: 0.5}, 2.0, 1.5).with_cutoff(grid_res * 0.5),
                  UniformElectricField.for_material((0.3, 0.8), 1, 60.0),
                  chem):
            sim.add_force_field(f)
    return sim


def nbody_points(n, seed=13, layout="blobs", grid_res=128):
    """Particle set for NBodyGravityField accelerations: positions and masses in reference
    index order.  layout "blobs": three Gaussian clusters of different widths; "uniform":
    uniform in the grid's interior; "clustered": 90 % of the particles within 0.05 cells of
    one point (leaves at the tree's maximum depth hold many bodies), the rest uniform;
    "duplicates": positions on a coarse lattice so that many coincide.  Masses are seeded in
    [0.1, 1]; every 11th particle has none (not a body, but still evaluated)."""
    from emerge_engine_b200.abi import PARTICLE_DTYPE
    rng = np.random.default_rng(seed)
    lo, hi = 4.0, grid_res - 4.0
    if layout == "blobs":
        centers = np.array([[0.3, 0.35], [0.7, 0.6], [0.45, 0.75]]) * grid_res
        widths = np.array([4.0, 9.0, 2.0])
        k = rng.integers(0, 3, n)
        x = centers[k] + rng.normal(size=(n, 2)) * widths[k, None]
    elif layout == "uniform":
        x = rng.uniform(lo, hi, (n, 2))
    elif layout == "clustered":
        x = rng.uniform(lo, hi, (n, 2))
        m = rng.random(n) < 0.9
        x[m] = grid_res * 0.4 + rng.uniform(-0.05, 0.05, (int(m.sum()), 2))
    elif layout == "duplicates":
        x = np.floor(rng.uniform(lo, hi, (n, 2)) / 4.0) * 4.0
    else:
        raise ValueError(layout)
    p = np.zeros(n, dtype=PARTICLE_DTYPE)
    p["x"] = np.clip(x, lo, hi).astype(np.float32)
    p["mass"] = rng.uniform(0.1, 1.0, n).astype(np.float32)
    p["mass"][::11] = 0.0
    p["f"] = np.array([1.0, 0.0, 0.0, 1.0], dtype=np.float32)
    p["initial_volume"] = 0.25
    p["volume"] = 0.25
    p["density"] = 1.0
    return p


def nbody_field(G=20.0, softening=1.0, theta=0.5, max_depth=8, max_bodies=4):
    from emerge_engine_b200 import NBodyGravityField
    f = NBodyGravityField.new(G, softening, theta)
    f.max_depth = max_depth
    f.max_bodies_per_node = max_bodies
    return f


def nbody_scene(sim_cls, grid_res=128, seed=13, dt=0.05, G=20.0, softening=1.0, theta=0.5,
                max_depth=8, max_bodies=4, pinned_every=0, scale=1, **sim_kw):
    """Self-gravitating clumps: three NeoHookean (400, 200) blocks (sides 18, 14, 10 cells,
    times `scale`) at 4 ppc with seeded jitter and initial velocities in a grid_res^2 grid
    without gravity, pulled together by NBodyGravityField(G, softening, theta) (tree shape
    max_depth, max_bodies); every pinned_every-th particle pinned (0: none)."""
    cfg = SimConfig.standard(grid_res, dt, (0.0, 0.0))
    sim = sim_cls.empty(cfg, **sim_kw).with_default_material(NeoHookeanMaterial.new(400.0, 200.0))
    for k, (cx, cy, side) in enumerate(((0.3, 0.4, 18), (0.68, 0.55, 14), (0.5, 0.75, 10))):
        s = SpawnRegion.for_sim(cfg)
        side = side * scale
        s.spacing, s.box_size, s.box_center = 0.5, (side, side), (grid_res * cx, grid_res * cy)
        s.position_jitter, s.rng_seed, s.initial_velocity_scale = 0.3, seed + k, 1.0
        sim.add_body(s)
    if pinned_every:
        p = sim.particles()
        p["pinned"][::pinned_every] = 1
        sim.set_particles(p)
    sim.add_force_field(nbody_field(G, softening, theta, max_depth, max_bodies))
    return sim


def sleep_scene(sim_cls, threshold=0.05, grid_res=96, seed=9, dt=0.05, **sim_kw):
    """Sleep partition: NeoHookean (400, 200) at 4 ppc in a grid_res^2 grid, gravity (0, -1),
    sleep_threshold `threshold`.  Tag 1: a 32 x 10 block resting on the floor (asleep after
    its first substep); tag 2: a disk of radius 6 launched at (6, -1) toward it (wakes it on
    contact); tag 3: an 8 x 8 block with activation 0.5, which never sleeps."""
    cfg = SimConfig.standard(grid_res, dt, (0.0, -1.0))
    cfg.sleep_threshold = threshold
    t = cfg.boundary_thickness
    sim = sim_cls.empty(cfg, **sim_kw).with_default_material(NeoHookeanMaterial.new(400.0, 200.0))
    a = SpawnRegion.for_sim(cfg)
    a.spacing, a.box_size, a.box_center = 0.5, (32, 10), (56.0, t + 1 + 5.0)
    a.position_jitter, a.rng_seed = 0.3, seed
    b = SpawnRegion.for_sim(cfg).disk(6.0)
    b.spacing, b.box_center, b.position_jitter, b.rng_seed = 0.5, (30.0, 14.0), 0.3, seed + 1
    c = SpawnRegion.for_sim(cfg)
    c.spacing, c.box_size, c.box_center = 0.5, (8, 8), (80.0, 50.0)
    for s in (a, b, c):
        sim.add_body(s)
    p = sim.particles()
    p["v"][p["user_tag"] == 2] = (6.0, -1.0)
    p["activation"][p["user_tag"] == 3] = 0.5
    sim.set_particles(p)
    return sim


def model_blocks(sim_cls, grid_res=1024, target_particles=4_000_000, seed=11, gravity=-1.0,
                 dt=0.05, **sim_kw):
    """The seven constitutive models beyond the core set at scale: the seeded block partition
    of mixed_granular (16-128-cell blocks, 4 ppc) with each block's material uniform over
    ZOO's Corotated, VonMises, Rankine, mu(I), Viscoelastic, GranularFluid and Bingham
    (temperature and activation left at zero)."""
    kinds = sorted(ZOO)
    cfg = SimConfig.standard(grid_res, dt, (0.0, gravity))
    sim = sim_cls.empty(cfg, **sim_kw).with_default_material(ZOO[kinds[0]][0]())
    for k in range(1, len(kinds)):
        sim = sim.with_material(k, ZOO[kinds[k]][0]())
    rng = np.random.default_rng(seed)
    for (x0, y0, w, h, _) in granular_blocks(grid_res, target_particles, seed):
        mid = int(rng.integers(len(kinds)))
        s = SpawnRegion.for_sim(cfg)
        s.spacing, s.box_size = 0.5, (w, h)
        s.box_center = (x0 + w / 2.0, y0 + h / 2.0)
        s.material_id = mid
        s.position_jitter = 0.2
        s.rng_seed = (seed * 7919 + x0 * 131 + y0) & 0xFFFFFFFF
        mass = ZOO[kinds[mid]][1]
        if mass is not None:
            s.mass_override = mass
        sim.add_body(s)
    return sim


def field_dam_break(sim_cls, grid_res=1024, column=512, asflip=0.5, **sim_kw):
    """The dam break with ASFLIP (asflip_blend 0.5) and three force fields in this order: a
    gravity well at the grid centre (G = 0.5, mass 2e4, softening 8, cutoff grid_res / 2),
    a linear drag toward (0.2, 0) on the fluid (coefficient 0.05) and a radial confinement
    of radius 0.45 grid_res (stiffness 0.5)."""
    from emerge_engine_b200 import GravityWellField, LinearDragField, RadialConfinementField
    sim = dam_break(sim_cls, grid_res=grid_res, column=column, **sim_kw)
    c = grid_res * 0.5
    for f in (GravityWellField.point((c, c), 2e4, 0.5, 8.0).with_cutoff(grid_res * 0.5),
              LinearDragField.new((0.2, 0.0), 0.05, LinearDragField.ALL_MATERIALS),
              RadialConfinementField.new((c, c), grid_res * 0.45, 0.5)):
        sim.add_force_field(f)
    return sim


def sleep_slab(sim_cls, grid_res=1024, slab=512, seed=21, threshold=0.05, **sim_kw):
    """Sleep partition at scale: a NeoHookean (400, 200) slab of slab x slab / 2 cells at
    4 ppc resting on the floor, which falls asleep after its first substep, and a disk of
    radius 40 launched into it at (12, -2), which wakes the part it reaches; sleep
    threshold `threshold`."""
    cfg = SimConfig.standard(grid_res, 0.05, (0.0, -1.0))
    cfg.asflip_blend = 0.0
    cfg.sleep_threshold = threshold
    sim = sim_cls.empty(cfg, **sim_kw).with_default_material(NeoHookeanMaterial.new(400.0, 200.0))
    t = cfg.boundary_thickness
    a = SpawnRegion.for_sim(cfg)
    a.spacing, a.box_size = 0.5, (slab, slab // 2)
    a.box_center = (grid_res - t - 4 - slab / 2.0, t + 1 + slab / 4.0)
    a.position_jitter, a.rng_seed = 0.3, seed
    b = SpawnRegion.for_sim(cfg).disk(40.0)
    b.spacing, b.box_center = 0.5, (grid_res - t - 8 - slab - 48.0, t + 60.0)
    b.position_jitter, b.rng_seed = 0.3, seed + 1
    sim.add_body(a)
    tag = sim.add_body(b)
    p = sim.particles()
    p["v"][p["user_tag"] == tag] = (12.0, -2.0)
    sim.set_particles(p)
    return sim


def contact_scene(sim_cls, grid_res=96, seed=13, dt=0.05, friction=0.5, grip=None, asflip=0.0,
                  sleep=0.0, **sim_kw):
    """Multi-field contact: a NeoHookean (400, 200) slab on the floor (contact group 0) and a
    block of the same material with contact_group 1 falling onto it at (1.5, -3), 4 ppc,
    SimConfig.contact_friction `friction`, optional DirectionalContactGrip `grip`,
    SimConfig.asflip_blend `asflip`, SimConfig.sleep_threshold `sleep`."""
    cfg = SimConfig.standard(grid_res, dt, (0.0, -1.0))
    cfg.contact_friction = friction
    cfg.asflip_blend = asflip
    cfg.sleep_threshold = sleep
    t = cfg.boundary_thickness
    sim = sim_cls.empty(cfg, **sim_kw).with_default_material(NeoHookeanMaterial.new(400.0, 200.0))
    if grip is not None:
        sim.set_contact_grip(grip)
    a = SpawnRegion.for_sim(cfg)
    a.spacing, a.box_size, a.box_center = 0.5, (48, 12), (grid_res / 2.0, t + 1 + 6.0)
    a.position_jitter, a.rng_seed = 0.3, seed
    b = SpawnRegion.for_sim(cfg)
    b.spacing, b.box_size, b.box_center = 0.5, (14, 10), (grid_res / 2.0 - 6.0, t + 1 + 12 + 6.0)
    b.position_jitter, b.rng_seed = 0.3, seed + 1
    sim.add_body(a)
    tag = sim.add_body(b)
    p = sim.particles()
    g = p["user_tag"] == tag
    p["contact_group"][g] = 1
    p["v"][g] = (1.5, -3.0)
    sim.set_particles(p)
    return sim


def mixture_scene(sim_cls, grid_res=96, seed=17, dt=0.05, drag=5.0, iterations=2, **sim_kw):
    """Two-phase mixture: a DruckerPrager sand block (solid phase, 1e5 / 0.3, 4 ppc at 1600)
    on the floor with a block of water (NewtonianFluid 1000 / 1e4, fluid phase, 4 ppc at
    rho0) resting on part of it, mixture_drag_coefficient `drag`,
    mixture_pressure_iterations `iterations`."""
    from emerge_engine_b200 import FLUID_PHASE, SOLID_PHASE, WithMixturePhase
    cfg = SimConfig.standard(grid_res, dt, (0.0, -1.0))
    cfg.mixture_drag_coefficient = drag
    cfg.mixture_pressure_iterations = iterations
    t = cfg.boundary_thickness
    sim = (sim_cls.empty(cfg, **sim_kw)
           .with_default_material(WithMixturePhase(DruckerPragerMaterial.cohesionless(1e5, 0.3),
                                                   SOLID_PHASE))
           .with_material(1, WithMixturePhase(NewtonianFluidMaterial.low_viscosity(1000.0, 1e4),
                                              FLUID_PHASE)))
    a = SpawnRegion.for_sim(cfg)
    a.spacing, a.box_size, a.box_center = 0.5, (40, 16), (grid_res / 2.0, t + 1 + 8.0)
    a.position_jitter, a.rng_seed, a.mass_override = 0.3, seed, 1600.0 * 0.25
    b = SpawnRegion.for_sim(cfg)
    b.spacing, b.box_size, b.material_id = 0.5, (20, 10), 1
    b.box_center = (grid_res / 2.0 - 8.0, t + 1 + 16 + 5.0)
    b.position_jitter, b.rng_seed, b.mass_override = 0.3, seed + 1, 1000.0 * 0.25
    sim.add_body(a)
    sim.add_body(b)
    return sim


def contact_slab(sim_cls, grid_res=1024, slab=(896, 192), block=(320, 256), seed=23, **sim_kw):
    """Multi-field contact at scale: a NeoHookean (400, 200) slab of `slab` cells at 4 ppc on
    the floor and a grip block (contact_group 1) of `block` cells on top of it, thrown at
    (1.5, -3), with DirectionalContactGrip(0.1, 0.9, (1, 0)); the two touch from the start."""
    from emerge_engine_b200 import DirectionalContactGrip
    cfg = SimConfig.standard(grid_res, 0.05, (0.0, -1.0))
    t = cfg.boundary_thickness
    sim = sim_cls.empty(cfg, **sim_kw).with_default_material(NeoHookeanMaterial.new(400.0, 200.0))
    sim.set_contact_grip(DirectionalContactGrip(0.1, 0.9, (1.0, 0.0)))
    a = SpawnRegion.for_sim(cfg)
    a.spacing, a.box_size = 0.5, slab
    a.box_center = (grid_res / 2.0, t + 1 + slab[1] / 2.0)
    a.position_jitter, a.rng_seed = 0.3, seed
    b = SpawnRegion.for_sim(cfg)
    b.spacing, b.box_size = 0.5, block
    b.box_center = (grid_res / 2.0 - block[0] / 4.0, t + 1 + slab[1] + block[1] / 2.0 + 0.5)
    b.position_jitter, b.rng_seed = 0.3, seed + 1
    sim.add_body(a)
    tag = sim.add_body(b)
    p = sim.particles()
    g = p["user_tag"] == tag
    p["contact_group"][g] = 1
    p["v"][g] = (1.5, -3.0)
    sim.set_particles(p)
    return sim


def mixture_overlap(sim_cls, grid_res=1024, side=362, seed=29, drag=5.0, iterations=2, **sim_kw):
    """Two-phase mixture at scale, without gravity (the reference's two-phase drag test,
    tests/solver.rs:1888-1990, at scale): a DruckerPrager sand square (1e5 / 0.3, solid phase)
    and a water square (NewtonianFluid 1000 / 1e4, fluid phase), `side` cells at 4 ppc each,
    overlapping in the middle of the domain, the water moving through the sand at (0, -3);
    particle masses of 125 give the overlap the water's rest density.
    mixture_drag_coefficient `drag`, mixture_pressure_iterations `iterations`."""
    from emerge_engine_b200 import FLUID_PHASE, SOLID_PHASE, WithMixturePhase
    cfg = SimConfig.standard(grid_res, 0.05, (0.0, 0.0))
    cfg.mixture_drag_coefficient = drag
    cfg.mixture_pressure_iterations = iterations
    sim = (sim_cls.empty(cfg, **sim_kw)
           .with_default_material(WithMixturePhase(DruckerPragerMaterial.cohesionless(1e5, 0.3),
                                                   SOLID_PHASE))
           .with_material(1, WithMixturePhase(NewtonianFluidMaterial.low_viscosity(1000.0, 1e4),
                                              FLUID_PHASE)))
    tags = []
    for k in range(2):
        s = SpawnRegion.for_sim(cfg)
        s.spacing, s.box_size, s.material_id = 0.5, (side, side), k
        s.box_center = (grid_res / 2.0, grid_res / 2.0)
        s.position_jitter, s.rng_seed, s.mass_override = 0.3, seed + k, 125.0
        tags.append(sim.add_body(s))
    p = sim.particles()
    p["v"][p["user_tag"] == tags[1]] = (0.0, -3.0)
    sim.set_particles(p)
    return sim


def region_stats64(particles, center, radius):
    """BodyState statistics (spacetime/solver/query.rs:109-142) of the particles with
    |x - center|^2 <= radius^2, summed in float64 from a particle array.  Two bit-identical
    particle sets give identical values, unlike the reference's f32 running sums, whose
    rounding (~1e-5 relative over 1e5 particles) depends on the iteration order."""
    x = particles["x"].astype(np.float64)
    c = np.asarray(center, dtype=np.float64)
    sel = ((x - c) ** 2).sum(1) <= float(radius) ** 2
    p = particles[sel]
    n = int(sel.sum())
    if n == 0:
        return dict(count=0)
    f = p["f"].astype(np.float64)
    det = f[:, 0] * f[:, 3] - f[:, 2] * f[:, 1]
    jp = p["plastic_volume_ratio"].astype(np.float64)
    return dict(count=n, avg_volume_ratio=float(jp.mean()), max_volume_ratio=float(jp.max()),
                avg_speed=float(np.linalg.norm(p["v"].astype(np.float64), axis=1).mean()),
                avg_det_f=float(det.mean()), avg_density=float(p["density"].astype(np.float64).mean()),
                centroid=[float(v) for v in x[sel].mean(0)])
