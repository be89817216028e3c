"""Generates tests/golden/region_100_steps.json: the oracle's state statistics after 10 and
100 frames (Simulation::step calls) of two seeded scenes, for the check that region_state
statistics agree within 1e-3 after 100 steps.

    python tests/golden/make_region_100.py

Scenes (tests/scenes.py): the dam break at 262,144 particles (256 x 256-cell column on a
512^2 grid) and the mixed granular scene on a 256^2 grid (~160k particles of DruckerPrager
sand, Stomakhin snow and NACC soil).  The oracle runs with correctly rounded exp / log / pow /
sin / sinh (oracle_set_correctly_rounded), which is what the device's reference-order mode
evaluates, so that mode can be held to a tight bar; the fast path is held to 1e-3.
Recorded per checkpoint: the substeps of every frame, total mass and momentum (f64 sums
over particles), the sum of |m v| (the momentum scale), the oracle's region_state for three
regions (f32 running sums, as the reference), the same statistics summed in f64 from the
particle array (tests/scenes.py region_stats64), and a SHA-256 of the particle array.
A second oracle run feeds the same particles in a shuffled index order (the reference sums
P2G contributions in particle order, transfer/p2g.rs:16-23): its f64 statistics measure how
far the reference itself moves under a change of summation order after 10 and 100 frames.
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import OracleSimulation, correctly_rounded_math  # noqa: E402
from tests import scenes  # noqa: E402

SCENES = {
    "dam_break_262k": dict(builder=lambda cls: scenes.dam_break(cls, grid_res=512, column=256),
                           regions={"domain": ((256.0, 256.0), 400.0), "corner": ((64.0, 64.0), 48.0),
                                    "floor": ((200.0, 40.0), 40.0)}),
    "granular_256": dict(builder=lambda cls: scenes.mixed_granular(cls, grid_res=256,
                                                                   target_particles=120_000),
                         regions={"domain": ((128.0, 128.0), 200.0), "left": ((64.0, 64.0), 40.0),
                                  "right": ((180.0, 90.0), 30.0)}),
}
CHECKPOINTS = (10, 100)


def summary(sim, regions, perm=None):
    p = sim.particles()
    if perm is not None:  # back to the original index order
        inv = np.empty_like(perm)
        inv[perm] = np.arange(len(perm))
        p = p[inv]
    m = p["mass"].astype(np.float64)
    v = p["v"].astype(np.float64)
    out = {"particles": int(len(p)), "mass": float(m.sum()),
           "momentum": [float(x) for x in (m[:, None] * v).sum(0)],
           "momentum_scale": float((m * np.linalg.norm(v, axis=1)).sum()),
           "sha256": hashlib.sha256(np.ascontiguousarray(p).tobytes()).hexdigest(),
           "regions": {}, "stats64": {}}
    for key, (c, r) in regions.items():
        out["stats64"][key] = scenes.region_stats64(p, c, r)
        if perm is not None:
            continue
        b = sim.region_state(c, r)
        out["regions"][key] = dict(center=list(c), radius=r, count=int(b.count),
                                   avg_volume_ratio=b.avg_volume_ratio,
                                   max_volume_ratio=b.max_volume_ratio, avg_speed=b.avg_speed,
                                   avg_det_f=b.avg_det_f, avg_density=b.avg_density,
                                   centroid=list(b.centroid))
    return out


def run(spec, perm_seed=None):
    sim = spec["builder"](OracleSimulation)
    perm = None
    if perm_seed is not None:
        p = sim.particles()
        perm = np.random.default_rng(perm_seed).permutation(len(p))
        sim.set_particles(p[perm])
    subs, rec = [], {}
    for frame in range(1, max(CHECKPOINTS) + 1):
        sim.step()
        subs.append(int(sim.last_substeps()))
        if frame in CHECKPOINTS:
            rec[str(frame)] = summary(sim, spec["regions"], perm)
    return subs, rec


def main():
    data = {"math": "correctly rounded exp/log/pow/sin/sinh (oracle_set_correctly_rounded)"}
    with correctly_rounded_math():
        for name, spec in SCENES.items():
            t0 = time.time()
            subs, rec = run(spec)
            subs_r, rec_r = run(spec, perm_seed=1)
            data[name] = {"substeps": subs, "checkpoints": rec,
                          "reordered": {"substeps": subs_r,
                                        "checkpoints": {k: {"stats64": v["stats64"],
                                                            "momentum": v["momentum"]}
                                                        for k, v in rec_r.items()}},
                          "oracle_seconds": time.time() - t0}
            print(name, f"{time.time() - t0:.0f} s", flush=True)
    with open(os.path.join(HERE, "region_100_steps.json"), "w") as f:
        json.dump(data, f, indent=1)


if __name__ == "__main__":
    main()
