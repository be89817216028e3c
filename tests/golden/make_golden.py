"""Generates the golden fixtures in this directory from the CPU oracle.

    python tests/golden/make_golden.py

The reference crate (Rust) cannot be built in this environment and ships no golden
trajectories, so these fixtures record the oracle (a restatement of the reference CPU step,
pinned by the reference's known-answer tests) on seeded scenes:
  quickstart_step1.npz / quickstart_step60.npz  -- full particle state of the README scene
  dam_break_128_step1.npz                        -- every 16th particle of 16384
  granular_256_region.json                       -- region_state after one frame
  granular_256_substep1.npz                      -- every 32nd particle after one substep
                                                    (frame dt = 1e-3, below the CFL bound)
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import OracleSimulation  # noqa: E402
from tests import scenes  # noqa: E402


def save(name, arr):
    np.savez_compressed(os.path.join(HERE, name), particles=arr.view(np.uint8))


def main():
    sim = scenes.quickstart(OracleSimulation)
    sim.step()
    save("quickstart_step1.npz", sim.particles())
    sim.step_n(59)
    save("quickstart_step60.npz", sim.particles())
    sim = scenes.dam_break(OracleSimulation, grid_res=128, column=64)
    sim.step()
    save("dam_break_128_step1.npz", sim.particles()[::16].copy())
    sim = scenes.mixed_granular(OracleSimulation, grid_res=256, target_particles=120_000)
    sim.step()
    out = {}
    for key, (c, r) in {"center": ((128.0, 128.0), 200.0), "left": ((64.0, 64.0), 40.0)}.items():
        b = sim.region_state(c, r)
        out[key] = dict(center=c, radius=r, count=b.count, avg_volume_ratio=b.avg_volume_ratio,
                        max_volume_ratio=b.max_volume_ratio, avg_speed=b.avg_speed,
                        avg_det_f=b.avg_det_f, avg_density=b.avg_density, centroid=b.centroid,
                        substeps=sim.last_substeps())
    with open(os.path.join(HERE, "granular_256_region.json"), "w") as f:
        json.dump(out, f, indent=1)
    sim = scenes.mixed_granular(OracleSimulation, grid_res=256, target_particles=120_000, dt=1e-3)
    sim.step()
    assert sim.last_substeps() == 1
    save("granular_256_substep1.npz", sim.particles()[::32].copy())


if __name__ == "__main__":
    main()
