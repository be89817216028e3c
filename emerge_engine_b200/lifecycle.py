"""Particle-set edits of the reference `Simulation` that take a host predicate
(solver/particles.rs:177-205, solver/lifecycle.rs:237-310), restated on the reference-order
particle array (structured numpy array of `emerge_particle`).  Each returns the new array
and the new active-zone size; the simulation then replaces its particle set.  Shared by the
CUDA `Simulation` and the oracle so both apply the same edits.
"""
from __future__ import annotations

import numpy as np

from .abi import PARTICLE_DTYPE, Particle

f32 = np.float32


def as_particle(row) -> Particle:
    """One structured-array row as the `Particle` struct the predicates receive."""
    return Particle.from_buffer_copy(np.ascontiguousarray(row).tobytes())


def _swap(p: np.ndarray, a: int, b: int) -> None:
    if a != b:
        t = p[a].copy()
        p[a] = p[b]
        p[b] = t


def remove_particles(p: np.ndarray, active: int, predicate) -> tuple:
    """remove_particles (particles.rs:177-205): stable retain of the particles the predicate
    rejects, then the swap partition that moves sleeping particles to the back.
    Returns (particles, active_count, removed)."""
    keep = np.array([not predicate(as_particle(r)) for r in p], dtype=bool)
    out = p[keep].copy()
    removed = len(p) - len(out)
    if removed == 0:
        return p, active, 0
    write = 0
    for read in range(len(out)):
        if not out["sleeping"][read]:
            _swap(out, write, read)
            write += 1
    return out, write, removed


def retain_particles(p: np.ndarray, active: int, predicate) -> tuple:
    """retain_particles (lifecycle.rs:237-253): stable retain; every survivor is in the
    active zone afterwards (active_count = new length)."""
    keep = np.array([bool(predicate(as_particle(r))) for r in p], dtype=bool)
    out = p[keep].copy()
    return out, len(out)


class _Lcg:
    """LcgRng (solver/mod.rs:154-175)."""

    def __init__(self, seed: int):
        self.state = seed & 0xFFFFFFFF

    def next_f32(self) -> np.float32:
        self.state = (self.state * 1664525 + 1013904223) & 0xFFFFFFFF
        return f32(f32(self.state) / f32(4294967296.0))


def split_particles(p: np.ndarray, active: int, should_split, jitter: float) -> tuple:
    """split_particles (lifecycle.rs:271-310): every active particle the predicate selects
    becomes two awake children with half mass and volumes, jittered by LcgRng(0xC0FFEE11)
    draws in [-jitter, jitter); sleeping particles follow unchanged."""
    rng = _Lcg(0xC0FFEE11)
    jit = f32(jitter)
    rows = []
    for i in range(active):
        r = p[i]
        if should_split(as_particle(r)):
            for _ in range(2):
                c = r.copy()
                c["mass"] = f32(c["mass"] * f32(0.5))
                c["initial_volume"] = f32(c["initial_volume"] * f32(0.5))
                c["volume"] = f32(c["volume"] * f32(0.5))
                jx = f32(f32(f32(rng.next_f32() - f32(0.5)) * f32(2.0)) * jit)
                jy = f32(f32(f32(rng.next_f32() - f32(0.5)) * f32(2.0)) * jit)
                c["x"][0] = f32(c["x"][0] + jx)
                c["x"][1] = f32(c["x"][1] + jy)
                c["sleeping"] = 0
                rows.append(c)
        else:
            rows.append(r.copy())
    n_active = len(rows)
    rows += [p[i].copy() for i in range(active, len(p))]
    out = np.array(rows, dtype=PARTICLE_DTYPE) if rows else np.zeros(0, dtype=PARTICLE_DTYPE)
    return out, n_active


def wake_tag(p: np.ndarray, active: int, tag: int) -> tuple:
    """wake_tag (particles.rs:271-290): the tag's sleeping particles, in ascending index
    order, each swapped with the first sleeping particle (wake_particle, :252-268)."""
    p = p.copy()
    for i in [k for k in range(len(p)) if p["user_tag"][k] == tag and p["sleeping"][k]]:
        if not p["sleeping"][i]:
            continue
        p["sleeping"][i] = 0
        _swap(p, i, active)
        active += 1
    return p, active


def sleep_tag(p: np.ndarray, active: int, tag: int) -> tuple:
    """sleep_tag (particles.rs:292-312): the tag's awake particles, in descending index order,
    each swapped with the last active particle (sleep_particle, :227-245)."""
    p = p.copy()
    for i in sorted((k for k in range(len(p)) if p["user_tag"][k] == tag and not p["sleeping"][k]),
                    reverse=True):
        if p["sleeping"][i] or active == 0:
            continue
        p["sleeping"][i] = 1
        _swap(p, i, active - 1)
        active -= 1
    return p, active
