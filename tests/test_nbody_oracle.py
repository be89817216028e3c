"""NBodyGravityField on the CPU: the oracle's Barnes-Hut restatement (oracle/emerge_oracle.cpp)
against a second, independent restatement in Python float32 arithmetic below (the same
algorithm, n_body.rs:63-283, written as the reference's own recursive insertion), bit for bit;
against closed forms (two bodies, the direct O(N^2) sum when no node is far); and the
reference's orbit-helper tests (n_body.rs:431-455)."""
import math

import numpy as np
import pytest

from emerge_engine_b200 import NBodyGravityField, SimConfig, orbit
from oracle.oracle import OracleSimulation
from tests import scenes

f32 = np.float32


class _Node:
    """Node of n_body.rs:110-214, every operation in float32."""

    def __init__(self, center, half, depth):
        self.center, self.half, self.depth = center, half, depth
        self.mass, self.com = f32(0.0), (f32(0.0), f32(0.0))
        self.bodies = []
        self.children = None

    def quadrant(self, p):
        return int(p[0] >= self.center[0]) | (int(p[1] < self.center[1]) << 1)

    def insert(self, b, pos, mass, max_depth, max_bodies):
        nt = f32(self.mass + mass[b])
        if nt > 0:
            self.com = (f32(f32(f32(self.com[0] * self.mass) + f32(pos[b][0] * mass[b])) / nt),
                        f32(f32(f32(self.com[1] * self.mass) + f32(pos[b][1] * mass[b])) / nt))
            self.mass = nt
        if self.depth >= max_depth or (len(self.bodies) < max_bodies and self.children is None):
            self.bodies.append(b)
            return
        if self.children is None:
            q = f32(self.half * f32(0.5))
            self.children = [_Node((f32(self.center[0] + (q if k & 1 else -q)),
                                    f32(self.center[1] + (-q if k & 2 else q))), q, self.depth + 1)
                             for k in range(4)]
            old, self.bodies = self.bodies, []
            for e in old:
                self.children[self.quadrant(pos[e])].insert(e, pos, mass, max_depth, max_bodies)
        self.children[self.quadrant(pos[b])].insert(b, pos, mass, max_depth, max_bodies)

    def accel(self, idx, p, pos, mass, index, g, soft, theta):
        eps2 = f32(soft * soft)
        dx, dy = f32(p[0] - self.center[0]), f32(p[1] - self.center[1])
        dist = f32(np.sqrt(f32(f32(dx * dx) + f32(dy * dy))))
        if not (dist < soft or self.mass <= 0) and f32(f32(self.half * f32(2.0)) / dist) < theta:
            return _pull(f32(self.com[0] - p[0]), f32(self.com[1] - p[1]), self.mass, g, eps2)
        total = (f32(0.0), f32(0.0))
        if self.children is None:
            for b in self.bodies:
                if index[b] == idx:
                    continue
                rx, ry = f32(pos[b][0] - p[0]), f32(pos[b][1] - p[1])
                if f32(f32(rx * rx) + f32(ry * ry)) < eps2:
                    continue
                a = _pull(rx, ry, mass[b], g, eps2)
                total = (f32(total[0] + a[0]), f32(total[1] + a[1]))
            return total
        for c in self.children:
            a = c.accel(idx, p, pos, mass, index, g, soft, theta)
            total = (f32(total[0] + a[0]), f32(total[1] + a[1]))
        return total


def _pull(rx, ry, m, g, eps2):
    ns = f32(f32(f32(rx * rx) + f32(ry * ry)) + eps2)
    with np.errstate(all="ignore"):
        scale = f32(f32(g * m) / f32(ns * f32(np.sqrt(ns))))
    if not np.isfinite(scale):
        return f32(0.0), f32(0.0)
    return f32(rx * scale), f32(ry * scale)


def python_accelerations(p, g, soft, theta, max_depth=8, max_bodies=4):
    """Field::acceleration of NBodyGravityField for every particle (prepare + acceleration)."""
    g, soft, theta = f32(g), f32(soft), f32(theta)
    x = p["x"].astype(np.float32)
    sel = [i for i in range(len(p)) if p["mass"][i] > 0]
    pos = [(x[i, 0], x[i, 1]) for i in sel]
    mass = [p["mass"][i] for i in sel]
    if not sel:
        root = _Node((f32(0.0), f32(0.0)), f32(1000.0), 0)
    else:
        mn_x = min(q[0] for q in pos)
        mn_y = min(q[1] for q in pos)
        mx_x = max(q[0] for q in pos)
        mx_y = max(q[1] for q in pos)
        pad = f32(f32(f32(f32(mx_x - mn_x) + f32(mx_y - mn_y)) * f32(0.1)) + f32(1.0))
        mn_x, mn_y, mx_x, mx_y = f32(mn_x - pad), f32(mn_y - pad), f32(mx_x + pad), f32(mx_y + pad)
        root = _Node((f32(f32(mn_x + mx_x) * f32(0.5)), f32(f32(mn_y + mx_y) * f32(0.5))),
                     f32(max(f32(mx_x - mn_x), f32(mx_y - mn_y)) * f32(0.5)), 0)
        for b in range(len(sel)):
            root.insert(b, pos, mass, max_depth, max_bodies)
    out = np.zeros((len(p), 2), dtype=np.float32)
    for i in range(len(p)):
        out[i] = root.accel(i, (x[i, 0], x[i, 1]), pos, mass, sel, g, soft, theta)
    return out


def oracle_with(p, field, grid_res=128):
    sim = OracleSimulation.empty(SimConfig.standard(grid_res, 0.05, (0.0, 0.0)))
    sim.add_particles(p)
    sim.add_force_field(field)
    return sim


@pytest.mark.parametrize("layout,n,g,soft,theta,depth,maxb", [
    ("blobs", 300, 20.0, 1.0, 0.5, 8, 4),
    ("uniform", 250, 5.0, 0.5, 1.0, 8, 4),
    ("blobs", 200, 20.0, 2.0, 0.3, 3, 1),
    ("clustered", 220, 10.0, 0.01, 0.7, 4, 2),
    ("duplicates", 260, 1.0, 1.0, 0.5, 8, 0),
    ("uniform", 120, 3.0, 0.5, 0.5, 0, 4),
])
def test_oracle_tree_matches_the_python_restatement_bit_for_bit(layout, n, g, soft, theta, depth, maxb):
    p = scenes.nbody_points(n, seed=n + depth, layout=layout)
    field = scenes.nbody_field(g, soft, theta, depth, maxb)
    got = oracle_with(p, field).field_accelerations()
    want = python_accelerations(p, g, soft, theta, depth, maxb)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


def test_two_bodies_pull_by_the_plummer_law():
    p = scenes.nbody_points(2, layout="uniform")
    p["mass"] = [2.0, 3.0]
    p["x"] = [[40.0, 50.0], [43.0, 54.0]]
    a = oracle_with(p, scenes.nbody_field(G=7.0, softening=0.5, theta=0.5)).field_accelerations()
    r = np.array([3.0, 4.0])
    s = 7.0 / (25.0 + 0.25) ** 1.5
    np.testing.assert_allclose(a[0], 3.0 * s * r, rtol=1e-6)
    np.testing.assert_allclose(a[1], -2.0 * s * r, rtol=1e-6)


def test_no_far_node_gives_the_direct_sum():
    """theta far below any width/distance ratio: every pair is summed directly."""
    p = scenes.nbody_points(400, seed=3, layout="blobs")
    g, soft = 5.0, 0.7
    a = oracle_with(p, scenes.nbody_field(G=g, softening=soft, theta=1e-6)).field_accelerations()
    x, m = p["x"].astype(np.float64), p["mass"].astype(np.float64)
    d = x[None, :, :] - x[:, None, :]
    r2 = (d ** 2).sum(-1)
    ns = r2 + soft * soft
    w = np.where((r2 >= soft * soft) & (m[None, :] > 0), g * m[None, :] / ns ** 1.5, 0.0)
    np.fill_diagonal(w, 0.0)
    want = (w[:, :, None] * d).sum(1)
    np.testing.assert_allclose(a, want, rtol=2e-5, atol=1e-6 * np.abs(want).max())


def test_barnes_hut_approximates_the_direct_sum():
    """Monopole nodes opened by box width over distance to the box center (the reference's
    criterion): median error 0.4 %, worst 22 % of the RMS acceleration on this set."""
    p = scenes.nbody_points(600, seed=4, layout="blobs")
    exact = oracle_with(p, scenes.nbody_field(theta=1e-6)).field_accelerations().astype(np.float64)
    bh = oracle_with(p, scenes.nbody_field(theta=0.5)).field_accelerations().astype(np.float64)
    rms = np.sqrt((np.linalg.norm(exact, axis=1) ** 2).mean())
    err = np.linalg.norm(bh - exact, axis=1) / rms
    assert np.median(err) < 1e-2 and err.max() < 0.3


def test_empty_and_massless_sets_pull_nothing():
    p = scenes.nbody_points(30, layout="uniform")
    p["mass"] = 0.0
    a = oracle_with(p, scenes.nbody_field()).field_accelerations()
    assert np.all(a == 0.0)


def test_theta_is_validated():
    for bad in (0.0, -0.5, 1.5, float("nan")):
        with pytest.raises(ValueError):
            NBodyGravityField.new(1.0, 1.0, bad)
    NBodyGravityField.new(1.0, 1.0, 1.0)


# n_body.rs:431-455
def test_orbit_escape_is_sqrt2_times_circular():
    vc = orbit.circular_velocity(1.0, 100.0, 10.0)
    ve = orbit.escape_velocity(1.0, 100.0, 10.0)
    assert abs(ve / vc - math.sqrt(2.0)) < 1e-5


def test_orbit_circular_is_a_zero_eccentricity_ellipse():
    vc = orbit.circular_velocity(0.5, 200.0, 25.0)
    ve = orbit.elliptical_velocity(0.5, 200.0, 25.0, 0.0, True)
    assert abs(vc - ve) < 1e-4


def test_orbit_zero_radius_is_safe():
    assert orbit.circular_velocity(1.0, 1.0, 0.0) == 0.0
    assert orbit.escape_velocity(1.0, 1.0, 0.0) == 0.0
    assert orbit.circular_velocity_softened(1.0, 1.0, 0.0, 0.0) == 0.0
    r, e = 5.0, 1.0
    assert orbit.circular_velocity_softened(2.0, 3.0, r, e) == pytest.approx(
        r * math.sqrt(2.0 * 3.0 / (r * r + e * e) ** 1.5), rel=1e-6)
