"""Pins the CPU oracle of the learned closure: analytic MLP gradients against central
finite differences (float64), Adam against its closed form after one step, the bfloat16
rounding, and the Drucker-Prager smooth branch against the C++ oracle's return mapping
(DruckerPragerMaterial::project, sand.rs:156-194)."""
import ctypes

import numpy as np
import pytest

from oracle import closure_oracle as co


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    p = co.init_params(5, dtype=np.float64)
    x = rng.normal(size=(7, co.IN))
    t = rng.normal(size=(7, co.OUT))
    _, g = co.loss_and_grad(p, x, t)
    idx = rng.choice(co.NPARAMS, size=120, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        fd = (co.loss_and_grad(p + e, x, t)[0] - co.loss_and_grad(p - e, x, t)[0]) / (2 * h)
        assert g[i] == pytest.approx(fd, rel=1e-5, abs=1e-9)


def test_adam_first_step_is_lr_sign():
    # with m = v = 0 the bias-corrected first step is lr * g / (|g| + eps') = lr * sign(g)
    g = np.array([0.5, -2.0, 1e-3, 0.0])
    p, m, v = co.adam_step(np.zeros(4), np.zeros(4), np.zeros(4), g, 1, lr=0.01, eps=1e-30)
    np.testing.assert_allclose(p[:3], -0.01 * np.sign(g[:3]), rtol=1e-12)
    assert p[3] == 0.0


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0, 1e-30], np.float32)
    r = co.to_bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie rounds to even
    assert r[2] == np.float32(1.0078125)
    bits = r.view(np.uint32)
    assert np.all(bits & 0xFFFF == 0)
    assert abs(r[3] - x[3]) <= abs(x[3]) * 2.0 ** -8


def test_dp_smooth_branch_matches_oracle_return_mapping(oracle_lib):
    """Targets computed from the network inputs agree with the oracle's dp_project."""
    from oracle.oracle import oracle_material
    from emerge_engine_b200 import DruckerPragerMaterial
    L = oracle_lib
    mat = DruckerPragerMaterial.cohesionless(1e5, 0.2)
    mc = oracle_material(mat)
    pm = mat.params()
    f32 = np.float32
    rng = np.random.default_rng(11)
    lam, mu = f32(mat.lambda_), f32(mat.mu)
    hits = 0
    for _ in range(400):
        sigma = rng.uniform(0.9, 1.1, size=2).astype(np.float32)
        lvs = f32(rng.uniform(-0.05, 0.05))
        q = f32(rng.uniform(0, 0.5))
        out = (ctypes.c_float * 2)()
        dq = ctypes.c_float()
        proj = L.oracle_dp_project(ctypes.byref(mc), (ctypes.c_float * 2)(*sigma), float(lvs),
                                   float(q), out, ctypes.byref(dq))
        eps = np.log(sigma) + lvs * f32(0.5)
        # alpha(q) (sand.rs:135) in f32
        phi = f32(pm.dp_h0) + (f32(pm.dp_h1) * q - f32(pm.dp_h3)) * np.exp(-f32(pm.dp_h2) * q)
        s = np.sin(f32(phi))
        alpha = f32(np.sqrt(f32(2.0) / f32(3.0))) * (f32(2.0) * s) / (f32(3.0) - s)
        x = co.dp_features(eps[None, :], alpha, (lam + mu) / mu, f32(mat.cohesion) / (f32(2) * mu))
        tgt, on = co.dp_smooth_targets(x)
        s = np.exp(x[0, 5])
        if on[0]:
            hits += 1
            assert proj == 1
            np.testing.assert_allclose(np.exp(tgt[0, :2] * s), np.array(out[:2]), rtol=1e-5)
            assert tgt[0, 2] * s == pytest.approx(dq.value, rel=1e-4, abs=1e-6)
    assert hits > 20
