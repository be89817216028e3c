"""CPU oracle of the learned closure (test infrastructure only; nothing in the product
imports it).

Restates in numpy what the device closure computes, so the device kernels can be checked:
  * the MLP 6 -> 64 -> 64 -> 64 -> 3 with SiLU hidden layers, its MSE loss and gradients
    (plain reverse-mode differentiation, FP32), checked here against central finite
    differences in float64;
  * Adam with bias correction (Kingma & Ba 2015, Algorithm 1);
  * the BF16 tensor-core inference: weights and hidden activations rounded to bfloat16
    (round to nearest even), FP32 accumulation;
  * the smooth plastic branch of the Drucker-Prager return mapping
    (DruckerPragerMaterial::project, sand.rs:156-194) from the network's inputs, to check
    logged (input, target) pairs;
  * the relative error of the principal Kirchhoff stress the closure is judged by
    (sand.rs:220-231 and nacc.rs:236-249 in principal axes, scale-free).

Parameter layout (FP32, 8963 values): W1[6][64] b1[64] W2[64][64] b2[64] W3[64][64] b3[64]
W4[64][3] b4[3], W[k][n] with k the input index.
"""
from __future__ import annotations

import numpy as np

IN, H, OUT = 6, 64, 3
SHAPES = [("W1", (IN, H)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)),
          ("b3", (H,)), ("W4", (H, OUT)), ("b4", (OUT,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(p):
    out, off = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = p[off:off + n].reshape(shape)
        off += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name]).reshape(-1) for name, _ in SHAPES])


def init_params(seed, dtype=np.float32):
    rng = np.random.default_rng(seed)
    d = {}
    for name, shape in SHAPES:
        if name.startswith("W"):
            a = np.sqrt(6.0 / (shape[0] + shape[1]))
            d[name] = rng.uniform(-a, a, size=shape)
        else:
            d[name] = rng.normal(0.0, 0.1, size=shape)
    return pack(d).astype(dtype)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, x):
    w = unpack(p)
    z1 = x @ w["W1"] + w["b1"]
    a1 = silu(z1)
    z2 = a1 @ w["W2"] + w["b2"]
    a2 = silu(z2)
    z3 = a2 @ w["W3"] + w["b3"]
    a3 = silu(z3)
    y = a3 @ w["W4"] + w["b4"]
    return y, (z1, a1, z2, a2, z3, a3)


def loss_and_grad(p, x, t):
    """MSE over all outputs of the batch, and its gradient w.r.t. the parameters."""
    w = unpack(p)
    y, (z1, a1, z2, a2, z3, a3) = forward(p, x)
    n = y.size
    loss = np.sum((y - t) ** 2) / n
    dy = 2.0 * (y - t) / n
    g = {"W4": a3.T @ dy, "b4": dy.sum(0)}
    d3 = (dy @ w["W4"].T) * dsilu(z3)
    g["W3"], g["b3"] = a2.T @ d3, d3.sum(0)
    d2 = (d3 @ w["W3"].T) * dsilu(z2)
    g["W2"], g["b2"] = a1.T @ d2, d2.sum(0)
    d1 = (d2 @ w["W2"].T) * dsilu(z1)
    g["W1"], g["b1"] = x.T @ d1, d1.sum(0)
    return loss, pack(g)


def adam_step(p, m, v, g, step, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    m = beta1 * m + (1.0 - beta1) * g
    v = beta2 * v + (1.0 - beta2) * g * g
    mh = m / (1.0 - beta1 ** step)
    vh = v / (1.0 - beta2 ** step)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v


def to_bf16(a):
    """Rounds float32 values to bfloat16 (round to nearest even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = rounded.astype(np.uint32).view(np.float32)
    return np.where(np.isfinite(a), out, a)


def forward_bf16(p, x):
    """The tensor-core inference: BF16 weights, inputs and hidden activations, FP32 sums."""
    w = {k: to_bf16(v) for k, v in unpack(np.asarray(p, np.float32)).items()}
    b = unpack(np.asarray(p, np.float32))
    a = to_bf16(x)
    for L in ("1", "2", "3"):
        z = a.astype(np.float64) @ w["W" + L].astype(np.float64) + b["b" + L]
        a = to_bf16(silu(z).astype(np.float32))
    y = a.astype(np.float64) @ w["W4"].astype(np.float64) + b["b4"]
    return y.astype(np.float32)


def dp_features(eps, alpha, ratio, cohesion_term):
    """Network inputs of the Drucker-Prager closure: strains in units of the trial
    deviatoric norm s, (eps / s, alpha, (lambda+mu)/mu, cohesion/(2 mu s), ln s)."""
    eps = np.asarray(eps, np.float32)
    trace = eps[:, 0] + eps[:, 1]
    dev = eps - (trace * np.float32(0.5))[:, None]
    s = np.sqrt(dev[:, 0] * dev[:, 0] + dev[:, 1] * dev[:, 1]).astype(np.float32)
    return np.column_stack([eps[:, 0] / s, eps[:, 1] / s, alpha, ratio, cohesion_term / s,
                            np.log(s)]).astype(np.float32)


def dp_smooth_targets(x):
    """Drucker-Prager smooth plastic branch (sand.rs:156-194) from the network inputs
    (dp_features): returns (h1 / s, h2 / s, gamma / s) and a mask of the rows on that branch
    (gamma > 0, trace <= 0).  With eps / s given, the mapping needs no s: it is invariant
    under scaling of the strains."""
    x = np.asarray(x, np.float32)
    e = x[:, :2]
    trace = e[:, 0] + e[:, 1]
    dev = e - (trace * np.float32(0.5))[:, None]
    dev_norm = np.sqrt(dev[:, 0] * dev[:, 0] + dev[:, 1] * dev[:, 1])  # = 1 up to rounding
    g = dev_norm + x[:, 3] * trace * x[:, 2] - x[:, 4]
    on = (dev_norm > 0) & (trace <= 0) & (g > 0)
    safe = np.where(dev_norm > 0, dev_norm, 1.0)
    h = e - g[:, None] * (dev / safe[:, None])
    return np.column_stack([h, g]).astype(np.float32), on


def principal_stress(model, x, y):
    """Principal Kirchhoff stress of outputs y (log singular values first; Drucker-Prager
    in units of s = exp(x[:, 5]), NACC as the correction of x's log singular values),
    scale-free: Drucker-Prager in units of mu, NACC in units of kappa."""
    unit = np.exp(np.asarray(x[:, 5], np.float64)) if model == 0 else 1.0
    # NACC outputs: the plastic correction ln(sv') - ln(sv)
    off0 = 0.0 if model == 0 else np.asarray(x[:, 0], np.float64)
    off1 = 0.0 if model == 0 else np.asarray(x[:, 1], np.float64)
    a = np.exp(np.asarray(y[:, 0], np.float64) * unit + off0)
    b = np.exp(np.asarray(y[:, 1], np.float64) * unit + off1)
    j = a * b
    if model == 0:
        lam = x[:, 3] - 1.0
        vol = lam * (j - 1.0) * j
        return np.column_stack([2 * (a - 1) * a + vol, 2 * (b - 1) * b + vol])
    jj = np.maximum(j, 1e-6)
    ht = 0.5 * (a * a + b * b)
    vol = 0.5 * (jj * jj - 1.0)
    mk = x[:, 3]
    return np.column_stack([mk / jj * (a * a - ht) + vol, mk / jj * (b * b - ht) + vol])


def stress_rel_err(model, x, y_pred, y_ref):
    sp, sr = principal_stress(model, x, y_pred), principal_stress(model, x, y_ref)
    return np.linalg.norm(sp - sr, axis=1) / np.maximum(np.linalg.norm(sr, axis=1), 1e-6)
