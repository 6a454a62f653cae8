"""CPU restatement of the learned initial guess (TEST INFRASTRUCTURE ONLY).

The network of include/gmilos.h (gm_mlp: 4 nl -> 256 -> 256 -> 9, GELU) in
numpy FP64, with the engine kernels' rounding points restated so that their
outputs and gradients can be checked against it: inputs standardised in FP32
and rounded to BF16, weights rounded to BF16, hidden activations rounded to
BF16 after GELU, the output gradient rounded to BF16, and every product and
sum then in FP64 (the kernels accumulate the same BF16 operands in FP32 on
the tensor cores, g-milos_b200/csrc/gm_mlp.cu).  With quantize=False it is the
plain FP64 network, whose gradients tests/test_mlp_oracle.py checks against
finite differences.  The learned guess has no counterpart in the reference:
its training targets are the reference's model parameters (Init_Model,
defines.h:94-106) in the engine's 9-output encoding.

Only tests/ and bench.py's checks import this module.
"""
import math

import numpy as np

IN, HID, OUT, OUT_PAD = 128, 256, 9, 16
DEG = math.pi / 180.0


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    nan = np.isnan(a)
    if nan.any():
        out[nan] = np.nan
    return out


SQRT_2_OVER_PI = math.sqrt(2.0 / math.pi)


def _sigmoid_2u(z):
    """s = (1 + tanh u) / 2 = 1 / (1 + exp(-2u)), u = sqrt(2/pi) (z + 0.044715 z^3),
    and d(2u)/dz."""
    z = np.asarray(z, dtype=np.float64)
    u2 = 2.0 * SQRT_2_OVER_PI * z * (1.0 + 0.044715 * z * z)
    du2 = 2.0 * SQRT_2_OVER_PI * (1.0 + 3 * 0.044715 * z * z)
    with np.errstate(over="ignore"):
        s = 1.0 / (1.0 + np.exp(-u2))
    return s, du2


def gelu(z):
    """GELU in its tanh form (Hendrycks & Gimpel, 2016)."""
    s, _ = _sigmoid_2u(z)
    return np.asarray(z, dtype=np.float64) * s


def gelu_grad(z):
    s, du2 = _sigmoid_2u(z)
    return s + np.asarray(z, dtype=np.float64) * s * (1.0 - s) * du2


def targets(models):
    """The 9 outputs of models [n][11]: eta0, vlos, Doppler width, damping,
    S0, S1, B cos gamma, B sin gamma cos 2 phi, B sin gamma sin 2 phi."""
    m = np.asarray(models, dtype=np.float64)
    g, ph = m[:, 5] * DEG, 2.0 * m[:, 6] * DEG
    return np.stack([m[:, 0], m[:, 2], m[:, 3], m[:, 4], m[:, 7], m[:, 8], m[:, 1] * np.cos(g),
                     m[:, 1] * np.sin(g) * np.cos(ph), m[:, 1] * np.sin(g) * np.sin(ph)], axis=1)


def outputs_to_models(y, guess, fix):
    """9 de-standardised outputs -> models [n][11] within the reference's
    ranges (milosUtils.cu:160-238); fixed parameters, v_mac and the filling
    factor from the guess model."""
    y = np.asarray(y, dtype=np.float64)
    bl, bq, bu = y[:, 6], y[:, 7], y[:, 8]
    bt = np.sqrt(bq * bq + bu * bu)
    phi = 0.5 * np.arctan2(bu, bq) / DEG
    phi = np.where(phi < 0, phi + 180.0, phi)
    v = np.stack([np.clip(y[:, 0], 1, 2500), np.minimum(np.sqrt(bl * bl + bt * bt), 5000),
                  np.clip(y[:, 1], -20, 20), np.clip(y[:, 2], 1e-4, 0.6), np.clip(y[:, 3], 1e-4, 10),
                  np.arctan2(bt, bl) / DEG, phi, np.clip(y[:, 4], 1e-4, 2), np.clip(y[:, 5], 1e-4, 2)], axis=1)
    m = np.tile(np.asarray(guess, dtype=np.float64), (len(y), 1))
    for i in range(9):
        if fix[i]:
            m[:, i] = np.where(np.isfinite(v[:, i]), v[:, i], m[:, i])
    return m


def params(net):
    """float64 copies of a gm_mlp's arrays (net.arrays() of the binding)."""
    return {k: np.asarray(v, dtype=np.float64) for k, v in net.arrays().items()}


def inputs(p, iquv, quantize=True):
    """Standardised inputs [n][128]: (x - mean) * scale in FP32, BF16-rounded."""
    x = np.asarray(iquv, dtype=np.float32).reshape(len(iquv), -1)
    X = np.zeros((len(x), IN), dtype=np.float32)
    F = x.shape[1]
    X[:, :F] = (x - p["in_mean"][:F].astype(np.float32)) * p["in_scale"][:F].astype(np.float32)
    return bf16(X) if quantize else X.astype(np.float64)


def forward(p, X, quantize=True):
    """Forward pass on standardised inputs X [n][128]; every intermediate."""
    q = bf16 if quantize else (lambda a: np.asarray(a, dtype=np.float64))
    W1, W2, W3 = q(p["w1"]), q(p["w2"]), q(p["w3"])
    z1 = X @ W1.T + p["b1"]
    h1 = q(gelu(z1))
    z2 = h1 @ W2.T + p["b2"]
    h2 = q(gelu(z2))
    out = h2 @ W3.T + p["b3"][:OUT]
    return {"X": X, "z1": z1, "h1": h1, "z2": z2, "h2": h2, "out": out, "W1": W1, "W2": W2, "W3": W3}


def loss_and_grads(p, X, Y, quantize=True):
    """Mean squared error over the batch and the 9 standardised outputs, and
    its gradients (w1, b1, w2, b2, w3, b3), as the training kernels form
    them: bias gradients are column sums of the BF16-rounded output
    gradients of each layer."""
    q = bf16 if quantize else (lambda a: np.asarray(a, dtype=np.float64))
    f = forward(p, X, quantize)
    n = len(X)
    d = f["out"] - Y
    loss = float((d * d).sum() / (n * OUT))
    g3 = q(2.0 * d / (n * OUT))
    dh2 = g3 @ f["W3"]
    g2 = q(dh2 * gelu_grad(f["z2"]))
    dh1 = g2 @ f["W2"]
    g1 = q(dh1 * gelu_grad(f["z1"]))
    grads = {"w3": g3.T @ f["h2"], "b3": g3.sum(axis=0), "w2": g2.T @ f["h1"], "b2": g2.sum(axis=0),
             "w1": g1.T @ X, "b1": g1.sum(axis=0)}
    return loss, grads


def standardised_targets(p, models):
    t = targets(models)
    return (t - p["out_mean"][:OUT]) / p["out_scale"][:OUT]


def predict(p, iquv, guess, fix):
    """Start models the network gives for iquv [n][4][nl]."""
    f = forward(p, inputs(p, iquv))
    y = (f["out"] + 0.0) * p["out_scale"][:OUT] + p["out_mean"][:OUT]
    return outputs_to_models(y, guess, fix), y
