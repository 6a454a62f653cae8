"""Shared fixtures: line, grids, synthetic truth models, observations."""
import numpy as np

import oracle as O

GUESS = (40.0, 1000.0, 0.2, 0.03, 0.05, 150.0, 110.0, 0.35, 0.5, 0.0, 1.0)   # run/guess.mod
FREE9 = (1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0)


def kat():
    g = np.load(__file__.replace("helpers.py", "golden/kat_synthesis.npz"))
    return g


def fe_line():
    return O.fe6173()


def grid(nl=30, step=35.0, first=None):
    """Centred grid of nl samples at `step` mA (default: the -350:35:665 grid)."""
    l0, _ = fe_line()
    if first is None:
        first = -350.0 if nl == 30 else -step * (nl // 2)
    last = first + step * (nl - 1)
    return O.grid_lambda(l0, first, step, last), O.grid_offsets_mA(first, step, last)


def truth_models(n, rng, alpha_range=None, normalise=True):
    """Uniform draws in the ranges of the headline benchmark (eta0 1-30, B 0-3000 G,
    vlos +-3 km/s, Doppler width 20-60 mA, damping 0-0.5, angles 0-180 deg,
    S0 0.1-0.5, S1 0.3-1.0); S0, S1 rescaled by the continuum S0+S1 so the
    profiles are normalised to the continuum."""
    t = np.zeros((n, 11))
    t[:, 0] = rng.uniform(1, 30, n)
    t[:, 1] = rng.uniform(0, 3000, n)
    t[:, 2] = rng.uniform(-3, 3, n)
    t[:, 3] = rng.uniform(0.020, 0.060, n)
    t[:, 4] = rng.uniform(0, 0.5, n)
    t[:, 5] = rng.uniform(0, 180, n)
    t[:, 6] = rng.uniform(0, 180, n)
    t[:, 7] = rng.uniform(0.1, 0.5, n)
    t[:, 8] = rng.uniform(0.3, 1.0, n)
    t[:, 10] = 1.0 if alpha_range is None else rng.uniform(*alpha_range, n)
    if normalise:
        ic = t[:, 7] + t[:, 8]
        t[:, 7] /= ic
        t[:, 8] /= ic
    return t


def observations(cfg, truth, rng, noise=1e-3, slight=None, slight_per_pixel=False):
    obs = O.synth_batch_f(cfg, truth, slight=slight, slight_per_pixel=slight_per_pixel)
    if noise:
        obs = obs + rng.normal(0, noise, obs.shape).astype(np.float32)
    return np.ascontiguousarray(obs, dtype=np.float32)


def stray_profile(cfg):
    """Field-free ME profile used as the stray-light source."""
    m = np.array([10.0, 0.0, 0.0, 0.03, 0.1, 0.0, 0.0, 0.3, 0.7, 0.0, 1.0])
    return O.synth_f(cfg, m).astype(np.float32)


def normwise(a, b):
    """max over Stokes rows of ||a - b|| / ||b|| (last axis = wavelength)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    num = np.sqrt(((a - b) ** 2).sum(axis=-1))
    den = np.sqrt((b ** 2).sum(axis=-1))
    return num / np.maximum(den, 1e-300)


def rel_to_I(a, b):
    """Per-Stokes error norm in units of the Stokes-I norm of b (polarisation
    measured in units of the intensity, as inversion codes quote it); a and b
    are [..., 4, nl]."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    num = np.sqrt(((a - b) ** 2).sum(axis=-1))
    den = np.sqrt((b[..., 0:1, :] ** 2).sum(axis=-1))
    return num / np.maximum(den, 1e-300)


def rf_rel(a, b):
    """Per-parameter error of response functions [..., 4, nt, nl]: norm over
    Stokes and wavelength of the difference / norm of b's column."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    num = np.sqrt(((a - b) ** 2).sum(axis=(-3, -1)))
    den = np.sqrt((b ** 2).sum(axis=(-3, -1)))
    return np.where(den > 0, num / np.maximum(den, 1e-300), num)


def angle_diff(a, b, period=180.0):
    d = np.abs(np.asarray(a) - np.asarray(b)) % period
    return np.minimum(d, period - d)


def fits_agree(ma, mb):
    """Per pixel: two fitted models [P][11] agree to |dB| < 1 G, |d gamma| and
    |d phi| < 0.1 deg (phi modulo 180) and |d vlos| < 5 m/s."""
    return ((np.abs(ma[:, 1] - mb[:, 1]) < 1.0) & (angle_diff(ma[:, 5], mb[:, 5], 360) < 0.1)
            & (angle_diff(ma[:, 6], mb[:, 6]) < 0.1) & (np.abs(ma[:, 2] - mb[:, 2]) < 0.005))


def random_net(seed, nl=30, realistic=True):
    """A learned-guess network with random weights and biases, standardised
    (when realistic) to the truth-model distribution so that its outputs land
    inside the parameter ranges."""
    import gmilos_b200 as G
    import mlp_oracle as M
    net = G.mlp_new(nl, seed)
    a = net.arrays()
    rng = np.random.default_rng(seed)
    a["b1"][:] = rng.normal(0, 0.1, a["b1"].shape)
    a["b2"][:] = rng.normal(0, 0.1, a["b2"].shape)
    a["w3"][:] *= 10.0
    a["b3"][:M.OUT] = rng.normal(0, 0.1, M.OUT)
    if realistic:
        t = M.targets(truth_models(4096, rng))
        a["out_mean"][:M.OUT] = t.mean(axis=0)
        a["out_scale"][:M.OUT] = t.std(axis=0)
        a["in_mean"][:4 * nl] = rng.normal(0, 0.1, 4 * nl)
        a["in_scale"][:4 * nl] = rng.uniform(5, 20, 4 * nl)
    return net


def invert_each_kernel(engine, gcfg, obs, **kw):
    """Yields ("waves", out) and ("fused", out): `obs` inverted once by the
    wave-synchronous kernels and once by the fused persistent kernel under
    the configuration `gcfg` (restored to the automatic choice afterwards).
    Calls of a few thousand pixels run the fused kernel by default, so the
    inversion parity tests run both kernels against one oracle result."""
    import gmilos_b200 as G
    try:
        for name, kernel in (("waves", G.KERNEL_WAVES), ("fused", G.KERNEL_FUSED)):
            gcfg.kernel = kernel
            engine.configure(gcfg)
            out = engine.invert(obs, **kw)
            launches = engine.stats()["kernel_launches"]
            if len(obs):
                assert (launches > 2) if name == "waves" else (launches <= 2), (name, launches)
            yield name, out
    finally:
        gcfg.kernel = G.KERNEL_AUTO
        engine.configure(gcfg)
