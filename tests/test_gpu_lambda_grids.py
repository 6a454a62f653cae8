"""Per-pixel wavelength grids (gm_config.lambda_per_pixel / lambda_map).

Each pixel carries its own absolute wavelengths -- the case of a
wavelength-shifted field of view, which the reference's 4-D wavelength FITS
(utilsFits.c:1488-1500) was meant to describe -- while the PSF taps stay
global.  The oracle is pixel-wise, so each pixel is checked against the
oracle configured on that pixel's grid, with the tolerances of the
single-grid parity tests:
  synthesis          <= 2e-6 of the reference-faithful FP32 oracle (error
                      norm per Stokes in units of the Stokes-I norm)
  classical estimates B, vlos, gamma, phi within 1e-6 relative (FP64)
  full inversions    as the single-grid inversions: >= 95 % agree, and agree
                      or chi2 no worse on >= 99 %
A map whose rows all equal the configured grid must give bit-identical
results to the configured grid itself."""
import numpy as np
import pytest

import gmilos_b200 as G
import helpers as H
import oracle as O

pytestmark = pytest.mark.gpu

ZG = G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0)


@pytest.fixture(scope="module")
def engine():
    e = G.Engine(0)
    yield e
    e.close()


def shifted_grids(P, rng, nl=30, shift_mA=25.0, stretch=0.01):
    """Grids of the -350:35:665 mA layout shifted by up to +-shift_mA and
    stretched by up to +-stretch per pixel (an etalon-like wavelength drift
    across the field)."""
    lam, off = H.grid(nl)
    l0, _ = H.fe_line()
    sh = rng.uniform(-shift_mA, shift_mA, P) / 1000.0
    st = 1.0 + rng.uniform(-stretch, stretch, P)
    return lam, l0 + (lam[None, :] - l0) * st[:, None] + sh[:, None]


def ocfg_for(lam_p, psf=None, fix=H.FREE9, **kw):
    l0, zo = H.fe_line()
    return O.make_cfg(lam_p, l0, zo, psf=psf, fix=fix, init=H.GUESS, **kw)


def observe(lmap, truth, rng, psf=None, sl=None, fix=H.FREE9, noise=1e-3):
    obs = np.stack([O.synth_f(ocfg_for(lmap[p], psf, fix), truth[p], slight=sl) for p in range(len(truth))])
    obs = obs + rng.normal(0, noise, obs.shape)
    return np.ascontiguousarray(obs, dtype=np.float32)


@pytest.mark.parametrize("psf,stray,mac", [(False, False, False), (True, True, False), (True, False, True)])
def test_synthesis_on_per_pixel_grids(engine, psf, stray, mac):
    rng = np.random.default_rng(1200 + 2 * psf + mac)
    P = 96
    lam, lmap = shifted_grids(P, rng)
    l0, _ = H.fe_line()
    p = O.psf_gauss(100.0, lam) if psf else None
    sl = H.stray_profile(ocfg_for(lam)) if stray else None
    fix = H.FREE9[:10] + (1 if stray else 0,)
    t = H.truth_models(P, rng, alpha_range=(0.7, 1.0) if stray else None)
    if mac:
        t[:, 9] = rng.uniform(0.3, 2.0, P)
    engine.configure(G.make_config(lam, l0, ZG, psf=p, fix=fix, init=H.GUESS, slight=sl, lambda_map=lmap))
    s = engine.synthesize(t)
    ref = np.stack([O.synth_f(ocfg_for(lmap[k], p, fix), t[k], slight=sl) for k in range(P)])
    err = H.rel_to_I(s, ref)
    assert err.max() < 2e-6, err.max()
    # the grids matter: the same models on the configured grid differ
    engine.configure(G.make_config(lam, l0, ZG, psf=p, fix=fix, init=H.GUESS, slight=sl))
    assert H.rel_to_I(engine.synthesize(t), ref).max() > 1e-3


def test_classical_estimates_on_per_pixel_grids(engine):
    rng = np.random.default_rng(1300)
    P = 64
    lam, lmap = shifted_grids(P, rng)
    l0, _ = H.fe_line()
    t = H.truth_models(P, rng)
    obs = observe(lmap, t, rng)
    engine.configure(G.make_config(lam, l0, ZG, init=H.GUESS, lambda_map=lmap))
    m = engine.classical(obs)
    for k in range(P):
        r = O.classical(ocfg_for(lmap[k]), obs[k], model=H.GUESS, for_init=0)
        np.testing.assert_allclose(m[k, [1, 2, 5, 6, 7]], r[[1, 2, 5, 6, 7]], rtol=1e-6, atol=1e-9)


@pytest.mark.parametrize("psf,stray", [(False, False), (True, True)])
def test_inversion_on_per_pixel_grids(engine, psf, stray):
    rng = np.random.default_rng(1400 + psf)
    P = 256
    lam, lmap = shifted_grids(P, rng)
    l0, _ = H.fe_line()
    p = O.psf_gauss(100.0, lam) if psf else None
    sl = H.stray_profile(ocfg_for(lam)) if stray else None
    fix = H.FREE9[:10] + (1 if stray else 0,)
    t = H.truth_models(P, rng, alpha_range=(0.7, 1.0) if stray else None)
    obs = observe(lmap, t, rng, psf=p, sl=sl, fix=fix)
    gcfg = G.make_config(lam, l0, ZG, psf=p, fix=fix, init=H.GUESS, slight=sl, numerics=1, lambda_map=lmap)
    mr = np.zeros((P, 11))
    cr = np.zeros(P)
    for k in range(P):
        mr[k], cr[k], _, _, _ = O.lm_f(ocfg_for(lmap[k], p, fix), obs[k], slight=sl)
    for name, out in H.invert_each_kernel(engine, gcfg, obs):
        mg, cg = out["model64"], out["chi2"]
        no_worse = cg <= cr * (1 + 1e-3) + 1e-6
        ok = H.fits_agree(mg, mr) & no_worse
        print("%s: agree %.4f  chi2-no-worse %.4f" % (name, ok.mean(), no_worse.mean()))
        assert ok.mean() >= 0.95, name
        assert (ok | no_worse).mean() >= 0.99, name


def test_uniform_map_equals_configured_grid(engine):
    """Rows that all equal the configured grid: bit-identical results, for the
    10-term kernel and for the macroturbulence-capable one."""
    rng = np.random.default_rng(1500)
    P = 200
    lam, _ = H.grid()
    l0, _ = H.fe_line()
    p = O.psf_gauss(100.0, lam)
    t = H.truth_models(P, rng)
    obs = observe(np.repeat(lam[None], P, 0), t, rng, psf=p)
    for mac0 in (0.0, 0.5):
        init = list(H.GUESS)
        init[9] = mac0
        a_cfg = G.make_config(lam, l0, ZG, psf=p, init=init)
        b_cfg = G.make_config(lam, l0, ZG, psf=p, init=init, lambda_map=np.repeat(lam[None], P, 0))
        engine.configure(a_cfg)
        a = engine.invert(obs)
        engine.configure(b_cfg)
        b = engine.invert(obs)
        np.testing.assert_array_equal(a["model64"], b["model64"])
        np.testing.assert_array_equal(a["chi2"], b["chi2"])
        np.testing.assert_array_equal(a["iters"], b["iters"])


def test_device_map_and_errors(engine):
    import torch
    rng = np.random.default_rng(1600)
    P = 32
    lam, lmap = shifted_grids(P, rng)
    l0, _ = H.fe_line()
    t = H.truth_models(P, rng)
    obs = observe(lmap, t, rng)
    engine.configure(G.make_config(lam, l0, ZG, init=H.GUESS, lambda_map=lmap))
    host = engine.invert(obs)
    dmap = torch.tensor(lmap, dtype=torch.float64, device="cuda")
    engine.configure(G.make_config(lam, l0, ZG, init=H.GUESS, lambda_map=dmap))
    dev = engine.invert(obs)
    np.testing.assert_array_equal(host["model64"], dev["model64"])
    # a configuration that asks for per-pixel grids without a map
    c = G.make_config(lam, l0, ZG, init=H.GUESS)
    c.lambda_per_pixel = 1
    engine.configure(c)
    with pytest.raises(G.GmError) as e:
        engine.invert(obs)
    assert e.value.status == 1
    # serving shares one grid between requests
    engine.configure(G.make_config(lam, l0, ZG, init=H.GUESS, lambda_map=lmap))
    with pytest.raises(G.GmError) as e:
        engine.submit(obs, np.empty((P, 11), np.float32))
    assert e.value.status == 5
