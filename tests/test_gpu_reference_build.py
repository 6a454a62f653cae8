"""The engine against the reference's own routines, on the GPU.

Two comparison builds of the reference's per-pixel code (oracle/build_ref.py):
the host build (libgmref_cpu.so) and the sm_100a build (libgmref_gpu.so, the
reference's lm_mils with its own launch geometry, streams and device heap,
child launches run in-thread).  The engine runs through its C ABI.

  - One LM iteration (miter = 1, classical-estimate start): the engine in
    ACCURATE numerics against the host build; model p99 <= 1e-4 relative,
    chi2 <= 1e-4 relative, identical accept/reject.
  - Full inversions of a cube with PSF and stray light: the engine in
    REFERENCE numerics (the reference's __sincosf / __fdividef) against the
    sm_100a build on identical inputs: median chi2 within 1 %, parameters
    agreeing (|dB| < 1 G, angles < 0.1 deg, vlos < 5 m/s) on >= 75 % of
    pixels, the engine's chi2 worse (by > 1e-3) on no more pixels than the
    reference's is worse (+1 %), and truth recovery no worse.
Skipped when the libraries are not built.
"""
import numpy as np
import pytest

import gmilos_b200 as G
import helpers as H
import oracle as O

ref = pytest.importorskip("ref")
pytestmark = pytest.mark.gpu

FIX = (1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 1)


@pytest.fixture(scope="module")
def engine():
    e = G.Engine(0)
    yield e
    e.close()


def setups(psf, stray, miter=50, numerics=0, fix=FIX):
    lam, _ = H.grid(30)
    l0, zo = H.fe_line()
    zg = G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0)
    p = O.psf_gauss(100.0, lam) if psf else None
    ocfg = O.make_cfg(lam, l0, zo, psf=p, fix=fix, init=H.GUESS, miter=miter)
    sl = H.stray_profile(ocfg) if stray else None
    gcfg = G.make_config(lam, l0, zg, psf=p, fix=fix, init=H.GUESS, slight=sl, miter=miter,
                         numerics=numerics)
    return ocfg, ref.setup_from_cfg(ocfg), gcfg, sl


def cube(ocfg, sl, n, seed):
    rng = np.random.default_rng(seed)
    t = H.truth_models(n, rng, alpha_range=(0.7, 1.0) if sl is not None else None)
    return t, H.observations(ocfg, t, rng, slight=sl)


@pytest.mark.skipif(not ref.available(), reason="libgmref_cpu.so not built")
@pytest.mark.parametrize("psf,stray", [(False, False), (True, True)])
def test_one_iteration_matches_reference_host_build(engine, psf, stray):
    fix = FIX if stray else H.FREE9
    ocfg, s, gcfg, sl = setups(psf, stray, miter=1, numerics=G.NUMERICS_ACCURATE, fix=fix)
    t, obs = cube(ocfg, sl, 1024, 21)
    engine.configure(gcfg)
    out = engine.invert(obs)
    mr, cr, ir, _ = ref.invert_cpu(s, obs, slight=sl)
    rel = np.abs(out["model64"] - mr) / np.maximum(np.abs(mr), 1e-3)
    crel = np.abs(out["chi2"] - cr) / cr
    print("one iteration vs reference host build: model rel p50 %.2e p99 %.2e max %.2e, chi2 rel max %.2e"
          % (np.percentile(rel[:, :9], 50), np.percentile(rel[:, :9], 99), rel[:, :9].max(), crel.max()))
    assert (out["iters"] == ir).all()
    assert np.percentile(rel[:, :9], 99) < 1e-4
    assert np.percentile(crel, 99) < 1e-4


@pytest.mark.skipif(not ref.available(gpu=True), reason="libgmref_gpu.so not built")
def test_inversions_match_reference_gpu_build(engine):
    ocfg, s, gcfg, sl = setups(True, True, numerics=G.NUMERICS_REFERENCE)
    # 16 384 pixels: the shares of pixels where either side ends worse are
    # ~10 % each, so their difference has a standard deviation of ~0.34 %
    # and the 1 % margin below is ~3 sigma (on 4096 pixels single seeds
    # swing by +-1.2 % either way)
    t, obs = cube(ocfg, sl, 16384, 22)
    engine.configure(gcfg)
    out = engine.invert(obs)
    mr, cr, ir, _, rep = ref.invert_gpu(s, obs, slight=sl, nstreams=16)
    assert rep["malloc_failures"] == 0
    mg, cg = out["model64"], out["chi2"]
    agree = ((np.abs(mg[:, 1] - mr[:, 1]) < 1.0) & (H.angle_diff(mg[:, 5], mr[:, 5], 360) < 0.1)
             & (H.angle_diff(mg[:, 6], mr[:, 6]) < 0.1) & (np.abs(mg[:, 2] - mr[:, 2]) < 0.005))
    worse_g = ~agree & (cg > cr * (1 + 1e-3) + 1e-6)
    worse_r = ~agree & (cr > cg * (1 + 1e-3) + 1e-6)
    rec_g = (np.abs(mg[:, 1] - t[:, 1]) < 50).mean()
    rec_r = (np.abs(mr[:, 1] - t[:, 1]) < 50).mean()
    print("vs reference sm_100a build: agree %.4f, engine chi2 worse %.4f, reference chi2 worse %.4f, "
          "median chi2 %.4f / %.4f, iters %.1f / %.1f, |dB-truth|<50G %.4f / %.4f"
          % (agree.mean(), worse_g.mean(), worse_r.mean(), np.median(cg), np.median(cr),
             out["iters"].mean(), ir.mean(), rec_g, rec_r))
    assert np.median(cg) == pytest.approx(np.median(cr), rel=0.01)
    # Two FP32 implementations of the same LM trajectory part ways wherever
    # rounding flips an accept/reject decision (the reference's host and GPU
    # builds agree on ~84 % of these pixels); where they part, neither side
    # is systematically better.
    assert agree.mean() >= 0.75
    assert worse_g.mean() <= worse_r.mean() + 0.01
    assert rec_g >= rec_r - 0.01


@pytest.mark.skipif(not ref.available(), reason="libgmref_cpu.so not built")
@pytest.mark.parametrize("fix", [FIX, (1,) * 11])
def test_macroturbulence_iteration_matches_reference_host_build(engine, fix):
    """One iteration with macroturbulence: the fixed-v_mac 10-term path and
    the 11-term path (lm_mils_11, FP64 step) against the reference's host
    build, ACCURATE numerics."""
    lam, _ = H.grid(30)
    l0, zo = H.fe_line()
    zg = G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0)
    p = O.psf_gauss(100.0, lam)
    init = list(H.GUESS)
    init[9] = 0.5
    ocfg = O.make_cfg(lam, l0, zo, psf=p, fix=fix, init=init, miter=1)
    sl = H.stray_profile(ocfg)
    gcfg = G.make_config(lam, l0, zg, psf=p, fix=fix, init=init, slight=sl, miter=1,
                         numerics=G.NUMERICS_ACCURATE)
    rng = np.random.default_rng(23 + sum(fix))
    t = H.truth_models(1024, rng, alpha_range=(0.7, 1.0))
    t[:, 9] = rng.uniform(0.3, 2.0, len(t))
    obs = H.observations(ocfg, t, rng, slight=sl)
    engine.configure(gcfg)
    out = engine.invert(obs)
    mr, cr, ir, _ = ref.invert_cpu(ref.setup_from_cfg(ocfg), obs, slight=sl)
    rel = np.abs(out["model64"] - mr) / np.maximum(np.abs(mr), 1e-3)
    crel = np.abs(out["chi2"] - cr) / cr
    print("v_mac one iteration (%d terms): model rel p99 %.2e, chi2 rel p99 %.2e"
          % (engine.nterms, np.percentile(rel, 99), np.percentile(crel, 99)))
    assert (out["iters"] == ir).all()
    assert np.percentile(rel, 99) < 1e-4
    assert np.percentile(crel, 99) < 1e-4
