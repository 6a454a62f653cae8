"""The engine against the reference's own routines, on the GPU.

Two comparison builds of the reference's per-pixel code (oracle/build_ref.py):
the host build (libgmref_cpu.so) and the sm_100a build (libgmref_gpu.so, the
reference's lm_mils with its own launch geometry, streams and device heap,
child launches run in-thread).  The engine runs through its C ABI.

  - One LM iteration (miter = 1, classical-estimate start): the engine in
    ACCURATE numerics against the host build, and in REFERENCE numerics
    (the reference's __sincosf / __fdividef) against the sm_100a build;
    model p99 <= 1e-4 relative, chi2 <= 1e-4 relative, the same
    accept/reject decisions.
  - Full inversions of a cube with PSF and stray light: the engine in
    REFERENCE numerics against the sm_100a build on identical inputs: median
    chi2 within 1 %, parameters agreeing (|dB| < 1 G, angles < 0.1 deg,
    vlos < 5 m/s) on at least the share (-2 %) on which the reference's own
    host build agrees with its sm_100a build, the engine's chi2 worse (by
    > 1e-3) on no more pixels than the reference's is worse (+1 %), and
    truth recovery no worse.
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
    mr, cr, ir, _ = ref.invert_cpu(s, obs, slight=sl)
    for name, out in H.invert_each_kernel(engine, gcfg, obs):
        rel = np.abs(out["model64"] - mr) / np.maximum(np.abs(mr), 1e-3)
        crel = np.abs(out["chi2"] - cr) / cr
        print("%s, one iteration vs reference host build: model rel p50 %.2e p99 %.2e max %.2e, "
              "chi2 rel max %.2e" % (name, np.percentile(rel[:, :9], 50), np.percentile(rel[:, :9], 99),
                                     rel[:, :9].max(), crel.max()))
        assert (out["iters"] == ir).all(), name
        assert np.percentile(rel[:, :9], 99) < 1e-4, name
        assert np.percentile(crel, 99) < 1e-4, name


@pytest.mark.skipif(not (ref.available(gpu=True) and ref.available()),
                    reason="libgmref_gpu.so / libgmref_cpu.so not built")
def test_inversions_match_reference_gpu_build(engine):
    """Full inversions (PSF, stray light, 9 ME + alpha, <= 50 iterations).
    Two FP32 implementations of the same LM trajectory part ways wherever
    rounding flips one accept/reject decision, so the bar for the engine is
    the reference's own: the engine agrees with the reference's sm_100a build
    on at least as many pixels (-2 %) as the reference's host build does with
    that same sm_100a build, on the same pixels; where fits part, neither
    side is systematically better."""
    ocfg, s, gcfg, sl = setups(True, True, numerics=G.NUMERICS_REFERENCE)
    # 16 384 pixels: the shares of pixels where either side ends worse are
    # ~10 % each, so their difference has a standard deviation of ~0.34 %
    # and the 1 % margin below is ~3 sigma (on 4096 pixels single seeds
    # swing by +-1.2 % either way); the agreement shares have a standard
    # deviation of ~0.35 %, so the 2 % margin is over 4 sigma
    t, obs = cube(ocfg, sl, 16384, 22)
    engine.configure(gcfg)
    out = engine.invert(obs)
    mr, cr, ir, _, rep = ref.invert_gpu(s, obs, slight=sl, nstreams=16)
    assert rep["malloc_failures"] == 0
    mh, ch, ih, _ = ref.invert_cpu(s, obs, slight=sl)
    mg, cg = out["model64"], out["chi2"]
    agree = H.fits_agree(mg, mr)
    agree_ref = H.fits_agree(mh, mr)
    worse_g = ~agree & (cg > cr * (1 + 1e-3) + 1e-6)
    worse_r = ~agree & (cr > cg * (1 + 1e-3) + 1e-6)
    worse_h = ~agree_ref & (ch > cr * (1 + 1e-3) + 1e-6)
    worse_hr = ~agree_ref & (cr > ch * (1 + 1e-3) + 1e-6)
    rec_g = (np.abs(mg[:, 1] - t[:, 1]) < 50).mean()
    rec_r = (np.abs(mr[:, 1] - t[:, 1]) < 50).mean()
    print("vs reference sm_100a build: engine agrees %.4f (chi2 worse %.4f, reference's worse %.4f); "
          "reference host build agrees %.4f (chi2 worse %.4f, GPU build's worse %.4f); "
          "median chi2 %.4f / %.4f / %.4f, iters %.1f / %.1f / %.1f, |dB-truth|<50G %.4f / %.4f"
          % (agree.mean(), worse_g.mean(), worse_r.mean(), agree_ref.mean(), worse_h.mean(),
             worse_hr.mean(), np.median(cg), np.median(cr), np.median(ch), out["iters"].mean(),
             ir.mean(), ih.mean(), rec_g, rec_r))
    assert np.median(cg) == pytest.approx(np.median(cr), rel=0.01)
    assert agree.mean() >= agree_ref.mean() - 0.02
    assert worse_g.mean() <= worse_r.mean() + 0.01
    assert rec_g >= rec_r - 0.01


@pytest.mark.skipif(not (ref.available(gpu=True) and ref.available()),
                    reason="libgmref_gpu.so / libgmref_cpu.so not built")
@pytest.mark.parametrize("psf,stray", [(False, False), (True, True)])
def test_one_iteration_reference_numerics_vs_reference_gpu_build(engine, psf, stray):
    """One LM iteration (miter = 1, classical-estimate start) in REFERENCE
    numerics -- the reference's __sincosf / __fdividef in the solve and the
    angles -- against the reference's own sm_100a build.  The two builds
    round the synthesis, the response functions and the normal equations
    differently (FMA contraction chosen by two compilations; both sum the
    normal equations in FP32, the reference each Stokes parameter in
    sequence, lib.cu:65-118, the engine per lane and then as a tree over
    the lanes), and the 18-step Jacobi with the hardware trigonometry
    amplifies last-bit differences of alpha into step differences
    (measured: model p99 5e-5 to 1e-4, chi2 p99 1.6e-4 to 1.9e-4,
    99.3-99.6 % of pixels within 1e-3, the largest difference 5 % of
    a parameter -- a step-size difference, far below a whole step, so no
    accept/reject decision differs).  The same step by the reference's own
    host build (libm trigonometry) lands within 1e-3 of its sm_100a build
    on only 0.4-2.9 % of the pixels (p99 0.13-0.27): the engine must
    reproduce the sm_100a build's step better than that build's own host
    compilation does."""
    fix = FIX if stray else H.FREE9
    ocfg, s, gcfg, sl = setups(psf, stray, miter=1, numerics=G.NUMERICS_REFERENCE, fix=fix)
    t, obs = cube(ocfg, sl, 4096, 24)
    mr, cr, ir, _, rep = ref.invert_gpu(s, obs, slight=sl, nstreams=16)
    assert rep["malloc_failures"] == 0
    # the reference's own host build against its sm_100a build, same step
    mh, ch, ih, _ = ref.invert_cpu(s, obs, slight=sl)
    relh = np.abs(mh - mr) / np.maximum(np.abs(mr), 1e-3)
    crelh = np.abs(ch - cr) / cr
    sameh = (relh[:, :9].max(axis=1) < 1e-3).mean()
    print("one iteration, reference host build vs its sm_100a build: same decision %.4f, model rel "
          "p50 %.2e p99 %.2e max %.2e, chi2 rel p99 %.2e"
          % (sameh, np.percentile(relh[:, :9], 50), np.percentile(relh[:, :9], 99), relh[:, :9].max(),
             np.percentile(crelh, 99)))
    for name, out in H.invert_each_kernel(engine, gcfg, obs):
        rel = np.abs(out["model64"] - mr) / np.maximum(np.abs(mr), 1e-3)
        crel = np.abs(out["chi2"] - cr) / cr
        # the output is the last accepted model: a different accept/reject
        # decision shows as a whole step's difference, far above 1e-3
        same = (rel[:, :9].max(axis=1) < 1e-3).mean()
        print("%s, one iteration, REFERENCE numerics vs reference sm_100a build: same decision %.4f, "
              "model rel p50 %.2e p99 %.2e max %.2e, chi2 rel p99 %.2e"
              % (name, same, np.percentile(rel[:, :9], 50), np.percentile(rel[:, :9], 99), rel[:, :9].max(),
                 np.percentile(crel, 99)))
        assert (out["iters"] == ir).all(), name
        assert same >= 0.99 and same > sameh, name
        assert np.percentile(rel[:, :9], 99) < np.percentile(relh[:, :9], 99), name
        assert rel[:, :9].max() < 0.2, name
        assert np.percentile(rel[:, :9], 99) < 2e-4, name
        assert np.percentile(crel, 99) < 5e-4, name


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
    mr, cr, ir, _ = ref.invert_cpu(ref.setup_from_cfg(ocfg), obs, slight=sl)
    for name, out in H.invert_each_kernel(engine, gcfg, obs):
        rel = np.abs(out["model64"] - mr) / np.maximum(np.abs(mr), 1e-3)
        crel = np.abs(out["chi2"] - cr) / cr
        print("%s, v_mac one iteration (%d terms): model rel p99 %.2e, chi2 rel p99 %.2e"
              % (name, engine.nterms, np.percentile(rel, 99), np.percentile(crel, 99)))
        assert (out["iters"] == ir).all(), name
        assert np.percentile(rel, 99) < 1e-4, name
        assert np.percentile(crel, 99) < 1e-4, name
