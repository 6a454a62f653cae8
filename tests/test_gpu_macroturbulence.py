"""Macroturbulence and the 11-term path on the GPU against the oracle.

The reference convolves the profiles with a Gaussian macroturbulence kernel
when v_mac > 1e-4 (fgauss.cu:16-63, mil_sinrf.cu:101-116), with the PSF
folded into the kernel; the response functions go through the kernel and
v_mac's own RF through its derivative (me_der.cu:117-156).  With v_mac and
alpha both free it runs its 11-term kernel (lm_mils_11,
milosUtils.cu:713-850) whose step is an FP64 SVD solve (mil_svd,
milosUtils.cu:280-325).

Tolerances are those of the 10-term tests: synthesis <= 2e-6 of the
Stokes-I norm against the reference-faithful FP32 oracle and <= 1e-5 against
FP64; RF columns <= max(1e-4, 10 x the reference arithmetic's own deviation
from FP64); one LM step (ACCURATE numerics, identical state) p99 <= 1e-4;
full inversions >= 95 % agreeing outright and >= 99 % agreeing or with a
chi2 no worse (1e-3).
"""
import numpy as np
import pytest

import gmilos_b200 as G
import helpers as H
import oracle as O

pytestmark = pytest.mark.gpu

FIX10 = (1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 1)     # 9 ME + alpha, v_mac fixed
FIX11 = (1,) * 11                             # v_mac and alpha free: 11 terms


@pytest.fixture(scope="module")
def engine():
    e = G.Engine(0)
    yield e
    e.close()


def configs(nl=30, psf=True, stray=True, fix=FIX10, mac0=0.6, **kw):
    l0, zo = H.fe_line()
    zg = G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0)
    lam, _ = H.grid(nl)
    p = O.psf_gauss(100.0, lam) if psf else None
    init = list(H.GUESS)
    init[9] = mac0
    okw = {k: v for k, v in kw.items() if k in ("miter",)}
    ocfg = O.make_cfg(lam, l0, zo, psf=p, fix=fix, init=init, **okw)
    sl = H.stray_profile(ocfg) if stray else None
    gkw = {k: v for k, v in kw.items() if k in ("miter", "numerics", "init_mode")}
    gcfg = G.make_config(lam, l0, zg, psf=p, fix=fix, init=init, slight=sl, **gkw)
    return ocfg, gcfg, sl


def truth(n, rng, stray=True):
    t = H.truth_models(n, rng, alpha_range=(0.7, 1.0) if stray else None)
    t[:, 9] = rng.uniform(0.2, 3.0, n)
    return t


@pytest.mark.parametrize("nl,psf,stray,fix", [(30, False, False, FIX10), (30, True, True, FIX10),
                                              (30, True, True, FIX11), (31, True, False, FIX10),
                                              (64, True, True, FIX11), (45, False, True, FIX11)])
def test_synthesis_and_rf_with_macroturbulence(engine, nl, psf, stray, fix):
    rng = np.random.default_rng(700 + nl)
    ocfg, gcfg, sl = configs(nl, psf, stray, fix)
    t = truth(96, rng, stray)
    t[::8, 9] = 0.0                           # some pixels without macroturbulence
    engine.configure(gcfg)
    s, rf = engine.synthesize(t, rf=True)
    nt = engine.nterms
    assert rf.shape[2] == nt == ocfg.nterms
    worst = 0.0
    for p in range(len(t)):
        sl64 = None if sl is None else sl.astype(np.float64)
        s64, r64 = O.synth_d(ocfg, t[p], slight=sl64, rf=True)
        s32, r32 = O.synth_f(ocfg, t[p], slight=sl, rf=True)
        assert H.rel_to_I(s[p], s32).max() < 2e-6
        assert H.rel_to_I(s[p], s64).max() < 1e-5
        own = H.rf_rel(r32, r64)
        bound = np.maximum(1e-4, 10 * own)
        cols = list(range(9)) + ([9] if (stray or nt == 11) else []) + ([10] if nt == 11 else [])
        worst = max(worst, (H.rf_rel(rf[p], r64) / bound)[cols].max())
    assert worst < 1.0, worst


@pytest.mark.parametrize("fix", [FIX10, FIX11])
def test_one_step_with_macroturbulence(engine, fix):
    rng = np.random.default_rng(710 + len(fix) + sum(fix))
    ocfg, gcfg, sl = configs(fix=fix, numerics=G.NUMERICS_ACCURATE)
    t = truth(256, rng)
    obs = H.observations(ocfg, t, rng, slight=sl)
    start = t.copy()
    start[:, 1] = np.clip(t[:, 1] * rng.uniform(0.8, 1.2, len(t)) + 50, 0, None)
    start[:, 2] += rng.uniform(-0.3, 0.3, len(t))
    start[:, 9] = np.clip(t[:, 9] * rng.uniform(0.7, 1.3, len(t)), 0.05, None)
    engine.configure(gcfg)
    d, trial, c0, c1 = engine.lm_step(obs, start, 0.1)
    nt = engine.nterms
    rel = []
    for p in range(len(t)):
        dr, tr, c1r, c0r = O.lm_step_f(ocfg, start[p], obs[p], 0.1, slight=sl)
        assert c0[p] == pytest.approx(c0r, rel=1e-4)
        ref = np.asarray(dr[:nt], dtype=np.float64)
        rel.append(np.linalg.norm(d[p, :nt] - ref) / max(np.linalg.norm(ref), 1e-30))
    rel = np.array(rel)
    assert np.percentile(rel, 99) < 1e-4 and rel.max() < 1e-3, (np.percentile(rel, [50, 99]), rel.max())


@pytest.mark.parametrize("fix", [FIX10, FIX11])
def test_inversions_with_macroturbulence(engine, fix):
    rng = np.random.default_rng(720 + sum(fix))
    ocfg, gcfg, sl = configs(fix=fix, numerics=G.NUMERICS_ACCURATE)
    t = truth(1024, rng)
    obs = H.observations(ocfg, t, rng, slight=sl)
    mr, cr, ir, ar, fr = O.lm_batch_f(ocfg, obs, slight=sl)
    for name, out in H.invert_each_kernel(engine, gcfg, obs):
        mg, cg = out["model64"], out["chi2"]
        ok = H.fits_agree(mg, mr)
        no_worse = cg <= cr * (1 + 1e-3) + 1e-6
        print("%s: agree %.4f  chi2-no-worse %.4f  iters %.1f / %.1f  mac %.3f / %.3f"
              % (name, ok.mean(), no_worse.mean(), out["iters"].mean(), ir.mean(), np.median(mg[:, 9]),
                 np.median(mr[:, 9])))
        assert ok.mean() >= 0.95, name
        assert (ok | no_worse).mean() >= 0.99, name
