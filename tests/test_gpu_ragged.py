"""Ragged batches on the GPU (gm_invert_rois through gmilos_b200.batch): ROIs
of 16 to 512 px a side on centred 35 mA grids of 12 to 60 samples, each with
its own PSF taps, the per-pixel early stop on an accepted chi2 gain below
1e-4, all in one launch sequence per samples-per-lane class.

  - pixels are independent: every ROI's results in the batch equal those of
    the ROI alone, bit for bit, and so do the results of a graph replay and
    of any resident-block limit the autotuner tries;
  - the ragged-batch kernels against the plain inversion of each ROI on its
    own grid (the same LM arithmetic compiled as other kernels: equal to
    rounding, fits agree on nearly every pixel);
  - every pixel of the small ROIs against the faithful oracle.
"""
import numpy as np
import pytest

import gmilos_b200 as G
from gmilos_b200 import batch
import helpers as H
import oracle as O

pytestmark = pytest.mark.gpu

ZG = G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0)
STOP = 1e-4
L0 = 6173.3356


def psf_for(lam):
    return O.psf_gauss(100.0, lam)


def base_config(numerics=0):
    lam, _ = H.grid(30)
    return G.make_config(lam, L0, ZG, init=H.GUESS, stop_dchi2=STOP, numerics=numerics)


def make_rois(eng, seed, sides, nls):
    """Observations synthesised by the engine on each ROI's grid, with its
    PSF, noise 1e-3."""
    rng = np.random.default_rng(seed)
    out = []
    for side, nl in zip(sides, nls):
        lam, _ = H.grid(int(nl))
        eng.configure(G.make_config(lam, L0, ZG, psf=psf_for(lam), init=H.GUESS))
        t = H.truth_models(int(side) ** 2, rng)
        o = eng.synthesize(t)
        out.append((np.ascontiguousarray(o + rng.normal(0, 1e-3, o.shape).astype(np.float32)), lam))
    return out


@pytest.fixture(scope="module")
def engine():
    e = G.Engine(0)
    yield e
    e.close()


@pytest.fixture(scope="module")
def rois(engine):
    sides = [512, 16, 24, 100, 16, 48, 200, 24, 64, 16]
    nls = [30, 12, 60, 45, 31, 20, 33, 57, 12, 30]
    return make_rois(engine, 41, sides, nls)


def test_batch_equals_rois_alone(engine, rois):
    engine.configure(base_config())
    got, st = batch.invert_rois(engine, rois, psf_for)
    print("batch: %d px, %d grids, %d launches, lane occupancy %.3f, %.1f ms"
          % (st["pixels"], st["grids"], st["launches"], st["lane_occupancy"], st["device_ms"]))
    assert st["pixels"] == sum(len(a) for a, _ in rois)
    assert st["grids"] == len({len(l) for _, l in rois})
    assert 0.3 < st["lane_occupancy"] < 1.0
    for (a, lam), g in zip(rois, got):
        alone, _ = batch.invert_rois(engine, [(a, lam)], psf_for)
        for k in ("model", "chi2", "iters", "status"):
            np.testing.assert_array_equal(g[k], alone[0][k], err_msg=k)
    # early stop: far fewer trials than the iteration limit
    assert np.mean(np.concatenate([g["iters"] for g in got])) < 40


def test_graph_replay_and_tuning_change_nothing(engine, rois):
    engine.configure(base_config())
    plain, _ = batch.invert_rois(engine, rois, psf_for)
    tuned, st1 = batch.invert_rois(engine, rois, psf_for, autotune=True)
    first, st2 = batch.invert_rois(engine, rois, psf_for, use_graph=True, autotune=True)
    again, st3 = batch.invert_rois(engine, rois, psf_for, use_graph=True, autotune=True)
    print("tuned limits trial %d accept %d; graph replayed %d / %d; %.1f ms direct, %.1f ms replayed"
          % (st1["cap_trial"], st1["cap_accept"], st2["graph_replayed"], st3["graph_replayed"],
             st1["device_ms"], st3["device_ms"]))
    assert st2["graph_replayed"] == 0 and st3["graph_replayed"] == 1
    assert st1["cap_trial"] >= 1 and st1["cap_accept"] >= 1
    for outs in (tuned, first, again):
        for p, g in zip(plain, outs):
            for k in ("model", "chi2", "iters", "status"):
                np.testing.assert_array_equal(p[k], g[k], err_msg=k)


@pytest.mark.parametrize("numerics", [G.NUMERICS_REFERENCE, G.NUMERICS_ACCURATE])
def test_batch_against_plain_inversions(engine, rois, numerics):
    """The ragged-batch kernels and the one-grid wave kernels (chosen
    explicitly: small calls would otherwise run the fused kernel) run the
    same LM arithmetic.  At <= 32 samples they compile to the same results bit
    for bit; at 33..64 samples they round differently, and in REFERENCE
    numerics (hardware trigonometry in the solve) the trajectories then part
    on some pixels as between any two builds: neither side is worse more
    often, and in ACCURATE numerics the fits agree on nearly every pixel."""
    engine.configure(base_config(numerics=numerics))
    got, _ = batch.invert_rois(engine, rois, psf_for)
    worse_b, worse_p, agree, tot = 0, 0, 0, 0
    for (a, lam), g in zip(rois[1:6], got[1:6]):
        engine.configure(G.make_config(lam, L0, ZG, psf=psf_for(lam), init=H.GUESS, stop_dchi2=STOP,
                                       numerics=numerics, kernel=G.KERNEL_WAVES))
        ref = engine.invert(a)
        same = H.fits_agree(np.asarray(g["model"], dtype=np.float64), ref["model64"])
        wb = ~same & (g["chi2"] > ref["chi2"] * (1 + 1e-3) + 1e-6)
        wp = ~same & (ref["chi2"] > g["chi2"] * (1 + 1e-3) + 1e-6)
        agree += int(same.sum())
        worse_b += int(wb.sum())
        worse_p += int(wp.sum())
        tot += len(a)
        bitwise = (g["model"] == ref["model"]).all(axis=1).mean()
        print("numerics %d, nl %d: agree %.4f, batch worse %.4f, plain worse %.4f, bit-identical models %.4f"
              % (numerics, len(lam), same.mean(), wb.mean(), wp.mean(), bitwise))
        if len(lam) <= 32:
            assert bitwise == 1.0
    assert worse_b / tot <= worse_p / tot + 0.02
    if numerics == G.NUMERICS_ACCURATE:
        assert agree / tot >= 0.97


def test_batch_against_the_oracle(engine, rois):
    """Every pixel of the small ROIs (<= 24 px a side) against the oracle in
    the numerics whose LM steps it follows."""
    engine.configure(base_config(numerics=G.NUMERICS_ACCURATE))
    small = [r for r in rois if len(r[0]) <= 24 * 24]
    got, _ = batch.invert_rois(engine, small, psf_for)
    ok = []
    for (a, lam), g in zip(small, got):
        ocfg = O.make_cfg(lam, L0, H.fe_line()[1], psf=psf_for(lam), init=H.GUESS, stop_dchi2=STOP)
        mr, cr, _, _, _ = O.lm_batch_f(ocfg, a, nthreads=0)
        mg, cg = np.asarray(g["model"], dtype=np.float64), g["chi2"]
        ok.append((cg <= cr * (1 + 1e-3) + 1e-6) | H.fits_agree(mg, mr))
    ok = np.concatenate(ok)
    print("oracle: agree or chi2 no worse on %.4f of %d pixels" % (ok.mean(), len(ok)))
    assert ok.mean() >= 0.97


def test_ragged_batch_refuses_what_it_cannot_do(engine, rois):
    lam, _ = H.grid(30)
    sl = np.ones((4, 30), np.float32)
    engine.configure(G.make_config(lam, L0, ZG, init=H.GUESS, slight=sl, fix=(1,) * 9 + (0, 1)))
    with pytest.raises(G.GmError):
        batch.invert_rois(engine, rois[:2], psf_for)


def test_empty_rois_and_empty_batch(engine, rois):
    """A ROI without pixels in a batch changes nothing for the others, and a
    batch without pixels returns at once."""
    engine.configure(base_config())
    some = [rois[1], rois[2], rois[4]]
    empty = (np.zeros((0, 4, len(rois[3][1])), np.float32), rois[3][1])
    plain, st = batch.invert_rois(engine, some, psf_for)
    mixed, st2 = batch.invert_rois(engine, [some[0], empty, some[1], some[2]], psf_for)
    assert st2["pixels"] == st["pixels"]
    assert len(mixed[1]["model"]) == 0
    for p, g in zip(plain, [mixed[0], mixed[2], mixed[3]]):
        for k in ("model", "chi2", "iters", "status"):
            np.testing.assert_array_equal(p[k], g[k], err_msg=k)
    none, st0 = batch.invert_rois(engine, [empty], psf_for)
    assert st0["pixels"] == 0 and len(none[0]["model"]) == 0
    nothing, stn = batch.invert_rois(engine, [], psf_for)
    assert stn["pixels"] == 0 and nothing == []
