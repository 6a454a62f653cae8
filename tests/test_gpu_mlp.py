"""The learned initial guess on the GPU: its tensor-core inference and
training kernels against the CPU restatement (oracle/mlp_oracle.py), and
what a trained network gains an inversion over the classical start.

  - inference: the start models the network gives (gm_mlp_predict) equal the
    oracle's on the same BF16 roundings, to FP32 accumulation order (a few
    BF16 roundings of hidden activations may flip);
  - gradients: one batch's loss and every weight and bias gradient
    (gm_mlp_gradients) equal the oracle's to 1 % (normwise), cosine > 0.9999;
  - training on pixels synthesised by the engine (the 30-sample grid, PSF,
    noise 1e-3) lowers the loss, and inversions started from the trained
    guess (GM_INIT_LEARNED, with the classical start kept wherever it has the
    lower chi2) converge in fewer iterations to no worse a chi2 and no worse
    a recovery of the truth than inversions from the classical start.
"""
import numpy as np
import pytest

import gmilos_b200 as G
import helpers as H
import mlp_oracle as M
import oracle as O

pytestmark = pytest.mark.gpu

ZG = G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0)


@pytest.fixture(scope="module")
def engine():
    e = G.Engine(0)
    yield e
    e.close()


def config(nl=30, psf=True, **kw):
    lam, _ = H.grid(nl)
    l0, zo = H.fe_line()
    p = O.psf_gauss(100.0, lam) if psf else None
    return (O.make_cfg(lam, l0, zo, psf=p, init=H.GUESS),
            G.make_config(lam, l0, ZG, psf=p, init=H.GUESS, **kw))


def observations(ocfg, n, seed):
    rng = np.random.default_rng(seed)
    t = H.truth_models(n, rng)
    return t, H.observations(ocfg, t, rng)


@pytest.mark.parametrize("nl,n", [(30, 1000), (20, 300)])
def test_inference_matches_oracle(engine, nl, n):
    ocfg, gcfg = config(nl)
    net = H.random_net(11 + nl, nl)
    _, obs = observations(ocfg, n, 5 + nl)
    engine.configure(gcfg)
    got = engine.mlp_predict(net, obs)
    want, _ = M.predict(M.params(net), obs, H.GUESS, H.FREE9)
    p = M.params(net)
    err = np.abs(M.targets(got) - M.targets(want)) / p["out_scale"][:M.OUT]
    print("inference vs oracle (nl %d): standardised output error p50 %.2e p99 %.2e max %.2e"
          % (nl, np.median(err), np.percentile(err, 99), err.max()))
    assert np.percentile(err, 99) < 5e-3 and np.median(err) < 5e-4
    np.testing.assert_array_equal(got[:, 9:], np.tile(np.asarray(H.GUESS)[9:], (n, 1)))


def test_inference_with_tiles_in_flight_matches_oracle(engine):
    """Enough pixels that every CTA of the persistent inference kernel runs
    tiles through both of its slots and starts a second pair (3 tiles per
    CTA on 148 SMs, one CTA 4, the last tile partial): the outputs equal
    the oracle's as they do for small calls."""
    ocfg, gcfg = config(30)
    net = H.random_net(61, 30)
    n = 148 * 128 * 3 + 77
    rng = np.random.default_rng(62)
    engine.configure(gcfg)
    obs = engine.synthesize(H.truth_models(n, rng))
    obs = np.ascontiguousarray(obs + rng.normal(0, 1e-3, obs.shape).astype(np.float32))
    got = engine.mlp_predict(net, obs)
    want, _ = M.predict(M.params(net), obs, H.GUESS, H.FREE9)
    p = M.params(net)
    err = np.abs(M.targets(got) - M.targets(want)) / p["out_scale"][:M.OUT]
    print("inference with tiles in flight (%d px): standardised output error p50 %.2e p99 %.2e max %.2e"
          % (n, np.median(err), np.percentile(err, 99), err.max()))
    assert np.percentile(err, 99) < 5e-3 and np.median(err) < 5e-4


def test_gradients_match_oracle(engine):
    ocfg, gcfg = config()
    net = H.random_net(21)
    truth, obs = observations(ocfg, 512, 22)
    engine.configure(gcfg)
    loss, g = engine.mlp_gradients(net, obs, truth)
    p = M.params(net)
    X = M.inputs(p, obs)
    Y = M.standardised_targets(p, truth).astype(np.float32).astype(np.float64)
    lo, go = M.loss_and_grads(p, X, Y)
    print("loss engine %.6f oracle %.6f" % (loss, lo))
    assert loss == pytest.approx(lo, rel=1e-3)
    ga = g.arrays()
    for name in ("w1", "b1", "w2", "b2", "w3", "b3"):
        a = np.asarray(ga[name], dtype=np.float64)
        b = go[name]
        if name == "b3":
            a = a[:M.OUT]
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        cos = float((a * b).sum() / (np.linalg.norm(a) * np.linalg.norm(b)))
        print("%s: relative error %.2e, cosine %.7f" % (name, rel, cos))
        assert rel < 1e-2 and cos > 0.9999, name
    # the unused inputs (past 4 nl) get no gradient
    assert not np.any(np.asarray(ga["w1"])[:, 120:])


def test_training_and_what_the_learned_guess_gains(engine):
    ocfg, gcfg = config(stop_dchi2=1e-4)
    rng = np.random.default_rng(31)
    n = 1 << 17
    truth = H.truth_models(n, rng)
    engine.configure(gcfg)
    clean = engine.synthesize(truth)
    obs = np.ascontiguousarray(clean + rng.normal(0, 1e-3, clean.shape).astype(np.float32))
    net = G.mlp_new(30, 3)
    losses = engine.mlp_train(net, obs, truth, epochs=6, batch=8192, lr=2e-3)
    print("training loss per epoch:", np.round(losses, 4))
    assert losses[-1] < 0.5 * losses[0]
    assert net.steps == 6 * (n // 8192)
    # a cube the network has not seen
    tt = H.truth_models(4096, rng)
    ct = engine.synthesize(tt)
    ob = np.ascontiguousarray(ct + rng.normal(0, 1e-3, ct.shape).astype(np.float32))
    plain = engine.invert(ob)
    lam, _ = H.grid(30)
    l0, _ = H.fe_line()
    engine.configure(G.make_config(lam, l0, ZG, psf=O.psf_gauss(100.0, lam), init=H.GUESS, stop_dchi2=1e-4,
                                   init_mode=G.INIT_LEARNED, mlp=net))
    learned = engine.invert(ob)
    took = ((learned["status"] & G.PIX_LEARNED_INIT) != 0).mean()
    dB_p = np.median(np.abs(plain["model64"][:, 1] - tt[:, 1]))
    dB_l = np.median(np.abs(learned["model64"][:, 1] - tt[:, 1]))
    print("learned start kept on %.1f%% of pixels; mean iterations %.2f -> %.2f; median chi2 %.4f -> %.4f; "
          "median |B - truth| %.1f -> %.1f G"
          % (100 * took, plain["iters"].mean(), learned["iters"].mean(), np.median(plain["chi2"]),
             np.median(learned["chi2"]), dB_p, dB_l))
    assert took > 0.5
    assert learned["iters"].mean() < 0.9 * plain["iters"].mean()
    assert np.median(learned["chi2"]) <= 1.01 * np.median(plain["chi2"])
    assert dB_l <= 1.05 * dB_p + 1.0


def test_learned_mode_needs_a_network_for_its_grid(engine):
    _, gcfg = config(init_mode=G.INIT_LEARNED)
    with pytest.raises(G.GmError):
        engine.configure(gcfg)
    _, g20 = config(nl=20, init_mode=G.INIT_LEARNED, mlp=G.mlp_new(30))
    with pytest.raises(G.GmError):
        engine.configure(g20)


def test_misaligned_device_profiles_rejected(engine):
    """The kernels read profiles in 16-byte vectors: a device array that
    starts 4 bytes past a boundary is refused on the host, before any
    launch, and the context stays usable."""
    import torch
    ocfg, gcfg = config(30)
    net = H.random_net(3, 30)
    _, obs = observations(ocfg, 256, 9)
    engine.configure(gcfg)
    flat = torch.zeros(obs.size + 1, dtype=torch.float32, device="cuda")
    flat[1:] = torch.from_numpy(np.ascontiguousarray(obs, dtype=np.float32).ravel()).cuda()
    bad = flat[1:].view(obs.shape)
    assert bad.data_ptr() % 16 == 4
    with pytest.raises(G.GmError, match="16-byte"):
        engine.mlp_predict(net, bad)
    good = torch.from_numpy(np.ascontiguousarray(obs, dtype=np.float32)).cuda()
    got = engine.mlp_predict(net, good).cpu().numpy()
    want = engine.mlp_predict(net, obs)
    assert np.array_equal(got, want)
