"""GPU parity: the CUDA engine (through the C ABI) against the CPU oracle.

The engine has two numerics modes.  REFERENCE uses the hardware sin/cos and
fast division the reference uses inside its 10x10 Jacobi solver; their
absolute error (a few 1e-7) is amplified by the badly scaled normal matrix
into step differences of ~1e-3, which no CPU code can reproduce.  ACCURATE
uses correctly rounded trigonometry there and is the mode in which the GPU
algorithm is compared step by step with the oracle.

Tolerances (floating point):
  synthesis          <= 1e-5 of the FP64 oracle, error norm per Stokes in
                      units of the Stokes-I norm; <= 2e-6 of the reference-
                      faithful FP32 oracle; known-answer vector <= 2e-6
  response functions per parameter column: <= 1e-4 of the FP64 oracle or
                      <= 10x the deviation of the reference's own FP32
                      arithmetic from FP64, whichever is larger
  one LM step        <= 1e-4 relative step difference (99th percentile) from
                      the reference-faithful oracle at an identical state
  full inversions    |dB| < 1 G, |d angles| < 0.1 deg, |d vlos| < 5 m/s and
                      chi2 no worse (1e-3) on >= 95 % of pixels, and agree or
                      chi2 no worse on >= 99 %; the oracle against itself
                      with 1-ulp input perturbations reaches 97-99 % / 99 %.
"""
import numpy as np
import pytest

import gmilos_b200 as G
import helpers as H
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    e = G.Engine(0)
    yield e
    e.close()


def configs(nl=30, psf=False, stray=False, fix=H.FREE9, **kw):
    l0, zo = H.fe_line()
    zg = G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0)
    lam, off = H.grid(nl)
    p = O.psf_gauss(100.0, lam) if psf else None
    ocfg = O.make_cfg(lam, l0, zo, psf=p, fix=fix, init=H.GUESS, **{k: v for k, v in kw.items()
                                                                       if k in ("miter", "ilambda", "logclambda", "weight", "classical_init")})
    sl = H.stray_profile(ocfg) if stray else None
    gkw = {k: v for k, v in kw.items() if k in ("miter", "ilambda", "logclambda", "weight", "init_mode",
                                                 "numerics", "kernel")}
    gcfg = G.make_config(lam, l0, zg, psf=p, fix=fix, init=H.GUESS, slight=sl, **gkw)
    return ocfg, gcfg, sl


# ------------------------------------------------------------ synthesis
def test_known_answer_vector(engine):
    """data/synthesis_gpu.per: the reference's synthesis of run/init.mod with
    the CRISP PSF, reproduced by the GPU synthesis."""
    g = H.kat()
    l0 = float(g["lambda0"])
    first, step, last = g["grid"]
    lam = G.grid_lambda(l0, first, step, last)
    off = G.grid_offsets_mA(first, step, last)
    psf = G.psf_from_table(g["psf_x_mA"], g["psf_y"], off, step)
    cfg = G.make_config(lam, l0, G.zeeman_from_levels(*g["quantum"], 1.0), psf=psf)
    engine.configure(cfg)
    s = engine.synthesize(g["model"][None, :].copy())
    assert H.normwise(s[0], g["per_iquv"]).max() < 2e-6


@pytest.mark.parametrize("nl,psf,stray", [(30, False, False), (30, True, False), (30, True, True),
                                          (31, True, False), (12, False, False), (64, True, True),
                                          (45, False, True)])
def test_synthesis_matches_oracle(engine, nl, psf, stray):
    rng = np.random.default_rng(100 + nl)
    ocfg, gcfg, sl = configs(nl, psf, stray, fix=H.FREE9[:10] + (1 if stray else 0,))
    t = H.truth_models(256, rng, alpha_range=(0.7, 1.0) if stray else None)
    engine.configure(gcfg)
    s = engine.synthesize(t)
    s64 = np.stack([O.synth_d(ocfg, m, slight=None if sl is None else sl.astype(np.float64)) for m in t])
    s32 = O.synth_batch_f(ocfg, t, slight=sl)
    e64 = H.rel_to_I(s, s64)
    e32 = H.rel_to_I(s, s32)
    assert e64.max() < 1e-5, e64.max()
    assert e32.max() < 2e-6, e32.max()


@pytest.mark.parametrize("nl,psf,stray", [(30, False, False), (30, True, True), (64, True, False)])
@pytest.mark.parametrize("numerics", [0, 1])
def test_response_functions_match_oracle(engine, nl, psf, stray, numerics):
    rng = np.random.default_rng(200 + nl)
    ocfg, gcfg, sl = configs(nl, psf, stray, fix=(1,) * 9 + (0, 1 if stray else 0), numerics=numerics)
    t = H.truth_models(128, rng, alpha_range=(0.7, 1.0) if stray else None)
    engine.configure(gcfg)
    s, rf = engine.synthesize(t, rf=True)
    worst64, worst32 = 0.0, 0.0
    for p in range(len(t)):
        sl64 = None if sl is None else sl.astype(np.float64)
        _, r64 = O.synth_d(ocfg, t[p], slight=sl64, rf=True)
        _, r32 = O.synth_f(ocfg, t[p], slight=sl, rf=True)
        own = H.rf_rel(r32, r64)                 # the reference arithmetic's own deviation
        bound = np.maximum(1e-4, 10 * own)       # large only for near-zero columns
        worst64 = max(worst64, (H.rf_rel(rf[p], r64) / bound)[:10].max())
        if numerics == 1:
            worst32 = max(worst32, (H.rf_rel(rf[p], r32) / bound)[:10].max())
    assert worst64 < 1.0, worst64
    assert worst32 < 1.0, worst32


def test_float32_and_float64_models_agree(engine):
    rng = np.random.default_rng(3)
    _, gcfg, _ = configs()
    engine.configure(gcfg)
    t = H.truth_models(64, rng)
    a = engine.synthesize(t)
    b = engine.synthesize(t.astype(np.float32))
    np.testing.assert_allclose(a, b, rtol=1e-4, atol=1e-5)


# ------------------------------------------------------------ one LM step
@pytest.mark.parametrize("psf,flambda", [(False, 0.1), (True, 0.1), (True, 1e-3), (False, 10.0)])
def test_one_lm_step_matches_reference(engine, psf, flambda):
    """One iteration from an identical state: the damped normal equations, the
    18-step parallel-Jacobi solve and the step limits against the faithful
    oracle (required: within 1e-4), with accurate trigonometry."""
    rng = np.random.default_rng(300)
    ocfg, gcfg, _ = configs(psf=psf, numerics=1)
    t = H.truth_models(256, rng)
    obs = H.observations(ocfg, t, rng)
    start = t.copy()
    start[:, 1] = np.clip(t[:, 1] * rng.uniform(0.8, 1.2, len(t)) + 50, 0, None)
    start[:, 2] += rng.uniform(-0.3, 0.3, len(t))
    start[:, 5] = np.clip(start[:, 5] + rng.uniform(-10, 10, len(t)), 1, 179)
    start[:, 6] = (start[:, 6] + rng.uniform(-10, 10, len(t))) % 180
    engine.configure(gcfg)
    d, trial, c0, c1 = engine.lm_step(obs, start, flambda)
    rel = []
    for p in range(len(t)):
        dr, tr, c1r, c0r = O.lm_step_f(ocfg, start[p], obs[p], flambda)
        assert c0[p] == pytest.approx(c0r, rel=1e-4)
        rel.append(np.linalg.norm(d[p, :9] - dr[:9]) / max(np.linalg.norm(dr[:9]), 1e-30))
    rel = np.array(rel)
    assert np.percentile(rel, 99) < 1e-4 and rel.max() < 1e-3, (np.percentile(rel, [50, 99]), rel.max())


# ------------------------------------------------------------ full inversions
def close_enough(mg, cg, mr, cr):
    return ((np.abs(mg[:, 1] - mr[:, 1]) < 1.0) & (H.angle_diff(mg[:, 5], mr[:, 5], 360) < 0.1)
            & (H.angle_diff(mg[:, 6], mr[:, 6]) < 0.1) & (np.abs(mg[:, 2] - mr[:, 2]) < 0.005)
            & (cg <= cr * (1 + 1e-3) + 1e-6))


@pytest.mark.parametrize("psf,stray", [(False, False), (True, True)])
def test_inversion_matches_reference(engine, psf, stray):
    """Full LM inversions against the faithful oracle.  Both follow the same
    algorithm in FP32; pixels agree unless rounding flips an accept/reject
    decision, after which both trajectories are still valid fits.  Pixels
    where parameters differ must then have a chi2 no worse than the oracle's
    (within 1e-3) on >= 99 %, and >= 95 % must agree to the stated
    tolerances outright."""
    rng = np.random.default_rng(400 + psf)
    fix = H.FREE9[:10] + (1 if stray else 0,)
    ocfg, gcfg, sl = configs(psf=psf, stray=stray, fix=fix, numerics=1)
    t = H.truth_models(1024, rng, alpha_range=(0.7, 1.0) if stray else None)
    obs = H.observations(ocfg, t, rng, slight=sl)
    mr, cr, ir, ar, fr = O.lm_batch_f(ocfg, obs, slight=sl, nthreads=0)
    for name, out in H.invert_each_kernel(engine, gcfg, obs, fitted=True):
        mg, cg = out["model64"], out["chi2"]
        ok = close_enough(mg, cg, mr, cr)
        no_worse = cg <= cr * (1 + 1e-3) + 1e-6
        print("%s: agree %.4f  chi2-no-worse %.4f  iters gpu %.1f ref %.1f"
              % (name, ok.mean(), no_worse.mean(), out["iters"].mean(), ir.mean()))
        assert ok.mean() >= 0.95, name
        assert (ok | no_worse).mean() >= 0.99, name
        same = ok & (out["iters"] == ir)
        # where the trajectories agree, the fitted profiles agree too; the
        # fitted output is the last trial, which may be a rejected step taken
        # with a large damping, and rounding can still move that one
        frel = H.rel_to_I(out["fitted"][same], fr[same]).max(axis=-1)
        assert (frel < 1e-4).mean() >= 0.98, (name, np.percentile(frel, [50, 99]))


@pytest.mark.parametrize("nl", [30, 45])
def test_wave_and_fused_kernels_agree(engine, nl):
    """The wave-synchronous kernels (the default) and the fused persistent
    kernel run the same LM arithmetic, compiled in different kernels: after
    one trial the models agree to float rounding, and full inversions match
    the oracle equally well (trajectories then part where rounding flips an
    accept/reject decision, as between any two builds)."""
    rng = np.random.default_rng(730 + nl)
    fix = H.FREE9[:10] + (1,)
    ocfg, gcfg, sl = configs(nl=nl, psf=True, stray=True, fix=fix, numerics=1)
    t = H.truth_models(1024, rng, alpha_range=(0.7, 1.0))
    obs = H.observations(ocfg, t, rng, slight=sl)
    mr, cr, _, _, _ = O.lm_batch_f(ocfg, obs, slight=sl, nthreads=0)
    res = {}
    for mode, kernel in (("waves", G.KERNEL_WAVES), ("fused", G.KERNEL_FUSED)):
        gcfg.kernel = kernel
        engine.configure(gcfg)
        full = engine.invert(obs)
        launches = engine.stats()["kernel_launches"]
        _, g1, _ = configs(nl=nl, psf=True, stray=True, fix=fix, numerics=1, miter=1, kernel=kernel)
        engine.configure(g1)
        res[mode] = (full, launches, engine.invert(obs)["model64"])
    (w, lw, w1), (f, lf, f1) = res["waves"], res["fused"]
    assert lw > lf
    rel = np.abs(w1 - f1) / np.maximum(np.abs(f1), 1e-3)
    assert (rel.max(axis=1) < 1e-4).mean() >= 0.99, np.percentile(rel.max(axis=1), [50, 99])
    okw = close_enough(w["model64"], w["chi2"], mr, cr).mean()
    okf = close_enough(f["model64"], f["chi2"], mr, cr).mean()
    print("oracle agreement: waves %.4f fused %.4f" % (okw, okf))
    assert okw >= 0.95 and okf >= 0.95 and abs(okw - okf) <= 0.03
    assert np.median(w["chi2"]) == pytest.approx(np.median(f["chi2"]), rel=1e-2)


def test_small_calls_run_the_fused_kernel(engine):
    """Under GM_KERNEL_AUTO a call of fewer than 16 384 pixels (with a PSF)
    runs the fused persistent kernel (pre-pass + one launch), a larger one
    the wave kernels (pre-pass + 101 launches); GM_KERNEL_WAVES keeps the
    small call on the wave kernels.  Both fit equally well."""
    rng = np.random.default_rng(745)
    ocfg, gcfg, _ = configs(psf=True)
    small = H.observations(ocfg, H.truth_models(4096, rng), rng)
    large = H.observations(ocfg, H.truth_models(16384, rng), rng)
    engine.configure(gcfg)
    fused = engine.invert(small)
    assert engine.stats()["kernel_launches"] == 2
    engine.invert(large)
    assert engine.stats()["kernel_launches"] == 2 + 2 * 50
    gcfg.kernel = G.KERNEL_WAVES
    engine.configure(gcfg)
    waves = engine.invert(small)
    assert engine.stats()["kernel_launches"] == 2 + 2 * 50
    assert np.median(waves["chi2"]) == pytest.approx(np.median(fused["chi2"]), rel=1e-2)
    assert abs(waves["iters"].mean() - fused["iters"].mean()) < 0.5


def test_wave_state_within_the_hbm_budget():
    """The wave kernels keep about 4 KB of LM state per pixel of a chunk in
    the context's budget; a budget with room for fewer than 16 384 pixels
    of it runs the fused kernel instead (pre-pass + one launch), and both
    give equally good fits."""
    rng = np.random.default_rng(740)
    ocfg, gcfg, _ = configs(psf=True)
    obs = H.observations(ocfg, H.truth_models(20000, rng), rng)
    res = {}
    for budget in (60 << 20, 300 << 20):
        with G.Engine(0, hbm_budget=budget) as e:
            e.configure(gcfg)
            out = e.invert(obs)
            res[budget] = (out, e.stats()["kernel_launches"])
    (f, lf), (w, lw) = res[60 << 20], res[300 << 20]
    assert lf == 2 and lw == 2 * 51
    assert np.median(w["chi2"]) == pytest.approx(np.median(f["chi2"]), rel=1e-2)
    assert abs(w["iters"].mean() - f["iters"].mean()) < 0.5


def test_calls_on_two_streams_take_the_scratch_in_turn(engine):
    """Device-buffer calls return at launch; two calls on different streams
    share the context's scratch (counters, wave state), so the second waits
    for the first on the device: both results equal the calls run alone."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(750)
    ocfg, gcfg, _ = configs(psf=True)
    engine.configure(gcfg)
    cubes = [torch.from_numpy(H.observations(ocfg, H.truth_models(20000, rng), rng)).cuda() for _ in range(2)]
    alone = [engine.invert(c) for c in cubes]
    torch.cuda.synchronize()
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    outs = []
    for c, st in zip(cubes, streams):
        o = {"model": torch.empty((len(c), 11), dtype=torch.float32, device="cuda"), "model64": None,
             "chi2": torch.empty(len(c), dtype=torch.float32, device="cuda"),
             "iters": torch.empty(len(c), dtype=torch.int32, device="cuda"),
             "accepted": None, "status": None, "fitted": None}
        engine.invert(c, out=o, stream=st.cuda_stream)
        outs.append(o)
    torch.cuda.synchronize()
    for o, a in zip(outs, alone):
        for k in ("model", "chi2", "iters"):
            np.testing.assert_array_equal(o[k].cpu().numpy(), a[k].cpu().numpy(), err_msg=k)


def test_inversion_edge_cases(engine):
    rng = np.random.default_rng(500)
    ocfg, gcfg, _ = configs(numerics=1)
    t = H.truth_models(37, rng)                         # not a multiple of the warps per block
    obs = H.observations(ocfg, t, rng)
    obs[3] = np.nan                                     # a bad pixel
    obs[5, 0, :3] = -1.0                                # leading "ghost" samples
    mr, cr, ir, ar, fr = O.lm_batch_f(ocfg, obs)
    good = np.ones(len(t), bool)
    good[3] = False
    for name, out in H.invert_each_kernel(engine, gcfg, obs):
        assert out["iters"].min() >= 1 and out["iters"].max() <= 50, name
        ok = close_enough(out["model64"][good], out["chi2"][good], mr[good], cr[good])
        nw = out["chi2"][good] <= cr[good] * (1 + 1e-3) + 1e-6
        assert (ok | nw).mean() >= 0.95, name
        assert out["status"][3] & (G.PIX_NONFINITE | G.PIX_INIT_NAN), name
    # an empty request is fine
    engine.configure(gcfg)
    empty = np.zeros((0, 4, 30), np.float32)
    o0 = engine.invert(empty)
    assert o0["chi2"].shape == (0,)


def test_results_do_not_depend_on_scheduling(engine):
    """Work stealing changes which warp takes a pixel, never its result."""
    rng = np.random.default_rng(600)
    ocfg, gcfg, _ = configs(psf=True)
    t = H.truth_models(300, rng)
    obs = H.observations(ocfg, t, rng)
    for kernel in (G.KERNEL_WAVES, G.KERNEL_FUSED):
        gcfg.kernel = kernel
        engine.configure(gcfg)
        a = engine.invert(obs)
        b = engine.invert(obs[::-1].copy())
        np.testing.assert_array_equal(a["model"], b["model"][::-1])
        np.testing.assert_array_equal(a["chi2"], b["chi2"][::-1])
        single = engine.invert(obs[7:8].copy())
        np.testing.assert_array_equal(single["model"][0], a["model"][7])


def test_pipelined_host_inversion_equals_one_launch(engine):
    """A cube in host memory of at least two 131 072-pixel chunks goes up in
    chunks on two streams, each inverted by its own launch; the results must
    be those of one launch over the same cube in device memory, bit for bit,
    including the per-pixel stray-light and wavelength maps (offset per
    chunk) and the fitted profiles; the iteration count sums over chunks."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(710)
    P = 300000
    fix = (1,) * 9 + (0, 1)
    ocfg, _, sl = configs(psf=True, stray=True, fix=fix)
    lam, _ = H.grid(30)
    l0, _ = H.fe_line()
    t = H.truth_models(P, rng, alpha_range=(0.7, 1.0))
    obs = H.observations(ocfg, t, rng, slight=sl)
    slmap = (sl[None] * rng.uniform(0.9, 1.1, (P, 1, 1))).astype(np.float32)
    lmap = lam[None, :] + rng.uniform(-0.01, 0.01, (P, 1))
    engine.configure(G.make_config(lam, l0, G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0),
                                   psf=O.psf_gauss(100.0, lam), fix=fix, init=H.GUESS, slight=slmap,
                                   slight_per_pixel=True, lambda_map=lmap))
    host = engine.invert(obs, fitted=True)
    st = engine.stats()
    dev = engine.invert(torch.from_numpy(obs).cuda(), fitted=True)
    torch.cuda.synchronize()
    # two chunks, each with the same kernels
    assert st["kernel_launches"] >= 2 and st["kernel_launches"] % 2 == 0
    for k in ("model", "model64", "chi2", "iters", "accepted", "status", "fitted"):
        np.testing.assert_array_equal(host[k], dev[k].cpu().numpy(), err_msg=k)
    assert st["iterations"] == int(host["iters"].sum())


def test_pipelined_host_inversion_in_three_chunks(engine):
    """A host cube large enough for a short first chunk and two long ones
    (131 072 + 2 x 284 464 pixels, alternating streams) gives the results of
    one launch over the cube in device memory, bit for bit."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(711)
    P = 700000
    fix = (1,) * 9 + (0, 1)
    ocfg, gcfg, sl = configs(psf=True, stray=True, fix=fix)
    engine.configure(gcfg)
    t = H.truth_models(P, rng, alpha_range=(0.7, 1.0))
    obs = engine.synthesize(t)
    obs = np.ascontiguousarray(obs + rng.normal(0, 1e-3, obs.shape).astype(np.float32))
    host = engine.invert(obs)
    st = engine.stats()
    dev = engine.invert(torch.from_numpy(obs).cuda())
    torch.cuda.synchronize()
    assert st["pixels"] == P
    for k in ("model", "model64", "chi2", "iters", "accepted", "status"):
        np.testing.assert_array_equal(host[k], dev[k].cpu().numpy(), err_msg=k)
    assert st["iterations"] == int(host["iters"].sum())


def test_classical_prepass_equals_in_kernel_estimates(engine):
    """gm_invert forms the classical start models in a pre-pass kernel;
    gm_invert_noalloc forms them inside the fused inversion kernel with the
    same device code: with gm_invert on the fused kernel too, the inversions
    agree bit for bit."""
    import ctypes as C
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(720)
    fix = (1,) * 9 + (0, 1)
    ocfg, gcfg, sl = configs(psf=True, stray=True, fix=fix, kernel=G.KERNEL_FUSED)
    obs = H.observations(ocfg, H.truth_models(4096, rng, alpha_range=(0.7, 1.0)), rng, slight=sl)
    engine.configure(gcfg)
    a = engine.invert(obs)
    d = torch.from_numpy(obs).cuda()
    P, nl = len(obs), obs.shape[2]
    model = torch.empty((P, 11), dtype=torch.float32, device="cuda")
    chi2 = torch.empty(P, dtype=torch.float32, device="cuda")
    iters = torch.empty(P, dtype=torch.int32, device="cuda")
    status = torch.empty(P, dtype=torch.int32, device="cuda")
    st = G.lib().gm_invert_noalloc(C.byref(gcfg), G._ptr(d), P, nl, G._ptr(model), G._ptr(chi2), G._ptr(iters),
                                   None, G._ptr(status), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == G.GM_OK
    torch.cuda.synchronize()
    np.testing.assert_array_equal(a["model"], model.cpu().numpy())
    np.testing.assert_array_equal(a["chi2"], chi2.cpu().numpy())
    np.testing.assert_array_equal(a["iters"], iters.cpu().numpy())
    np.testing.assert_array_equal(a["status"].astype(np.int64), status.cpu().numpy().astype(np.int64))


def test_device_and_host_buffers_agree(engine):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(700)
    ocfg, gcfg, _ = configs(psf=True)
    engine.configure(gcfg)
    obs = H.observations(ocfg, H.truth_models(64, rng), rng)
    a = engine.invert(obs)
    b = engine.invert(torch.from_numpy(obs).cuda())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(a["model"], b["model"].cpu().numpy())
    # the reference-facing call with caller-owned host buffers
    m = np.zeros((64, 11), np.float32)
    c = np.zeros(64, np.float32)
    engine.invert_plain(obs, m, chi2=c)
    np.testing.assert_array_equal(m, a["model"])


@pytest.mark.parametrize("nl,psf", [(31, True), (45, True), (60, True)])
def test_inversion_across_grid_sizes(engine, nl, psf):
    """Centred grids of 12 to 60 samples at 35 mA: one sample per lane up to
    32 samples, two above (the kernel's second lane layout), against the
    faithful oracle with the full-inversion tolerances."""
    rng = np.random.default_rng(500 + nl)
    ocfg, gcfg, _ = configs(nl=nl, psf=psf, numerics=1)
    t = H.truth_models(512, rng)
    obs = H.observations(ocfg, t, rng)
    mr, cr, ir, ar, fr = O.lm_batch_f(ocfg, obs, nthreads=0)
    for name, out in H.invert_each_kernel(engine, gcfg, obs):
        ok = close_enough(out["model64"], out["chi2"], mr, cr)
        no_worse = out["chi2"] <= cr * (1 + 1e-3) + 1e-6
        print("nl %d %s: agree %.4f  chi2-no-worse %.4f" % (nl, name, ok.mean(), no_worse.mean()))
        assert ok.mean() >= 0.95, name
        assert (ok | no_worse).mean() >= 0.99, name


def test_twelve_sample_grid(engine):
    """The shortest grid of the benchmark set (12 samples, +-210 mA) cuts the
    wings of strongly split, shifted lines, and the fit is ill-conditioned:
    single LM steps match the faithful oracle as on 30 samples (required:
    99th percentile of the relative step difference < 1e-4), but ~8 % of
    trajectories part after a rounding-level difference (every kernel
    generation here shows the same share).  Where they part, neither side may
    end with the better chi2 systematically: on 2048 pixels the share where
    the engine is worse may exceed the oracle's by at most 2 % (about 2.5
    standard deviations), and the median chi2 agrees within 1 %."""
    rng = np.random.default_rng(512)
    ocfg, gcfg, _ = configs(nl=12, numerics=1)
    t = H.truth_models(2048, rng)
    obs = H.observations(ocfg, t, rng)
    engine.configure(gcfg)
    start = t[:256].copy()
    start[:, 1] = np.clip(start[:, 1] * rng.uniform(0.8, 1.2, 256) + 50, 0, None)
    start[:, 2] += rng.uniform(-0.3, 0.3, 256)
    d, _, _, _ = engine.lm_step(obs[:256], start, 0.1)
    rel = np.array([np.linalg.norm(d[p, :9] - O.lm_step_f(ocfg, start[p], obs[p], 0.1)[0][:9])
                    / max(np.linalg.norm(O.lm_step_f(ocfg, start[p], obs[p], 0.1)[0][:9]), 1e-30)
                    for p in range(256)])
    assert np.percentile(rel, 99) < 1e-4, np.percentile(rel, [50, 99])
    mr, cr, ir, ar, fr = O.lm_batch_f(ocfg, obs, nthreads=0)
    for name, out in H.invert_each_kernel(engine, gcfg, obs):
        mg, cg = out["model64"], out["chi2"]
        agree = close_enough(mg, cg, mr, cr)
        worse_g = ~agree & (cg > cr * (1 + 1e-3) + 1e-6)
        worse_r = ~agree & (cr > cg * (1 + 1e-3) + 1e-6)
        print("nl 12 %s: agree %.4f  engine worse %.4f  oracle worse %.4f  median chi2 %.4f / %.4f"
              % (name, agree.mean(), worse_g.mean(), worse_r.mean(), np.median(cg), np.median(cr)))
        assert agree.mean() >= 0.88, name
        assert worse_g.mean() <= worse_r.mean() + 0.02, name
        assert np.median(cg) == pytest.approx(np.median(cr), rel=0.01), name


@pytest.mark.parametrize("fix", [(1, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0),      # 7 free, S0 S1 fixed
                                 (1, 1, 1, 0, 0, 1, 1, 1, 1, 0, 0)])     # Doppler width, damping fixed
def test_fixed_parameter_sets(engine, fix):
    rng = np.random.default_rng(800)
    ocfg, gcfg, _ = configs(psf=True, fix=fix, numerics=1)
    t = H.truth_models(256, rng)
    t[:, 7] = H.GUESS[7]
    t[:, 8] = H.GUESS[8]
    if not fix[3]:
        t[:, 3] = H.GUESS[3]
        t[:, 4] = H.GUESS[4]
    obs = H.observations(ocfg, t, rng)
    mr, cr, ir, ar, fr = O.lm_batch_f(ocfg, obs)
    for name, out in H.invert_each_kernel(engine, gcfg, obs):
        for i in range(11):
            if not fix[i] and i not in (1, 2, 5, 6):
                assert (out["model64"][:, i] == H.GUESS[i]).all(), name
        assert close_enough(out["model64"], out["chi2"], mr, cr).mean() >= 0.95, name


def test_stray_light_map_per_pixel(engine):
    rng = np.random.default_rng(900)
    fix = (1,) * 9 + (0, 1)
    l0, zo = H.fe_line()
    lam, _ = H.grid()
    ocfg = O.make_cfg(lam, l0, zo, fix=fix, init=H.GUESS)
    base = H.stray_profile(ocfg)
    P = 128
    slmap = (base[None] * rng.uniform(0.9, 1.1, (P, 1, 1))).astype(np.float32)
    t = H.truth_models(P, rng, alpha_range=(0.7, 1.0))
    obs = H.observations(ocfg, t, rng, slight=slmap, slight_per_pixel=True)
    gcfg = G.make_config(lam, l0, G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0), fix=fix, init=H.GUESS,
                         slight=slmap, slight_per_pixel=True, numerics=1)
    mr, cr, ir, ar, fr = O.lm_batch_f(ocfg, obs, slight=slmap, slight_per_pixel=True)
    for name, out in H.invert_each_kernel(engine, gcfg, obs):
        assert close_enough(out["model64"], out["chi2"], mr, cr).mean() >= 0.95, name
        assert np.abs(out["model64"][:, 10] - mr[:, 10]).max() < 0.05, name


@pytest.mark.parametrize("weight,logc", [((1, 0, 0, 1), 0), ((1, 1, 1, 1), 1)])
def test_zero_weights_and_logclambda(engine, weight, logc):
    """Q, U unweighted (azimuth unconstrained) or the log-chi2 damping
    schedule: the GPU fit is as good as the oracle's."""
    rng = np.random.default_rng(1000)
    ocfg, gcfg, _ = configs(weight=weight, logclambda=logc, numerics=1)
    t = H.truth_models(256, rng)
    obs = H.observations(ocfg, t, rng)
    mr, cr, ir, ar, fr = O.lm_batch_f(ocfg, obs)
    for name, out in H.invert_each_kernel(engine, gcfg, obs):
        ok = close_enough(out["model64"], out["chi2"], mr, cr)
        nw = out["chi2"] <= cr * (1 + 1e-3) + 1e-6
        assert (ok | nw).mean() >= 0.95, name
        assert np.median(out["chi2"]) == pytest.approx(np.median(cr), rel=0.02), name


@pytest.mark.parametrize("psf", [False, True])
def test_reference_numerics_fit_quality(engine, psf):
    """With the reference's own intrinsics the trajectories follow the
    reference GPU arithmetic; against the oracle the fits must be equally good:
    same chi2 distribution and the same recovery of the truth."""
    rng = np.random.default_rng(1200)
    ocfg, gcfg, _ = configs(psf=psf, numerics=0)
    t = H.truth_models(1024, rng)
    obs = H.observations(ocfg, t, rng)
    mr, cr, ir, ar, fr = O.lm_batch_f(ocfg, obs)
    rec_r = (np.abs(mr[:, 1] - t[:, 1]) < 50).mean()
    for name, out in H.invert_each_kernel(engine, gcfg, obs):
        assert np.median(out["chi2"]) == pytest.approx(np.median(cr), rel=0.02), name
        rec_g = (np.abs(out["model64"][:, 1] - t[:, 1]) < 50).mean()
        assert abs(rec_g - rec_r) < 0.03, name
        assert abs(out["iters"].mean() - ir.mean()) < 2.0, name


def test_invalid_configurations_are_errors(engine):
    _, gcfg, _ = configs()
    gcfg.noise = 0.0
    with pytest.raises(G.GmError) as e:
        engine.configure(gcfg)
    assert e.value.status == 1
    _, gcfg, _ = configs()
    gcfg.numerics = 7
    with pytest.raises(G.GmError) as e:
        engine.configure(gcfg)
    assert e.value.status == 1


def test_grid_synthesis_matches_synthesis(engine):
    """The fine-grid generator without PSF equals the synthesis kernel on the
    same grid."""
    rng = np.random.default_rng(1100)
    ocfg, gcfg, _ = configs()
    engine.configure(gcfg)
    t = H.truth_models(64, rng)
    a = engine.synthesize(t)
    offs = np.array(ocfg.lambda_[:30]) - ocfg.lambda0
    b = engine.synthesize_grid(t, np.ascontiguousarray(offs))
    assert H.rel_to_I(b, a).max() < 1e-6
