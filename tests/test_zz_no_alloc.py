"""gm_invert_noalloc: the inversion entry point for callers that cannot
allocate device memory -- real-time reduction loops that must not stall on
the allocator, frameworks that own every device byte through their own pool.
It takes the configuration and device buffers directly and keeps its scratch
in a fixed device array inside the library.

Collected last on purpose (file name), so a run that stops at the first
failure has run every other test first.  It must pass alone in a fresh
process and after the other tests, so it assumes nothing about earlier calls.
"""
import ctypes as C

import numpy as np
import pytest

import gmilos_b200 as G
import helpers as H
import oracle as O

pytestmark = pytest.mark.gpu

# (grid samples, stray light: None, "global" profile or "map" per pixel)
CASES = [(30, None), (30, "global"), (45, "global"), (60, "map")]


def _setup(nl, stray, torch):
    rng = np.random.default_rng(4242 + nl + (0 if stray is None else len(stray)))
    l0, zo = H.fe_line()
    lam, _ = H.grid(nl)
    psf = O.psf_gauss(100.0, lam)
    fix = (1,) * 9 + (0, 0 if stray is None else 1)
    ocfg = O.make_cfg(lam, l0, zo, psf=psf, fix=fix, init=H.GUESS)
    P = 300
    truth = H.truth_models(P, rng, alpha_range=None if stray is None else (0.7, 1.0))
    sl = sl_dev = None
    if stray == "global":
        sl = H.stray_profile(ocfg)
    elif stray == "map":
        base = H.stray_profile(ocfg)
        sl = (base[None] * rng.uniform(0.9, 1.1, (P, 1, 1))).astype(np.float32)
        sl_dev = torch.from_numpy(sl).cuda()
    obs = H.observations(ocfg, truth, rng, slight=sl, slight_per_pixel=stray == "map")
    zg = G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0)
    # the allocating entry point on the same (fused) kernel, for comparison
    ref_cfg = G.make_config(lam, l0, zg, psf=psf, fix=fix, init=H.GUESS, slight=sl,
                            slight_per_pixel=stray == "map", kernel=G.KERNEL_FUSED)
    # the no-alloc call: a per-pixel map must already be device memory
    cfg = G.make_config(lam, l0, zg, psf=psf, fix=fix, init=H.GUESS,
                        slight=sl_dev if stray == "map" else sl, slight_per_pixel=stray == "map")
    return cfg, ref_cfg, obs, sl_dev


def _outputs(torch, P, nl):
    dev = "cuda"
    return {"model": torch.full((P, 11), -1.0, dtype=torch.float32, device=dev),
            "chi2": torch.full((P,), -1.0, dtype=torch.float32, device=dev),
            "iters": torch.full((P,), -1, dtype=torch.int32, device=dev),
            "fitted": torch.zeros((P, 4, nl), dtype=torch.float32, device=dev),
            "status": torch.zeros((P,), dtype=torch.int32, device=dev)}


def _call(torch, cfg, obs_dev, out):
    P, _, nl = obs_dev.shape
    stream = torch.cuda.current_stream().cuda_stream
    return G.lib().gm_invert_noalloc(C.byref(cfg), G._ptr(obs_dev), P, nl, G._ptr(out["model"]),
                                     G._ptr(out["chi2"]), G._ptr(out["iters"]), G._ptr(out["fitted"]),
                                     G._ptr(out["status"]), C.c_void_p(stream))


@pytest.mark.parametrize("nl,stray", CASES)
def test_noalloc_matches_gm_invert_twice(nl, stray):
    """Two calls in a row give the results of the allocating entry point on
    the same (fused) inversion kernel, and the calls after the first one
    leave the device's free memory unchanged (nothing allocated)."""
    torch = pytest.importorskip("torch")
    cfg, ref_cfg, obs, _keep = _setup(nl, stray, torch)
    with G.Engine(0) as eng:
        eng.configure(ref_cfg)
        ref = eng.invert(obs, fitted=True)
    obs_dev = torch.from_numpy(obs).cuda()
    P = len(obs)
    outs = [_outputs(torch, P, nl) for _ in range(3)]
    # the first call of the process on this device sets up the scratch
    # address and loads the kernels; it may be this one
    assert _call(torch, cfg, obs_dev, outs[0]) == G.GM_OK
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for k in (1, 2):
        st = _call(torch, cfg, obs_dev, outs[k])
        assert st == G.GM_OK, G.STATUS_NAMES.get(st, st)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0, "a no-alloc call changed the device's free memory"
    for k in (1, 2):
        got = {n: v.cpu().numpy() for n, v in outs[k].items()}
        np.testing.assert_allclose(got["model"], ref["model"], rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(got["chi2"], ref["chi2"], rtol=1e-6)
        np.testing.assert_array_equal(got["iters"], ref["iters"])
        np.testing.assert_array_equal(got["status"], ref["status"])
        # the fitted profile is the last trial's synthesis, as the reference
        # returns its working profile (milosUtils.cu:606); a rejected last
        # trial of a pixel that wandered can be non-finite, in both calls alike
        np.testing.assert_array_equal(np.isfinite(got["fitted"]), np.isfinite(ref["fitted"]))
        fin = np.isfinite(ref["fitted"]).all(axis=(1, 2))
        assert fin.mean() > 0.9
        assert H.rel_to_I(got["fitted"][fin], ref["fitted"][fin]).max() < 1e-6


def test_noalloc_rejects_what_it_cannot_do():
    torch = pytest.importorskip("torch")
    cfg, _, obs, _ = _setup(30, None, torch)
    P, _, nl = obs.shape
    model = torch.empty((P, 11), dtype=torch.float32, device="cuda")
    host_model = np.empty((P, 11), np.float32)
    lib = G.lib()
    # host memory would need staging buffers: rejected
    assert lib.gm_invert_noalloc(C.byref(cfg), G._ptr(obs), P, nl, G._ptr(model), None, None, None,
                                 None, None) == 1
    obs_dev = torch.from_numpy(obs).cuda()
    assert lib.gm_invert_noalloc(C.byref(cfg), G._ptr(obs_dev), P, nl, G._ptr(host_model), None, None,
                                 None, None, None) == 1
    # a per-pixel stray map in host memory
    host_map = np.ones((P, 4, nl), np.float32)
    mcfg = G.make_config(np.asarray(cfg.lambda_[:nl]), cfg.lambda0, cfg.zeeman, slight=host_map,
                         slight_per_pixel=True)
    assert lib.gm_invert_noalloc(C.byref(mcfg), G._ptr(obs_dev), P, nl, G._ptr(model), None, None,
                                 None, None, None) == 1
    # wrong grid length
    assert lib.gm_invert_noalloc(C.byref(cfg), G._ptr(obs_dev), P, nl + 1, G._ptr(model), None, None,
                                 None, None, None) == 1
    # a grid longer than the scratch and the kernels allow
    big = G.Config.from_buffer_copy(cfg)
    big.nl = G.MAX_NL + 1
    assert lib.gm_invert_noalloc(C.byref(big), G._ptr(obs_dev), P, big.nl, G._ptr(model), None, None,
                                 None, None, None) == 1
