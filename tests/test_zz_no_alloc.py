"""gm_invert_noalloc: the inversion entry point for callers that cannot
allocate device memory (graph-captured or real-time pipelines, frameworks
that own every device byte).  It takes the configuration and device buffers
directly and keeps its scratch in a fixed device array inside the library.

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


def _setup(stray):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(4242 + stray)
    l0, zo = H.fe_line()
    lam, _ = H.grid()
    psf = O.psf_gauss(100.0, lam)
    fix = (1,) * 9 + (0, 1 if stray else 0)
    ocfg = O.make_cfg(lam, l0, zo, psf=psf, fix=fix, init=H.GUESS)
    sl = H.stray_profile(ocfg) if stray else None
    truth = H.truth_models(300, rng, alpha_range=(0.7, 1.0) if stray else None)
    obs = H.observations(ocfg, truth, rng, slight=sl)
    cfg = G.make_config(lam, l0, G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0), psf=psf, fix=fix,
                        init=H.GUESS, slight=sl)
    return torch, cfg, obs


def _noalloc(torch, cfg, obs_dev):
    P, _, nl = obs_dev.shape
    dev = obs_dev.device
    out = {"model": torch.full((P, 11), -1.0, dtype=torch.float32, device=dev),
           "chi2": torch.full((P,), -1.0, dtype=torch.float32, device=dev),
           "iters": torch.full((P,), -1, dtype=torch.int32, device=dev),
           "fitted": torch.zeros((P, 4, nl), dtype=torch.float32, device=dev),
           "status": torch.zeros((P,), dtype=torch.int32, device=dev)}
    stream = torch.cuda.current_stream().cuda_stream
    st = G.lib().gm_invert_noalloc(C.byref(cfg), G._ptr(obs_dev), P, nl, G._ptr(out["model"]),
                                   G._ptr(out["chi2"]), G._ptr(out["iters"]), G._ptr(out["fitted"]),
                                   G._ptr(out["status"]), C.c_void_p(stream))
    assert st == G.GM_OK, G.STATUS_NAMES.get(st, st)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


@pytest.mark.parametrize("stray", [0, 1])
def test_noalloc_matches_gm_invert_twice(stray, monkeypatch):
    """Two calls in a row give the results of the allocating entry point on
    the same (fused) inversion kernel; gm_invert's default wave-synchronous
    kernels agree with it to rounding."""
    torch, cfg, obs = _setup(stray)
    monkeypatch.setenv("GMILOS_INVERT_KERNEL", "fused")
    with G.Engine(0) as eng:
        eng.configure(cfg)
        ref = eng.invert(obs, fitted=True)
    obs_dev = torch.from_numpy(obs).cuda()
    for _ in range(2):
        got = _noalloc(torch, cfg, obs_dev)
        np.testing.assert_allclose(got["model"], ref["model"], rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(got["chi2"], ref["chi2"], rtol=1e-6)
        np.testing.assert_array_equal(got["iters"], ref["iters"])
        np.testing.assert_array_equal(got["status"], ref["status"])
        assert H.rel_to_I(got["fitted"], ref["fitted"]).max() < 1e-6


def test_noalloc_rejects_what_it_cannot_do():
    torch, cfg, obs = _setup(0)
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
    # wrong grid length
    assert lib.gm_invert_noalloc(C.byref(cfg), G._ptr(obs_dev), P, nl + 1, G._ptr(model), None, None,
                                 None, None, None) == 1
    # a grid longer than the scratch and the kernels allow
    big = G.Config.from_buffer_copy(cfg)
    big.nl = G.MAX_NL + 1
    assert lib.gm_invert_noalloc(C.byref(big), G._ptr(obs_dev), P, big.nl, G._ptr(model), None, None,
                                 None, None, None) == 1
