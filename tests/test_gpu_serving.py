"""Serving: continuous batching of inversion requests (gm_submit / gm_poll).

Requests of different sizes, memory spaces and free-parameter masks are
submitted together; each must come back exactly (bit for bit) as the same
inversion run alone through gm_invert, because pixels are independent and
the kernel's per-pixel arithmetic does not depend on which launch, lane or
chunk carried it.  Admission against the HBM budget, cancellation and the
reported latencies are checked too."""
import threading
import time

import numpy as np
import pytest

import gmilos_b200 as G
import helpers as H
import oracle as O

pytestmark = pytest.mark.gpu

FIX9A = (1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 1)
FIX7A = (1, 1, 1, 1, 1, 1, 1, 0, 0, 0, 1)     # S0, S1 fixed


def config(fix=FIX9A, **kw):
    lam, _ = H.grid(30)
    l0, zo = H.fe_line()
    psf = O.psf_gauss(100.0, lam)
    ocfg = O.make_cfg(lam, l0, zo, psf=psf, fix=FIX9A)
    sl = H.stray_profile(ocfg)
    gcfg = G.make_config(lam, l0, G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0), psf=psf, fix=fix,
                         init=H.GUESS, slight=sl, **kw)
    return ocfg, gcfg, sl


def cube(n, seed):
    ocfg, _, sl = config()
    rng = np.random.default_rng(seed)
    t = H.truth_models(n, rng, alpha_range=(0.7, 1.0))
    return H.observations(ocfg, t, rng, slight=sl)


def alone(obs, fix):
    _, gcfg, _ = config(fix)
    with G.Engine(0) as e:
        e.configure(gcfg)
        out = e.invert(obs)
    return out


def test_results_are_the_same_alone_and_in_the_mix():
    import torch
    sizes = [1, 37, 5000, 70000, 300, 9000]
    fixes = [FIX9A, FIX7A, FIX9A, FIX7A, FIX9A, FIX7A]
    data = [cube(n, 100 + k) for k, n in enumerate(sizes)]
    _, gcfg, _ = config()
    with G.Engine(0) as e:
        e.configure(gcfg)
        e.serving_options(streams=4, chunk_pixels=4096, max_active=3)
        reqs = []
        for k, (obs, fix) in enumerate(zip(data, fixes)):
            if k % 2:   # device buffers
                d = torch.tensor(obs, device="cuda")
                model = torch.empty((len(obs), 11), dtype=torch.float32, device="cuda")
                chi2 = torch.empty(len(obs), dtype=torch.float32, device="cuda")
                iters = torch.empty(len(obs), dtype=torch.int32, device="cuda")
                src = d
            else:       # host buffers
                src = obs
                model = np.empty((len(obs), 11), np.float32)
                chi2 = np.empty(len(obs), np.float32)
                iters = np.empty(len(obs), np.int32)
            t = e.submit(src, model, chi2=chi2, iters=iters, fix=fix)
            reqs.append((t, src, model, chi2, iters))
        lat = []
        for t, src, model, chi2, iters in reqs:
            assert e.poll(t) == 0
            lat.append((e.last_latency_ms, e.last_queue_ms))
    for k, (t, src, model, chi2, iters) in enumerate(reqs):
        ref = alone(data[k], fixes[k])
        m = model.cpu().numpy() if hasattr(model, "cpu") else model
        c = chi2.cpu().numpy() if hasattr(chi2, "cpu") else chi2
        it = iters.cpu().numpy() if hasattr(iters, "cpu") else iters
        np.testing.assert_array_equal(m, ref["model"])
        np.testing.assert_array_equal(c, ref["chi2"])
        np.testing.assert_array_equal(it, ref["iters"])
    for latency, queued in lat:
        assert latency > 0 and 0 <= queued <= latency


def test_admission_against_the_hbm_budget():
    obs = cube(2000, 7)
    per_request = obs.nbytes + 2000 * (11 * 4 + 4 + 4)
    _, gcfg, _ = config()
    with G.Engine(0, hbm_budget=int(per_request * 1.5)) as e:
        e.configure(gcfg)
        outs = []
        for k in range(4):   # only one fits at a time: they run one after another
            m = np.empty((len(obs), 11), np.float32)
            c = np.empty(len(obs), np.float32)
            it = np.empty(len(obs), np.int32)
            # every buffer of a request stays alive until its poll returns
            outs.append((e.submit(obs, m, chi2=c, iters=it), m, c, it))
        for t, m, c, it in outs:
            assert e.poll(t) == 0
        for t, m, c, it in outs[1:]:
            np.testing.assert_array_equal(m, outs[0][1])
        big = cube(5000, 8)
        with pytest.raises(G.GmError) as err:
            e.submit(big, np.empty((5000, 11), np.float32))
        assert err.value.status == 3


def test_cancel_and_poll_timeout():
    obs = cube(20000, 9)
    _, gcfg, _ = config()
    with G.Engine(0) as e:
        e.configure(gcfg)
        e.serving_options(streams=2, chunk_pixels=65536, max_active=1)
        bufs = [np.empty((len(obs), 11), np.float32) for _ in range(3)]
        ts = [e.submit(obs, b) for b in bufs]
        e.cancel(ts[2])                      # still queued behind the first
        assert e.poll(ts[2]) == 7            # cancelled
        assert e.poll(ts[0]) == 0 and e.poll(ts[1]) == 0
        np.testing.assert_array_equal(bufs[0], bufs[1])
        t = e.submit(obs, bufs[2])
        st = e.poll(t, timeout_us=1)
        assert st in (0, 6)
        assert e.poll(t) == 0


def test_concurrent_submitters():
    """Several host threads submitting and polling at once."""
    data = [cube(3000 + 500 * k, 200 + k) for k in range(6)]
    _, gcfg, _ = config()
    results = {}
    with G.Engine(0) as e:
        e.configure(gcfg)

        def worker(k):
            m = np.empty((len(data[k]), 11), np.float32)
            t = e.submit(data[k], m)
            assert e.poll(t) == 0
            results[k] = m

        th = [threading.Thread(target=worker, args=(k,)) for k in range(6)]
        for x in th:
            x.start()
        for x in th:
            x.join(timeout=120)
    for k in range(6):
        np.testing.assert_array_equal(results[k], alone(data[k], FIX9A)["model"])


@pytest.mark.parametrize("policy", [G.SERVE_FIFO, G.SERVE_SHORTEST_FIRST, G.SERVE_RESPONSE_RATIO])
def test_every_policy_gives_the_lone_results(policy):
    """The serving policies decide only which request's chunk a free lane
    takes next: results stay those of each request inverted alone, and the
    shortest-first and response-ratio policies finish a small request
    submitted after a large one first."""
    sizes = [60000, 500, 3000]
    data = [cube(n, 200 + k) for k, n in enumerate(sizes)]
    _, gcfg, _ = config()
    with G.Engine(0) as e:
        e.configure(gcfg)
        e.serving_options(streams=2, chunk_pixels=4096, max_active=4)
        e.serving_policy(policy)
        outs = [(np.empty((n, 11), np.float32), np.empty(n, np.float32)) for n in sizes]
        tickets = [e.submit(d, o[0], chi2=o[1]) for d, o in zip(data, outs)]
        lat = []
        for t in tickets:
            assert e.poll(t) == 0
            lat.append(e.last_latency_ms)
        with pytest.raises(G.GmError):
            e.serving_policy(7)
    for d, (model, chi2) in zip(data, outs):
        ref = alone(d, FIX9A)
        np.testing.assert_array_equal(model, ref["model"])
        np.testing.assert_array_equal(chi2, ref["chi2"])
    if policy in (G.SERVE_SHORTEST_FIRST, G.SERVE_RESPONSE_RATIO):
        assert lat[1] < lat[0]
