#!/usr/bin/env python
"""Headline benchmark: converged pixels/s of the Milne-Eddington inversion.

Workload (the reference's full-cube case): 1024 x 1024 pixels x 4 Stokes x
30 wavelengths (Fe I 6173.3356 A, -350:35:665 mA), FP32, normalised to the
continuum.  Truth parameters drawn uniformly (eta0 1-30, B 0-3000 G, vlos
+-3 km/s, Doppler width 20-60 mA, damping 0-0.5, gamma/phi 0-180 deg,
S0 0.1-0.5, S1 0.3-1.0 rescaled to unit continuum), stray light of 0-30 %
(filling factor alpha 0.7-1.0) against a fixed field-free profile.  The
observations are synthesised on a 1 mA grid, convolved with a Gaussian PSF
of FWHM 100 mA sampled at 1 mA, resampled to the 30 samples, plus Gaussian
noise of 1e-3 Ic.  The inversion fits 9 ME parameters + alpha with at most 50
LM iterations, PSF and stray light modelled with the reference's semantics
(the 1 mA PSF table linearly interpolated at the grid offsets).  Synthetic
data stand in for an observed cube.

One step = one inversion of the whole cube.  Inputs (480 MB) exceed the
126 MB L2, so no flush is needed between steps.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (os.path.join(ROOT, "g-milos_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

LAMBDA0 = 6173.3356
GRID = (-350.0, 35.0, 665.0)
FWHM_MA = 100.0
NOISE = 1e-3
GUESS = (40.0, 1000.0, 0.2, 0.03, 0.05, 150.0, 110.0, 0.35, 0.5, 0.0, 1.0)   # run/guess.mod
FIX = (1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 1)          # 9 ME parameters + alpha
STRAY_MODEL = (10.0, 0.0, 0.0, 0.03, 0.1, 0.0, 0.0, 0.3, 0.7, 0.0, 1.0)
# --vmac-free: the reference's 11-term path (v_mac and alpha both free), v_mac starting at 0.5 km/s
FIX11 = (1,) * 11
GUESS_VMAC = GUESS[:9] + (0.5, 1.0)
MAXITER = 50

# DRAM bytes (read + write) per pixel of one inversion (classical pre-pass
# and every trial / accept wave), measured with ncu (dram__bytes_read.sum +
# dram__bytes_write.sum summed over the 102 launches of an inversion) on
# 65 536-pixel inversions of this workload with the current kernels;
# traffic grows with the pixel count.
DRAM_BYTES_PER_PIXEL = 206500.0

# Algorithmic FLOPs per pixel (per-wavelength costs counted from the formulas)
C_VOIGT, C_RTE, C_DVOIGT, C_DRTE = 100, 85, 23, 870


def flops_model(nl, ntaps, n_free, s0_free, psf, stray, ncomp=3):
    """Algorithmic FLOPs of one pixel: F_trial (one synthesis + chi2 + solve),
    F_acc (response functions + normal equations at an accepted model) and
    F_init (classical estimates + the initial synthesis and RF)."""
    n = n_free
    n_conv = n - (1 if s0_free else 0)
    f_trial = nl * (ncomp * C_VOIGT + C_RTE) + (8 * nl * ntaps if psf else 0) + (12 * nl if stray else 0) \
        + 12 * nl + (n ** 3 / 3 + 2 * n ** 2)
    f_acc = nl * (ncomp * C_DVOIGT + C_DRTE) + (8 * nl * ntaps * n_conv if psf else 0) \
        + (4 * nl * n if stray else 0) + 8 * nl * (n * (n + 1) / 2 + n)
    f_init = 40 * nl + f_trial + f_acc
    return f_trial, f_acc, f_init


def truth_models(n, rng):
    t = np.zeros((n, 11))
    t[:, 0] = rng.uniform(1, 30, n)
    t[:, 1] = rng.uniform(0, 3000, n)
    t[:, 2] = rng.uniform(-3, 3, n)
    t[:, 3] = rng.uniform(0.020, 0.060, n)
    t[:, 4] = rng.uniform(0, 0.5, n)
    t[:, 5] = rng.uniform(0, 180, n)
    t[:, 6] = rng.uniform(0, 180, n)
    t[:, 7] = rng.uniform(0.1, 0.5, n)
    t[:, 8] = rng.uniform(0.3, 1.0, n)
    ic = t[:, 7] + t[:, 8]
    t[:, 7] /= ic
    t[:, 8] /= ic
    t[:, 10] = rng.uniform(0.7, 1.0, n)
    return t


def grid():
    first, step, last = GRID
    n = int(((last - first) / step) + 1)
    off = np.empty(n)
    off[0] = first
    lam = np.empty(n)
    lam[0] = LAMBDA0 + first / 1000.0
    for i in range(1, n):
        off[i] = off[i - 1] + step
        lam[i] = lam[i - 1] + step / 1000.0
    return lam, off


def psf_table():
    """Gaussian PSF of FWHM 100 mA sampled at 1 mA over +-2750 mA (the layout
    of the reference's .psf files)."""
    x = np.arange(-2750.0, 2750.5, 1.0)
    sigma = FWHM_MA / (2 * np.sqrt(2 * np.log(2)))
    return x, np.exp(-0.5 * (x / sigma) ** 2)


def fine_operator(off):
    """Fine 1 mA grid covering the samples +-6 sigma, and the matrix that
    convolves a fine profile with the PSF and samples it at `off`."""
    sigma = FWHM_MA / (2 * np.sqrt(2 * np.log(2)))
    half = int(np.ceil(6 * sigma))
    fine = np.arange(off[0] - half, off[-1] + half + 0.5, 1.0)
    W = np.exp(-0.5 * ((off[:, None] - fine[None, :]) / sigma) ** 2)
    W /= W.sum(axis=1, keepdims=True)
    return fine, W


# ----------------------------------------------------------------- engine arm
def clocks_sampler(dev_index, stop, out):
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    try:
        p = subprocess.Popen(["nvidia-smi", "-i", str(dev_index), "--query-gpu=" + q,
                              "--format=csv,noheader,nounits", "-lms", "200"],
                             stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    except Exception:
        return
    while not stop.is_set():
        line = p.stdout.readline()
        if not line:
            break
        out.append(line.strip())
    p.terminate()


def summarize_clocks(lines):
    sm, mx, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for l in lines:
        f = [x.strip() for x in l.split(",")]
        if len(f) < 9:
            continue
        try:
            sm.append(float(f[1]))
            mx.append(float(f[2]))
        except ValueError:
            continue
        for i, n in enumerate(names):
            if f[5 + i].lower().startswith("active"):
                reasons.add(n)
    if not sm:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
    return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
            "samples": len(sm)}


def make_cube_gpu(eng, truth, off, slight, rng_seed, torch):
    """Observations on the device: fine-grid ME synthesis by the engine's grid
    kernel, PSF convolution + resampling as one matmul, stray mix, noise."""
    fine, W = fine_operator(off)
    fine_A = np.ascontiguousarray(fine / 1000.0)
    Wt = torch.tensor(W.T, dtype=torch.float32, device="cuda")
    P = truth.shape[0]
    nl = len(off)
    out = torch.empty((P, 4, nl), dtype=torch.float32, device="cuda")
    tm = torch.tensor(truth, dtype=torch.float64, device="cuda")
    offs_d = torch.tensor(fine_A, dtype=torch.float64, device="cuda")
    chunk = 32768
    for a in range(0, P, chunk):
        b = min(P, a + chunk)
        f = eng.synthesize_grid(tm[a:b].contiguous(), offs_d)
        out[a:b] = torch.matmul(f, Wt)
        del f
    alpha = tm[:, 10].to(torch.float32)[:, None, None]
    sl = torch.tensor(slight, dtype=torch.float32, device="cuda")[None]
    out = alpha * out + (1 - alpha) * sl
    g = torch.Generator(device="cuda")
    g.manual_seed(rng_seed)
    out += NOISE * torch.randn(out.shape, generator=g, device="cuda", dtype=torch.float32)
    torch.cuda.synchronize()
    return out.contiguous()


def stray_profile_cpu(off):
    """Field-free ME profile seen through the same 1 mA PSF (the fixed stray
    light source), computed with the engine-independent CPU oracle only for
    the reference arm; the engine arm computes it with the engine."""
    import oracle as O
    return _fine_synth_cpu(O, np.array([STRAY_MODEL]), off)[0]


def _fine_synth_cpu(O, models, off):
    l0, z = O.fe6173()
    fine, W = fine_operator(off)
    P = models.shape[0]
    prof = np.zeros((P, 4, len(fine)), dtype=np.float32)
    for a in range(0, len(fine), 128):
        b = min(len(fine), a + 128)
        lam = LAMBDA0 + fine[a:b] / 1000.0
        if b - a < 2:
            lam = np.array([lam[0], lam[0] + 1e-3])
        cfg = O.make_cfg(lam, l0, z)
        prof[:, :, a:b] = O.synth_batch_f(cfg, models)[:, :, :b - a]
    return (prof @ W.T.astype(np.float32)).astype(np.float32)


def run_engine(args):
    import torch
    import torch.distributed as dist
    import gmilos_b200 as G

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    lam, off = grid()
    x, y = psf_table()
    psf = G.psf_from_table(x, y, off, GRID[1])
    eng = G.Engine(local)
    zee = G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0)
    # stray profile: ME synthesis of the field-free model through the 1 mA PSF
    cfg0 = G.make_config(lam, LAMBDA0, zee, fix=FIX, init=GUESS)
    eng.configure(cfg0)
    fine, W = fine_operator(off)
    sl_fine = eng.synthesize_grid(np.array([STRAY_MODEL]), np.ascontiguousarray(fine / 1000.0))
    slight = (sl_fine @ W.T.astype(np.float32))[0].astype(np.float32)
    fix, guess = (FIX11, GUESS_VMAC) if args.vmac_free else (FIX, GUESS)
    cfg = G.make_config(lam, LAMBDA0, zee, psf=psf, fix=fix, init=guess, miter=MAXITER, slight=slight)
    eng.configure(cfg)

    rng = np.random.default_rng(args.seed + rank)
    P = args.pixels
    truth = truth_models(P, rng)
    obs = make_cube_gpu(eng, truth, off, slight, args.seed + 1000 + rank, torch)
    nl = len(off)
    dev = obs.device
    outs = {"model": torch.empty((P, 11), dtype=torch.float32, device=dev),
            "model64": None,
            "chi2": torch.empty(P, dtype=torch.float32, device=dev),
            "iters": torch.empty(P, dtype=torch.int32, device=dev),
            "accepted": torch.empty(P, dtype=torch.int32, device=dev),
            "status": torch.empty(P, dtype=torch.int32, device=dev),
            "fitted": None}
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    for _ in range(args.warmup):
        eng.invert(obs, out=outs, stream=sptr)
    torch.cuda.synchronize()

    stop = threading.Event()
    clk = []
    th = threading.Thread(target=clocks_sampler, args=(local, stop, clk), daemon=True)
    th.start()
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    iters_sum = 0
    acc_sum = 0
    t_start.record(stream)
    for k in range(args.steps):
        evs[k][0].record(stream)
        eng.invert(obs, out=outs, stream=sptr)
        evs[k][1].record(stream)
    t_end.record(stream)
    torch.cuda.synchronize()
    launches_per_step = int(eng.stats()["kernel_launches"])
    if world > 1:
        dist.barrier()
    stop.set()
    iters_sum = int(outs["iters"].sum().item())
    acc_sum = int(outs["accepted"].sum().item())
    total_ms = t_start.elapsed_time(t_end)
    launch_ms = [a.elapsed_time(b) for a, b in evs]
    ms_t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    total_ms = float(ms_t.item())
    ms_per_step = total_ms / args.steps
    value = P * world / (ms_per_step / 1e3)

    # end to end through the public C ABI with pinned host buffers
    obs_h = obs.cpu().pin_memory()
    model_h = torch.empty((P, 11), dtype=torch.float32).pin_memory()
    chi_h = torch.empty(P, dtype=torch.float32).pin_memory()
    it_h = torch.empty(P, dtype=torch.int32).pin_memory()
    e2e_ms = []
    for k in range(max(1, min(args.steps, 3)) + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng.invert_plain(obs_h.numpy(), model_h.numpy(), chi2=chi_h.numpy(), iters=it_h.numpy())
        t1 = time.perf_counter()
        if k > 0:
            e2e_ms.append((t1 - t0) * 1e3)
    e2e_t = torch.tensor([float(np.mean(e2e_ms))], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = P * world / (float(e2e_t.item()) / 1e3)
    h2d = obs_h.numel() * 4
    d2h = (model_h.numel() + chi_h.numel() + it_h.numel()) * 4

    # roofline of the inversion kernel: algorithmic FLOPs / launch duration
    ftr, facc, finit = flops_model(nl, nl, n_free=sum(fix), s0_free=fix[7], psf=True, stray=True)
    flops_launch = P * finit + iters_sum * ftr + acc_sum * facc
    launch_avg = float(np.mean(launch_ms))
    achieved = flops_launch / (launch_avg / 1e3) / 1e12
    fp32_peak, fp64_peak = eng.measure_peaks()
    # special-function side: MUFU operations per sample (10 per trial, 5 per
    # accepted step) plus the 2 sincos of the field angles per trial; the
    # initial point counts as one trial and one accepted step
    sfu_launch = (iters_sum + P) * (10 * nl + 4) + (acc_sum + P) * 5 * nl
    sfu_achieved = sfu_launch / (launch_avg / 1e3) / 1e9
    sfu_peak = eng.measure_sfu_peak()
    clocks = summarize_clocks(clk)

    result = {
        "metric": METRIC,
        "value": value, "unit": "pixels/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (f64 Voigt polynomials and model parameters)", "data": "synthetic",
        "config": {"workload": "full cube %dx%d px x 4 Stokes x 30 lambda, Fe I 6173 A, PSF FWHM 100 mA "
                               "(1 mA table), stray light alpha 0.7-1.0, noise 1e-3 Ic" % (int(np.sqrt(P)), int(np.sqrt(P))) if int(np.sqrt(P)) ** 2 == P
                               else "%d px x 4 x 30 lambda, PSF, stray light" % P,
                   "pixels_per_gpu": P, "nlambda": nl, "free_parameters": int(sum(fix)), "max_iterations": MAXITER,
                   "terms": 11 if args.vmac_free else 10,
                   "mean_iterations": iters_sum / P, "mean_accepted": acc_sum / P,
                   "l2_policy": "inputs 480 MB per GPU > 126 MB L2, no flush", "parallelism": "replicas (weak scaling, no collective)"},
        "e2e": {"value": e2e_value, "unit": "pixels/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches_per_step * args.steps,
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                     "frac": achieved / fp32_peak if fp32_peak else None,
                     "traffic": DRAM_BYTES_PER_PIXEL * P,
                     "traffic_note": "bytes per inversion (pre-pass + trial/accept waves), scaled from an ncu "
                                     "capture of a 65536-pixel inversion",
                     "kernels": "one step = classical pre-pass + %d trial_kernel / accept_kernel launches "
                                "(wave-synchronous LM); achieved = algorithmic FLOPs / the step's device time"
                                % (launches_per_step - 1),
                     "peak_source": "measured FFMA microbenchmark (gm_measure_peaks), burst",
                     "fp64_peak": fp64_peak,
                     "flops_per_launch": flops_launch, "launch_ms": launch_avg,
                     "sfu": {"ops_per_launch": sfu_launch, "achieved": sfu_achieved, "peak": sfu_peak,
                             "unit": "G MUFU ops/s", "frac": sfu_achieved / sfu_peak if sfu_peak else None,
                             "peak_source": "measured ex2.approx chains (gm_measure_sfu_peak), burst"}},
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(obs[: min(P, 200000)].cpu().numpy(), slight, psf, lam, seconds=args.cpu_seconds)
    if rank == 0 and world == 1 and args.serve_requests > 0:
        result["latency"] = serving_latency(eng, obs_h, args)
    if rank == 0 and world == 1 and args.ref_gpu_pixels > 0:
        import ref
        n = min(P, args.ref_gpu_pixels)
        if ref.available(gpu=True):
            try:
                rg = reference_gpu(obs[:n].cpu().numpy(), slight, psf, lam, nstreams=args.ref_gpu_streams)
                rep = rg["report"]
                cmp_ = _fit_comparison(outs["model"][:n].double().cpu().numpy(), outs["chi2"][:n].cpu().numpy(),
                                       outs["iters"][:n].cpu().numpy(), rg["model"], rg["chi2"], rg["iters"])
                host_vs_gpu = None
                if ref.available():
                    # the reference's own host build on the same pixels: how
                    # far two builds of the reference itself agree
                    s, _ = _ref_setup(lam, psf)
                    mh, ch, ih, _ = ref.invert_cpu(s, obs[:n].cpu().numpy(), slight=slight,
                                                   nthreads=os.cpu_count())
                    host_vs_gpu = _fit_comparison(mh, ch, ih, rg["model"], rg["chi2"], rg["iters"],
                                                  names=("host_build", "gpu_build"))
                result["reference_gpu"] = {
                    "what": "the reference's own lm_mils built for sm_100a (child launches run in-thread), "
                            "its launch geometry, streams and device heap, same cube",
                    "value": rg["value"], "e2e": rg["e2e"], "unit": "pixels/s",
                    "sample": "first %d pixels of the same cube" % n,
                    "geometry": {"blocks_per_stream": rep["num_blocks"], "threads_per_block": rep["threads_per_block"],
                                 "streams": rep["nstreams"], "registers": rep["regs"],
                                 "stack_bytes": rep["local_bytes"]},
                    "speedup_value": value / rg["value"], "speedup_e2e": e2e_value / rg["e2e"],
                    "fit_vs_engine": cmp_,
                    "reference_host_vs_gpu": host_vs_gpu}
            except Exception as exc:  # the comparison must not take the bench line down
                result["reference_gpu"] = {"unavailable": str(exc)[:200]}
        else:
            result["reference_gpu"] = {"unavailable": "oracle/_ref/libgmref_gpu.so not built"}
    if rank == 0 and world == 1 and args.config1:
        result["config1"] = config1_block(eng, args, torch)
    if rank == 0 and world == 1 and args.ragged_rois > 0:
        try:
            result["ragged"] = ragged_block(eng, args, torch)
        except Exception as exc:  # the block must not take the bench line down
            result["ragged"] = {"unavailable": str(exc)[:300]}
    if rank == 0 and world == 1 and args.mlp_train_pixels > 0:
        try:
            result["learned_init"] = learned_block(eng, args, torch)
        except Exception as exc:  # the block must not take the bench line down
            result["learned_init"] = {"unavailable": str(exc)[:300]}
    if rank == 0:
        print(json.dumps(result), flush=True)
    eng.close()
    if world > 1:
        dist.destroy_process_group()


def serving_latency(eng, obs_h, args, rate=None, n=None):
    """Serving under load: a Poisson stream of inversion requests, frames of
    side uniform in [side_min, side_max] px x 4 x 30 lambda with PSF and
    stray light, half of them with S0 and S1 fixed (7 ME + alpha free instead
    of 9 + alpha), host buffers in and out (pinned), through the engine's
    continuous-batching entry points (gm_submit / gm_poll).  Latency is
    submit -> results in host memory, taken by the engine.  Frames are cut
    from the bench cube, tiled when a frame is larger than the cube.  Beside
    the latency percentiles: per frame-size class, and the stretch (latency
    over the frame's inversion time at the engine's unloaded rate), which
    takes the frame size out."""
    import torch
    rate = args.serve_rate if rate is None else rate
    n = args.serve_requests if n is None else n
    rng = np.random.default_rng(args.seed + 77 + int(rate * 100))
    sides = rng.integers(args.serve_side_min, args.serve_side_max + 1, n)
    npix = (sides.astype(np.int64) ** 2)
    fix7 = (1, 1, 1, 1, 1, 1, 1, 0, 0, 0, 1)
    mixes = [FIX if k % 2 == 0 else fix7 for k in range(n)]
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
    P = obs_h.shape[0]
    reps = int(np.ceil(npix.max() / P))
    pool = obs_h if reps <= 1 else torch.cat([obs_h] * reps).pin_memory()
    starts = rng.integers(0, max(1, pool.shape[0] - int(npix.max()) + 1), n)
    outs = [(torch.empty((int(k), 11), dtype=torch.float32).pin_memory(),
             torch.empty(int(k), dtype=torch.float32).pin_memory(),
             torch.empty(int(k), dtype=torch.int32).pin_memory()) for k in npix]
    tickets = [None] * n
    t0 = time.perf_counter()
    for k in range(n):
        delay = t0 + arrivals[k] - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        frame = pool[int(starts[k]): int(starts[k]) + int(npix[k])]
        tickets[k] = eng.submit(frame, outs[k][0], chi2=outs[k][1], iters=outs[k][2], fix=mixes[k])
    lat, queue = [], []
    for k in range(n):
        st = eng.poll(tickets[k])
        if st != 0:
            raise RuntimeError("serving request %d failed with status %d" % (k, st))
        lat.append(eng.last_latency_ms)
        queue.append(eng.last_queue_ms)
    t_end = t0 + max(arrivals[k] + lat[k] / 1e3 for k in range(n))
    lat = np.array(lat)
    span = t_end - t0
    alone_ms = npix / args.serve_unloaded_rate * 1e3
    stretch = lat / alone_ms
    edges = np.linspace(args.serve_side_min, args.serve_side_max + 1, 5)
    classes = []
    for a, b in zip(edges[:-1], edges[1:]):
        m = (sides >= a) & (sides < b)
        if m.sum():
            classes.append({"sides": [int(a), int(b) - 1], "requests": int(m.sum()),
                            "p50_ms": float(np.percentile(lat[m], 50)), "p99_ms": float(np.percentile(lat[m], 99))})
    return {"what": "Poisson stream of %d requests at %.2f req/s, frames %d^2-%d^2 px x 4 x 30 lambda, "
                    "PSF + stray light, half with S0/S1 fixed; host buffers; continuous batching "
                    "(%d lanes, %d-pixel chunks, %s policy, HBM budget %s)"
                    % (n, rate, args.serve_side_min, args.serve_side_max, 4, 65536, args.serve_policy,
                       "%d GB" % args.serve_budget_gb if args.serve_budget_gb else "whole device"),
            "rate": rate, "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "p99_over_p50": float(np.percentile(lat, 99) / np.percentile(lat, 50)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max()),
            "mean_queue_ms": float(np.mean(queue)),
            "stretch_p50": float(np.percentile(stretch, 50)), "stretch_p99": float(np.percentile(stretch, 99)),
            "by_size": classes,
            "pixels_per_s": float(npix.sum() / span), "offered_pixels_per_s": float(npix.sum() / arrivals[-1]),
            "requests": n, "pixels": int(npix.sum())}


SERVE_POLICIES = {"round_robin": 0, "fifo": 1, "shortest_first": 2, "response_ratio": 3}


def run_serve_sweep(args):
    """--serve-sweep: the serving stream at each of the given arrival rates,
    on a context whose HBM budget is --serve-budget-gb, one JSON line."""
    import torch
    import gmilos_b200 as G
    torch.cuda.set_device(0)
    lam, off = grid()
    x, y = psf_table()
    psf = G.psf_from_table(x, y, off, GRID[1])
    eng = G.Engine(0, hbm_budget=int(args.serve_budget_gb) << 30)
    zee = G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0)
    eng.configure(G.make_config(lam, LAMBDA0, zee, fix=FIX, init=GUESS))
    fine, W = fine_operator(off)
    sl_fine = eng.synthesize_grid(np.array([STRAY_MODEL]), np.ascontiguousarray(fine / 1000.0))
    slight = (sl_fine @ W.T.astype(np.float32))[0].astype(np.float32)
    eng.configure(G.make_config(lam, LAMBDA0, zee, psf=psf, fix=FIX, init=GUESS, miter=MAXITER, slight=slight))
    eng.serving_policy(SERVE_POLICIES[args.serve_policy])
    P = args.pixels
    rng = np.random.default_rng(args.seed)
    obs = make_cube_gpu(eng, truth_models(P, rng), off, slight, args.seed + 1000, torch)
    obs_h = obs.cpu().pin_memory()
    del obs
    rates = [float(r) for r in args.serve_sweep.split(",")]
    out = {"metric": "serving latency", "policy": args.serve_policy, "budget_gb": args.serve_budget_gb,
           "unloaded_rate_pixels_per_s": args.serve_unloaded_rate, "sweep": []}
    for r in rates:
        out["sweep"].append(serving_latency(eng, obs_h, args, rate=r, n=args.serve_requests))
    print(json.dumps(out), flush=True)
    eng.close()


FIX9 = (1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0)         # the 9 ME parameters


def config1_block(eng, args, torch, reps=10):
    """The reference's CPU-runnable case as specified: a 64 x 64 px cube x 4
    Stokes x 30 lambda on the same grid and line, truth drawn from the same
    ranges, noise 1e-3 Ic, no PSF, no stray light, 9 free parameters, at
    most 50 iterations.  The engine inverts it device-resident (CUDA-event
    time) and end to end from host memory (gm_invert); the reference's own
    per-pixel routines, built host-side, invert the whole cube on every host
    thread.  Both fits are compared pixel by pixel."""
    import gmilos_b200 as G
    import ref
    lam, off = grid()
    zee = G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0)
    cfg = G.make_config(lam, LAMBDA0, zee, fix=FIX9, init=GUESS, miter=MAXITER)
    eng.configure(cfg)
    rng = np.random.default_rng(args.seed + 64)
    P = 64 * 64
    truth = truth_models(P, rng)
    truth[:, 10] = 1.0
    obs = eng.synthesize(truth)
    obs = np.ascontiguousarray(obs + rng.normal(0, NOISE, obs.shape).astype(np.float32))
    obs_d = torch.from_numpy(obs).cuda()
    stream = torch.cuda.current_stream()
    out = None
    for _ in range(3):
        out = eng.invert(obs_d, out=out, stream=stream.cuda_stream)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    torch.cuda.synchronize()
    evs[0].record(stream)
    for _ in range(reps):
        eng.invert(obs_d, out=out, stream=stream.cuda_stream)
    evs[1].record(stream)
    torch.cuda.synchronize()
    dev_ms = evs[0].elapsed_time(evs[1]) / reps
    obs_h = torch.from_numpy(obs).pin_memory()
    model_h = torch.empty((P, 11), dtype=torch.float32).pin_memory()
    chi_h = torch.empty(P, dtype=torch.float32).pin_memory()
    it_h = torch.empty(P, dtype=torch.int32).pin_memory()
    e2e = []
    for k in range(reps + 1):
        t0 = time.perf_counter()
        eng.invert_plain(obs_h.numpy(), model_h.numpy(), chi2=chi_h.numpy(), iters=it_h.numpy())
        if k:
            e2e.append(time.perf_counter() - t0)
    res = {"workload": "64x64 px x 4 Stokes x 30 lambda, no PSF, no stray light, 9 free, <= 50 iterations, "
                       "noise 1e-3 Ic",
           "engine": {"value": P / (dev_ms / 1e3), "unit": "pixels/s", "ms": dev_ms,
                      "e2e": P / float(np.mean(e2e)), "mean_iterations": float(out["iters"].float().mean())}}
    if ref.available():
        import oracle as O
        l0, z = O.fe6173()
        s = ref.setup_from_cfg(O.make_cfg(lam, l0, z, fix=FIX9, init=GUESS, miter=MAXITER))
        nthreads = os.cpu_count()
        times = []
        for k in range(3):
            t0 = time.perf_counter()
            mr, cr, ir, _ = ref.invert_cpu(s, obs, nthreads=nthreads)
            times.append(time.perf_counter() - t0)
        cpu_value = P / float(np.mean(times))
        res["reference_cpu"] = {"value": cpu_value, "unit": "pixels/s", "cores": nthreads,
                                "kind": "reference", "sample": "the whole 4096-pixel cube, 3 runs"}
        res["speedup_e2e_vs_reference_cpu"] = res["engine"]["e2e"] / cpu_value
        res["fit_vs_reference"] = _fit_comparison(out["model64"].cpu().numpy(), out["chi2"].cpu().numpy(),
                                                  out["iters"].cpu().numpy(), mr, cr, ir)
    return res


def ragged_block(eng, args, torch):
    """Ragged batch: 64 ROIs, side lengths uniform in 16-512 px, centred
    35 mA grids of 12-60 samples (same line, truth ranges, noise 1e-3 Ic, no
    PSF), early stop at an accepted chi2 gain below 1e-4, 9 free, <= 50
    iterations.  The whole batch goes to gm_invert_rois: one persistent
    launch sequence per samples-per-lane class, autotuned on the first call,
    then timed direct and as a replayed CUDA graph; beside it the same ROIs
    inverted one gm_invert call each on their own grid."""
    import gmilos_b200 as G
    rng = np.random.default_rng(args.seed + 3)
    zee = G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0)
    dev = torch.device("cuda")
    lam30, _ = grid()
    eng.configure(G.make_config(lam30, LAMBDA0, zee, fix=FIX9, init=GUESS, miter=MAXITER))
    rois = []
    for k in range(args.ragged_rois):
        side = int(rng.integers(16, 513))
        nl = int(rng.integers(12, 61))
        off = 35.0 * (np.arange(nl) - nl // 2)
        lam = LAMBDA0 + off / 1000.0
        t = truth_models(side * side, rng)
        t[:, 10] = 1.0
        o = eng.synthesize_grid(torch.tensor(t, dtype=torch.float64, device=dev),
                                torch.tensor(off / 1000.0, dtype=torch.float64, device=dev))
        o += NOISE * torch.randn(o.shape, device=dev, dtype=torch.float32)
        rois.append((o.contiguous(), lam, None))
    torch.cuda.synchronize()
    P = sum(int(a.shape[0]) for a, _, _ in rois)
    eng.configure(G.make_config(lam30, LAMBDA0, zee, fix=FIX9, init=GUESS, miter=MAXITER, stop_dchi2=1e-4))
    _, tuned = eng.invert_rois(rois, autotune=True)
    _, direct = eng.invert_rois(rois, autotune=True)
    _, cap = eng.invert_rois(rois, use_graph=True, autotune=True)
    reps = [eng.invert_rois(rois, use_graph=True, autotune=True)[1] for _ in range(2)]
    outs, _ = eng.invert_rois(rois, use_graph=True, autotune=True)
    graph_ms = float(np.mean([r["device_ms"] for r in reps]))
    # the same ROIs one call each on their own grid (device-resident, no graph)
    stream = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    cfgs = [G.make_config(lam, LAMBDA0, zee, fix=FIX9, init=GUESS, miter=MAXITER, stop_dchi2=1e-4)
            for _, lam, _ in rois]
    torch.cuda.synchronize()
    ev[0].record(stream)
    t0 = time.perf_counter()
    for (a, _, _), c in zip(rois, cfgs):
        eng.configure(c)
        eng.invert(a, stream=stream.cuda_stream)
    ev[1].record(stream)
    torch.cuda.synchronize()
    per_roi_wall = time.perf_counter() - t0
    per_roi_ms = ev[0].elapsed_time(ev[1])
    iters = np.concatenate([o["iters"].cpu().numpy() for o in outs])
    return {"workload": "%d ROIs, sides 16-512 px, centred 35 mA grids of 12-60 samples, %d px in all, no PSF, "
                        "noise 1e-3 Ic, early stop dchi2 < 1e-4" % (len(rois), P),
            "pixels": P, "grids": tuned["grids"], "mean_iterations": float(iters.mean()),
            "lane_occupancy": direct["lane_occupancy"],
            "tuned_blocks_per_sm": {"trial": tuned["cap_trial"], "accept": tuned["cap_accept"]},
            "direct": {"pixels_per_s": P / (direct["device_ms"] / 1e3), "ms": direct["device_ms"],
                       "launches": direct["launches"]},
            "graph": {"pixels_per_s": P / (graph_ms / 1e3), "ms": graph_ms, "replayed": reps[-1]["graph_replayed"],
                      "capture_call_ms": cap["device_ms"]},
            "one_call_per_roi": {"pixels_per_s": P / (per_roi_ms / 1e3), "ms": per_roi_ms,
                                 "wall_s": per_roi_wall}}


def _timed_inversions(eng, obs_d, torch, reps):
    """Device time per inversion (CUDA events over `reps` calls after one
    untimed call) and the last call's outputs."""
    stream = torch.cuda.current_stream()
    out = eng.invert(obs_d, stream=stream.cuda_stream)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    torch.cuda.synchronize()
    ev[0].record(stream)
    for _ in range(reps):
        eng.invert(obs_d, out=out, stream=stream.cuda_stream)
    ev[1].record(stream)
    torch.cuda.synchronize()
    return ev[0].elapsed_time(ev[1]) / reps, out


def learned_block(eng, args, torch, reps=3):
    """The learned initial guess (MLP 120 -> 256 -> 256 -> 9, GELU, BF16
    weights, FP32 accumulation): trained by the engine's own tensor-core
    kernels on pixels its ME synthesis generates (the 30-sample grid, the
    PSF of the headline cube, truth from the same ranges, noise 1e-3 Ic),
    then used as the start model of a cube it has not seen, against the
    plain GPU form (classical start, the reference's stop rule) on the same
    cube: pixels/s, iterations, chi2 and the error against the truth."""
    import gmilos_b200 as G
    lam, off = grid()
    x, y = psf_table()
    psf = G.psf_from_table(x, y, off, GRID[1])
    zee = G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0)
    mk = lambda **kw: G.make_config(lam, LAMBDA0, zee, psf=psf, fix=FIX9, init=GUESS, miter=MAXITER, **kw)
    eng.configure(mk())
    dev = torch.device("cuda")

    def cube(n, seed):
        rng = np.random.default_rng(seed)
        t = truth_models(n, rng)
        t[:, 10] = 1.0
        td = torch.tensor(t, dtype=torch.float64, device=dev)
        o = eng.synthesize(td)
        g = torch.Generator(device=dev)
        g.manual_seed(seed)
        o += NOISE * torch.randn(o.shape, generator=g, device=dev, dtype=torch.float32)
        torch.cuda.synchronize()
        return t, td, o.contiguous()

    n_train = args.mlp_train_pixels
    _, t_train, o_train = cube(n_train, args.seed + 400)
    # one short run on a throwaway network first, so that the timed call
    # does not include loading the training kernels
    warm = G.mlp_new(len(lam), args.seed + 1)
    nw = min(16384, n_train // 128 * 128)
    eng.mlp_train(warm, o_train[:nw], t_train[:nw], epochs=1, batch=nw, lr=2e-3, seed=args.seed)
    net = G.mlp_new(len(lam), args.seed)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses = eng.mlp_train(net, o_train, t_train, epochs=args.mlp_epochs, batch=16384, lr=2e-3, seed=args.seed)
    train_s = time.perf_counter() - t0
    del o_train, t_train
    # algorithmic FLOPs per training sample: forward 2 (120*256 + 256*256 + 256*9),
    # backward twice that (activation and weight gradients)
    f_fwd = 2 * (120 * 256 + 256 * 256 + 256 * 9)
    P = args.mlp_eval_pixels
    truth, _, obs = cube(P, args.seed + 500)
    # inference alone (includes uploading and packing the network)
    eng.configure(mk())
    eng.mlp_predict(net, obs)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record()
    for _ in range(reps):
        starts = eng.mlp_predict(net, obs)
    ev[1].record()
    torch.cuda.synchronize()
    infer_ms = ev[0].elapsed_time(ev[1]) / reps
    res = {"workload": "train %d px (%d epochs, batch 16384); evaluate on %d px x 4 x 30 lambda, PSF, noise 1e-3 Ic, "
                       "9 free, <= 50 iterations" % (n_train, args.mlp_epochs, P),
           "training": {"seconds": train_s, "loss_per_epoch": [float(v) for v in losses],
                        "samples_per_s": n_train * args.mlp_epochs / train_s,
                        "tflops_algorithmic": 3 * f_fwd * n_train * args.mlp_epochs / train_s / 1e12},
           "inference": {"ms": infer_ms, "pixels_per_s": P / (infer_ms / 1e3),
                         "tflops_algorithmic": f_fwd * P / (infer_ms / 1e3) / 1e12}}
    variants = {"plain": mk(), "plain_early_stop": mk(stop_dchi2=1e-4),
                "learned": mk(init_mode=G.INIT_LEARNED, mlp=net),
                "learned_early_stop": mk(init_mode=G.INIT_LEARNED, mlp=net, stop_dchi2=1e-4)}
    for name, cfg in variants.items():
        eng.configure(cfg)
        ms, out = _timed_inversions(eng, obs, torch, reps)
        m = out["model64"].cpu().numpy()
        chi = out["chi2"].cpu().numpy()
        st = out["status"].cpu().numpy()
        res[name] = {"pixels_per_s": P / (ms / 1e3), "ms": ms,
                     "mean_iterations": float(out["iters"].float().mean()),
                     "median_chi2": float(np.median(chi)),
                     "learned_start_share": float(((st & G.PIX_LEARNED_INIT) != 0).mean()),
                     "median_abs_error": {"B_G": float(np.median(np.abs(m[:, 1] - truth[:, 1]))),
                                          "vlos_kms": float(np.median(np.abs(m[:, 2] - truth[:, 2]))),
                                          "gamma_deg": float(np.median(np.abs(m[:, 5] - truth[:, 5]))),
                                          "phi_deg": float(np.median(np.minimum(np.abs(m[:, 6] - truth[:, 6]) % 180,
                                                                                180 - np.abs(m[:, 6] - truth[:, 6]) % 180)))}}
    res["speedup_learned_early_stop_vs_plain"] = res["learned_early_stop"]["pixels_per_s"] / res["plain"]["pixels_per_s"]
    # the network's own start models against the truth
    s = starts.cpu().numpy()
    res["start_models_median_abs_error"] = {"B_G": float(np.median(np.abs(s[:, 1] - truth[:, 1]))),
                                            "vlos_kms": float(np.median(np.abs(s[:, 2] - truth[:, 2])))}
    return res


# ----------------------------------------------------------------- reference arms
def _ref_setup(lam, psf):
    """The reference's configuration for this workload (oracle/ref.py)."""
    import oracle as O
    import ref
    l0, z = O.fe6173()
    cfg = O.make_cfg(lam, l0, z, psf=psf, fix=FIX, init=GUESS, miter=MAXITER)
    return ref.setup_from_cfg(cfg), cfg


def cpu_baseline(obs, slight, psf, lam, seconds=15.0, nthreads=0):
    """Time the CPU implementation of the path on a bounded sample of the
    workload: the reference's own routines compiled host-side
    (oracle/_ref/libgmref_cpu.so, kind "reference") when built, else the
    oracle's restatement (kind "port")."""
    import oracle as O
    import ref
    nthreads = nthreads or os.cpu_count()
    s, cfg = _ref_setup(lam, psf)
    if ref.available():
        run = lambda o: ref.invert_cpu(s, o, slight=slight, nthreads=nthreads)
        kind = "reference"
    else:
        run = lambda o: O.lm_batch_f(cfg, o, slight=slight, nthreads=nthreads)
        kind = "port"
    probe = min(len(obs), max(256, 16 * nthreads))
    t0 = time.perf_counter()
    run(np.ascontiguousarray(obs[:probe]))
    rate = probe / (time.perf_counter() - t0)
    n = int(min(len(obs), max(probe, rate * seconds)))
    t0 = time.perf_counter()
    run(np.ascontiguousarray(obs[:n]))
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "pixels/s", "cores": nthreads, "kind": kind,
            "sample": "%d pixels of the same cube (first %d), %.1f s" % (n, n, dt)}


def reference_gpu(obs, slight, psf, lam, nstreams=16):
    """The reference's own lm_mils built for sm_100a (oracle/_ref/
    libgmref_gpu.so) on host buffers, with its launch geometry: blocks per
    stream = occupancy per SM, 32 threads per block, `nstreams` streams.
    Returns pixels / event-timed kernel time (gmilos.cu:1196-1220), the same
    with H2D/D2H included, and the fit results for the equal-chi2 check."""
    import ref
    s, _ = _ref_setup(lam, psf)
    m, chi, it, _, rep = ref.invert_gpu(s, np.ascontiguousarray(obs), slight=slight, nstreams=nstreams)
    P = len(obs)
    return {"value": P / (rep["kernel_ms"] / 1e3), "e2e": P / (rep["e2e_ms"] / 1e3), "report": rep,
            "model": m, "chi2": chi, "iters": it}


def _fit_comparison(mg, cg, ig, mr, cr, ir, names=("engine", "reference")):
    """Agreement of two fits of the same pixels (|dB| < 1 G, angles < 0.1 deg,
    vlos < 5 m/s) and, where they part, on which side chi2 is worse."""
    agree = ((np.abs(mg[:, 1] - mr[:, 1]) < 1.0)
             & (np.minimum(np.abs(mg[:, 5] - mr[:, 5]) % 360, 360 - np.abs(mg[:, 5] - mr[:, 5]) % 360) < 0.1)
             & (np.minimum(np.abs(mg[:, 6] - mr[:, 6]) % 180, 180 - np.abs(mg[:, 6] - mr[:, 6]) % 180) < 0.1)
             & (np.abs(mg[:, 2] - mr[:, 2]) < 0.005))
    return {"median_chi2": [float(np.median(cg)), float(np.median(cr))],
            "mean_iterations": [float(np.mean(ig)), float(np.mean(ir))],
            "agree": float(agree.mean()),
            names[0] + "_chi2_worse": float((~agree & (cg > cr * (1 + 1e-3) + 1e-6)).mean()),
            names[1] + "_chi2_worse": float((~agree & (cr > cg * (1 + 1e-3) + 1e-6)).mean())}


def _reference_sample(args):
    """A bounded sample of the workload synthesised on the CPU (oracle), so
    that no engine code runs in the reference arms."""
    import oracle as O
    lam, off = grid()
    x, y = psf_table()
    psf = O.psf_from_table(x, y, off, GRID[1])
    slight = stray_profile_cpu(off)
    rng = np.random.default_rng(args.seed)
    truth = truth_models(args.ref_pixels, rng)
    obs = _fine_synth_cpu(O, truth, off)
    a = truth[:, 10][:, None, None].astype(np.float32)
    obs = a * obs + (1 - a) * slight[None]
    obs += (NOISE * np.random.default_rng(args.seed + 1000).standard_normal(obs.shape)).astype(np.float32)
    return np.ascontiguousarray(obs, dtype=np.float32), slight, psf, lam


METRIC = "converged pixels/s (1024^2 x 4 x 30 lambda, PSF, stray light, 9 ME + alpha free, <=50 LM iterations)"


def run_reference(args):
    """--impl reference: the reference's own per-pixel routines compiled
    host-side, on every host thread, on a bounded sample per step."""
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    obs, slight, psf, lam = _reference_sample(args)
    nthreads = os.cpu_count()
    times = []
    base = None
    for k in range(args.warmup + args.steps):
        b = cpu_baseline(obs, slight, psf, lam, seconds=args.ref_seconds, nthreads=nthreads)
        if k >= args.warmup:
            times.append(b["value"])
            base = b
    value = float(np.mean(times))
    result = {
        "metric": METRIC,
        "value": value, "unit": "pixels/s", "n_gpus": int(os.environ.get("WORLD_SIZE", 1)), "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "impl": "reference",
        "config": {"workload": "full cube 1024x1024 px x 4 Stokes x 30 lambda (bounded sample per step)",
                   "pixels_per_gpu": 1024 * 1024, "nlambda": 30},
        "cpu_baseline": {"value": value, "unit": "pixels/s", "cores": nthreads, "kind": base["kind"],
                         "sample": base["sample"]},
        "e2e": {"value": value, "unit": "pixels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(result), flush=True)


def run_reference_gpu(args):
    """--impl reference_gpu: the reference's own lm_mils built for sm_100a,
    one inversion of a bounded sample per step (pixels / event-timed kernel
    time, as the reference reports it; e2e adds its H2D and D2H copies)."""
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    import ref
    if not ref.available(gpu=True):
        print(json.dumps({"impl": "reference_gpu", "unavailable": "oracle/_ref/libgmref_gpu.so not built"}))
        return
    obs, slight, psf, lam = _reference_sample(args)
    vals, e2es, rep = [], [], None
    for k in range(args.warmup + args.steps):
        rg = reference_gpu(obs, slight, psf, lam, nstreams=args.ref_gpu_streams)
        if k >= args.warmup:
            vals.append(rg["value"])
            e2es.append(rg["e2e"])
            rep = rg["report"]
    P = len(obs)
    result = {
        "metric": METRIC, "value": float(np.mean(vals)), "unit": "pixels/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": P / float(np.mean(vals)) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "impl": "reference_gpu",
        "config": {"workload": "%d px of the full-cube workload x 4 Stokes x 30 lambda" % P,
                   "blocks_per_stream": rep["num_blocks"], "threads_per_block": rep["threads_per_block"],
                   "streams": rep["nstreams"], "registers": rep["regs"], "stack_bytes": rep["local_bytes"],
                   "heap_bytes": rep["heap_bytes"]},
        "e2e": {"value": float(np.mean(e2es)), "unit": "pixels/s", "h2d_bytes_per_step": obs.nbytes,
                "d2h_bytes_per_step": P * (11 * 8 + 4 + 4) + obs.nbytes},
    }
    print(json.dumps(result), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference", "reference_gpu"])
    ap.add_argument("--pixels", type=int, default=1024 * 1024)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-pixels", type=int, default=65536)
    ap.add_argument("--ref-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-gpu-pixels", type=int, default=65536,
                    help="pixels of the cube run through the reference's sm_100a build (0: skip)")
    ap.add_argument("--ref-gpu-streams", type=int, default=16)
    ap.add_argument("--serve-requests", type=int, default=40,
                    help="requests of the serving-latency phase, per rate with --serve-sweep (0: skip)")
    ap.add_argument("--serve-rate", type=float, default=1.0, help="mean arrivals per second")
    ap.add_argument("--serve-side-min", type=int, default=256)
    ap.add_argument("--serve-side-max", type=int, default=2048)
    ap.add_argument("--serve-policy", default="response_ratio", choices=sorted(SERVE_POLICIES))
    ap.add_argument("--serve-budget-gb", type=int, default=150, help="HBM budget of the serving context")
    ap.add_argument("--serve-unloaded-rate", type=float, default=3.1e6,
                    help="pixels/s of an unloaded host-memory inversion (the stretch's denominator)")
    ap.add_argument("--serve-sweep", default="",
                    help="comma-separated arrival rates: run only the serving stream at each (one JSON line)")
    ap.add_argument("--vmac-free", action="store_true",
                    help="free v_mac too (the reference's 11-term path, lm_mils_11), v_mac starting at 0.5 km/s")
    ap.add_argument("--no-config1", dest="config1", action="store_false",
                    help="skip the 64x64 no-PSF case (engine and the reference's CPU routines)")
    ap.add_argument("--mlp-train-pixels", type=int, default=1 << 22,
                    help="training pixels of the learned initial guess (0: skip that block)")
    ap.add_argument("--mlp-epochs", type=int, default=8)
    ap.add_argument("--ragged-rois", type=int, default=64, help="ROIs of the ragged-batch block (0: skip it)")
    ap.add_argument("--mlp-eval-pixels", type=int, default=1 << 20)
    args = ap.parse_args()
    if args.serve_sweep:
        run_serve_sweep(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.impl == "reference_gpu":
        run_reference_gpu(args)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
