"""Python binding of the B200 Milne-Eddington inversion engine (libgmilos.so).

A thin ctypes layer over the C ABI declared in include/gmilos.h.  Arrays may
be numpy arrays (host memory) or torch CUDA tensors (device memory); the
engine copies host data itself.  There is no CPU fallback: every entry point
needs the compiled library and a CUDA device, and raises otherwise.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgmilos.so")
PKG_ROOT = os.path.dirname(HERE)
MAX_NL = 64
NPAR = 11
ABI_VERSION = 3
PARAM_NAMES = ("eta0", "B", "vlos", "dopp", "aa", "gm", "az", "S0", "S1", "mac", "alfa")

GM_OK = 0
STATUS_NAMES = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of memory / over budget",
                4: "not configured", 5: "unsupported", 6: "timeout", 7: "cancelled", 8: "I/O error"}

PIX_INIT_NAN = 0x01
PIX_MAXITER = 0x02
PIX_LAMBDA_EXIT = 0x04
PIX_CHI2_EXIT = 0x08
PIX_NONFINITE = 0x10
PIX_BAD_INPUT = 0x20

INIT_CLASSICAL, INIT_GIVEN, INIT_PER_PIXEL, INIT_LEARNED = 0, 1, 2, 3
PIX_LEARNED_INIT = 0x40
MLP_IN, MLP_HIDDEN, MLP_OUT, MLP_OUT_PAD = 128, 256, 9, 16
NUMERICS_REFERENCE, NUMERICS_ACCURATE = 0, 1
KERNEL_AUTO, KERNEL_FUSED, KERNEL_WAVES = 0, 1, 2
SERVE_ROUND_ROBIN, SERVE_FIFO, SERVE_SHORTEST_FIRST, SERVE_RESPONSE_RATIO = 0, 1, 2, 3

# Symbols include/gmilos.h declares (checked by the tests against the .so).
EXPORTS = ("gm_create", "gm_destroy", "gm_last_error", "gm_status_string", "gm_config_defaults",
           "gm_configure", "gm_invert", "gm_invert_ex", "gm_synthesize", "gm_synthesize_f64",
           "gm_synthesize_grid", "gm_lm_step", "gm_submit", "gm_poll", "gm_cancel", "gm_zeeman_from_levels",
           "gm_psf_gaussian", "gm_psf_from_table", "gm_get_stats", "gm_measure_peaks", "gm_measure_sfu_peak",
           "gm_invert_noalloc", "gm_classical", "gm_serving_options", "gm_wave_state_bytes",
           "gm_mlp_init", "gm_mlp_train_defaults", "gm_mlp_train", "gm_mlp_gradients", "gm_mlp_predict",
           "gm_invert_rois", "gm_serving_policy")


class GmError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        super().__init__("gmilos: %s%s" % (STATUS_NAMES.get(status, status), (": " + msg) if msg else ""))


class Zeeman(C.Structure):
    _fields_ = [("n_pi", C.c_int), ("n_sig", C.c_int),
                ("nub", C.c_float * 10), ("nup", C.c_float * 10), ("nur", C.c_float * 10),
                ("web", C.c_float * 10), ("wep", C.c_float * 10), ("wer", C.c_float * 10),
                ("gl", C.c_float), ("gu", C.c_float), ("geff", C.c_float), ("fo", C.c_float)]


class Mlp(C.Structure):
    """gm_mlp: the learned initial guess (FP32 parameters, standardisation)."""
    _fields_ = [("abi_version", C.c_int), ("nl", C.c_int), ("steps", C.c_int64),
                ("in_mean", C.c_float * MLP_IN), ("in_scale", C.c_float * MLP_IN),
                ("out_mean", C.c_float * MLP_OUT_PAD), ("out_scale", C.c_float * MLP_OUT_PAD),
                ("w1", (C.c_float * MLP_IN) * MLP_HIDDEN), ("b1", C.c_float * MLP_HIDDEN),
                ("w2", (C.c_float * MLP_HIDDEN) * MLP_HIDDEN), ("b2", C.c_float * MLP_HIDDEN),
                ("w3", (C.c_float * MLP_HIDDEN) * MLP_OUT), ("b3", C.c_float * MLP_OUT_PAD)]

    def arrays(self):
        """numpy views (no copies) of the parameters and standardisation."""
        a = lambda name, shape: np.ctypeslib.as_array(getattr(self, name)).reshape(shape)
        return {"in_mean": a("in_mean", (MLP_IN,)), "in_scale": a("in_scale", (MLP_IN,)),
                "out_mean": a("out_mean", (MLP_OUT_PAD,)), "out_scale": a("out_scale", (MLP_OUT_PAD,)),
                "w1": a("w1", (MLP_HIDDEN, MLP_IN)), "b1": a("b1", (MLP_HIDDEN,)),
                "w2": a("w2", (MLP_HIDDEN, MLP_HIDDEN)), "b2": a("b2", (MLP_HIDDEN,)),
                "w3": a("w3", (MLP_OUT, MLP_HIDDEN)), "b3": a("b3", (MLP_OUT_PAD,))}


class TrainOpts(C.Structure):
    _fields_ = [("epochs", C.c_int), ("batch", C.c_int), ("lr", C.c_float), ("weight_decay", C.c_float),
                ("seed", C.c_uint64)]


class Config(C.Structure):
    _fields_ = [("abi_version", C.c_int), ("nl", C.c_int), ("lambda0", C.c_double),
                ("lambda_", C.c_double * MAX_NL), ("zeeman", Zeeman), ("use_psf", C.c_int),
                ("psf", C.c_double * MAX_NL), ("mu", C.c_float), ("weight", C.c_float * 4),
                ("noise", C.c_float), ("fix", C.c_int * NPAR), ("init_model", C.c_double * NPAR),
                ("init_mode", C.c_int), ("miter", C.c_int), ("ilambda", C.c_float),
                ("toplim", C.c_double), ("logclambda", C.c_int), ("stop_dchi2", C.c_double),
                ("use_slight", C.c_int), ("slight_per_pixel", C.c_int),
                ("slight", C.POINTER(C.c_float)), ("reference_quirks", C.c_int),
                ("numerics", C.c_int), ("lambda_per_pixel", C.c_int),
                ("lambda_map", C.POINTER(C.c_double)), ("kernel", C.c_int),
                ("mlp", C.POINTER(Mlp))]


class Request(C.Structure):
    _fields_ = [("iquv", C.c_void_p), ("npix", C.c_int64), ("nl", C.c_int),
                ("model", C.c_void_p), ("chi2", C.c_void_p), ("iters", C.c_void_p),
                ("status", C.c_void_p), ("fix", C.POINTER(C.c_int)),
                ("latency_ms", C.POINTER(C.c_double)), ("queue_ms", C.POINTER(C.c_double))]


class Roi(C.Structure):
    _fields_ = [("iquv", C.c_void_p), ("npix", C.c_int64), ("nl", C.c_int), ("lambda_", C.c_void_p),
                ("psf", C.c_void_p), ("model", C.c_void_p), ("chi2", C.c_void_p), ("iters", C.c_void_p),
                ("status", C.c_void_p)]


class BatchOpts(C.Structure):
    _fields_ = [("use_graph", C.c_int), ("autotune", C.c_int)]


class BatchStats(C.Structure):
    _fields_ = [("pixels", C.c_int64), ("grids", C.c_int), ("launches", C.c_int), ("graph_replayed", C.c_int),
                ("cap_trial", C.c_int), ("cap_accept", C.c_int), ("device_ms", C.c_float),
                ("lane_occupancy", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("pixels", C.c_int64), ("iterations", C.c_int64), ("accepted", C.c_int64),
                ("kernel_ms", C.c_float), ("grid_blocks", C.c_int), ("block_threads", C.c_int),
                ("warps_per_block", C.c_int), ("kernel_launches", C.c_int)]


_lib = None


def lib():
    """Load libgmilos.so; raises if the extension was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise GmError(5, "libgmilos.so not built (run `make -C %s` or __graft_entry__.build())" % PKG_ROOT)
        L = C.CDLL(LIB_PATH)
        vp, i64 = C.c_void_p, C.c_int64
        L.gm_create.argtypes = [C.c_int, C.c_size_t, C.POINTER(vp)]
        L.gm_destroy.argtypes = [vp]
        L.gm_last_error.argtypes = [vp]
        L.gm_last_error.restype = C.c_char_p
        L.gm_status_string.argtypes = [C.c_int]
        L.gm_status_string.restype = C.c_char_p
        L.gm_config_defaults.argtypes = [C.POINTER(Config)]
        L.gm_config_defaults.restype = None
        L.gm_configure.argtypes = [vp, C.POINTER(Config)]
        L.gm_invert.argtypes = [vp, vp, i64, C.c_int, vp, vp, vp, vp, vp, vp]
        L.gm_invert_ex.argtypes = [vp, vp, i64, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        L.gm_lm_step.argtypes = [vp, vp, i64, C.c_int, vp, C.c_float, vp, vp, vp, vp, vp]
        L.gm_synthesize.argtypes = [vp, vp, i64, vp, vp, vp]
        L.gm_synthesize_f64.argtypes = [vp, vp, i64, vp, vp, vp]
        L.gm_synthesize_grid.argtypes = [vp, vp, i64, vp, C.c_int, vp, vp]
        L.gm_classical.argtypes = [vp, vp, i64, C.c_int, vp, vp]
        L.gm_serving_options.argtypes = [vp, C.c_int, i64, C.c_int]
        L.gm_serving_policy.argtypes = [vp, C.c_int]
        L.gm_submit.argtypes = [vp, C.POINTER(Request), C.POINTER(C.c_uint64)]
        L.gm_poll.argtypes = [vp, C.c_uint64, C.c_int]
        L.gm_cancel.argtypes = [vp, C.c_uint64]
        L.gm_zeeman_from_levels.argtypes = [C.c_double] * 7 + [C.POINTER(Zeeman)]
        L.gm_psf_gaussian.argtypes = [C.c_double, vp, C.c_int, vp]
        L.gm_psf_from_table.argtypes = [vp, vp, C.c_int, vp, C.c_int, C.c_double, vp]
        L.gm_get_stats.argtypes = [vp, C.POINTER(Stats)]
        L.gm_measure_peaks.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.gm_measure_sfu_peak.argtypes = [vp, C.POINTER(C.c_double)]
        L.gm_invert_noalloc.argtypes = [C.POINTER(Config), vp, i64, C.c_int, vp, vp, vp, vp, vp, vp]
        L.gm_wave_state_bytes.argtypes = [C.c_int, C.c_int, i64]
        L.gm_wave_state_bytes.restype = C.c_size_t
        L.gm_mlp_init.argtypes = [C.POINTER(Mlp), C.c_int, C.c_uint64]
        L.gm_mlp_train_defaults.argtypes = [C.POINTER(TrainOpts)]
        L.gm_mlp_train_defaults.restype = None
        L.gm_mlp_train.argtypes = [vp, C.POINTER(Mlp), vp, vp, i64, C.POINTER(TrainOpts), vp]
        L.gm_mlp_gradients.argtypes = [vp, C.POINTER(Mlp), vp, vp, i64, C.POINTER(Mlp), C.POINTER(C.c_float)]
        L.gm_mlp_predict.argtypes = [vp, C.POINTER(Mlp), vp, i64, vp, vp]
        L.gm_invert_rois.argtypes = [vp, C.POINTER(Roi), C.c_int, C.POINTER(BatchOpts), C.POINTER(BatchStats), vp]
        _lib = L
    return _lib


def _ptr(a):
    """Raw pointer of a numpy array or torch tensor (None -> NULL)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return C.c_void_p(a.data_ptr())
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return C.c_void_p(a.ctypes.data)


def _check(st, ctx=None):
    if st != GM_OK:
        msg = lib().gm_last_error(ctx).decode() if ctx else ""
        raise GmError(st, msg)


# ------------------------------------------------------------------ set-up
def zeeman_from_levels(sl, ll, jl, su, lu, ju, fos=1.0):
    z = Zeeman()
    _check(lib().gm_zeeman_from_levels(sl, ll, jl, su, lu, ju, fos, C.byref(z)))
    return z


def fe6173():
    """Fe I 6173.3356 A (atomic-parameter entry `5P 1.0- 5D 0.0`)."""
    return 6173.3356, zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0)


def grid_offsets_mA(first_mA, step_mA, last_mA):
    n = int(((last_mA - first_mA) / step_mA) + 1)
    off = np.empty(n)
    off[0] = first_mA
    for i in range(1, n):
        off[i] = off[i - 1] + step_mA
    return off


def grid_lambda(lambda0, first_mA, step_mA, last_mA):
    """Absolute wavelengths of a .grid line, accumulated like gmilos.cu:184-189."""
    n = int(((last_mA - first_mA) / step_mA) + 1)
    lam = np.empty(n)
    lam[0] = lambda0 + first_mA / 1000.0
    for i in range(1, n):
        lam[i] = lam[i - 1] + step_mA / 1000.0
    return lam


def psf_gaussian(fwhm_mA, lam):
    lam = np.ascontiguousarray(lam, dtype=np.float64)
    out = np.zeros(len(lam))
    _check(lib().gm_psf_gaussian(fwhm_mA, _ptr(lam), len(lam), _ptr(out)))
    return out


def mlp_new(nl, seed=0):
    """A fresh learned-guess network for grids of nl samples (gm_mlp_init)."""
    net = Mlp()
    _check(lib().gm_mlp_init(C.byref(net), int(nl), int(seed)))
    return net


def wave_state_bytes(nl, miter, pixels):
    """Device bytes of wave-kernel LM state for a chunk of `pixels` pixels
    (gm_wave_state_bytes): what an HBM budget must leave room for."""
    return int(lib().gm_wave_state_bytes(int(nl), int(miter), int(pixels)))


def psf_from_table(x_mA, y, offsets_mA, step_mA):
    x = np.ascontiguousarray(x_mA, dtype=np.float64)
    yy = np.ascontiguousarray(y, dtype=np.float64)
    off = np.ascontiguousarray(offsets_mA, dtype=np.float64)
    out = np.zeros(len(off))
    _check(lib().gm_psf_from_table(_ptr(x), _ptr(yy), len(x), _ptr(off), len(off), step_mA, _ptr(out)))
    return out


def make_config(lam, lambda0, zeeman, psf=None, mu=1.0, weight=(1, 1, 1, 1), noise=1e-6,
                fix=(1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0), init=None, init_mode=INIT_CLASSICAL,
                miter=50, ilambda=0.1, toplim=1e-12, logclambda=0, stop_dchi2=0.0,
                slight=None, slight_per_pixel=False, reference_quirks=1, numerics=0,
                lambda_map=None, kernel=KERNEL_AUTO, mlp=None):
    """Engine configuration (gm_config).  lambda_map: optional per-pixel
    wavelength grids [P][nl] (absolute, A; numpy or a CUDA tensor of float64),
    read at each call like a per-pixel stray map; `lam` then only sizes the
    grid and the PSF stays `psf`.  kernel: KERNEL_AUTO (the fused kernel for
    calls of fewer than 16384 pixels, 32768 without a PSF, else the
    wave-synchronous kernels where they cover the call), KERNEL_FUSED (the
    fused kernel for every call) or KERNEL_WAVES (the wave kernels wherever
    they cover the call).  mlp: a trained Mlp for init_mode INIT_LEARNED."""
    c = Config()
    lib().gm_config_defaults(C.byref(c))
    lam = np.asarray(lam, dtype=np.float64)
    if len(lam) > MAX_NL:
        raise ValueError("at most %d wavelength samples" % MAX_NL)
    c.nl = len(lam)
    c.lambda0 = lambda0
    for i, v in enumerate(lam):
        c.lambda_[i] = v
    c.zeeman = zeeman
    c.use_psf = 0 if psf is None else 1
    if psf is not None:
        for i, v in enumerate(psf):
            c.psf[i] = v
    c.mu = mu
    for i in range(4):
        c.weight[i] = weight[i]
    c.noise = noise
    for i in range(NPAR):
        c.fix[i] = int(fix[i])
    if init is not None:
        for i in range(NPAR):
            c.init_model[i] = init[i]
    c.init_mode = init_mode
    c.miter = miter
    c.ilambda = ilambda
    c.toplim = toplim
    c.logclambda = logclambda
    c.stop_dchi2 = stop_dchi2
    c.reference_quirks = reference_quirks
    c.numerics = numerics
    c.kernel = kernel
    c._mlp_ref = mlp
    if mlp is not None:
        c.mlp = C.pointer(mlp)
    c._slight_ref = None
    c._lambda_ref = None
    if lambda_map is not None:
        c.lambda_per_pixel = 1
        if hasattr(lambda_map, "data_ptr"):
            c._lambda_ref = lambda_map
            c.lambda_map = C.cast(C.c_void_p(lambda_map.data_ptr()), C.POINTER(C.c_double))
        else:
            arr = np.ascontiguousarray(lambda_map, dtype=np.float64)
            if arr.ndim != 2 or arr.shape[1] != len(lam):
                raise ValueError("lambda_map must be [P][nl]")
            c._lambda_ref = arr
            c.lambda_map = arr.ctypes.data_as(C.POINTER(C.c_double))
    if slight is not None:
        c.use_slight = 1
        c.slight_per_pixel = 1 if slight_per_pixel else 0
        if hasattr(slight, "data_ptr"):
            c.slight = C.cast(C.c_void_p(slight.data_ptr()), C.POINTER(C.c_float))
        else:
            arr = np.ascontiguousarray(slight, dtype=np.float32)
            c._slight_ref = arr
            c.slight = arr.ctypes.data_as(C.POINTER(C.c_float))
    return c


# ------------------------------------------------------------------ engine
class Engine:
    """One engine context on one CUDA device (gm_create / gm_destroy)."""

    def __init__(self, device=0, hbm_budget=0):
        self._ctx = C.c_void_p()
        _check(lib().gm_create(device, hbm_budget, C.byref(self._ctx)))
        self.cfg = None

    def close(self):
        if self._ctx:
            lib().gm_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def configure(self, cfg):
        _check(lib().gm_configure(self._ctx, C.byref(cfg)), self._ctx)
        self.cfg = cfg

    @property
    def nl(self):
        return self.cfg.nl

    @property
    def nterms(self):
        """Terms of the normal equations: 11 when v_mac and alpha are both free."""
        return 11 if (self.cfg.fix[9] and self.cfg.fix[10]) else 10

    def invert(self, iquv, init_models=None, fitted=False, out=None, stream=None):
        """Invert a cube iquv [P][4][nl] (numpy: host; torch CUDA tensor: device).

        Returns dict(model [P][11] f32, model64 [P][11] f64, chi2, iters, accepted,
        status, fitted [P][4][nl] or None) in the same memory space as the input."""
        P = int(iquv.shape[0])
        nl = self.nl
        if tuple(iquv.shape[1:]) != (4, nl):
            raise ValueError("iquv must be [P][4][%d]" % nl)
        if out is None:
            out = self._alloc_outputs(iquv, P, nl, fitted)
        st = lib().gm_invert_ex(self._ctx, _ptr(iquv), P, nl, _ptr(init_models), _ptr(out["model"]),
                                _ptr(out["model64"]), _ptr(out["chi2"]), _ptr(out["iters"]),
                                _ptr(out["accepted"]), _ptr(out["fitted"]), _ptr(out["status"]),
                                C.c_void_p(stream) if stream else None)
        _check(st, self._ctx)
        return out

    def invert_plain(self, iquv, model, chi2=None, iters=None, fitted=None, status=None, stream=None):
        """gm_invert: the reference-facing call with caller-owned buffers."""
        P = int(iquv.shape[0])
        st = lib().gm_invert(self._ctx, _ptr(iquv), P, self.nl, _ptr(model), _ptr(chi2), _ptr(iters),
                             _ptr(fitted), _ptr(status), C.c_void_p(stream) if stream else None)
        _check(st, self._ctx)

    @staticmethod
    def _alloc_outputs(like, P, nl, fitted):
        if hasattr(like, "data_ptr"):
            import torch
            dev = like.device
            mk = lambda shape, dt: torch.empty(shape, dtype=dt, device=dev)
            f32, f64, i32 = torch.float32, torch.float64, torch.int32
        else:
            mk = lambda shape, dt: np.empty(shape, dtype=dt)
            f32, f64, i32 = np.float32, np.float64, np.int32
        o = {"model": mk((P, NPAR), f32), "model64": mk((P, NPAR), f64), "chi2": mk((P,), f32),
             "iters": mk((P,), i32), "accepted": mk((P,), i32), "status": mk((P,), i32),
             "fitted": mk((P, 4, nl), f32) if fitted else None}
        return o

    def lm_step(self, iquv, models, flambda):
        """One LM iteration from explicit states: (delta [P][nterms], trial [P][11],
        chi2_start [P], chi2_trial [P]) as host numpy arrays."""
        P = int(iquv.shape[0])
        models = np.ascontiguousarray(models, dtype=np.float64)
        d = np.empty((P, self.nterms), dtype=np.float32)
        t = np.empty((P, NPAR), dtype=np.float64)
        c0 = np.empty(P, dtype=np.float32)
        c1 = np.empty(P, dtype=np.float32)
        _check(lib().gm_lm_step(self._ctx, _ptr(iquv), P, self.nl, _ptr(models), float(flambda),
                                _ptr(d), _ptr(t), _ptr(c0), _ptr(c1), None), self._ctx)
        return d, t, c0, c1

    def synthesize(self, models, rf=False, stream=None):
        """Synthesis (+ response functions [P][4][nterms][nl]) of models [P][11] (float64 or float32)."""
        P = int(models.shape[0])
        nl, nt = self.nl, self.nterms
        is_t = hasattr(models, "data_ptr")
        if is_t:
            import torch
            spec = torch.empty((P, 4, nl), dtype=torch.float32, device=models.device)
            r = torch.empty((P, 4, nt, nl), dtype=torch.float32, device=models.device) if rf else None
            f64 = models.dtype == torch.float64
        else:
            spec = np.empty((P, 4, nl), dtype=np.float32)
            r = np.empty((P, 4, nt, nl), dtype=np.float32) if rf else None
            f64 = models.dtype == np.float64
        fn = lib().gm_synthesize_f64 if f64 else lib().gm_synthesize
        _check(fn(self._ctx, _ptr(models), P, _ptr(spec), _ptr(r), C.c_void_p(stream) if stream else None),
               self._ctx)
        return (spec, r) if rf else spec

    def synthesize_grid(self, models, offsets_A, stream=None):
        """Pure ME profiles (no PSF / stray light) of models [P][11] f64 on offsets [A]."""
        P = int(models.shape[0])
        n = int(offsets_A.shape[0])
        if hasattr(models, "data_ptr"):
            import torch
            out = torch.empty((P, 4, n), dtype=torch.float32, device=models.device)
        else:
            out = np.empty((P, 4, n), dtype=np.float32)
        _check(lib().gm_synthesize_grid(self._ctx, _ptr(models), P, _ptr(offsets_A), n, _ptr(out),
                                        C.c_void_p(stream) if stream else None), self._ctx)
        return out

    def classical(self, iquv):
        """Classical estimates only (the NumberOfCycles < 0 mode): models [P][11] f64."""
        P = int(iquv.shape[0])
        out = np.empty((P, NPAR), dtype=np.float64)
        _check(lib().gm_classical(self._ctx, _ptr(iquv), P, self.nl, _ptr(out), None), self._ctx)
        return out

    def serving_options(self, streams=4, chunk_pixels=65536, max_active=16):
        _check(lib().gm_serving_options(self._ctx, int(streams), int(chunk_pixels), int(max_active)),
               self._ctx)

    def serving_policy(self, policy):
        """SERVE_ROUND_ROBIN, SERVE_FIFO, SERVE_SHORTEST_FIRST or SERVE_RESPONSE_RATIO
        (gm_serving_policy)."""
        _check(lib().gm_serving_policy(self._ctx, int(policy)), self._ctx)

    def submit(self, iquv, model, chi2=None, iters=None, status=None, fix=None):
        """Queue an inversion (continuous batching).  The engine reads and
        writes the arrays until poll() returns for the ticket; this object
        keeps them alive until then."""
        r = Request()
        r.iquv = _ptr(iquv)
        r.npix = int(iquv.shape[0])
        r.nl = self.nl
        r.model = _ptr(model)
        r.chi2 = _ptr(chi2)
        r.iters = _ptr(iters)
        r.status = _ptr(status)
        if fix is not None:
            arr = (C.c_int * NPAR)(*[int(x) for x in fix])
            r.fix = C.cast(arr, C.POINTER(C.c_int))
        times = (C.c_double * 2)(-1.0, -1.0)
        r.latency_ms = C.cast(C.byref(times, 0), C.POINTER(C.c_double))
        r.queue_ms = C.cast(C.byref(times, C.sizeof(C.c_double)), C.POINTER(C.c_double))
        t = C.c_uint64()
        _check(lib().gm_submit(self._ctx, C.byref(r), C.byref(t)), self._ctx)
        if not hasattr(self, "_times"):
            self._times = {}
        self._times[t.value] = (times, (iquv, model, chi2, iters, status))
        return t.value

    def poll(self, ticket, timeout_us=-1):
        """Status of the request (0 when done); its latency and queueing time
        [ms] are then in last_latency_ms / last_queue_ms."""
        st = lib().gm_poll(self._ctx, ticket, timeout_us)
        if st != 6:   # not a timeout: the ticket is consumed
            entry = getattr(self, "_times", {}).pop(ticket, None)
            if entry is not None:
                times = entry[0]
                self.last_latency_ms, self.last_queue_ms = times[0], times[1]
        return st

    def cancel(self, ticket):
        _check(lib().gm_cancel(self._ctx, ticket), self._ctx)

    def measure_peaks(self):
        """(fp32, fp64) FMA peaks of this device in TFLOP/s."""
        a, b = C.c_double(), C.c_double()
        _check(lib().gm_measure_peaks(self._ctx, C.byref(a), C.byref(b)), self._ctx)
        return a.value, b.value

    def measure_sfu_peak(self):
        """Special-function-unit (MUFU) throughput of this device, G ops/s."""
        a = C.c_double()
        _check(lib().gm_measure_sfu_peak(self._ctx, C.byref(a)), self._ctx)
        return a.value

    # ------------------------------------------------------- ragged batches
    def invert_rois(self, rois, use_graph=False, autotune=False, stream=None):
        """Invert a ragged batch in one call (gm_invert_rois).  rois: list of
        (iquv [P][4][nl], lambda [nl] absolute wavelengths, psf [nl] or None);
        iquv numpy (host) or CUDA tensors (device).  Returns one output dict
        per ROI (model [P][11], chi2, iters, status, in the ROI's memory
        space) and the batch statistics."""
        keep = []
        arr = (Roi * max(1, len(rois)))()
        outs = []
        for i, (iquv, lam, psf) in enumerate(rois):
            P, nl = int(iquv.shape[0]), int(iquv.shape[2])
            lam = np.ascontiguousarray(lam, dtype=np.float64)
            ps = None if psf is None else np.ascontiguousarray(psf, dtype=np.float64)
            o = self._alloc_outputs(iquv, P, nl, False)
            keep += [lam, ps, iquv]
            r = arr[i]
            r.iquv, r.npix, r.nl = _ptr(iquv), P, nl
            r.lambda_ = lam.ctypes.data
            r.psf = None if ps is None else ps.ctypes.data
            r.model, r.chi2, r.iters, r.status = _ptr(o["model"]), _ptr(o["chi2"]), _ptr(o["iters"]), _ptr(o["status"])
            outs.append({k: o[k] for k in ("model", "chi2", "iters", "status")})
        opts = BatchOpts(int(bool(use_graph)), int(bool(autotune)))
        st = BatchStats()
        _check(lib().gm_invert_rois(self._ctx, arr, len(rois), C.byref(opts), C.byref(st),
                                    C.c_void_p(stream) if stream else None), self._ctx)
        return outs, {k: getattr(st, k) for k, _ in BatchStats._fields_}

    # ------------------------------------------------------- learned guess
    def mlp_train(self, net, iquv, truth, epochs=8, batch=16384, lr=2e-3, weight_decay=0.0, seed=1):
        """Train `net` (an Mlp, in place) on profiles iquv [n][4][nl] and the
        models that made them, truth [n][11] (numpy or CUDA tensors).
        Returns the mean loss of each epoch."""
        o = TrainOpts()
        lib().gm_mlp_train_defaults(C.byref(o))
        o.epochs, o.batch, o.lr, o.weight_decay, o.seed = int(epochs), int(batch), float(lr), float(weight_decay), \
            int(seed)
        loss = np.zeros(max(1, int(epochs)), dtype=np.float32)
        _check(lib().gm_mlp_train(self._ctx, C.byref(net), _ptr(iquv), _ptr(truth), int(iquv.shape[0]),
                                  C.byref(o), _ptr(loss)), self._ctx)
        return loss

    def mlp_gradients(self, net, iquv, truth):
        """(loss, gradients as an Mlp) of one batch (n a multiple of 128)."""
        g = Mlp()
        loss = C.c_float()
        _check(lib().gm_mlp_gradients(self._ctx, C.byref(net), _ptr(iquv), _ptr(truth), int(iquv.shape[0]),
                                      C.byref(g), C.byref(loss)), self._ctx)
        return loss.value, g

    def mlp_predict(self, net, iquv):
        """Start models [n][11] (float64) the network predicts for iquv."""
        n = int(iquv.shape[0])
        if hasattr(iquv, "data_ptr"):
            import torch
            out = torch.empty((n, NPAR), dtype=torch.float64, device=iquv.device)
        else:
            out = np.empty((n, NPAR), dtype=np.float64)
        _check(lib().gm_mlp_predict(self._ctx, C.byref(net), _ptr(iquv), n, _ptr(out), None), self._ctx)
        return out

    def stats(self):
        s = Stats()
        _check(lib().gm_get_stats(self._ctx, C.byref(s)), self._ctx)
        return {k: getattr(s, k) for k, _ in Stats._fields_}
