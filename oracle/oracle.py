"""ctypes wrapper of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / reference legs as the checker.  The engine under
g-milos_b200/ never imports this module.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
MAXNL = 128
NPAR = 11
PARAM_NAMES = ("eta0", "B", "vlos", "dopp", "aa", "gm", "az", "S0", "S1", "mac", "alfa")


class Zeeman(C.Structure):
    _fields_ = [("n_pi", C.c_int), ("n_sig", C.c_int),
                ("nub", C.c_double * 10), ("nup", C.c_double * 10), ("nur", C.c_double * 10),
                ("web", C.c_double * 10), ("wep", C.c_double * 10), ("wer", C.c_double * 10),
                ("gl", C.c_double), ("gu", C.c_double), ("geff", C.c_double), ("fo", C.c_double)]


class Cfg(C.Structure):
    _fields_ = [("nl", C.c_int), ("nterms", C.c_int),
                ("lambda_", C.c_double * MAXNL), ("lambda0", C.c_double),
                ("z", Zeeman), ("use_psf", C.c_int), ("psf", C.c_double * MAXNL),
                ("mu", C.c_double), ("weight", C.c_double * 4), ("noise", C.c_double),
                ("fix", C.c_int * NPAR), ("init", C.c_double * NPAR),
                ("miter", C.c_int), ("ilambda", C.c_double), ("toplim", C.c_double),
                ("logclambda", C.c_int), ("classical_init", C.c_int),
                ("alpha_rf_mixed", C.c_int), ("stop_dchi2", C.c_double)]


def build():
    subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        fp = C.POINTER(C.c_float)
        ip = C.POINTER(C.c_int)
        cp = C.POINTER(Cfg)
        L.orc_cuanten.argtypes = [C.c_double] * 7 + [C.POINTER(Zeeman)]
        L.orc_psf_gauss.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, dp]
        L.orc_psf_center_shift.argtypes = [dp, C.c_int, C.c_double]
        L.orc_psf_center_shift.restype = C.c_double
        L.orc_psf_linear.argtypes = [dp, dp, C.c_int, dp, C.c_int, C.c_double, dp]
        L.orc_synth_d.argtypes = [cp, dp, dp, dp, dp]
        L.orc_synth_f.argtypes = [cp, dp, fp, fp, fp]
        L.orc_classical.argtypes = [C.c_double, dp, C.c_int, fp, dp, C.c_int, C.c_double]
        L.orc_svdcordic_f.argtypes = [fp, fp, fp]
        L.orc_svdcordic_d.argtypes = [dp, dp, dp]
        L.orc_solve_f.argtypes = [fp, fp, fp]
        L.orc_svdcmp.argtypes = [dp, C.c_int, C.c_int, dp, dp]
        L.orc_normal_f.argtypes = [cp, dp, fp, fp, fp, fp, fp]
        L.orc_lm_step_f.argtypes = [cp, dp, fp, fp, C.c_float, fp, dp, fp, fp]
        L.orc_lm_f.argtypes = [cp, fp, fp, dp, fp, ip, ip, fp]
        L.orc_lm_d.argtypes = [cp, fp, fp, dp, dp, ip, ip, dp]
        L.orc_lm_batch_f.argtypes = [cp, C.c_long, fp, fp, C.c_int, dp, fp, ip, ip, fp, C.c_int]
        L.orc_synth_batch_f.argtypes = [cp, C.c_long, dp, fp, C.c_int, fp, C.c_int]
        L.orc_max_threads.restype = C.c_int
        L.orc_set_mo_scale.argtypes = [C.c_double]
        _lib = L
    return _lib


def _p(a, t):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(t))


def _d(a):
    return _p(a, C.c_double)


def _f(a):
    return _p(a, C.c_float)


def _i(a):
    return _p(a, C.c_int)


# ---------------------------------------------------------------- helpers
def cuanten(sl, ll, jl, su, lu, ju, fos=1.0):
    z = Zeeman()
    lib().orc_cuanten(sl, ll, jl, su, lu, ju, fos, C.byref(z))
    return z


def fe6173():
    """Fe I 6173.3356 A, LINES entry 5P 1.0- 5D 0.0 (S=(5-1)/2, L=P/D)."""
    return 6173.3356, cuanten(2, 1, 1.0, 2, 2, 0.0, 1.0)


def grid_offsets_mA(first_mA, step_mA, last_mA):
    """Offsets of a .grid line, accumulated like gmilos.cu:171-176."""
    n = int(((last_mA - first_mA) / step_mA) + 1)
    off = np.empty(n)
    off[0] = first_mA
    for i in range(1, n):
        off[i] = off[i - 1] + step_mA
    return off


def grid_lambda(lambda0, first_mA, step_mA, last_mA):
    """Absolute wavelengths, accumulated like gmilos.cu:184-189."""
    n = int(((last_mA - first_mA) / step_mA) + 1)
    lam = np.empty(n)
    lam[0] = lambda0 + first_mA / 1000.0
    for i in range(1, n):
        lam[i] = lam[i - 1] + step_mA / 1000.0
    return lam


def psf_from_table(x_mA, y, offsets_mA, step_mA):
    n = len(offsets_mA)
    off = np.ascontiguousarray(offsets_mA, dtype=np.float64)
    shift = lib().orc_psf_center_shift(_d(off), n, step_mA / 1000.0)
    out = np.zeros(n)
    x = np.ascontiguousarray(x_mA, dtype=np.float64)
    yy = np.ascontiguousarray(y, dtype=np.float64)
    lib().orc_psf_linear(_d(x), _d(yy), len(x), _d(off), n, shift, _d(out))
    return out


def psf_gauss(fwhm_mA, lam):
    n = len(lam)
    out = np.zeros(n)
    lib().orc_psf_gauss(fwhm_mA, lam[1] - lam[0], lam[0], lam[n // 2], n, _d(out))
    return out


def make_cfg(lam, lambda0, zeeman, psf=None, mu=1.0, weight=(1, 1, 1, 1), noise=1e-6,
             fix=(1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0), init=None, miter=50, ilambda=0.1,
             toplim=1e-12, logclambda=0, classical_init=1, alpha_rf_mixed=1, nterms=None,
             stop_dchi2=0.0):
    c = Cfg()
    lam = np.asarray(lam, dtype=np.float64)
    c.nl = len(lam)
    assert c.nl <= MAXNL
    c.nterms = nterms if nterms is not None else (11 if (fix[9] and fix[10]) else 10)
    for i, v in enumerate(lam):
        c.lambda_[i] = v
    c.lambda0 = lambda0
    c.z = zeeman
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
    if init is None:
        init = (40.0, 1000.0, 0.2, 0.03, 0.05, 150.0, 110.0, 0.35, 0.5, 0.0, 1.0)   # run/guess.mod
    for i in range(NPAR):
        c.init[i] = init[i]
    c.miter = miter
    c.ilambda = ilambda
    c.toplim = toplim
    c.logclambda = logclambda
    c.classical_init = classical_init
    c.alpha_rf_mixed = alpha_rf_mixed
    c.stop_dchi2 = stop_dchi2
    return c


# ---------------------------------------------------------------- model
def synth_d(cfg, model, slight=None, rf=False):
    nl, nt = cfg.nl, cfg.nterms
    m = np.ascontiguousarray(model, dtype=np.float64)
    sl = None if slight is None else np.ascontiguousarray(slight, dtype=np.float64)
    spec = np.zeros(4 * nl)
    r = np.zeros(4 * nt * nl) if rf else None
    lib().orc_synth_d(C.byref(cfg), _d(m), _d(sl), _d(spec), _d(r))
    spec = spec.reshape(4, nl)
    return (spec, r.reshape(4, nt, nl)) if rf else spec


def synth_f(cfg, model, slight=None, rf=False):
    nl, nt = cfg.nl, cfg.nterms
    m = np.ascontiguousarray(model, dtype=np.float64)
    sl = None if slight is None else np.ascontiguousarray(slight, dtype=np.float32)
    spec = np.zeros(4 * nl, dtype=np.float32)
    r = np.zeros(4 * nt * nl, dtype=np.float32) if rf else None
    lib().orc_synth_f(C.byref(cfg), _d(m), _f(sl), _f(spec), _f(r))
    spec = spec.reshape(4, nl)
    return (spec, r.reshape(4, nt, nl)) if rf else spec


def synth_batch_f(cfg, models, slight=None, slight_per_pixel=False, nthreads=0):
    models = np.ascontiguousarray(models, dtype=np.float64)
    P = models.shape[0]
    sl = None if slight is None else np.ascontiguousarray(slight, dtype=np.float32)
    out = np.zeros((P, 4, cfg.nl), dtype=np.float32)
    lib().orc_synth_batch_f(C.byref(cfg), P, _d(models), _f(sl), int(slight_per_pixel),
                            _f(out), nthreads)
    return out


def classical(cfg, obs, model=None, for_init=1):
    m = np.array(model if model is not None else list(cfg.init), dtype=np.float64)
    o = np.ascontiguousarray(obs, dtype=np.float32).reshape(-1)
    lam = np.array(cfg.lambda_[:cfg.nl])
    lib().orc_classical(cfg.lambda0, _d(lam), cfg.nl, _f(o), _d(m), for_init, cfg.z.geff)
    return m


def svdcordic_f(a):
    a = np.ascontiguousarray(a, dtype=np.float32).reshape(100)
    w = np.zeros(10, dtype=np.float32)
    v = np.zeros(100, dtype=np.float32)
    lib().orc_svdcordic_f(_f(a), _f(w), _f(v))
    return w, v.reshape(10, 10)


def svdcordic_d(a):
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(100)
    w = np.zeros(10)
    v = np.zeros(100)
    lib().orc_svdcordic_d(_d(a), _d(w), _d(v))
    return w, v.reshape(10, 10)


def solve_f(h, beta):
    h = np.ascontiguousarray(h, dtype=np.float32).reshape(100)
    b = np.ascontiguousarray(beta, dtype=np.float32)
    d = np.zeros(10, dtype=np.float32)
    lib().orc_solve_f(_f(h), _f(b), _f(d))
    return d


def svdcmp(a):
    a = np.array(a, dtype=np.float64)
    m, n = a.shape
    aa = np.ascontiguousarray(a).reshape(-1)
    w = np.zeros(n)
    v = np.zeros(n * n)
    lib().orc_svdcmp(_d(aa), m, n, _d(w), _d(v))
    return aa.reshape(m, n), w, v.reshape(n, n)


def normal_f(cfg, model, obs, slight=None):
    nt = cfg.nterms
    m = np.ascontiguousarray(model, dtype=np.float64)
    o = np.ascontiguousarray(obs, dtype=np.float32).reshape(-1)
    sl = None if slight is None else np.ascontiguousarray(slight, dtype=np.float32)
    al = np.zeros(nt * nt, dtype=np.float32)
    be = np.zeros(nt, dtype=np.float32)
    chi = np.zeros(1, dtype=np.float32)
    lib().orc_normal_f(C.byref(cfg), _d(m), _f(o), _f(sl), _f(al), _f(be), _f(chi))
    return al.reshape(nt, nt), be, float(chi[0])


def lm_step_f(cfg, model, obs, flambda, slight=None):
    m = np.ascontiguousarray(model, dtype=np.float64)
    o = np.ascontiguousarray(obs, dtype=np.float32).reshape(-1)
    sl = None if slight is None else np.ascontiguousarray(slight, dtype=np.float32)
    delta = np.zeros(cfg.nterms, dtype=np.float32)
    trial = np.zeros(NPAR)
    c1 = np.zeros(1, dtype=np.float32)
    c0 = np.zeros(1, dtype=np.float32)
    lib().orc_lm_step_f(C.byref(cfg), _d(m), _f(o), _f(sl), flambda, _f(delta), _d(trial),
                        _f(c1), _f(c0))
    return delta, trial, float(c1[0]), float(c0[0])


def lm_f(cfg, obs, slight=None):
    o = np.ascontiguousarray(obs, dtype=np.float32).reshape(-1)
    sl = None if slight is None else np.ascontiguousarray(slight, dtype=np.float32)
    m = np.zeros(NPAR)
    chi = np.zeros(1, dtype=np.float32)
    it = np.zeros(1, dtype=np.int32)
    acc = np.zeros(1, dtype=np.int32)
    fit = np.zeros(4 * cfg.nl, dtype=np.float32)
    lib().orc_lm_f(C.byref(cfg), _f(o), _f(sl), _d(m), _f(chi), _i(it), _i(acc), _f(fit))
    return m, float(chi[0]), int(it[0]), int(acc[0]), fit.reshape(4, cfg.nl)


def lm_batch_f(cfg, obs, slight=None, slight_per_pixel=False, nthreads=0):
    obs = np.ascontiguousarray(obs, dtype=np.float32)
    P = obs.shape[0]
    sl = None if slight is None else np.ascontiguousarray(slight, dtype=np.float32)
    m = np.zeros((P, NPAR))
    chi = np.zeros(P, dtype=np.float32)
    it = np.zeros(P, dtype=np.int32)
    acc = np.zeros(P, dtype=np.int32)
    fit = np.zeros((P, 4, cfg.nl), dtype=np.float32)
    lib().orc_lm_batch_f(C.byref(cfg), P, _f(obs), _f(sl), int(slight_per_pixel), _d(m),
                         _f(chi), _i(it), _i(acc), _f(fit), nthreads)
    return m, chi, it, acc, fit
