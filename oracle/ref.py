"""ctypes wrapper of the reference's own per-pixel routines, built from its
sources by oracle/build_ref.py (libgmref_cpu.so: host C++ with OpenMP;
libgmref_gpu.so: sm_100a with the reference's launch geometry).

TEST AND BENCHMARK INFRASTRUCTURE ONLY: imported by tests/ and by bench.py's
reference and cpu_baseline legs, as the thing compared against.  The engine
under g-milos_b200/ never imports this module.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CPU_LIB = os.path.join(HERE, "_ref", "libgmref_cpu.so")
GPU_LIB = os.path.join(HERE, "_ref", "libgmref_gpu.so")
MAXNL = 50
FE6173_QUANTUM = (2.0, 1.0, 1.0, 2.0, 2.0, 0.0)


class Setup(C.Structure):
    _fields_ = [("nl", C.c_int), ("lambda_", C.c_double * MAXNL), ("lambda0", C.c_double),
                ("quantum", C.c_double * 6), ("use_psf", C.c_int), ("psf", C.c_double * MAXNL),
                ("weight", C.c_float * 4), ("noise", C.c_float), ("mu", C.c_float),
                ("ilambda", C.c_float), ("toplim", C.c_double), ("miter", C.c_int),
                ("logclambda", C.c_int), ("fix", C.c_int * 11), ("init", C.c_double * 11)]


class GpuReport(C.Structure):
    _fields_ = [("kernel_ms", C.c_float), ("e2e_ms", C.c_float), ("num_blocks", C.c_int),
                ("threads_per_block", C.c_int), ("n_rte_parallel", C.c_int),
                ("nstreams", C.c_int), ("heap_bytes", C.c_ulonglong),
                ("stack_bytes", C.c_ulonglong), ("local_bytes", C.c_ulonglong),
                ("regs", C.c_int), ("malloc_failures", C.c_uint), ("cuda_error", C.c_int),
                ("msg", C.c_char * 256)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["msg"] = self.msg.decode(errors="replace")
        return d


def available(gpu=False):
    return os.path.exists(GPU_LIB if gpu else CPU_LIB)


_cpu = None
_gpu = None


def _p(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def cpu_lib():
    global _cpu
    if _cpu is None:
        if not os.path.exists(CPU_LIB):
            raise FileNotFoundError(f"{CPU_LIB} not built (python oracle/build_ref.py)")
        L = C.CDLL(CPU_LIB)
        sp = C.POINTER(Setup)
        fp, dp, ip = C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.gmref_cpu_invert.argtypes = [sp, fp, C.c_longlong, fp, C.c_int, dp, fp, ip, fp, C.c_int]
        L.gmref_cpu_synth.argtypes = [sp, dp, fp, fp, fp, C.c_int]
        L.gmref_cpu_cuantic.argtypes = [sp, fp]
        L.gmref_cpu_max_threads.restype = C.c_int
        _cpu = L
    return _cpu


def gpu_lib():
    global _gpu
    if _gpu is None:
        if not os.path.exists(GPU_LIB):
            raise FileNotFoundError(f"{GPU_LIB} not built (python oracle/build_ref.py)")
        L = C.CDLL(GPU_LIB)
        sp = C.POINTER(Setup)
        fp, dp, ip = C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.gmref_gpu_invert.argtypes = [sp, fp, C.c_longlong, fp, C.c_int, C.c_int, dp, fp, ip,
                                       fp, C.POINTER(GpuReport)]
        _gpu = L
    return _gpu


def setup_from_cfg(cfg, quantum=FE6173_QUANTUM):
    """A reference setup carrying the same configuration as an oracle Cfg."""
    s = Setup()
    s.nl = cfg.nl
    if cfg.nl > MAXNL:
        raise ValueError(f"the reference supports at most {MAXNL} samples")
    for i in range(cfg.nl):
        s.lambda_[i] = cfg.lambda_[i]
        s.psf[i] = cfg.psf[i]
    s.lambda0 = cfg.lambda0
    for i in range(6):
        s.quantum[i] = quantum[i]
    s.use_psf = cfg.use_psf
    for i in range(4):
        s.weight[i] = cfg.weight[i]
    s.noise = cfg.noise
    s.mu = cfg.mu
    s.ilambda = cfg.ilambda
    s.toplim = cfg.toplim
    s.miter = cfg.miter
    s.logclambda = cfg.logclambda
    for i in range(11):
        s.fix[i] = cfg.fix[i]
        s.init[i] = cfg.init[i]
    return s


def max_threads():
    return cpu_lib().gmref_cpu_max_threads()


def cuantic(setup):
    out = np.zeros(66, dtype=np.float32)
    if cpu_lib().gmref_cpu_cuantic(C.byref(setup), _p(out, C.c_float)):
        raise RuntimeError("gmref_cpu_cuantic failed")
    return out


def synth(setup, model, slight=None, rf=False, nterms=10):
    nl = setup.nl
    m = np.ascontiguousarray(model, dtype=np.float64)
    sl = None if slight is None else np.ascontiguousarray(slight, dtype=np.float32)
    spec = np.zeros(4 * nl, dtype=np.float32)
    r = np.zeros(4 * nterms * nl, dtype=np.float32) if rf else None
    if cpu_lib().gmref_cpu_synth(C.byref(setup), _p(m, C.c_double), _p(sl, C.c_float),
                                 _p(spec, C.c_float), _p(r, C.c_float), int(nterms)):
        raise RuntimeError("gmref_cpu_synth failed")
    spec = spec.reshape(4, nl)
    return (spec, r.reshape(4, nterms, nl)) if rf else spec


def invert_cpu(setup, obs, slight=None, slight_per_pixel=False, nthreads=0, fitted=False):
    obs = np.ascontiguousarray(obs, dtype=np.float32)
    P = obs.shape[0]
    sl = None if slight is None else np.ascontiguousarray(slight, dtype=np.float32)
    m = np.zeros((P, 11))
    chi = np.zeros(P, dtype=np.float32)
    it = np.zeros(P, dtype=np.int32)
    fit = np.zeros((P, 4, setup.nl), dtype=np.float32) if fitted else None
    rc = cpu_lib().gmref_cpu_invert(C.byref(setup), _p(obs, C.c_float), P, _p(sl, C.c_float),
                                    int(slight_per_pixel), _p(m, C.c_double),
                                    _p(chi, C.c_float), _p(it, C.c_int), _p(fit, C.c_float),
                                    int(nthreads))
    if rc:
        raise RuntimeError(f"gmref_cpu_invert failed ({rc})")
    return m, chi, it, fit


def invert_gpu(setup, obs, slight=None, slight_per_pixel=False, nstreams=16, fitted=False):
    obs = np.ascontiguousarray(obs, dtype=np.float32)
    P = obs.shape[0]
    sl = None if slight is None else np.ascontiguousarray(slight, dtype=np.float32)
    m = np.zeros((P, 11))
    chi = np.zeros(P, dtype=np.float32)
    it = np.zeros(P, dtype=np.int32)
    fit = np.zeros((P, 4, setup.nl), dtype=np.float32) if fitted else None
    rep = GpuReport()
    rc = gpu_lib().gmref_gpu_invert(C.byref(setup), _p(obs, C.c_float), P, _p(sl, C.c_float),
                                    int(slight_per_pixel), int(nstreams), _p(m, C.c_double),
                                    _p(chi, C.c_float), _p(it, C.c_int), _p(fit, C.c_float),
                                    C.byref(rep))
    if rc:
        raise RuntimeError(f"gmref_gpu_invert failed ({rc}): {rep.msg.decode(errors='replace')}")
    return m, chi, it, fit, rep.as_dict()
