"""Python binding of the file-format library (include/gmilos_io.h), part of
libgmilos.so: control files, models, grids, line lists, PSF tables, .per
profiles and FITS cubes in the reference's formats.  Host-only: none of
these calls needs a GPU."""
import ctypes as C

import numpy as np

from . import GmError, lib as _engine_lib

PATH = 4096
NPAR = 11


class Trol(C.Structure):
    _fields_ = [("ncycles", C.c_int), ("observed", C.c_char * PATH), ("stray", C.c_char * PATH),
                ("psf", C.c_char * PATH), ("use_psf", C.c_int), ("fwhm_mA", C.c_double),
                ("wavelength", C.c_char * PATH), ("grid", C.c_char * PATH), ("use_grid", C.c_int),
                ("lines", C.c_char * PATH), ("abundances", C.c_char * PATH),
                ("init_model", C.c_char * PATH), ("init_model2", C.c_char * PATH),
                ("weight", C.c_float * 4), ("auto_nodes", C.c_int), ("fix", C.c_int * NPAR),
                ("fix2", C.c_int * NPAR), ("invert_filling_factor", C.c_int), ("mu", C.c_float),
                ("sn_i", C.c_int), ("noise", C.c_double), ("continuum_contrast", C.c_int),
                ("ilambda", C.c_float), ("use_fft", C.c_int), ("logclambda", C.c_int),
                ("nstreams", C.c_int), ("device", C.c_int)]


_io = None


def lib():
    global _io
    if _io is None:
        L = _engine_lib()
        vp, cp, dp, fp, ip = C.c_void_p, C.c_char_p, C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_int)
        L.gm_io_last_error.restype = C.c_char_p
        L.gm_io_trol_defaults.argtypes = [C.POINTER(Trol)]
        L.gm_io_trol_defaults.restype = None
        L.gm_io_read_trol.argtypes = [cp, C.POINTER(Trol)]
        L.gm_io_read_model.argtypes = [cp, dp]
        L.gm_io_write_model.argtypes = [cp, dp, C.c_int, C.c_float]
        L.gm_io_read_grid.argtypes = [cp, ip, dp, dp, dp]
        L.gm_io_grid_wavelengths.argtypes = [C.c_double] * 4 + [dp, dp, C.c_int]
        L.gm_io_read_line.argtypes = [cp, C.c_int, dp, dp]
        L.gm_io_read_psf_table.argtypes = [cp, dp, dp, C.c_int, ip]
        L.gm_io_read_per.argtypes = [cp, C.c_int, fp, dp]
        L.gm_io_write_per.argtypes = [cp, C.c_int, C.c_int, dp, fp]
        L.gm_fits_read_cube.argtypes = [cp, C.c_int, C.POINTER(vp)]
        L.gm_fits_cube_dims.argtypes = [vp, ip, ip, ip]
        L.gm_fits_cube_dims.restype = None
        L.gm_fits_cube_data.argtypes = [vp]
        L.gm_fits_cube_data.restype = fp
        L.gm_fits_cube_free.argtypes = [vp]
        L.gm_fits_cube_free.restype = None
        L.gm_fits_write_profiles.argtypes = [cp, vp, fp]
        L.gm_fits_write_models.argtypes = [cp, C.c_int, C.c_int, dp, ip, fp, C.c_int]
        L.gm_fits_read_stray.argtypes = [cp, C.c_int, C.POINTER(fp), ip, ip, ip]
        L.gm_fits_read_lambda.argtypes = [cp, dp, C.c_int, ip, ip]
        L.gm_fits_read_lambda_map.argtypes = [cp, C.POINTER(dp), ip, ip, ip, ip, ip]
        L.gm_fits_write_image.argtypes = [cp, C.c_int, C.POINTER(C.c_int64), fp, C.POINTER(C.c_char_p), C.c_int]
        L.gm_io_free.argtypes = [vp]
        L.gm_io_free.restype = None
        _io = L
    return _io


def _b(path):
    return str(path).encode()


def _check(st):
    if st != 0:
        raise GmError(st, lib().gm_io_last_error().decode(errors="replace"))


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _i(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def read_trol(path):
    t = Trol()
    _check(lib().gm_io_read_trol(_b(path), C.byref(t)))
    return t


def read_model(path, base=None):
    m = np.zeros(NPAR) if base is None else np.array(base, dtype=np.float64)
    _check(lib().gm_io_read_model(_b(path), _d(m)))
    return m


def write_model(path, model, iters=0, chi2=0.0):
    m = np.ascontiguousarray(model, dtype=np.float64)
    _check(lib().gm_io_write_model(_b(path), _d(m), int(iters), float(chi2)))


def read_grid(path):
    idx = C.c_int()
    a, s, b = C.c_double(), C.c_double(), C.c_double()
    _check(lib().gm_io_read_grid(_b(path), C.byref(idx), C.byref(a), C.byref(s), C.byref(b)))
    return idx.value, a.value, s.value, b.value


def grid_wavelengths(lambda0, first, step, last, cap=256):
    off = np.zeros(cap)
    lam = np.zeros(cap)
    n = lib().gm_io_grid_wavelengths(lambda0, first, step, last, _d(off), _d(lam), cap)
    return off[:n], lam[:n]


def read_line(path, index):
    l0 = C.c_double()
    q = np.zeros(6)
    _check(lib().gm_io_read_line(_b(path), int(index), C.byref(l0), _d(q)))
    return l0.value, q


def read_psf_table(path, cap=200000):
    x = np.zeros(cap)
    y = np.zeros(cap)
    n = C.c_int()
    _check(lib().gm_io_read_psf_table(_b(path), _d(x), _d(y), cap, C.byref(n)))
    return x[:n.value], y[:n.value]


def read_per(path, nl):
    iquv = np.zeros(4 * nl, dtype=np.float32)
    off = np.zeros(nl)
    _check(lib().gm_io_read_per(_b(path), nl, _f(iquv), _d(off)))
    return iquv.reshape(4, nl), off


def write_per(path, line_index, offsets, iquv):
    off = np.ascontiguousarray(offsets, dtype=np.float64)
    s = np.ascontiguousarray(iquv, dtype=np.float32).reshape(-1)
    _check(lib().gm_io_write_per(_b(path), int(line_index), len(off), _d(off), _f(s)))


def read_cube(path, nl=0):
    """(pixels [rows*cols][4][nl], rows, cols); pixel p = col * rows + row."""
    h = C.c_void_p()
    _check(lib().gm_fits_read_cube(_b(path), int(nl), C.byref(h)))
    try:
        r, c, n = C.c_int(), C.c_int(), C.c_int()
        lib().gm_fits_cube_dims(h, C.byref(r), C.byref(c), C.byref(n))
        P = r.value * c.value
        ptr = lib().gm_fits_cube_data(h)
        data = np.ctypeslib.as_array(ptr, shape=(P * 4 * n.value,)).copy().reshape(P, 4, n.value)
    finally:
        lib().gm_fits_cube_free(h)
    return data, r.value, c.value


def write_profiles_like(path, like_path, iquv, nl):
    h = C.c_void_p()
    _check(lib().gm_fits_read_cube(_b(like_path), int(nl), C.byref(h)))
    try:
        s = np.ascontiguousarray(iquv, dtype=np.float32).reshape(-1)
        _check(lib().gm_fits_write_profiles(_b(path), h, _f(s)))
    finally:
        lib().gm_fits_cube_free(h)


def write_models(path, rows, cols, models, iters=None, chi2=None, with_chi2=True):
    m = np.ascontiguousarray(models, dtype=np.float64)
    it = None if iters is None else np.ascontiguousarray(iters, dtype=np.int32)
    ch = None if chi2 is None else np.ascontiguousarray(chi2, dtype=np.float32)
    _check(lib().gm_fits_write_models(_b(path), int(rows), int(cols), _d(m),
                                      None if it is None else _i(it), None if ch is None else _f(ch),
                                      int(with_chi2)))


def read_stray(path, nl):
    out = C.POINTER(C.c_float)()
    pp, r, c = C.c_int(), C.c_int(), C.c_int()
    _check(lib().gm_fits_read_stray(_b(path), int(nl), C.byref(out), C.byref(pp), C.byref(r), C.byref(c)))
    n = 4 * nl * (r.value * c.value if pp.value else 1)
    arr = np.ctypeslib.as_array(out, shape=(n,)).copy()
    lib().gm_io_free(C.cast(out, C.c_void_p))
    if pp.value:
        return arr.reshape(r.value * c.value, 4, nl), True
    return arr.reshape(4, nl), False


def read_lambda(path, cap=256):
    lam = np.zeros(cap)
    n, idx = C.c_int(), C.c_int()
    _check(lib().gm_fits_read_lambda(_b(path), _d(lam), cap, C.byref(n), C.byref(idx)))
    return lam[:n.value], idx.value


def read_lambda_map(path):
    """Wavelength FITS with one grid or per-pixel grids (gm_fits_read_lambda_map):
    (grids [nl] or [P][nl], line index, per_pixel, rows, cols)."""
    out = C.POINTER(C.c_double)()
    pp, r, c, n, idx = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
    _check(lib().gm_fits_read_lambda_map(_b(path), C.byref(out), C.byref(pp), C.byref(r), C.byref(c),
                                         C.byref(n), C.byref(idx)))
    P = r.value * c.value if pp.value else 1
    g = np.ctypeslib.as_array(out, shape=(P * n.value,)).copy()
    lib().gm_io_free(C.cast(out, C.c_void_p))
    g = g.reshape(P, n.value) if pp.value else g
    return g, idx.value, bool(pp.value), r.value, c.value


def write_image(path, data, cards=()):
    """data: numpy array whose LAST axis is NAXIS1 (C order = FITS order)."""
    a = np.ascontiguousarray(data, dtype=np.float32)
    naxes = (C.c_int64 * a.ndim)(*reversed(a.shape))
    cs = (C.c_char_p * max(1, len(cards)))(*[c.encode() for c in cards])
    _check(lib().gm_fits_write_image(_b(path), a.ndim, naxes, _f(a.reshape(-1)), cs, len(cards)))


def read_image(path):
    """Minimal FITS reader for tests: (data with NAXIS1 last, {key: value})."""
    raw = open(path, "rb").read()
    cards, off = {}, 0
    while True:
        block = raw[off:off + 2880]
        off += 2880
        done = False
        for i in range(36):
            card = block[80 * i:80 * (i + 1)].decode("ascii")
            key = card[:8].strip()
            if key == "END":
                done = True
                break
            if card[8:10] == "= ":
                cards[key] = card[10:].split("/")[0].strip().strip("'").strip()
        if done:
            break
    naxis = int(cards["NAXIS"])
    shape = [int(cards["NAXIS%d" % (k + 1)]) for k in range(naxis)]
    bitpix = int(cards["BITPIX"])
    dt = {-32: ">f4", -64: ">f8", 16: ">i2", 32: ">i4"}[bitpix]
    n = int(np.prod(shape))
    data = np.frombuffer(raw, dtype=dt, count=n, offset=off).astype(np.float64)
    return data.reshape(list(reversed(shape))), cards
