"""The C ABI library without a GPU: it loads, exports what include/gmilos.h
declares, its host-side set-up helpers agree with the oracle, and it fails
loudly (an error status, no fallback) when no CUDA device is present."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import gmilos_b200 as G
import helpers as H
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "gmilos.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(gm_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_function():
    names = header_functions()
    assert set(names) == set(G.EXPORTS), names
    lib = C.CDLL(G.LIB_PATH)
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", G.LIB_PATH], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(r"\bT %s\b" % n, out), n


def test_library_exports_every_file_format_function():
    txt = open(os.path.join(ROOT, "include", "gmilos_io.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = sorted(set(re.findall(r"\b(gm_(?:io|fits)_[a-z0-9_]+)\s*\(", txt)))
    assert len(names) >= 20, names
    out = subprocess.run(["nm", "-D", "--defined-only", G.LIB_PATH], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(r"\bT %s\b" % n, out), n


def test_wave_state_bytes():
    """Per pixel of a chunk: the 576-byte LM record, the staging block of
    (27 LPL + 1) x 32 floats and three list entries; 16 bytes of counters per
    wave (1 + max(miter, 1) waves) and 256 bytes of alignment slack."""
    per1 = 576 + 4 * (27 * 1 + 1) * 32 + 12
    per2 = 576 + 4 * (27 * 2 + 1) * 32 + 12
    assert G.wave_state_bytes(30, 50, 1000) == 1000 * per1 + 16 * 51 + 256
    assert G.wave_state_bytes(32, 50, 1000) == 1000 * per1 + 16 * 51 + 256
    assert G.wave_state_bytes(33, 50, 1000) == 1000 * per2 + 16 * 51 + 256
    assert G.wave_state_bytes(30, 0, 10) == 10 * per1 + 16 * 2 + 256
    assert G.wave_state_bytes(30, 50, 0) == 16 * 51 + 256
    for bad in ((0, 50, 10), (G.MAX_NL + 1, 50, 10), (30, 50, -1)):
        assert G.wave_state_bytes(*bad) == 0
    # a full 2^20-pixel chunk at nl <= 32: about 4.2 KB per pixel
    assert 4.1e3 < G.wave_state_bytes(30, 50, 1 << 20) / (1 << 20) < 4.3e3


def test_status_strings():
    lib = G.lib()
    assert lib.gm_status_string(0) == b"ok"
    assert lib.gm_status_string(5) == b"unsupported"


def test_config_defaults_follow_reference():
    c = G.Config()
    G.lib().gm_config_defaults(C.byref(c))
    assert c.abi_version == G.ABI_VERSION
    assert list(c.weight) == [1.0] * 4
    assert c.noise == pytest.approx(1e-6)
    assert c.ilambda == pytest.approx(0.1)
    assert c.toplim == 1e-12
    assert c.mu == 1.0
    assert c.reference_quirks == 1
    assert c.lambda_per_pixel == 0 and not c.lambda_map


def test_per_pixel_wavelength_map_binding():
    lam = np.linspace(6172.9, 6173.9, 30)
    lmap = np.repeat(lam[None], 5, 0) + np.arange(5)[:, None] * 1e-3
    c = G.make_config(lam, 6173.3356, G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0), lambda_map=lmap)
    assert c.lambda_per_pixel == 1
    assert c.lambda_map[4 * 30 + 29] == lmap[4, 29]
    with pytest.raises(ValueError):
        G.make_config(lam, 6173.3356, G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0), lambda_map=lmap[:, :10])


@pytest.mark.parametrize("levels", [(2, 1, 1.0, 2, 2, 0.0), (2, 2, 0.0, 3, 2, 1.0),
                                    (2, 1, 2.0, 2, 1, 3.0), (3, 3, 5.0, 3, 0, 4.0),
                                    (2.5, 0, 2.5, 1.5, 2, 2.5)])
def test_zeeman_matches_oracle(levels):
    a = G.zeeman_from_levels(*levels, 1.0)
    b = O.cuanten(*levels, 1.0)
    assert (a.n_pi, a.n_sig) == (b.n_pi, b.n_sig)
    for f in ("nub", "nup", "nur", "web", "wep", "wer"):
        np.testing.assert_allclose(list(getattr(a, f)), list(getattr(b, f)), rtol=1e-6, atol=1e-7)
    assert a.geff == pytest.approx(b.geff, rel=1e-6)


def test_psf_helpers_match_oracle():
    g = H.kat()
    off = G.grid_offsets_mA(-350, 35, 665)
    np.testing.assert_array_equal(G.psf_from_table(g["psf_x_mA"], g["psf_y"], off, 35.0),
                                  O.psf_from_table(g["psf_x_mA"], g["psf_y"], off, 35.0))
    lam = G.grid_lambda(6173.3356, -350, 35, 665)
    np.testing.assert_array_equal(G.psf_gaussian(100.0, lam), O.psf_gauss(100.0, lam))


def test_invalid_arguments_are_errors():
    with pytest.raises(G.GmError):
        G.zeeman_from_levels(2, 1, -1.0, 2, 2, 0.0)
    with pytest.raises(G.GmError):
        G.psf_gaussian(-5.0, np.arange(30.0))


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_no_device_is_an_error_not_a_fallback():
    with pytest.raises(G.GmError) as e:
        G.Engine(0)
    assert e.value.status == 2
