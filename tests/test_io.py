"""The reference's file formats (include/gmilos_io.h): control file, models,
grids, line list, PSF tables, .per profiles and FITS cubes.  Host-only.

Files are written here in the reference's layouts; where the reference's own
example files are present (its run/ directory) they are parsed as well."""
import os

import numpy as np
import pytest

import gmilos_b200.io as gio

from build_ref import locate_reference

REF = locate_reference() or ""

FIELDS = ["Number of cycles          (*)", "Observed profiles          (*)", "Stray light file             ",
          "PSF file                     ", "Wavelength grid file      (s)", "Atomic parameters file       ",
          "Abundances file              ", "Initial guess model 1     (*)", "Initial guess model 2        ",
          "Weight for Stokes I          ", "Weight for Stokes Q          ", "Weight for Stokes U          ",
          "Weight for Stokes V          ", "AUTOMATIC SELECT. OF NODES?  ", "Nodes for S_0 1              ",
          "Nodes for S_1 1              ", "Nodes for eta0 1             ", "Nodes for magnetic field 1   ",
          "Nodes for LOS velocity 1     ", "Nodes for gamma 1            ", "Nodes for phi 1              ",
          "Nodes for lambda_doppler 1   ", "Nodes for damping 1          ", "Invert macroturbulence 1     ",
          "Nodes for S_0 2              ", "Nodes for S_1 2              ", "Nodes for eta0 2             ",
          "Nodes for magnetic field 2   ", "Nodes for LOS velocity 2     ", "Nodes for gamma 2            ",
          "Nodes for phi 2              ", "Nodes for lambda_doppler 2   ", "Nodes for damping 2          ",
          "Invert macroturbulence 2?    ", "Invert filling factor?       ", "Invert stray light factor?   ",
          "mu=cos (theta)               ", "Estimated S/N for I          ", "Continuum contrast           ",
          "Initial diagonal element     ", "Use FFT for convolutions     ", "Diagonal element acceleration",
          "Number of Streams            ", "Device number                "]


def write_trol(path, values):
    with open(path, "w") as f:
        for name, v in zip(FIELDS, values):
            f.write("%s:%-20s ! comment\n" % (name, v))


def fe_lines(path):
    with open(path, "w") as f:
        f.write("1=FE 1   6173.3356    1.0  2.223 -2.880   5P 1.0- 5D 0.0  0.266  7.868e-15\n")
        f.write("3=FE 1   6302.494    1.0  3.69  -1.16    5P 1.0- 5D 0.0\n")
        f.write("12=FE 1  7090.3835    1.0   4.23 -1.21    6S 2.5- 4D 2.5\n")


def grid_file(path, idx=1, a=-350, s=35, b=665):
    with open(path, "w") as f:
        f.write("header line\n\nLine indices : Initial lambda Step Final lambda\n")
        f.write("-----------------------------------------------------------------------\n")
        f.write("%d                       :        %s,            %s,           %s\n" % (idx, a, s, b))


def test_control_file(tmp_path):
    psf = tmp_path / "p.psf"
    psf.write_text("-10.0 0.1\n0.0 1.0\n10.0 0.1\n")
    grid = tmp_path / "g.grid"
    grid_file(grid)
    vals = ["25", "obs.fits", "", str(psf), str(grid), "LINES", "", "guess.mod", "", "1", "0.5", "0.5", "2",
            "", "1", "0", "1", "1", "1", "1", "1", "1", "1", "1", "", "", "", "", "", "", "", "", "", "",
            "", "1", "0.9", "500", "", "0.01", "0", "1", "16", "3"]
    write_trol(tmp_path / "a.mtrol", vals)
    t = gio.read_trol(tmp_path / "a.mtrol")
    assert t.ncycles == 25 and t.observed == b"obs.fits" and t.stray == b""
    assert t.use_psf == 1 and t.fwhm_mA == 0 and t.use_grid == 1 and t.grid == str(grid).encode()
    assert list(t.weight) == [1.0, 0.5, 0.5, 2.0]
    # S0, S1, eta0, B, vlos, gamma, phi, dopp, damping, mac in the file's order
    assert list(t.fix) == [1, 1, 1, 1, 1, 1, 1, 1, 0, 1, 1]
    assert t.mu == pytest.approx(0.9) and t.sn_i == 500 and t.noise == pytest.approx(4e-6)
    assert t.ilambda == pytest.approx(0.01) and t.logclambda == 1 and t.nstreams == 16 and t.device == 3
    # a number in the PSF field is a Gaussian FWHM; empty fields keep defaults
    vals[3] = "90.5"
    vals[9] = ""
    vals[37] = ""
    vals[39] = ""
    write_trol(tmp_path / "b.mtrol", vals)
    t = gio.read_trol(tmp_path / "b.mtrol")
    assert t.use_psf == 1 and t.fwhm_mA == pytest.approx(90.5)
    assert t.weight[0] == 1.0 and t.noise == pytest.approx(1e-6) and t.ilambda == pytest.approx(0.1)
    vals[3] = ""
    write_trol(tmp_path / "c.mtrol", vals)
    assert gio.read_trol(tmp_path / "c.mtrol").use_psf == 0
    # a PSF file with another extension is an error, as in the reference
    bad = tmp_path / "p.txt"
    bad.write_text("0 1\n")
    vals[3] = str(bad)
    write_trol(tmp_path / "d.mtrol", vals)
    with pytest.raises(gio.GmError):
        gio.read_trol(tmp_path / "d.mtrol")
    # short files are errors
    (tmp_path / "e.mtrol").write_text("Number of cycles: 3\n")
    with pytest.raises(gio.GmError):
        gio.read_trol(tmp_path / "e.mtrol")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "run")), reason="reference example files absent")
def test_reference_example_files(monkeypatch):
    monkeypatch.chdir(REF)
    t = gio.read_trol("run/invert.mtrol")
    assert t.ncycles == 100 and t.observed == b"data/synthesis_gpu.per"
    assert t.use_psf == 1 and t.use_grid == 1 and t.grid == b"run/malla.grid"
    assert list(t.fix) == [1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0]
    assert t.noise == pytest.approx(1e-6) and t.nstreams == 4
    assert gio.read_trol("run/synthesis.mtrol").ncycles == 0
    idx, a, s, b = gio.read_grid("run/malla.grid")
    assert (idx, a, s, b) == (1, -350.0, 35.0, 665.0)
    l0, q = gio.read_line("run/LINES", 1)
    assert l0 == pytest.approx(6173.3356) and list(q) == [2, 1, 1.0, 2, 2, 0.0]
    m = gio.read_model("run/guess.mod")
    assert list(m) == [40, 1000, 0.2, 0.03, 0.05, 150, 110, 0.35, 0.5, 0, 1]
    x, y = gio.read_psf_table("run/CRISP_6173_1mA.psf")
    assert len(x) > 5000 and x[0] == -2750.0 and np.all(np.diff(x) > 0)
    off, _ = gio.grid_wavelengths(l0, a, s, b)
    per, poff = gio.read_per("data/synthesis_gpu.per", len(off))
    np.testing.assert_allclose(poff, off, atol=1e-6)
    assert per.shape == (4, 30) and 0.5 < per[0, 0] < 1.0


def test_models_grids_lines_psf_per(tmp_path):
    mod = tmp_path / "m.mod"
    mod.write_text("eta_0:          20\nmagnetic field: 1100\nLOS velocity:   0.2\nDoppler width:  0.03\n"
                   "damping:        0.05\ngamma:          120\nphi:            150\nS_0:            0.35\n"
                   "S_1:            0.5\nv_mac:          0\nfilling factor: 1---\n")
    m = gio.read_model(mod)
    assert list(m) == [20, 1100, 0.2, 0.03, 0.05, 120, 150, 0.35, 0.5, 0, 1]
    gio.write_model(tmp_path / "o.mod", m * 1.5, iters=17, chi2=1.25)
    m2 = gio.read_model(tmp_path / "o.mod")
    np.testing.assert_allclose(m2, m * 1.5, rtol=1e-6)
    txt = (tmp_path / "o.mod").read_text()
    assert "# Iterations        :17" in txt and "chisqr" in txt
    # absent keys keep the caller's values
    (tmp_path / "p.mod").write_text("magnetic field: 7\n")
    np.testing.assert_array_equal(gio.read_model(tmp_path / "p.mod", base=np.arange(11.0)),
                                  [0, 7, 2, 3, 4, 5, 6, 7, 8, 9, 10])
    grid_file(tmp_path / "x.grid", 3, -120.5, 21.53, 1000)
    assert gio.read_grid(tmp_path / "x.grid") == (3, -120.5, 21.53, 1000.0)
    off, lam = gio.grid_wavelengths(6302.494, -350, 35, 665)
    assert len(off) == 30 and off[-1] == pytest.approx(665) and lam[0] == pytest.approx(6302.144)
    fe_lines(tmp_path / "LINES")
    l0, q = gio.read_line(tmp_path / "LINES", 3)
    assert l0 == pytest.approx(6302.494) and list(q) == [2, 1, 1.0, 2, 2, 0.0]
    l0, q = gio.read_line(tmp_path / "LINES", 12)
    # even multiplicity: S = (6 - 1) / 2 in integer arithmetic, as the reference stores it
    assert list(q) == [2, 0, 2.5, 1, 2, 2.5]
    with pytest.raises(gio.GmError):
        gio.read_line(tmp_path / "LINES", 9)
    (tmp_path / "t.psf").write_text("\t-2.0    1e-3\n\t-1.0    0.5\n\t0.0    1.0\n\t1.0    0.5\n")
    x, y = gio.read_psf_table(tmp_path / "t.psf")
    np.testing.assert_array_equal(x, [-2, -1, 0, 1])
    rng = np.random.default_rng(0)
    prof = rng.normal(size=(4, 30)).astype(np.float32)
    gio.write_per(tmp_path / "a.per", 1, off, prof)
    back, boff = gio.read_per(tmp_path / "a.per", 30)
    np.testing.assert_allclose(back, prof, rtol=1e-6)
    np.testing.assert_allclose(boff, off, atol=1e-6)
    with pytest.raises(gio.GmError):
        gio.read_per(tmp_path / "a.per", 31)


CT = {"row": "HPLN-TAN", "col": "HPLT-TAN", "lam": "WAVE-GRI", "stokes": "STOKES"}


def cube_file(path, pix, rows, cols, order, ctype=True):
    """pix [P][4][nl] with p = col * rows + row, written with the FITS axes
    in `order` (NAXIS1 first)."""
    nl = pix.shape[2]
    size = {"row": rows, "col": cols, "lam": nl, "stokes": 4}
    arr = np.zeros([size[a] for a in reversed(order)], dtype=np.float32)
    for r in range(rows):
        for c in range(cols):
            p = c * rows + r
            for s in range(4):
                for l in range(nl):
                    idx = {"row": r, "col": c, "lam": l, "stokes": s}
                    arr[tuple(idx[a] for a in reversed(order))] = pix[p, s, l]
    cards = []
    if ctype:
        for k, a in enumerate(order):
            cards.append("CTYPE%d  = '%-8s'           / axis %d" % (k + 1, CT[a], k + 1))
    cards.append("OBSERVER= 'synthetic'          / kept in the fitted-profile file")
    gio.write_image(path, arr, cards)


@pytest.mark.parametrize("order,ctype", [(("lam", "stokes", "row", "col"), True),
                                         (("row", "col", "lam", "stokes"), True),
                                         (("stokes", "lam", "col", "row"), True),
                                         (("lam", "stokes", "row", "col"), False),
                                         (("stokes", "lam", "row", "col"), False)])
def test_fits_cube_axes_and_round_trip(tmp_path, order, ctype):
    rng = np.random.default_rng(1)
    # without CTYPE keywords the axes are told apart by length (Stokes the
    # shortest, wavelength the next), so the spatial axes must be longer
    rows, cols, nl = (7, 5, 12) if ctype else (17, 15, 12)
    pix = rng.normal(size=(rows * cols, 4, nl)).astype(np.float32)
    cube_file(tmp_path / "in.fits", pix, rows, cols, order, ctype)
    got, r, c = gio.read_cube(tmp_path / "in.fits", nl)
    assert (r, c) == (rows, cols)
    np.testing.assert_array_equal(got, pix)
    # fitted profiles keep the input's axes and user cards
    gio.write_profiles_like(tmp_path / "out.fits", tmp_path / "in.fits", pix * 2, nl)
    back, r2, c2 = gio.read_cube(tmp_path / "out.fits", nl)
    np.testing.assert_array_equal(back, pix * 2)
    _, cards = gio.read_image(tmp_path / "out.fits")
    assert cards["OBSERVER"] == "synthetic" and cards["BITPIX"] == "-32"
    with pytest.raises(gio.GmError):
        gio.read_cube(tmp_path / "in.fits", nl + 1)


def test_fits_models_and_stray_and_lambda(tmp_path):
    rows, cols = 3, 4
    P = rows * cols
    models = np.arange(P * 11, dtype=np.float64).reshape(P, 11)
    iters = np.arange(P, dtype=np.int32) + 100
    chi2 = np.linspace(1, 2, P).astype(np.float32)
    gio.write_models(tmp_path / "m.fits", rows, cols, models, iters, chi2)
    data, cards = gio.read_image(tmp_path / "m.fits")
    assert data.shape == (13, cols, rows) and cards["NAXIS1"] == str(rows)
    for r in range(rows):
        for c in range(cols):
            p = c * rows + r
            np.testing.assert_allclose(data[:11, c, r], models[p])
            assert data[11, c, r] == iters[p] and data[12, c, r] == pytest.approx(chi2[p])
    gio.write_models(tmp_path / "n.fits", rows, cols, models, iters, None, with_chi2=False)
    assert gio.read_image(tmp_path / "n.fits")[0].shape == (12, cols, rows)
    nl = 9
    prof = np.arange(4 * nl, dtype=np.float32).reshape(4, nl)
    gio.write_image(tmp_path / "s1.fits", prof)             # NAXIS1 = wavelength
    gio.write_image(tmp_path / "s2.fits", prof.T.copy())    # NAXIS1 = Stokes
    for f in ("s1.fits", "s2.fits"):
        s, per_pixel = gio.read_stray(tmp_path / f, nl)
        assert not per_pixel
        np.testing.assert_array_equal(s, prof)
    pix = np.random.default_rng(2).normal(size=(P, 4, nl)).astype(np.float32)
    cube_file(tmp_path / "s4.fits", pix, rows, cols, ("lam", "stokes", "row", "col"))
    s, per_pixel = gio.read_stray(tmp_path / "s4.fits", nl)
    assert per_pixel
    np.testing.assert_array_equal(s, pix)
    lam = 6173.3356 + np.arange(nl) * 0.035
    gio.write_image(tmp_path / "l.fits", np.stack([np.full(nl, 1.0), lam]).astype(np.float32))
    got, idx = gio.read_lambda(tmp_path / "l.fits")
    assert idx == 1
    np.testing.assert_allclose(got, lam.astype(np.float32))


def write_f64_image(path, data):
    """BITPIX -64 image, NAXIS1 = the last numpy axis (wavelengths kept exact)."""
    a = np.ascontiguousarray(data, dtype=">f8")
    cards = ["SIMPLE  = %20s" % "T", "BITPIX  = %20d" % -64, "NAXIS   = %20d" % a.ndim]
    cards += ["NAXIS%-3d= %20d" % (i + 1, n) for i, n in enumerate(reversed(a.shape))]
    cards.append("END")
    hdr = "".join(c.ljust(80) for c in cards)
    hdr = hdr.ljust((len(hdr) + 2879) // 2880 * 2880)
    body = a.tobytes()
    body += b"\0" * ((-len(body)) % 2880)
    with open(path, "wb") as f:
        f.write(hdr.encode() + body)


def lambda_map_planes(grids, rows, cols, line_index=1):
    """[1 + nl][cols][rows] planes of a per-pixel wavelength FITS; pixel p =
    col * rows + row as in the cube reader."""
    P, nl = grids.shape
    arr = np.zeros((nl + 1, cols, rows))
    arr[0] = line_index
    for r in range(rows):
        for c in range(cols):
            arr[1:, c, r] = grids[c * rows + r]
    return arr


def test_per_pixel_wavelength_fits(tmp_path):
    rows, cols, nl = 3, 4, 7
    P = rows * cols
    rng = np.random.default_rng(11)
    grids = 6173.0 + np.arange(nl) * 0.035 + rng.uniform(-0.02, 0.02, (P, 1))
    arr = lambda_map_planes(grids, rows, cols)
    write_f64_image(tmp_path / "lmap3.fits", arr)
    write_f64_image(tmp_path / "lmap4.fits", arr[None])
    for f in ("lmap3.fits", "lmap4.fits"):
        g, idx, per_pixel, r, c = gio.read_lambda_map(tmp_path / f)
        assert per_pixel and (r, c) == (rows, cols) and idx == 1
        np.testing.assert_array_equal(g, grids)
    # one grid, 2-D: line index row, wavelength row
    write_f64_image(tmp_path / "l2.fits", np.stack([np.full(nl, 2.0), grids[0]]))
    g, idx, per_pixel, r, c = gio.read_lambda_map(tmp_path / "l2.fits")
    assert not per_pixel and idx == 2
    np.testing.assert_array_equal(g, grids[0])
    with pytest.raises(gio.GmError):          # the 2-D reader points to the map reader
        gio.read_lambda(tmp_path / "lmap3.fits")
    arr[0, 1, 2] = 2                           # one line per run
    write_f64_image(tmp_path / "bad.fits", arr)
    with pytest.raises(gio.GmError):
        gio.read_lambda_map(tmp_path / "bad.fits")
