"""The `gmilos` command-line front end end to end: control file in, the
reference's output files out (synthesis, classical estimates, .per and FITS
inversions), checked against the known-answer vector, the oracle and the
engine's own API on the same inputs."""
import os
import subprocess

import numpy as np
import pytest

import gmilos_b200 as G
import gmilos_b200.io as gio
import helpers as H
import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "g-milos_b200", "bin", "gmilos")

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


def setup_dir(d, ncycles, observed="", stray="", init=None, stray_free=0, mac_free=0, wavelength="malla.grid"):
    """Line list, grid, PSF table and guess model of the known-answer case."""
    g = H.kat()
    (d / "LINES").write_text("1=FE 1   6173.3356    1.0  2.223 -2.880   5P 1.0- 5D 0.0  0.266  7.868e-15\n")
    first, step, last = g["grid"]
    (d / "malla.grid").write_text("Line indices : Initial lambda Step Final lambda\n"
                                  "------------------------------------------------\n"
                                  "1          :   %r,   %r,   %r\n" % (float(first), float(step), float(last)))
    with open(d / "crisp.psf", "w") as f:
        for x, y in zip(g["psf_x_mA"], g["psf_y"]):
            f.write("\t%.1f    %.7e\n" % (x, y))
    m = g["model"] if init is None else init
    names = ["eta_0", "magnetic field", "LOS velocity", "Doppler width", "damping", "gamma", "phi", "S_0",
             "S_1", "v_mac", "filling factor"]
    (d / "guess.mod").write_text("".join("%s: %.10g\n" % (n, v) for n, v in zip(names, m)))
    vals = [str(ncycles), observed, stray, "crisp.psf", wavelength, "LINES", "", "guess.mod", "", "1", "1",
            "1", "1", "", "1", "1", "1", "1", "1", "1", "1", "1", "1", str(mac_free)] + [""] * 10 + \
           ["", str(stray_free), "1", "1000", "", "0.1", "0", "0", "4", "0"]
    with open(d / "run.mtrol", "w") as f:
        for name, v in zip(FIELDS, vals):
            f.write("%s:%-20s ! comment\n" % (name, v))
    return g


def run_cli(d):
    assert os.path.exists(CLI), "g-milos_b200/bin/gmilos not built"
    r = subprocess.run([CLI, "run.mtrol", "--quiet"], cwd=d, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout


def kat_config(g, d, **kw):
    """The engine configuration the CLI builds, from the files it reads."""
    l0 = float(g["lambda0"])
    first, step, last = g["grid"]
    lam = G.grid_lambda(l0, first, step, last)
    off = G.grid_offsets_mA(first, step, last)
    x, y = gio.read_psf_table(d / "crisp.psf")
    psf = G.psf_from_table(x, y, off, step)
    return lam, off, psf, G.make_config(lam, l0, G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0), psf=psf, **kw)


def test_synthesis_mode_reproduces_the_known_answer(tmp_path):
    g = setup_dir(tmp_path, 0)
    run_cli(tmp_path)
    spec, off = gio.read_per(tmp_path / "guess.per", 30)
    np.testing.assert_allclose(off, g["per_offsets_mA"], atol=1e-6)
    assert H.normwise(spec, g["per_iquv"]).max() < 2e-6


def test_per_inversion_matches_the_engine_api(tmp_path):
    g = setup_dir(tmp_path, 50, observed="obs.per", init=H.GUESS)
    gio.write_per(tmp_path / "obs.per", 1, g["per_offsets_mA"], g["per_iquv"])
    run_cli(tmp_path)
    m = gio.read_model(tmp_path / "obs_model.mod")
    fit, _ = gio.read_per(tmp_path / "obs_stokes.per", 30)
    obs, _ = gio.read_per(tmp_path / "obs.per", 30)
    lam, off, psf, cfg = kat_config(g, tmp_path, init=H.GUESS, miter=50)
    with G.Engine(0) as e:
        e.configure(cfg)
        out = e.invert(np.ascontiguousarray(obs[None], dtype=np.float32), fitted=True)
    np.testing.assert_allclose(m, out["model64"][0], rtol=2e-6, atol=2e-6)
    np.testing.assert_allclose(fit, out["fitted"][0], rtol=1e-5, atol=1e-7)
    # the known-answer profile comes from run/init.mod: the fit recovers it
    assert abs(m[1] - g["model"][1]) < 5 and abs(m[5] - g["model"][5]) < 0.5


def test_fits_inversion_with_stray_light(tmp_path):
    g = setup_dir(tmp_path, 40, observed="cube.fits", stray="stray.per", init=list(H.GUESS[:10]) + [0.9],
                  stray_free=1)
    lam, off, psf, _ = kat_config(g, tmp_path)
    l0, zo = H.fe_line()
    ocfg = O.make_cfg(lam, l0, zo, psf=psf, fix=(1,) * 9 + (0, 1))
    gio.write_per(tmp_path / "stray.per", 1, np.trunc(off), H.stray_profile(ocfg))
    sl, _ = gio.read_per(tmp_path / "stray.per", 30)
    rng = np.random.default_rng(5)
    rows, cols = 6, 5
    t = H.truth_models(rows * cols, rng, alpha_range=(0.7, 1.0))
    obs = H.observations(ocfg, t, rng, slight=sl)
    from test_io import cube_file
    cube_file(tmp_path / "cube.fits", obs, rows, cols, ("lam", "stokes", "row", "col"))
    run_cli(tmp_path)
    planes, cards = gio.read_image(tmp_path / "cube_mod.fits")
    assert planes.shape == (13, cols, rows)
    fitted, r, c = gio.read_cube(tmp_path / "cube_stokes.fits", 30)
    assert (r, c) == (rows, cols)
    init = list(H.GUESS[:10]) + [0.9]
    cfg = G.make_config(lam, l0, G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0), psf=psf,
                        fix=(1,) * 9 + (0, 1), init=init, miter=40, slight=sl)
    with G.Engine(0) as e:
        e.configure(cfg)
        out = e.invert(obs, fitted=True)
    for rr in range(rows):
        for cc in range(cols):
            p = cc * rows + rr
            np.testing.assert_allclose(planes[:11, cc, rr], out["model"][p], rtol=1e-6)
            assert planes[11, cc, rr] == out["iters"][p]
            assert planes[12, cc, rr] == pytest.approx(out["chi2"][p], rel=1e-6)
    np.testing.assert_allclose(fitted, out["fitted"], rtol=1e-6, atol=1e-7)


def test_classical_estimates_mode(tmp_path):
    g = setup_dir(tmp_path, -1, observed="cube.fits", init=H.GUESS)
    lam, off, psf, _ = kat_config(g, tmp_path)
    l0, zo = H.fe_line()
    ocfg = O.make_cfg(lam, l0, zo, psf=psf)
    rng = np.random.default_rng(6)
    rows, cols = 4, 3
    t = H.truth_models(rows * cols, rng)
    obs = H.observations(ocfg, t, rng)
    from test_io import cube_file
    cube_file(tmp_path / "cube.fits", obs, rows, cols, ("stokes", "lam", "col", "row"))
    run_cli(tmp_path)
    planes, _ = gio.read_image(tmp_path / "cube_model_ce.fits")
    for rr in range(rows):
        for cc in range(cols):
            p = cc * rows + rr
            ref = O.classical(ocfg, obs[p], model=H.GUESS, for_init=0)
            got = planes[:11, cc, rr]
            for k in (1, 2, 5, 6, 7):      # B, vlos, gamma, phi and S0 = B_los
                assert got[k] == pytest.approx(ref[k], rel=1e-5, abs=1e-4), (k, got[k], ref[k])
            assert planes[11, cc, rr] == 0 and planes[12, cc, rr] == 0


def test_fits_inversion_on_per_pixel_wavelength_grids(tmp_path):
    """A per-pixel wavelength FITS (rows x cols x (1 + nl)): the CLI inverts
    each pixel on its own grid, with the PSF of the first pixel's grid, as the
    engine API does with lambda_map."""
    from test_io import cube_file, lambda_map_planes, write_f64_image
    g = setup_dir(tmp_path, 30, observed="cube.fits", init=H.GUESS, wavelength="lmap.fits")
    rows, cols = 5, 4
    P = rows * cols
    rng = np.random.default_rng(7)
    l0, zo = H.fe_line()
    first, step, last = g["grid"]
    lam0 = G.grid_lambda(l0, first, step, last)
    grids = lam0[None] + rng.uniform(-0.02, 0.02, (P, 1))
    write_f64_image(tmp_path / "lmap.fits", lambda_map_planes(grids, rows, cols))
    off0 = (grids[0] - l0) * 1000.0
    x, y = gio.read_psf_table(tmp_path / "crisp.psf")
    psf = G.psf_from_table(x, y, off0, (grids[0][1] - grids[0][0]) * 1000.0)
    t = H.truth_models(P, rng)
    obs = np.stack([O.synth_f(O.make_cfg(grids[p], l0, zo, psf=psf), t[p]) for p in range(P)])
    obs = np.ascontiguousarray(obs + rng.normal(0, 1e-3, obs.shape), dtype=np.float32)
    cube_file(tmp_path / "cube.fits", obs, rows, cols, ("lam", "stokes", "row", "col"))
    run_cli(tmp_path)
    planes, _ = gio.read_image(tmp_path / "cube_mod.fits")
    cfg = G.make_config(grids[0], l0, G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0), psf=psf,
                        init=H.GUESS, miter=30, lambda_map=grids)
    one = G.make_config(grids[0], l0, G.zeeman_from_levels(2, 1, 1.0, 2, 2, 0.0, 1.0), psf=psf,
                        init=H.GUESS, miter=30)
    with G.Engine(0) as e:
        e.configure(cfg)
        out = e.invert(obs)
        e.configure(one)
        single = e.invert(obs)
    for rr in range(rows):
        for cc in range(cols):
            p = cc * rows + rr
            np.testing.assert_allclose(planes[:11, cc, rr], out["model"][p], rtol=1e-6)
            assert planes[11, cc, rr] == out["iters"][p]
    # the map is applied per pixel: pixel 0, whose grid is the single grid,
    # comes out bit-identical to a single-grid run; every other pixel differs
    np.testing.assert_array_equal(out["model64"][0], single["model64"][0])
    assert (np.abs(out["model64"][1:] - single["model64"][1:]).max(axis=1) > 0).all()
