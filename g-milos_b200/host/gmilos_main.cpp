// gmilos_main.cpp -- the command-line front end: `gmilos <control.mtrol>`,
// a drop-in for the reference's gmilos (gmilos.cu:86-1341) on top of the
// engine's C ABI (include/gmilos.h) and the format library
// (include/gmilos_io.h).
//
// Modes (Number of cycles in the control file):
//   < 0  classical estimates only     -> <base>_model_ce.mod / .fits
//   = 0  synthesis of the guess model -> <base>.per
//   > 0  Levenberg-Marquardt inversion -> <base>_model.mod + <base>_stokes.per
//                                         (.per input), or <base>_mod.fits +
//                                         <base>_stokes.fits (.fits input)
// <base> is the observed-profile file's path without its extension (the
// guess model's when no observed file is named).
//
// Options: --numerics reference|accurate (default reference), --device N
// (overrides the control file), --quiet.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "gmilos.h"
#include "gmilos_io.h"

namespace {

bool g_quiet = false;

void note(const char* fmt, const std::string& a = "", double b = 0) {
  if (!g_quiet) {
    std::printf(fmt, a.c_str(), b);
    std::fflush(stdout);
  }
}

int die(const std::string& msg) {
  std::fprintf(stderr, "gmilos: %s\n", msg.c_str());
  return 1;
}

std::string base_name(const std::string& p) {
  const size_t slash = p.rfind('/');
  const size_t dot = p.rfind('.');
  if (dot == std::string::npos || (slash != std::string::npos && dot < slash)) return p;
  return p.substr(0, dot);
}

std::string ext(const std::string& p) {
  const size_t dot = p.rfind('.');
  return dot == std::string::npos ? "" : p.substr(dot);
}

bool exists(const std::string& p) {
  if (p.empty()) return false;
  FILE* f = std::fopen(p.c_str(), "rb");
  if (!f) return false;
  std::fclose(f);
  return true;
}

struct Cleanup {
  gm_ctx* ctx = nullptr;
  gm_fits_cube* cube = nullptr;
  float* stray = nullptr;
  double* lambda_map = nullptr;
  ~Cleanup() {
    if (ctx) gm_destroy(ctx);
    if (cube) gm_fits_cube_free(cube);
    if (stray) gm_io_free(stray);
    if (lambda_map) gm_io_free(lambda_map);
  }
};

}  // namespace

int main(int argc, char** argv) {
  std::string trol_path;
  int numerics = GM_NUMERICS_REFERENCE, device = -1;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--numerics" && i + 1 < argc) {
      const std::string v = argv[++i];
      if (v == "reference") numerics = GM_NUMERICS_REFERENCE;
      else if (v == "accurate") numerics = GM_NUMERICS_ACCURATE;
      else return die("--numerics takes reference or accurate");
    } else if (a == "--device" && i + 1 < argc) {
      device = std::atoi(argv[++i]);
    } else if (a == "--quiet") {
      g_quiet = true;
    } else if (a[0] != '-' && trol_path.empty()) {
      trol_path = a;
    } else {
      return die("usage: gmilos <control.mtrol> [--numerics reference|accurate] [--device N] [--quiet]");
    }
  }
  if (trol_path.empty())
    return die("usage: gmilos <control.mtrol> [--numerics reference|accurate] [--device N] [--quiet]");

  gm_trol t;
  if (gm_io_read_trol(trol_path.c_str(), &t) != GM_OK) return die(gm_io_last_error());
  if (device < 0) device = t.device;

  gm_config cfg;
  gm_config_defaults(&cfg);
  if (t.init_model[0] && gm_io_read_model(t.init_model, cfg.init_model) != GM_OK)
    return die(gm_io_last_error());
  // stray light only with a filling factor below 1 (gmilos.cu:163-167)
  if (cfg.init_model[GM_NPAR - 1] < 1 && !exists(t.stray))
    return die("filling factor below 1 in the guess model and no stray-light file");

  // ---- wavelengths and the line
  double lambda[GM_MAX_NL], offsets[GM_MAX_NL], quantum[6], lambda0 = 0, step_mA = 0;
  int nl = 0, line_index = 0, lam_rows = 1, lam_cols = 1;
  Cleanup res;
  if (t.use_grid) {
    double first, last;
    if (gm_io_read_grid(t.grid, &line_index, &first, &step_mA, &last) != GM_OK) return die(gm_io_last_error());
    if (gm_io_read_line(t.lines, line_index, &lambda0, quantum) != GM_OK) return die(gm_io_last_error());
    nl = gm_io_grid_wavelengths(lambda0, first, step_mA, last, offsets, lambda, GM_MAX_NL);
    if (nl < 2) return die("the grid must have 2.." + std::to_string(GM_MAX_NL) + " samples");
  } else {
    // one grid (2-D FITS) or per-pixel grids (rows x cols x (1 + nl)); with
    // per-pixel grids the first pixel's grid sets the PSF and the offsets
    // written with .per outputs
    double* grids = nullptr;
    int per_pixel = 0;
    if (gm_fits_read_lambda_map(t.wavelength, &grids, &per_pixel, &lam_rows, &lam_cols, &nl, &line_index) != GM_OK)
      return die(gm_io_last_error());
    res.lambda_map = grids;
    if (nl < 2 || nl > GM_MAX_NL) return die("the wavelength file must have 2.." + std::to_string(GM_MAX_NL) + " samples");
    for (int i = 0; i < nl; ++i) lambda[i] = grids[i];
    if (per_pixel) {
      cfg.lambda_per_pixel = 1;
      cfg.lambda_map = grids;
    }
    if (gm_io_read_line(t.lines, line_index, &lambda0, quantum) != GM_OK) return die(gm_io_last_error());
    for (int i = 0; i < nl; ++i) offsets[i] = (lambda[i] - lambda0) * 1000.0;
    step_mA = (lambda[1] - lambda[0]) * 1000.0;
  }
  cfg.nl = nl;
  cfg.lambda0 = lambda0;
  for (int i = 0; i < nl; ++i) cfg.lambda[i] = lambda[i];
  if (gm_zeeman_from_levels(quantum[0], quantum[1], quantum[2], quantum[3], quantum[4], quantum[5], 1.0,
                            &cfg.zeeman) != GM_OK)
    return die("cannot build the Zeeman pattern of line " + std::to_string(line_index));

  // ---- PSF: a Gaussian of the given FWHM or a table (gmilos.cu:241-300)
  cfg.use_psf = t.use_psf;
  if (t.use_psf) {
    if (t.fwhm_mA > 0) {
      if (gm_psf_gaussian(t.fwhm_mA, lambda, nl, cfg.psf) != GM_OK) return die("Gaussian PSF failed");
    } else {
      std::vector<double> x(200000), y(200000);
      int n = 0;
      if (gm_io_read_psf_table(t.psf, x.data(), y.data(), (int)x.size(), &n) != GM_OK)
        return die(gm_io_last_error());
      if (std::trunc(offsets[0]) < std::trunc(x[0]) || std::trunc(offsets[nl - 1]) > std::trunc(x[n - 1]))
        return die("the PSF table covers less than the wavelength grid");
      if (gm_psf_from_table(x.data(), y.data(), n, offsets, nl, step_mA, cfg.psf) != GM_OK)
        return die("PSF interpolation failed");
    }
  }

  cfg.mu = t.mu;
  for (int s = 0; s < 4; ++s) cfg.weight[s] = t.weight[s];
  cfg.noise = (float)t.noise;
  for (int i = 0; i < GM_NPAR; ++i) cfg.fix[i] = t.fix[i];
  cfg.ilambda = t.ilambda;
  cfg.logclambda = t.logclambda;
  cfg.miter = t.ncycles > 0 ? t.ncycles : 1;
  cfg.init_mode = GM_INIT_CLASSICAL;
  cfg.numerics = numerics;

  // ---- stray light: one profile (.per or 2-D FITS) or a map (4-D FITS)
  int stray_rows = 0, stray_cols = 0;
  if (exists(t.stray)) {
    if (ext(t.stray) == ".per") {
      res.stray = (float*)std::malloc(sizeof(float) * 4 * nl);
      std::vector<double> so(nl);
      if (gm_io_read_per(t.stray, nl, res.stray, so.data()) != GM_OK) return die(gm_io_last_error());
      for (int i = 0; i < nl; ++i)   // offsets must match the grid (utilsFits.c:1557-1560)
        if (so[i] != std::trunc(offsets[i])) return die("stray-light offsets differ from the grid");
      cfg.slight_per_pixel = 0;
    } else {
      int per_pixel = 0;
      if (gm_fits_read_stray(t.stray, nl, &res.stray, &per_pixel, &stray_rows, &stray_cols) != GM_OK)
        return die(gm_io_last_error());
      cfg.slight_per_pixel = per_pixel;
    }
    cfg.use_slight = 1;
    cfg.slight = res.stray;
  }

  if (gm_create(device, 0, &res.ctx) != GM_OK) return die("no CUDA device / engine context");
  if (gm_configure(res.ctx, &cfg) != GM_OK) return die(gm_last_error(res.ctx));

  const std::string base = base_name(t.observed[0] ? t.observed : t.init_model);
  const std::string obs = t.observed;
  const bool per_input = ext(obs) == ".per";
  const bool fits_input = ext(obs) == ".fits";

  // ---- synthesis
  if (t.ncycles == 0) {
    if (cfg.slight_per_pixel) return die("synthesis takes one stray-light profile, not a map");
    if (cfg.lambda_per_pixel) return die("synthesis takes one wavelength grid, not per-pixel grids");
    std::vector<float> spec(4 * nl);
    if (gm_synthesize_f64(res.ctx, cfg.init_model, 1, spec.data(), nullptr, nullptr) != GM_OK)
      return die(gm_last_error(res.ctx));
    const std::string out = base + ".per";
    if (gm_io_write_per(out.c_str(), line_index, nl, offsets, spec.data()) != GM_OK) return die(gm_io_last_error());
    note("SYNTHESIS DONE: %s\n", out);
    return 0;
  }

  // ---- observed profiles
  std::vector<float> one;
  const float* iquv = nullptr;
  int64_t P = 0;
  int rows = 1, cols = 1;
  if (per_input) {
    one.resize(4 * nl);
    if (gm_io_read_per(obs.c_str(), nl, one.data(), nullptr) != GM_OK) return die(gm_io_last_error());
    iquv = one.data();
    P = 1;
  } else if (fits_input) {
    if (gm_fits_read_cube(obs.c_str(), nl, &res.cube) != GM_OK) return die(gm_io_last_error());
    gm_fits_cube_dims(res.cube, &rows, &cols, nullptr);
    iquv = gm_fits_cube_data(res.cube);
    P = (int64_t)rows * cols;
  } else {
    return die("observed profiles must be a .per or .fits file");
  }
  if (cfg.slight_per_pixel && (stray_rows != rows || stray_cols != cols))
    return die("the stray-light map's dimensions differ from the observed cube's");
  if (cfg.lambda_per_pixel && (!fits_input || lam_rows != rows || lam_cols != cols))
    return die("per-pixel wavelength grids need a FITS cube of the same rows and columns");
  if (cfg.slight_per_pixel) {
    // the per-pixel map travels with the call (gm_invert_ex reads cfg.slight)
  }

  std::vector<double> models((size_t)P * GM_NPAR);
  std::vector<float> chi2((size_t)P, 0.f);
  std::vector<int> iters((size_t)P, 0);

  if (t.ncycles < 0) {
    if (gm_classical(res.ctx, iquv, P, nl, models.data(), nullptr) != GM_OK) return die(gm_last_error(res.ctx));
    if (per_input) {
      const std::string out = base + "_model_ce.mod";
      if (gm_io_write_model(out.c_str(), models.data(), 0, 0.f) != GM_OK) return die(gm_io_last_error());
      note("CLASSICAL ESTIMATES: %s\n", out);
    } else {
      const std::string out = base + "_model_ce.fits";
      if (gm_fits_write_models(out.c_str(), rows, cols, models.data(), iters.data(), chi2.data(), 1) != GM_OK)
        return die(gm_io_last_error());
      note("CLASSICAL ESTIMATES: %s\n", out);
    }
    return 0;
  }

  std::vector<float> fitted((size_t)P * 4 * nl);
  const auto t0 = std::chrono::steady_clock::now();
  if (gm_invert_ex(res.ctx, iquv, P, nl, nullptr, nullptr, models.data(), chi2.data(), iters.data(), nullptr,
                   fitted.data(), nullptr, nullptr) != GM_OK)
    return die(gm_last_error(res.ctx));
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  note("FINISH EXECUTION OF INVERSION: %s%f seconds\n", "", secs);

  if (per_input) {
    const std::string m = base + "_model.mod", s = base + "_stokes.per";
    if (gm_io_write_model(m.c_str(), models.data(), iters[0], chi2[0]) != GM_OK) return die(gm_io_last_error());
    if (gm_io_write_per(s.c_str(), line_index, nl, offsets, fitted.data()) != GM_OK) return die(gm_io_last_error());
    note("INVERTED MODEL SAVED IN FILE: %s\n", m);
  } else {
    const std::string m = base + "_mod.fits", s = base + "_stokes.fits";
    if (gm_fits_write_models(m.c_str(), rows, cols, models.data(), iters.data(), chi2.data(), 1) != GM_OK)
      return die(gm_io_last_error());
    if (gm_fits_write_profiles(s.c_str(), res.cube, fitted.data()) != GM_OK) return die(gm_io_last_error());
    note("INVERTED MODELS SAVED IN FILE: %s\n", m);
  }
  return 0;
}
