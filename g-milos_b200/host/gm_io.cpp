// gm_io.cpp -- the reference's file formats (include/gmilos_io.h): control
// file, models, grids, line list, PSF tables, .per profiles and a small
// single-HDU FITS reader/writer of this project's own.
#include "gmilos_io.h"

#include <sys/stat.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

gm_status io_fail(gm_status s, const std::string& msg) {
  g_err = msg;
  return s;
}

bool file_exists(const std::string& p) {
  struct stat st;
  return !p.empty() && stat(p.c_str(), &st) == 0 && S_ISREG(st.st_mode);
}

// extension including the dot, or "" (file_ext, readConfig.c:2312-2326:
// the extension must be alphanumeric)
std::string extension(const std::string& p) {
  const size_t d = p.rfind('.');
  if (d == std::string::npos) return "";
  for (size_t i = d + 1; i < p.size(); ++i)
    if (!std::isalnum((unsigned char)p[i])) return "";
  return p.substr(d);
}

void copy_str(char* dst, const std::string& s) {
  std::strncpy(dst, s.c_str(), GM_IO_PATH - 1);
  dst[GM_IO_PATH - 1] = '\0';
}

bool read_lines(const char* path, std::vector<std::string>* out) {
  std::ifstream f(path);
  if (!f) return false;
  std::string line;
  while (std::getline(f, line)) out->push_back(line);
  return true;
}

// The value of a "name : value ! comment" line: the first whitespace-
// delimited token after the first ':'; a token that opens the comment is
// an empty value.
std::string trol_value(const std::string& line) {
  const size_t c = line.find(':');
  if (c == std::string::npos) return "";
  size_t i = c + 1;
  while (i < line.size() && std::isspace((unsigned char)line[i])) ++i;
  size_t j = i;
  while (j < line.size() && !std::isspace((unsigned char)line[j])) ++j;
  std::string tok = line.substr(i, j - i);
  if (!tok.empty() && tok[0] == '!') return "";
  return tok;
}

bool parse_int(const std::string& tok, int* v) {
  if (tok.empty()) return false;
  char* end = nullptr;
  errno = 0;
  const long x = std::strtol(tok.c_str(), &end, 0);   // like %i: decimal, 0x.., 0..
  if (end == tok.c_str()) return false;
  *v = (int)x;
  return true;
}

bool parse_float(const std::string& tok, float* v) {
  if (tok.empty()) return false;
  char* end = nullptr;
  const float x = std::strtof(tok.c_str(), &end);
  if (end == tok.c_str()) return false;
  *v = x;
  return true;
}

// ---------------------------------------------------------------- FITS
constexpr int kBlock = 2880;
constexpr int kCard = 80;

struct Card {
  std::string key, raw;
};

struct FitsImage {
  int bitpix = 0;
  std::vector<int64_t> naxes;
  std::vector<Card> cards;      // every card before END
  double bscale = 1.0, bzero = 0.0;
  std::vector<double> data;     // physical values, file order
};

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

// value field of a card: a quoted string (with '' for a quote) or the text
// before a '/' comment
std::string card_value(const std::string& raw) {
  if (raw.size() < 10 || raw[8] != '=') return "";
  std::string v = raw.substr(10);
  size_t i = 0;
  while (i < v.size() && v[i] == ' ') ++i;
  if (i < v.size() && v[i] == '\'') {
    std::string out;
    for (size_t k = i + 1; k < v.size(); ++k) {
      if (v[k] == '\'') {
        if (k + 1 < v.size() && v[k + 1] == '\'') {
          out += '\'';
          ++k;
        } else {
          break;
        }
      } else {
        out += v[k];
      }
    }
    // trailing blanks of a FITS string are not significant
    while (!out.empty() && out.back() == ' ') out.pop_back();
    return out;
  }
  const size_t slash = v.find('/');
  return trim(slash == std::string::npos ? v : v.substr(0, slash));
}

uint64_t be_read(const unsigned char* p, int n) {
  uint64_t v = 0;
  for (int i = 0; i < n; ++i) v = (v << 8) | p[i];
  return v;
}

gm_status fits_read(const char* path, FitsImage* img) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return io_fail(GM_ERR_IO, std::string("cannot open ") + path);
  std::vector<char> block(kBlock);
  bool end = false;
  int nblocks = 0;
  while (!end) {
    if (!f.read(block.data(), kBlock)) return io_fail(GM_ERR_IO, std::string("truncated FITS header: ") + path);
    ++nblocks;
    for (int c = 0; c < kBlock / kCard; ++c) {
      std::string raw(block.data() + c * kCard, kCard);
      std::string key = trim(raw.substr(0, 8));
      if (key == "END") {
        end = true;
        break;
      }
      img->cards.push_back({key, raw});
    }
    if (nblocks > 10000) return io_fail(GM_ERR_IO, "FITS header without END");
  }
  auto find = [&](const std::string& k, std::string* v) {
    for (const Card& c : img->cards)
      if (c.key == k) {
        *v = card_value(c.raw);
        return true;
      }
    return false;
  };
  std::string v;
  if (!find("SIMPLE", &v) || v != "T") return io_fail(GM_ERR_IO, std::string("not a FITS primary HDU: ") + path);
  if (!find("BITPIX", &v)) return io_fail(GM_ERR_IO, "FITS without BITPIX");
  img->bitpix = std::atoi(v.c_str());
  if (!find("NAXIS", &v)) return io_fail(GM_ERR_IO, "FITS without NAXIS");
  const int naxis = std::atoi(v.c_str());
  if (naxis < 1 || naxis > 8) return io_fail(GM_ERR_IO, "unsupported NAXIS");
  int64_t n = 1;
  for (int a = 1; a <= naxis; ++a) {
    if (!find("NAXIS" + std::to_string(a), &v)) return io_fail(GM_ERR_IO, "FITS without NAXISn");
    const int64_t len = std::atoll(v.c_str());
    if (len < 1) return io_fail(GM_ERR_IO, "empty FITS axis");
    img->naxes.push_back(len);
    n *= len;
  }
  if (find("BSCALE", &v)) img->bscale = std::atof(v.c_str());
  if (find("BZERO", &v)) img->bzero = std::atof(v.c_str());
  const int bytes = std::abs(img->bitpix) / 8;
  if (!(img->bitpix == -32 || img->bitpix == -64 || img->bitpix == 8 || img->bitpix == 16 ||
        img->bitpix == 32 || img->bitpix == 64))
    return io_fail(GM_ERR_IO, "unsupported BITPIX");
  std::vector<unsigned char> raw((size_t)n * bytes);
  if (!f.read((char*)raw.data(), (std::streamsize)raw.size()))
    return io_fail(GM_ERR_IO, std::string("truncated FITS data: ") + path);
  img->data.resize((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    const uint64_t u = be_read(raw.data() + (size_t)i * bytes, bytes);
    double x;
    switch (img->bitpix) {
      case -32: {
        uint32_t w = (uint32_t)u;
        float fv;
        std::memcpy(&fv, &w, 4);
        x = fv;
        break;
      }
      case -64: {
        double dv;
        std::memcpy(&dv, &u, 8);
        x = dv;
        break;
      }
      case 8: x = (double)(uint8_t)u; break;
      case 16: x = (double)(int16_t)(uint16_t)u; break;
      case 32: x = (double)(int32_t)(uint32_t)u; break;
      default: x = (double)(int64_t)u; break;
    }
    img->data[(size_t)i] = img->bzero + img->bscale * x;
  }
  return GM_OK;
}

std::string fixed_card(const std::string& key, const std::string& value, const std::string& comment = "") {
  char buf[kCard + 1];
  std::snprintf(buf, sizeof(buf), "%-8.8s= %20s%s%s", key.c_str(), value.c_str(),
                comment.empty() ? "" : " / ", comment.c_str());
  std::string s(buf);
  s.resize(kCard, ' ');
  return s;
}

bool structural(const std::string& key) {
  if (key == "SIMPLE" || key == "BITPIX" || key == "NAXIS" || key == "EXTEND" || key == "BSCALE" ||
      key == "BZERO" || key == "END")
    return true;
  return key.size() > 5 && key.compare(0, 5, "NAXIS") == 0 &&
         std::all_of(key.begin() + 5, key.end(), [](char ch) { return std::isdigit((unsigned char)ch); });
}

gm_status fits_write(const char* path, const std::vector<int64_t>& naxes, const float* data,
                     const std::vector<std::string>& extra_cards) {
  std::vector<std::string> cards;
  cards.push_back(fixed_card("SIMPLE", "T", "conforms to the FITS standard"));
  cards.push_back(fixed_card("BITPIX", "-32", "IEEE single precision"));
  cards.push_back(fixed_card("NAXIS", std::to_string(naxes.size())));
  for (size_t a = 0; a < naxes.size(); ++a)
    cards.push_back(fixed_card("NAXIS" + std::to_string(a + 1), std::to_string(naxes[a])));
  for (const std::string& c : extra_cards) {
    std::string s = c;
    s.resize(kCard, ' ');
    cards.push_back(s);
  }
  std::string end = "END";
  end.resize(kCard, ' ');
  cards.push_back(end);
  std::string header;
  for (const std::string& c : cards) header += c;
  header.resize(((header.size() + kBlock - 1) / kBlock) * kBlock, ' ');
  int64_t n = 1;
  for (int64_t a : naxes) n *= a;
  std::vector<unsigned char> body((size_t)n * 4);
  for (int64_t i = 0; i < n; ++i) {
    uint32_t w;
    std::memcpy(&w, data + i, 4);
    for (int b = 0; b < 4; ++b) body[(size_t)i * 4 + b] = (unsigned char)(w >> (24 - 8 * b));
  }
  body.resize(((body.size() + kBlock - 1) / kBlock) * kBlock, 0);
  std::remove(path);
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  if (!f) return io_fail(GM_ERR_IO, std::string("cannot create ") + path);
  f.write(header.data(), (std::streamsize)header.size());
  f.write((const char*)body.data(), (std::streamsize)body.size());
  if (!f) return io_fail(GM_ERR_IO, std::string("write failed: ") + path);
  return GM_OK;
}

// axis roles of a 4-D Stokes cube (readFitsSpectroImage, utilsFits.c:267-370)
struct Axes {
  int row = -1, col = -1, lambda = -1, stokes = -1;
};

gm_status infer_axes(const FitsImage& img, Axes* ax) {
  if (img.naxes.size() != 4) return io_fail(GM_ERR_IO, "a Stokes cube needs NAXIS = 4");
  std::string ct[4];
  bool all = true;
  for (int a = 0; a < 4; ++a) {
    bool found = false;
    for (const Card& c : img.cards)
      if (c.key == "CTYPE" + std::to_string(a + 1)) {
        ct[a] = card_value(c.raw);
        found = true;
      }
    all = all && found;
  }
  if (all) {
    for (int a = 0; a < 4; ++a) {
      if (ct[a] == "WAVE-GRI") ax->lambda = a;
      else if (ct[a] == "HPLN-TAN") ax->row = a;
      else if (ct[a] == "HPLT-TAN") ax->col = a;
      else if (ct[a] == "STOKES") ax->stokes = a;
    }
    if (ax->row < 0 || ax->col < 0 || ax->lambda < 0 || ax->stokes < 0)
      return io_fail(GM_ERR_IO, "CTYPE1..4 must name WAVE-GRI, STOKES, HPLN-TAN and HPLT-TAN");
    return GM_OK;
  }
  // without the keywords: Stokes is the shortest axis, wavelength the next
  // shortest, the two remaining axes rows then columns
  int64_t best = INT64_MAX;
  for (int a = 0; a < 4; ++a)
    if (img.naxes[a] < best) {
      best = img.naxes[a];
      ax->stokes = a;
    }
  best = INT64_MAX;
  for (int a = 0; a < 4; ++a)
    if (a != ax->stokes && img.naxes[a] < best) {
      best = img.naxes[a];
      ax->lambda = a;
    }
  for (int a = 0; a < 4; ++a) {
    if (a == ax->stokes || a == ax->lambda) continue;
    if (ax->row < 0) ax->row = a;
    else ax->col = a;
  }
  return GM_OK;
}

}  // namespace

struct gm_fits_cube {
  int rows = 0, cols = 0, nl = 0;
  Axes ax;
  std::vector<int64_t> naxes;
  std::vector<std::string> cards;   // non-structural header cards of the input
  std::vector<float> pix;           // [rows*cols][4][nl]
};

extern "C" {

const char* gm_io_last_error(void) { return g_err.c_str(); }

void gm_io_free(void* p) { std::free(p); }

void gm_io_trol_defaults(gm_trol* t) {
  std::memset(t, 0, sizeof(*t));
  for (int s = 0; s < 4; ++s) t->weight[s] = 1.f;
  t->noise = 1e-3 * 1e-3;      // NOISE_SIGMA^2
  t->ilambda = 0.1f;
  t->mu = 1.f;
  t->nstreams = 2;
  t->device = 0;
}

gm_status gm_io_read_trol(const char* path, gm_trol* t) {
  gm_io_trol_defaults(t);
  std::vector<std::string> L;
  if (!read_lines(path, &L)) return io_fail(GM_ERR_IO, std::string("cannot open control file ") + path);
  if (L.size() < 44) return io_fail(GM_ERR_IO, "control file has fewer than 44 lines");
  auto v = [&](int i) { return trol_value(L[i]); };
  if (!parse_int(v(0), &t->ncycles)) return io_fail(GM_ERR_IO, "Number of cycles is not an integer");
  copy_str(t->observed, v(1));
  copy_str(t->stray, v(2));
  copy_str(t->psf, v(3));
  // PSF: a .psf file, else a number = FWHM [mA] (0 or none: no PSF)
  // (readConfig.c:1485-1510)
  const std::string psf = v(3);
  if (!file_exists(psf)) {
    const double fwhm = std::atof(psf.c_str());
    t->use_psf = fwhm != 0 ? 1 : 0;
    t->fwhm_mA = fwhm != 0 ? fwhm : -1;
  } else {
    if (extension(psf) != ".psf") return io_fail(GM_ERR_IO, "the PSF file's extension is not .psf: " + psf);
    t->use_psf = 1;
    t->fwhm_mA = 0;
  }
  const std::string wl = v(4);
  if (file_exists(wl)) {
    if (extension(wl) == ".grid") {
      copy_str(t->grid, wl);
      t->use_grid = 1;
    } else if (extension(wl) == ".fits") {
      copy_str(t->wavelength, wl);
      t->use_grid = 0;
    } else {
      return io_fail(GM_ERR_IO, "the wavelength file must be .grid or .fits: " + wl);
    }
  } else {
    copy_str(t->wavelength, wl);
  }
  copy_str(t->lines, v(5));
  copy_str(t->abundances, v(6));
  copy_str(t->init_model, v(7));
  copy_str(t->init_model2, v(8));
  for (int s = 0; s < 4; ++s) parse_float(v(9 + s), &t->weight[s]);
  parse_int(v(13), &t->auto_nodes);
  // free flags, in the control file's order
  static const int order[10] = {7, 8, 0, 1, 2, 5, 6, 3, 4, 9};
  for (int k = 0; k < 10; ++k) parse_int(v(14 + k), &t->fix[order[k]]);
  for (int k = 0; k < 10; ++k) parse_int(v(24 + k), &t->fix2[order[k]]);
  parse_int(v(34), &t->invert_filling_factor);
  parse_int(v(35), &t->fix[10]);
  parse_float(v(36), &t->mu);
  if (parse_int(v(37), &t->sn_i) && t->sn_i != 0) {
    const double n = 1.0 / t->sn_i;
    t->noise = n * n;
  }
  parse_int(v(38), &t->continuum_contrast);
  parse_float(v(39), &t->ilambda);
  parse_int(v(40), &t->use_fft);
  parse_int(v(41), &t->logclambda);
  parse_int(v(42), &t->nstreams);
  parse_int(v(43), &t->device);
  return GM_OK;
}

gm_status gm_io_read_model(const char* path, double model[GM_NPAR]) {
  std::vector<std::string> L;
  if (!read_lines(path, &L)) return io_fail(GM_ERR_IO, std::string("cannot open model file ") + path);
  static const struct {
    const char* key;
    int idx;
  } keys[] = {{"magnetic field", 1}, {"gamma", 5},  {"phi", 6},     {"eta_0", 0},
              {"Doppler width", 3},  {"damping", 4}, {"filling factor", 10}, {"v_mac", 9},
              {"LOS velocity", 2},   {"S_0", 7},     {"S_1", 8}};
  for (const std::string& line : L) {
    const size_t c = line.find(':');
    if (c == std::string::npos) continue;
    const std::string name = line.substr(0, c);
    char* end = nullptr;
    const double x = std::strtod(line.c_str() + c + 1, &end);
    if (end == line.c_str() + c + 1) continue;
    for (const auto& k : keys)
      if (name.find(k.key) != std::string::npos) model[k.idx] = x;
  }
  return GM_OK;
}

gm_status gm_io_write_model(const char* path, const double m[GM_NPAR], int iters, float chi2) {
  FILE* f = std::fopen(path, "w");
  if (!f) return io_fail(GM_ERR_IO, std::string("cannot create ") + path);
  std::fprintf(f, "eta_0               :%lf\n", m[0]);
  std::fprintf(f, "magnetic field [G]  :%lf\n", m[1]);
  std::fprintf(f, "LOS velocity[km/s]  :%lf\n", m[2]);
  std::fprintf(f, "Doppler width [A]   :%lf\n", m[3]);
  std::fprintf(f, "damping             :%lf\n", m[4]);
  std::fprintf(f, "gamma [deg]         :%lf\n", m[5]);
  std::fprintf(f, "phi  [deg]          :%lf\n", m[6]);
  std::fprintf(f, "S_0                 :%lf\n", m[7]);
  std::fprintf(f, "S_1                 :%lf\n", m[8]);
  std::fprintf(f, "v_mac [km/s]        :%lf\n", m[9]);
  std::fprintf(f, "filling factor      :%lf\n", m[10]);
  std::fprintf(f, "# Iterations        :%d\n", iters);
  std::fprintf(f, "chisqr              :%le\n", (double)chi2);
  std::fprintf(f, "\n\n");
  std::fclose(f);
  return GM_OK;
}

gm_status gm_io_read_grid(const char* path, int* line_index, double* first_mA, double* step_mA,
                          double* last_mA) {
  std::vector<std::string> L;
  if (!read_lines(path, &L)) return io_fail(GM_ERR_IO, std::string("cannot open grid file ") + path);
  for (size_t i = 0; i + 1 < L.size(); ++i) {
    if (L[i].compare(0, 6, "------") != 0) continue;
    const std::string& d = L[i + 1];
    const size_t c = d.find(':');
    if (c == std::string::npos) break;
    char* end = nullptr;
    const long idx = std::strtol(d.c_str(), &end, 10);
    if (end == d.c_str()) break;
    double v[3];
    const char* p = d.c_str() + c + 1;
    for (int k = 0; k < 3; ++k) {
      v[k] = std::strtod(p, &end);
      if (end == p) return io_fail(GM_ERR_IO, "grid line needs initial, step, final");
      p = end;
      while (*p == ' ' || *p == '\t') ++p;
      if (k < 2) {
        if (*p != ',') return io_fail(GM_ERR_IO, "grid values must be separated by commas");
        ++p;
      }
    }
    *line_index = (int)idx;
    *first_mA = v[0];
    *step_mA = v[1];
    *last_mA = v[2];
    return GM_OK;
  }
  return io_fail(GM_ERR_IO, "no grid line after a ------ header line");
}

int gm_io_grid_wavelengths(double lambda0, double first_mA, double step_mA, double last_mA,
                           double* offsets_mA, double* lambda, int cap) {
  if (step_mA == 0) return 0;
  const int n = (int)(((last_mA - first_mA) / step_mA) + 1);
  if (n < 1 || n > cap) return 0;
  double off = first_mA, lam = lambda0 + first_mA / 1000.0;
  for (int i = 0; i < n; ++i) {
    if (i > 0) {
      off += step_mA;
      lam += step_mA / 1000.0;
    }
    if (offsets_mA) offsets_mA[i] = off;
    if (lambda) lambda[i] = lam;
  }
  return n;
}

gm_status gm_io_read_line(const char* path, int line_index, double* lambda0, double quantum[6]) {
  std::vector<std::string> L;
  if (!read_lines(path, &L)) return io_fail(GM_ERR_IO, std::string("cannot open line list ") + path);
  auto orbital = [](char ch, double* l) {
    static const char letters[] = "SPDFGHJ";
    const char* p = std::strchr(letters, ch);
    if (!p || !ch) return false;
    *l = (double)(p - letters);
    return true;
  };
  for (const std::string& line : L) {
    const size_t eq = line.find('=');
    if (eq == std::string::npos) continue;
    char* end = nullptr;
    const long idx = std::strtol(line.c_str(), &end, 10);
    if (end == line.c_str() || idx != line_index) continue;
    std::istringstream ss(line.substr(eq + 1));
    std::vector<std::string> tok;
    std::string t;
    while (ss >> t) tok.push_back(t);
    // element, ionisation, centre, then the term of each level: "5P 1.0- 5D 0.0"
    if (tok.size() < 3) return io_fail(GM_ERR_IO, "short line-list entry");
    *lambda0 = std::atof(tok[2].c_str());
    for (size_t k = 1; k + 2 < tok.size(); ++k) {
      if (tok[k].empty() || tok[k].back() != '-') continue;
      const std::string lo = tok[k - 1], up = tok[k + 1];
      const std::string jlo = tok[k].substr(0, tok[k].size() - 1), jup = tok[k + 2];
      if (lo.size() < 2 || up.size() < 2) break;
      // S = (multiplicity - 1) / 2 in integer arithmetic, as the reference
      // stores it (readConfig.c:478-479)
      const int mlo = std::atoi(lo.substr(0, lo.size() - 1).c_str());
      const int mup = std::atoi(up.substr(0, up.size() - 1).c_str());
      double llo, lup;
      if (!orbital(lo.back(), &llo) || !orbital(up.back(), &lup))
        return io_fail(GM_ERR_IO, "unknown orbital letter in line " + std::to_string(line_index));
      quantum[0] = (double)((mlo - 1) / 2);
      quantum[1] = llo;
      quantum[2] = std::atof(jlo.c_str());
      quantum[3] = (double)((mup - 1) / 2);
      quantum[4] = lup;
      quantum[5] = std::atof(jup.c_str());
      return GM_OK;
    }
    return io_fail(GM_ERR_IO, "no level terms in line " + std::to_string(line_index));
  }
  return io_fail(GM_ERR_IO, "line " + std::to_string(line_index) + " not in the line list");
}

gm_status gm_io_read_psf_table(const char* path, double* x_mA, double* y, int cap, int* n) {
  std::vector<std::string> L;
  if (!read_lines(path, &L)) return io_fail(GM_ERR_IO, std::string("cannot open PSF file ") + path);
  int k = 0;
  for (const std::string& line : L) {
    char* end = nullptr;
    const double a = std::strtod(line.c_str(), &end);
    if (end == line.c_str()) continue;
    const char* p = end;
    const double b = std::strtod(p, &end);
    if (end == p) continue;
    if (k >= cap) return io_fail(GM_ERR_IO, "PSF table longer than the buffer");
    x_mA[k] = a;
    y[k] = b;
    ++k;
  }
  *n = k;
  return k > 1 ? GM_OK : io_fail(GM_ERR_IO, "PSF table is empty");
}

gm_status gm_io_read_per(const char* path, int nl, float* iquv, double* offsets_mA) {
  std::vector<std::string> L;
  if (!read_lines(path, &L)) return io_fail(GM_ERR_IO, std::string("cannot open profile file ") + path);
  int k = 0;
  for (const std::string& line : L) {
    if (k >= nl) break;
    double v[6];
    const char* p = line.c_str();
    int got = 0;
    for (; got < 6; ++got) {
      char* end = nullptr;
      v[got] = std::strtod(p, &end);
      if (end == p) break;
      p = end;
    }
    if (got == 0) continue;
    if (got < 6) return io_fail(GM_ERR_IO, "a profile line needs index, offset, I, Q, U, V");
    if (offsets_mA) offsets_mA[k] = v[1];
    for (int s = 0; s < 4; ++s) iquv[s * nl + k] = (float)v[2 + s];
    ++k;
  }
  if (k != nl)
    return io_fail(GM_ERR_IO, std::string("profile file has fewer samples than the grid: ") + path);
  return GM_OK;
}

gm_status gm_io_write_per(const char* path, int line_index, int nl, const double* offsets_mA,
                          const float* iquv) {
  FILE* f = std::fopen(path, "w");
  if (!f) return io_fail(GM_ERR_IO, std::string("cannot create ") + path);
  for (int k = 0; k < nl; ++k)
    std::fprintf(f, "%d\t%f\t%e\t%e\t%e\t%e\n", line_index, offsets_mA[k], (double)iquv[k],
                 (double)iquv[nl + k], (double)iquv[2 * nl + k], (double)iquv[3 * nl + k]);
  std::fclose(f);
  return GM_OK;
}

// ---------------------------------------------------------------- FITS API
gm_status gm_fits_read_cube(const char* path, int nl_expected, gm_fits_cube** out) {
  FitsImage img;
  gm_status st = fits_read(path, &img);
  if (st != GM_OK) return st;
  Axes ax;
  if ((st = infer_axes(img, &ax)) != GM_OK) return st;
  if (img.naxes[ax.stokes] != 4) return io_fail(GM_ERR_IO, "the Stokes axis must have 4 planes");
  if (nl_expected > 0 && img.naxes[ax.lambda] != nl_expected)
    return io_fail(GM_ERR_IO, "the cube's wavelength axis differs from the grid");
  gm_fits_cube* c = new gm_fits_cube;
  c->ax = ax;
  c->naxes = img.naxes;
  c->rows = (int)img.naxes[ax.row];
  c->cols = (int)img.naxes[ax.col];
  c->nl = (int)img.naxes[ax.lambda];
  for (const Card& cd : img.cards)
    if (!structural(cd.key)) c->cards.push_back(cd.raw);
  const int64_t P = (int64_t)c->rows * c->cols;
  c->pix.assign((size_t)P * 4 * c->nl, 0.f);
  const int64_t* n = img.naxes.data();
  int64_t idx[4];
  size_t e = 0;
  for (idx[3] = 0; idx[3] < n[3]; ++idx[3])
    for (idx[2] = 0; idx[2] < n[2]; ++idx[2])
      for (idx[1] = 0; idx[1] < n[1]; ++idx[1])
        for (idx[0] = 0; idx[0] < n[0]; ++idx[0], ++e) {
          const int64_t p = idx[ax.col] * c->rows + idx[ax.row];
          c->pix[(size_t)(p * 4 + idx[ax.stokes]) * c->nl + idx[ax.lambda]] = (float)img.data[e];
        }
  *out = c;
  return GM_OK;
}

void gm_fits_cube_dims(const gm_fits_cube* c, int* rows, int* cols, int* nl) {
  if (rows) *rows = c->rows;
  if (cols) *cols = c->cols;
  if (nl) *nl = c->nl;
}

float* gm_fits_cube_data(gm_fits_cube* c) { return c->pix.data(); }

void gm_fits_cube_free(gm_fits_cube* c) { delete c; }

gm_status gm_fits_write_profiles(const char* path, const gm_fits_cube* like, const float* iquv) {
  const int64_t* n = like->naxes.data();
  std::vector<float> out((size_t)(n[0] * n[1] * n[2] * n[3]));
  int64_t idx[4];
  size_t e = 0;
  const Axes& ax = like->ax;
  for (idx[3] = 0; idx[3] < n[3]; ++idx[3])
    for (idx[2] = 0; idx[2] < n[2]; ++idx[2])
      for (idx[1] = 0; idx[1] < n[1]; ++idx[1])
        for (idx[0] = 0; idx[0] < n[0]; ++idx[0], ++e) {
          const int64_t p = idx[ax.col] * like->rows + idx[ax.row];
          out[e] = iquv[(size_t)(p * 4 + idx[ax.stokes]) * like->nl + idx[ax.lambda]];
        }
  return fits_write(path, like->naxes, out.data(), like->cards);
}

gm_status gm_fits_write_models(const char* path, int rows, int cols, const double* models,
                               const int* iters, const float* chi2, int with_chi2) {
  if (rows < 1 || cols < 1 || !models) return io_fail(GM_ERR_INVALID, "bad model image");
  const int planes = 12 + (with_chi2 ? 1 : 0);
  const int64_t P = (int64_t)rows * cols;
  std::vector<float> out((size_t)(P * planes));
  for (int k = 0; k < planes; ++k)
    for (int64_t p = 0; p < P; ++p) {
      float v;
      if (k < 11) v = (float)models[p * 11 + k];
      else if (k == 11) v = iters ? (float)iters[p] : 0.f;
      else v = chi2 ? chi2[p] : 0.f;
      out[(size_t)(k * P + p)] = v;
    }
  return fits_write(path, {rows, cols, planes}, out.data(), {});
}

gm_status gm_fits_read_stray(const char* path, int nl, float** out, int* per_pixel, int* rows, int* cols) {
  FitsImage img;
  gm_status st = fits_read(path, &img);
  if (st != GM_OK) return st;
  if (img.naxes.size() == 2) {
    const int64_t a = img.naxes[0], b = img.naxes[1];
    const int64_t nls = a > b ? a : b;
    if (nls != nl || (a > b ? b : a) != 4) return io_fail(GM_ERR_IO, "stray-light profile must be [4][nl]");
    float* s = (float*)std::malloc(sizeof(float) * 4 * nl);
    for (int64_t j = 0; j < b; ++j)
      for (int64_t i = 0; i < a; ++i) {
        const double v = img.data[(size_t)(j * a + i)];
        // wavelength along NAXIS1: file order is already [4][nl]
        if (a == nls) s[j * nl + i] = (float)v;
        else s[i * nl + j] = (float)v;
      }
    *out = s;
    *per_pixel = 0;
    if (rows) *rows = 1;
    if (cols) *cols = 1;
    return GM_OK;
  }
  if (img.naxes.size() == 4) {
    gm_fits_cube* c = nullptr;
    st = gm_fits_read_cube(path, nl, &c);
    if (st != GM_OK) return st;
    float* s = (float*)std::malloc(sizeof(float) * c->pix.size());
    std::memcpy(s, c->pix.data(), sizeof(float) * c->pix.size());
    *out = s;
    *per_pixel = 1;
    if (rows) *rows = c->rows;
    if (cols) *cols = c->cols;
    gm_fits_cube_free(c);
    return GM_OK;
  }
  return io_fail(GM_ERR_IO, "stray-light FITS must have 2 or 4 axes");
}

gm_status gm_fits_read_lambda(const char* path, double* lambda, int cap, int* nl, int* line_index) {
  FitsImage img;
  gm_status st = fits_read(path, &img);
  if (st != GM_OK) return st;
  if (img.naxes.size() != 2 || img.naxes[1] < 2)
    return io_fail(GM_ERR_IO, "wavelength FITS must be 2-D: line index row, wavelength row "
                              "(per-pixel grids: gm_fits_read_lambda_map)");
  const int64_t n = img.naxes[0];
  if (n > cap) return io_fail(GM_ERR_IO, "too many wavelengths");
  *line_index = (int)img.data[(size_t)(n - 1)];
  for (int64_t i = 0; i < n; ++i) lambda[i] = img.data[(size_t)(n + i)];
  *nl = (int)n;
  return GM_OK;
}

gm_status gm_fits_read_lambda_map(const char* path, double** out, int* per_pixel, int* rows, int* cols,
                                  int* nl, int* line_index) {
  *out = nullptr;
  FitsImage img;
  gm_status st = fits_read(path, &img);
  if (st != GM_OK) return st;
  const size_t na = img.naxes.size();
  if (na == 2) {   // one grid: row 1 the line index, row 2 the wavelengths
    const int64_t n = img.naxes[0];
    if (img.naxes[1] < 2 || n < 2) return io_fail(GM_ERR_IO, "wavelength FITS must hold a line index and >= 2 wavelengths");
    double* g = (double*)std::malloc(sizeof(double) * (size_t)n);
    *line_index = (int)img.data[(size_t)(n - 1)];
    for (int64_t i = 0; i < n; ++i) g[i] = img.data[(size_t)(n + i)];
    *out = g;
    *per_pixel = 0;
    *rows = *cols = 1;
    *nl = (int)n;
    return GM_OK;
  }
  // per-pixel grids: NAXIS1 = rows, NAXIS2 = cols, NAXIS3 = 1 + nl (plane 0
  // the line index, planes 1..nl the wavelengths), NAXIS4 = 1 if present
  if ((na != 3 && na != 4) || (na == 4 && img.naxes[3] != 1) || img.naxes[2] < 3)
    return io_fail(GM_ERR_IO, "per-pixel wavelength FITS must be rows x cols x (1 + nl)");
  const int64_t R = img.naxes[0], Cc = img.naxes[1], n = img.naxes[2] - 1, P = R * Cc;
  const int idx = (int)img.data[0];
  for (int64_t p = 0; p < P; ++p)
    if ((int)img.data[(size_t)p] != idx) return io_fail(GM_ERR_IO, "per-pixel wavelength FITS: one line index for all pixels");
  double* m = (double*)std::malloc(sizeof(double) * (size_t)(P * n));
  for (int64_t l = 0; l < n; ++l)
    for (int64_t p = 0; p < P; ++p) m[(size_t)(p * n + l)] = img.data[(size_t)((l + 1) * P + p)];
  *out = m;
  *per_pixel = 1;
  *rows = (int)R;
  *cols = (int)Cc;
  *nl = (int)n;
  *line_index = idx;
  return GM_OK;
}

gm_status gm_fits_write_image(const char* path, int naxis, const int64_t* naxes, const float* data,
                              const char* const* cards, int ncards) {
  std::vector<int64_t> ax(naxes, naxes + naxis);
  std::vector<std::string> c;
  for (int i = 0; i < ncards; ++i) c.push_back(cards[i]);
  return fits_write(path, ax, data, c);
}

}  // extern "C"
