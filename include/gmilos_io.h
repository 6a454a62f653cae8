/* gmilos_io.h -- the reference's on-disk formats on either side of the
 * inversion path, for C/C++ hosts (and, through ctypes, for Python):
 *
 *   control file (.mtrol)   readTrolFile, readConfig.c:1421-2101
 *   model (.mod)            readInitialModel, readConfig.c:495-545; the
 *                           inverted-model writer of gmilos.cu:839-858
 *   wavelength grid (.grid) readMallaGrid, readConfig.c:626-660
 *   line list (LINES)       readFileCuanticLines, readConfig.c:388-493
 *   PSF table (.psf)        readPSFFile, readConfig.c:673-702
 *   profiles (.per)         the readers of gmilos.cu:317-335 and
 *                           readPerStrayLightFile, utilsFits.c:1532-1576;
 *                           the writer of gmilos.cu:582-590
 *   FITS cubes              readFitsSpectroImage, utilsFits.c:267-657 (axes
 *                           from CTYPEn, else from their lengths);
 *                           writeFitsImageModels, utilsFits.c:2403-2525;
 *                           writeFitsImageProfiles, utilsFits.c:2777-2950;
 *                           readFitsStrayLightFile, utilsFits.c:1578-1896;
 *                           readFitsLambdaToArray, utilsFits.c:1446-1530
 *
 * The FITS code is this project's own reader/writer of single-HDU images
 * (FITS Standard 4.0: 2880-byte blocks, 80-character cards, big-endian
 * IEEE data); CFITSIO is not used.  Pixel order of every cube in memory is
 * the reference's: pixel p = col * rows + row (rows along the HPLN-TAN axis,
 * columns along HPLT-TAN), each pixel [4][nl].
 *
 * Every function returns GM_OK or an error status; a message is available
 * from gm_io_last_error() (thread-local). */
#ifndef GMILOS_IO_H
#define GMILOS_IO_H

#include <stdint.h>

#include "gmilos.h"

#ifdef __cplusplus
extern "C" {
#endif

#define GM_IO_PATH 4096

/* The control file, field by field in the reference's fixed line order. */
typedef struct {
    int ncycles;                  /* Number of cycles: < 0 classical estimates,
                                     0 synthesis, > 0 LM iterations */
    char observed[GM_IO_PATH];    /* Observed profiles (.per or .fits) */
    char stray[GM_IO_PATH];       /* Stray light file (.per or .fits) or empty */
    char psf[GM_IO_PATH];         /* PSF field as written */
    int use_psf;                  /* 1 when a PSF applies */
    double fwhm_mA;               /* > 0: Gaussian of this FWHM instead of a table */
    char wavelength[GM_IO_PATH];  /* .fits wavelength file, when not a grid */
    char grid[GM_IO_PATH];        /* .grid file */
    int use_grid;
    char lines[GM_IO_PATH];       /* Atomic parameters file */
    char abundances[GM_IO_PATH];  /* not used by the inversion */
    char init_model[GM_IO_PATH];  /* Initial guess model 1 (.mod) */
    char init_model2[GM_IO_PATH]; /* not used by the inversion */
    float weight[4];              /* Weight for Stokes I, Q, U, V */
    int auto_nodes;               /* not used by the inversion */
    int fix[GM_NPAR];             /* free flags, the reference's fix[] order */
    int fix2[GM_NPAR];            /* second component: not used by the inversion */
    int invert_filling_factor;    /* not used by the inversion */
    float mu;
    int sn_i;                     /* Estimated S/N for I */
    double noise;                 /* (1/S/N)^2 when S/N is given, else 1e-6 */
    int continuum_contrast;       /* not used by the inversion */
    float ilambda;                /* Initial diagonal element */
    int use_fft;                  /* not used (direct convolution) */
    int logclambda;               /* Diagonal element acceleration */
    int nstreams;                 /* Number of Streams (reference GPU launch) */
    int device;                   /* Device number */
} gm_trol;

const char *gm_io_last_error(void);

/* defaults of loadInitialValues (readConfig.c:704-744) */
void gm_io_trol_defaults(gm_trol *t);
gm_status gm_io_read_trol(const char *path, gm_trol *t);

/* .mod: "name: value" lines matched by key substrings (eta_0, magnetic field,
 * LOS velocity, Doppler width, damping, gamma, phi, S_0, S_1, v_mac, filling
 * factor); absent keys keep the values model[] holds on entry. */
gm_status gm_io_read_model(const char *path, double model[GM_NPAR]);
/* the inverted-model file: the 11 parameters, iterations and chi2 */
gm_status gm_io_write_model(const char *path, const double model[GM_NPAR], int iters, float chi2);

gm_status gm_io_read_grid(const char *path, int *line_index, double *first_mA, double *step_mA,
                          double *last_mA);
/* offsets [mA] and absolute wavelengths [A] of a grid, accumulated sample by
 * sample as the reference does (gmilos.cu:171-196); returns the sample count
 * (0 on error) and fills at most cap entries */
int gm_io_grid_wavelengths(double lambda0, double first_mA, double step_mA, double last_mA,
                           double *offsets_mA, double *lambda, int cap);

/* Line line_index of the line list: centre [A] and the lower / upper levels'
 * S, L, J (S from the multiplicity, L from the spectroscopic letter). */
gm_status gm_io_read_line(const char *path, int line_index, double *lambda0, double quantum[6]);

/* PSF table: offsets [mA] and values, at most cap rows; *n = rows read */
gm_status gm_io_read_psf_table(const char *path, double *x_mA, double *y, int cap, int *n);

/* .per: nl lines "index offset I Q U V"; iquv [4][nl]; offsets may be NULL */
gm_status gm_io_read_per(const char *path, int nl, float *iquv, double *offsets_mA);
gm_status gm_io_write_per(const char *path, int line_index, int nl, const double *offsets_mA,
                          const float *iquv);

/* ---- FITS ---- */
typedef struct gm_fits_cube gm_fits_cube;

/* A Stokes cube: 4 axes (CTYPE WAVE-GRI, STOKES, HPLN-TAN, HPLT-TAN, or
 * inferred from the axis lengths as the reference does), nl_expected
 * wavelength samples (0: any).  BITPIX -32 as the reference requires; -64
 * is converted. */
gm_status gm_fits_read_cube(const char *path, int nl_expected, gm_fits_cube **out);
void gm_fits_cube_dims(const gm_fits_cube *c, int *rows, int *cols, int *nl);
/* the pixels [rows*cols][4][nl], pixel p = col * rows + row */
float *gm_fits_cube_data(gm_fits_cube *c);
void gm_fits_cube_free(gm_fits_cube *c);

/* Fitted profiles with the input cube's axes and header cards. */
gm_status gm_fits_write_profiles(const char *path, const gm_fits_cube *like, const float *iquv);

/* Model planes: NAXIS1 = rows, NAXIS2 = cols, NAXIS3 = 12 (+1 with chi2):
 * the 11 parameters, iterations, chi2; pixel p at (row, col) as read. */
gm_status gm_fits_write_models(const char *path, int rows, int cols, const double *models,
                               const int *iters, const float *chi2, int with_chi2);

/* Stray light: one profile (2-D, [4][nl] in either axis order; *per_pixel
 * = 0) or a map with the cube's layout (4-D; *per_pixel = 1).  *out is
 * malloc'd [4][nl] or [P][4][nl]; free with gm_io_free. */
gm_status gm_fits_read_stray(const char *path, int nl, float **out, int *per_pixel, int *rows,
                             int *cols);

/* Wavelength file: NAXIS = 2, row 1 = line index, row 2 = wavelengths [A]
 * (readFitsLambdaToArray, utilsFits.c:1446-1487). */
gm_status gm_fits_read_lambda(const char *path, double *lambda, int cap, int *nl, int *line_index);

/* Wavelength file with one grid (2-D, as above; *per_pixel = 0, *out [nl])
 * or per-pixel grids (*per_pixel = 1, *out [P][nl], pixel p = col * rows +
 * row as in gm_fits_read_cube): NAXIS1 = rows, NAXIS2 = cols, NAXIS3 =
 * 1 + nl, optional NAXIS4 = 1; plane 0 holds the line index (the same in
 * every pixel), planes 1..nl the pixel's wavelengths [A] -- the 2-D layout
 * with pixels added.  The reference meant its 4-D branch for this
 * (utilsFits.c:1488-1500) but reads it into a NULL pointer.  BITPIX -64
 * keeps the wavelengths exact.  *out is malloc'd; free with gm_io_free. */
gm_status gm_fits_read_lambda_map(const char *path, double **out, int *per_pixel, int *rows, int *cols,
                                  int *nl, int *line_index);

/* Generic single-HDU float image (for tests and tools): naxes[0] fastest. */
gm_status gm_fits_write_image(const char *path, int naxis, const int64_t *naxes, const float *data,
                              const char *const *cards, int ncards);

void gm_io_free(void *p);

#ifdef __cplusplus
}
#endif
#endif
