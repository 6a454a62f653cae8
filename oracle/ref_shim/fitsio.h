/* Stand-in for CFITSIO's header, used only when the reference's per-pixel
 * sources are compiled for the comparison builds.  Those sources include it
 * for the declarations of their FITS image structure (defines.h), which
 * needs one constant: the length of a FITS header card plus terminator.
 * No CFITSIO function is declared or called. */
#ifndef GM_SHIM_FITSIO_H
#define GM_SHIM_FITSIO_H
#define FLEN_CARD 81
#endif
