/*
 * mtb_fits.h -- FITS cube writer for the Stokes images.
 *
 * Writes what mt-imager's ImageManager writes through cfitsio and casacore
 * (code/mt-imager/lib/components/ImageManager.cpp:59-236): one primary HDU,
 * BITPIX -32, NAXIS = 4 with axes (l, m, Stokes, frequency), a SIN projection
 * centred on the phase centre at pixel (nx/2, ny/2) (0-based), CDELT1 = -l
 * increment, BUNIT 'JY/BEAM'.  Channels are written as they are finished, in
 * any order; each channel is the [P][ny][nx] image mtb_finalize produces.
 * cfitsio is not used: the file is written directly in 2880-byte blocks,
 * big-endian.
 */
#ifndef MTB_FITS_H
#define MTB_FITS_H

#include "mtb.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mtb_fits mtb_fits;

typedef struct mtb_fits_header {
    int nx, ny, nstokes, nchan;
    double l_increment, m_increment;   /* radians                                   */
    double ra_deg, dec_deg;            /* phase centre                              */
    const double *freqs_hz;            /* [nchan]; the axis is written linear from
                                          freqs_hz[0] with the mean spacing         */
    const int *stokes;                 /* [nstokes] FITS codes: 1 I, 2 Q, 3 U, 4 V   */
    const char *telescope;             /* may be NULL                               */
    const char *observer;              /* may be NULL                               */
    double obs_mjd;                    /* observation start, MJD (UTC); 0: omitted  */
} mtb_fits_header;

/* Creates the file (replacing an existing one), writes the header and sizes
 * the data area (zero-filled). */
int mtb_fits_create(const char *path, const mtb_fits_header *h, mtb_fits **out);
/* Writes channel `chan` from host memory float [nstokes][ny][nx]. */
int mtb_fits_write_channel(mtb_fits *f, int chan, const float *image);
/* Flushes and closes the file. */
int mtb_fits_close(mtb_fits *f);

#ifdef __cplusplus
}
#endif
#endif /* MTB_FITS_H */
