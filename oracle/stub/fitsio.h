/* Empty stand-in for cfitsio's header.
 *
 * The reference's inversion core (ME_SOLVER, LM_FIT, FADDEEVA, SVD, INV_INIT,
 * RINPUT, RANDOM_NUMBER, LOG_ERROR, STR, ALLOCATION) includes <fitsio.h> through
 * Src/RINPUT.h:6 but uses no cfitsio symbol; only Src/IO.c does, and IO.c is not
 * part of the oracle build.  cfitsio is not installed in this image, so this
 * header lets the core compile unmodified.
 */
#pragma once
