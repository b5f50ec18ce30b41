/*
 * sharp_almhelpers.h -- standard a_lm layouts.  Same names and meaning as
 * the reference's libsharp/sharp_almhelpers.h.
 */
#ifndef SHARP_B200_ALMHELPERS_H
#define SHARP_B200_ALMHELPERS_H

#include "sharp_lowlevel.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Healpix_cxx layout: m-major, mvstart[m] = stride*m*(2*lmax+1-m)/2.
   Replaces sharp_make_triangular_alm_info, sharp_almhelpers.h:44. */
void sharp_make_triangular_alm_info (int lmax, int mmax, int stride,
  sharp_alm_info **alm_info);

/* Fortran Healpix layout: mvstart[m] = stride*m*(lmax+1).
   Replaces sharp_make_rectangular_alm_info, sharp_almhelpers.h:50. */
void sharp_make_rectangular_alm_info (int lmax, int mmax, int stride,
  sharp_alm_info **alm_info);

#ifdef __cplusplus
}
#endif

#endif
