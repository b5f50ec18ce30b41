/*
 * sharp_geomhelpers.h -- ready-made map geometries (HEALPix and iso-latitude
 * grids).  Same names and argument meaning as the reference's
 * libsharp/sharp_geomhelpers.h, so callers compile unchanged.
 */
#ifndef SHARP_B200_GEOMHELPERS_H
#define SHARP_B200_GEOMHELPERS_H

#include "sharp_lowlevel.h"

#ifdef __cplusplus
extern "C" {
#endif

/* HEALPix RING geometry of resolution nside; weight (2*nside entries, or
   NULL for all ones) multiplies the 4*pi/npix quadrature weight per ring.
   Replaces sharp_make_weighted_healpix_geom_info, sharp_geomhelpers.h:46. */
void sharp_make_weighted_healpix_geom_info (int nside, int stride,
  const double *weight, sharp_geom_info **geom_info);

/* Replaces the static inline sharp_make_healpix_geom_info,
   sharp_geomhelpers.h:52-55. */
static inline void sharp_make_healpix_geom_info (int nside, int stride,
  sharp_geom_info **geom_info)
  { sharp_make_weighted_healpix_geom_info (nside, stride, NULL, geom_info); }

/* Gauss-Legendre grid.  Replaces sharp_make_gauss_geom_info,
   sharp_geomhelpers.h:66. */
void sharp_make_gauss_geom_info (int nrings, int nphi, double phi0,
  int stride_lon, int stride_lat, sharp_geom_info **geom_info);

/* Equidistant grid without polar rings (Fejer's first rule).  Replaces
   sharp_make_fejer1_geom_info, sharp_geomhelpers.h:84. */
void sharp_make_fejer1_geom_info (int nrings, int nphi, double phi0,
  int stride_lon, int stride_lat, sharp_geom_info **geom_info);

/* Old name of the Fejer-1 grid.  Replaces the static inline
   sharp_make_ecp_geom_info, sharp_geomhelpers.h:89-94. */
static inline void sharp_make_ecp_geom_info (int nrings, int nphi, double phi0,
  int stride_lon, int stride_lat, sharp_geom_info **geom_info)
  {
  sharp_make_fejer1_geom_info (nrings, nphi, phi0, stride_lon, stride_lat,
    geom_info);
  }

/* Equidistant grid including the poles (Clenshaw-Curtis).  Replaces
   sharp_make_cc_geom_info, sharp_geomhelpers.h:108. */
void sharp_make_cc_geom_info (int nrings, int ppring, double phi0,
  int stride_lon, int stride_lat, sharp_geom_info **geom_info);

/* Equidistant grid, Fejer's second rule.  Replaces
   sharp_make_fejer2_geom_info, sharp_geomhelpers.h:123. */
void sharp_make_fejer2_geom_info (int nrings, int ppring, double phi0,
  int stride_lon, int stride_lat, sharp_geom_info **geom_info);

/* McEwen-Wiaux grid (no quadrature weights).  Replaces
   sharp_make_mw_geom_info, sharp_geomhelpers.h:135. */
void sharp_make_mw_geom_info (int nrings, int ppring, double phi0,
  int stride_lon, int stride_lat, sharp_geom_info **geom_info);

#ifdef __cplusplus
}
#endif

#endif
