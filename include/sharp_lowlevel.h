/*
 * sharp_lowlevel.h -- C ABI of the B200 spherical-harmonic transform engine.
 *
 * This header declares exactly the types and entry points that callers of
 * libsharp's low-level interface bind to, so existing C/C++/Fortran callers
 * (Healpix_cxx alm2map/map2alm via sharp_cxxjob<T>, conviqt_v4, the Fortran
 * bind(c) wrapper) relink against libsharp_b200.so unchanged.
 *
 * Struct layouts must stay byte-identical to the reference because callers
 * index geometry pairs directly.  Each declaration names the reference
 * declaration it replaces (zonca/planck-levelS, libsharp/sharp_lowlevel.h).
 *
 * Work runs on the current CUDA device.  Host pointers are accepted
 * everywhere (data are staged through HBM); see sharp_b200.h for the
 * device-pointer, batched, mixed-precision and adjoint extensions.
 */
#ifndef SHARP_B200_LOWLEVEL_H
#define SHARP_B200_LOWLEVEL_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One iso-latitude ring.  Replaces sharp_ringinfo, sharp_lowlevel.h:43-48. */
typedef struct
  {
  double theta, phi0, weight, cth, sth;
  ptrdiff_t ofs;
  int nph, stride;
  } sharp_ringinfo;

/* Two rings mirrored about the equator (r1 north); r2.nph==-1 when the ring
   has no partner.  Replaces sharp_ringpair, sharp_lowlevel.h:52-56. */
typedef struct
  {
  sharp_ringinfo r1,r2;
  } sharp_ringpair;

/* Map geometry.  Replaces sharp_geom_info, sharp_lowlevel.h:60-64. */
typedef struct
  {
  sharp_ringpair *pair;
  int npairs, nphmax;
  } sharp_geom_info;

/* a_lm layout: index(l,mval[mi]) = mvstart[mi] + stride*l.
   Replaces sharp_alm_info, sharp_lowlevel.h:71-86. */
typedef struct
  {
  int lmax;
  int nm;
  int *mval;
  int flags;
  ptrdiff_t *mvstart;
  ptrdiff_t stride;
  } sharp_alm_info;

/* m=0 coefficients stored as reals only; mvstart counts reals.
   Replaces sharp_almflags, sharp_lowlevel.h:89-93. */
typedef enum { SHARP_PACKED = 1 } sharp_almflags;

/* Replaces sharp_make_alm_info, sharp_lowlevel.h:106. */
void sharp_make_alm_info (int lmax, int mmax, int stride,
  const ptrdiff_t *mstart, sharp_alm_info **alm_info);
/* Replaces sharp_make_general_alm_info, sharp_lowlevel.h:119. */
void sharp_make_general_alm_info (int lmax, int nm, int stride, const int *mval,
  const ptrdiff_t *mvstart, int flags, sharp_alm_info **alm_info);
/* Replaces sharp_alm_index, sharp_lowlevel.h:125. */
ptrdiff_t sharp_alm_index (const sharp_alm_info *self, int l, int mi);
/* Replaces sharp_destroy_alm_info, sharp_lowlevel.h:127. */
void sharp_destroy_alm_info (sharp_alm_info *info);

/* Sorts rings by sin(theta), pairs north/south rings and sorts the pairs by
   (nph, phi0, cth) as the reference does.  wgt==NULL means weight 1.
   Replaces sharp_make_geom_info, sharp_lowlevel.h:147. */
void sharp_make_geom_info (int nrings, const int *nph, const ptrdiff_t *ofs,
  const int *stride, const double *phi0, const double *theta,
  const double *wgt, sharp_geom_info **geom_info);
/* Replaces sharp_destroy_geom_info, sharp_lowlevel.h:152.  Also releases any
   device tables cached for this geometry. */
void sharp_destroy_geom_info (sharp_geom_info *info);

/* Job types.  Replaces sharp_jobtype, sharp_lowlevel.h:160-167. */
typedef enum { SHARP_YtW=0,
               SHARP_MAP2ALM=SHARP_YtW,
               SHARP_Y=1,
               SHARP_ALM2MAP=SHARP_Y,
               SHARP_Yt=2,
               SHARP_WY=3,
               SHARP_ALM2MAP_DERIV1=4
             } sharp_jobtype;

/* Job flags.  Replaces sharp_jobflags, sharp_lowlevel.h:170-191.  Bits 8-19
   carry the B200 extensions declared in sharp_b200.h. */
typedef enum { SHARP_DP              = 1<<4,
               SHARP_ADD             = 1<<5,
               SHARP_REAL_HARMONICS  = 1<<6,
               SHARP_NO_FFT          = 1<<7,
               SHARP_USE_WEIGHTS     = 1<<20,
               SHARP_NO_OPENMP       = 1<<21,
               SHARP_NVMAX           = (1<<4)-1
             } sharp_jobflags;

/* Runs one transform job: ntrans simultaneous SHTs of the given type and spin.
   alm/map are arrays of host pointers (ntrans*nalm and ntrans*nmaps of them;
   complex double/double with SHARP_DP, complex float/float otherwise).
   Outputs are overwritten unless SHARP_ADD.  time (seconds, wall clock) and
   opcnt (floating-point operation estimate) may be NULL.
   Replaces sharp_execute, sharp_lowlevel.h:222-224. */
void sharp_execute (sharp_jobtype type, int spin, void *alm, void *map,
  const sharp_geom_info *geom_info, const sharp_alm_info *alm_info, int ntrans,
  int flags, double *time, unsigned long long *opcnt);

/* Chunking knobs of the reference job driver, accepted and stored for ABI
   compatibility.  The GPU engine keeps whole transforms resident in HBM and
   does not split ring pairs into chunks.
   Replace sharp_set_chunksize_min / sharp_set_nchunks_max,
   sharp_lowlevel.h:226-227. */
void sharp_set_chunksize_min(int new_chunksize_min);
void sharp_set_nchunks_max(int new_nchunks_max);

/* Largest m with non-negligible Y_lm on a ring of the given sin/cos(theta)
   (same rule as the reference).  Replaces sharp_get_mlim,
   sharp_internal.h:64. */
int sharp_get_mlim (int lmax, int spin, double sth, double cth);

/* Vector-length hint of the low flag bits: accepted and ignored, so the
   largest hint is 1 and the oracle answers 1.  Replace sharp_get_nv_max and
   sharp_nv_oracle, sharp_internal.h:62-63. */
int sharp_get_nv_max (void);
int sharp_nv_oracle (sharp_jobtype type, int spin, int ntrans);

/* Start-up banner of the reference's tools (printed to stdout), and the
   argument-count check that prints the usage and exits(1) on a mismatch.
   Replace sharp_announce and sharp_module_startup, sharp_announce.h:35-37. */
void sharp_announce (const char *name);
void sharp_module_startup (const char *name, int argc, int argc_expected,
  const char *argv_expected, int verbose);

#ifdef __cplusplus
}
#endif

#endif
