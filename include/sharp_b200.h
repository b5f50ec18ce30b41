/*
 * sharp_b200.h -- extensions of the B200 transform engine beyond the
 * reference ABI.  None of these has a counterpart in the reference except
 * where a comment names one; the reference-compatible surface is in
 * sharp_lowlevel.h, sharp_geomhelpers.h and sharp_almhelpers.h.
 */
#ifndef SHARP_B200_EXT_H
#define SHARP_B200_EXT_H

#include "sharp_lowlevel.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Extra job flags, in bits the reference leaves unused (8-19). */
enum {
  /* Apply the transpose of the named job type:
     Y (ALM2MAP) -> Yt, YtW (MAP2ALM) -> WY, Yt -> Y, WY -> YtW.
     Yt is the exact adjoint of Y under <a,b> = sum_{m=0} Re(a*b)
     + 2 sum_{m>0} Re(a*b) on a_lm and the plain dot product on maps. */
  SHARP_ADJOINT = 1<<8,
  /* Mixed-precision execution of alm2map and map2alm (any spin):
     the recurrence stays FP64 on the CUDA cores; its values are quantised
     to 32-bit fixed point against an analytic bound, the other operand to
     signed base-256 digits, and the Legendre contraction runs exactly in
     integers on the int8 tensor cores (int32 accumulation, combined in
     64-bit integers and scaled to FP64 per l-tile).  Results are within
     1e-6 relative L2 of the FP64 path (typically 1e-8).  Other job types
     ignore the flag. */
  SHARP_MIXED   = 1<<9,
  /* Subtract the result from the output arrays (maps or a_lm) instead of
     overwriting them: the counterpart of SHARP_ADD, with which it may not be
     combined.  It lets an iteration such as map2alm_iter form its residual
     inside the transform instead of in a separate pass over the data. */
  SHARP_SUBTRACT = 1<<10
};

/* Message of the last failed call on this thread ("" when none). */
const char *sharp_b200_last_error(void);
void sharp_b200_clear_error(void);
/* 1 (default, the reference's behaviour): print the message and exit(1) on a
   bad argument or a CUDA failure.  0: return early and keep the message for
   sharp_b200_last_error().  The environment variable
   SHARP_B200_ABORT_ON_ERROR=0 selects 0 at start-up. */
void sharp_b200_set_abort_on_error(int on);

/* Same job semantics as sharp_execute, but every alm/map pointer is a device
   address on the current CUDA device and the work is enqueued on `stream`
   (a cudaStream_t; NULL = legacy default stream) without host
   synchronisation.  time (if non-NULL) receives the enqueue time only. */
void sharp_b200_execute_device (sharp_jobtype type, int spin, void *alm,
  void *map, const sharp_geom_info *geom_info, const sharp_alm_info *alm_info,
  int ntrans, int flags, void *stream, double *time,
  unsigned long long *opcnt);

/* Waits for the work enqueued on `stream` (a cudaStream_t; NULL = legacy
   default stream) and reports whether a SHARP_MIXED transform on the device
   gave up on one of its bounded internal waits (its outputs are then not
   valid), or whether the stream failed.  Device-pointer callers use it to
   learn of such a failure for the call that had it; without it the failure
   is reported at the start of the next SHARP_MIXED call.  Returns 0, or -1
   after a failure (message in sharp_b200_last_error(); in the default abort
   mode the failure ends the process as other errors do). */
int sharp_b200_check_device_errors (void *stream);

/* A new geometry holding the ring pairs pairs[0..npairs) of geom_info
   (indices into geom_info->pair), the ring structs copied unchanged; free it
   with sharp_destroy_geom_info.  It serves the decomposition of one transform
   over several GPUs by ring pairs (each GPU runs its subset; the analysis
   sums the partial a_lm over the GPUs), which takes the place of the
   reference's MPI job driver sharp_execute_mpi (libsharp/sharp_mpi.h:80-83)
   for the ring side.  Returns 0, or -1 on a bad argument (message in
   sharp_b200_last_error()). */
int sharp_b200_make_subset_geom_info (const sharp_geom_info *geom_info,
  const int *pairs, int npairs, sharp_geom_info **subset);

/* Drops the device tables cached for this geometry (sharp_destroy_geom_info
   calls it). */
void sharp_b200_forget_geometry (const sharp_geom_info *geom_info);

/* Frees every cached device table and workspace of the calling process. */
void sharp_b200_release_cache (void);

/* Device memory of the library's workspace pool on the current device:
   *reserved = bytes the pool keeps mapped (freed workspace stays mapped for
   the next job until sharp_b200_release_cache), *used = bytes of live
   workspace.  Returns 0, or -1 (both set to 0) before the first job on this
   device.  No counterpart in the reference. */
int sharp_b200_workspace_bytes (unsigned long long *reserved, unsigned long long *used);

/* Number of CUDA kernels this library has launched in the calling process. */
unsigned long long sharp_b200_kernel_launches (void);

/* Per-kernel timing with CUDA events recorded on the launching stream around
   every kernel of the library (off by default; costs two event records per
   launch).  on=1 starts collecting, on=0 stops and discards. */
void sharp_b200_profile (int on);
/* Waits for the recorded events and returns the summed milliseconds of all
   launches of one kernel family since profiling started ("legendre_synth",
   "legendre_anal", "mixed_synth_spin0", "mixed_synth_spin",
   "mixed_anal_spin0", "mixed_anal_spin", "mixed_image", "ring_synth",
   "ring_anal", "stage_alm", "scatter_alm"); *launches (if non-NULL)
   receives their number. */
double sharp_b200_profile_ms (const char *family, unsigned long long *launches);

/* One job of a batch: the arguments of sharp_execute. */
typedef struct {
  sharp_jobtype type;
  int spin;
  void *alm;                          /* ntrans * nalm pointers, as sharp_execute */
  void *map;                          /* ntrans * nmaps pointers */
  const sharp_geom_info *geom_info;
  const sharp_alm_info *alm_info;
  int ntrans;
  int flags;
} sharp_b200_job;

/* Runs a batch of jobs of uneven geometry, lmax and spin (for example many
   spin-0 and spin-2 maps at several HEALPix resolutions, or the alm2map and
   map2alm halves of a round trip).  No counterpart in the reference, whose
   callers loop over sharp_execute.  Jobs that share type, spin, flags and
   the same geom_info and alm_info objects are merged into one job of up to
   100 transforms, so the batched kernels (SHARP_MIXED) see them together.
   Every output equals that of sharp_execute on its own job, run in list
   order (neither the merge nor the scheduling changes any arithmetic).
   Jobs must not share output arrays.
   device_ptrs = 0: host arrays; the jobs take effect in list order: a job
   may read host arrays that an earlier job of the batch writes (its input
   copies wait for those output copies; in such a batch only consecutive
   jobs are merged).  All merged jobs run as one pipelined sequence of pieces
   (host->device copies, compute and device->host copies overlapped across
   the whole batch); returns after the results are copied back.
   device_ptrs = 1: device arrays; the jobs must be independent (no job reads
   another's output), any compatible jobs are merged, and the merged jobs
   run side by side on up to four library streams forked from `stream` and
   joined back to it (work ordered after what `stream` holds, later work on
   `stream` after the batch), without host synchronisation.  opcnt (if
   non-NULL) receives the summed operation count.  Returns the number of
   merged groups executed, or -1 after a failure in non-abort mode. */
int sharp_b200_execute_batch (const sharp_b200_job *jobs, int njobs,
  int device_ptrs, void *stream, unsigned long long *opcnt);

/* How sharp_b200_execute_batch would merge `jobs` (same arguments): returns
   the number of merged groups and, if group_of_job is non-NULL, each job's
   group index (groups numbered in order of first appearance), or -1 after
   an argument error in non-abort mode.  Host work only: nothing runs on the
   GPU and no array is read. */
int sharp_b200_batch_groups (const sharp_b200_job *jobs, int njobs,
  int device_ptrs, int *group_of_job);

/* Spin-0 alm2map without any device allocation.  No counterpart in the
   reference: it serves callers that cannot call cudaMalloc when they need a
   transform (GPU memory owned by another allocator such as a framework's
   caching pool or an arena reserved at start-up, or a no-allocation policy
   after initialisation).  Same result as sharp_b200_execute_device(
   SHARP_ALM2MAP, 0, ..., SHARP_DP) with one transform: alm (complex double,
   layout alm_info, not SHARP_PACKED) and map (double) are device pointers,
   ring pixels of map are overwritten, work is enqueued on `stream`.
   All scratch lives in one fixed 32 MiB __device__ array that every GPU
   loading the library holds until exit (about Nside 256 / lmax 512 fits);
   larger problems are rejected: the call returns -1 and
   sharp_b200_last_error() says how much scratch they would need.  Other
   failures follow the library's abort policy (in non-abort mode: -1).
   Returns 0 on success.  The first call on each device looks up the array's
   address.  All calls share the array:
   calls that overlap on the GPU race and must be serialised by the caller. */
int sharp_b200_alm2map_noalloc (const sharp_geom_info *geom_info,
  const sharp_alm_info *alm_info, const void *alm, void *map, void *stream);

#ifdef __cplusplus
}
#endif

#endif
