// Device-side plan structures and kernel launchers of the transform engine.
//
// Data layout in HBM (one job, FP64 internal arithmetic):
//   * ring pairs are re-ordered by decreasing mlim (sharp_get_mlim), so the
//     pairs that take part at a given m form the prefix [0, count_m[m]);
//   * staged a_lm  A[(moff[m] + l - m) * ncA + comp]   (double2), scaled by the
//     recurrence normalisation c_l (and norm_l for spin > 0); each m segment
//     is followed by kPad zero entries so l-blocks may run past lmax;
//   * phase       P[((p * ncm + comp) * 2 + hemisphere) * (mmax + 1) + m]
//     (double2): ring-major, so the ring FFT reads and writes contiguous rows
//     and the Legendre kernels write one element per (m, pair, comp, ring).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

#include "sht_internal.h"

namespace sht {

constexpr int kMaxRadices = 24;

// Factorisation of one complex FFT length.
struct FftDesc {
  int n;        // real ring length
  int N;        // complex FFT length (n/2 for even n, n for odd n)
  int tw;       // offset of exp(-2 pi i j/n), j<n, in the twiddle table
  int nrad;
  int rad[kMaxRadices];
  int blue;     // 1: the size-class kernels run a Bluestein convolution of length M
  int M;       // power-of-two convolution length >= 2N - 1
  long long bhat;   // offset of the transformed chirp in the digit order of the
                    // radix-4 stages (/M), or -1 when no generic-class ring uses it
  long long bhat2;  // the same in the digit order of the radix-16 register passes,
                    // or -1 when no register-Bluestein ring uses it
  long long chirp;  // with bhat2: offset of c_j = exp(-pi i j^2/N), j < N, in natural
                    // order (the register kernels read it coalesced), else -1
};

// Host half of a geometry plan (build_geom_host, no device calls): what the
// cached plans upload and the allocation-free synthesis places in its fixed
// scratch.  Pairs are in internal (decreasing mlim) order; per-ring entries
// are indexed 2*p + hemisphere.
struct GeomHost {
  int npairs = 0, nphmax = 0, nmax_complex = 0;
  int P = 2;                          // largest Bluestein convolution length (>= 2)
  int synth_tile = 256;
  std::vector<int> order, count_m, mlim_sorted;
  std::vector<int2> synth_items, mixed_items;
  std::vector<double> cth, sth, phi0, weight;
  std::vector<int> nph, stride, fft;
  std::vector<long long> ofs;
  std::vector<FftDesc> descs;
  std::vector<int> tw_n, tw_off;      // per distinct length: n and table offset
  std::vector<int> blue_idx;          // descriptors with a radix-4 chirp transform (bhat)
  std::vector<int> blue2_idx;         // descriptors with a register-pass one (bhat2)
  long long tw_total = 0, bhat_total = 0, chirp_total = 0;
  std::vector<int> cls_N, cls_start, cls_count, cls_bufA, cls_bufB, cls_pairs;
  // pairs whose rings run the power-of-two register FFT (pow2_ring_length):
  // complex length pw_N[c], listed at pw_pairs[pw_start[c] .. +pw_count[c])
  std::vector<int> pw_N, pw_start, pw_count, pw_pairs;
  // pairs whose rings run the register Bluestein convolution
  // (blue_ring_length): length pb_M[c], listed at pb_pairs[pb_start[c] ..)
  std::vector<int> pb_M, pb_start, pb_count, pb_pairs;
  long long map_lo = 0, map_hi = 0;
  bool map_covered = false;
};
// Shared memory of the register ring kernels (pw_entries(N) buffer entries
// of the ring kernels, the phi0 rotation slices and the twiddle slices of
// the power-of-two analysis), in double2 entries.
inline size_t pow2_ring_smem_entries(int N, int mmax) {
  const int n = N - 1;
  return size_t(n + (n >> 4) + (n >> 8) + 1) + 64 + mmax / 64 + 2 + 64 + N / 64 + 1;
}
constexpr size_t kRingSmemLimit = 227 * 1024;
// Complex FFT length N of a ring that the power-of-two ring kernels take
// (n = 2N pixels with N in {1024, 2048, 4096, 8192}, unit stride, no alias
// folding: mm <= N), else 0.
inline int pow2_ring_length(int nph, int stride, int mm) {
  if (nph <= 0 || (nph & 1) || stride != 1) return 0;
  const int N = nph / 2;
  if (N != 1024 && N != 2048 && N != 4096 && N != 8192) return 0;
  return mm <= N ? N : 0;
}
// Convolution length M of a ring that the register Bluestein kernels take,
// else 0: even nph with M in {1024, 2048, 4096, 8192} (any stride, any alias
// folding) whose complex length either calls for a Bluestein convolution by
// the cost model of the size classes or exceeds 1024 (there the size-class
// kernel, one 1024-thread CTA per SM, ran the mixed-radix Stockham passes
// about twice as slowly per ring as the register convolution).
constexpr int kRegBluesteinMinN = 1024;
inline int blue_ring_length(int nph, const FftDesc &d) {
  if (nph <= 0 || (nph & 1)) return 0;
  if (!d.blue && d.N <= kRegBluesteinMinN) return 0;
  return (d.M == 1024 || d.M == 2048 || d.M == 4096 || d.M == 8192) ? d.M : 0;
}
GeomHost build_geom_host(const sharp_geom_info *g, int lmax, int mmax, int spin);

// Per-geometry device tables (pairs in internal mlim order).
struct GeomPlan {
  const void *key = nullptr;
  uint64_t hash = 0;
  int lmax = -1, mmax = -1, spin = -1;
  int npairs = 0, nphmax = 0, nmax_complex = 0;
  std::vector<int> count_m;          // host copy, mmax+1 entries
  std::vector<int> order;            // internal index -> reference pair index
  std::vector<int2> synth_items;     // (m, tile) work list for synthesis
  int synth_tile = 0;
  std::vector<int2> mixed_items;     // (m, tile of 256 pairs) for the tensor-core path
  // device arrays
  double *cth = nullptr, *sth = nullptr;
  int *mlim = nullptr, *count = nullptr;
  int2 *items = nullptr;
  int2 *mitems = nullptr;
  // per ring (index 2*p + h)
  double *phi0 = nullptr, *weight = nullptr;
  long long *ofs = nullptr;
  int *nph = nullptr, *stride = nullptr, *fft = nullptr;
  FftDesc *fdesc = nullptr;
  double2 *twiddle = nullptr;
  double2 *bhat = nullptr;           // Bluestein chirp transforms
  double2 *chirp = nullptr;          // chirps of the register Bluestein lengths
  double2 *wpow2 = nullptr;          // exp(-2 pi i j/P), j<P, P = largest M
  int P = 2;
  // ring FFT size classes: pairs whose largest complex FFT length is
  // <= cls_N[c], listed at cls_pairs[cls_start[c] .. +cls_count[c])
  std::vector<int> cls_N, cls_start, cls_count, cls_bufA, cls_bufB;
  int *cls_pairs = nullptr;
  // power-of-two register-FFT classes (see GeomHost)
  std::vector<int> pw_N, pw_start, pw_count;
  int *pw_pairs = nullptr;
  // register-Bluestein classes (see GeomHost)
  std::vector<int> pb_M, pb_start, pb_count;
  int *pb_pairs = nullptr;
  long long map_lo = 0, map_hi = 0;  // pixel index extent [lo, hi)
  bool map_covered = false;          // rings tile [lo,hi) exactly
  GeomPlan() = default;
  GeomPlan(const GeomPlan &) = delete;   // owns device memory
  GeomPlan &operator=(const GeomPlan &) = delete;
  ~GeomPlan();
};

// Recurrence coefficient tables for (lmax, mmax, spin).
struct CoefPlan {
  int lmax = -1, mmax = -1, spin = -1;
  long long total = 0;               // table length incl. padding
  std::vector<long long> moff;       // host copy
  long long *d_moff = nullptr;
  double *alpha = nullptr;           // spin 0: alpha; spin>0: a
  double *beta = nullptr;            // spin>0: b = a * fx1
  double *cfac = nullptr;            // c_l
  double *seed = nullptr;            // spin 0: mfac[m]; spin>0: prefac mantissa
  int *seed_exp = nullptr;           // spin>0: prefac exponent (base 2)
  double2 *mx_coef = nullptr;        // mixed analysis: (alpha_l, c_l 2^30 / b_l), lazily built
  CoefPlan() = default;
  CoefPlan(const CoefPlan &) = delete;
  CoefPlan &operator=(const CoefPlan &) = delete;
  ~CoefPlan();
};

// a_lm addressing for one alm_info.
struct AlmPlan {
  const void *key = nullptr;
  uint64_t hash = 0;
  int lmax = 0, mmax = 0;
  bool packed = false;
  long long stride = 0;
  long long lo = 0, hi = 0;          // extent in complex (or real if packed) units
  bool covered = false;              // every element in [lo,hi) is an a_lm
  long long *mvstart = nullptr;      // indexed by m
  AlmPlan() = default;
  AlmPlan(const AlmPlan &) = delete;
  AlmPlan &operator=(const AlmPlan &) = delete;
  ~AlmPlan();
};

struct JobDesc {
  int type;        // SHARP_ALM2MAP, SHARP_MAP2ALM, SHARP_ALM2MAP_DERIV1
  int spin;
  int nmaps, nalm;
  int ntrans;
  int flags;
  int lmax, mmax;
  bool dp;
};

// Mixed-precision tensor-core synthesis (sht_mixed.cu)
bool mixed_synth_supported(const JobDesc &job);
void launch_mixed_synth(const JobDesc &job, const GeomPlan &gp, const CoefPlan &cp,
                        const double2 *A, int ncA, double2 *phase, int ncm, int *d_err,
                        cudaStream_t st);
bool mixed_anal_supported(const JobDesc &job);
void launch_mixed_anal(const JobDesc &job, const GeomPlan &gp, CoefPlan &cp,
                       const double2 *phase, int ncm, double2 *Aout, int ncA, int *d_err,
                       cudaStream_t st);

// Kernel launchers (sht_legendre.cu)
void launch_coef_tables(CoefPlan &cp, cudaStream_t st);
void launch_legendre_synth(const JobDesc &job, const GeomPlan &gp, const CoefPlan &cp,
                           const double2 *A, int ncA, int comp0, int nt,
                           double2 *phase, int ncm, int pcomp0, cudaStream_t st);
void launch_legendre_anal(const JobDesc &job, const GeomPlan &gp, const CoefPlan &cp,
                          const double2 *phase, int ncm, int pcomp0, int nt,
                          double *Aout, int ncA, int comp0, cudaStream_t st);

// Ring FFT and staging launchers (sht_ring.cu)
void launch_twiddles(GeomPlan &gp, int ntw, const std::vector<int> &tw_n,
                     const std::vector<int> &tw_off, cudaStream_t st);
void launch_bluestein_setup(GeomPlan &gp, const GeomHost &h, cudaStream_t st);
void launch_twiddles_preplaced(double2 *tw, const int *d_n, const int *d_off, int ntab,
                               cudaStream_t st);
void launch_bluestein_setup_preplaced(const GeomPlan &gp, const int *d_blue_idx, int nblue,
                                      const int *d_blue2_idx, int nblue2, cudaStream_t st);
// map_lo / alm_lo: index (in elements of the user array) that the device
// pointers in maps_dev / alm_dev point at (0 when they are the user's own
// device arrays, the extent start when they are staged copies).
// Ring FFT shared memory.  Entries of the high twiddle slice for ring lengths
// up to 2 nmax_complex, and the double2 entries of one CTA: buffers A and B,
// the phi0 shift slices (64 + mmax/64 + 2), the twiddle slices of the ring
// length and of the Bluestein convolution length P (64 + P/64 + 2).
inline int ring_twiddle_hi_entries(int nmax_complex) { return (2 * nmax_complex) / 64 + 2; }
inline size_t ring_fft_smem_entries(int bufA, int bufB, int mmax, int nmax_complex, int P) {
  return size_t(bufA) + bufB + (64 + mmax / 64 + 2) + (64 + ring_twiddle_hi_entries(nmax_complex)) +
         (64 + P / 64 + 2);
}

void launch_phase2ring(const JobDesc &job, const GeomPlan &gp, long long map_lo,
                       const double2 *phase, int ncm, void *const *maps_dev, int nmapptr,
                       cudaStream_t st);
void launch_ring2phase(const JobDesc &job, const GeomPlan &gp, long long map_lo,
                       const void *const *maps_dev, int nmapptr, double2 *phase, int ncm,
                       cudaStream_t st);
void launch_phase2ring_direct(const JobDesc &job, const GeomPlan &gp, long long map_lo,
                              const double2 *phase, int ncm, void *const *maps_dev, int nmapptr,
                              cudaStream_t st);
void launch_ring2phase_direct(const JobDesc &job, const GeomPlan &gp, long long map_lo,
                              const void *const *maps_dev, int nmapptr, double2 *phase,
                              int ncm, cudaStream_t st);
void launch_stage_alm(const JobDesc &job, const AlmPlan &ap, long long alm_lo,
                      const CoefPlan &cp, const double *norm_l, const void *const *alm_dev,
                      int nalmptr, double2 *A, int ncA, cudaStream_t st);
void launch_scatter_alm(const JobDesc &job, const AlmPlan &ap, long long alm_lo,
                        const CoefPlan &cp, const double *norm_l, const double *Aout, int ncA,
                        void *const *alm_dev, int nalmptr, cudaStream_t st);

// Launch accounting: every launcher wraps its kernel in a ProfScope, which
// counts the launch and, when profiling is on, records CUDA events on the
// launching stream around it.
class ProfScope {
 public:
  ProfScope(const char *family, cudaStream_t st);
  ~ProfScope();
  ProfScope(const ProfScope &) = delete;
  ProfScope &operator=(const ProfScope &) = delete;

 private:
  const char *family_;
  cudaStream_t st_;
  cudaEvent_t start_ = nullptr;
};

void check_cuda(cudaError_t e, const char *what, const char *file, int line);
#define SHT_CUDA(call) ::sht::check_cuda((call), #call, __FILE__, __LINE__)

// Stream-ordered workspace allocation from the library's own memory pool on
// the current device (free with cudaFreeAsync, never cudaFree, which leaves
// the pool's accounting wrong).  The pool keeps freed memory mapped across
// synchronizes (release threshold unlimited), so a transform after a
// synchronize does not map gigabytes of workspace again, and being the
// library's own it leaves the settings of the process's default pool alone.
// Plan-lifetime tables use cudaMalloc.  ws_trim() hands the unused memory
// back (sharp_b200_release_cache); ws_bytes() reports the pool's size.
cudaError_t ws_alloc_bytes(void **p, size_t bytes, cudaStream_t st);
template <typename T>
inline cudaError_t ws_alloc(T **p, size_t bytes, cudaStream_t st) {
  return ws_alloc_bytes(reinterpret_cast<void **>(p), bytes, st);
}
void ws_trim();
bool ws_bytes(unsigned long long *reserved, unsigned long long *used);

}  // namespace sht
