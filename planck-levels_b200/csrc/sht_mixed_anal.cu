// Mixed-precision batched analysis (map2alm Legendre step) on the
// 5th-generation tensor cores, spin 0.
//
// For NB transforms sharing geometry and lmax the analysis of order m is
//   A_l[col] = sum_p lambda_l(p) N_p[col] + (-1)^(l-m) sum_p lambda_l(p) S_p[col]
// with N/S the north/south ring phases (weights already applied) and
// col = (transform, re/im).  As in the synthesis, the FP64 recurrence stays on
// the CUDA cores and the contraction runs exactly in integers on
// tcgen05.mma.kind::i8, here with the roles of the operands turned around:
//
//  * A (M = 64 consecutive l, K = (ring pair, byte)): the words
//    u_l(p) = 2^31 + round(lambda_l(p) 2^30 / b_l), b_l = sqrt((2l+1)/4pi) the
//    analytic bound, one magic-constant DFMA each; a producer thread owns one
//    ring pair and writes one 4-byte word per l.
//  * B (N = (half, column, weight), K = (ring pair, byte)): the Toeplitz
//    expansion of the signed base-256 digits of the ring phases, quantised per
//    group of 256 ring pairs and (half, column) against the group's maximum.
//    It is built once per group in shared memory and stays there while the
//    group sweeps all l.
//  * D (int32, TMEM): per l-tile the exact class sums over the group's ring
//    pairs.  Two tiles share one TMEM column set (lanes 0-15 and 16-31 of
//    each subpartition), two sets alternate; a pair is read back one lane per
//    l, its class sums combined exactly in 64-bit integers, corrected for the
//    2^31 offset and scaled in FP64, and added to the output (one CTA per m,
//    so no atomics).
//    Like the FP64 kernels, the output holds sum_p mu_l(p) phi_p with the
//    rescaled recurrence values mu_l = lambda_l / c_l; c_l is applied when the
//    a_lm are scattered.
//
// Warp roles (288 threads): warps 0-7 each own 32 ring pairs of the current
// group; warp 8 (lane 0) stages each l-tile's recurrence coefficients into
// shared memory (cp.async.bulk) and issues its MMAs.  Every wait is bounded;
// a timeout is reported through the error word.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "sht_device.h"
#include "sht_recurrence.cuh"
#include "sht_tc.cuh"

namespace sht {

namespace {

constexpr int kAW = 8;                        // producer warps
constexpr int kAGroup = 32 * kAW;             // ring pairs per group (K extent)
constexpr int kAM = 64;                       // l rows per tile (MMA M)
constexpr int kAThreads = 32 * (kAW + 1);
constexpr int kAKB = 4 * kAGroup;             // K bytes of a group
constexpr int kAClasses = 5;                  // byte-product weights 2^16 .. 2^48
// A slice of one warp and tile (64 l x 32 ring pairs, K-major, no swizzle):
// the 8-row groups are contiguous (SBO = 128) and the 8 K core matrices lie
// kALBO = 8*128 + 16 bytes apart, so the per-l 4-byte stores of a warp hit 32
// distinct banks with 112 bytes of padding per slice.
constexpr int kALBO = (kAM / 8) * 128 + 16;
constexpr int kASlice = 7 * kALBO + (kAM / 8) * 128;
constexpr int kACoef = kAM * 16;              // one tile's (alpha, cq) pairs

template <int NB_>
struct AShape {
  static constexpr int NB = NB_;
  static constexpr int NCOL = 2 * NB;                  // real columns
  static constexpr int NH = 2 * NCOL;                  // (half, column): north, then south
  static constexpr int NPR = kAClasses * NH;           // B rows used
  static constexpr int NP = (NPR + 15) / 16 * 16;      // MMA N
  // B (NP x 1024 bytes of K): row groups contiguous, K core matrices BLBO
  // apart (conflict-free per-ring stores, as for A)
  static constexpr int BLBO = (NP / 8) * 128 + 16;
  static constexpr int BBYTES = ((kAKB / 16 - 1) * BLBO + (NP / 8) * 128 + 127) / 128 * 128;
  static constexpr int SMEM = 2 * kAW * kASlice + BBYTES + 2 * kACoef;
  // TMEM: a pair of tiles shares one column set (lanes 0-15 / 16-31 of each
  // subpartition); two column sets
  static constexpr uint32_t NCOLS = 2 * NP <= 32 ? 32 : 2 * NP <= 64 ? 64 : 2 * NP <= 128 ? 128
                                    : 2 * NP <= 256 ? 256 : 512;
  static_assert(NP <= 256 && 2 * NP <= 512, "TMEM / MMA N shape");
  static_assert(SMEM + 4096 <= 232448, "shared memory");
};

__device__ __forceinline__ void sts_u32(uint32_t a, uint32_t v) {
  asm volatile("st.shared.b32 [%0], %1;" :: "r"(a), "r"(v) : "memory");
}
__device__ __forceinline__ void producers_sync() {
  asm volatile("bar.sync 1, %0;" :: "n"(kAGroup) : "memory");
}

// Per-m coefficient table of the analysis: (alpha_l, c_l 2^30 / b_l).
__global__ void mixed_anal_coef_kernel(int lmax, int mmax, const long long *__restrict__ moff,
                                       const double *__restrict__ alpha,
                                       const double *__restrict__ cfac,
                                       double2 *__restrict__ out) {
  const int m = blockIdx.x;
  if (m > mmax) return;
  const long long base = moff[m];
  const int L = lmax - m + 1 + kPad;
  for (int i = threadIdx.x; i < L; i += blockDim.x) {
    const int l = m + i;
    const double b = sqrt((2.0 * l + 1.0) / (4.0 * M_PI));
    out[base + i] = make_double2(alpha[base + i], cfac[base + i] * kQ / b);
  }
}

// Reads back a pair of tiles of class sums (tiles 2f and 2f+1 of the group:
// lanes 0-15 and 16-31 of this warp's subpartition, column set f & 1) and
// adds the FP64 result to the output.  The five class sums of a column are
// combined exactly in 64-bit integers: T = sum_w D_w 2^(8(w-2)).
template <class S>
__device__ __forceinline__ void flush_pair(uint32_t tmem, int f, int ntile, int m, int lmax,
                                           long long mo, const double2 *__restrict__ cf,
                                           const double *s_fscale, const double *s_corr,
                                           double2 *__restrict__ Aout, int ncA, int comp0,
                                           int warp, int lane) {
  const int k = warp & 3;
  const uint32_t base = tmem + (uint32_t(32 * k) << 16) + uint32_t((f & 1) * S::NP);
  uint32_t v[S::NP];
#pragma unroll
  for (int q = 0; q < S::NP; q += 16) tmem_ld16(base + q, *reinterpret_cast<uint32_t(*)[16]>(v + q));
  tmem_ld_wait();
  const int t = 2 * f + (lane >> 4);
  const int l = m + t * kAM + 16 * k + (lane & 15);
  if (t >= ntile || l > lmax) return;
  // the output is sum_p mu_l phi (the scatter applies c_l): lambda was
  // quantised as c_l mu_l 2^30 / b_l, so the row factor is b_l / c_l = 2^30 / cq_l
  const double b = kQ / __ldg(cf + l).y;
  const double sg = ((l - m) & 1) ? -b : b;
  double R[S::NH];
#pragma unroll
  for (int h = 0; h < S::NH; ++h) {
    const uint32_t *d = v + h * kAClasses;
    const long long P = (long long)int(d[0]) + ((long long)int(d[1]) << 8) +
                        ((long long)int(d[2]) << 16) + ((long long)int(d[3]) << 24);
    const double Pd = __longlong_as_double(P + 0x4338000000000000LL) - 6755399441055744.0;
    R[h] = (fma(i2d_exact(d[4]), 4294967296.0, Pd) - s_corr[h]) * s_fscale[h];
  }
  double2 *out = Aout + (mo + l) * ncA + comp0;
#pragma unroll
  for (int j = 0; j < S::NB; ++j) {
    double2 o = out[j];
    o.x += b * R[2 * j] + sg * R[S::NCOL + 2 * j];
    o.y += b * R[2 * j + 1] + sg * R[S::NCOL + 2 * j + 1];
    out[j] = o;
  }
}

template <class S>
__global__ void __launch_bounds__(kAThreads, 1)
mixed_anal_kernel(const int *__restrict__ count, const double *__restrict__ cth,
                  const double *__restrict__ sth, const int *__restrict__ nph_ring,
                  const long long *__restrict__ moff, const double2 *__restrict__ coef,
                  const double *__restrict__ mfac, const double2 *__restrict__ phase, int ncm,
                  int pcomp0, int lmax, int ms, double2 *__restrict__ Aout, int ncA, int comp0,
                  int *__restrict__ err) {
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ uint64_t full_a[2], done[2], cfull[2];
  __shared__ uint32_t tslot;
  __shared__ double s_red[kAW][S::NH];
  __shared__ long long s_psum[kAW][S::NH];
  __shared__ double s_amax[S::NH], s_fscale[S::NH], s_corr[S::NH];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m = blockIdx.x;
  const int cnt = count[m];
  const long long mo = moff[m] - m;
  const int ntile = (lmax - m + kAM) / kAM;
  const int ngroup = (cnt + kAGroup - 1) / kAGroup;
  const int njobs = ngroup * ntile;
  unsigned char *sA = sm;
  unsigned char *sB = sm + 2 * kAW * kASlice;
  unsigned char *sC = sB + S::BBYTES;
  const uint32_t sA32 = smem_u32(sA), sB32 = smem_u32(sB), sC32 = smem_u32(sC);
  const double2 *cf = coef + mo;   // cf[l]: (alpha_l, cq_l)

  if (tid == 0) {
    for (int i = 0; i < 2; ++i) {
      mbar_init(&full_a[i], kAW);
      mbar_init(&done[i], 1);
      mbar_init(&cfull[i], 1);
    }
    fence_mbar_init();
  }
  if (warp == 0) {
    tmem_alloc(&tslot, S::NCOLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tslot;

  if (warp == kAW) {
    // ------- coefficient loader and MMA issuer (lane 0 issues) -------
    auto load_coef = [&](int j) {
      const int l0 = m + (j % ntile) * kAM;
      mbar_arrive_tx(&cfull[j & 1], kACoef);
      bulk_g2s(sC + (j & 1) * kACoef, cf + l0, kACoef, &cfull[j & 1]);
    };
    if (lane == 0)
      for (int j = 0; j < 2 && j < njobs; ++j) load_coef(j);
    __syncwarp();
    constexpr uint32_t idesc = make_idesc_i8(kAM, S::NP);
    const uint64_t b0 = make_desc(sB32, S::BLBO, 128);
    bool ok = true;
    int issued = -1;
    for (int J = 0; J < njobs; ++J) {
      const int st = J & 1;
      if (!__all_sync(0xffffffffu, mbar_wait(&full_a[st], (J >> 1) & 1))) {
        ok = false;
        break;
      }
      tc_fence_after();
      if (lane == 0) {
        // the producers are done with this job's coefficients
        if (J + 2 < njobs) load_coef(J + 2);
        const int t = J % ntile;
        const uint32_t d = tmem + (uint32_t(16 * (t & 1)) << 16) + uint32_t(((t >> 1) & 1) * S::NP);
        const uint64_t a0 = make_desc(sA32 + st * kAW * kASlice, kALBO, 128);
        // the start-address field (bits 0-13, 16-byte units) is advanced per K-step
#pragma unroll
        for (int k = 0; k < kAKB / 32; ++k)
          mma_i8(d, a0 + uint64_t(((k / 4) * kASlice + (k % 4) * 2 * kALBO) >> 4),
                 b0 + uint64_t((2 * k * S::BLBO) >> 4), idesc, k > 0 ? 1u : 0u);
        mma_commit(&done[st]);
      }
      __syncwarp();
      issued = J;
    }
    if (!ok) {
      if (lane == 0) *reinterpret_cast<volatile int *>(err) = 1;
      if (issued >= 0) mbar_wait(&done[issued & 1], (issued >> 1) & 1);
    }
  } else {
    // ---------------- producers: one ring pair per thread ----------------
    // All producer warps run the same loops (named barriers inside); a wait
    // that gives up clears ok, after which the warp skips waits and reads of
    // TMEM but keeps its place in the barriers.
    bool ok = true;
    const uint32_t bcol = (tid >> 2) * S::BLBO + 4 * (tid & 3);   // this pair's K column of B
    for (int r = S::NPR; r < S::NP; ++r)                           // unused B rows stay zero
      sts_u32(sB32 + (r >> 3) * 128 + (r & 7) * 16 + bcol, 0u);
    const double sgn_mfac = (m & 1) ? -mfac[m] : mfac[m];
    int J = 0;
    for (int g = 0; g < ngroup; ++g) {
      const int p = g * kAGroup + tid;
      const bool valid = p < cnt;
      const bool has_s = valid && nph_ring[2 * p + 1] > 0;
      // ring phases of this pair: (north, south) x (transform, re/im)
      double ph[S::NH];
#pragma unroll
      for (int j = 0; j < S::NB; ++j) {
        const long long row = ((long long)(valid ? p : 0) * ncm + pcomp0 + j) * 2 * ms;
        const double2 n = valid ? phase[row + m] : make_double2(0.0, 0.0);
        const double2 s = has_s ? phase[row + ms + m] : make_double2(0.0, 0.0);
        ph[2 * j] = n.x;
        ph[2 * j + 1] = n.y;
        ph[S::NCOL + 2 * j] = s.x;
        ph[S::NCOL + 2 * j + 1] = s.y;
      }
      // group maxima per (half, column)
#pragma unroll
      for (int i = 0; i < S::NH; ++i) {
        double a = fabs(ph[i]);
#pragma unroll
        for (int o = 16; o; o >>= 1) a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
        if (lane == 0) s_red[warp][i] = a;
      }
      producers_sync();
      if (tid < S::NH) {
        double a = 0.0;
        for (int w = 0; w < kAW; ++w) a = fmax(a, s_red[w][tid]);
        s_amax[tid] = a;
      }
      producers_sync();
      // quantise, write this pair's K column of the Toeplitz B tile
#pragma unroll
      for (int i = 0; i < S::NH; ++i) {
        const double amax = s_amax[i];
        const int q = amax > 0.0 ? static_cast<int>(llrint(ph[i] * (kQ / amax))) : 0;
        int d[4], r = q;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          d[k] = ((r + 128) & 255) - 128;
          r = (r - d[k]) >> 8;
        }
        d[3] = r;
#pragma unroll
        for (int w = 2; w <= 6; ++w) {
          uint32_t word = 0;
#pragma unroll
          for (int k = 0; k < 4; ++k)
            if (w - k >= 0 && w - k <= 3) word |= uint32_t(uint8_t(int8_t(d[w - k]))) << (8 * k);
          const int row = i * kAClasses + (w - 2);
          sts_u32(sB32 + (row >> 3) * 128 + (row & 7) * 16 + bcol, word);
        }
        long long ps = q;
#pragma unroll
        for (int o = 16; o; o >>= 1) ps += __shfl_xor_sync(0xffffffffu, ps, o);
        if (lane == 0) s_psum[warp][i] = ps;
      }
      producers_sync();
      if (tid < S::NH) {
        long long ps = 0;
        for (int w = 0; w < kAW; ++w) ps += s_psum[w][tid];
        // flush units: T = S / 2^16, so the offset correction is 2^15 sum q and
        // the scale amax / 2^44
        s_corr[tid] = 32768.0 * double(ps);
        s_fscale[tid] = s_amax[tid] * 0x1p-44;
      }
      producers_sync();

      // recurrence seed of this pair
      const double x = valid ? cth[p] : 0.0;
      double mu0 = 0.0, mu1;
      int E;
      bool act, live;
      {
        XD sd = valid ? xd_pow(sth[p], m) : XD{0.0, 0};
        sd = xd_norm(sd.v * sgn_mfac, sd.e);
        mu1 = sd.v;
        E = sd.e;
        live = valid && sd.v != 0.0;
        act = live && E >= -kSwitchExp;
        if (act) mu1 = ldexp(mu1, E);
      }
      int fnext = 0;   // next tile pair of this group to read back
      for (int t = 0; t < ntile; ++t, ++J) {
        const int st = J & 1;
        if (ok) {
          // A stage of job J-2 is reused; this job's coefficients are staged
          bool w = J < 2 || mbar_wait(&done[st], ((J >> 1) - 1) & 1);
          w = w && mbar_wait(&cfull[st], (J >> 1) & 1);
          ok = __all_sync(0xffffffffu, w);
          // tiles t-3, t-2 are complete once done(J-2) has been seen
          if (ok && (t & 1) && t >= 3) {
            if ((warp >> 2) == (fnext & 1)) {
              tc_fence_after();
              flush_pair<S>(tmem, fnext, ntile, m, lmax, mo, cf, s_fscale, s_corr, Aout, ncA,
                            comp0, warp, lane);
            }
            ++fnext;
          }
        }
        const uint32_t slice = sA32 + (st * kAW + warp) * kASlice + (lane >> 2) * kALBO +
                               4 * (lane & 3);
        const uint32_t cs = sC32 + st * kACoef;
        const int l0 = m + t * kAM;
#pragma unroll 1
        for (int blk = 0; blk < kAM / 16; ++blk) {
          const int lb = l0 + 16 * blk;
          if (lb > lmax) {
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              const int r = 16 * blk + i;
              sts_u32(slice + (r >> 3) * 128 + (r & 7) * 16, 0x80000000u);
            }
            continue;
          }
          double2 c[16];
#pragma unroll
          for (int i = 0; i < 16; ++i) c[i] = lds_f64x2(cs + (16 * blk + i) * 16);
          const bool all = __all_sync(0xffffffffu, act);
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const double cq = (all || act) ? c[i].y : 0.0;
            const int r = 16 * blk + i;
            sts_u32(slice + (r >> 3) * 128 + (r & 7) * 16, quant(mu1, cq));
            const double nx = fma(c[i].x * x, mu1, -mu0);
            mu0 = mu1;
            mu1 = nx;
          }
          // every 16 l-steps: bookkeeping of pairs still in the scaled regime
          if (live && !act) {
            live = renorm_pair(mu1, mu0, E);
            if (live && E >= -kSwitchExp) {
              mu1 = ldexp(mu1, E);
              mu0 = ldexp(mu0, E);
              act = true;
            }
          }
        }
        fence_async_smem();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&full_a[st]);
      }
      // end of the group: read back the pairs still in TMEM
      if (ok) ok = __all_sync(0xffffffffu, mbar_wait(&done[(J - 1) & 1], ((J - 1) >> 1) & 1));
      for (; 2 * fnext < ntile; ++fnext)
        if (ok && (warp >> 2) == (fnext & 1)) {
          tc_fence_after();
          flush_pair<S>(tmem, fnext, ntile, m, lmax, mo, cf, s_fscale, s_corr, Aout, ncA, comp0,
                        warp, lane);
        }
      // B, the scales and the TMEM columns are reused by the next group
      tc_fence_before();
      producers_sync();
      tc_fence_after();
    }
    if (!ok && lane == 0) *reinterpret_cast<volatile int *>(err) = 1;
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, S::NCOLS);
  }
}

template <class S>
void launch_anal_shape(const JobDesc &job, const GeomPlan &gp, const CoefPlan &cp,
                       const double2 *phase, int ncm, int t0, double2 *Aout, int ncA,
                       int *d_err, cudaStream_t st) {
  ProfScope ps("legendre_anal", st);
  auto k = mixed_anal_kernel<S>;
  SHT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, S::SMEM));
  k<<<job.mmax + 1, kAThreads, S::SMEM, st>>>(gp.count, gp.cth, gp.sth, gp.nph, cp.d_moff,
                                              cp.mx_coef, cp.seed, phase, ncm, t0, job.lmax,
                                              job.mmax + 1, Aout, ncA, t0, d_err);
  SHT_CUDA(cudaGetLastError());
}

}  // namespace

bool mixed_anal_supported(const JobDesc &job) {
  return job.type == SHARP_MAP2ALM && job.spin == 0 && job.ntrans >= 1;
}

void launch_mixed_anal(const JobDesc &job, const GeomPlan &gp, CoefPlan &cp,
                       const double2 *phase, int ncm, double2 *Aout, int ncA, int *d_err,
                       cudaStream_t st) {
  if (!cp.mx_coef) {
    // a tile's coefficients are copied whole: kAM entries of slack at the end
    const size_t n = size_t(cp.total) + kAM;
    SHT_CUDA(cudaMallocAsync(&cp.mx_coef, sizeof(double2) * n, st));
    SHT_CUDA(cudaMemsetAsync(cp.mx_coef, 0, sizeof(double2) * n, st));
    mixed_anal_coef_kernel<<<cp.mmax + 1, 256, 0, st>>>(cp.lmax, cp.mmax, cp.d_moff, cp.alpha,
                                                        cp.cfac, cp.mx_coef);
    SHT_CUDA(cudaGetLastError());
  }
  for (int t0 = 0; t0 < job.ntrans;) {
    const int nb = std::min(job.ntrans - t0, 4);
    switch (nb) {
      case 4: launch_anal_shape<AShape<4>>(job, gp, cp, phase, ncm, t0, Aout, ncA, d_err, st); break;
      case 3: launch_anal_shape<AShape<3>>(job, gp, cp, phase, ncm, t0, Aout, ncA, d_err, st); break;
      case 2: launch_anal_shape<AShape<2>>(job, gp, cp, phase, ncm, t0, Aout, ncA, d_err, st); break;
      default: launch_anal_shape<AShape<1>>(job, gp, cp, phase, ncm, t0, Aout, ncA, d_err, st); break;
    }
    t0 += nb;
  }
}

}  // namespace sht
