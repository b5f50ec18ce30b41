// Mixed-precision batched analysis (map2alm Legendre step) on the
// 5th-generation tensor cores, spin 0 and spin s > 0.
//
// For NB transforms sharing geometry and lmax the analysis of order m is, per
// output column (transform, component, re/im),
//   spin 0:  A_l = sum_p lambda_l(p) N_p + (-1)^(l-m) sum_p lambda_l(p) S_p
//   spin s:  A_l = sum_p [mu+_l(p) Hn+_p + mu-_l(p) Hn-_p]
//                + (-1)^(l-mhi) sum_p [mu+_l(p) Hs+_p + mu-_l(p) Hs-_p]
// with N/S the north/south ring phases (weights applied) and, for spin, Hn/Hs
// the north/south parts of the combined Q/U phase factors of the two
// Wigner-d recurrences (the even/odd factors of the FP64 kernel are
// Hn +- Hs).  As in the synthesis, the FP64 recurrence stays on the CUDA
// cores and the contraction runs exactly in integers on tcgen05.mma.kind::i8,
// here with the roles of the operands turned around:
//
//  * A (M = 64 consecutive l, K = (ring pair, value, byte)): the words
//    u_l(p) = 2^31 + round(lambda_l(p) 2^30 / b_l) with the analytic bound
//    b_l (sqrt((2l+1)/4pi) at spin 0; 1 for each of d^l_{m,+-s}), one
//    magic-constant DFMA each; a producer thread owns one ring pair and
//    writes one (spin: two) 4-byte words per l.
//  * B (N = (half, column, weight), K as A): the Toeplitz expansion of the
//    signed base-256 digits of the phase factors, quantised per group of ring
//    pairs and (half, column) against the group's maximum.  It is built once
//    per group in shared memory and stays there while the group sweeps all l.
//  * D (int32, TMEM): per l-tile the exact class sums over the group's ring
//    pairs.  Two tiles share one TMEM column set (lanes 0-15 and 16-31 of
//    each subpartition), two sets alternate; a pair is read back one lane per
//    l, its class sums combined exactly in 64-bit integers, corrected for the
//    2^31 offset and scaled in FP64, and added to the output (one CTA per m,
//    so no atomics).
//    Like the FP64 kernels, the output holds sums of the rescaled recurrence
//    values mu_l = lambda_l / c_l; c_l is applied when the a_lm are scattered.
//
// Warp roles: spin 0: 8 producer warps (256 ring pairs per group); spin s:
// 4 producer warps (128 ring pairs, two recurrences each).  Four flusher
// warps (one per TMEM subpartition) read the class sums back and update the
// output while the producers run the next tiles.  The last warp (lane 0)
// stages each l-tile's recurrence coefficients into shared memory
// (cp.async.bulk) and issues its MMAs.  Every wait is bounded; a timeout is
// reported through the error word.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "sht_device.h"
#include "sht_recurrence.cuh"
#include "sht_tc.cuh"

namespace sht {

namespace {

constexpr int kAM = 64;                       // l rows per tile (MMA M)
constexpr int kAClasses = 5;                  // byte-product weights 2^16 .. 2^48
// A slice of one warp and tile (64 l x the warp's ring pairs, K-major, no
// swizzle): the 8-row groups are contiguous (SBO = 128) and the K core
// matrices lie kALBO = 8*128 + 16 bytes apart, so the per-l stores of a warp
// spread over all 32 banks.
constexpr int kALBO = (kAM / 8) * 128 + 16;

constexpr int ceil16(int x) { return (x + 15) / 16 * 16; }

template <bool SPIN_, int NB_>
struct AShape {
  static constexpr bool SPIN = SPIN_;
  static constexpr int NB = NB_;
  static constexpr int TY = SPIN ? 2 : 1;              // recurrence values per pair and l
  static constexpr int PW = SPIN ? 4 : 8;              // producer warps
  static constexpr int G = 32 * PW;                    // ring pairs per group
  static constexpr int FW = 4;                         // flusher warps (one per TMEM subpartition)
  static constexpr int THREADS = 32 * (PW + FW + 1);
  static constexpr int KB = 4 * TY * G;                // K bytes of a group
  static constexpr int KCM = 8 * TY;                   // K core matrices per warp slice
  static constexpr int SLICE = (KCM - 1) * kALBO + (kAM / 8) * 128;
  static constexpr int CE = SPIN ? 32 : 16;            // coefficient bytes per l
  static constexpr int COEF = kAM * CE;                // one tile's coefficients
  static constexpr int OUT = SPIN ? 4 : 2;             // real outputs per transform
  static constexpr int NCOL = OUT * NB;
  static constexpr int NH = 2 * NCOL;                  // (half, column): north, then south
  static constexpr int NPR = kAClasses * NH;           // B rows used
  static constexpr int NP = ceil16(NPR);               // MMA N
  // B (NP x KB): row groups contiguous, K core matrices BLBO apart
  static constexpr int BLBO = (NP / 8) * 128 + 16;
  static constexpr int BBYTES = ((KB / 16 - 1) * BLBO + (NP / 8) * 128 + 127) / 128 * 128;
  static constexpr int SMEM = 2 * PW * SLICE + BBYTES + 2 * COEF;
  // TMEM: a pair of tiles shares one column set (lane halves); two sets
  static constexpr uint32_t NCOLS = 2 * NP <= 32 ? 32 : 2 * NP <= 64 ? 64 : 2 * NP <= 128 ? 128
                                    : 2 * NP <= 256 ? 256 : 512;
  static_assert(KB == 1024, "K extent of a group");
  static_assert(NP <= 256 && 2 * NP <= 512, "TMEM / MMA N shape");
  static_assert(SMEM + 4096 <= 232448, "shared memory");
};

__device__ __forceinline__ void sts_u32(uint32_t a, uint32_t v) {
  asm volatile("st.shared.b32 [%0], %1;" :: "r"(a), "r"(v) : "memory");
}
__device__ __forceinline__ void sts_u32x2(uint32_t a, uint32_t x, uint32_t y) {
  asm volatile("st.shared.v2.b32 [%0], {%1, %2};" :: "r"(a), "r"(x), "r"(y) : "memory");
}
template <int N>
__device__ __forceinline__ void producers_sync() {
  asm volatile("bar.sync 1, %0;" :: "n"(N) : "memory");
}

// Per-m coefficient table of the analysis, for l = m .. lmax + kPad:
// spin 0: (alpha_l, c_l 2^30 / b_l); spin s: (a_l, b_l), (c_l 2^30, 0).
__global__ void mixed_anal_coef_kernel(int lmax, int mmax, int spin,
                                       const long long *__restrict__ moff,
                                       const double *__restrict__ ca,
                                       const double *__restrict__ cb,
                                       const double *__restrict__ cfac,
                                       double2 *__restrict__ out) {
  const int m = blockIdx.x;
  if (m > mmax) return;
  const long long base = moff[m];
  const int L = lmax - m + 1 + kPad;
  for (int i = threadIdx.x; i < L; i += blockDim.x) {
    const int l = m + i;
    if (spin == 0) {
      const double b = sqrt((2.0 * l + 1.0) / (4.0 * M_PI));
      out[base + i] = make_double2(ca[base + i], cfac[base + i] * kQ / b);
    } else {
      out[2 * (base + i)] = make_double2(ca[base + i], cb[base + i]);
      out[2 * (base + i) + 1] = make_double2(cfac[base + i] * kQ, 0.0);
    }
  }
}

// Reads back a pair of tiles of class sums (tiles 2f and 2f+1 of the group:
// lanes 0-15 and 16-31 of this warp's subpartition, TMEM column set `set`)
// and adds the FP64 result to the output.  The five class sums of a column
// are combined exactly in 64-bit integers: T = sum_w D_w 2^(8(w-2)).
template <class S>
__device__ __forceinline__ void flush_pair(uint32_t tmem, int set, int f, int ntile, int l0,
                                           int lmax, long long mo,
                                           const double2 *__restrict__ coef,
                                           const double *s_fscale, const double *s_corr,
                                           double2 *__restrict__ Aout, int ncA, int comp0,
                                           int warp, int lane) {
  const int k = warp & 3;
  const uint32_t base = tmem + (uint32_t(32 * k) << 16) + uint32_t(set * S::NP);
  const int t = 2 * f + (lane >> 4);
  const int l = l0 + t * kAM + 16 * k + (lane & 15);
  const bool row = t < ntile && l <= lmax;
  // the output entries and the row factor are fetched before the TMEM reads
  double2 *out = Aout + (mo + (row ? l : l0)) * ncA + comp0;
  double2 o[S::NCOL / 2];
#pragma unroll
  for (int j = 0; j < S::NCOL / 2; ++j) o[j] = row ? out[j] : make_double2(0.0, 0.0);
  const double cq = !row ? 1.0 : S::SPIN ? __ldg(coef + 2 * (mo + l) + 1).x
                                         : __ldg(coef + mo + l).y;
  uint32_t v[S::NP];
#pragma unroll
  for (int q = 0; q < S::NP; q += 16) tmem_ld16(base + q, *reinterpret_cast<uint32_t(*)[16]>(v + q));
  tmem_ld_wait();
  if (!row) return;
  // the output is sum_p mu_l phi (the scatter applies c_l): lambda was
  // quantised as c_l mu_l 2^30 / b_l, so the row factor is b_l / c_l = 2^30 / cq_l
  const double b = kQ / cq;
  const double sg = ((l - l0) & 1) ? -b : b;
  double R[S::NH];
#pragma unroll
  for (int h = 0; h < S::NH; ++h) {
    const uint32_t *d = v + h * kAClasses;
    const long long P = (long long)int(d[0]) + ((long long)int(d[1]) << 8) +
                        ((long long)int(d[2]) << 16) + ((long long)int(d[3]) << 24);
    const double Pd = __longlong_as_double(P + 0x4338000000000000LL) - 6755399441055744.0;
    R[h] = (fma(i2d_exact(d[4]), 4294967296.0, Pd) - s_corr[h]) * s_fscale[h];
  }
#pragma unroll
  for (int j = 0; j < S::NCOL / 2; ++j) {
    o[j].x += b * R[2 * j] + sg * R[S::NCOL + 2 * j];
    o[j].y += b * R[2 * j + 1] + sg * R[S::NCOL + 2 * j + 1];
    out[j] = o[j];
  }
}

// Jobs run group-major (group g of ring pairs, l-tile t); tiles 2f, 2f+1 of a
// group form pair P = g * npg + f (npg pairs per group), whose class sums
// live in TMEM column set P mod 2.
//
// Barriers (all waits bounded):
//   full_a[st]  producers -> issuer: A stage st holds job J's words
//   done[st]    issuer -> producers: job J's MMAs are complete (A stage and,
//               after a group's last job, B may be rewritten)
//   cfull[st]   bulk copy -> producers: job J's coefficients are staged
//   dfull[set]  issuer -> flushers: pair P's class sums are complete
//   dfree[set]  flushers -> issuer: pair P has been read back
//   sfull[sl]   producers -> flushers: the scales of group g (slot g mod 2)
//   sfree[sl]   flushers -> producers: group g has been read back
template <class S>
__global__ void __launch_bounds__(S::THREADS, 1)
mixed_anal_kernel(const int *__restrict__ count, const double *__restrict__ cth,
                  const double *__restrict__ sth, const int *__restrict__ nph_ring,
                  const long long *__restrict__ moff, const double2 *__restrict__ coef,
                  const double *__restrict__ pre_v, const int *__restrict__ pre_e, int spin,
                  const double2 *__restrict__ phase, int ncm, int pcomp0, int lmax, int ms,
                  double2 *__restrict__ Aout, int ncA, int comp0, int *__restrict__ err) {
  constexpr int PW = S::PW;
  constexpr int FW = S::FW;                  // flusher warps PW .. PW+3
  constexpr int LW = PW + FW;                // coefficient loader and MMA issuer
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ uint64_t full_a[2], done[2], cfull[2], dfull[2], dfree[2], sfull[2], sfree[2];
  __shared__ uint32_t tslot;
  __shared__ double s_red[PW][S::NH];
  __shared__ long long s_psum[PW][S::NH];
  __shared__ double s_amax[S::NH], s_fscale[2][S::NH], s_corr[2][S::NH];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m = blockIdx.x;
  const int mhi = max(m, spin);
  const int cnt = count[m];
  const long long mo = moff[m] - m;
  const int ntile = mhi <= lmax ? (lmax - mhi + kAM) / kAM : 0;
  const int npg = (ntile + 1) / 2;
  const int ngroup = (cnt + S::G - 1) / S::G;
  const int njobs = ngroup * ntile;
  unsigned char *sA = sm;
  unsigned char *sB = sm + 2 * PW * S::SLICE;
  unsigned char *sC = sB + S::BBYTES;
  const uint32_t sA32 = smem_u32(sA), sB32 = smem_u32(sB), sC32 = smem_u32(sC);
  constexpr int CW = S::CE / 16;                       // double2 entries per l
  const double2 *cf = coef + CW * mo;                  // cf[CW l]: coefficients of l

  if (tid == 0) {
    for (int i = 0; i < 2; ++i) {
      mbar_init(&full_a[i], PW);
      mbar_init(&done[i], 1);
      mbar_init(&cfull[i], 1);
      mbar_init(&dfull[i], 1);
      mbar_init(&dfree[i], FW);
      mbar_init(&sfull[i], 1);
      mbar_init(&sfree[i], FW);
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

  if (warp == LW) {
    // ------- coefficient loader and MMA issuer (lane 0 issues) -------
    auto load_coef = [&](int j) {
      const int l0 = mhi + (j % ntile) * kAM;
      mbar_arrive_tx(&cfull[j & 1], S::COEF);
      bulk_g2s(sC + (j & 1) * S::COEF, cf + CW * l0, S::COEF, &cfull[j & 1]);
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
      const int g = J / ntile, t = J - g * ntile;
      const int P = g * npg + (t >> 1), set = P & 1;
      bool w = mbar_wait(&full_a[st], (J >> 1) & 1);
      // the pair's column set is free once pair P-2 has been read back
      if ((t & 1) == 0 && P >= 2) w = w && mbar_wait(&dfree[set], ((P >> 1) - 1) & 1);
      if (!__all_sync(0xffffffffu, w)) {
        ok = false;
        break;
      }
      tc_fence_after();
      if (lane == 0) {
        // the producers are done with this job's coefficients
        if (J + 2 < njobs) load_coef(J + 2);
        const uint32_t d = tmem + (uint32_t(16 * (t & 1)) << 16) + uint32_t(set * S::NP);
        const uint64_t a0 = make_desc(sA32 + st * PW * S::SLICE, kALBO, 128);
        // K-step k covers bytes [32k, 32k+32): warp slice k / (4 TY), core
        // matrices 2 (k mod 4 TY) and the next; the start-address field (bits
        // 0-13, 16-byte units) is advanced per K-step
#pragma unroll
        for (int k = 0; k < S::KB / 32; ++k)
          mma_i8(d,
                 a0 + uint64_t(((k / (4 * S::TY)) * S::SLICE + (k % (4 * S::TY)) * 2 * kALBO) >> 4),
                 b0 + uint64_t((2 * k * S::BLBO) >> 4), idesc, k > 0 ? 1u : 0u);
        mma_commit(&done[st]);
        if ((t & 1) || t == ntile - 1) mma_commit(&dfull[set]);
      }
      __syncwarp();
      issued = J;
    }
    if (!ok) {
      if (lane == 0) *reinterpret_cast<volatile int *>(err) = 1;
      if (issued >= 0) mbar_wait(&done[issued & 1], (issued >> 1) & 1);
    }
  } else if (warp >= PW) {
    // ---- flushers: warp PW + k reads lanes 32k .. 32k+31 of every pair ----
    bool ok = true;
    for (int g = 0; g < ngroup; ++g) {
      const int sl = g & 1;
      if (ok) ok = __all_sync(0xffffffffu, mbar_wait(&sfull[sl], (g >> 1) & 1));
      for (int f = 0; f < npg; ++f) {
        const int P = g * npg + f;
        if (ok) ok = __all_sync(0xffffffffu, mbar_wait(&dfull[P & 1], (P >> 1) & 1));
        if (ok) {
          tc_fence_after();
          flush_pair<S>(tmem, P & 1, f, ntile, mhi, lmax, mo, coef, s_fscale[sl], s_corr[sl],
                        Aout, ncA, comp0, warp, lane);
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&dfree[P & 1]);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&sfree[sl]);
    }
    if (!ok && lane == 0) *reinterpret_cast<volatile int *>(err) = 1;
  } else {
    // ---------------- producers: one ring pair per thread ----------------
    // All producer warps run the same loops (named barriers inside); a wait
    // that gives up clears ok, after which the warp skips waits but keeps
    // its place in the barriers.
    bool ok = true;
    // this pair's K segment of B: 4 TY bytes
    const uint32_t bcol = ((tid * 4 * S::TY) >> 4) * S::BLBO + ((tid * 4 * S::TY) & 15);
    for (int r = S::NPR; r < S::NP; ++r) {  // unused B rows stay zero
      const uint32_t a = sB32 + (r >> 3) * 128 + (r & 7) * 16 + bcol;
      if constexpr (S::SPIN) sts_u32x2(a, 0u, 0u); else sts_u32(a, 0u);
    }
    const double flip = ((mhi - m + spin) & 1) ? -1.0 : 1.0;
    const double sgn_mfac = (m & 1) ? -pre_v[m] : pre_v[m];
    int J = 0;
    for (int g = 0; g < ngroup; ++g) {
      const int sl = g & 1;
      const int p = g * S::G + tid;
      const bool valid = p < cnt;
      const bool has_s = valid && nph_ring[2 * p + 1] > 0;
      // phase factors of this pair: val[type][half * NCOL + column]
      double val[S::TY][S::NH];
#pragma unroll
      for (int j = 0; j < S::NB; ++j) {
        if constexpr (!S::SPIN) {
          const long long row = ((long long)(valid ? p : 0) * ncm + pcomp0 + j) * 2 * ms;
          const double2 n = valid ? phase[row + m] : make_double2(0.0, 0.0);
          const double2 s = has_s ? phase[row + ms + m] : make_double2(0.0, 0.0);
          val[0][2 * j] = n.x;
          val[0][2 * j + 1] = n.y;
          val[0][S::NCOL + 2 * j] = s.x;
          val[0][S::NCOL + 2 * j + 1] = s.y;
        } else {
          const long long rq = ((long long)(valid ? p : 0) * ncm + pcomp0 + 2 * j) * 2 * ms;
          const long long ru = ((long long)(valid ? p : 0) * ncm + pcomp0 + 2 * j + 1) * 2 * ms;
          const double2 qn = valid ? phase[rq + m] : make_double2(0.0, 0.0);
          const double2 un = valid ? phase[ru + m] : make_double2(0.0, 0.0);
          double2 qs = has_s ? phase[rq + ms + m] : make_double2(0.0, 0.0);
          double2 us = has_s ? phase[ru + ms + m] : make_double2(0.0, 0.0);
          qs.x *= flip; qs.y *= flip; us.x *= flip; us.y *= flip;
          // outputs (G.re, G.im, C.re, C.im); type 0: mu+, type 1: mu-
          double *np_ = &val[0][4 * j], *nm_ = &val[1][4 * j];
          double *sp_ = &val[0][S::NCOL + 4 * j], *sm_ = &val[1][S::NCOL + 4 * j];
          np_[0] = qn.x + un.y; nm_[0] = qn.x - un.y; sp_[0] = qs.x - us.y; sm_[0] = qs.x + us.y;
          np_[1] = qn.y - un.x; nm_[1] = qn.y + un.x; sp_[1] = qs.y + us.x; sm_[1] = qs.y - us.x;
          np_[2] = un.x - qn.y; nm_[2] = un.x + qn.y; sp_[2] = us.x + qs.y; sm_[2] = us.x - qs.y;
          np_[3] = un.y + qn.x; nm_[3] = un.y - qn.x; sp_[3] = us.y - qs.x; sm_[3] = us.y + qs.x;
        }
      }
      // group maxima per (half, column) over pairs and values
#pragma unroll
      for (int i = 0; i < S::NH; ++i) {
        double a = fabs(val[0][i]);
        if constexpr (S::SPIN) a = fmax(a, fabs(val[S::TY - 1][i]));
#pragma unroll
        for (int o = 16; o; o >>= 1) a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
        if (lane == 0) s_red[warp][i] = a;
      }
      producers_sync<S::G>();
      if (tid < S::NH) {
        double a = 0.0;
        for (int w = 0; w < PW; ++w) a = fmax(a, s_red[w][tid]);
        s_amax[tid] = a;
      }
      producers_sync<S::G>();
      // quantise, write this pair's K segment of the Toeplitz B tile (the
      // MMAs of the previous group are complete: its last done was seen)
#pragma unroll
      for (int i = 0; i < S::NH; ++i) {
        const double amax = s_amax[i];
        uint32_t word[S::TY][5];
        long long ps = 0;
#pragma unroll
        for (int ty = 0; ty < S::TY; ++ty) {
          const int q = amax > 0.0 ? static_cast<int>(llrint(val[ty][i] * (kQ / amax))) : 0;
          ps += q;
          int d[4], r = q;
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            d[k] = ((r + 128) & 255) - 128;
            r = (r - d[k]) >> 8;
          }
          d[3] = r;
#pragma unroll
          for (int w = 2; w <= 6; ++w) {
            uint32_t wd = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k)
              if (w - k >= 0 && w - k <= 3) wd |= uint32_t(uint8_t(int8_t(d[w - k]))) << (8 * k);
            word[ty][w - 2] = wd;
          }
        }
#pragma unroll
        for (int w = 0; w < 5; ++w) {
          const int row = i * kAClasses + w;
          const uint32_t a = sB32 + (row >> 3) * 128 + (row & 7) * 16 + bcol;
          if constexpr (S::SPIN) sts_u32x2(a, word[0][w], word[S::TY - 1][w]);
          else sts_u32(a, word[0][w]);
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) ps += __shfl_xor_sync(0xffffffffu, ps, o);
        if (lane == 0) s_psum[warp][i] = ps;
      }
      // the scale slot of group g-2 is free once its pairs have been read back
      if (g >= 2 && ok) ok = __all_sync(0xffffffffu, mbar_wait(&sfree[sl], ((g >> 1) - 1) & 1));
      producers_sync<S::G>();
      if (tid < S::NH) {
        long long ps = 0;
        for (int w = 0; w < PW; ++w) ps += s_psum[w][tid];
        // flush units: T = S / 2^16, so the offset correction is 2^15 sum q and
        // the scale amax / 2^44
        s_corr[sl][tid] = 32768.0 * double(ps);
        s_fscale[sl][tid] = s_amax[tid] * 0x1p-44;
      }
      producers_sync<S::G>();
      if (tid == 0) mbar_arrive(&sfull[sl]);

      // recurrence seed(s) of this pair
      const double x = valid ? cth[p] : 0.0;
      double mu0 = 0.0, mu1 = 0.0, mm0 = 0.0, mm1 = 0.0;
      int E = 0, Em = 0;
      bool act, live;
      if constexpr (!S::SPIN) {
        const XD sd = valid ? xd_pow_log(sth[p], m, sgn_mfac) : XD{0.0, 0};
        mu1 = sd.v;
        E = sd.e;
        live = valid && sd.v != 0.0;
        act = live && E >= -kSwitchExp;
        if (act) mu1 = ldexp(mu1, E);
      } else {
        live = spin_start_log(valid, x, valid ? sth[p] : 0.0, m, spin, pre_v[m], pre_e[m], mu0,
                              mu1, mm0, mm1, E, Em, act);
      }
      for (int t = 0; t < ntile; ++t, ++J) {
        const int st = J & 1;
        if (ok) {
          // A stage of job J-2 is reused; this job's coefficients are staged
          bool w = J < 2 || mbar_wait(&done[st], ((J >> 1) - 1) & 1);
          w = w && mbar_wait(&cfull[st], (J >> 1) & 1);
          ok = __all_sync(0xffffffffu, w);
        }
        const uint32_t slice = sA32 + (st * PW + warp) * S::SLICE +
                               (S::SPIN ? (lane >> 1) * kALBO + 8 * (lane & 1)
                                        : (lane >> 2) * kALBO + 4 * (lane & 3));
        const uint32_t cs = sC32 + st * S::COEF;
        const int l0 = mhi + t * kAM;
#pragma unroll 1
        for (int blk = 0; blk < kAM / 16; ++blk) {
          const int lb = l0 + 16 * blk;
          if (lb > lmax) {
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              const int r = 16 * blk + i;
              const uint32_t a = slice + (r >> 3) * 128 + (r & 7) * 16;
              if constexpr (S::SPIN) sts_u32x2(a, 0x80000000u, 0x80000000u);
              else sts_u32(a, 0x80000000u);
            }
            continue;
          }
          const bool all = __all_sync(0xffffffffu, act);
          if constexpr (!S::SPIN) {
            double2 c[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) c[i] = lds_f64x2(cs + (16 * blk + i) * 16);
            uint32_t u[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              const double cq = (all || act) ? c[i].y : 0.0;
              u[i] = quant(mu1, cq);
              const double nx = fma(c[i].x * x, mu1, -mu0);
              mu0 = mu1;
              mu1 = nx;
            }
            // stores after the steps: no store waits on its quantisation
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              const int r = 16 * blk + i;
              sts_u32(slice + (r >> 3) * 128 + (r & 7) * 16, u[i]);
            }
          } else {
#pragma unroll
            for (int h8 = 0; h8 < 2; ++h8) {
              double2 ab[8];
              double cq[8];
#pragma unroll
              for (int i = 0; i < 8; ++i) {
                const int li = 16 * blk + 8 * h8 + i;
                ab[i] = lds_f64x2(cs + li * 32);
                cq[i] = lds_f64x2(cs + li * 32 + 16).x;
              }
              uint32_t up[8], um[8];
#pragma unroll
              for (int i = 0; i < 8; ++i) {
                const double q = (all || act) ? cq[i] : 0.0;
                up[i] = quant(mu1, q);
                um[i] = quant(mm1, q);
                const double np_ = fma(fma(ab[i].x, x, -ab[i].y), mu1, -mu0);
                const double nm_ = fma(fma(ab[i].x, x, ab[i].y), mm1, -mm0);
                mu0 = mu1;
                mu1 = np_;
                mm0 = mm1;
                mm1 = nm_;
              }
#pragma unroll
              for (int i = 0; i < 8; ++i) {
                const int r = 16 * blk + 8 * h8 + i;
                sts_u32x2(slice + (r >> 3) * 128 + (r & 7) * 16, up[i], um[i]);
              }
            }
          }
          // every 16 l-steps: bookkeeping of pairs still in the scaled regime
          if constexpr (!S::SPIN) {
            if (live && !act) {
              live = renorm_pair(mu1, mu0, E);
              if (live && E >= -kSwitchExp) {
                mu1 = ldexp(mu1, E);
                mu0 = ldexp(mu0, E);
                act = true;
              }
            }
          } else {
            spin_renorm(live, act, mu0, mu1, mm0, mm1, E, Em);
          }
        }
        fence_async_smem();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&full_a[st]);
      }
      // B is rewritten by the next group once the last MMA of this one is done
      if (ok && ntile > 0)
        ok = __all_sync(0xffffffffu, mbar_wait(&done[(J - 1) & 1], ((J - 1) >> 1) & 1));
      tc_fence_before();
      producers_sync<S::G>();
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
  ProfScope ps(S::SPIN ? "mixed_anal_spin" : "mixed_anal_spin0", st);
  auto k = mixed_anal_kernel<S>;
  SHT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, S::SMEM));
  const int per = S::SPIN ? 2 : 1;   // maps and a_lm components per transform
  k<<<job.mmax + 1, S::THREADS, S::SMEM, st>>>(gp.count, gp.cth, gp.sth, gp.nph, cp.d_moff,
                                               cp.mx_coef, cp.seed, cp.seed_exp, job.spin, phase,
                                               ncm, t0 * per, job.lmax, job.mmax + 1, Aout, ncA,
                                               t0 * per, d_err);
  SHT_CUDA(cudaGetLastError());
}

}  // namespace

bool mixed_anal_supported(const JobDesc &job) {
  return job.type == SHARP_MAP2ALM && job.ntrans >= 1;
}

void launch_mixed_anal(const JobDesc &job, const GeomPlan &gp, CoefPlan &cp,
                       const double2 *phase, int ncm, double2 *Aout, int ncA, int *d_err,
                       cudaStream_t st) {
  if (!cp.mx_coef) {
    // a tile's coefficients are copied whole: kAM entries of slack at the end
    const size_t n = (size_t(cp.total) + kAM) * (cp.spin == 0 ? 1 : 2);
    SHT_CUDA(cudaMallocAsync(&cp.mx_coef, sizeof(double2) * n, st));
    SHT_CUDA(cudaMemsetAsync(cp.mx_coef, 0, sizeof(double2) * n, st));
    mixed_anal_coef_kernel<<<cp.mmax + 1, 256, 0, st>>>(cp.lmax, cp.mmax, cp.spin, cp.d_moff,
                                                        cp.alpha, cp.beta, cp.cfac, cp.mx_coef);
    SHT_CUDA(cudaGetLastError());
  }
  for (int t0 = 0; t0 < job.ntrans;) {
    int nb;
    if (job.spin == 0) {
      nb = std::min(job.ntrans - t0, 4);
      switch (nb) {
        case 4: launch_anal_shape<AShape<false, 4>>(job, gp, cp, phase, ncm, t0, Aout, ncA, d_err, st); break;
        case 3: launch_anal_shape<AShape<false, 3>>(job, gp, cp, phase, ncm, t0, Aout, ncA, d_err, st); break;
        case 2: launch_anal_shape<AShape<false, 2>>(job, gp, cp, phase, ncm, t0, Aout, ncA, d_err, st); break;
        default: launch_anal_shape<AShape<false, 1>>(job, gp, cp, phase, ncm, t0, Aout, ncA, d_err, st); break;
      }
    } else {
      nb = std::min(job.ntrans - t0, 2);
      if (nb == 2) launch_anal_shape<AShape<true, 2>>(job, gp, cp, phase, ncm, t0, Aout, ncA, d_err, st);
      else launch_anal_shape<AShape<true, 1>>(job, gp, cp, phase, ncm, t0, Aout, ncA, d_err, st);
    }
    t0 += nb;
  }
}

}  // namespace sht
