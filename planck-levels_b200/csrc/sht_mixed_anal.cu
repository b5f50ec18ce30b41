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
// cores and the contraction runs exactly in integers on tcgen05.mma.kind::i8:
//
//  * A (tensor memory, M = 128 rows, K = (ring pair, value, byte)): the
//    Toeplitz expansion of the signed base-256 digits of the group's phase
//    factors, quantised per group of ring pairs and (half, column) against the
//    group's maximum; row (hc, w) holds class w of (half, column) hc.  Built
//    once per group, it stays in TMEM while the group sweeps all l, so the
//    MMAs read only the B operand from shared memory.
//  * B (shared memory, N = 80 consecutive l, K as A): the words
//    u_l(p) = 2^31 + round(lambda_l(p) 2^30 / b_l) with the analytic bound
//    b_l (sqrt((2l+1)/4pi) at spin 0; 1 for each of d^l_{m,+-s}), one
//    magic-constant DFMA each; a producer thread owns one ring pair and
//    writes one (spin: two) 4-byte words per l.
//  * D (int32, TMEM, 128 lanes x 80 columns per l-tile, two buffers): the
//    exact class sums over the group's ring pairs.  A tile is read back
//    through shared memory, its five class sums per (l, half, column)
//    combined exactly in 64-bit integers, corrected for the 2^31 offset and
//    scaled in FP64, and added to the output (one CTA per m: no atomics).
//    Like the FP64 kernels, the output holds sums of the rescaled recurrence
//    values mu_l = lambda_l / c_l; c_l is applied when the a_lm are scattered.
//
// Warp roles: spin 0: 8 producer warps (256 ring pairs per group, up to 6
// transforms per launch); spin s: 4 producer warps (128 ring pairs, two
// recurrences each, up to 3 transforms).  Four flusher warps (one per TMEM
// subpartition) read the class sums back and update the output while the
// producers run the next tiles.  The last warp (lane 0) stages each l-tile's
// recurrence coefficients into shared memory (cp.async.bulk) and issues its
// MMAs.  Every wait is bounded; a timeout is reported through the error word.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "sht_device.h"
#include "sht_recurrence.cuh"
#include "sht_tc.cuh"

namespace sht {

namespace {

constexpr int kAM = 80;                       // l per tile (MMA N; a multiple of 16)
constexpr int kAClasses = 5;                  // byte-product weights 2^16 .. 2^48
constexpr int kHCW = 6;                       // (half, column) groups per TMEM subpartition
// B slice of one producer warp and tile (kAM l x the warp's ring pairs,
// K-major, no swizzle): the 8-row groups are contiguous (SBO = 128) and the K
// core matrices lie kALBO = (kAM/8)*128 + 16 bytes apart, so the per-l stores
// of a warp spread over all 32 banks.  An MMA of N = 80 costs about what one
// of N = 64 does (the issue floor), so 80 l per tile cut the MMA time per l.
constexpr int kALBO = (kAM / 8) * 128 + 16;
constexpr int kFRow = 4 * kAM + 16;           // flush staging row (bytes)

// TMEM row (lane) of class w of (half, column) group hc: six groups of five
// rows per 32-lane subpartition, so a subpartition holds whole groups.
__host__ __device__ constexpr int arow(int hc, int w) {
  return 32 * (hc / kHCW) + kAClasses * (hc % kHCW) + w;
}

template <bool SPIN_, int NB_>
struct AShape {
  static constexpr bool SPIN = SPIN_;
  static constexpr int NB = NB_;
  static constexpr int TY = SPIN ? 2 : 1;              // recurrence values per pair and l
  static constexpr int PW = SPIN ? 4 : 8;              // producer warps
  static constexpr int FW = 4;                         // flusher warps (one per subpartition)
  static constexpr int G = 32 * PW;                    // ring pairs per group
  static constexpr int THREADS = 32 * (PW + FW + 1);
  static constexpr int KB = 4 * TY * G;                // K bytes of a group
  static constexpr int ACOLS = KB / 4;                 // TMEM columns of the A operand
  static constexpr int KCM = 8 * TY;                   // K core matrices per warp slice
  static constexpr int SLICE = (KCM - 1) * kALBO + (kAM / 8) * 128;
  static constexpr int STAGES = 2 * PW * SLICE;        // both B stages
  static constexpr int CE = SPIN ? 32 : 16;            // coefficient bytes per l
  static constexpr int COEF = kAM * CE;                // one tile's coefficients
  static constexpr int OUT = SPIN ? 4 : 2;             // real outputs per transform
  static constexpr int NCOL = OUT * NB;
  static constexpr int NH = 2 * NCOL;                  // (half, column): north, then south
  static constexpr int AROW = KB + 16;                 // A staging row (bytes)
  static constexpr int FLUSH = FW * 32 * kFRow;        // flush staging
  static constexpr int SMEM = STAGES + FLUSH + 2 * COEF;
  static constexpr uint32_t NCOLS = 512;               // A: 256 columns, D: 2 x kAM
  static_assert(ACOLS + 2 * kAM <= 512, "TMEM capacity");
  static_assert(KB == 1024, "K extent of a group");
  static_assert(NH <= 4 * kHCW, "(half, column) groups fit the four subpartitions");
  static_assert(arow(4 * kHCW - 1, kAClasses - 1) * AROW + KB <= STAGES, "A staging");
  static_assert(SMEM + 4096 <= 232448, "shared memory");
};

__device__ __forceinline__ void sts_u32(uint32_t a, uint32_t v) {
  asm volatile("st.shared.b32 [%0], %1;" :: "r"(a), "r"(v) : "memory");
}
__device__ __forceinline__ void sts_u32x2(uint32_t a, uint32_t x, uint32_t y) {
  asm volatile("st.shared.v2.b32 [%0], {%1, %2};" :: "r"(a), "r"(x), "r"(y) : "memory");
}
__device__ __forceinline__ uint4 lds_u32x4(uint32_t a) {
  uint4 v;
  asm volatile("ld.shared.v4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a));
  return v;
}
__device__ __forceinline__ uint32_t lds_u32(uint32_t a) {
  uint32_t v;
  asm volatile("ld.shared.b32 %0, [%1];" : "=r"(v) : "r"(a));
  return v;
}
template <int N>
__device__ __forceinline__ void producers_sync() {
  asm volatile("bar.sync 1, %0;" :: "n"(N) : "memory");
}
template <int N>
__device__ __forceinline__ void named_sync(int id) {
  asm volatile("bar.sync %0, %1;" :: "r"(id), "n"(N) : "memory");
}
// Instruction descriptor: D s32, A s8, B u8, both K-major, M = m, N = n.
__host__ __device__ constexpr uint32_t make_idesc_s8u8(int m, int n) {
  return (2u << 4) | (1u << 7) | (0u << 10) | (uint32_t(n >> 3) << 17) |
         (uint32_t(m >> 4) << 24);
}

// Per-m coefficient table of the analysis, for l = m .. lmax + kPad:
// spin 0: (alpha_l, c_l 2^30 / b_l); spin s: (a_l, b_l), (c_l 2^30, 1 / c_l)
// (the second entry of the spin record is the flush's row factor).
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
      const double c = cfac[base + i];
      out[2 * (base + i) + 1] = make_double2(c * kQ, c != 0.0 ? 1.0 / c : 0.0);
    }
  }
}

// Jobs run group-major (group g of ring pairs, l-tile t), J = g * ntile + t;
// the class sums of job J live in TMEM D buffer J mod 2.
//
// Barriers (all waits bounded):
//   full_a[st]  producers -> issuer: B stage st holds job J's words (and, for
//               a group's first job, the group's A operand is in TMEM)
//   done[st]    issuer -> producers: job J's MMAs are complete (B stage and,
//               after a group's last job, A may be rewritten)
//   cfull[st]   bulk copy -> producers: job J's coefficients are staged
//   dfull[d]    issuer -> flushers: job J's class sums are complete
//   dfree[d]    flushers -> issuer: job J's class sums have been read
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
  const int ngroup = (cnt + S::G - 1) / S::G;
  const int njobs = ngroup * ntile;
  unsigned char *sB = sm;                              // B stages; A staging at group start
  unsigned char *sF = sm + S::STAGES;                  // flush staging
  unsigned char *sC = sF + S::FLUSH;                   // coefficient stages
  const uint32_t sB32 = smem_u32(sB), sF32 = smem_u32(sF), sC32 = smem_u32(sC);
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
  const uint32_t tmem = tslot;                 // A: columns [0, 256); D: 256 + kAM d

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
    constexpr uint32_t idesc = make_idesc_s8u8(128, kAM);
    bool ok = true;
    int issued = -1;
    for (int J = 0; J < njobs; ++J) {
      const int st = J & 1;
      bool w = mbar_wait(&full_a[st], (J >> 1) & 1);
      // D buffer st is free once job J-2 has been read back
      if (J >= 2) w = w && mbar_wait(&dfree[st], ((J >> 1) - 1) & 1);
      if (!__all_sync(0xffffffffu, w)) {
        ok = false;
        break;
      }
      tc_fence_after();
      if (lane == 0) {
        // the producers are done with this job's coefficients
        if (J + 2 < njobs) load_coef(J + 2);
        const uint32_t d = tmem + uint32_t(S::ACOLS + st * kAM);
        const uint64_t b0 = make_desc(sB32 + st * PW * S::SLICE, kALBO, 128);
        // K-step k covers bytes [32k, 32k+32): A columns 8k .. 8k+7; B warp
        // slice k / (4 TY), core matrices 2 (k mod 4 TY) and the next (the
        // start-address field, 16-byte units, is advanced per K-step)
#pragma unroll
        for (int k = 0; k < S::KB / 32; ++k)
          mma_i8_tmem_a(d, tmem + uint32_t(8 * k),
                        b0 + uint64_t(((k / (4 * S::TY)) * S::SLICE +
                                       (k % (4 * S::TY)) * 2 * kALBO) >> 4),
                        idesc, k > 0 ? 1u : 0u);
        mma_commit(&done[st]);
        mma_commit(&dfull[st]);
      }
      __syncwarp();
      issued = J;
    }
    if (!ok) {
      if (lane == 0) *reinterpret_cast<volatile int *>(err) = 1;
      if (issued >= 0) mbar_wait(&done[issued & 1], (issued >> 1) & 1);
    }
  } else if (warp >= PW) {
    // ---- flushers: warp PW + k reads lanes 32k .. 32k+31 of each tile ----
    const int k = warp - PW;                   // == warp mod 4: its TMEM subpartition
    const int ft = tid - 32 * PW;              // 0 .. 127
    constexpr int kItems = (kAM * (S::NCOL / 2) + 32 * FW - 1) / (32 * FW);
    const uint32_t frow = sF32 + (32 * k + lane) * kFRow;
    bool ok = true;
    int J = 0;
    for (int g = 0; g < ngroup; ++g) {
      const int sl = g & 1;
      if (ok) ok = __all_sync(0xffffffffu, mbar_wait(&sfull[sl], (g >> 1) & 1));
      const double *fsc = s_fscale[sl], *fco = s_corr[sl];
      for (int t = 0; t < ntile; ++t, ++J) {
        const int d = J & 1;
        // items (l, complex output jo), real columns 2 jo, 2 jo + 1 of both
        // halves: their output entries and row factors do not depend on the
        // class sums, so they are fetched before the wait
        const int l0 = mhi + t * kAM;
        double2 po[kItems];
        double pcq[kItems];
#pragma unroll
        for (int u = 0; u < kItems; ++u) {
          const int it = ft + u * 32 * FW;
          const int l = l0 + (it % kAM);
          const bool v = ok && it < kAM * (S::NCOL / 2) && l <= lmax;
          po[u] = v ? Aout[(mo + l) * ncA + comp0 + it / kAM] : make_double2(0.0, 0.0);
          // spin s: the row factor 1 / c_l itself; spin 0: c_l 2^30 / b_l
          pcq[u] = !v ? 1.0 : S::SPIN ? __ldg(coef + 2 * (mo + l) + 1).y : __ldg(coef + mo + l).y;
        }
        if (ok) ok = __all_sync(0xffffffffu, mbar_wait(&dfull[d], (J >> 1) & 1));
        // staging of the previous tile is no longer read
        named_sync<32 * FW>(2);
        if (ok) {
          tc_fence_after();
          uint32_t v[kAM];
#pragma unroll
          for (int q = 0; q < kAM; q += 16)
            tmem_ld16(tmem + (uint32_t(32 * k) << 16) + uint32_t(S::ACOLS + d * kAM + q),
                      *reinterpret_cast<uint32_t(*)[16]>(v + q));
          tmem_ld_wait();
#pragma unroll
          for (int q = 0; q < kAM; q += 4) sts_u32x4(frow + 4 * q, v[q], v[q + 1], v[q + 2], v[q + 3]);
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&dfree[d]);
        named_sync<32 * FW>(2);
        if (ok) {
#pragma unroll
          for (int u = 0; u < kItems; ++u) {
            const int it = ft + u * 32 * FW;
            const int li = it % kAM, jo = it / kAM;
            const int l = l0 + li;
            if (it >= kAM * (S::NCOL / 2) || l > lmax) continue;
            double R[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const int hc = (e >> 1) * S::NCOL + 2 * jo + (e & 1);
              uint32_t c[kAClasses];
#pragma unroll
              for (int w = 0; w < kAClasses; ++w) c[w] = lds_u32(sF32 + arow(hc, w) * kFRow + 4 * li);
              const long long P = (long long)int(c[0]) + ((long long)int(c[1]) << 8) +
                                  ((long long)int(c[2]) << 16) + ((long long)int(c[3]) << 24);
              const double Pd = __longlong_as_double(P + 0x4338000000000000LL) - 6755399441055744.0;
              R[e] = (fma(i2d_exact(c[4]), 4294967296.0, Pd) - fco[hc]) * fsc[hc];
            }
            // lambda was quantised as c_l mu_l 2^30 / b_l: row factor
            // b_l / c_l = 2^30 / cq_l (spin s: b_l = 1, read from the table)
            const double b = S::SPIN ? pcq[u] : kQ / pcq[u];
            const double sg = ((l - mhi) & 1) ? -b : b;
            double2 o = po[u];
            o.x += b * R[0] + sg * R[2];
            o.y += b * R[1] + sg * R[3];
            Aout[(mo + l) * ncA + comp0 + jo] = o;
          }
        }
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
    const double flip = ((mhi - m + spin) & 1) ? -1.0 : 1.0;
    const double sgn_mfac = (m & 1) ? -pre_v[m] : pre_v[m];
    const int sp = warp & 3;                   // this warp's TMEM subpartition
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
      // quantise; the A words of this pair go to the staging rows (the B
      // stages are free: the previous group's last MMA has completed)
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
        for (int w = 0; w < kAClasses; ++w) {
          const uint32_t a = sB32 + arow(i, w) * S::AROW + 4 * S::TY * tid;
          if constexpr (S::SPIN) sts_u32x2(a, word[0][w], word[S::TY - 1][w]);
          else sts_u32(a, word[0][w]);
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) ps += __shfl_xor_sync(0xffffffffu, ps, o);
        if (lane == 0) s_psum[warp][i] = ps;
      }
      // the scale slot of group g-2 is free once its tiles have been read back
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
      // A rows of this warp's subpartition (lane = row) into TMEM; the PW / 4
      // warps of a subpartition split the columns
      {
        constexpr int per = S::ACOLS / (PW / 4);
        const int c0 = (warp >> 2) * per;
        const uint32_t src = sB32 + (32 * sp + lane) * S::AROW + 4 * c0;
        const uint32_t dst = tmem + (uint32_t(32 * sp) << 16) + uint32_t(c0);
#pragma unroll 1
        for (int c = 0; c < per; c += 16) {
          uint32_t wv[16];
#pragma unroll
          for (int q = 0; q < 16; q += 4) {
            // lanes 30, 31 of a subpartition are padding rows (zero)
            const uint4 x = lane < kAClasses * kHCW ? lds_u32x4(src + 4 * (c + q))
                                                    : make_uint4(0u, 0u, 0u, 0u);
            wv[q] = x.x; wv[q + 1] = x.y; wv[q + 2] = x.z; wv[q + 3] = x.w;
          }
          tmem_st16(dst + uint32_t(c), wv);
        }
        tmem_st_wait();
      }
      tc_fence_before();
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
          // B stage of job J-2 is reused; this job's coefficients are staged
          bool w = J < 2 || mbar_wait(&done[st], ((J >> 1) - 1) & 1);
          w = w && mbar_wait(&cfull[st], (J >> 1) & 1);
          ok = __all_sync(0xffffffffu, w);
        }
        const uint32_t slice = sB32 + (st * PW + warp) * S::SLICE +
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
      // A (TMEM) and the staging rows are rewritten by the next group once
      // the last MMA of this one is done
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
    // a table of the plan (freed with it by cudaFree), not workspace
    SHT_CUDA(cudaMalloc(&cp.mx_coef, sizeof(double2) * n));
    SHT_CUDA(cudaMemsetAsync(cp.mx_coef, 0, sizeof(double2) * n, st));
    mixed_anal_coef_kernel<<<cp.mmax + 1, 256, 0, st>>>(cp.lmax, cp.mmax, cp.spin, cp.d_moff,
                                                        cp.alpha, cp.beta, cp.cfac, cp.mx_coef);
    SHT_CUDA(cudaGetLastError());
  }
  for (int t0 = 0; t0 < job.ntrans;) {
    int nb;
    if (job.spin == 0) {
      nb = std::min(job.ntrans - t0, 6);
      switch (nb) {
        case 6: launch_anal_shape<AShape<false, 6>>(job, gp, cp, phase, ncm, t0, Aout, ncA, d_err, st); break;
        case 5: launch_anal_shape<AShape<false, 5>>(job, gp, cp, phase, ncm, t0, Aout, ncA, d_err, st); break;
        case 4: launch_anal_shape<AShape<false, 4>>(job, gp, cp, phase, ncm, t0, Aout, ncA, d_err, st); break;
        case 3: launch_anal_shape<AShape<false, 3>>(job, gp, cp, phase, ncm, t0, Aout, ncA, d_err, st); break;
        case 2: launch_anal_shape<AShape<false, 2>>(job, gp, cp, phase, ncm, t0, Aout, ncA, d_err, st); break;
        default: launch_anal_shape<AShape<false, 1>>(job, gp, cp, phase, ncm, t0, Aout, ncA, d_err, st); break;
      }
    } else {
      nb = std::min(job.ntrans - t0, 3);
      switch (nb) {
        case 3: launch_anal_shape<AShape<true, 3>>(job, gp, cp, phase, ncm, t0, Aout, ncA, d_err, st); break;
        case 2: launch_anal_shape<AShape<true, 2>>(job, gp, cp, phase, ncm, t0, Aout, ncA, d_err, st); break;
        default: launch_anal_shape<AShape<true, 1>>(job, gp, cp, phase, ncm, t0, Aout, ncA, d_err, st); break;
      }
    }
    t0 += nb;
  }
}

}  // namespace sht
