// Mixed-precision batched synthesis on the 5th-generation tensor cores.
//
// For NB transforms sharing geometry and lmax, the Legendre step of alm2map
// is, per order m and tile of 128 ring pairs, the contraction
//   R[ring, col] = sum_l lambda_l(ring) * a_l[col]
// split by the parity of l - max(m, s) (north/south symmetry), with
// col = (transform, component, re/im).  The recurrence for lambda stays FP64
// (one thread per ring pair, exponent-tracked as in the FP64 kernels).  The
// contraction runs exactly in integers on tcgen05.mma.kind::i8:
//
//  * lambda is bounded analytically, |lambda_lm| <= sqrt((2l+1)/4pi) for
//    spin 0 and |d^l_{m,+-s}| <= 1 for spin s (so |r+ +- r-| <= 2), so
//    q_l = round(lambda_l * 2^30 / b_l) fits 31 bits.  One DFMA with the
//    constant 1.5*2^52 + 2^31 leaves u_l = q_l + 2^31 in the low word of the
//    result: its four bytes are the unsigned int8 digits of the A operand,
//    stored as they are (K index = 4*l + byte).
//  * a_l * b_l is quantised per (m, column) to p_l = round(. * 2^30 / max),
//    written as four signed int8 digits d_0..d_3.  The B operand is the
//    Toeplitz expansion B[(l,k), (col,w)] = d_{w-k}, w = 2..6, so one MMA
//    accumulates the byte products of equal weight 2^(8w) in one int32
//    column; products of weight below 2^16 are dropped (relative size 2^-30).
//  * int32 accumulation over all l is exact (|sum| < 2^29 for lmax <= 8192),
//    so TMEM is read once per tile; the epilogue forms
//    sum_w D_w 2^(8w) - 2^31 sum_l p_l in FP64 and rescales.
//
// Warp roles (288 threads): warps 0-7 each own 32 ring pairs (two row sets
// of 128, each its own MMA M dimension and TMEM accumulators, sharing the B
// tiles), run the recurrence and write the A tiles of a 32-l chunk; lane 0
// of warp 8 streams the per-chunk block (recurrence coefficients,
// quantisation factors, B tiles) with cp.async.bulk and issues the MMAs.
// Chunks are pipelined through mbarriers (A tiles double-buffered,
// coefficient blocks prefetched four deep); every wait is bounded and a
// timeout is reported through an error word (mapped host memory) after the
// accumulators are released.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <vector>

#include "sht_device.h"
#include "sht_recurrence.cuh"
#include "sht_tc.cuh"

namespace sht {

namespace {

constexpr int kMC = 32;          // l-steps per chunk
constexpr int kLP = kMC / 2;     // l-steps of one parity per chunk
constexpr int kKB = 4 * kLP;     // K bytes of one parity tile (64)
constexpr int kRows = 128;       // ring pairs per row set (MMA M)
constexpr int kRS = 2;           // row sets per CTA (256 ring pairs, 8 producer warps)
constexpr int kClasses = 5;      // byte-product weights 2^16 .. 2^48
constexpr int kSA = 2;           // A-tile stages
constexpr int kSB = 4;           // coefficient/B-block stages
constexpr int kThreads = 32 * (4 * kRS + 1);
constexpr int kTileBytes = kRows * kKB;                        // one A tile (8 KiB)

// Byte offset of element (row, kbyte) in a K-major tile whose rows are
// kKB bytes long.
__host__ __device__ constexpr int tile_off(int row, int kb) {
  return ((row >> 3) * (kKB / 16) + (kb >> 4)) * 128 + (row & 7) * 16 + (kb & 15);
}

// 16 l-steps of the spin-0 recurrence for one ring pair: quantised words of
// the even-offset (ue) and odd-offset (uo) values.  ALL: every lane of the
// warp is in the IEEE regime (no per-lane masking of the quantisation).
template <bool ALL>
__device__ __forceinline__ void steps16_s0(uint32_t cf, double x, bool act, double &mu0,
                                           double &mu1, uint32_t *ue, uint32_t *uo) {
  double2 c[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) c[k] = lds_f64x2(cf + 16 * k);  // (alpha_l, cq_l)
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const double q0 = (ALL || act) ? c[2 * j].y : 0.0;
    const double q1 = (ALL || act) ? c[2 * j + 1].y : 0.0;
    ue[j] = quant(mu1, q0);
    const double nm = fma(c[2 * j].x * x, mu1, -mu0);
    uo[j] = quant(nm, q1);
    const double nn = fma(c[2 * j + 1].x * x, nm, -mu1);
    mu0 = nm;
    mu1 = nn;
  }
}

// 8 l-steps of the spin-s recurrences (mu+, mu-): words of r+ + r- (uw)
// and r- - r+ (ux), even (e) and odd (o) offsets.
template <bool ALL>
__device__ __forceinline__ void steps8_sp(uint32_t cf, double x, bool act, double &mp0,
                                          double &mp1, double &mm0, double &mm1, uint32_t *uwe,
                                          uint32_t *uxe, uint32_t *uwo, uint32_t *uxo) {
  double2 ab[8], cq[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    ab[k] = lds_f64x2(cf + 32 * k);       // (a_l, b_l)
    cq[k] = lds_f64x2(cf + 32 * k + 16);  // (cq_l, 0)
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const double q0 = (ALL || act) ? cq[2 * j].x : 0.0;
    const double q1 = (ALL || act) ? cq[2 * j + 1].x : 0.0;
    {
      const uint32_t up = quant(mp1, q0), um = quant(mm1, q0);
      uwe[j] = up + um - 0x80000000u;
      uxe[j] = um - up + 0x80000000u;
    }
    const double2 a0 = ab[2 * j], a1 = ab[2 * j + 1];
    const double np_ = fma(fma(a0.x, x, -a0.y), mp1, -mp0);
    const double nm_ = fma(fma(a0.x, x, a0.y), mm1, -mm0);
    {
      const uint32_t up = quant(np_, q1), um = quant(nm_, q1);
      uwo[j] = up + um - 0x80000000u;
      uxo[j] = um - up + 0x80000000u;
    }
    const double nnp = fma(fma(a1.x, x, -a1.y), np_, -mp1);
    const double nnm = fma(fma(a1.x, x, a1.y), nm_, -mm1);
    mp0 = np_;
    mp1 = nnp;
    mm0 = nm_;
    mm1 = nnm;
  }
}

// --------------------------------------------------------------------------
// Compile-time shape of one kernel instance.
// --------------------------------------------------------------------------
template <int T_, int NCOMP_, int NB_>
struct Shape {
  static constexpr int T = T_;                 // value types (1: lambda; 2: r+ + r-, r- - r+)
  static constexpr int NCOMP = NCOMP_;         // a_lm components per transform
  static constexpr int NB = NB_;               // transforms per launch
  static constexpr int NCOL = 2 * NCOMP * NB;  // real columns
  static constexpr int NPR = kClasses * NCOL;  // B rows used
  static constexpr int NP = (NPR + 15) / 16 * 16;
  static constexpr int PS = NP <= 256 ? NP : NP / 2;  // MMA N per instruction
  static constexpr int CE = (T == 1) ? 16 : 32;       // coefficient bytes per l
  static constexpr int COEF = kMC * CE;
  static constexpr int BLK = COEF + 2 * NP * kKB;     // per-chunk block
  static constexpr int ATILES = T * 2;                // A tiles per row set
  static constexpr int TCOLS = ATILES * NP;           // TMEM columns per row set
  static constexpr int ALLCOLS = kRS * TCOLS;
  static constexpr uint32_t NCOLS =
      ALLCOLS <= 32 ? 32 : ALLCOLS <= 64 ? 64 : ALLCOLS <= 128 ? 128 : ALLCOLS <= 256 ? 256 : 512;
  static constexpr int SMEM = kSB * BLK + kSA * kRS * ATILES * kTileBytes;
  static constexpr int MINB = NCOLS <= 256 ? 2 : 1;   // CTAs per SM the TMEM allows
  static_assert(NP % PS == 0 && PS % 16 == 0 && PS <= 256, "MMA N shape");
  static_assert(ALLCOLS <= 512, "TMEM capacity");
  static_assert(BLK % 16 == 0, "bulk copy granularity");
};

// --------------------------------------------------------------------------
// Per-call image of the a_lm and coefficients: per (m, chunk) one block
// [coefficients | B tile even | B tile odd], plus per-m epilogue constants
// epi[m] = {scale[col], 2^31 * sum_even p[col], 2^31 * sum_odd p[col]}.
// One CTA per m.  A first pass over the m segment of A (rows read
// contiguously, each thread on one component) finds the quantisation scale
// of every column; then each chunk's block is assembled in shared memory
// (the chunk's A rows staged there first; warp w forms the words of the
// columns col = w (mod 8), lane = l within the chunk) and written out
// whole with 16-byte stores, padding rows and l > lmax as zeros, so the
// image needs no zero fill.
// --------------------------------------------------------------------------
template <class S>
__global__ void __launch_bounds__(256)
mixed_image_kernel(int lmax, int spin, const long long *__restrict__ moff,
                   const double *__restrict__ ca, const double *__restrict__ cb,
                   const double *__restrict__ cfac, const long long *__restrict__ ioff,
                   const double2 *__restrict__ A, int ncA, int comp0,
                   unsigned char *__restrict__ img, double *__restrict__ epi) {
  constexpr int NCOL = S::NCOL, NCU = NCOL / 2;   // real columns, complex components
  constexpr int G = 256 / NCU;                    // l-groups of the scale pass
  constexpr int CPW = (NCOL + 7) / 8;             // columns per warp
  __shared__ __align__(16) unsigned char blk[S::BLK];
  __shared__ double2 arow[kMC][NCU];
  __shared__ double red[G][NCOL];
  __shared__ double inv[NCOL];
  const int m = blockIdx.x;
  const int lbase = max(m, spin);
  if (lbase > lmax) return;
  const long long mo = moff[m] - m;
  const int nch = (lmax - lbase + kMC) / kMC;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  unsigned char *base = img + ioff[m];
  double *ep = epi + (long long)m * 3 * NCOL;
  auto bound = [&](int l) { return spin == 0 ? sqrt((2.0 * l + 1.0) / (4.0 * M_PI)) : 2.0; };
  // a_l * b_l of component c (both columns), zero where cfac is zero
  auto scaled = [&](int l, int c) {
    const double f = cfac[mo + l];
    if (f == 0.0) return make_double2(0.0, 0.0);
    const double2 a = A[(mo + l) * ncA + comp0 + c];
    const double b = bound(l);
    return make_double2(a.x / f * b, a.y / f * b);
  };
  // ---- scale pass: column maxima ----
  if (tid < G * NCU) {
    const int c = tid % NCU, g = tid / NCU;
    double mr = 0.0, mi = 0.0;
    for (int l = lbase + g; l <= lmax; l += G) {
      const double2 v = scaled(l, c);
      mr = fmax(mr, fabs(v.x));
      mi = fmax(mi, fabs(v.y));
    }
    red[g][2 * c] = mr;
    red[g][2 * c + 1] = mi;
  }
  __syncthreads();
  if (tid < NCOL) {
    double amax = 0.0;
    for (int g = 0; g < G; ++g) amax = fmax(amax, red[g][tid]);
    inv[tid] = amax > 0.0 ? kQ / amax : 0.0;
    ep[tid] = amax / (kQ * kQ);
  }
  long long psum[CPW];
#pragma unroll
  for (int k = 0; k < CPW; ++k) psum[k] = 0;
  // ---- blocks ----
  for (int ch = 0; ch < nch; ++ch) {
    const int l0 = lbase + ch * kMC;
    for (int i = tid; i < S::BLK / 16; i += 256)
      reinterpret_cast<uint4 *>(blk)[i] = make_uint4(0u, 0u, 0u, 0u);
    for (int i = tid; i < kMC * NCU; i += 256) {
      const int r = i / NCU, c = i - r * NCU;
      arow[r][c] = (l0 + r <= lmax) ? scaled(l0 + r, c) : make_double2(0.0, 0.0);
    }
    __syncthreads();
    // coefficient entries (alpha_l, cq_l) or (a_l, b_l, cq_l, 0)
    if (tid < kMC) {
      const int l = l0 + tid;
      double *cf = reinterpret_cast<double *>(blk) + tid * (S::CE / 8);
      const double cq = cfac[mo + l] * kQ / bound(l);
      cf[0] = ca[mo + l];
      if (spin == 0) {
        cf[1] = cq;
      } else {
        cf[1] = cb[mo + l];
        cf[2] = cq;
        cf[3] = 0.0;
      }
    }
    if (l0 + lane <= lmax) {
      unsigned char *tile = blk + kMC * S::CE + (lane & 1) * S::NP * kKB;
      const int jj = lane >> 1;
#pragma unroll
      for (int k = 0; k < CPW; ++k) {
        const int col = warp + 8 * k;
        if (col >= NCOL) break;
        const double2 v = arow[lane][col >> 1];
        const int p = static_cast<int>(llrint(((col & 1) ? v.y : v.x) * inv[col]));
        // signed base-256 digits, each in [-128, 127]
        int d[4], r = p;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          d[q] = ((r + 128) & 255) - 128;
          r = (r - d[q]) >> 8;
        }
        d[3] = r;
        psum[k] += p;
#pragma unroll
        for (int w = 2; w <= 6; ++w) {
          uint32_t word = 0;
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (w - q >= 0 && w - q <= 3) word |= uint32_t(uint8_t(int8_t(d[w - q]))) << (8 * q);
          const int row = col * kClasses + (w - 2);
          *reinterpret_cast<uint32_t *>(tile + tile_off(row, 4 * jj)) = word;
        }
      }
    }
    __syncthreads();
    uint4 *dst = reinterpret_cast<uint4 *>(base + (long long)ch * S::BLK);
    for (int i = tid; i < S::BLK / 16; i += 256) dst[i] = reinterpret_cast<const uint4 *>(blk)[i];
    __syncthreads();
  }
  // parity sums: lanes of equal parity (xor with even offsets keeps parity)
#pragma unroll
  for (int k = 0; k < CPW; ++k) {
    const int col = warp + 8 * k;
#pragma unroll
    for (int o = 16; o >= 2; o >>= 1) psum[k] += __shfl_xor_sync(0xffffffffu, psum[k], o);
    if (col < NCOL && lane < 2) ep[(1 + lane) * NCOL + col] = 2147483648.0 * double(psum[k]);
  }
}

// --------------------------------------------------------------------------
// Epilogue: per ring pair, the exact int32 class sums of every (type, parity,
// column) -> FP64 (sum_w D_w 2^(8w) - 2^31 sum p, times the column scale),
// then the north/south phases.  TMEM is streamed 16 columns at a time and a
// transform is finalised as soon as its columns are complete, so only a few
// accumulators are live at once.
// --------------------------------------------------------------------------
template <class S>
__device__ __forceinline__ void epilogue(uint32_t lane_base, const double *__restrict__ ep,
                                         bool valid, bool has_s, int p, int m, int mhi, int spin,
                                         double2 *__restrict__ phase, int ncm, int pcomp0,
                                         int ms) {
  constexpr int CPT = 2 * S::NCOMP;      // real columns per transform
  constexpr int RPT = kClasses * CPT;    // B rows per transform
  double R[S::T][2][S::NCOL];
#pragma unroll
  for (int q = 0; q < S::NPR; q += 16) {
    uint32_t v[S::T][2][16];
#pragma unroll
    for (int t = 0; t < S::T; ++t)
#pragma unroll
      for (int par = 0; par < 2; ++par)
        tmem_ld16(lane_base + uint32_t((t * 2 + par) * S::NP + q), v[t][par]);
    tmem_ld_wait();
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const int row = q + i;
      if (row < S::NPR) {
        const int col = row / kClasses, w = row % kClasses + 2;
        const double wt = double(1ull << (8 * w));
#pragma unroll
        for (int t = 0; t < S::T; ++t)
#pragma unroll
          for (int par = 0; par < 2; ++par) {
            if (w == 2) R[t][par][col] = -ep[(1 + par) * S::NCOL + col];
            R[t][par][col] = fma(i2d_exact(v[t][par][i]), wt, R[t][par][col]);
          }
      }
    }
    // transforms whose last row lies in this group are complete
#pragma unroll
    for (int j = 0; j < S::NB; ++j) {
      const int last = (j + 1) * RPT - 1;
      if (last < q || last >= q + 16) continue;
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        const double sc = ep[j * CPT + c];
#pragma unroll
        for (int t = 0; t < S::T; ++t)
#pragma unroll
          for (int par = 0; par < 2; ++par) R[t][par][j * CPT + c] *= sc;
      }
      if (!valid) continue;
      if constexpr (S::T == 1) {
        const long long row = ((long long)(p * ncm + pcomp0 + j) * 2) * ms;
        const double er = R[0][0][2 * j], ei = R[0][0][2 * j + 1];
        const double orr = R[0][1][2 * j], oi = R[0][1][2 * j + 1];
        phase[row + m] = make_double2(er + orr, ei + oi);
        if (has_s) phase[row + ms + m] = make_double2(er - orr, ei - oi);
      } else {
        const double flip = ((mhi - m + spin) & 1) ? -1.0 : 1.0;
        constexpr int X = S::T - 1;
        // columns of transform j: G re, G im, C re, C im
        const double2 gwe = make_double2(R[0][0][4 * j], R[0][0][4 * j + 1]);
        const double2 gwo = make_double2(R[0][1][4 * j], R[0][1][4 * j + 1]);
        const double2 gxe = make_double2(R[X][0][4 * j], R[X][0][4 * j + 1]);
        const double2 gxo = make_double2(R[X][1][4 * j], R[X][1][4 * j + 1]);
        const double2 cwe = make_double2(R[0][0][4 * j + 2], R[0][0][4 * j + 3]);
        const double2 cwo = make_double2(R[0][1][4 * j + 2], R[0][1][4 * j + 3]);
        const double2 cxe = make_double2(R[X][0][4 * j + 2], R[X][0][4 * j + 3]);
        const double2 cxo = make_double2(R[X][1][4 * j + 2], R[X][1][4 * j + 3]);
        // q1 = Gwe + i Cxo, q2 = Gwo + i Cxe, u1 = Cwe - i Gxo, u2 = Cwo - i Gxe
        const double2 q1 = make_double2(gwe.x - cxo.y, gwe.y + cxo.x);
        const double2 q2 = make_double2(gwo.x - cxe.y, gwo.y + cxe.x);
        const double2 u1 = make_double2(cwe.x + gxo.y, cwe.y - gxo.x);
        const double2 u2 = make_double2(cwo.x + gxe.y, cwo.y - gxe.x);
        const long long rq = ((long long)(p * ncm + pcomp0 + 2 * j) * 2) * ms;
        const long long ru = ((long long)(p * ncm + pcomp0 + 2 * j + 1) * 2) * ms;
        phase[rq + m] = make_double2(q1.x + q2.x, q1.y + q2.y);
        phase[ru + m] = make_double2(u1.x + u2.x, u1.y + u2.y);
        if (has_s) {
          phase[rq + ms + m] = make_double2(flip * (q1.x - q2.x), flip * (q1.y - q2.y));
          phase[ru + ms + m] = make_double2(flip * (u1.x - u2.x), flip * (u1.y - u2.y));
        }
      }
    }
  }
}

// --------------------------------------------------------------------------
// The synthesis kernel.
// --------------------------------------------------------------------------
template <class S>
__global__ void __launch_bounds__(kThreads, S::MINB)
mixed_synth_kernel(const int2 *__restrict__ items, const int *__restrict__ count,
                   const double *__restrict__ cth, const double *__restrict__ sth,
                   const int *__restrict__ nph_ring, const double *__restrict__ pre_v,
                   const int *__restrict__ pre_e, int spin, const unsigned char *__restrict__ img,
                   const long long *__restrict__ ioff, const double *__restrict__ epi, int lmax,
                   double2 *__restrict__ phase, int ncm, int pcomp0, int ms,
                   int *__restrict__ err) {
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ uint64_t full_b[kSB], full_a[kSA], done[kSA];
  __shared__ uint32_t tslot;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int2 it = items[blockIdx.x];
  const int m = it.x;
  const int mhi = max(m, spin);
  const int cnt = count[m];
  const int nch = mhi <= lmax ? (lmax - mhi + kMC) / kMC : 0;
  const unsigned char *img_m = img + ioff[m];
  unsigned char *sB = sm;                         // kSB blocks
  unsigned char *sA = sm + kSB * S::BLK;          // kSA x kRS x ATILES tiles

  if (tid == 0) {
    for (int i = 0; i < kSB; ++i) mbar_init(&full_b[i], 1);
    for (int i = 0; i < kSA; ++i) {
      mbar_init(&full_a[i], 4 * kRS);
      mbar_init(&done[i], 1);
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

  if (warp == 4 * kRS) {
    // ---------------- loader / MMA issuer (lane 0 issues) ----------------
    if (nch > 0) {
      if (lane == 0) {
        const int npre = nch < kSB ? nch : kSB;
        for (int c = 0; c < npre; ++c) {
          mbar_arrive_tx(&full_b[c], S::BLK);
          bulk_g2s(sB + c * S::BLK, img_m + (long long)c * S::BLK, S::BLK, &full_b[c]);
        }
      }
      __syncwarp();
      constexpr uint32_t idesc = make_idesc_i8(128, S::PS);
      bool ok = true;
      int issued = -1;
      for (int c = 0; c < nch; ++c) {
        const int sa = c % kSA, sb = c % kSB;
        const bool ready =
            mbar_wait(&full_a[sa], (c / kSA) & 1) && mbar_wait(&full_b[sb], (c / kSB) & 1);
        if (!__all_sync(0xffffffffu, ready)) {
          ok = false;
          break;
        }
        tc_fence_after();
        if (lane == 0) {
          const uint32_t a0 = smem_u32(sA + sa * kRS * S::ATILES * kTileBytes);
          const uint32_t b0 = smem_u32(sB + sb * S::BLK + S::COEF);
#pragma unroll
          for (int rs = 0; rs < kRS; ++rs)
#pragma unroll
          for (int t = 0; t < S::T; ++t)
#pragma unroll
            for (int par = 0; par < 2; ++par) {
              const uint32_t at = a0 + ((rs * S::T + t) * 2 + par) * kTileBytes;
              const uint32_t bt = b0 + par * S::NP * kKB;
#pragma unroll
              for (int pc = 0; pc < S::NP / S::PS; ++pc)
#pragma unroll
                for (int s = 0; s < kKB / 32; ++s) {
                  const uint32_t d =
                      tmem + uint32_t(rs * S::TCOLS + (t * 2 + par) * S::NP + pc * S::PS);
                  mma_i8(d, make_desc(at + s * 256, 128, 512),
                         make_desc(bt + (pc * S::PS / 8) * 512 + s * 256, 128, 512), idesc,
                         (c > 0 || s > 0) ? 1u : 0u);
                }
            }
          mma_commit(&done[sa]);
        }
        __syncwarp();
        issued = c;
        // refill the block of chunk c-1 (its MMAs are normally complete by now)
        const int cr = c - 1 + kSB;
        if (c >= 1 && cr < nch) {
          if (!__all_sync(0xffffffffu, mbar_wait(&done[(c - 1) % kSA], ((c - 1) / kSA) & 1))) {
            ok = false;
            break;
          }
          if (lane == 0) {
            const int sr = cr % kSB;
            mbar_arrive_tx(&full_b[sr], S::BLK);
            bulk_g2s(sB + sr * S::BLK, img_m + (long long)cr * S::BLK, S::BLK, &full_b[sr]);
          }
          __syncwarp();
        }
      }
      if (!ok) {
        if (lane == 0) *reinterpret_cast<volatile int *>(err) = 1;
        // let MMAs in flight drain (a commit tracks all earlier MMAs)
        if (issued >= 0) mbar_wait(&done[issued % kSA], (issued / kSA) & 1);
      }
    }
  } else {
    // ---------------- producers: one ring pair per thread ----------------
    const int rs = warp >> 2;                  // row set of this warp
    const int row = tid & (kRows - 1);         // MMA row / TMEM lane
    const int p = it.y * (kRS * kRows) + tid;
    const bool valid = p < cnt;
    const double x = valid ? cth[p] : 0.0;
    bool ok = true;
    double mu0, mu1, mm0 = 0.0, mm1 = 0.0;
    int E, Em = 0;
    bool act, live;
    if constexpr (S::T == 1) {
      const XD sd = valid ? xd_pow_log(sth[p], m, (m & 1) ? -pre_v[m] : pre_v[m]) : XD{0.0, 0};
      mu0 = 0.0;
      mu1 = sd.v;
      E = sd.e;
      live = valid && sd.v != 0.0;
      act = live && E >= -kSwitchExp;
      if (act) mu1 = ldexp(mu1, E);
    } else {
      live = spin_start_log(valid, x, valid ? sth[p] : 0.0, m, spin, pre_v[m], pre_e[m], mu0,
                            mu1, mm0, mm1, E, Em, act);
    }
    for (int c = 0; c < nch; ++c) {
      const int sa = c % kSA, sb = c % kSB;
      const bool w1 = mbar_wait(&full_b[sb], (c / kSB) & 1);
      const bool w2 = c < kSA || mbar_wait(&done[sa], ((c / kSA) - 1) & 1);
      if (!__all_sync(0xffffffffu, w1 && w2)) {
        ok = false;
        break;
      }
      unsigned char *at = sA + (sa * kRS + rs) * S::ATILES * kTileBytes;
      const uint32_t at32 = smem_u32(at);
      uint32_t u[S::T][2][kLP];
      const uint32_t cf = smem_u32(sB + sb * S::BLK);
      // this thread's row of every A tile, four l of one parity per store,
      // written as soon as the steps that make them are done
      auto store4 = [&](int o) {
#pragma unroll
        for (int t = 0; t < S::T; ++t)
#pragma unroll
          for (int par = 0; par < 2; ++par)
            sts_u32x4(at32 + (t * 2 + par) * kTileBytes + tile_off(row, 4 * o), u[t][par][o],
                      u[t][par][o + 1], u[t][par][o + 2], u[t][par][o + 3]);
      };
#pragma unroll
      for (int h = 0; h < 2; ++h) {  // two blocks of 16 l-steps
        const bool all = __all_sync(0xffffffffu, act);
        if constexpr (S::T == 1) {
          if (all)
            steps16_s0<true>(cf + h * 16 * S::CE, x, act, mu0, mu1, &u[0][0][8 * h],
                             &u[0][1][8 * h]);
          else
            steps16_s0<false>(cf + h * 16 * S::CE, x, act, mu0, mu1, &u[0][0][8 * h],
                              &u[0][1][8 * h]);
          store4(8 * h);
          store4(8 * h + 4);
        } else {
#pragma unroll
          for (int g = 0; g < 2; ++g) {
            const uint32_t cg = cf + (h * 16 + 8 * g) * S::CE;
            const int o = 8 * h + 4 * g;
            if (all)
              steps8_sp<true>(cg, x, act, mu0, mu1, mm0, mm1, &u[0][0][o], &u[S::T - 1][0][o],
                              &u[0][1][o], &u[S::T - 1][1][o]);
            else
              steps8_sp<false>(cg, x, act, mu0, mu1, mm0, mm1, &u[0][0][o], &u[S::T - 1][0][o],
                               &u[0][1][o], &u[S::T - 1][1][o]);
            store4(o);
          }
        }
        // every 16 l-steps: bookkeeping of rings still in the scaled regime
        if constexpr (S::T == 1) {
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
      __syncwarp();
      if (lane == 0) mbar_arrive(&full_a[sa]);
    }
    // epilogue: exact int32 class sums -> FP64 -> phase
    if (ok && nch > 0) {
      const int cl = nch - 1;
      if (!__all_sync(0xffffffffu, mbar_wait(&done[cl % kSA], (cl / kSA) & 1))) ok = false;
    }
    if (!ok) {
      if (lane == 0) *reinterpret_cast<volatile int *>(err) = 1;
    } else if (nch > 0) {
      tc_fence_after();
      epilogue<S>(tmem + (uint32_t((warp & 3) * 32) << 16) + uint32_t(rs * S::TCOLS),
                  epi + (long long)m * 3 * S::NCOL, valid,
                  valid ? nph_ring[2 * p + 1] > 0 : false, p, m, mhi, spin, phase, ncm, pcomp0,
                  ms);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, S::NCOLS);
  }
}

template <class S>
void launch_shape(const JobDesc &job, const GeomPlan &gp, const CoefPlan &cp, const double2 *A,
                  int ncA, int t0, double2 *phase, int ncm, int *d_err, cudaStream_t st) {
  const int mmax = job.mmax, lmax = job.lmax, spin = job.spin;
  std::vector<long long> ioff(mmax + 1);
  long long tot = 0;
  for (int m = 0; m <= mmax; ++m) {
    ioff[m] = tot;
    const int lbase = m > spin ? m : spin;
    if (lbase <= lmax) tot += (long long)((lmax - lbase + kMC) / kMC) * S::BLK;
  }
  if (tot == 0) return;
  unsigned char *img = nullptr;
  long long *d_ioff = nullptr;
  double *epi = nullptr;
  const size_t epi_bytes = sizeof(double) * 3 * S::NCOL * (mmax + 1);
  SHT_CUDA(::sht::ws_alloc(&img, size_t(tot), st));
  SHT_CUDA(::sht::ws_alloc(&d_ioff, sizeof(long long) * (mmax + 1), st));
  SHT_CUDA(::sht::ws_alloc(&epi, epi_bytes, st));
  SHT_CUDA(cudaMemcpyAsync(d_ioff, ioff.data(), sizeof(long long) * (mmax + 1),
                           cudaMemcpyHostToDevice, st));
  SHT_CUDA(cudaMemsetAsync(epi, 0, epi_bytes, st));
  {
    ProfScope ps("mixed_image", st);
    mixed_image_kernel<S><<<mmax + 1, 256, 0, st>>>(lmax, spin, cp.d_moff, cp.alpha, cp.beta,
                                                    cp.cfac, d_ioff, A, ncA, t0 * S::NCOMP, img,
                                                    epi);
    SHT_CUDA(cudaGetLastError());
  }
  {
    ProfScope ps(S::T == 1 ? "mixed_synth_spin0" : "mixed_synth_spin", st);
    auto k = mixed_synth_kernel<S>;
    SHT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, S::SMEM));
    k<<<int(gp.mixed_items.size()), kThreads, S::SMEM, st>>>(
        gp.mitems, gp.count, gp.cth, gp.sth, gp.nph, cp.seed, cp.seed_exp, spin, img, d_ioff,
        epi, lmax, phase, ncm, t0 * S::NCOMP, mmax + 1, d_err);
    SHT_CUDA(cudaGetLastError());
  }
  SHT_CUDA(cudaFreeAsync(img, st));
  SHT_CUDA(cudaFreeAsync(d_ioff, st));
  SHT_CUDA(cudaFreeAsync(epi, st));
}

}  // namespace

// ---------------------------------------------------------------------------
// Launcher: staged FP64 a_lm (A, as for the FP64 path) -> image -> kernel,
// in groups of up to 6 (spin 0) or 3 (spin > 0) transforms.
// ---------------------------------------------------------------------------
bool mixed_synth_supported(const JobDesc &job) {
  return job.type == SHARP_ALM2MAP && job.ntrans >= 1;
}

// Largest number of transforms per launch (SHARP_B200_MIXED_GROUP, default
// 6 for spin 0 and 3 for spin > 0; values above those are clamped).
int mixed_group_cap() {
  static int cap = [] {
    const char *e = getenv("SHARP_B200_MIXED_GROUP");
    const int v = e ? atoi(e) : 0;
    return v > 0 ? v : 1 << 30;
  }();
  return cap;
}

void launch_mixed_synth(const JobDesc &job, const GeomPlan &gp, const CoefPlan &cp,
                        const double2 *A, int ncA, double2 *phase, int ncm, int *d_err,
                        cudaStream_t st) {
  if (gp.mixed_items.empty()) return;  // no ring pair has an active m
  for (int t0 = 0; t0 < job.ntrans;) {
    const int left = std::min(job.ntrans - t0, mixed_group_cap());
    int nb;
#define SHT_MX(TV, CV, NBV) \
  launch_shape<Shape<TV, CV, NBV>>(job, gp, cp, A, ncA, t0, phase, ncm, d_err, st)
    if (job.spin == 0) {
      nb = left >= 12 ? 12 : std::min(left, 6);
      switch (nb) {
        case 12: SHT_MX(1, 1, 12); break;
        case 6: SHT_MX(1, 1, 6); break;
        case 5: SHT_MX(1, 1, 5); break;
        case 4: SHT_MX(1, 1, 4); break;
        case 3: SHT_MX(1, 1, 3); break;
        case 2: SHT_MX(1, 1, 2); break;
        default: SHT_MX(1, 1, 1); break;
      }
    } else {
      nb = std::min(left, 3);
      switch (nb) {
        case 3: SHT_MX(2, 2, 3); break;
        case 2: SHT_MX(2, 2, 2); break;
        default: SHT_MX(2, 2, 1); break;
      }
    }
#undef SHT_MX
    t0 += nb;
  }
}

}  // namespace sht
