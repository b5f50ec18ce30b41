// Associated-Legendre (spin 0) and Wigner-d (spin s, first derivatives)
// recurrences of the spherical-harmonic transform, FP64, sm_100a.
//
// Reference: libsharp/sharp_core_inc.c:182-293 (seeds, scaled run-up) and
// libsharp/sharp_core_inc2.c:32-619 (synthesis/analysis kernels),
// coefficients libsharp/sharp_ylmgen_c.c:44-198.
//
// Design (not a translation of the SIMD code):
//  * one thread owns R ring pairs, lanes of a warp hold consecutive pairs, so
//    recurrence coefficients and staged a_lm are warp-uniform broadcast loads;
//  * the three-term recurrence is rewritten with a per-l normalisation c_l
//    (lambda_l = c_l mu_l) so that every step is mu_{l+1} = t_l mu_l - mu_{l-1}
//    with t_l = alpha_l x (spin 0) or a_l x -/+ b_l (spin s): 2 FP64 ops per
//    step instead of 3; c_l is folded into the staged a_lm;
//  * seeds sin^m(theta) etc. are formed as (mantissa, exponent) pairs; while
//    the recurrence value is below 2^-kSwitchExp it runs scaled (exponent
//    renormalised once per l-block, nothing accumulated), then switches to
//    plain IEEE values.  Skipped terms are < 2^-88 of the leading ones;
//  * analysis reduces over rings with a warp transpose-reduction and a fixed
//    cross-warp order: no atomics, bitwise repeatable results.
#include <cuda_pipeline.h>
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "sht_device.h"
#include "sht_recurrence.cuh"

namespace sht {

namespace {

// Lane i ends up with sum over the warp of v[i] (recursive halving).
__device__ __forceinline__ double warp_transpose_reduce32(double (&v)[32]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) {
    const bool up = (lane & s) != 0;
#pragma unroll
    for (int i = 0; i < s; ++i) {
      const double send = up ? v[i] : v[i + s];
      const double keep = up ? v[i + s] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, s);
    }
  }
  return v[0];
}

// ---------------------------------------------------------------------------
// Coefficient tables (one thread per m)
// ---------------------------------------------------------------------------
__global__ void coef_spin0_kernel(int lmax, int mmax, const long long *__restrict__ moff,
                                  double *__restrict__ alpha, double *__restrict__ cfac) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m > mmax) return;
  const long long base = moff[m];
  const int L = lmax - m + 1;
  // f0[l], f1[l] as libsharp/sharp_ylmgen_c.c:160-168 (root/iroot products)
  double c_lm1 = 1.0, c_l = 1.0;  // c_{l-1}, c_l at l=m (c_{m-1} unused)
  for (int i = 0; i < L; ++i) {
    const int l = m + i;
    double f0, f1;
    if (l == m) {
      f0 = sqrt(double(2 * m + 3));
      f1 = 0.0;
    } else {
      const double tmp = sqrt(double(2 * l + 3)) * (1.0 / sqrt(double(l + 1 + m))) *
                         (1.0 / sqrt(double(l + 1 - m)));
      f0 = tmp * sqrt(double(2 * l + 1));
      f1 = tmp * sqrt(double(l + m)) * sqrt(double(l - m)) * (1.0 / sqrt(double(2 * l - 1)));
    }
    // c_{l+1} = f1[l] c_{l-1} (l >= m+1), c_{m+1} = 1
    const double c_lp1 = (l == m) ? 1.0 : f1 * c_lm1;
    cfac[base + i] = c_l;
    alpha[base + i] = (l < lmax) ? f0 * c_l / c_lp1 : 0.0;
    c_lm1 = c_l;
    c_l = c_lp1;
  }
  for (int i = L; i < L + kPad; ++i) {
    cfac[base + i] = 0.0;
    alpha[base + i] = 0.0;
  }
}

__global__ void coef_spin_kernel(int lmax, int mmax, int s, const long long *__restrict__ moff,
                                 double *__restrict__ a, double *__restrict__ b,
                                 double *__restrict__ cfac) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m > mmax) return;
  const long long base = moff[m];
  const int L = lmax - m + 1;
  const int mhi = max(m, s);
  for (int i = 0; i < L + kPad; ++i) {
    a[base + i] = 0.0;
    b[base + i] = 0.0;
    cfac[base + i] = 0.0;
  }
  // fx[l+1] for the step l -> l+1, libsharp/sharp_ylmgen_c.c:172-183
  double c_lm1 = 1.0, c_l = 1.0;
  for (int l = mhi; l <= lmax; ++l) {
    double fx0 = 0.0, fx1 = 0.0, fx2 = 0.0;
    if (l < lmax) {
      const double t = sqrt(1.0 / (l + m + 1.0)) * sqrt(1.0 / (l - m + 1.0)) *
                       sqrt(1.0 / (l + s + 1.0)) * sqrt(1.0 / (l - s + 1.0));
      fx0 = (l + 1.0) * (2 * l + 1.0) * t;
      fx1 = (l == 0) ? 0.0 : double(m) * s * (1.0 / l) * (1.0 / (l + 1.0));
      const double t2 = sqrt((l + m) / (l + m + 1.0)) * sqrt((l - m) / (l - m + 1.0)) *
                        sqrt((l + s) / (l + s + 1.0)) * sqrt((l - s) / (l - s + 1.0));
      fx2 = (l == 0) ? 0.0 : t2 * (l + 1.0) * (1.0 / l);
    }
    const double c_lp1 = (l == mhi) ? 1.0 : fx2 * c_lm1;
    const int i = l - m;
    cfac[base + i] = c_l;
    if (l < lmax) {
      const double al = fx0 * c_l / c_lp1;
      a[base + i] = al;
      b[base + i] = al * fx1;
    }
    c_lm1 = c_l;
    c_l = c_lp1;
  }
}

// ---------------------------------------------------------------------------
// Phase rows: phase[((p * ncm + comp) * 2 + hemisphere) * ms + m], ms = mmax+1
// (ring-major so the ring FFT reads and writes contiguous m runs).
// ---------------------------------------------------------------------------
__device__ __forceinline__ long long phase_row(int p, int ncm, int comp, int h, int ms) {
  return ((long long)(p * ncm + comp) * 2 + h) * ms;
}

// ---------------------------------------------------------------------------
// Coefficient staging.  Recurrence coefficients and staged a_lm are consumed
// in chunks of kChunk l-steps, copied global -> shared with cp.async into one
// of three buffers two chunks ahead of their use.  Synthesis warps stage
// privately (a __syncwarp publishes a chunk, no CTA barrier); analysis CTAs
// share the buffers and merge the publishing barrier with the one of their
// cross-warp reduction.  Inside a chunk all lanes read the same words.
// ---------------------------------------------------------------------------
constexpr int kChunk = 32;
constexpr int kWarps = 4;  // 128-thread CTAs

__device__ __forceinline__ void copy8(double *dst, const double *src) {
  __pipeline_memcpy_async(dst, src, sizeof(double));
}
__device__ __forceinline__ void copy16(double2 *dst, const double2 *src) {
  __pipeline_memcpy_async(dst, src, sizeof(double2));
}

// ---------------------------------------------------------------------------
// Spin-0 synthesis: phase_m(p) = sum_l lambda_lm(theta_p) a_lm, split into
// even (p1) and odd (p2) l-m; north = p1+p2, south = p1-p2.
// ---------------------------------------------------------------------------
template <int NT, int R>
__global__ void __launch_bounds__(128)
synth_spin0_kernel(const int2 *__restrict__ items, const int *__restrict__ count,
                   const double *__restrict__ cth, const double *__restrict__ sth,
                   const int *__restrict__ nph_ring, const long long *__restrict__ moff,
                   const double *__restrict__ alpha, const double *__restrict__ mfac,
                   const double2 *__restrict__ A, int ncA, int comp0, int lmax,
                   double2 *__restrict__ phase, int ncm, int pcomp0, int ms) {
  __shared__ double s_al[kWarps][3][kChunk];
  __shared__ double2 s_A[kWarps][3][kChunk * NT];
  const int2 it = items[blockIdx.x];
  const int m = it.x;
  const int cnt = count[m];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long mo = moff[m] - m;  // table index of l is mo + l
  const double *al = alpha + mo;
  const double2 *Am = A + mo * ncA + comp0;
  const int nchunks = (lmax - m + kChunk) / kChunk;
  auto stage = [&](int ch) {
    if (ch < nchunks) {
      const int lc = m + ch * kChunk;
      const int b = ch % 3;
      for (int t = lane; t < kChunk; t += 32) copy8(&s_al[w][b][t], al + lc + t);
      for (int t = lane; t < kChunk * NT; t += 32)
        copy16(&s_A[w][b][t], Am + (long long)(lc + t / NT) * ncA + t % NT);
    }
    __pipeline_commit();
  };
  stage(0);
  stage(1);

  double x[R], mu0[R], mu1[R];
  int E[R];
  bool act[R], live[R];
  double2 p1[R][NT], p2[R][NT];
  const double sgn_mfac = (m & 1) ? -mfac[m] : mfac[m];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int p = it.y * (128 * R) + r * 128 + threadIdx.x;
    const bool valid = p < cnt;
    x[r] = valid ? cth[p] : 0.0;
    XD sd = valid ? xd_pow(sth[p], m) : XD{0.0, 0};
    sd = xd_norm(sd.v * sgn_mfac, sd.e);
    mu0[r] = 0.0;
    mu1[r] = sd.v;
    E[r] = sd.e;
    live[r] = valid && sd.v != 0.0;
    act[r] = live[r] && E[r] >= -kSwitchExp;
    if (act[r]) mu1[r] = ldexp(mu1[r], E[r]);
#pragma unroll
    for (int j = 0; j < NT; ++j) p1[r][j] = p2[r][j] = make_double2(0.0, 0.0);
  }

  for (int ch = 0; ch < nchunks; ++ch) {
    __pipeline_wait_prior(1);
    __syncwarp();
    stage(ch + 2);
    const double *ca = s_al[w][ch % 3];
    const double2 *cA = s_A[w][ch % 3];
#pragma unroll
    for (int sb = 0; sb < kChunk; sb += kLBlock) {
#pragma unroll 4
      for (int i = sb; i < sb + kLBlock; i += 2) {
        const double a0 = ca[i], a1 = ca[i + 1];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const double nm = fma(a0 * x[r], mu1[r], -mu0[r]);
          const double nn = fma(a1 * x[r], nm, -mu1[r]);
          if (act[r]) {
#pragma unroll
            for (int j = 0; j < NT; ++j) {
              const double2 A0 = cA[i * NT + j], A1 = cA[(i + 1) * NT + j];
              p1[r][j].x = fma(mu1[r], A0.x, p1[r][j].x);
              p1[r][j].y = fma(mu1[r], A0.y, p1[r][j].y);
              p2[r][j].x = fma(nm, A1.x, p2[r][j].x);
              p2[r][j].y = fma(nm, A1.y, p2[r][j].y);
            }
          }
          mu0[r] = nm;
          mu1[r] = nn;
        }
      }
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if (live[r] && !act[r]) {
          live[r] = renorm_pair(mu1[r], mu0[r], E[r]);
          if (live[r] && E[r] >= -kSwitchExp) {
            mu1[r] = ldexp(mu1[r], E[r]);
            mu0[r] = ldexp(mu0[r], E[r]);
            act[r] = true;
          }
        }
      }
    }
  }

#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int p = it.y * (128 * R) + r * 128 + threadIdx.x;
    if (p >= cnt) continue;
    const bool has_s = nph_ring[2 * p + 1] > 0;
#pragma unroll
    for (int j = 0; j < NT; ++j) {
      const long long row = phase_row(p, ncm, pcomp0 + j, 0, ms);
      phase[row + m] = make_double2(p1[r][j].x + p2[r][j].x, p1[r][j].y + p2[r][j].y);
      if (has_s)
        phase[row + ms + m] = make_double2(p1[r][j].x - p2[r][j].x, p1[r][j].y - p2[r][j].y);
    }
  }
}

// ---------------------------------------------------------------------------
// Spin-s synthesis (DERIV=false: E/B -> Q/U; DERIV=true: a -> d/dtheta,
// d/dphi with spin-1 functions).  Two recurrences mu+ / mu- share a_l, b_l.
// ---------------------------------------------------------------------------
template <int NT, int R, bool DERIV>
__global__ void __launch_bounds__(128)
synth_spin_kernel(const int2 *__restrict__ items, const int *__restrict__ count,
                  const double *__restrict__ cth, const double *__restrict__ sth,
                  const int *__restrict__ nph_ring, const long long *__restrict__ moff,
                  const double *__restrict__ ca, const double *__restrict__ cb,
                  const double *__restrict__ pre_v, const int *__restrict__ pre_e, int s,
                  const double2 *__restrict__ A, int ncA, int comp0, int lmax,
                  double2 *__restrict__ phase, int ncm, int pcomp0, int ms) {
  constexpr int NA = DERIV ? 1 : 2;  // staged alm components per transform
  constexpr int NC = NA * NT;        // staged alm entries per l
  __shared__ double2 s_ab[kWarps][3][kChunk];  // (a_l, b_l)
  __shared__ double2 s_A[kWarps][3][kChunk * NC];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int2 it = items[blockIdx.x];
  const int m = it.x;
  const int cnt = count[m];
  const int mhi = max(m, s);
  const long long mo = moff[m] - m;
  const double *aa = ca + mo;
  const double *bb = cb + mo;
  const double2 *Am = A + mo * ncA + comp0;
  const int nchunks = (lmax - mhi + kChunk) / kChunk;
  auto stage = [&](int ch) {
    if (ch < nchunks) {
      const int lc = mhi + ch * kChunk;
      const int b = ch % 3;
      for (int t = lane; t < 2 * kChunk; t += 32) {
        double *dst = reinterpret_cast<double *>(&s_ab[w][b][t >> 1]) + (t & 1);
        copy8(dst, ((t & 1) ? bb : aa) + lc + (t >> 1));
      }
      for (int t = lane; t < kChunk * NC; t += 32)
        copy16(&s_A[w][b][t], Am + (long long)(lc + t / NC) * ncA + t % NC);
    }
    __pipeline_commit();
  };
  stage(0);
  stage(1);

  double x[R], mp0[R], mp1[R], mm0[R], mm1[R];
  int Ep[R], Em[R];
  bool act[R], live[R];
  double2 q1[R][NT], q2[R][NT], u1[R][NT], u2[R][NT];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int p = it.y * (128 * R) + r * 128 + threadIdx.x;
    const bool valid = p < cnt;
    x[r] = valid ? cth[p] : 0.0;
    live[r] = spin_start(valid, x[r], valid ? sth[p] : 0.0, m, s, pre_v[m], pre_e[m], mp0[r],
                         mp1[r], mm0[r], mm1[r], Ep[r], Em[r], act[r]);
#pragma unroll
    for (int j = 0; j < NT; ++j)
      q1[r][j] = q2[r][j] = u1[r][j] = u2[r][j] = make_double2(0.0, 0.0);
  }

  for (int ch = 0; ch < nchunks; ++ch) {
    __pipeline_wait_prior(1);
    __syncwarp();
    stage(ch + 2);
    const double2 *cab = s_ab[w][ch % 3];
    const double2 *cA = s_A[w][ch % 3];
#pragma unroll
    for (int sb = 0; sb < kChunk; sb += kLBlock) {
#pragma unroll 2
      for (int i = sb; i < sb + kLBlock; i += 2) {
        const double2 ab0 = cab[i], ab1 = cab[i + 1];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          // even offset from mhi: px = p1, py = p2
          if (act[r]) {
            const double lw = mp1[r] + mm1[r], lx = mm1[r] - mp1[r];
#pragma unroll
            for (int j = 0; j < NT; ++j) {
              const double2 G0 = cA[i * NC + NA * j];
              q1[r][j].x = fma(G0.x, lw, q1[r][j].x);
              q1[r][j].y = fma(G0.y, lw, q1[r][j].y);
              u2[r][j].x = fma(G0.y, lx, u2[r][j].x);
              u2[r][j].y = fma(-G0.x, lx, u2[r][j].y);
              if (!DERIV) {
                const double2 C0 = cA[i * NC + NA * j + 1];
                u1[r][j].x = fma(C0.x, lw, u1[r][j].x);
                u1[r][j].y = fma(C0.y, lw, u1[r][j].y);
                q2[r][j].x = fma(-C0.y, lx, q2[r][j].x);
                q2[r][j].y = fma(C0.x, lx, q2[r][j].y);
              }
            }
          }
          const double np_ = fma(fma(ab0.x, x[r], -ab0.y), mp1[r], -mp0[r]);
          const double nm_ = fma(fma(ab0.x, x[r], ab0.y), mm1[r], -mm0[r]);
          // odd offset: px = p2, py = p1
          if (act[r]) {
            const double lw = np_ + nm_, lx = nm_ - np_;
#pragma unroll
            for (int j = 0; j < NT; ++j) {
              const double2 G1 = cA[(i + 1) * NC + NA * j];
              q2[r][j].x = fma(G1.x, lw, q2[r][j].x);
              q2[r][j].y = fma(G1.y, lw, q2[r][j].y);
              u1[r][j].x = fma(G1.y, lx, u1[r][j].x);
              u1[r][j].y = fma(-G1.x, lx, u1[r][j].y);
              if (!DERIV) {
                const double2 C1 = cA[(i + 1) * NC + NA * j + 1];
                u2[r][j].x = fma(C1.x, lw, u2[r][j].x);
                u2[r][j].y = fma(C1.y, lw, u2[r][j].y);
                q1[r][j].x = fma(-C1.y, lx, q1[r][j].x);
                q1[r][j].y = fma(C1.x, lx, q1[r][j].y);
              }
            }
          }
          const double nnp = fma(fma(ab1.x, x[r], -ab1.y), np_, -mp1[r]);
          const double nnm = fma(fma(ab1.x, x[r], ab1.y), nm_, -mm1[r]);
          mp0[r] = np_;
          mp1[r] = nnp;
          mm0[r] = nm_;
          mm1[r] = nnm;
        }
      }
#pragma unroll
      for (int r = 0; r < R; ++r)
        spin_renorm(live[r], act[r], mp0[r], mp1[r], mm0[r], mm1[r], Ep[r], Em[r]);
    }
  }

  const double flip = ((mhi - m + s) & 1) ? -1.0 : 1.0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int p = it.y * (128 * R) + r * 128 + threadIdx.x;
    if (p >= cnt) continue;
    const bool has_s = nph_ring[2 * p + 1] > 0;
#pragma unroll
    for (int j = 0; j < NT; ++j) {
      const long long rq = phase_row(p, ncm, pcomp0 + 2 * j, 0, ms);
      const long long ru = phase_row(p, ncm, pcomp0 + 2 * j + 1, 0, ms);
      phase[rq + m] = make_double2(q1[r][j].x + q2[r][j].x, q1[r][j].y + q2[r][j].y);
      phase[ru + m] = make_double2(u1[r][j].x + u2[r][j].x, u1[r][j].y + u2[r][j].y);
      if (has_s) {
        phase[rq + ms + m] = make_double2(flip * (q1[r][j].x - q2[r][j].x),
                                          flip * (q1[r][j].y - q2[r][j].y));
        phase[ru + ms + m] = make_double2(flip * (u1[r][j].x - u2[r][j].x),
                                          flip * (u1[r][j].y - u2[r][j].y));
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Analysis.  One CTA of 128 threads per m loops over tiles of 128*R ring
// pairs.  Per l-block (LB steps, LB*VPL == 32 values) every lane accumulates
// its R rings' contributions; a warp transpose-reduction leaves one sum per
// lane, kept in a per-warp shared array for the whole chunk.  At the next
// chunk's barrier (the same one that publishes staged coefficients) warp 0
// adds the four warps' sums in a fixed order to Aout, which this CTA owns:
// no atomics, bitwise repeatable, one barrier per 32 l-steps.
// ---------------------------------------------------------------------------
template <int VPL>
__device__ __forceinline__ void flush_chunk(const double (*wred)[kChunk * VPL / 32][32], int lane,
                                            int l0, long long mo, int ncA, int comp0,
                                            double *__restrict__ Aout) {
  constexpr int LB = 32 / VPL;
#pragma unroll 1
  for (int sb = 0; sb < kChunk / LB; ++sb) {
    const double acc = (wred[0][sb][lane] + wred[1][sb][lane]) +
                       (wred[2][sb][lane] + wred[3][sb][lane]);
    const int l = l0 + sb * LB + lane / VPL;
    Aout[((mo + l) * ncA + comp0) * 2 + lane % VPL] += acc;
  }
}

template <int NT, int R>
__global__ void __launch_bounds__(128)
anal_spin0_kernel(const int *__restrict__ count, const double *__restrict__ cth,
                  const double *__restrict__ sth, const int *__restrict__ nph_ring,
                  const long long *__restrict__ moff, const double *__restrict__ alpha,
                  const double *__restrict__ mfac, const double2 *__restrict__ phase, int ncm,
                  int pcomp0, int lmax, int ms, double *__restrict__ Aout, int ncA,
                  int comp0) {
  constexpr int VPL = 2 * NT;
  constexpr int LB = 32 / VPL;
  constexpr int NSB = kChunk / LB;
  static_assert(LB % 2 == 0 && kChunk % LB == 0, "l-block must be even and divide a chunk");
  __shared__ double wred[2][kWarps][NSB][32];
  __shared__ double s_al[3][kChunk];
  const int m = blockIdx.x;
  const int cnt = count[m];
  const long long mo = moff[m] - m;
  const double *al = alpha + mo;
  const double sgn_mfac = (m & 1) ? -mfac[m] : mfac[m];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nchunks = (lmax - m + kChunk) / kChunk;
  auto stage = [&](int ch) {
    if (ch < nchunks)
      for (int t = threadIdx.x; t < kChunk; t += blockDim.x)
        copy8(&s_al[ch % 3][t], al + m + ch * kChunk + t);
    __pipeline_commit();
  };

  for (int tb = 0; tb < cnt; tb += 128 * R) {
    stage(0);
    stage(1);
    double x[R], mu0[R], mu1[R];
    int E[R];
    bool act[R], live[R];
    double2 P1[R][NT], P2[R][NT];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int p = tb + r * 128 + threadIdx.x;
      const bool valid = p < cnt;
      x[r] = valid ? cth[p] : 0.0;
      XD sd = valid ? xd_pow(sth[p], m) : XD{0.0, 0};
      sd = xd_norm(sd.v * sgn_mfac, sd.e);
      mu0[r] = 0.0;
      mu1[r] = sd.v;
      E[r] = sd.e;
      live[r] = valid && sd.v != 0.0;
      act[r] = live[r] && E[r] >= -kSwitchExp;
      if (act[r]) mu1[r] = ldexp(mu1[r], E[r]);
      const bool has_s = valid && nph_ring[2 * p + 1] > 0;
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        const long long row = phase_row(valid ? p : 0, ncm, pcomp0 + j, 0, ms);
        const double2 n = valid ? phase[row + m] : make_double2(0.0, 0.0);
        const double2 sv = has_s ? phase[row + ms + m] : make_double2(0.0, 0.0);
        P1[r][j] = make_double2(n.x + sv.x, n.y + sv.y);
        P2[r][j] = make_double2(n.x - sv.x, n.y - sv.y);
      }
    }

    for (int ch = 0; ch < nchunks; ++ch) {
      __pipeline_wait_prior(1);
      __syncthreads();
      stage(ch + 2);
      if (ch > 0 && warp == 0)
        flush_chunk<VPL>(wred[(ch - 1) & 1], lane, m + (ch - 1) * kChunk, mo, ncA, comp0, Aout);
      const double *ca = s_al[ch % 3];
#pragma unroll 1
      for (int sb = 0; sb < NSB; ++sb) {
        double v[32];
#pragma unroll
        for (int k = 0; k < 32; ++k) v[k] = 0.0;
        bool any = false;
#pragma unroll
        for (int i = 0; i < LB; i += 2) {
          const double a0 = ca[sb * LB + i], a1 = ca[sb * LB + i + 1];
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const double nm = fma(a0 * x[r], mu1[r], -mu0[r]);
            const double nn = fma(a1 * x[r], nm, -mu1[r]);
            if (act[r]) {
#pragma unroll
              for (int j = 0; j < NT; ++j) {
                v[i * VPL + 2 * j] = fma(mu1[r], P1[r][j].x, v[i * VPL + 2 * j]);
                v[i * VPL + 2 * j + 1] = fma(mu1[r], P1[r][j].y, v[i * VPL + 2 * j + 1]);
                v[(i + 1) * VPL + 2 * j] = fma(nm, P2[r][j].x, v[(i + 1) * VPL + 2 * j]);
                v[(i + 1) * VPL + 2 * j + 1] =
                    fma(nm, P2[r][j].y, v[(i + 1) * VPL + 2 * j + 1]);
              }
            }
            mu0[r] = nm;
            mu1[r] = nn;
          }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
          any |= act[r];
          if (live[r] && !act[r] && ((sb + 1) * LB) % kLBlock == 0) {
            live[r] = renorm_pair(mu1[r], mu0[r], E[r]);
            if (live[r] && E[r] >= -kSwitchExp) {
              mu1[r] = ldexp(mu1[r], E[r]);
              mu0[r] = ldexp(mu0[r], E[r]);
              act[r] = true;
            }
          }
        }
        wred[ch & 1][warp][sb][lane] =
            __any_sync(0xffffffffu, any) ? warp_transpose_reduce32(v) : 0.0;
      }
    }
    __pipeline_wait_prior(0);
    __syncthreads();
    if (warp == 0)
      flush_chunk<VPL>(wred[(nchunks - 1) & 1], lane, m + (nchunks - 1) * kChunk, mo, ncA, comp0,
                       Aout);
    __syncthreads();
  }
}

// Spin-s analysis (E/B from Q/U): per l, (G.re, G.im, C.re, C.im) per
// transform (saddstep2, libsharp/sharp_core_inc2.c:338-364), written directly
// in terms of mu+ and mu- (lw = mu+ + mu-, lx = mu- - mu+):
//   lw X - lx Y = mu+ (X+Y) + mu- (X-Y),   lw X + lx Y = mu+ (X-Y) + mu- (X+Y)
// so each output takes 2 FMAs and lw, lx are never formed.  H?p / H?m hold
// the combined phase factors of mu+ / mu- for even (e) and odd (o) l-mhi.
template <int NT, int R>
__global__ void __launch_bounds__(128)
anal_spin_kernel(const int *__restrict__ count, const double *__restrict__ cth,
                 const double *__restrict__ sth, const int *__restrict__ nph_ring,
                 const long long *__restrict__ moff, const double *__restrict__ ca,
                 const double *__restrict__ cb, const double *__restrict__ pre_v,
                 const int *__restrict__ pre_e, int s, const double2 *__restrict__ phase,
                 int ncm, int pcomp0, int lmax, int ms, double *__restrict__ Aout, int ncA,
                 int comp0) {
  constexpr int VPL = 4 * NT;
  constexpr int LB = 32 / VPL;
  constexpr int NSB = kChunk / LB;
  static_assert(LB % 2 == 0 && kChunk % LB == 0, "l-block must be even and divide a chunk");
  __shared__ double wred[2][kWarps][NSB][32];
  __shared__ double2 s_ab[3][kChunk];
  const int m = blockIdx.x;
  const int cnt = count[m];
  const int mhi = max(m, s);
  const long long mo = moff[m] - m;
  const double *aa = ca + mo;
  const double *bb = cb + mo;
  const double flip = ((mhi - m + s) & 1) ? -1.0 : 1.0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nchunks = (lmax - mhi + kChunk) / kChunk;
  auto stage = [&](int ch) {
    if (ch < nchunks)
      for (int t = threadIdx.x; t < 2 * kChunk; t += blockDim.x) {
        double *dst = reinterpret_cast<double *>(&s_ab[ch % 3][t >> 1]) + (t & 1);
        copy8(dst, ((t & 1) ? bb : aa) + mhi + ch * kChunk + (t >> 1));
      }
    __pipeline_commit();
  };

  for (int tb = 0; tb < cnt; tb += 128 * R) {
    stage(0);
    stage(1);
    double x[R], mp0[R], mp1[R], mm0[R], mm1[R];
    int Ep[R], Em[R];
    bool act[R], live[R];
    // [r][j][k]: k = G.re, G.im, C.re, C.im
    double Hep[R][NT][4], Hem[R][NT][4], Hop[R][NT][4], Hom[R][NT][4];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int p = tb + r * 128 + threadIdx.x;
      const bool valid = p < cnt;
      x[r] = valid ? cth[p] : 0.0;
      live[r] = spin_start(valid, x[r], valid ? sth[p] : 0.0, m, s, pre_v[m], pre_e[m],
                           mp0[r], mp1[r], mm0[r], mm1[r], Ep[r], Em[r], act[r]);
      const bool has_s = valid && nph_ring[2 * p + 1] > 0;
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        const long long rq = phase_row(valid ? p : 0, ncm, pcomp0 + 2 * j, 0, ms);
        const long long ru = phase_row(valid ? p : 0, ncm, pcomp0 + 2 * j + 1, 0, ms);
        const double2 qn = valid ? phase[rq + m] : make_double2(0.0, 0.0);
        const double2 un = valid ? phase[ru + m] : make_double2(0.0, 0.0);
        double2 qs = has_s ? phase[rq + ms + m] : make_double2(0.0, 0.0);
        double2 us = has_s ? phase[ru + ms + m] : make_double2(0.0, 0.0);
        qs.x *= flip; qs.y *= flip; us.x *= flip; us.y *= flip;
        const double2 P1q = make_double2(qn.x + qs.x, qn.y + qs.y);
        const double2 P2q = make_double2(qn.x - qs.x, qn.y - qs.y);
        const double2 P1u = make_double2(un.x + us.x, un.y + us.y);
        const double2 P2u = make_double2(un.x - us.x, un.y - us.y);
        // even offset: px = p1, py = p2
        //   G.re = lw P1q.re - lx P2u.im   G.im = lw P1q.im + lx P2u.re
        //   C.re = lw P1u.re + lx P2q.im   C.im = lw P1u.im - lx P2q.re
        Hep[r][j][0] = P1q.x + P2u.y; Hem[r][j][0] = P1q.x - P2u.y;
        Hep[r][j][1] = P1q.y - P2u.x; Hem[r][j][1] = P1q.y + P2u.x;
        Hep[r][j][2] = P1u.x - P2q.y; Hem[r][j][2] = P1u.x + P2q.y;
        Hep[r][j][3] = P1u.y + P2q.x; Hem[r][j][3] = P1u.y - P2q.x;
        // odd offset: px = p2, py = p1
        Hop[r][j][0] = P2q.x + P1u.y; Hom[r][j][0] = P2q.x - P1u.y;
        Hop[r][j][1] = P2q.y - P1u.x; Hom[r][j][1] = P2q.y + P1u.x;
        Hop[r][j][2] = P2u.x - P1q.y; Hom[r][j][2] = P2u.x + P1q.y;
        Hop[r][j][3] = P2u.y + P1q.x; Hom[r][j][3] = P2u.y - P1q.x;
      }
    }

    for (int ch = 0; ch < nchunks; ++ch) {
      __pipeline_wait_prior(1);
      __syncthreads();
      stage(ch + 2);
      if (ch > 0 && warp == 0)
        flush_chunk<VPL>(wred[(ch - 1) & 1], lane, mhi + (ch - 1) * kChunk, mo, ncA, comp0,
                         Aout);
      const double2 *cab = s_ab[ch % 3];
#pragma unroll 1
      for (int sb = 0; sb < NSB; ++sb) {
        double v[32];
#pragma unroll
        for (int k = 0; k < 32; ++k) v[k] = 0.0;
        bool any = false;
#pragma unroll
        for (int i = 0; i < LB; i += 2) {
          const double2 ab0 = cab[sb * LB + i], ab1 = cab[sb * LB + i + 1];
#pragma unroll
          for (int r = 0; r < R; ++r) {
            if (act[r]) {
#pragma unroll
              for (int j = 0; j < NT; ++j)
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                  double &o = v[i * VPL + 4 * j + k];
                  o = fma(mp1[r], Hep[r][j][k], fma(mm1[r], Hem[r][j][k], o));
                }
            }
            const double np_ = fma(fma(ab0.x, x[r], -ab0.y), mp1[r], -mp0[r]);
            const double nm_ = fma(fma(ab0.x, x[r], ab0.y), mm1[r], -mm0[r]);
            if (act[r]) {
#pragma unroll
              for (int j = 0; j < NT; ++j)
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                  double &o = v[(i + 1) * VPL + 4 * j + k];
                  o = fma(np_, Hop[r][j][k], fma(nm_, Hom[r][j][k], o));
                }
            }
            const double nnp = fma(fma(ab1.x, x[r], -ab1.y), np_, -mp1[r]);
            const double nnm = fma(fma(ab1.x, x[r], ab1.y), nm_, -mm1[r]);
            mp0[r] = np_;
            mp1[r] = nnp;
            mm0[r] = nm_;
            mm1[r] = nnm;
          }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
          any |= act[r];
          if (((sb + 1) * LB) % kLBlock == 0)
            spin_renorm(live[r], act[r], mp0[r], mp1[r], mm0[r], mm1[r], Ep[r], Em[r]);
        }
        wred[ch & 1][warp][sb][lane] =
            __any_sync(0xffffffffu, any) ? warp_transpose_reduce32(v) : 0.0;
      }
    }
    __pipeline_wait_prior(0);
    __syncthreads();
    if (warp == 0)
      flush_chunk<VPL>(wred[(nchunks - 1) & 1], lane, mhi + (nchunks - 1) * kChunk, mo, ncA,
                       comp0, Aout);
    __syncthreads();
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
void launch_coef_tables(CoefPlan &cp, cudaStream_t st) {
  ProfScope ps("coef_tables", st);
  const int threads = 128;
  const int blocks = (cp.mmax + 1 + threads - 1) / threads;
  if (cp.spin == 0)
    coef_spin0_kernel<<<blocks, threads, 0, st>>>(cp.lmax, cp.mmax, cp.d_moff, cp.alpha, cp.cfac);
  else
    coef_spin_kernel<<<blocks, threads, 0, st>>>(cp.lmax, cp.mmax, cp.spin, cp.d_moff, cp.alpha,
                                                 cp.beta, cp.cfac);
  SHT_CUDA(cudaGetLastError());
}

void launch_legendre_synth(const JobDesc &job, const GeomPlan &gp, const CoefPlan &cp,
                           const double2 *A, int ncA, int comp0, int nt, double2 *phase,
                           int ncm, int pcomp0, cudaStream_t st) {
  const int nitems = int(gp.synth_items.size());
  if (nitems == 0) return;
  ProfScope ps("legendre_synth", st);
  constexpr int R = 2;
  SHT_REQUIRE(gp.synth_tile == 128 * R, "synthesis tile mismatch");
  const bool deriv = job.type == SHARP_ALM2MAP_DERIV1;
  if (job.spin == 0 && !deriv) {
#define SHT_S0(NTV)                                                                           \
  synth_spin0_kernel<NTV, R><<<nitems, 128, 0, st>>>(                                         \
      gp.items, gp.count, gp.cth, gp.sth, gp.nph, cp.d_moff, cp.alpha, cp.seed, A, ncA, comp0, \
      job.lmax, phase, ncm, pcomp0, job.mmax + 1)
    if (nt == 1) SHT_S0(1);
    else if (nt == 2) SHT_S0(2);
    else SHT_S0(4);
#undef SHT_S0
  } else {
#define SHT_SS(NTV, DV)                                                                         \
  synth_spin_kernel<NTV, R, DV><<<nitems, 128, 0, st>>>(                                        \
      gp.items, gp.count, gp.cth, gp.sth, gp.nph, cp.d_moff, cp.alpha, cp.beta, cp.seed,        \
      cp.seed_exp, cp.spin, A, ncA, comp0, job.lmax, phase, ncm, pcomp0, job.mmax + 1)
    if (deriv) {
      if (nt == 1) SHT_SS(1, true);
      else SHT_SS(2, true);
    } else {
      if (nt == 1) SHT_SS(1, false);
      else SHT_SS(2, false);
    }
#undef SHT_SS
  }
  SHT_CUDA(cudaGetLastError());
}

void launch_legendre_anal(const JobDesc &job, const GeomPlan &gp, const CoefPlan &cp,
                          const double2 *phase, int ncm, int pcomp0, int nt, double *Aout,
                          int ncA, int comp0, cudaStream_t st) {
  const int nblocks = job.mmax + 1;
  ProfScope ps("legendre_anal", st);
  if (job.spin == 0) {
#define SHT_A0(NTV)                                                                       \
  anal_spin0_kernel<NTV, 4><<<nblocks, 128, 0, st>>>(                                     \
      gp.count, gp.cth, gp.sth, gp.nph, cp.d_moff, cp.alpha, cp.seed, phase, ncm, pcomp0, \
      job.lmax, job.mmax + 1, Aout, ncA, comp0)
    if (nt == 1) SHT_A0(1);
    else if (nt == 2) SHT_A0(2);
    else SHT_A0(4);
#undef SHT_A0
  } else {
#define SHT_AS(NTV)                                                                        \
  anal_spin_kernel<NTV, 2><<<nblocks, 128, 0, st>>>(                                       \
      gp.count, gp.cth, gp.sth, gp.nph, cp.d_moff, cp.alpha, cp.beta, cp.seed, cp.seed_exp, \
      cp.spin, phase, ncm, pcomp0, job.lmax, job.mmax + 1, Aout, ncA, comp0)
    if (nt == 1) SHT_AS(1);
    else SHT_AS(2);
#undef SHT_AS
  }
  SHT_CUDA(cudaGetLastError());
}

}  // namespace sht
