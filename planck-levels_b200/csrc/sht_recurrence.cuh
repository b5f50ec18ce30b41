// Exponent-tracked seeds shared by the FP64 and mixed-precision Legendre
// kernels (device-only, internal linkage in each translation unit).
#pragma once

#include <cuda_runtime.h>

#include "sht_internal.h"

namespace sht {
namespace {

// ---------------------------------------------------------------------------
// (mantissa, exponent) numbers for the seeds
// ---------------------------------------------------------------------------
struct XD {
  double v;  // |v| in [0.5,1) or 0
  int e;
};

__device__ __forceinline__ XD xd_norm(double v, int e) {
  int k;
  double mnt = frexp(v, &k);
  return {mnt, e + k};
}

__device__ __forceinline__ XD xd_mul(XD a, XD b) { return xd_norm(a.v * b.v, a.e + b.e); }

__device__ XD xd_pow(double base, int n) {
  XD r{1.0, 0};
  XD b = xd_norm(base, 0);
  while (n) {
    if (n & 1) r = xd_mul(r, b);
    n >>= 1;
    if (n) b = xd_mul(b, b);
  }
  return xd_norm(r.v, r.e);
}

// Renormalises a scaled pair (mu_cur, mu_prev) * 2^E so that the larger one
// lies in [0.5,1); returns false if both are zero.
__device__ __forceinline__ bool renorm_pair(double &cur, double &prev, int &E) {
  double big = fmax(fabs(cur), fabs(prev));
  if (big == 0.0) return false;
  int k;
  frexp(big, &k);
  cur = ldexp(cur, -k);
  prev = ldexp(prev, -k);
  E += k;
  return true;
}

// ---------------------------------------------------------------------------
// Spin-s seeds: the two Wigner-d recurrences mu+ / mu- of one ring start at
// l = max(m, s) from (cos(theta/2), sin(theta/2)) powers and a per-m
// prefactor, as exponent-tracked numbers.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void spin_seed(double cth, double sth, int m, int s, double pre_v,
                                          int pre_e, XD &sp, XD &sm) {
  // libsharp/sharp_core_inc.c:223-271 and sharp_ylmgen_c.c:186-196
  double c2 = fmax(sqrt((1.0 + cth) * 0.5), 1e-15);
  double s2 = fmax(sqrt((1.0 - cth) * 0.5), 1e-15);
  if (sth < 0.0) {
    if (cth < 0.0) c2 = -c2;
    if (cth > 0.0) s2 = -s2;
  }
  const int mhi = max(m, s);
  int cosPow, sinPow;
  bool preMinus_p, preMinus_m;
  if (mhi == m) {
    cosPow = mhi + s;
    sinPow = mhi - s;
    preMinus_p = preMinus_m = ((mhi - s) & 1) != 0;
  } else {
    cosPow = mhi + m;
    sinPow = mhi - m;
    preMinus_p = false;
    preMinus_m = ((mhi + m) & 1) != 0;
  }
  const XD pre{pre_v, pre_e};
  sp = xd_mul(xd_mul(pre, xd_pow(c2, cosPow)), xd_pow(s2, sinPow));
  sm = xd_mul(xd_mul(pre, xd_pow(c2, sinPow)), xd_pow(s2, cosPow));
  if (preMinus_p) sp.v = -sp.v;
  if (preMinus_m) sm.v = -sm.v;
  if (s & 1) sp.v = -sp.v;
}

// Starts the two spin recurrences of one ring; returns whether it is live.
__device__ __forceinline__ bool spin_start(bool valid, double x, double sth, int m, int s,
                                           double pre_v, int pre_e, double &mp0, double &mp1,
                                           double &mm0, double &mm1, int &Ep, int &Em,
                                           bool &act) {
  XD sp{0.0, 0}, sm{0.0, 0};
  if (valid) spin_seed(x, sth, m, s, pre_v, pre_e, sp, sm);
  mp0 = mm0 = 0.0;
  mp1 = sp.v;
  mm1 = sm.v;
  Ep = sp.e;
  Em = sm.e;
  const bool live = valid && (sp.v != 0.0 || sm.v != 0.0);
  const int emax = max(sp.v != 0.0 ? Ep : -0x3fffffff, sm.v != 0.0 ? Em : -0x3fffffff);
  act = live && emax >= -kSwitchExp;
  if (act) {
    mp1 = ldexp(mp1, Ep);
    mm1 = ldexp(mm1, Em);
  }
  return live;
}

// ---------------------------------------------------------------------------
// Seeds from base-2 logarithms, for the mixed-precision kernels: a product of
// powers b_i^k_i is formed as 2^L, L = sum k_i log2|b_i|, and split into a
// mantissa 2^(L - E) in [0.5, 1) and the exponent E.  The relative error is
// about |L| 2^-52 (below 1e-11 for powers up to 8192), far below the 2^-30
// quantisation step of the mixed contraction, at a fraction of the cost of
// the exact square-and-multiply seeds.
// ---------------------------------------------------------------------------
__device__ __forceinline__ XD xd_from_log2(double L, bool neg) {
  const double e = floor(L) + 1.0;
  const double v = exp2(L - e);
  return xd_norm(neg ? -v : v, int(e));
}

// sign * |pre| * |base|^k as an exponent-tracked number (zero if pre or a
// positive power of a zero base vanishes)
__device__ __forceinline__ XD xd_pow_log(double base, int k, double pre) {
  if (pre == 0.0 || (k > 0 && base == 0.0)) return XD{0.0, 0};
  const double L = (k > 0 ? k * log2(fabs(base)) : 0.0) + log2(fabs(pre));
  return xd_from_log2(L, (pre < 0.0) != (base < 0.0 && (k & 1)));
}

// spin_start with the seeds of spin_seed formed from logarithms
__device__ __forceinline__ bool spin_start_log(bool valid, double x, double sth, int m, int s,
                                               double pre_v, int pre_e, double &mp0,
                                               double &mp1, double &mm0, double &mm1, int &Ep,
                                               int &Em, bool &act) {
  XD sp{0.0, 0}, sm{0.0, 0};
  if (valid && pre_v != 0.0) {
    double c2 = fmax(sqrt((1.0 + x) * 0.5), 1e-15);
    double s2 = fmax(sqrt((1.0 - x) * 0.5), 1e-15);
    if (sth < 0.0) {
      if (x < 0.0) c2 = -c2;
      if (x > 0.0) s2 = -s2;
    }
    const int mhi = max(m, s);
    int cosPow, sinPow;
    bool preMinus_p, preMinus_m;
    if (mhi == m) {
      cosPow = mhi + s;
      sinPow = mhi - s;
      preMinus_p = preMinus_m = ((mhi - s) & 1) != 0;
    } else {
      cosPow = mhi + m;
      sinPow = mhi - m;
      preMinus_p = false;
      preMinus_m = ((mhi + m) & 1) != 0;
    }
    const double lc = log2(fabs(c2)), ls = log2(fabs(s2));
    const double lp = log2(fabs(pre_v)) + pre_e;
    const bool npre = pre_v < 0.0, nc = c2 < 0.0, ns = s2 < 0.0;
    const bool negp = npre ^ (nc && (cosPow & 1)) ^ (ns && (sinPow & 1)) ^ preMinus_p ^ (s & 1);
    const bool negm = npre ^ (nc && (sinPow & 1)) ^ (ns && (cosPow & 1)) ^ preMinus_m;
    sp = xd_from_log2(lp + cosPow * lc + sinPow * ls, negp);
    sm = xd_from_log2(lp + sinPow * lc + cosPow * ls, negm);
  }
  mp0 = mm0 = 0.0;
  mp1 = sp.v;
  mm1 = sm.v;
  Ep = sp.e;
  Em = sm.e;
  const bool live = valid && (sp.v != 0.0 || sm.v != 0.0);
  const int emax = max(sp.v != 0.0 ? Ep : -0x3fffffff, sm.v != 0.0 ? Em : -0x3fffffff);
  act = live && emax >= -kSwitchExp;
  if (act) {
    mp1 = ldexp(mp1, Ep);
    mm1 = ldexp(mm1, Em);
  }
  return live;
}

// End-of-block bookkeeping of a ring still in the scaled (skip) regime.
__device__ __forceinline__ void spin_renorm(bool &live, bool &act, double &mp0, double &mp1,
                                            double &mm0, double &mm1, int &Ep, int &Em) {
  if (!live || act) return;
  const bool lp = renorm_pair(mp1, mp0, Ep);
  const bool lm = renorm_pair(mm1, mm0, Em);
  live = lp || lm;
  const int emax = max(lp ? Ep : -0x3fffffff, lm ? Em : -0x3fffffff);
  if (live && emax >= -kSwitchExp) {
    mp1 = ldexp(mp1, Ep);
    mp0 = ldexp(mp0, Ep);
    mm1 = ldexp(mm1, Em);
    mm0 = ldexp(mm0, Em);
    act = true;
  }
}

}  // namespace
}  // namespace sht
