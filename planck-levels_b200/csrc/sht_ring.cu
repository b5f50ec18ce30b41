// Ring stage of the transform: phase <-> ring pixels with the per-ring real
// FFT, phi0 rotation, quadrature weight and alias folding, plus the a_lm
// staging/scatter kernels.
//
// Reference behaviour: libsharp/sharp.c:253-353 (ringhelper_phase2ring /
// ring2phase), :481-606 (alm2almtmp / almtmp2alm), :608-669 (ring gathers
// and the SHARP_NO_FFT path); FFT conventions of libfftpack/ls_fft.c:130-212
// (unnormalised backward transform, FFTPACK half-complex order).
//
// Three kernel families, chosen per ring pair when the geometry plan is built:
//  * power-of-two rings (2N pixels, N = 1024 .. 8192, no alias folding): one
//    CTA per ring and component, radix-16 passes in registers
//    (phase2ring_pow2_kernel / ring2phase_pow2_kernel);
//  * long even rings that need a Bluestein convolution of length M = 1024 ..
//    8192 (the polar HEALPix rings): the same register passes around the
//    chirp product (phase2ring_blue_kernel / ring2phase_blue_kernel);
//  * all other rings, in size classes (phase2ring_kernel / ring2phase_kernel),
//    described here.
//
// Size classes: one CTA owns one (ring pair, component) and runs both
// hemispheres.  The FFT
// is a Stockham auto-sort mixed-radix transform in shared memory: even ring
// lengths n use a complex FFT of length n/2 on packed (x_2j + i x_2j+1) data;
// odd lengths a complex FFT of length n.  Radix-2/3/4/5/8 stages and a generic
// prime stage share one code path (each thread computes whole outputs, so
// large prime factors parallelise over outputs).  Twiddles come from a
// per-length table exp(-2 pi i j/n) computed once per geometry; each ring
// copies two short slices of it into shared memory (e mod 64 and 64 (e/64))
// and forms exp(-2 pi i e/n) as their product, so no butterfly waits on a
// global load.  Lengths with large prime factors use a power-of-two
// Bluestein convolution in place (run_bluestein).  The buffers are indexed
// through Buf, which swizzles entries inside blocks of 8 so that the
// butterflies' power-of-two strided accesses do not share bank groups.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "sht_device.h"
#include "sht_tc.cuh"   // mbarriers and bulk copies

namespace sht {

namespace {

constexpr double kSqrtHalf = 0.707106781186547572737310929369;
constexpr double kSqrtTwo = 1.414213562373095145474621858739;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) {
  return make_double2(a.x * s, a.y * s);
}
// FFT buffer (shared memory, or a CTA's slot of global scratch) whose element
// index is swizzled inside aligned blocks of 8 entries (16-byte units):
// e -> e ^ ((e >> 3) & 7).  The butterflies' strided stores (2, 4 or 8
// entries apart) and contiguous runs then spread over the bank groups of a
// 128-byte wavefront.  The map permutes each block, so a buffer of a
// multiple of 8 entries holds the indices [0, size); elementwise work on
// two buffers stored the same way may index them directly.
struct Buf {
  double2 *p;
  __device__ __forceinline__ double2 &operator[](int e) const { return p[e ^ ((e >> 3) & 7)]; }
};

// exp(-2 pi i e/n), 0 <= e < n, read from the per-length global table
struct TwGlobal {
  const double2 *__restrict__ W;
  __device__ __forceinline__ double2 operator()(int e) const { return __ldg(W + e); }
};
// the same from two shared-memory slices: lo[e mod 64] * hi[e / 64]
constexpr int kTwLo = 64;
struct TwShared {
  const double2 *lo, *hi;
  __device__ __forceinline__ double2 operator()(int e) const {
    return cmul(hi[e >> 6], lo[e & (kTwLo - 1)]);
  }
};
// Copies the slices of the table W (n entries) into lo (64) and hi (n/64 + 1).
__device__ void load_twshared(double2 *lo, double2 *hi, const double2 *__restrict__ W, int n) {
  const int nhi = (n + kTwLo - 1) / kTwLo;
  for (int t = threadIdx.x; t < kTwLo + nhi; t += blockDim.x) {
    if (t < kTwLo) lo[t] = t < n ? __ldg(W + t) : make_double2(1.0, 0.0);
    else hi[t - kTwLo] = __ldg(W + kTwLo * (t - kTwLo));
  }
}

// ---------------------------------------------------------------------------
// Stockham auto-sort passes.  For radix R and Ns = product of the radices
// already applied, butterfly j (0 <= j < N/R, k = j mod Ns) reads
// x_r = src[j + r N/R], twiddles x_r *= w_N^{+-r k N/(Ns R)}, applies the
// R-point DFT and writes y_q to dst[(j - k) R + k + q Ns].
// ---------------------------------------------------------------------------
constexpr double kC5a = 0.30901699437494742410;   // cos(2 pi/5)
constexpr double kC5b = -0.80901699437494742410;  // cos(4 pi/5)
constexpr double kS5a = 0.95105651629515357212;   // sin(2 pi/5)
constexpr double kS5b = 0.58778525229247312917;   // sin(4 pi/5)
constexpr double kS3 = 0.86602540378443864676;    // sin(2 pi/3)
constexpr double kR2 = 0.70710678118654752440;    // cos(pi/4)

__device__ __forceinline__ double2 mul_i(double2 a) { return make_double2(-a.y, a.x); }

template <int R>
__device__ __forceinline__ void small_dft(double2 (&v)[R], bool inv) {
  if constexpr (R == 2) {
    const double2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (R == 4) {
    const double2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
    const double2 c = cadd(v[1], v[3]), d = csub(v[1], v[3]);
    const double2 id = mul_i(d);  // i d
    v[0] = cadd(a, c);
    v[2] = csub(a, c);
    v[1] = inv ? cadd(b, id) : csub(b, id);
    v[3] = inv ? csub(b, id) : cadd(b, id);
  } else if constexpr (R == 3) {
    const double2 t = cadd(v[1], v[2]);
    const double2 u = make_double2(v[0].x - 0.5 * t.x, v[0].y - 0.5 * t.y);
    const double2 d = cscale(mul_i(csub(v[1], v[2])), inv ? kS3 : -kS3);
    v[0] = cadd(v[0], t);
    v[1] = cadd(u, d);
    v[2] = csub(u, d);
  } else if constexpr (R == 8) {
    // 8 = 2 x 4: DFT-2 over n1 of x[4 n1 + n2], twiddles w8^n2 on the odd
    // outputs, DFT-4 over n2; output X[k1 + 2 k2]
    double2 a0[4], a1[4];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
      a0[n2] = cadd(v[n2], v[n2 + 4]);
      a1[n2] = csub(v[n2], v[n2 + 4]);
    }
    const double sg = inv ? 1.0 : -1.0;   // w8^e = (cos(e pi/4), sg sin(e pi/4))
    a1[1] = cmul(a1[1], make_double2(kR2, sg * kR2));
    a1[2] = make_double2(-sg * a1[2].y, sg * a1[2].x);     // times (0, sg)
    a1[3] = cmul(a1[3], make_double2(-kR2, sg * kR2));
    small_dft<4>(a0, inv);
    small_dft<4>(a1, inv);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) {
      v[2 * k2] = a0[k2];
      v[2 * k2 + 1] = a1[k2];
    }
  } else if constexpr (R == 5) {
    const double2 a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
    const double2 a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
    const double2 x0 = v[0];
    const double2 r1 = make_double2(x0.x + kC5a * a1.x + kC5b * a2.x, x0.y + kC5a * a1.y + kC5b * a2.y);
    const double2 r2 = make_double2(x0.x + kC5b * a1.x + kC5a * a2.x, x0.y + kC5b * a1.y + kC5a * a2.y);
    const double sg = inv ? 1.0 : -1.0;
    const double2 i1 = cscale(mul_i(make_double2(kS5a * b1.x + kS5b * b2.x, kS5a * b1.y + kS5b * b2.y)), sg);
    const double2 i2 = cscale(mul_i(make_double2(kS5b * b1.x - kS5a * b2.x, kS5b * b1.y - kS5a * b2.y)), sg);
    v[0] = make_double2(x0.x + a1.x + a2.x, x0.y + a1.y + a2.y);
    v[1] = cadd(r1, i1);
    v[4] = csub(r1, i1);
    v[2] = cadd(r2, i2);
    v[3] = csub(r2, i2);
  }
}

template <int R, class TW>
__device__ void stockham_small(Buf src, Buf dst, int N, int Ns, bool inv,
                               const TW &tw, int step) {
  const int NR = N / R;
  const int sf = N / (Ns * R);
  for (int j = threadIdx.x; j < NR; j += blockDim.x) {
    const int k = j % Ns;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[j + r * NR];
    if (Ns > 1) {
      // w^r for r = 1 .. R-1 from one table entry (relative error below
      // R ulp, far under the FP64 tolerance of the transform)
      double2 w1 = tw(k * sf * step);
      if (inv) w1.y = -w1.y;
      double2 w = w1;
#pragma unroll
      for (int r = 1; r < R; ++r) {
        v[r] = cmul(v[r], w);
        if (r + 1 < R) w = cmul(w, w1);
      }
    }
    small_dft<R>(v, inv);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int q = 0; q < R; ++q) dst[base + q * Ns] = v[q];
  }
}

// Generic prime radix: each thread computes whole outputs (parallel over
// the N outputs, so a large prime factor does not serialise a few threads).
template <class TW>
__device__ void stockham_generic(Buf src, Buf dst, int N, int R, int Ns,
                                 bool inv, const TW &tw, int step) {
  const int NR = N / R;
  const int sf = N / (Ns * R);
  for (int item = threadIdx.x; item < N; item += blockDim.x) {
    const int j = item / R;
    const int q = item - j * R;
    const int k = j % Ns;
    const int ang = (sf * (k + q * Ns)) % N;
    int e = 0;
    double2 acc = make_double2(0.0, 0.0);
    for (int r = 0; r < R; ++r) {
      double2 w = tw(e * step);
      if (inv) w.y = -w.y;
      const double2 v = src[j + r * NR];
      acc.x = fma(v.x, w.x, fma(-v.y, w.y, acc.x));
      acc.y = fma(v.x, w.y, fma(v.y, w.x, acc.y));
      e += ang;
      if (e >= N) e -= N;
    }
    dst[(j - k) * R + k + q * Ns] = acc;
  }
}

// Complex FFT of length d.N in buffers a/b; returns the buffer holding the
// result.  Callers synchronise before; the function synchronises after each
// pass.
template <class TW>
__device__ double2 *run_fft(const FftDesc &d, double2 *a, double2 *b, bool inv, const TW &W) {
  const int step = d.n / d.N;
  int Ns = 1;
  double2 *src = a, *dst = b;   // raw; each pass indexes them through Buf
  for (int s = 0; s < d.nrad; ++s) {
    const int R = d.rad[s];
    switch (R) {
      case 2: stockham_small<2>(Buf{src}, Buf{dst}, d.N, Ns, inv, W, step); break;
      case 3: stockham_small<3>(Buf{src}, Buf{dst}, d.N, Ns, inv, W, step); break;
      case 4: stockham_small<4>(Buf{src}, Buf{dst}, d.N, Ns, inv, W, step); break;
      case 5: stockham_small<5>(Buf{src}, Buf{dst}, d.N, Ns, inv, W, step); break;
      case 8: stockham_small<8>(Buf{src}, Buf{dst}, d.N, Ns, inv, W, step); break;
      default: stockham_generic(Buf{src}, Buf{dst}, d.N, R, Ns, inv, W, step); break;
    }
    __syncthreads();
    Ns *= R;
    double2 *t = src;
    src = dst;
    dst = t;
  }
  return src;
}

// ---------------------------------------------------------------------------
// Bluestein transform for lengths with large prime factors:
// X_k = c_k sum_j (x_j c_j) conj(c_{k-j}), c_j = exp(-pi i j^2/N), evaluated
// as a power-of-two convolution of length M >= 2N-1: in-place radix-4
// decimation in frequency (digit-reversed output), product with the chirp
// transform precomputed in the same order, the inverse stages back to
// natural order.  The inverse transform is conj(forward(conj x)).
// ---------------------------------------------------------------------------
template <class TW>
__device__ __forceinline__ double2 chirp_of(int j, int n, int N, const TW &Wn) {
  // j < N <= n <= 2^15, so j^2 fits 32 bits
  const unsigned jj = unsigned(j) * unsigned(j);
  if ((n & 1) == 0) return Wn(int(jj % unsigned(n)));  // exp(-2 pi i (j^2 mod n)/n)
  double sn, cs;
  sincospi(-double(jj % (2u * unsigned(n))) / n, &sn, &cs);
  return make_double2(cs, sn);
}

// In-place decimation in frequency of length M = 2^lg (output in the
// digit order of the stages): one radix-2 stage when lg is odd, then radix-4
// stages.  A stage of length len maps x_{i + j len/4} (j < 4) to
// y_r = W_len^{ir} sum_j x_{i + j len/4} (-i)^{jr}, stored at i + r len/4.
template <class TW>
__device__ __forceinline__ void dif_stage4(const Buf &a, int M, int len, const TW &Wp, int P) {
  const int q = len >> 2, st = P / len, lq = 31 - __clz(q);
  for (int t = threadIdx.x; t < (M >> 2); t += blockDim.x) {
    const int i = t & (q - 1);
    const int b0 = (t >> lq) * len + i;
    const double2 x0 = a[b0], x1 = a[b0 + q], x2 = a[b0 + 2 * q], x3 = a[b0 + 3 * q];
    const double2 s02 = cadd(x0, x2), d02 = csub(x0, x2);
    const double2 s13 = cadd(x1, x3), d13 = csub(x1, x3);
    const double2 md13 = make_double2(d13.y, -d13.x);  // -i (x1 - x3)
    a[b0] = cadd(s02, s13);
    a[b0 + q] = cmul(cadd(d02, md13), Wp(i * st));
    a[b0 + 2 * q] = cmul(csub(s02, s13), Wp(2 * i * st));
    a[b0 + 3 * q] = cmul(csub(d02, md13), Wp(3 * i * st));
  }
  __syncthreads();
}

// One stage of the inverse (conjugate twiddles), undoing dif_stage4.
template <class TW>
__device__ __forceinline__ void dit_stage4(const Buf &a, int M, int len, const TW &Wp, int P) {
  const int q = len >> 2, st = P / len, lq = 31 - __clz(q);
  for (int t = threadIdx.x; t < (M >> 2); t += blockDim.x) {
    const int i = t & (q - 1);
    const int b0 = (t >> lq) * len + i;
    const double2 z0 = a[b0];
    const double2 z1 = cmul(a[b0 + q], cconj(Wp(i * st)));
    const double2 z2 = cmul(a[b0 + 2 * q], cconj(Wp(2 * i * st)));
    const double2 z3 = cmul(a[b0 + 3 * q], cconj(Wp(3 * i * st)));
    const double2 s02 = cadd(z0, z2), d02 = csub(z0, z2);
    const double2 s13 = cadd(z1, z3), d13 = csub(z1, z3);
    const double2 pd13 = make_double2(-d13.y, d13.x);  // i (z1 - z3)
    a[b0] = cadd(s02, s13);
    a[b0 + q] = cadd(d02, pd13);
    a[b0 + 2 * q] = csub(s02, s13);
    a[b0 + 3 * q] = csub(d02, pd13);
  }
  __syncthreads();
}

template <class TW>
__device__ void dif_inplace(double2 *buf, int M, const TW &Wp, int P) {
  const Buf a{buf};
  const int lg = 31 - __clz(M);
  int len = M;
  if (lg & 1) {
    const int half = len >> 1, st = P / len;
    for (int t = threadIdx.x; t < half; t += blockDim.x) {
      const double2 u = a[t], v = a[t + half];
      a[t] = cadd(u, v);
      a[t + half] = cmul(csub(u, v), Wp(t * st));
    }
    __syncthreads();
    len = half;
  }
  for (; len >= 4; len >>= 2) dif_stage4(a, M, len, Wp, P);
}

// Bluestein convolution of x (buf[0, N)) with the chirp: the stages of
// dif_inplace, the product with the transformed chirp bh (stored in the same
// digit order and swizzle) and the inverse stages, with three sweeps merged:
//  * the chirp pre-multiplication into the first DIF stage, whose inputs at
//    and beyond M/2 >= N are the zero padding;
//  * the last DIF stage (length 4: unit twiddles), the product and the first
//    inverse stage, which all act on the same four consecutive entries;
//  * the last inverse stage into the chirp post-multiplication, of which
//    only the outputs k < N are needed.
// The result X_k (k < N) is left in buf[0, N).
template <class TW>
__device__ void run_bluestein(const FftDesc &d, double2 *raw, bool inv, const TW &Wn,
                              const TW &Wp, int P, const double2 *__restrict__ bhat) {
  const Buf a{raw};
  const Buf bh{const_cast<double2 *>(bhat + d.bhat)};   // read only
  const int M = d.M, N = d.N, lg = 31 - __clz(M);
  auto pre = [&](int j) {   // x_j c_j (conjugated input for the inverse transform)
    double2 x = a[j];
    if (inv) x.y = -x.y;
    return cmul(x, chirp_of(j, d.n, N, Wn));
  };
  const double2 zero = make_double2(0.0, 0.0);
  int len;
  if (lg & 1) {
    const int half = M >> 1, st = P / M;
    for (int t = threadIdx.x; t < half; t += blockDim.x) {
      const double2 u = t < N ? pre(t) : zero;
      a[t] = u;
      a[t + half] = cmul(u, Wp(t * st));
    }
    len = half;
  } else {
    const int q = M >> 2, st = P / M;
    for (int t = threadIdx.x; t < q; t += blockDim.x) {
      const double2 x0 = t < N ? pre(t) : zero;
      const double2 x1 = t + q < N ? pre(t + q) : zero;
      const double2 md1 = make_double2(x1.y, -x1.x);   // -i x1
      a[t] = cadd(x0, x1);
      a[t + q] = cmul(cadd(x0, md1), Wp(t * st));
      a[t + 2 * q] = cmul(csub(x0, x1), Wp(2 * t * st));
      a[t + 3 * q] = cmul(csub(x0, md1), Wp(3 * t * st));
    }
    len = q;
  }
  __syncthreads();
  for (; len >= 16; len >>= 2) dif_stage4(a, M, len, Wp, P);
  for (int t = threadIdx.x; t < (M >> 2); t += blockDim.x) {
    const int b0 = 4 * t;
    double2 y[4];
    {
      const double2 x0 = a[b0], x1 = a[b0 + 1], x2 = a[b0 + 2], x3 = a[b0 + 3];
      const double2 s02 = cadd(x0, x2), d02 = csub(x0, x2);
      const double2 s13 = cadd(x1, x3), d13 = csub(x1, x3);
      const double2 md13 = make_double2(d13.y, -d13.x);
      y[0] = cadd(s02, s13);
      y[1] = cadd(d02, md13);
      y[2] = csub(s02, s13);
      y[3] = csub(d02, md13);
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) y[r] = cmul(y[r], __ldg(&bh[b0 + r]));
    const double2 s02 = cadd(y[0], y[2]), d02 = csub(y[0], y[2]);
    const double2 s13 = cadd(y[1], y[3]), d13 = csub(y[1], y[3]);
    const double2 pd13 = make_double2(-d13.y, d13.x);
    a[b0] = cadd(s02, s13);
    a[b0 + 1] = cadd(d02, pd13);
    a[b0 + 2] = csub(s02, s13);
    a[b0 + 3] = csub(d02, pd13);
  }
  __syncthreads();
  const int top = (lg & 1) ? (M >> 1) : M;   // length of the last radix-4 stage
  for (len = 16; len < top; len <<= 2) dit_stage4(a, M, len, Wp, P);
  auto post = [&](int k, double2 v) {
    double2 y = cmul(v, chirp_of(k, d.n, N, Wn));
    if (inv) y.y = -y.y;
    a[k] = y;
  };
  if (lg & 1) {
    // radix-4 stages end at M/2; the radix-2 stage's outputs k < N
    if (top >= 16) dit_stage4(a, M, top, Wp, P);
    const int half = M >> 1, st = P / M;
    for (int t = threadIdx.x; t < N; t += blockDim.x)
      post(t, cadd(a[t], cmul(a[t + half], cconj(Wp(t * st)))));
  } else {
    // the last radix-4 stage (length M): outputs i and i + M/4 (< N <= M/2)
    const int q = M >> 2, st = P / M;
    for (int i = threadIdx.x; i < q; i += blockDim.x) {
      const double2 z0 = a[i];
      const double2 z1 = cmul(a[i + q], cconj(Wp(i * st)));
      const double2 z2 = cmul(a[i + 2 * q], cconj(Wp(2 * i * st)));
      const double2 z3 = cmul(a[i + 3 * q], cconj(Wp(3 * i * st)));
      const double2 s02 = cadd(z0, z2), d02 = csub(z0, z2);
      const double2 s13 = cadd(z1, z3), d13 = csub(z1, z3);
      const double2 pd13 = make_double2(-d13.y, d13.x);
      if (i < N) post(i, cadd(s02, s13));
      if (i + q < N) post(i + q, cadd(d02, pd13));
    }
  }
  __syncthreads();
}

// Precomputes, per Bluestein length, DIF(b)/M with b_j = conj(c_j) for
// |j| < N (negative j wrapped to M-j).  One CTA per length, in global memory.
__global__ void bluestein_setup_kernel(const FftDesc *__restrict__ fdesc,
                                       const int *__restrict__ blue_idx,
                                       const double2 *__restrict__ twiddle,
                                       const double2 *__restrict__ wpow2, int P,
                                       double2 *__restrict__ bhat) {
  const FftDesc d = fdesc[blue_idx[blockIdx.x]];
  double2 *b = bhat + d.bhat;    // M (a power of two >= 64) entries, swizzled as Buf
  const TwGlobal Wn{twiddle + d.tw};
  for (int j = threadIdx.x; j < d.M; j += blockDim.x) {
    int jj = -1;
    if (j < d.N) jj = j;
    else if (j > d.M - d.N) jj = d.M - j;
    Buf{b}[j] = (jj >= 0) ? cconj(chirp_of(jj, d.n, d.N, Wn)) : make_double2(0.0, 0.0);
  }
  __syncthreads();
  dif_inplace(b, d.M, TwGlobal{wpow2}, P);
  const double inv_m = 1.0 / d.M;
  for (int j = threadIdx.x; j < d.M; j += blockDim.x) b[j] = cscale(b[j], inv_m);
}

template <typename T>
__device__ __forceinline__ void store_px(T *p, double v, bool add) {
  if (add) *p += T(v);
  else *p = T(v);
}

// e^{i m phi0} for m <= mm as hi[m >> 6] * lo[m & 63], built per ring in
// shared memory (about 64 + mm/64 sincos calls instead of mm).
constexpr int kShiftLo = 64;
__device__ void build_shift(double2 *lo, double2 *hi, int mm, double ph) {
  const int nhi = (mm >> 6) + 1;
  for (int t = threadIdx.x; t < kShiftLo + nhi; t += blockDim.x) {
    double sn, cs;
    if (t < kShiftLo) {
      sincos(t * ph, &sn, &cs);
      lo[t] = make_double2(cs, sn);
    } else {
      sincos(double(t - kShiftLo) * kShiftLo * ph, &sn, &cs);
      hi[t - kShiftLo] = make_double2(cs, sn);
    }
  }
}

__device__ __forceinline__ double2 shift_of(const double2 *lo, const double2 *hi, int m) {
  return cmul(hi[m >> 6], lo[m & (kShiftLo - 1)]);
}

// ---------------------------------------------------------------------------
// phase -> ring (synthesis).  Grid: (pairs of one size class, components).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(1024) phase2ring_kernel(const int *__restrict__ pairs, const int *__restrict__ mlim,
                                  const int *__restrict__ nph, const long long *__restrict__ ofs,
                                  const int *__restrict__ stride, const double *__restrict__ phi0,
                                  const double *__restrict__ weight, const int *__restrict__ fftidx,
                                  const FftDesc *__restrict__ fdesc,
                                  const double2 *__restrict__ twiddle,
                                  const double2 *__restrict__ wpow2, int P,
                                  const double2 *__restrict__ bhat,
                                  const double2 *__restrict__ phase, int ncm, int mmax, int flags,
                                  int nbufA, int nbufB, int twcap, T *const *__restrict__ maps,
                                  long long map_lo, double2 *__restrict__ gbuf, int npc,
                                  int nitems) {
  extern __shared__ double2 smem[];
  const int ms = mmax + 1;
  // SHARP_SUBTRACT: the negated result is added (negation is exact)
  const bool add = (flags & (SHARP_ADD | SHARP_SUBTRACT)) != 0;
  const double wscale = ((flags & SHARP_REAL_HARMONICS) ? kSqrtHalf : 1.0) *
                        ((flags & SHARP_SUBTRACT) ? -1.0 : 1.0);
  // buffers A/B in shared memory, or (rings too long for it) in this CTA's
  // slot of a global scratch; such CTAs loop over (pair, component) items
  const bool gb = gbuf != nullptr;
  double2 *bufA = gb ? gbuf + size_t(blockIdx.x) * (nbufA + nbufB) : smem;
  double2 *bufB = bufA + nbufA;
  double2 *slo = gb ? smem : smem + nbufA + nbufB;
  double2 *shi = slo + kShiftLo;
  // twiddle slices: ring length (twcap = 2 nmax/64 + 2 entries in hi), then
  // the Bluestein convolution length P
  double2 *twlo = shi + (mmax / kShiftLo + 2);
  double2 *twhi = twlo + kTwLo;
  double2 *pwlo = twhi + twcap;
  double2 *pwhi = pwlo + kTwLo;
  const TwShared tw{twlo, twhi}, pw{pwlo, pwhi};
  if (P > 0) load_twshared(pwlo, pwhi, wpow2, P);
  for (int it = gb ? blockIdx.x : 0; it < (gb ? nitems : 1); it += gb ? gridDim.x : 1) {
  const int p = gb ? pairs[it % npc] : pairs[blockIdx.x];
  const int c = gb ? it / npc : blockIdx.y;
  const int mm = min(mmax, mlim[p]);
  T *map = maps[c];
  for (int h = 0; h < 2; ++h) {
    const int ring = 2 * p + h;
    const int n = nph[ring];
    if (n <= 0) continue;
    const FftDesc d = fdesc[fftidx[ring]];
    const double wgt = ((flags & SHARP_USE_WEIGHTS) ? weight[ring] : 1.0) * wscale;
    const double ph = phi0[ring];
    const bool rot = fabs(ph) >= 1e-14;
    const int half = n / 2;  // highest bin kept (n odd: (n-1)/2)
    const Buf C{bufB}, Ab{bufA};
    const double2 *src = phase + ((long long)(p * ncm + c) * 2 + h) * ms;
    if (rot) build_shift(slo, shi, mm, ph);
    load_twshared(twlo, twhi, twiddle + d.tw, n);
    __syncthreads();
    // fold phase_m * wgt * e^{i m phi0} into bins 0..half (sharp.c:265-300);
    // as there, the direct term of m = 1 of a one-pixel ring is not added
    // (the reference's running bin index starts at 1 and wraps only after
    // its first use, sharp.c:282, :297)
    for (int k = threadIdx.x; k <= half; k += blockDim.x) {
      double2 acc = make_double2(0.0, 0.0);
      for (int m = k; m <= mm; m += n) {
        if (n == 1 && m == 1) continue;
        double2 t = cscale(src[m], wgt);
        if (rot) t = cmul(t, shift_of(slo, shi, m));
        acc = cadd(acc, t);
      }
      for (int m = (k == 0) ? n : n - k; m <= mm; m += n) {
        double2 t = cscale(src[m], wgt);
        if (rot) t = cmul(t, shift_of(slo, shi, m));
        acc = cadd(acc, cconj(t));
      }
      if (k == 0 || 2 * k == n) acc.y = 0.0;
      C[k] = acc;
    }
    __syncthreads();
    if ((n & 1) == 0) {
      // Z_k = (C_k + conj C_{N-k}) + i conj(W^k) (C_k - conj C_{N-k}), k < N
      for (int k = threadIdx.x; k < d.N; k += blockDim.x) {
        const double2 ck = C[k], cn = cconj(C[d.N - k]);
        const double2 sm = cadd(ck, cn), df = csub(ck, cn);
        const double2 w = tw(k);                    // exp(-2 pi i k/n)
        const double2 iw = make_double2(w.y, w.x);  // i * conj(w)
        Ab[k] = cadd(sm, cmul(iw, df));
      }
    } else {
      for (int k = threadIdx.x; k < n; k += blockDim.x)
        Ab[k] = (k <= half) ? C[k] : cconj(C[n - k]);
    }
    __syncthreads();
    double2 *res;
    if (d.blue) {
      run_bluestein(d, bufA, true, tw, pw, P, bhat);
      res = bufA;
    } else {
      res = run_fft(d, bufA, bufB, true, tw);
    }
    const long long o = ofs[ring] - map_lo;
    const long long st = stride[ring];
    const Buf Rs{res};
    if ((n & 1) == 0) {
      for (int j = threadIdx.x; j < d.N; j += blockDim.x) {
        const double2 z = Rs[j];
        store_px(map + o + (2 * j) * st, z.x, add);
        store_px(map + o + (2 * j + 1) * st, z.y, add);
      }
    } else {
      for (int j = threadIdx.x; j < n; j += blockDim.x) store_px(map + o + j * st, Rs[j].x, add);
    }
    __syncthreads();
  }
  }
}

// ---------------------------------------------------------------------------
// ring -> phase (analysis)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(1024) ring2phase_kernel(const int *__restrict__ pairs, const int *__restrict__ mlim,
                                  const int *__restrict__ nph, const long long *__restrict__ ofs,
                                  const int *__restrict__ stride, const double *__restrict__ phi0,
                                  const double *__restrict__ weight, const int *__restrict__ fftidx,
                                  const FftDesc *__restrict__ fdesc,
                                  const double2 *__restrict__ twiddle,
                                  const double2 *__restrict__ wpow2, int P,
                                  const double2 *__restrict__ bhat, double2 *__restrict__ phase,
                                  int ncm, int mmax, int flags, int nbufA, int nbufB, int twcap,
                                  const T *const *__restrict__ maps, long long map_lo,
                                  double2 *__restrict__ gbuf, int npc, int nitems) {
  extern __shared__ double2 smem[];
  const int ms = mmax + 1;
  const double wscale = (flags & SHARP_REAL_HARMONICS) ? kSqrtTwo : 1.0;
  const bool gb = gbuf != nullptr;  // as in phase2ring_kernel
  double2 *bufA = gb ? gbuf + size_t(blockIdx.x) * (nbufA + nbufB) : smem;
  double2 *bufB = bufA + nbufA;
  double2 *slo = gb ? smem : smem + nbufA + nbufB;
  double2 *shi = slo + kShiftLo;
  // twiddle slices: ring length (twcap = 2 nmax/64 + 2 entries in hi), then
  // the Bluestein convolution length P
  double2 *twlo = shi + (mmax / kShiftLo + 2);
  double2 *twhi = twlo + kTwLo;
  double2 *pwlo = twhi + twcap;
  double2 *pwhi = pwlo + kTwLo;
  const TwShared tw{twlo, twhi}, pw{pwlo, pwhi};
  if (P > 0) load_twshared(pwlo, pwhi, wpow2, P);
  for (int it = gb ? blockIdx.x : 0; it < (gb ? nitems : 1); it += gb ? gridDim.x : 1) {
  const int p = gb ? pairs[it % npc] : pairs[blockIdx.x];
  const int c = gb ? it / npc : blockIdx.y;
  const int mm = min(mmax, mlim[p]);
  const T *map = maps[c];
  for (int h = 0; h < 2; ++h) {
    const int ring = 2 * p + h;
    const int n = nph[ring];
    if (n <= 0) continue;
    const FftDesc d = fdesc[fftidx[ring]];
    const double wgt = ((flags & SHARP_USE_WEIGHTS) ? weight[ring] : 1.0) * wscale;
    const double ph = phi0[ring];
    const bool rot = fabs(ph) >= 1e-14;
    const long long o = ofs[ring] - map_lo;
    const long long st = stride[ring];
    if (rot) build_shift(slo, shi, mm, -ph);
    load_twshared(twlo, twhi, twiddle + d.tw, n);
    const Buf Ab{bufA};
    if ((n & 1) == 0) {
      for (int j = threadIdx.x; j < d.N; j += blockDim.x)
        Ab[j] = make_double2(double(map[o + (2 * j) * st]), double(map[o + (2 * j + 1) * st]));
    } else {
      for (int j = threadIdx.x; j < n; j += blockDim.x)
        Ab[j] = make_double2(double(map[o + j * st]), 0.0);
    }
    __syncthreads();
    double2 *res;
    if (d.blue) {
      run_bluestein(d, bufA, false, tw, pw, P, bhat);
      res = bufA;
    } else {
      res = run_fft(d, bufA, bufB, false, tw);
    }
    const Buf X{(res == bufA) ? bufB : bufA}, Rs{res};
    if ((n & 1) == 0) {
      // X_k = (Z_k + conj Z_{N-k})/2 - i W^k (Z_k - conj Z_{N-k})/2, k <= N
      for (int k = threadIdx.x; k <= d.N; k += blockDim.x) {
        const double2 zk = Rs[k == d.N ? 0 : k];
        const double2 zn = cconj(Rs[k == 0 ? 0 : d.N - k]);
        const double2 sm = cadd(zk, zn), df = csub(zk, zn);
        const double2 w = tw(k);
        const double2 mi_w = make_double2(w.y, -w.x);  // -i * w
        double2 xk = cscale(cadd(sm, cmul(mi_w, df)), 0.5);
        if (k == 0 || k == d.N) xk.y = 0.0;  // DC and Nyquist are real
        X[k] = xk;
      }
    } else {
      for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double2 xk = Rs[k];
        if (k == 0) xk.y = 0.0;
        X[k] = xk;
      }
    }
    __syncthreads();
    double2 *dst = phase + ((long long)(p * ncm + c) * 2 + h) * ms;
    for (int m = threadIdx.x; m <= mm; m += blockDim.x) {
      const int idx = m % n;
      double2 v = (idx < n - idx) ? X[idx] : cconj(X[n - idx]);
      v = cscale(v, wgt);
      if (rot) v = cmul(v, shift_of(slo, shi, m));
      dst[m] = v;
    }
    __syncthreads();
  }
  }
}

// ---------------------------------------------------------------------------
// Power-of-two rings (n = 2N real pixels, N = 1024 .. 8192; every equatorial
// HEALPix ring when Nside is a power of two) with no alias folding
// (mlim <= N): one CTA per ring and component, N/16 threads holding 16
// complex values each.  The complex FFT of length N runs as in-place
// decimation-in-frequency passes over one shared buffer: radix-16 passes in
// registers (a 16-point DFT as 4 x 4 with internal twiddles), then one pass
// of radix 2, 4 or 8 for the remaining factor; the output is in digit-
// reversed order, which the final global access undoes.  The packing of the
// real transform (the C_k / C_{N-k} twist) is fused into the global phase
// reads (synthesis) or the phase writes (analysis), so the buffer is read
// and written once per pass.  Buffer entries are padded (p + p/16 + p/256)
// so that the strided accesses of every pass spread over the bank groups.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int pw_pad(int p) { return p + (p >> 4) + (p >> 8); }
__host__ __device__ constexpr int pw_entries(int N) {
  return (N - 1) + ((N - 1) >> 4) + ((N - 1) >> 8) + 1;
}
__host__ __device__ constexpr int pw_passes16(int N) {
  return N >= 4096 ? 3 : 2;   // 1024 = 16^2 4, 2048 = 16^2 8, 4096 = 16^3, 8192 = 16^3 2
}
__host__ __device__ constexpr int pw_last(int N) {
  return N / (pw_passes16(N) == 3 ? 4096 : 256);
}

// cos(2 pi e / 16), e = 0 .. 15
__device__ __forceinline__ double cos16(int e) {
  switch (e & 15) {
    case 0: return 1.0;
    case 1: case 15: return 0.92387953251128675613;
    case 2: case 14: return 0.70710678118654752440;
    case 3: case 13: return 0.38268343236508977173;
    case 4: case 12: return 0.0;
    case 5: case 11: return -0.38268343236508977173;
    case 6: case 10: return -0.70710678118654752440;
    case 7: case 9: return -0.92387953251128675613;
    default: return -1.0;
  }
}
// exp(-+2 pi i e / 16) (INV: +); sin(2 pi e/16) = cos(2 pi (e - 4)/16)
template <bool INV>
__device__ __forceinline__ double2 w16(int e) {
  const double sn = cos16(e + 12);
  return make_double2(cos16(e), INV ? sn : -sn);
}

// 16-point DFT in place: v[n2 + 4 n1] -> X[k1 + 4 k2] = v[k1 + 4 k2]
template <bool INV>
__device__ __forceinline__ void dft16(double2 (&v)[16]) {
  double2 y[4][4];
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) {
    double2 t[4] = {v[n2], v[n2 + 4], v[n2 + 8], v[n2 + 12]};
    small_dft<4>(t, INV);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      const int e = n2 * k1;
      if (e == 0) y[k1][n2] = t[k1];
      else if (e == 4) y[k1][n2] = INV ? make_double2(-t[k1].y, t[k1].x)
                                       : make_double2(t[k1].y, -t[k1].x);
      else y[k1][n2] = cmul(t[k1], w16<INV>(e));
    }
  }
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    small_dft<4>(y[k1], INV);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = y[k1][k2];
  }
}

// One radix-16 DIF pass of length len (stride len/16) over the buffer;
// twiddles W_len^(k0 f) from a table W of exp(-2 pi i j/tl), j < tl (a
// multiple of len), so W_len^e = W[(tl/len) e].
// Inputs i >= NIN are taken as zero (not read).
// The arithmetic and stores of a pass on inputs already in registers: v[i]
// is the entry at base + s i (s = len/16, base = (u/s) len + k0, k0 = u mod s).
template <int N, bool INV>
__device__ __forceinline__ void pw_pass16_regs(double2 (&v)[16], double2 *buf, int len,
                                               const double2 *__restrict__ W, int tl) {
  const int s = len >> 4;
  const int u = threadIdx.x;
  const int k0 = u & (s - 1);
  const int base = (u / s) * len + k0;
  dft16<INV>(v);
  if (s > 1 && k0 > 0) {
    double2 w1 = __ldg(W + (tl / len) * k0);
    if (INV) w1.y = -w1.y;
    double2 w = w1;
#pragma unroll
    for (int f = 1; f < 16; ++f) {
      v[f] = cmul(v[f], w);
      if (f < 15) w = cmul(w, w1);
    }
  }
#pragma unroll
  for (int f = 0; f < 16; ++f) buf[pw_pad(base + s * f)] = v[f];
}

template <int N, bool INV, int NIN = 16>
__device__ __forceinline__ void pw_pass16(double2 *buf, int len, const double2 *__restrict__ W,
                                          int tl) {
  const int s = len >> 4;
  const int u = threadIdx.x;
  const int k0 = u & (s - 1);
  const int base = (u / s) * len + k0;
  double2 v[16];
#pragma unroll
  for (int i = 0; i < 16; ++i)
    v[i] = i < NIN ? buf[pw_pad(base + s * i)] : make_double2(0.0, 0.0);
  dft16<INV>(v);
  if (s > 1 && k0 > 0) {
    double2 w1 = __ldg(W + (tl / len) * k0);
    if (INV) w1.y = -w1.y;
    double2 w = w1;
#pragma unroll
    for (int f = 1; f < 16; ++f) {
      v[f] = cmul(v[f], w);
      if (f < 15) w = cmul(w, w1);
    }
  }
#pragma unroll
  for (int f = 0; f < 16; ++f) buf[pw_pad(base + s * f)] = v[f];
}

// The last pass (radix R = 2, 4 or 8 over blocks of R, no twiddles)
template <int N, int R, bool INV>
__device__ __forceinline__ void pw_pass_last(double2 *buf) {
#pragma unroll
  for (int q = 0; q < 16 / R; ++q) {
    const int b = threadIdx.x + (N / 16) * q;
    double2 v[R];
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = buf[pw_pad(b * R + i)];
    small_dft<R>(v, INV);
#pragma unroll
    for (int i = 0; i < R; ++i) buf[pw_pad(b * R + i)] = v[i];
  }
}

// The passes of pw_fft after the first (which the caller ran from registers
// with pw_pass16_regs and a __syncthreads).
template <int N, bool INV>
__device__ void pw_fft_rest(double2 *buf, const double2 *__restrict__ W, int tl) {
  int len = N >> 4;
#pragma unroll
  for (int q = 1; q < pw_passes16(N); ++q) {
    pw_pass16<N, INV>(buf, len, W, tl);
    __syncthreads();
    len >>= 4;
  }
  constexpr int RL = pw_last(N);
  if constexpr (RL > 1) {
    pw_pass_last<N, RL, INV>(buf);
    __syncthreads();
  }
}

template <int N, bool INV>
__device__ void pw_fft(double2 *buf, const double2 *__restrict__ W, int tl) {
  int len = N;
#pragma unroll
  for (int q = 0; q < pw_passes16(N); ++q) {
    pw_pass16<N, INV>(buf, len, W, tl);
    __syncthreads();
    len >>= 4;
  }
  constexpr int RL = pw_last(N);
  if constexpr (RL > 1) {
    pw_pass_last<N, RL, INV>(buf);
    __syncthreads();
  }
}

// The transposed pass of pw_pass16 with the opposite sign: inputs at the
// positions pw_pass16 writes, times conj(W_len^(k0 f)), then the 16-point
// DFT with positive sign.  Run in the reverse order of the passes of
// pw_fft<N, false>, the chain maps its digit-reversed output back to
// natural order and computes the unnormalised inverse DFT.  Outputs
// i >= NOUT are not stored.
template <int N, int NOUT = 16>
__device__ __forceinline__ void pw_pass16_back(double2 *buf, int len,
                                               const double2 *__restrict__ W, int tl) {
  const int s = len >> 4;
  const int u = threadIdx.x;
  const int k0 = u & (s - 1);
  const int base = (u / s) * len + k0;
  double2 v[16];
#pragma unroll
  for (int f = 0; f < 16; ++f) v[f] = buf[pw_pad(base + s * f)];
  if (s > 1 && k0 > 0) {
    double2 w1 = __ldg(W + (tl / len) * k0);
    w1.y = -w1.y;
    double2 w = w1;
#pragma unroll
    for (int f = 1; f < 16; ++f) {
      v[f] = cmul(v[f], w);
      if (f < 15) w = cmul(w, w1);
    }
  }
  dft16<true>(v);
#pragma unroll
  for (int i = 0; i < NOUT; ++i) buf[pw_pad(base + s * i)] = v[i];
}

// Buffer position of frequency k after pw_fft (digits reversed)
template <int N>
__device__ __forceinline__ int pw_pos(int k) {
  int p = 0, rem = k, stride = N;
#pragma unroll
  for (int q = 0; q < pw_passes16(N); ++q) {
    stride >>= 4;
    p += (rem & 15) * stride;
    rem >>= 4;
  }
  return p + rem;   // the last digit (radix pw_last(N)) has stride 1
}

// CTAs per SM the synthesis kernel is compiled for: three at N = 4096 (80
// registers, a few spilled; measured 8.9 against 9.5 ms per 12-transform
// synthesis at Nside 2048 with two), 128 registers for the shorter rings
__host__ __device__ constexpr int pow2_synth_min_blocks(int N) {
  return N == 4096 ? 3 : N == 2048 ? 4 : N == 1024 ? 8 : 1;
}

// phase -> ring.  Grid: (2 * pairs of this length, components).
template <typename T, int N>
__global__ void __launch_bounds__(N / 16, pow2_synth_min_blocks(N))
phase2ring_pow2_kernel(const int *__restrict__ pairs, const int *__restrict__ mlim,
                       const int *__restrict__ nph, const long long *__restrict__ ofs,
                       const double *__restrict__ phi0, const double *__restrict__ weight,
                       const int *__restrict__ fftidx, const FftDesc *__restrict__ fdesc,
                       const double2 *__restrict__ twiddle, const double2 *__restrict__ phase,
                       int ncm, int mmax, int flags, T *const *__restrict__ maps,
                       long long map_lo) {
  extern __shared__ double2 smem[];
  __shared__ uint64_t row_full;
  double2 *buf = smem;
  double2 *slo = smem + pw_entries(N);
  double2 *shi = slo + kShiftLo;
  // while the Z_k are formed the buffer holds the phase row (entries 0 .. mm
  // <= N) and, behind it where there is room (N >= 2048), the twiddle slices
  // W^k = twh[k / 64] twl[k mod 64], k < N
  constexpr bool kSlices = N + 1 + kTwLo + N / kTwLo <= pw_entries(N);
  double2 *twl = buf + (N + 1), *twh = twl + kTwLo;
  const int p = pairs[blockIdx.x >> 1], h = blockIdx.x & 1, c = blockIdx.y;
  const int ring = 2 * p + h;
  if (nph[ring] <= 0) return;        // unpaired ring: nothing in this hemisphere
  const int ms = mmax + 1;
  const int mm = min(mmax, mlim[p]);
  const bool add = (flags & (SHARP_ADD | SHARP_SUBTRACT)) != 0;
  const double wgt = ((flags & SHARP_USE_WEIGHTS) ? weight[ring] : 1.0) *
                     ((flags & SHARP_REAL_HARMONICS) ? kSqrtHalf : 1.0) *
                     ((flags & SHARP_SUBTRACT) ? -1.0 : 1.0);
  const double ph = phi0[ring];
  const bool rot = fabs(ph) >= 1e-14;
  const double2 *W = twiddle + fdesc[fftidx[ring]].tw;
  const double2 *src = phase + ((long long)(p * ncm + c) * 2 + h) * ms;
  // the phase row into shared memory by one bulk copy (16-byte aligned, a
  // multiple of 16 bytes), while the threads build the twiddle and phi0
  // slices
  if (threadIdx.x == 0) {
    mbar_init(&row_full, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_arrive_tx(&row_full, uint32_t(16 * (mm + 1)));
    bulk_g2s(buf, src, uint32_t(16 * (mm + 1)), &row_full);
  }
  if constexpr (kSlices) load_twshared(twl, twh, W, N);   // W: the table of 2N entries
  if (rot) build_shift(slo, shi, mm, ph);
  // a copy that did not complete within the bounded wait is redone by the
  // threads from global memory (the same values, so a late bulk write
  // changes nothing)
  if (__syncthreads_or(!mbar_wait(&row_full, 0))) {
    for (int m = threadIdx.x; m <= mm; m += N / 16) buf[m] = src[m];
    __syncthreads();
  }
  // t_m = phase_m wgt e^{i m phi0} (zero above mm); C_0 and C_N real
  auto tm = [&](int m) {
    if (m > mm) return make_double2(0.0, 0.0);
    double2 t = cscale(buf[m], wgt);
    if (rot) t = cmul(t, shift_of(slo, shi, m));
    return t;
  };
  // Z_k = (C_k + conj C_{N-k}) + i conj(W^k) (C_k - conj C_{N-k}), k < N,
  // for k = tid + (N/16) i: exactly this thread's inputs of the first pass,
  // which therefore runs from registers
  double2 v[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const int k = threadIdx.x + (N / 16) * i;
    double2 ck = tm(k), cn;
    if (k == 0) {
      ck.y = 0.0;
      const double2 tn = tm(N);
      cn = make_double2(tn.x + tn.x, 0.0);   // C_N = t_N + conj t_N
    } else {
      cn = tm(N - k);
    }
    cn = cconj(cn);
    const double2 sm = cadd(ck, cn), df = csub(ck, cn);
    const double2 w = kSlices ? cmul(twh[k >> 6], twl[k & (kTwLo - 1)]) : __ldg(W + k);
    const double2 iw = make_double2(w.y, w.x);   // i * conj(w)
    v[i] = cadd(sm, cmul(iw, df));
  }
  __syncthreads();   // the row and the slices are read; the first pass overwrites them
  pw_pass16_regs<N, true>(v, buf, N, W, 2 * N);
  __syncthreads();
  pw_fft_rest<N, true>(buf, W, 2 * N);
  // pixels 2j, 2j+1 = Re, Im z_j
  T *map = maps[c] + (ofs[ring] - map_lo);
#pragma unroll 4
  for (int s2 = 0; s2 < 16; ++s2) {
    const int j = threadIdx.x + (N / 16) * s2;
    const double2 z = buf[pw_pad(pw_pos<N>(j))];
    store_px(map + 2 * j, z.x, add);
    store_px(map + 2 * j + 1, z.y, add);
  }
}

// ring -> phase
template <typename T, int N>
__global__ void __launch_bounds__(N / 16)
ring2phase_pow2_kernel(const int *__restrict__ pairs, const int *__restrict__ mlim,
                       const int *__restrict__ nph, const long long *__restrict__ ofs,
                       const double *__restrict__ phi0, const double *__restrict__ weight,
                       const int *__restrict__ fftidx, const FftDesc *__restrict__ fdesc,
                       const double2 *__restrict__ twiddle, double2 *__restrict__ phase,
                       int ncm, int mmax, int flags, const T *const *__restrict__ maps,
                       long long map_lo) {
  extern __shared__ double2 smem[];
  double2 *buf = smem;
  double2 *slo = smem + pw_entries(N);
  double2 *shi = slo + kShiftLo;
  // twiddle slices for the unpacking: W^k = twh[k / 64] twl[k mod 64], k <= N
  double2 *twl = shi + (mmax / kShiftLo + 2), *twh = twl + kTwLo;
  const int p = pairs[blockIdx.x >> 1], h = blockIdx.x & 1, c = blockIdx.y;
  const int ring = 2 * p + h;
  if (nph[ring] <= 0) return;
  const int ms = mmax + 1;
  const int mm = min(mmax, mlim[p]);
  const double wgt = ((flags & SHARP_USE_WEIGHTS) ? weight[ring] : 1.0) *
                     ((flags & SHARP_REAL_HARMONICS) ? kSqrtTwo : 1.0);
  const double ph = phi0[ring];
  const bool rot = fabs(ph) >= 1e-14;
  const double2 *W = twiddle + fdesc[fftidx[ring]].tw;
  const T *map = maps[c] + (ofs[ring] - map_lo);
  if (rot) build_shift(slo, shi, mm, -ph);
  load_twshared(twl, twh, W, N + 1);   // W: the table of 2N entries
  // pixels 2j, 2j+1 for j = tid + (N/16) s2: this thread's inputs of the
  // first pass, which runs from registers
  double2 v[16];
#pragma unroll
  for (int s2 = 0; s2 < 16; ++s2) {
    const int j = threadIdx.x + (N / 16) * s2;
    v[s2] = make_double2(double(map[2 * j]), double(map[2 * j + 1]));
  }
  pw_pass16_regs<N, false>(v, buf, N, W, 2 * N);
  __syncthreads();
  pw_fft_rest<N, false>(buf, W, 2 * N);
  // X_k = (Z_k + conj Z_{N-k})/2 - i W^k (Z_k - conj Z_{N-k})/2, k <= N;
  // phase_m = X_m wgt e^{-i m phi0} for m <= mm (<= N: no folding)
  double2 *dst = phase + ((long long)(p * ncm + c) * 2 + h) * ms;
  for (int k = threadIdx.x; k <= mm; k += N / 16) {
    const double2 zk = buf[pw_pad(pw_pos<N>(k == N ? 0 : k))];
    const double2 zn = cconj(buf[pw_pad(pw_pos<N>(k == 0 ? 0 : N - k))]);
    const double2 sm = cadd(zk, zn), df = csub(zk, zn);
    const double2 w = cmul(twh[k >> 6], twl[k & (kTwLo - 1)]);
    const double2 mi_w = make_double2(w.y, -w.x);  // -i * w
    double2 xk = cscale(cadd(sm, cmul(mi_w, df)), 0.5);
    if (k == 0 || k == N) xk.y = 0.0;
    double2 v = cscale(xk, wgt);
    if (rot) v = cmul(v, shift_of(slo, shi, k));
    dst[k] = v;
  }
}

// ---------------------------------------------------------------------------
// Bluestein rings in registers: even rings n = 2N whose complex length N
// takes the Bluestein convolution with M in {1024, 2048, 4096, 8192} (the
// polar HEALPix rings nph = 4i whose i has a large prime factor), with any
// stride and any alias folding.  One CTA per ring and component, M/16
// threads.  The convolution reuses the radix-16 passes of the power-of-two
// rings over one padded shared buffer:
//  * forward passes over x_j c_j, c_j = exp(-pi i j^2/N), whose upper half
//    (j >= M/2 >= N) is the zero padding and is not read;
//  * the product with the chirp spectrum (DFT of b_j = conj c_j, |j| < N,
//    scaled by 1/M and stored in the passes' digit order) fused between the
//    last forward pass and the first transposed one, which act on the same
//    registers;
//  * the transposed passes back to natural order; of the last only the
//    lower half (the outputs k < N) is stored.
// X_k = c_k (x c * b)_k; the inverse transform is conj(forward(conj x)).
// The alias folding and the real-FFT twist run in the same buffer around
// the convolution, pairing k with N-k so that each thread updates its own
// entries in place.
// ---------------------------------------------------------------------------
// c_j from the ring's table exp(-2 pi i e/n): c_j = W[j^2 mod n] (n = 2N)
__device__ __forceinline__ double2 pb_chirp(const double2 *__restrict__ W, int j, int n) {
  return __ldg(W + int((unsigned(j) * unsigned(j)) % unsigned(n)));
}

// In place: natural-order input (upper half zero) -> M times the cyclic
// convolution with b, natural order, lower half.  W: exp(-2 pi i j/tl).
// The callers run the first forward pass themselves from registers
// (pw_pass16_regs on the entries tid + (M/16) i, i < 8, the rest zero,
// then a __syncthreads); this runs the rest.
template <int M>
__device__ void pb_convolve(double2 *buf, const double2 *__restrict__ W, int tl,
                            const double2 *__restrict__ bh) {
  constexpr int P16 = pw_passes16(M), RL = pw_last(M);
  constexpr int FWD = (RL > 1) ? P16 : P16 - 1;   // radix-16 passes before the product
  int len = M >> 4;
#pragma unroll
  for (int q = 1; q < FWD; ++q) {
    pw_pass16<M, false>(buf, len, W, tl);
    __syncthreads();
    len >>= 4;
  }
  if constexpr (RL > 1) {
    // last forward pass (radix RL, unit twiddles), product, its inverse
#pragma unroll
    for (int q = 0; q < 16 / RL; ++q) {
      const int b = threadIdx.x + (M / 16) * q;
      double2 v[RL];
#pragma unroll
      for (int i = 0; i < RL; ++i) v[i] = buf[pw_pad(b * RL + i)];
      small_dft<RL>(v, false);
#pragma unroll
      for (int i = 0; i < RL; ++i) v[i] = cmul(v[i], __ldg(bh + b * RL + i));
      small_dft<RL>(v, true);
#pragma unroll
      for (int i = 0; i < RL; ++i) buf[pw_pad(b * RL + i)] = v[i];
    }
  } else {
    // the radix-16 pass of length 16 (unit twiddles), product, its inverse
    const int b = threadIdx.x * 16;
    double2 v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = buf[pw_pad(b + i)];
    dft16<false>(v);
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = cmul(v[i], __ldg(bh + b + i));
    dft16<true>(v);
#pragma unroll
    for (int i = 0; i < 16; ++i) buf[pw_pad(b + i)] = v[i];
  }
  __syncthreads();
  len = (RL > 1) ? 16 * RL : 256;
#pragma unroll
  for (int q = 0; q < FWD; ++q) {
    if (q == FWD - 1) pw_pass16_back<M, 8>(buf, len, W, tl);
    else pw_pass16_back<M>(buf, len, W, tl);
    __syncthreads();
    len <<= 4;
  }
}

// Chirp spectra in the digit order of the register passes: one CTA per
// descriptor of blue2 (those of other lengths return at once).
template <int M>
__global__ void __launch_bounds__(M / 16)
bluestein_pw_setup_kernel(const FftDesc *__restrict__ fdesc, const int *__restrict__ blue2_idx,
                          const double2 *__restrict__ twiddle,
                          const double2 *__restrict__ wpow2, int P,
                          double2 *__restrict__ bhat, double2 *__restrict__ chirp) {
  extern __shared__ double2 smem[];
  const FftDesc &d = fdesc[blue2_idx[blockIdx.x]];
  if (d.M != M) return;
  const int N = d.N, n = d.n;
  const long long o = d.bhat2;
  const double2 *W = twiddle + d.tw;
  for (int j = threadIdx.x; j < N; j += M / 16) chirp[d.chirp + j] = pb_chirp(W, j, n);
  for (int j = threadIdx.x; j < M; j += M / 16) {
    const int jj = j < N ? j : (j > M - N ? M - j : -1);
    smem[pw_pad(j)] = jj >= 0 ? cconj(pb_chirp(W, jj, n)) : make_double2(0.0, 0.0);
  }
  __syncthreads();
  pw_fft<M, false>(smem, wpow2, P);
  for (int j = threadIdx.x; j < M; j += M / 16)
    bhat[o + j] = cscale(smem[pw_pad(j)], 1.0 / M);
}

// CTAs per SM the register Bluestein kernels are compiled for (at most 128
// registers: two CTAs of 256 threads at M = 4096 instead of one at ~150)
__host__ __device__ constexpr int blue_min_blocks(int M) {
  return M == 4096 ? 2 : M == 2048 ? 4 : M == 1024 ? 8 : 1;
}

// phase -> ring.  Grid: (2 * pairs of this length, components).
template <typename T, int M>
__global__ void __launch_bounds__(M / 16, blue_min_blocks(M))
phase2ring_blue_kernel(const int *__restrict__ pairs, const int *__restrict__ mlim,
                       const int *__restrict__ nph, const long long *__restrict__ ofs,
                       const int *__restrict__ stride, const double *__restrict__ phi0,
                       const double *__restrict__ weight, const int *__restrict__ fftidx,
                       const FftDesc *__restrict__ fdesc, const double2 *__restrict__ twiddle,
                       const double2 *__restrict__ wpow2, int P,
                       const double2 *__restrict__ bhat, const double2 *__restrict__ chirp,
                       const double2 *__restrict__ phase, int ncm, int mmax, int flags,
                       T *const *__restrict__ maps, long long map_lo, int stage_row) {
  constexpr int NT = M / 16;
  extern __shared__ double2 smem[];
  __shared__ uint64_t row_full;
  double2 *buf = smem;
  double2 *slo = smem + pw_entries(M);
  double2 *shi = slo + kShiftLo;
  // stage_row: the phase row (mm + 1 <= mmax + 1 entries) is copied into
  // shared memory behind the phi0 slices, so the alias fold reads it there
  double2 *srow = shi + (mmax / kShiftLo + 2);
  const int p = pairs[blockIdx.x >> 1], h = blockIdx.x & 1, c = blockIdx.y;
  const int ring = 2 * p + h;
  const int n = nph[ring];
  if (n <= 0) return;        // unpaired ring: nothing in this hemisphere
  const int N = n / 2;
  const FftDesc &fd = fdesc[fftidx[ring]];
  const double2 *W = twiddle + fd.tw;     // exp(-2 pi i e/n)
  const double2 *bh = bhat + fd.bhat2;
  const double2 *cz = chirp + fd.chirp;   // c_j, j < N
  const int ms = mmax + 1;
  const int mm = min(mmax, mlim[p]);
  const bool add = (flags & (SHARP_ADD | SHARP_SUBTRACT)) != 0;
  const double wgt = ((flags & SHARP_USE_WEIGHTS) ? weight[ring] : 1.0) *
                     ((flags & SHARP_REAL_HARMONICS) ? kSqrtHalf : 1.0) *
                     ((flags & SHARP_SUBTRACT) ? -1.0 : 1.0);
  const double ph = phi0[ring];
  const bool rot = fabs(ph) >= 1e-14;
  const double2 *src = phase + ((long long)(p * ncm + c) * 2 + h) * ms;
  if (stage_row) {
    if (threadIdx.x == 0) {
      mbar_init(&row_full, 1);
      fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      mbar_arrive_tx(&row_full, uint32_t(16 * (mm + 1)));
      bulk_g2s(srow, src, uint32_t(16 * (mm + 1)), &row_full);
    }
  }
  if (rot) build_shift(slo, shi, mm, ph);
  if (stage_row) {
    // a copy that did not complete within the bounded wait is redone by
    // the threads (the same values)
    if (__syncthreads_or(!mbar_wait(&row_full, 0))) {
      for (int m = threadIdx.x; m <= mm; m += NT) srow[m] = src[m];
    }
  }
  __syncthreads();
  const double2 *row = stage_row ? srow : src;
  auto tm = [&](int m) {
    double2 t = cscale(row[m], wgt);
    if (rot) t = cmul(t, shift_of(slo, shi, m));
    return t;
  };
  // C_k, k <= N: t_m folded onto bin m mod n, conj t_m onto (n - m) mod n
  // (sharp.c:265-300); C_0 and C_N real
  for (int k = threadIdx.x; k <= N; k += NT) {
    double2 acc = make_double2(0.0, 0.0);
    for (int m = k; m <= mm; m += n) acc = cadd(acc, tm(m));
    for (int m = (k == 0) ? n : n - k; m <= mm; m += n) acc = cadd(acc, cconj(tm(m)));
    if (k == 0 || k == N) acc.y = 0.0;
    buf[pw_pad(k)] = acc;
  }
  __syncthreads();
  // x_k = conj(Z_k) c_k with Z_k = (C_k + conj C_{N-k}) + i conj(W^k)
  // (C_k - conj C_{N-k}) for k < N, zero on [N, M/2): for k = tid + NT i,
  // i < 8, this thread's inputs of the first forward pass, which runs from
  // registers once every thread has read its C values
  double2 v[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const int k = threadIdx.x + NT * i;
    v[i] = make_double2(0.0, 0.0);
    if (i < 8 && k < N) {
      const double2 ck = buf[pw_pad(k)], cn = cconj(buf[pw_pad(N - k)]);
      const double2 sm = cadd(ck, cn), df = csub(ck, cn);
      const double2 w = __ldg(W + k);
      const double2 iw = make_double2(w.y, w.x);   // i * conj(w)
      v[i] = cmul(cconj(cadd(sm, cmul(iw, df))), __ldg(cz + k));
    }
  }
  __syncthreads();
  pw_pass16_regs<M, false>(v, buf, M, wpow2, P);
  __syncthreads();
  pb_convolve<M>(buf, wpow2, P, bh);
  // z_j = conj(c_j conv_j): pixels 2j, 2j+1 = Re, Im z_j
  T *map = maps[c] + (ofs[ring] - map_lo);
  const long long st = stride[ring];
  for (int j = threadIdx.x; j < N; j += NT) {
    const double2 z = cmul(buf[pw_pad(j)], __ldg(cz + j));
    store_px(map + (2 * j) * st, z.x, add);
    store_px(map + (2 * j + 1) * st, -z.y, add);
  }
}

// ring -> phase
template <typename T, int M>
__global__ void __launch_bounds__(M / 16, blue_min_blocks(M))
ring2phase_blue_kernel(const int *__restrict__ pairs, const int *__restrict__ mlim,
                       const int *__restrict__ nph, const long long *__restrict__ ofs,
                       const int *__restrict__ stride, const double *__restrict__ phi0,
                       const double *__restrict__ weight, const int *__restrict__ fftidx,
                       const FftDesc *__restrict__ fdesc, const double2 *__restrict__ twiddle,
                       const double2 *__restrict__ wpow2, int P,
                       const double2 *__restrict__ bhat, const double2 *__restrict__ chirp,
                       double2 *__restrict__ phase, int ncm, int mmax, int flags,
                       const T *const *__restrict__ maps, long long map_lo) {
  constexpr int NT = M / 16;
  extern __shared__ double2 smem[];
  double2 *buf = smem;
  double2 *slo = smem + pw_entries(M);
  double2 *shi = slo + kShiftLo;
  const int p = pairs[blockIdx.x >> 1], h = blockIdx.x & 1, c = blockIdx.y;
  const int ring = 2 * p + h;
  const int n = nph[ring];
  if (n <= 0) return;
  const int N = n / 2;
  const FftDesc &fd = fdesc[fftidx[ring]];
  const double2 *W = twiddle + fd.tw;
  const double2 *bh = bhat + fd.bhat2;
  const double2 *cz = chirp + fd.chirp;   // c_j, j < N
  const int ms = mmax + 1;
  const int mm = min(mmax, mlim[p]);
  const double wgt = ((flags & SHARP_USE_WEIGHTS) ? weight[ring] : 1.0) *
                     ((flags & SHARP_REAL_HARMONICS) ? kSqrtTwo : 1.0);
  const double ph = phi0[ring];
  const bool rot = fabs(ph) >= 1e-14;
  const T *map = maps[c] + (ofs[ring] - map_lo);
  const long long st = stride[ring];
  if (rot) build_shift(slo, shi, mm, -ph);
  // x_j c_j, x_j = pixels 2j + i (2j+1), zero on [N, M): for j = tid + NT i
  // this thread's inputs of the first forward pass, run from registers
  double2 v[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const int j = threadIdx.x + NT * i;
    v[i] = make_double2(0.0, 0.0);
    if (i < 8 && j < N)
      v[i] = cmul(make_double2(double(map[(2 * j) * st]), double(map[(2 * j + 1) * st])),
                  __ldg(cz + j));
  }
  pw_pass16_regs<M, false>(v, buf, M, wpow2, P);
  __syncthreads();
  pb_convolve<M>(buf, wpow2, P, bh);
  // Z_k = c_k conv_k (Z_N = Z_0);
  // X_k = (Z_k + conj Z_{N-k})/2 - i W^k (Z_k - conj Z_{N-k})/2, k <= N
  auto xout = [&](double2 zk, double2 zn, int k) {
    zn = cconj(zn);
    const double2 sm = cadd(zk, zn), df = csub(zk, zn);
    const double2 w = __ldg(W + k);
    const double2 mi_w = make_double2(w.y, -w.x);   // -i * w
    return cscale(cadd(sm, cmul(mi_w, df)), 0.5);
  };
  for (int k = threadIdx.x; 2 * k <= N; k += NT) {
    const int kk = N - k;
    const double2 zk = cmul(buf[pw_pad(k)], __ldg(cz + k));
    const double2 zn = (k == 0) ? zk : cmul(buf[pw_pad(kk)], __ldg(cz + kk));
    double2 xk = xout(zk, zn, k), xn = xout(zn, zk, kk);
    if (k == 0) { xk.y = 0.0; xn.y = 0.0; }   // DC and Nyquist are real
    buf[pw_pad(k)] = xk;
    if (kk != k) buf[pw_pad(kk)] = xn;
  }
  __syncthreads();
  // phase_m = X_{m mod n} (conjugated above N) wgt e^{-i m phi0}, m <= mm
  double2 *dst = phase + ((long long)(p * ncm + c) * 2 + h) * ms;
  for (int m = threadIdx.x; m <= mm; m += NT) {
    const int idx = m % n;
    double2 v = (idx <= N) ? buf[pw_pad(idx)] : cconj(buf[pw_pad(n - idx)]);
    v = cscale(v, wgt);
    if (rot) v = cmul(v, shift_of(slo, shi, m));
    dst[m] = v;
  }
}

// ---------------------------------------------------------------------------
// SHARP_NO_FFT: map entries are the complex phases themselves
// (libsharp/sharp.c:631-669); nph must equal mmax+1.
// ---------------------------------------------------------------------------
template <typename T2>
__global__ void phase2ring_direct_kernel(const int *__restrict__ mlim, const int *__restrict__ nph,
                                         const long long *__restrict__ ofs,
                                         const int *__restrict__ stride,
                                         const double *__restrict__ weight,
                                         const double2 *__restrict__ phase, int ncm,
                                         int mmax, int flags, T2 *const *__restrict__ maps,
                                         long long map_lo) {
  const int p = blockIdx.x, c = blockIdx.y;
  const int mm = min(mmax, mlim[p]);
  const bool add = (flags & (SHARP_ADD | SHARP_SUBTRACT)) != 0;
  T2 *map = maps[c];
  for (int h = 0; h < 2; ++h) {
    const int ring = 2 * p + h;
    const int n = nph[ring];
    if (n <= 0) continue;
    double wgt = (flags & SHARP_USE_WEIGHTS) ? n * weight[ring] : 1.0;
    if (flags & SHARP_REAL_HARMONICS) wgt *= kSqrtHalf;
    if (flags & SHARP_SUBTRACT) wgt = -wgt;
    const double2 *src = phase + ((long long)(p * ncm + c) * 2 + h) * (mmax + 1);
    for (int m = threadIdx.x; m <= mmax; m += blockDim.x) {
      const double2 v = (m <= mm) ? cscale(src[m], wgt) : make_double2(0.0, 0.0);
      T2 *px = map + (ofs[ring] - map_lo) + (long long)m * stride[ring];
      if (add) {
        px->x += decltype(px->x)(v.x);
        px->y += decltype(px->y)(v.y);
      } else {
        px->x = decltype(px->x)(v.x);
        px->y = decltype(px->y)(v.y);
      }
    }
  }
}

template <typename T2>
__global__ void ring2phase_direct_kernel(const int *__restrict__ mlim, const int *__restrict__ nph,
                                         const long long *__restrict__ ofs,
                                         const int *__restrict__ stride,
                                         const double *__restrict__ weight,
                                         double2 *__restrict__ phase, int ncm,
                                         int mmax, int flags, const T2 *const *__restrict__ maps,
                                         long long map_lo) {
  const int p = blockIdx.x, c = blockIdx.y;
  const int mm = min(mmax, mlim[p]);
  const T2 *map = maps[c];
  for (int h = 0; h < 2; ++h) {
    const int ring = 2 * p + h;
    const int n = nph[ring];
    if (n <= 0) continue;
    double wgt = (flags & SHARP_USE_WEIGHTS) ? n * weight[ring] : 1.0;
    if (flags & SHARP_REAL_HARMONICS) wgt *= kSqrtTwo;
    double2 *dst = phase + ((long long)(p * ncm + c) * 2 + h) * (mmax + 1);
    for (int m = threadIdx.x; m <= mm; m += blockDim.x) {
      const T2 v = map[(ofs[ring] - map_lo) + (long long)m * stride[ring]];
      dst[m] = make_double2(double(v.x) * wgt, double(v.y) * wgt);
    }
  }
}

// ---------------------------------------------------------------------------
// a_lm staging (alm2almtmp, sharp.c:481-545) and scatter (almtmp2alm,
// sharp.c:547-606).  Staged values carry c_l (recurrence normalisation),
// norm_l (spin > 0 / derivatives) and the real-harmonics m=0 factor.
// ---------------------------------------------------------------------------
// a_lm staging and scatter: one CTA per m moves the m segment between the
// caller's arrays (l contiguous in each of the nalmptr arrays) and the rows
// of A (the components of one l contiguous), through a shared-memory tile of
// 2^lgtl l-values by nalmptr components (leading dimension nalmptr | 1, odd,
// so both access patterns are free of bank conflicts).  Each side of the
// copy is then coalesced: a warp reads or writes consecutive l of one array,
// or consecutive components of one row.
template <typename T>
__global__ void __launch_bounds__(256)
stage_alm_kernel(int lmax, int nalmptr, const long long *__restrict__ mvstart,
                 long long astride, bool packed, long long alm_lo,
                 const long long *__restrict__ moff, const double *__restrict__ cfac,
                 const double *__restrict__ norm_l, bool use_norm, double norm_m0,
                 const T *const *__restrict__ alm, double2 *__restrict__ A, int ncA, int lgtl) {
  extern __shared__ double2 tile[];
  const int tl = 1 << lgtl, ld = nalmptr | 1;
  const int m = blockIdx.x;
  const long long mo = moff[m] - m;
  const long long base = mvstart[m];
  const int nl = lmax - m + 1 + kPad;
  for (int l0 = 0; l0 < nl; l0 += tl) {
    for (int e = threadIdx.x; e < tl * nalmptr; e += blockDim.x) {
      const int r = e & (tl - 1), c = e >> lgtl;
      const int l = m + l0 + r;
      double2 v = make_double2(0.0, 0.0);
      if (l <= lmax) {
        const T *a = alm[c];
        if (packed) {
          if (m == 0) {
            v.x = double(a[base + l * astride - alm_lo]);
          } else {
            const long long ri = base + 2 * l * astride - alm_lo;
            v = make_double2(double(a[ri]), double(a[ri + 1]));
          }
        } else {
          const long long ri = 2 * (base + l * astride - alm_lo);
          v.x = double(a[ri]);
          v.y = (m == 0) ? 0.0 : double(a[ri + 1]);
        }
        double f = cfac[mo + l];
        if (use_norm) f *= norm_l[l];
        if (m == 0) f *= norm_m0;
        v = cscale(v, f);
      }
      tile[r * ld + c] = v;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < tl * nalmptr; e += blockDim.x) {
      const int r = e / nalmptr, c = e - r * nalmptr;
      if (l0 + r < nl) A[(mo + m + l0 + r) * ncA + c] = tile[r * ld + c];
    }
    __syncthreads();
  }
}

template <typename T>
__global__ void __launch_bounds__(256)
scatter_alm_kernel(int lmax, int nalmptr, const long long *__restrict__ mvstart,
                   long long astride, bool packed, long long alm_lo,
                   const long long *__restrict__ moff, const double *__restrict__ cfac,
                   const double *__restrict__ norm_l, bool use_norm, double norm_m0, double sgn,
                   bool add, const double *__restrict__ Aout, int ncA,
                   T *const *__restrict__ alm, int lgtl) {
  extern __shared__ double2 tile[];
  const int tl = 1 << lgtl, ld = nalmptr | 1;
  const int m = blockIdx.x;
  const long long mo = moff[m] - m;
  const long long base = mvstart[m];
  const int nl = lmax - m + 1;
  const double2 *src = reinterpret_cast<const double2 *>(Aout);
  for (int l0 = 0; l0 < nl; l0 += tl) {
    for (int e = threadIdx.x; e < tl * nalmptr; e += blockDim.x) {
      const int r = e / nalmptr, c = e - r * nalmptr;
      if (l0 + r < nl) tile[r * ld + c] = src[(mo + m + l0 + r) * ncA + c];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < tl * nalmptr; e += blockDim.x) {
      const int r = e & (tl - 1), c = e >> lgtl;
      if (l0 + r >= nl) continue;
      const int l = m + l0 + r;
      const double2 v = tile[r * ld + c];
      double f = cfac[mo + l] * sgn;
      if (use_norm) f *= norm_l[l];
      double vr = v.x * f, vi = v.y * f;
      T *a = alm[c];
      if (m == 0) {
        vr *= norm_m0;
        if (packed) {
          T *px = a + (base + l * astride - alm_lo);
          *px = add ? T(*px + T(vr)) : T(vr);
        } else {
          T *px = a + 2 * (base + l * astride - alm_lo);
          if (add) {
            px[0] += T(vr);
          } else {
            px[0] = T(vr);
            px[1] = T(0);
          }
        }
      } else {
        T *px = packed ? a + (base + 2 * l * astride - alm_lo)
                       : a + 2 * (base + l * astride - alm_lo);
        if (add) {
          px[0] += T(vr);
          px[1] += T(vi);
        } else {
          px[0] = T(vr);
          px[1] = T(vi);
        }
      }
    }
    __syncthreads();
  }
}

__global__ void twiddle_kernel(int ntab, const int *__restrict__ tn, const int *__restrict__ toff,
                               double2 *__restrict__ tw) {
  const int t = blockIdx.y;
  if (t >= ntab) return;
  const int n = tn[t];
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    double s, c;
    sincospi(2.0 * j / n, &s, &c);
    tw[toff[t] + j] = make_double2(c, -s);
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
void launch_twiddles(GeomPlan &gp, int ntw, const std::vector<int> &tw_n,
                     const std::vector<int> &tw_off, cudaStream_t st) {
  if (tw_n.empty()) return;
  int *d_n = nullptr, *d_off = nullptr;
  const int nt = int(tw_n.size());
  SHT_CUDA(::sht::ws_alloc(&d_n, sizeof(int) * nt, st));
  SHT_CUDA(::sht::ws_alloc(&d_off, sizeof(int) * nt, st));
  SHT_CUDA(cudaMemcpyAsync(d_n, tw_n.data(), sizeof(int) * nt, cudaMemcpyHostToDevice, st));
  SHT_CUDA(cudaMemcpyAsync(d_off, tw_off.data(), sizeof(int) * nt, cudaMemcpyHostToDevice, st));
  (void)ntw;
  dim3 grid(8, nt);
  ProfScope ps("twiddles", st);
  twiddle_kernel<<<grid, 256, 0, st>>>(nt, d_n, d_off, gp.twiddle);
  SHT_CUDA(cudaGetLastError());
  SHT_CUDA(cudaFreeAsync(d_n, st));
  SHT_CUDA(cudaFreeAsync(d_off, st));
}

// Ring pairs are launched per size class (largest complex FFT length of
// the pair <= cls_N[c]) so small polar rings do not reserve the shared
// memory and threads of the largest rings.
namespace {

// The register-pass chirp spectra, one launch per convolution length.
void launch_bluestein_pw_setup(const GeomPlan &gp, const int *d_blue2_idx, int nblue2,
                               cudaStream_t st) {
  if (nblue2 <= 0) return;
  ProfScope ps("bluestein_setup", st);
  auto one = [&](auto kernel, int M) {
    const size_t smem = sizeof(double2) * pw_entries(M);
    SHT_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  int(smem)));
    kernel<<<nblue2, M / 16, smem, st>>>(gp.fdesc, d_blue2_idx, gp.twiddle, gp.wpow2, gp.P,
                                         gp.bhat, gp.chirp);
    SHT_CUDA(cudaGetLastError());
  };
  if (gp.P >= 1024) one(bluestein_pw_setup_kernel<1024>, 1024);
  if (gp.P >= 2048) one(bluestein_pw_setup_kernel<2048>, 2048);
  if (gp.P >= 4096) one(bluestein_pw_setup_kernel<4096>, 4096);
  if (gp.P >= 8192) one(bluestein_pw_setup_kernel<8192>, 8192);
}

}  // namespace

void launch_bluestein_setup(GeomPlan &gp, const GeomHost &h, cudaStream_t st) {
  const std::vector<int> &idx = h.blue_idx;
  // exp(-2 pi i j/P) for the power-of-two passes (computed even when unused)
  std::vector<int> pn{gp.P}, po{0};
  {
    int *d_n = nullptr, *d_off = nullptr;
    SHT_CUDA(::sht::ws_alloc(&d_n, sizeof(int), st));
    SHT_CUDA(::sht::ws_alloc(&d_off, sizeof(int), st));
    SHT_CUDA(cudaMemcpyAsync(d_n, pn.data(), sizeof(int), cudaMemcpyHostToDevice, st));
    SHT_CUDA(cudaMemcpyAsync(d_off, po.data(), sizeof(int), cudaMemcpyHostToDevice, st));
    ProfScope ps("twiddles", st);
    twiddle_kernel<<<dim3(8, 1), 256, 0, st>>>(1, d_n, d_off, gp.wpow2);
    SHT_CUDA(cudaGetLastError());
    SHT_CUDA(cudaFreeAsync(d_n, st));
    SHT_CUDA(cudaFreeAsync(d_off, st));
  }
  if (!idx.empty()) {
    int *d_idx = nullptr;
    SHT_CUDA(::sht::ws_alloc(&d_idx, sizeof(int) * idx.size(), st));
    SHT_CUDA(cudaMemcpyAsync(d_idx, idx.data(), sizeof(int) * idx.size(),
                             cudaMemcpyHostToDevice, st));
    ProfScope ps("bluestein_setup", st);
    bluestein_setup_kernel<<<int(idx.size()), 256, 0, st>>>(gp.fdesc, d_idx, gp.twiddle,
                                                            gp.wpow2, gp.P, gp.bhat);
    SHT_CUDA(cudaGetLastError());
    SHT_CUDA(cudaFreeAsync(d_idx, st));
  }
  const std::vector<int> &idx2 = h.blue2_idx;
  if (!idx2.empty()) {
    int *d_idx = nullptr;
    SHT_CUDA(::sht::ws_alloc(&d_idx, sizeof(int) * idx2.size(), st));
    SHT_CUDA(cudaMemcpyAsync(d_idx, idx2.data(), sizeof(int) * idx2.size(),
                             cudaMemcpyHostToDevice, st));
    launch_bluestein_pw_setup(gp, d_idx, int(idx2.size()), st);
    SHT_CUDA(cudaFreeAsync(d_idx, st));
  }
}

static size_t fft_smem(const GeomPlan &gp, int cls, int mmax) {
  return sizeof(double2) * ring_fft_smem_entries(gp.cls_bufA[cls], gp.cls_bufB[cls], mmax,
                                                 gp.nmax_complex, gp.P);
}
static int fft_twcap(const GeomPlan &gp) { return ring_twiddle_hi_entries(gp.nmax_complex); }
static int fft_threads(int N) { return N <= 256 ? 64 : N <= 1024 ? 256 : 1024; }

namespace {

// Launch shape of one size class.  A class whose buffers exceed the shared
// memory of a CTA keeps only the phi0 and twiddle slices there and runs its
// buffers in a global scratch of two slots per SM (persistent CTAs).
constexpr size_t kSmemLimit = 227 * 1024;
struct FftLaunch {
  dim3 grid;
  int thr = 0;
  size_t smem = 0;
  double2 *gbuf = nullptr;
  int npc = 0, nitems = 0;
};
FftLaunch plan_fft_launch(const GeomPlan &gp, int cls, int mmax, int ncomp, cudaStream_t st) {
  FftLaunch L;
  L.npc = gp.cls_count[cls];
  L.nitems = L.npc * ncomp;
  L.thr = fft_threads(gp.cls_N[cls]);
  L.smem = fft_smem(gp, cls, mmax);
  L.grid = dim3(L.npc, ncomp);
  if (L.smem > kSmemLimit) {
    int dev = 0, nsm = 0;
    SHT_CUDA(cudaGetDevice(&dev));
    SHT_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int slots = std::min(L.nitems, 2 * std::max(nsm, 1));
    L.grid = dim3(slots, 1);
    L.thr = 1024;
    L.smem = sizeof(double2) * ring_fft_smem_entries(0, 0, mmax, gp.nmax_complex, gp.P);
    SHT_CUDA(::sht::ws_alloc(&L.gbuf, sizeof(double2) * size_t(slots) *
                                          (gp.cls_bufA[cls] + gp.cls_bufB[cls]), st));
  }
  return L;
}

template <typename T>
void phase2ring_class(const JobDesc &job, const GeomPlan &gp, int cls, long long map_lo,
                      const double2 *phase, int ncm, void *const *maps_dev, int nmapptr,
                      cudaStream_t st) {
  const FftLaunch L = plan_fft_launch(gp, cls, job.mmax, nmapptr, st);
  auto k = phase2ring_kernel<T>;
  SHT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(L.smem)));
  k<<<L.grid, L.thr, L.smem, st>>>(gp.cls_pairs + gp.cls_start[cls], gp.mlim, gp.nph, gp.ofs,
                                   gp.stride, gp.phi0, gp.weight, gp.fft, gp.fdesc, gp.twiddle,
                                   gp.wpow2, gp.P, gp.bhat, phase, ncm, job.mmax, job.flags,
                                   gp.cls_bufA[cls], gp.cls_bufB[cls], fft_twcap(gp),
                                   reinterpret_cast<T *const *>(maps_dev), map_lo, L.gbuf, L.npc,
                                   L.nitems);
  SHT_CUDA(cudaGetLastError());
  if (L.gbuf) SHT_CUDA(cudaFreeAsync(L.gbuf, st));
}

template <typename T>
void ring2phase_class(const JobDesc &job, const GeomPlan &gp, int cls, long long map_lo,
                      const void *const *maps_dev, int nmapptr, double2 *phase, int ncm,
                      cudaStream_t st) {
  const FftLaunch L = plan_fft_launch(gp, cls, job.mmax, nmapptr, st);
  auto k = ring2phase_kernel<T>;
  SHT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(L.smem)));
  k<<<L.grid, L.thr, L.smem, st>>>(gp.cls_pairs + gp.cls_start[cls], gp.mlim, gp.nph, gp.ofs,
                                   gp.stride, gp.phi0, gp.weight, gp.fft, gp.fdesc, gp.twiddle,
                                   gp.wpow2, gp.P, gp.bhat, phase, ncm, job.mmax, job.flags,
                                   gp.cls_bufA[cls], gp.cls_bufB[cls], fft_twcap(gp),
                                   reinterpret_cast<const T *const *>(maps_dev), map_lo, L.gbuf,
                                   L.npc, L.nitems);
  SHT_CUDA(cudaGetLastError());
  if (L.gbuf) SHT_CUDA(cudaFreeAsync(L.gbuf, st));
}

}  // namespace

namespace {

size_t pow2_smem(int N, int mmax) {
  return sizeof(double2) * (size_t(pw_entries(N)) + kShiftLo + mmax / kShiftLo + 2);
}

template <typename T, int N>
void phase2ring_pow2(const JobDesc &job, const GeomPlan &gp, int cls, long long map_lo,
                     const double2 *phase, int ncm, void *const *maps_dev, int nmapptr,
                     cudaStream_t st) {
  auto k = phase2ring_pow2_kernel<T, N>;
  const size_t smem = pow2_smem(N, job.mmax);
  SHT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  k<<<dim3(2 * gp.pw_count[cls], nmapptr), N / 16, smem, st>>>(
      gp.pw_pairs + gp.pw_start[cls], gp.mlim, gp.nph, gp.ofs, gp.phi0, gp.weight, gp.fft,
      gp.fdesc, gp.twiddle, phase, ncm, job.mmax, job.flags,
      reinterpret_cast<T *const *>(maps_dev), map_lo);
  SHT_CUDA(cudaGetLastError());
}

template <typename T, int N>
void ring2phase_pow2(const JobDesc &job, const GeomPlan &gp, int cls, long long map_lo,
                     const void *const *maps_dev, int nmapptr, double2 *phase, int ncm,
                     cudaStream_t st) {
  auto k = ring2phase_pow2_kernel<T, N>;
  // plus the twiddle slices of the unpacking
  const size_t smem = pow2_smem(N, job.mmax) + sizeof(double2) * (kTwLo + N / kTwLo + 1);
  SHT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  k<<<dim3(2 * gp.pw_count[cls], nmapptr), N / 16, smem, st>>>(
      gp.pw_pairs + gp.pw_start[cls], gp.mlim, gp.nph, gp.ofs, gp.phi0, gp.weight, gp.fft,
      gp.fdesc, gp.twiddle, phase, ncm, job.mmax, job.flags,
      reinterpret_cast<const T *const *>(maps_dev), map_lo);
  SHT_CUDA(cudaGetLastError());
}

template <typename T, int M>
void phase2ring_blue(const JobDesc &job, const GeomPlan &gp, int cls, long long map_lo,
                     const double2 *phase, int ncm, void *const *maps_dev, int nmapptr,
                     cudaStream_t st) {
  auto k = phase2ring_blue_kernel<T, M>;
  // the phase row is staged in shared memory where that keeps the CTAs per
  // SM (M = 8192: one CTA per SM either way) and fits
  const size_t base = pow2_smem(M, job.mmax);
  const size_t with_row = base + sizeof(double2) * (job.mmax + 1);
  const int stage_row = (M == 8192 && with_row + 1024 <= 227 * 1024) ? 1 : 0;
  const size_t smem = stage_row ? with_row : base;
  SHT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  k<<<dim3(2 * gp.pb_count[cls], nmapptr), M / 16, smem, st>>>(
      gp.pb_pairs + gp.pb_start[cls], gp.mlim, gp.nph, gp.ofs, gp.stride, gp.phi0, gp.weight,
      gp.fft, gp.fdesc, gp.twiddle, gp.wpow2, gp.P, gp.bhat, gp.chirp, phase, ncm, job.mmax,
      job.flags, reinterpret_cast<T *const *>(maps_dev), map_lo, stage_row);
  SHT_CUDA(cudaGetLastError());
}

template <typename T, int M>
void ring2phase_blue(const JobDesc &job, const GeomPlan &gp, int cls, long long map_lo,
                     const void *const *maps_dev, int nmapptr, double2 *phase, int ncm,
                     cudaStream_t st) {
  auto k = ring2phase_blue_kernel<T, M>;
  const size_t smem = pow2_smem(M, job.mmax);
  SHT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  k<<<dim3(2 * gp.pb_count[cls], nmapptr), M / 16, smem, st>>>(
      gp.pb_pairs + gp.pb_start[cls], gp.mlim, gp.nph, gp.ofs, gp.stride, gp.phi0, gp.weight,
      gp.fft, gp.fdesc, gp.twiddle, gp.wpow2, gp.P, gp.bhat, gp.chirp, phase, ncm, job.mmax,
      job.flags, reinterpret_cast<const T *const *>(maps_dev), map_lo);
  SHT_CUDA(cudaGetLastError());
}

template <typename T>
void phase2ring_pow2_classes(const JobDesc &job, const GeomPlan &gp, long long map_lo,
                             const double2 *phase, int ncm, void *const *maps_dev, int nmapptr,
                             cudaStream_t st) {
  for (int c = 0; c < int(gp.pw_N.size()); ++c) {
    if (gp.pw_count[c] == 0) continue;
    switch (gp.pw_N[c]) {
      case 1024: phase2ring_pow2<T, 1024>(job, gp, c, map_lo, phase, ncm, maps_dev, nmapptr, st); break;
      case 2048: phase2ring_pow2<T, 2048>(job, gp, c, map_lo, phase, ncm, maps_dev, nmapptr, st); break;
      case 4096: phase2ring_pow2<T, 4096>(job, gp, c, map_lo, phase, ncm, maps_dev, nmapptr, st); break;
      default: phase2ring_pow2<T, 8192>(job, gp, c, map_lo, phase, ncm, maps_dev, nmapptr, st); break;
    }
  }
  for (int c = 0; c < int(gp.pb_M.size()); ++c) {
    if (gp.pb_count[c] == 0) continue;
    switch (gp.pb_M[c]) {
      case 1024: phase2ring_blue<T, 1024>(job, gp, c, map_lo, phase, ncm, maps_dev, nmapptr, st); break;
      case 2048: phase2ring_blue<T, 2048>(job, gp, c, map_lo, phase, ncm, maps_dev, nmapptr, st); break;
      case 4096: phase2ring_blue<T, 4096>(job, gp, c, map_lo, phase, ncm, maps_dev, nmapptr, st); break;
      default: phase2ring_blue<T, 8192>(job, gp, c, map_lo, phase, ncm, maps_dev, nmapptr, st); break;
    }
  }
}

template <typename T>
void ring2phase_pow2_classes(const JobDesc &job, const GeomPlan &gp, long long map_lo,
                             const void *const *maps_dev, int nmapptr, double2 *phase, int ncm,
                             cudaStream_t st) {
  for (int c = 0; c < int(gp.pw_N.size()); ++c) {
    if (gp.pw_count[c] == 0) continue;
    switch (gp.pw_N[c]) {
      case 1024: ring2phase_pow2<T, 1024>(job, gp, c, map_lo, maps_dev, nmapptr, phase, ncm, st); break;
      case 2048: ring2phase_pow2<T, 2048>(job, gp, c, map_lo, maps_dev, nmapptr, phase, ncm, st); break;
      case 4096: ring2phase_pow2<T, 4096>(job, gp, c, map_lo, maps_dev, nmapptr, phase, ncm, st); break;
      default: ring2phase_pow2<T, 8192>(job, gp, c, map_lo, maps_dev, nmapptr, phase, ncm, st); break;
    }
  }
  for (int c = 0; c < int(gp.pb_M.size()); ++c) {
    if (gp.pb_count[c] == 0) continue;
    switch (gp.pb_M[c]) {
      case 1024: ring2phase_blue<T, 1024>(job, gp, c, map_lo, maps_dev, nmapptr, phase, ncm, st); break;
      case 2048: ring2phase_blue<T, 2048>(job, gp, c, map_lo, maps_dev, nmapptr, phase, ncm, st); break;
      case 4096: ring2phase_blue<T, 4096>(job, gp, c, map_lo, maps_dev, nmapptr, phase, ncm, st); break;
      default: ring2phase_blue<T, 8192>(job, gp, c, map_lo, maps_dev, nmapptr, phase, ncm, st); break;
    }
  }
}

}  // namespace

void launch_phase2ring(const JobDesc &job, const GeomPlan &gp, long long map_lo,
                       const double2 *phase, int ncm, void *const *maps_dev, int nmapptr,
                       cudaStream_t st) {
  ProfScope ps("ring_synth", st);
  if (job.dp)
    phase2ring_pow2_classes<double>(job, gp, map_lo, phase, ncm, maps_dev, nmapptr, st);
  else
    phase2ring_pow2_classes<float>(job, gp, map_lo, phase, ncm, maps_dev, nmapptr, st);
  for (int cls = 0; cls < int(gp.cls_N.size()); ++cls) {
    if (gp.cls_count[cls] == 0) continue;
    if (job.dp)
      phase2ring_class<double>(job, gp, cls, map_lo, phase, ncm, maps_dev, nmapptr, st);
    else
      phase2ring_class<float>(job, gp, cls, map_lo, phase, ncm, maps_dev, nmapptr, st);
  }
}

void launch_ring2phase(const JobDesc &job, const GeomPlan &gp, long long map_lo,
                       const void *const *maps_dev, int nmapptr, double2 *phase, int ncm,
                       cudaStream_t st) {
  ProfScope ps("ring_anal", st);
  if (job.dp)
    ring2phase_pow2_classes<double>(job, gp, map_lo, maps_dev, nmapptr, phase, ncm, st);
  else
    ring2phase_pow2_classes<float>(job, gp, map_lo, maps_dev, nmapptr, phase, ncm, st);
  for (int cls = 0; cls < int(gp.cls_N.size()); ++cls) {
    if (gp.cls_count[cls] == 0) continue;
    if (job.dp)
      ring2phase_class<double>(job, gp, cls, map_lo, maps_dev, nmapptr, phase, ncm, st);
    else
      ring2phase_class<float>(job, gp, cls, map_lo, maps_dev, nmapptr, phase, ncm, st);
  }
}

void launch_phase2ring_direct(const JobDesc &job, const GeomPlan &gp, long long map_lo,
                              const double2 *phase, int ncm, void *const *maps_dev, int nmapptr,
                              cudaStream_t st) {
  if (gp.npairs == 0) return;
  dim3 grid(gp.npairs, nmapptr);
  ProfScope ps("ring_synth", st);
  if (job.dp)
    phase2ring_direct_kernel<double2><<<grid, 128, 0, st>>>(
        gp.mlim, gp.nph, gp.ofs, gp.stride, gp.weight, phase, ncm, job.mmax,
        job.flags, reinterpret_cast<double2 *const *>(maps_dev), map_lo);
  else
    phase2ring_direct_kernel<float2><<<grid, 128, 0, st>>>(
        gp.mlim, gp.nph, gp.ofs, gp.stride, gp.weight, phase, ncm, job.mmax,
        job.flags, reinterpret_cast<float2 *const *>(maps_dev), map_lo);
  SHT_CUDA(cudaGetLastError());
}

void launch_ring2phase_direct(const JobDesc &job, const GeomPlan &gp, long long map_lo,
                              const void *const *maps_dev, int nmapptr, double2 *phase,
                              int ncm, cudaStream_t st) {
  if (gp.npairs == 0) return;
  dim3 grid(gp.npairs, nmapptr);
  ProfScope ps("ring_anal", st);
  if (job.dp)
    ring2phase_direct_kernel<double2><<<grid, 128, 0, st>>>(
        gp.mlim, gp.nph, gp.ofs, gp.stride, gp.weight, phase, ncm, job.mmax,
        job.flags, reinterpret_cast<const double2 *const *>(maps_dev), map_lo);
  else
    ring2phase_direct_kernel<float2><<<grid, 128, 0, st>>>(
        gp.mlim, gp.nph, gp.ofs, gp.stride, gp.weight, phase, ncm, job.mmax,
        job.flags, reinterpret_cast<const float2 *const *>(maps_dev), map_lo);
  SHT_CUDA(cudaGetLastError());
}

// log2 of the staging tile's l extent: at least 32 l-values (a warp's
// worth of one array) and about 512 entries per tile (few components: more
// l-values, so the 256 threads stay busy), at most 256, and no more than
// 48 KiB of shared memory (nalmptr | 1 entries per l).
static int stage_tile_lg(int nalmptr) {
  const size_t ld = size_t(nalmptr | 1);
  int lg = 5;
  while (lg < 8 && (2 << lg) * nalmptr <= 512) ++lg;
  while (lg > 0 && (sizeof(double2) << lg) * ld > 48 * 1024) --lg;
  return lg;
}

void launch_stage_alm(const JobDesc &job, const AlmPlan &ap, long long alm_lo,
                      const CoefPlan &cp, const double *norm_l, const void *const *alm_dev,
                      int nalmptr, double2 *A, int ncA, cudaStream_t st) {
  const bool use_norm = job.spin > 0 || job.type == SHARP_ALM2MAP_DERIV1;
  const double norm_m0 = (job.flags & SHARP_REAL_HARMONICS) ? kSqrtTwo : 1.0;
  const int blocks = job.mmax + 1;
  const int lg = stage_tile_lg(nalmptr);
  const size_t smem = (sizeof(double2) << lg) * size_t(nalmptr | 1);
  ProfScope ps("stage_alm", st);
  if (job.dp)
    stage_alm_kernel<double><<<blocks, 256, smem, st>>>(
        job.lmax, nalmptr, ap.mvstart, ap.stride, ap.packed, alm_lo, cp.d_moff, cp.cfac, norm_l,
        use_norm, norm_m0, reinterpret_cast<const double *const *>(alm_dev), A, ncA, lg);
  else
    stage_alm_kernel<float><<<blocks, 256, smem, st>>>(
        job.lmax, nalmptr, ap.mvstart, ap.stride, ap.packed, alm_lo, cp.d_moff, cp.cfac, norm_l,
        use_norm, norm_m0, reinterpret_cast<const float *const *>(alm_dev), A, ncA, lg);
  SHT_CUDA(cudaGetLastError());
}

void launch_scatter_alm(const JobDesc &job, const AlmPlan &ap, long long alm_lo,
                        const CoefPlan &cp, const double *norm_l, const double *Aout, int ncA,
                        void *const *alm_dev, int nalmptr, cudaStream_t st) {
  const bool use_norm = job.spin > 0 || job.type == SHARP_ALM2MAP_DERIV1;
  const double norm_m0 = (job.flags & SHARP_REAL_HARMONICS) ? kSqrtHalf : 1.0;
  // SHARP_SUBTRACT: the negated result is added (negation is exact)
  const double sgn = (job.flags & SHARP_SUBTRACT) ? -1.0 : 1.0;
  const bool add = (job.flags & (SHARP_ADD | SHARP_SUBTRACT)) != 0;
  const int blocks = job.mmax + 1;
  const int lg = stage_tile_lg(nalmptr);
  const size_t smem = (sizeof(double2) << lg) * size_t(nalmptr | 1);
  ProfScope ps("scatter_alm", st);
  if (job.dp)
    scatter_alm_kernel<double><<<blocks, 256, smem, st>>>(
        job.lmax, nalmptr, ap.mvstart, ap.stride, ap.packed, alm_lo, cp.d_moff, cp.cfac, norm_l,
        use_norm, norm_m0, sgn, add, Aout, ncA, reinterpret_cast<double *const *>(alm_dev), lg);
  else
    scatter_alm_kernel<float><<<blocks, 256, smem, st>>>(
        job.lmax, nalmptr, ap.mvstart, ap.stride, ap.packed, alm_lo, cp.d_moff, cp.cfac, norm_l,
        use_norm, norm_m0, sgn, add, Aout, ncA, reinterpret_cast<float *const *>(alm_dev), lg);
  SHT_CUDA(cudaGetLastError());
}

// Table set-up without temporary allocations: the caller has already placed
// the per-table lengths/offsets (and the Bluestein descriptor indices) in
// device memory.
void launch_twiddles_preplaced(double2 *tw, const int *d_n, const int *d_off, int ntab,
                               cudaStream_t st) {
  if (ntab <= 0) return;
  ProfScope ps("twiddles", st);
  twiddle_kernel<<<dim3(8, ntab), 256, 0, st>>>(ntab, d_n, d_off, tw);
  SHT_CUDA(cudaGetLastError());
}

void launch_bluestein_setup_preplaced(const GeomPlan &gp, const int *d_blue_idx, int nblue,
                                      const int *d_blue2_idx, int nblue2, cudaStream_t st) {
  if (nblue > 0) {
    ProfScope ps("bluestein_setup", st);
    bluestein_setup_kernel<<<nblue, 256, 0, st>>>(gp.fdesc, d_blue_idx, gp.twiddle, gp.wpow2,
                                                  gp.P, gp.bhat);
    SHT_CUDA(cudaGetLastError());
  }
  launch_bluestein_pw_setup(gp, d_blue2_idx, nblue2, st);
}

}  // namespace sht
