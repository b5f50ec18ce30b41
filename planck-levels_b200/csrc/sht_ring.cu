// Ring stage of the transform: phase <-> ring pixels with the per-ring real
// FFT, phi0 rotation, quadrature weight and alias folding, plus the a_lm
// staging/scatter kernels.
//
// Reference behaviour: libsharp/sharp.c:253-353 (ringhelper_phase2ring /
// ring2phase), :481-606 (alm2almtmp / almtmp2alm), :608-669 (ring gathers
// and the SHARP_NO_FFT path); FFT conventions of libfftpack/ls_fft.c:130-212
// (unnormalised backward transform, FFTPACK half-complex order).
//
// One CTA owns one (ring pair, component) and runs both hemispheres.  The FFT
// is a Stockham auto-sort mixed-radix transform in shared memory: even ring
// lengths n use a complex FFT of length n/2 on packed (x_2j + i x_2j+1) data;
// odd lengths a complex FFT of length n.  Radix-2/3/4/5 stages and a generic
// prime stage share one code path (each thread computes whole outputs, so
// large prime factors parallelise over outputs).  Twiddles come from a
// per-length table exp(-2 pi i j/n) computed once per geometry.
#include <cuda_runtime.h>

#include <cmath>

#include "sht_device.h"

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

// One Stockham pass of radix R: Ns = product of the radices already done.
// out[(j/Ns)*Ns*R + k + q*Ns] = sum_r in[j + r*N/R] w_N^{sign r (N/(Ns R)) (k + q Ns)}
__device__ void stockham_pass(const double2 *src, double2 *dst, int N, int R, int Ns, bool inv,
                              const double2 *__restrict__ W, int step) {
  const int NR = N / R;
  const int sf = N / (Ns * R);
  for (int item = threadIdx.x; item < N; item += blockDim.x) {
    const int j = item / R;
    const int q = item - j * R;
    const int k = j % Ns;
    int ang = (sf * (k + q * Ns)) % N;
    int e = 0;
    double2 acc = make_double2(0.0, 0.0);
    for (int r = 0; r < R; ++r) {
      double2 w = __ldg(W + e * step);
      if (inv) w.y = -w.y;
      const double2 v = src[j + r * NR];
      acc.x = fma(v.x, w.x, fma(-v.y, w.y, acc.x));
      acc.y = fma(v.x, w.y, fma(v.y, w.x, acc.y));
      e += ang;
      if (e >= N) e -= N;
    }
    dst[(j / Ns) * Ns * R + k + q * Ns] = acc;
  }
}

// Complex FFT of length d.N in buffers a/b; returns the buffer holding the
// result.  Callers synchronise before and after.
__device__ double2 *run_fft(const FftDesc &d, double2 *a, double2 *b, bool inv,
                            const double2 *__restrict__ twiddle) {
  const double2 *W = twiddle + d.tw;
  const int step = d.n / d.N;
  int Ns = 1;
  double2 *src = a, *dst = b;
  for (int s = 0; s < d.nrad; ++s) {
    const int R = d.rad[s];
    stockham_pass(src, dst, d.N, R, Ns, inv, W, step);
    __syncthreads();
    Ns *= R;
    double2 *t = src;
    src = dst;
    dst = t;
  }
  return src;
}

template <typename T>
__device__ __forceinline__ void store_px(T *p, double v, bool add) {
  if (add) *p += T(v);
  else *p = T(v);
}

// ---------------------------------------------------------------------------
// phase -> ring (synthesis)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256)
phase2ring_kernel(const int *__restrict__ mlim, const int *__restrict__ nph,
                  const long long *__restrict__ ofs, const int *__restrict__ stride,
                  const double *__restrict__ phi0, const double *__restrict__ weight,
                  const int *__restrict__ fftidx, const FftDesc *__restrict__ fdesc,
                  const double2 *__restrict__ twiddle, const double2 *__restrict__ phase,
                  int ncm, int npairs, int mmax, int flags, T *const *__restrict__ maps,
                  long long map_lo) {
  extern __shared__ double2 smem[];
  const int p = blockIdx.x;
  const int c = blockIdx.y;
  const int mm = min(mmax, mlim[p]);
  const bool add = (flags & SHARP_ADD) != 0;
  double wscale = (flags & SHARP_REAL_HARMONICS) ? kSqrtHalf : 1.0;
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
    double2 *bufA = smem;
    double2 *bufB = smem + (d.N + 2);
    double2 *C = bufB;
    const double2 *src = phase + ((long long)p * ncm + c) * 2 + h;
    const long long mstride = (long long)npairs * ncm * 2;
    // fold phase[m] * wgt * e^{i m phi0} into bins 0..half (sharp.c:265-300)
    for (int k = threadIdx.x; k <= half; k += blockDim.x) {
      double2 acc = make_double2(0.0, 0.0);
      for (int m = k; m <= mm; m += n) {
        double2 t = cscale(src[m * mstride], wgt);
        if (rot) {
          double sn, cs;
          sincos(m * ph, &sn, &cs);
          t = cmul(t, make_double2(cs, sn));
        }
        acc = cadd(acc, t);
      }
      for (int m = (k == 0) ? n : n - k; m <= mm; m += n) {
        double2 t = cscale(src[m * mstride], wgt);
        if (rot) {
          double sn, cs;
          sincos(m * ph, &sn, &cs);
          t = cmul(t, make_double2(cs, sn));
        }
        acc = cadd(acc, cconj(t));
      }
      if (k == 0 || 2 * k == n) acc.y = 0.0;
      C[k] = acc;
    }
    __syncthreads();
    const double2 *W = twiddle + d.tw;
    if ((n & 1) == 0) {
      // Z_k = (C_k + conj C_{N-k}) + i conj(W^k) (C_k - conj C_{N-k}), k < N
      for (int k = threadIdx.x; k < d.N; k += blockDim.x) {
        const double2 ck = C[k], cn = cconj(C[d.N - k]);
        const double2 s = cadd(ck, cn), df = csub(ck, cn);
        const double2 w = __ldg(W + k);  // exp(-2 pi i k/n)
        const double2 iw = make_double2(w.y, w.x);  // i * conj(w)
        bufA[k] = cadd(s, cmul(iw, df));
      }
    } else {
      for (int k = threadIdx.x; k < n; k += blockDim.x)
        bufA[k] = (k <= half) ? C[k] : cconj(C[n - k]);
    }
    __syncthreads();
    double2 *res = run_fft(d, bufA, bufB, true, twiddle);
    const long long o = ofs[ring] - map_lo;
    const long long st = stride[ring];
    if ((n & 1) == 0) {
      for (int j = threadIdx.x; j < d.N; j += blockDim.x) {
        const double2 z = res[j];
        store_px(map + o + (2 * j) * st, z.x, add);
        store_px(map + o + (2 * j + 1) * st, z.y, add);
      }
    } else {
      for (int j = threadIdx.x; j < n; j += blockDim.x) store_px(map + o + j * st, res[j].x, add);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// ring -> phase (analysis)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256)
ring2phase_kernel(const int *__restrict__ mlim, const int *__restrict__ nph,
                  const long long *__restrict__ ofs, const int *__restrict__ stride,
                  const double *__restrict__ phi0, const double *__restrict__ weight,
                  const int *__restrict__ fftidx, const FftDesc *__restrict__ fdesc,
                  const double2 *__restrict__ twiddle, double2 *__restrict__ phase, int ncm,
                  int npairs, int mmax, int flags, const T *const *__restrict__ maps,
                  long long map_lo) {
  extern __shared__ double2 smem[];
  const int p = blockIdx.x;
  const int c = blockIdx.y;
  const int mm = min(mmax, mlim[p]);
  const double wscale = (flags & SHARP_REAL_HARMONICS) ? kSqrtTwo : 1.0;
  const T *map = maps[c];
  for (int h = 0; h < 2; ++h) {
    const int ring = 2 * p + h;
    const int n = nph[ring];
    if (n <= 0) continue;
    const FftDesc d = fdesc[fftidx[ring]];
    const double wgt = ((flags & SHARP_USE_WEIGHTS) ? weight[ring] : 1.0) * wscale;
    const double ph = phi0[ring];
    const bool rot = fabs(ph) >= 1e-14;
    double2 *bufA = smem;
    double2 *bufB = smem + (d.N + 2);
    const long long o = ofs[ring] - map_lo;
    const long long st = stride[ring];
    if ((n & 1) == 0) {
      for (int j = threadIdx.x; j < d.N; j += blockDim.x)
        bufA[j] = make_double2(double(map[o + (2 * j) * st]), double(map[o + (2 * j + 1) * st]));
    } else {
      for (int j = threadIdx.x; j < n; j += blockDim.x)
        bufA[j] = make_double2(double(map[o + j * st]), 0.0);
    }
    __syncthreads();
    double2 *res = run_fft(d, bufA, bufB, false, twiddle);
    double2 *X = (res == bufA) ? bufB : bufA;
    const double2 *W = twiddle + d.tw;
    if ((n & 1) == 0) {
      // X_k = (Z_k + conj Z_{N-k})/2 - i W^k (Z_k - conj Z_{N-k})/2, k <= N
      for (int k = threadIdx.x; k <= d.N; k += blockDim.x) {
        const double2 zk = res[k == d.N ? 0 : k];
        const double2 zn = cconj(res[k == 0 ? 0 : d.N - k]);
        const double2 s = cadd(zk, zn), df = csub(zk, zn);
        const double2 w = __ldg(W + k);
        const double2 mi_w = make_double2(w.y, -w.x);  // -i * w
        double2 xk = cscale(cadd(s, cmul(mi_w, df)), 0.5);
        if (k == 0 || k == d.N) xk.y = 0.0;  // DC and Nyquist are real
        X[k] = xk;
      }
    } else {
      for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double2 xk = res[k];
        if (k == 0) xk.y = 0.0;
        X[k] = xk;
      }
    }
    __syncthreads();
    double2 *dst = phase + ((long long)p * ncm + c) * 2 + h;
    const long long mstride = (long long)npairs * ncm * 2;
    for (int m = threadIdx.x; m <= mm; m += blockDim.x) {
      const int idx = m % n;
      double2 v;
      if (idx < n - idx) v = X[idx];
      else v = cconj(X[n - idx]);
      v = cscale(v, wgt);
      if (rot) {
        double sn, cs;
        sincos(m * ph, &sn, &cs);
        v = cmul(v, make_double2(cs, -sn));
      }
      dst[m * mstride] = v;
    }
    __syncthreads();
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
                                         const double2 *__restrict__ phase, int ncm, int npairs,
                                         int mmax, int flags, T2 *const *__restrict__ maps,
                                         long long map_lo) {
  const int p = blockIdx.x, c = blockIdx.y;
  const int mm = min(mmax, mlim[p]);
  const bool add = (flags & SHARP_ADD) != 0;
  T2 *map = maps[c];
  for (int h = 0; h < 2; ++h) {
    const int ring = 2 * p + h;
    const int n = nph[ring];
    if (n <= 0) continue;
    double wgt = (flags & SHARP_USE_WEIGHTS) ? n * weight[ring] : 1.0;
    if (flags & SHARP_REAL_HARMONICS) wgt *= kSqrtHalf;
    const double2 *src = phase + ((long long)p * ncm + c) * 2 + h;
    const long long mstride = (long long)npairs * ncm * 2;
    for (int m = threadIdx.x; m <= mmax; m += blockDim.x) {
      const double2 v = (m <= mm) ? cscale(src[m * mstride], wgt) : make_double2(0.0, 0.0);
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
                                         double2 *__restrict__ phase, int ncm, int npairs,
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
    double2 *dst = phase + ((long long)p * ncm + c) * 2 + h;
    const long long mstride = (long long)npairs * ncm * 2;
    for (int m = threadIdx.x; m <= mm; m += blockDim.x) {
      const T2 v = map[(ofs[ring] - map_lo) + (long long)m * stride[ring]];
      dst[m * mstride] = make_double2(double(v.x) * wgt, double(v.y) * wgt);
    }
  }
}

// ---------------------------------------------------------------------------
// a_lm staging (alm2almtmp, sharp.c:481-545) and scatter (almtmp2alm,
// sharp.c:547-606).  Staged values carry c_l (recurrence normalisation),
// norm_l (spin > 0 / derivatives) and the real-harmonics m=0 factor.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void stage_alm_kernel(int lmax, int nalmptr, const long long *__restrict__ mvstart,
                                 long long astride, bool packed, long long alm_lo,
                                 const long long *__restrict__ moff,
                                 const double *__restrict__ cfac,
                                 const double *__restrict__ norm_l, bool use_norm, double norm_m0,
                                 const T *const *__restrict__ alm, double2 *__restrict__ A,
                                 int ncA) {
  const int m = blockIdx.x;
  const long long mo = moff[m] - m;
  const long long base = mvstart[m];
  const int nl = lmax - m + 1 + kPad;
  for (int e = threadIdx.x; e < nl * nalmptr; e += blockDim.x) {
    const int l = m + e / nalmptr;
    const int c = e % nalmptr;
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
    A[(mo + l) * ncA + c] = v;
  }
}

template <typename T>
__global__ void scatter_alm_kernel(int lmax, int nalmptr, const long long *__restrict__ mvstart,
                                   long long astride, bool packed, long long alm_lo,
                                   const long long *__restrict__ moff,
                                   const double *__restrict__ cfac,
                                   const double *__restrict__ norm_l, bool use_norm,
                                   double norm_m0, bool add, const double *__restrict__ Aout,
                                   int ncA, T *const *__restrict__ alm) {
  const int m = blockIdx.x;
  const long long mo = moff[m] - m;
  const long long base = mvstart[m];
  const int nl = lmax - m + 1;
  for (int e = threadIdx.x; e < nl * nalmptr; e += blockDim.x) {
    const int l = m + e / nalmptr;
    const int c = e % nalmptr;
    const double *src = Aout + ((mo + l) * ncA + c) * 2;
    double f = cfac[mo + l];
    if (use_norm) f *= norm_l[l];
    double vr = src[0] * f, vi = src[1] * f;
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
      T *px = packed ? a + (base + 2 * l * astride - alm_lo) : a + 2 * (base + l * astride - alm_lo);
      if (add) {
        px[0] += T(vr);
        px[1] += T(vi);
      } else {
        px[0] = T(vr);
        px[1] = T(vi);
      }
    }
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
  SHT_CUDA(cudaMallocAsync(&d_n, sizeof(int) * nt, st));
  SHT_CUDA(cudaMallocAsync(&d_off, sizeof(int) * nt, st));
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

static size_t fft_smem(const GeomPlan &gp) { return sizeof(double2) * 2 * (gp.nmax_complex + 2); }

void launch_phase2ring(const JobDesc &job, const GeomPlan &gp, long long map_lo,
                       const double2 *phase, int ncm, void *const *maps_dev, int nmapptr,
                       cudaStream_t st) {
  if (gp.npairs == 0) return;
  dim3 grid(gp.npairs, nmapptr);
  const size_t sm = fft_smem(gp);
  ProfScope ps("ring_synth", st);
  if (job.dp) {
    auto k = phase2ring_kernel<double>;
    SHT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    k<<<grid, 256, sm, st>>>(gp.mlim, gp.nph, gp.ofs, gp.stride, gp.phi0, gp.weight, gp.fft,
                             gp.fdesc, gp.twiddle, phase, ncm, gp.npairs, job.mmax, job.flags,
                             reinterpret_cast<double *const *>(maps_dev), map_lo);
  } else {
    auto k = phase2ring_kernel<float>;
    SHT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    k<<<grid, 256, sm, st>>>(gp.mlim, gp.nph, gp.ofs, gp.stride, gp.phi0, gp.weight, gp.fft,
                             gp.fdesc, gp.twiddle, phase, ncm, gp.npairs, job.mmax, job.flags,
                             reinterpret_cast<float *const *>(maps_dev), map_lo);
  }
  SHT_CUDA(cudaGetLastError());
}

void launch_ring2phase(const JobDesc &job, const GeomPlan &gp, long long map_lo,
                       const void *const *maps_dev, int nmapptr, double2 *phase, int ncm,
                       cudaStream_t st) {
  if (gp.npairs == 0) return;
  dim3 grid(gp.npairs, nmapptr);
  const size_t sm = fft_smem(gp);
  ProfScope ps("ring_anal", st);
  if (job.dp) {
    auto k = ring2phase_kernel<double>;
    SHT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    k<<<grid, 256, sm, st>>>(gp.mlim, gp.nph, gp.ofs, gp.stride, gp.phi0, gp.weight, gp.fft,
                             gp.fdesc, gp.twiddle, phase, ncm, gp.npairs, job.mmax, job.flags,
                             reinterpret_cast<const double *const *>(maps_dev), map_lo);
  } else {
    auto k = ring2phase_kernel<float>;
    SHT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    k<<<grid, 256, sm, st>>>(gp.mlim, gp.nph, gp.ofs, gp.stride, gp.phi0, gp.weight, gp.fft,
                             gp.fdesc, gp.twiddle, phase, ncm, gp.npairs, job.mmax, job.flags,
                             reinterpret_cast<const float *const *>(maps_dev), map_lo);
  }
  SHT_CUDA(cudaGetLastError());
}

void launch_phase2ring_direct(const JobDesc &job, const GeomPlan &gp, long long map_lo,
                              const double2 *phase, int ncm, void *const *maps_dev, int nmapptr,
                              cudaStream_t st) {
  if (gp.npairs == 0) return;
  dim3 grid(gp.npairs, nmapptr);
  ProfScope ps("ring_synth", st);
  if (job.dp)
    phase2ring_direct_kernel<double2><<<grid, 128, 0, st>>>(
        gp.mlim, gp.nph, gp.ofs, gp.stride, gp.weight, phase, ncm, gp.npairs, job.mmax,
        job.flags, reinterpret_cast<double2 *const *>(maps_dev), map_lo);
  else
    phase2ring_direct_kernel<float2><<<grid, 128, 0, st>>>(
        gp.mlim, gp.nph, gp.ofs, gp.stride, gp.weight, phase, ncm, gp.npairs, job.mmax,
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
        gp.mlim, gp.nph, gp.ofs, gp.stride, gp.weight, phase, ncm, gp.npairs, job.mmax,
        job.flags, reinterpret_cast<const double2 *const *>(maps_dev), map_lo);
  else
    ring2phase_direct_kernel<float2><<<grid, 128, 0, st>>>(
        gp.mlim, gp.nph, gp.ofs, gp.stride, gp.weight, phase, ncm, gp.npairs, job.mmax,
        job.flags, reinterpret_cast<const float2 *const *>(maps_dev), map_lo);
  SHT_CUDA(cudaGetLastError());
}

void launch_stage_alm(const JobDesc &job, const AlmPlan &ap, long long alm_lo,
                      const CoefPlan &cp, const double *norm_l, const void *const *alm_dev,
                      int nalmptr, double2 *A, int ncA, cudaStream_t st) {
  const bool use_norm = job.spin > 0 || job.type == SHARP_ALM2MAP_DERIV1;
  const double norm_m0 = (job.flags & SHARP_REAL_HARMONICS) ? kSqrtTwo : 1.0;
  const int blocks = job.mmax + 1;
  ProfScope ps("stage_alm", st);
  if (job.dp)
    stage_alm_kernel<double><<<blocks, 256, 0, st>>>(
        job.lmax, nalmptr, ap.mvstart, ap.stride, ap.packed, alm_lo, cp.d_moff, cp.cfac, norm_l,
        use_norm, norm_m0, reinterpret_cast<const double *const *>(alm_dev), A, ncA);
  else
    stage_alm_kernel<float><<<blocks, 256, 0, st>>>(
        job.lmax, nalmptr, ap.mvstart, ap.stride, ap.packed, alm_lo, cp.d_moff, cp.cfac, norm_l,
        use_norm, norm_m0, reinterpret_cast<const float *const *>(alm_dev), A, ncA);
  SHT_CUDA(cudaGetLastError());
}

void launch_scatter_alm(const JobDesc &job, const AlmPlan &ap, long long alm_lo,
                        const CoefPlan &cp, const double *norm_l, const double *Aout, int ncA,
                        void *const *alm_dev, int nalmptr, cudaStream_t st) {
  const bool use_norm = job.spin > 0 || job.type == SHARP_ALM2MAP_DERIV1;
  const double norm_m0 = (job.flags & SHARP_REAL_HARMONICS) ? kSqrtHalf : 1.0;
  const bool add = (job.flags & SHARP_ADD) != 0;
  const int blocks = job.mmax + 1;
  ProfScope ps("scatter_alm", st);
  if (job.dp)
    scatter_alm_kernel<double><<<blocks, 256, 0, st>>>(
        job.lmax, nalmptr, ap.mvstart, ap.stride, ap.packed, alm_lo, cp.d_moff, cp.cfac, norm_l,
        use_norm, norm_m0, add, Aout, ncA, reinterpret_cast<double *const *>(alm_dev));
  else
    scatter_alm_kernel<float><<<blocks, 256, 0, st>>>(
        job.lmax, nalmptr, ap.mvstart, ap.stride, ap.packed, alm_lo, cp.d_moff, cp.cfac, norm_l,
        use_norm, norm_m0, add, Aout, ncA, reinterpret_cast<float *const *>(alm_dev));
  SHT_CUDA(cudaGetLastError());
}

}  // namespace sht
