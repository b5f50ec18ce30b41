// Host-side part of the C ABI: a_lm layouts, map geometries and error state.
//
// Geometry construction keeps the reference's observable behaviour (callers
// read geom_info->pair[] directly): rings sorted by sin(theta), north/south
// partners paired, pairs sorted by (nph, phi0, cth descending)
// (libsharp/sharp.c:122-135, 179-227).  Quadrature nodes and weights are the
// published rules the reference uses (Gauss-Legendre by Newton iteration;
// Fejer/Clenshaw-Curtis weights from Waldvogel 2006), computed here with our
// own code.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "sht_internal.h"
#include "sharp_almhelpers.h"
#include "sharp_geomhelpers.h"

namespace sht {

namespace {
thread_local std::string g_last_error;
int g_abort_mode = -1;  // -1: read the environment on first use
std::mutex g_err_mutex;
}  // namespace

bool abort_on_error() {
  std::lock_guard<std::mutex> lk(g_err_mutex);
  if (g_abort_mode < 0) {
    const char *e = std::getenv("SHARP_B200_ABORT_ON_ERROR");
    g_abort_mode = (e && e[0] == '0') ? 0 : 1;
  }
  return g_abort_mode == 1;
}

void record_error(const std::string &msg) { g_last_error = msg; }

void fail(const char *file, int line, const std::string &msg) {
  record_error(msg);
  if (abort_on_error()) {
    std::fprintf(stderr, "%s, %i:\n%s\n", file, line, msg.c_str());
    std::exit(1);
  }
  throw Failure{msg};
}

int get_mlim(int lmax, int spin, double sth, double cth) {
  // Largest m with non-negligible Y_lm on this ring (libsharp/sharp.c:66-78).
  double ofs = lmax * 0.01;
  if (ofs < 100.) ofs = 100.;
  double b = -2 * spin * std::fabs(cth);
  double t1 = lmax * sth + ofs;
  double c = double(spin) * spin - t1 * t1;
  double discr = b * b - 4 * c;
  if (discr <= 0) return lmax;
  double res = (-b + std::sqrt(discr)) / 2.;
  if (res > lmax) res = lmax;
  return int(res + 0.5);
}

}  // namespace sht

using sht::fail;

extern "C" {

const char *sharp_b200_last_error(void) { return sht::g_last_error.c_str(); }
void sharp_b200_clear_error(void) { sht::g_last_error.clear(); }
void sharp_b200_set_abort_on_error(int on) {
  std::lock_guard<std::mutex> lk(sht::g_err_mutex);
  sht::g_abort_mode = on ? 1 : 0;
}

// ---------------------------------------------------------------------------
// a_lm layouts
// ---------------------------------------------------------------------------
void sharp_make_general_alm_info(int lmax, int nm, int stride, const int *mval,
                                 const ptrdiff_t *mvstart, int flags,
                                 sharp_alm_info **alm_info) {
  auto *info = static_cast<sharp_alm_info *>(std::malloc(sizeof(sharp_alm_info)));
  info->lmax = lmax;
  info->nm = nm;
  info->mval = static_cast<int *>(std::malloc(sizeof(int) * std::max(nm, 1)));
  info->mvstart = static_cast<ptrdiff_t *>(std::malloc(sizeof(ptrdiff_t) * std::max(nm, 1)));
  info->stride = stride;
  info->flags = flags;
  for (int i = 0; i < nm; ++i) {
    info->mval[i] = mval[i];
    info->mvstart[i] = mvstart[i];
  }
  *alm_info = info;
}

void sharp_make_alm_info(int lmax, int mmax, int stride, const ptrdiff_t *mstart,
                         sharp_alm_info **alm_info) {
  std::vector<int> mval(mmax + 1);
  for (int i = 0; i <= mmax; ++i) mval[i] = i;
  sharp_make_general_alm_info(lmax, mmax + 1, stride, mval.data(), mstart, 0, alm_info);
}

ptrdiff_t sharp_alm_index(const sharp_alm_info *self, int l, int mi) {
  if (self->flags & SHARP_PACKED) {
    try {
      fail(__FILE__, __LINE__, "sharp_alm_index not applicable with SHARP_PACKED alms");
    } catch (const sht::Failure &) {
      return -1;
    }
  }
  return self->mvstart[mi] + self->stride * l;
}

void sharp_destroy_alm_info(sharp_alm_info *info) {
  if (!info) return;
  std::free(info->mval);
  std::free(info->mvstart);
  std::free(info);
}

void sharp_make_triangular_alm_info(int lmax, int mmax, int stride,
                                    sharp_alm_info **alm_info) {
  std::vector<int> mval(mmax + 1);
  std::vector<ptrdiff_t> start(mmax + 1);
  const ptrdiff_t tval = 2 * ptrdiff_t(lmax) + 1;
  for (ptrdiff_t m = 0; m <= mmax; ++m) {
    mval[m] = int(m);
    start[m] = stride * ((m * (tval - m)) >> 1);
  }
  sharp_make_general_alm_info(lmax, mmax + 1, stride, mval.data(), start.data(), 0, alm_info);
}

void sharp_make_rectangular_alm_info(int lmax, int mmax, int stride,
                                     sharp_alm_info **alm_info) {
  std::vector<int> mval(mmax + 1);
  std::vector<ptrdiff_t> start(mmax + 1);
  for (ptrdiff_t m = 0; m <= mmax; ++m) {
    mval[m] = int(m);
    start[m] = stride * m * (lmax + 1);
  }
  sharp_make_general_alm_info(lmax, mmax + 1, stride, mval.data(), start.data(), 0, alm_info);
}

// ---------------------------------------------------------------------------
// Geometry
// ---------------------------------------------------------------------------
static int cmp_ring_sth(const void *xa, const void *xb) {
  const auto *a = static_cast<const sharp_ringinfo *>(xa);
  const auto *b = static_cast<const sharp_ringinfo *>(xb);
  return (a->sth < b->sth) ? -1 : (a->sth > b->sth) ? 1 : 0;
}

static int cmp_pair(const void *xa, const void *xb) {
  const auto *a = static_cast<const sharp_ringpair *>(xa);
  const auto *b = static_cast<const sharp_ringpair *>(xb);
  if (a->r1.nph != b->r1.nph) return (a->r1.nph < b->r1.nph) ? -1 : 1;
  if (a->r1.phi0 != b->r1.phi0) return (a->r1.phi0 < b->r1.phi0) ? -1 : 1;
  return (a->r1.cth > b->r1.cth) ? -1 : 1;
}

static bool rel_close(double a, double b, double eps) {
  return std::fabs(a - b) < eps * std::fabs(b);
}

void sharp_make_geom_info(int nrings, const int *nph, const ptrdiff_t *ofs,
                          const int *stride, const double *phi0, const double *theta,
                          const double *wgt, sharp_geom_info **geom_info) {
  auto *info = static_cast<sharp_geom_info *>(std::malloc(sizeof(sharp_geom_info)));
  std::vector<sharp_ringinfo> rings(nrings);
  info->pair = static_cast<sharp_ringpair *>(
      std::malloc(sizeof(sharp_ringpair) * std::max(nrings, 1)));
  info->npairs = 0;
  info->nphmax = 0;
  for (int i = 0; i < nrings; ++i) {
    sharp_ringinfo &r = rings[i];
    r.theta = theta[i];
    r.cth = std::cos(theta[i]);
    r.sth = std::sin(theta[i]);
    r.weight = wgt ? wgt[i] : 1.;
    r.phi0 = phi0[i];
    r.ofs = ofs[i];
    r.stride = stride[i];
    r.nph = nph[i];
    info->nphmax = std::max(info->nphmax, nph[i]);
  }
  if (nrings > 0) std::qsort(rings.data(), nrings, sizeof(sharp_ringinfo), cmp_ring_sth);
  int pos = 0;
  while (pos < nrings) {
    sharp_ringpair &p = info->pair[info->npairs];
    std::memset(&p, 0, sizeof(p));
    p.r1 = rings[pos];
    if (pos < nrings - 1 && rel_close(rings[pos].cth, -rings[pos + 1].cth, 1e-12)) {
      if (rings[pos].cth > 0) {
        p.r2 = rings[pos + 1];
      } else {
        p.r1 = rings[pos + 1];
        p.r2 = rings[pos];
      }
      ++pos;
    } else {
      p.r2.nph = -1;
    }
    ++pos;
    ++info->npairs;
  }
  if (info->npairs > 0)
    std::qsort(info->pair, info->npairs, sizeof(sharp_ringpair), cmp_pair);
  *geom_info = info;
}

void sharp_b200_forget_geometry(const sharp_geom_info *info);  // device cache hook

// Copies the ring pairs pairs[0..npairs) of g (indices into g->pair, in the
// given order) into a new geometry; the ring structs are copied as they are,
// so theta, cos/sin(theta), weights and offsets stay bit-identical.
int sharp_b200_make_subset_geom_info(const sharp_geom_info *g, const int *pairs, int npairs,
                                     sharp_geom_info **geom_info) {
  if (!g || !geom_info || npairs < 0 || (npairs > 0 && !pairs)) {
    sht::record_error("sharp_b200_make_subset_geom_info: bad argument");
    return -1;
  }
  for (int i = 0; i < npairs; ++i)
    if (pairs[i] < 0 || pairs[i] >= g->npairs) {
      sht::record_error("sharp_b200_make_subset_geom_info: pair index out of range");
      return -1;
    }
  auto *info = static_cast<sharp_geom_info *>(std::malloc(sizeof(sharp_geom_info)));
  info->pair = static_cast<sharp_ringpair *>(
      std::malloc(sizeof(sharp_ringpair) * std::max(npairs, 1)));
  info->npairs = npairs;
  info->nphmax = 0;
  for (int i = 0; i < npairs; ++i) {
    info->pair[i] = g->pair[pairs[i]];
    info->nphmax = std::max(info->nphmax, std::max(info->pair[i].r1.nph, info->pair[i].r2.nph));
  }
  *geom_info = info;
  return 0;
}

void sharp_destroy_geom_info(sharp_geom_info *info) {
  if (!info) return;
  sharp_b200_forget_geometry(info);
  std::free(info->pair);
  std::free(info);
}

void sharp_make_weighted_healpix_geom_info(int nside, int stride, const double *weight,
                                           sharp_geom_info **geom_info) {
  const double pi = 3.141592653589793238462643383279502884197;
  const ptrdiff_t npix = ptrdiff_t(nside) * nside * 12;
  const ptrdiff_t ncap = 2 * ptrdiff_t(nside) * (nside - 1);
  const int nrings = 4 * nside - 1;
  std::vector<double> theta(nrings), wgt(nrings), phi0(nrings);
  std::vector<int> nph(nrings), strides(nrings, stride);
  std::vector<ptrdiff_t> ofs(nrings);
  for (int i = 0; i < nrings; ++i) {
    const int ring = i + 1;
    const ptrdiff_t northring = (ring > 2 * nside) ? 4 * nside - ring : ring;
    if (northring < nside) {
      theta[i] = 2 * std::asin(northring / (std::sqrt(6.) * nside));
      nph[i] = int(4 * northring);
      phi0[i] = pi / nph[i];
      ofs[i] = 2 * northring * (northring - 1) * stride;
    } else {
      const double fact1 = (8. * nside) / npix;
      const double costheta = (2 * nside - northring) * fact1;
      theta[i] = std::acos(costheta);
      nph[i] = 4 * nside;
      phi0[i] = ((northring - nside) & 1) ? 0. : pi / nph[i];
      ofs[i] = (ncap + (northring - nside) * nph[i]) * stride;
    }
    if (northring != ring) {  // southern hemisphere
      theta[i] = pi - theta[i];
      ofs[i] = (npix - nph[i]) * stride - ofs[i];
    }
    wgt[i] = 4. * pi / npix * (weight ? weight[northring - 1] : 1.);
  }
  sharp_make_geom_info(nrings, nph.data(), ofs.data(), strides.data(), phi0.data(),
                       theta.data(), wgt.data(), geom_info);
}

// Gauss-Legendre nodes (ascending) and weights on [-1,1] by Newton iteration
// on the three-term Legendre recurrence, started from the asymptotic guess
// cos(pi(4i-1)/(4n+2)) (Tricomi).  Same published method as the reference
// (libsharp/sharp_geomhelpers.c:105-156).
static void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w) {
  const double pi = 3.141592653589793238462643383279502884197;
  x.assign(n, 0.);
  w.assign(n, 0.);
  const int half = (n + 1) >> 1;
  const double t0 = 1 - (1 - 1. / n) / (8. * n * n);
  const double t1 = 1. / (4. * n + 2.);
  for (int i = 1; i <= half; ++i) {
    double x0 = std::cos(pi * ((i << 2) - 1) * t1) * t0;
    double dpdx = 0;
    bool last = false;
    for (int it = 0; it < 100; ++it) {
      double pm1 = 1.0, p = x0;
      for (int k = 2; k <= n; ++k) {
        const double pm2 = pm1;
        pm1 = p;
        p = x0 * pm1 + (k - 1.) / k * (x0 * pm1 - pm2);
      }
      const double omx2 = (std::fabs(x0) > 0.1) ? (1. + x0) * (1. - x0) : 1. - x0 * x0;
      dpdx = (pm1 - x0 * p) * n / omx2;
      const double dx = p / dpdx;
      x0 -= dx;
      if (last) break;
      if (std::fabs(dx) <= 3e-14) last = true;
    }
    const double omx2 = (std::fabs(x0) > 0.1) ? (1. + x0) * (1. - x0) : 1. - x0 * x0;
    x[i - 1] = -x0;
    x[n - i] = x0;
    w[i - 1] = w[n - i] = 2. / (omx2 * dpdx * dpdx);
  }
}

void sharp_make_gauss_geom_info(int nrings, int nphi, double phi0, int stride_lon,
                                int stride_lat, sharp_geom_info **geom_info) {
  const double pi = 3.141592653589793238462643383279502884197;
  std::vector<double> x, w;
  gauss_legendre(nrings, x, w);
  std::vector<double> theta(nrings), phis(nrings, phi0);
  std::vector<int> nph(nrings, nphi), strides(nrings, stride_lon);
  std::vector<ptrdiff_t> ofs(nrings);
  for (int i = 0; i < nrings; ++i) {
    theta[i] = std::acos(-x[i]);
    ofs[i] = ptrdiff_t(i) * stride_lat;
    w[i] *= 2 * pi / nphi;
  }
  sharp_make_geom_info(nrings, nph.data(), ofs.data(), strides.data(), phis.data(),
                       theta.data(), w.data(), geom_info);
}

// FFTPACK-convention backward real transform of a half-complex sequence
// [r0, r1, i1, r2, i2, ...] of length n, evaluated directly (O(n^2)) with an
// exact angle reduction; only used to build quadrature weights.
static void halfcomplex_backward(std::vector<double> &d) {
  const int n = int(d.size());
  if (n == 0) return;
  const double pi = 3.141592653589793238462643383279502884197;
  std::vector<double> c(n), s(n), out(n);
  for (int k = 0; k < n; ++k) {
    c[k] = std::cos(2 * pi * k / n);
    s[k] = std::sin(2 * pi * k / n);
  }
  for (int j = 0; j < n; ++j) {
    long double acc = d[0];
    for (int k = 1; 2 * k < n; ++k) {
      const long idx = (long(j) * k) % n;
      acc += 2.0L * ((long double)d[2 * k - 1] * c[idx] - (long double)d[2 * k] * s[idx]);
    }
    if ((n & 1) == 0) acc += (long double)d[n - 1] * ((j & 1) ? -1.0L : 1.0L);
    out[j] = double(acc);
  }
  d = out;
}

static void equidistant_geom(int nrings, int ppring, double phi0, int stride_lon,
                             int stride_lat, const std::vector<double> &theta,
                             const double *wgt, sharp_geom_info **geom_info) {
  std::vector<double> phis(nrings, phi0);
  std::vector<int> nph(nrings, ppring), strides(nrings, stride_lon);
  std::vector<ptrdiff_t> ofs(nrings);
  for (int i = 0; i < nrings; ++i) ofs[i] = ptrdiff_t(i) * stride_lat;
  sharp_make_geom_info(nrings, nph.data(), ofs.data(), strides.data(), phis.data(),
                       theta.data(), wgt, geom_info);
}

// Fejer-1 weights (Waldvogel 2006, BIT 46:195).
void sharp_make_fejer1_geom_info(int nrings, int ppring, double phi0, int stride_lon,
                                 int stride_lat, sharp_geom_info **geom_info) {
  const double pi = 3.141592653589793238462643383279502884197;
  std::vector<double> w(nrings, 0.), theta(nrings);
  w[0] = 2.;
  for (int k = 1; k <= (nrings - 1) / 2; ++k) {
    w[2 * k - 1] = 2. / (1. - 4. * k * k) * std::cos((k * pi) / nrings);
    w[2 * k] = 2. / (1. - 4. * k * k) * std::sin((k * pi) / nrings);
  }
  if ((nrings & 1) == 0) w[nrings - 1] = 0.;
  halfcomplex_backward(w);
  for (int m = 0; m < (nrings + 1) / 2; ++m) {
    theta[m] = pi * (m + 0.5) / nrings;
    theta[nrings - 1 - m] = pi - theta[m];
    w[m] = w[nrings - 1 - m] = w[m] * 2 * pi / (nrings * double(ppring));
  }
  equidistant_geom(nrings, ppring, phi0, stride_lon, stride_lat, theta, w.data(), geom_info);
}

// Clenshaw-Curtis weights (Waldvogel 2006).
void sharp_make_cc_geom_info(int nrings, int ppring, double phi0, int stride_lon,
                             int stride_lat, sharp_geom_info **geom_info) {
  const double pi = 3.141592653589793238462643383279502884197;
  const int n = nrings - 1;
  std::vector<double> w(nrings, 0.), theta(nrings);
  const double dw = -1. / (n * n - 1. + (n & 1));
  std::vector<double> v(n, 0.);
  v[0] = 2. + dw;
  for (int k = 1; k <= (n / 2 - 1); ++k) v[2 * k - 1] = 2. / (1. - 4. * k * k) + dw;
  v[2 * (n / 2) - 1] = (n - 3.) / (2 * (n / 2) - 1) - 1. - dw * ((2 - (n & 1)) * n - 1);
  halfcomplex_backward(v);
  for (int i = 0; i < n; ++i) w[i] = v[i];
  w[n] = w[0];
  for (int m = 0; m < (nrings + 1) / 2; ++m) {
    theta[m] = pi * m / (nrings - 1.);
    if (theta[m] < 1e-15) theta[m] = 1e-15;
    theta[nrings - 1 - m] = pi - theta[m];
    w[m] = w[nrings - 1 - m] = w[m] * 2 * pi / (n * double(ppring));
  }
  equidistant_geom(nrings, ppring, phi0, stride_lon, stride_lat, theta, w.data(), geom_info);
}

// Fejer-2 weights (Waldvogel 2006).
void sharp_make_fejer2_geom_info(int nrings, int ppring, double phi0, int stride_lon,
                                 int stride_lat, sharp_geom_info **geom_info) {
  const double pi = 3.141592653589793238462643383279502884197;
  const int n = nrings + 1;
  std::vector<double> v(n, 0.), w(nrings), theta(nrings);
  v[0] = 2.;
  for (int k = 1; k <= (n / 2 - 1); ++k) v[2 * k - 1] = 2. / (1. - 4. * k * k);
  v[2 * (n / 2) - 1] = (n - 3.) / (2 * (n / 2) - 1) - 1.;
  halfcomplex_backward(v);
  for (int m = 0; m < nrings; ++m) w[m] = v[m + 1];
  for (int m = 0; m < (nrings + 1) / 2; ++m) {
    theta[m] = pi * (m + 1) / (nrings + 1.);
    theta[nrings - 1 - m] = pi - theta[m];
    w[m] = w[nrings - 1 - m] = w[m] * 2 * pi / (n * double(ppring));
  }
  equidistant_geom(nrings, ppring, phi0, stride_lon, stride_lat, theta, w.data(), geom_info);
}

void sharp_make_mw_geom_info(int nrings, int ppring, double phi0, int stride_lon,
                             int stride_lat, sharp_geom_info **geom_info) {
  const double pi = 3.141592653589793238462643383279502884197;
  std::vector<double> theta(nrings);
  for (int m = 0; m < nrings; ++m) {
    theta[m] = pi * (2. * m + 1.) / (2. * nrings - 1.);
    if (theta[m] > pi - 1e-15) theta[m] = pi - 1e-15;
  }
  equidistant_geom(nrings, ppring, phi0, stride_lon, stride_lat, theta, nullptr, geom_info);
}

static int g_chunksize_min = 500, g_nchunks_max = 10;
void sharp_set_chunksize_min(int v) { g_chunksize_min = v; }
void sharp_set_nchunks_max(int v) { g_nchunks_max = v; }

// ---------------------------------------------------------------------------
// Helpers the reference exports beside the job interface (its test suite and
// tools call them): the m cut-off of a ring, the vector-length hint and its
// autotuner, and the start-up banner.
// ---------------------------------------------------------------------------
int sharp_get_mlim(int lmax, int spin, double sth, double cth) {
  return sht::get_mlim(lmax, spin, sth, cth);
}

// The low flag bits of a job select the reference's SIMD vector count (1..6);
// this engine has one kernel variant per job shape, so every hint is the same
// and the autotuner answers 1 without running anything.
int sharp_get_nv_max(void) { return 1; }
int sharp_nv_oracle(sharp_jobtype type, int spin, int ntrans) {
  if (type == SHARP_ALM2MAP_DERIV1) spin = 1;
  if (!(int(type) >= 0 && int(type) < 5)) fail(__FILE__, __LINE__, "bad type");
  if (ntrans <= 0) fail(__FILE__, __LINE__, "bad number of simultaneous transforms");
  if (spin < 0) fail(__FILE__, __LINE__, "bad spin");
  return 1;
}

void sharp_announce(const char *name) {
  const size_t n = std::strlen(name);
  std::printf("\n+-");
  for (size_t i = 0; i < n; ++i) std::printf("-");
  std::printf("-+\n| %s |\n+-", name);
  for (size_t i = 0; i < n; ++i) std::printf("-");
  std::printf("-+\n\n");
  std::printf("Spherical-harmonic transforms: libsharp_b200 (CUDA, sm_100a)\n\n");
}

void sharp_module_startup(const char *name, int argc, int argc_expected,
                          const char *argv_expected, int verbose) {
  if (verbose) sharp_announce(name);
  if (argc == argc_expected) return;
  if (verbose) std::fprintf(stderr, "Usage: %s %s\n", name, argv_expected);
  std::exit(1);
}

}  // extern "C"
