// Job driver of the C ABI: validation with the reference's error semantics,
// cached device plans (geometry, recurrence coefficients, a_lm layout), host
// staging and the per-job kernel sequence.
//
// Reference driver: libsharp/sharp.c:762-880 (sharp_execute_job,
// sharp_build_job_common, sharp_execute).  The reference splits ring pairs
// into chunks and loops over m with OpenMP; here a whole job stays resident
// in HBM and runs as: stage a_lm -> Legendre synthesis -> ring FFT (alm2map),
// or ring FFT -> Legendre analysis -> scatter a_lm (map2alm).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <cstdio>
#include <functional>
#include <tuple>
#include <map>
#include <set>
#include <memory>
#include <mutex>
#include <numeric>
#include <vector>

#include "sht_device.h"

namespace sht {

void check_cuda(cudaError_t e, const char *what, const char *file, int line) {
  if (e == cudaSuccess) return;
  fail(file, line, std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

namespace {

// flags whose jobs update the output arrays instead of overwriting them
constexpr int kAccumulate = SHARP_ADD | SHARP_SUBTRACT;

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------
uint64_t fnv1a(const void *data, size_t n, uint64_t h = 1469598103934665603ull) {
  const auto *p = static_cast<const unsigned char *>(data);
  for (size_t i = 0; i < n; ++i) {
    h ^= p[i];
    h *= 1099511628211ull;
  }
  return h;
}

template <typename T>
T *dev_upload(const std::vector<T> &v, cudaStream_t st) {
  T *d = nullptr;
  const size_t bytes = sizeof(T) * std::max<size_t>(v.size(), 1);
  SHT_CUDA(cudaMalloc(&d, bytes));
  if (!v.empty())
    SHT_CUDA(cudaMemcpyAsync(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st));
  return d;
}

template <typename T>
void dev_free(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}

std::vector<int> factor_fft(int N) {
  std::vector<int> r;
  int n = N;
  while (n % 8 == 0) { r.push_back(8); n /= 8; }
  while (n % 4 == 0) { r.push_back(4); n /= 4; }
  while (n % 2 == 0) { r.push_back(2); n /= 2; }
  for (int p = 3; n > 1; p += 2)
    while (n % p == 0) { r.push_back(p); n /= p; }
  return r;
}

uint64_t hash_geom(const sharp_geom_info *g) {
  uint64_t h = fnv1a(&g->npairs, sizeof(int));
  h = fnv1a(&g->nphmax, sizeof(int), h);
  if (g->npairs > 0) h = fnv1a(g->pair, sizeof(sharp_ringpair) * g->npairs, h);
  return h;
}

uint64_t hash_alm(const sharp_alm_info *a) {
  uint64_t h = fnv1a(&a->lmax, sizeof(int));
  h = fnv1a(&a->nm, sizeof(int), h);
  h = fnv1a(&a->flags, sizeof(int), h);
  h = fnv1a(&a->stride, sizeof(ptrdiff_t), h);
  if (a->nm > 0) {
    h = fnv1a(a->mval, sizeof(int) * a->nm, h);
    h = fnv1a(a->mvstart, sizeof(ptrdiff_t) * a->nm, h);
  }
  return h;
}

std::mutex g_cache_mutex;
std::map<const void *, std::vector<std::unique_ptr<GeomPlan>>> g_geom_cache;
std::vector<std::unique_ptr<CoefPlan>> g_coef_cache;
std::map<const void *, std::unique_ptr<AlmPlan>> g_alm_cache;

}  // namespace

// workspace pools, one per device, created on first use
static std::mutex g_pool_mutex;
static std::vector<cudaMemPool_t> g_pools;

cudaError_t ws_alloc_bytes(void **p, size_t bytes, cudaStream_t st) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  cudaMemPool_t pool = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_pool_mutex);
    if (int(g_pools.size()) <= dev) g_pools.resize(dev + 1, nullptr);
    if (!g_pools[dev]) {
      cudaMemPoolProps props = {};
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      cudaMemPool_t created = nullptr;
      e = cudaMemPoolCreate(&created, &props);
      if (e != cudaSuccess) return e;
      uint64_t keep = UINT64_MAX;
      e = cudaMemPoolSetAttribute(created, cudaMemPoolAttrReleaseThreshold, &keep);
      if (e != cudaSuccess) {
        cudaMemPoolDestroy(created);
        return e;
      }
      g_pools[dev] = created;
    }
    pool = g_pools[dev];
  }
  return cudaMallocFromPoolAsync(p, bytes, pool, st);
}

void ws_trim() {
  std::lock_guard<std::mutex> lk(g_pool_mutex);
  for (cudaMemPool_t pool : g_pools)
    if (pool) cudaMemPoolTrimTo(pool, 0);
}

bool ws_bytes(unsigned long long *reserved, unsigned long long *used) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  std::lock_guard<std::mutex> lk(g_pool_mutex);
  if (int(g_pools.size()) <= dev || !g_pools[dev]) return false;
  uint64_t r = 0, u = 0;
  if (cudaMemPoolGetAttribute(g_pools[dev], cudaMemPoolAttrReservedMemCurrent, &r) != cudaSuccess ||
      cudaMemPoolGetAttribute(g_pools[dev], cudaMemPoolAttrUsedMemCurrent, &u) != cudaSuccess)
    return false;
  if (reserved) *reserved = r;
  if (used) *used = u;
  return true;
}

// ---------------------------------------------------------------------------
// Host half of a geometry plan (no device calls): pairs in decreasing mlim
// order, the per-m counts and work lists, per-ring tables, one FFT
// descriptor per distinct ring length (radices, Bluestein choice, twiddle and
// chirp offsets) and the FFT size classes.  The cached plans and the
// allocation-free synthesis both build on it.
// ---------------------------------------------------------------------------
GeomHost build_geom_host(const sharp_geom_info *g, int lmax, int mmax, int spin) {
  GeomHost h;
  const int np = g->npairs;
  h.npairs = np;
  h.nphmax = g->nphmax;
  std::vector<int> mlim(np);
  for (int i = 0; i < np; ++i) mlim[i] = get_mlim(lmax, spin, g->pair[i].r1.sth, g->pair[i].r1.cth);
  h.order.resize(np);
  std::iota(h.order.begin(), h.order.end(), 0);
  std::stable_sort(h.order.begin(), h.order.end(),
                   [&](int a, int b) { return mlim[a] > mlim[b]; });
  // count_m[m] = number of pairs with mlim >= m (a prefix of the sorted order)
  std::vector<int> hist(mmax + 1, 0);
  for (int i = 0; i < np; ++i)
    if (mlim[i] >= 0) hist[std::min(mlim[i], mmax)] += 1;
  h.count_m.assign(mmax + 1, 0);
  int run = 0;
  for (int m = mmax; m >= 0; --m) {
    run += hist[m];
    h.count_m[m] = run;
  }
  for (int m = 0; m <= mmax; ++m)
    for (int t = 0; t * h.synth_tile < h.count_m[m]; ++t) h.synth_items.push_back({m, t});
  for (int m = 0; m <= mmax; ++m)
    for (int t = 0; t * 256 < h.count_m[m]; ++t) h.mixed_items.push_back({m, t});

  h.cth.resize(np);
  h.sth.resize(np);
  h.mlim_sorted.resize(np);
  h.phi0.resize(2 * np);
  h.weight.resize(2 * np);
  h.nph.resize(2 * np);
  h.stride.resize(2 * np);
  h.fft.assign(2 * np, 0);
  h.ofs.resize(2 * np);
  std::map<int, int> len_index;
  long long lo = 0, hi = 0;
  bool first = true, unit_stride = true;
  std::vector<std::pair<long long, long long>> spans;
  for (int p = 0; p < np; ++p) {
    const sharp_ringpair &pr = g->pair[h.order[p]];
    h.cth[p] = pr.r1.cth;
    h.sth[p] = pr.r1.sth;
    h.mlim_sorted[p] = mlim[h.order[p]];
    for (int hh = 0; hh < 2; ++hh) {
      const sharp_ringinfo &r = hh ? pr.r2 : pr.r1;
      const int i = 2 * p + hh;
      const bool present = (hh == 0) || r.nph > 0;
      h.nph[i] = present ? r.nph : -1;
      h.phi0[i] = present ? r.phi0 : 0.0;
      h.weight[i] = present ? r.weight : 0.0;
      h.ofs[i] = present ? r.ofs : 0;
      h.stride[i] = present ? r.stride : 1;
      if (!present || r.nph <= 0) continue;
      auto it = len_index.find(r.nph);
      if (it == len_index.end()) {
        FftDesc d{};
        d.n = r.nph;
        d.N = (r.nph & 1) ? r.nph : r.nph / 2;
        d.tw = int(h.tw_total);
        auto rad = factor_fft(d.N);
        SHT_REQUIRE(int(rad.size()) <= kMaxRadices, "ring length has too many factors");
        d.nrad = int(rad.size());
        for (int k = 0; k < d.nrad; ++k) d.rad[k] = rad[k];
        // Stockham cost ~ N * sum(generic radices); Bluestein ~ M log2 M + 2N
        // (power-of-two convolution of length M >= 2N-1)
        long long direct = 0;
        for (int rr : rad) direct += (rr > 5 && rr != 8) ? rr : 1;
        direct *= d.N;
        int M = 1, lg = 0;
        while (M < 2 * d.N - 1) { M <<= 1; ++lg; }
        const long long blue_cost = 2ll * ((long long)M * lg + 2ll * d.N);
        d.blue = (d.N > 16 && blue_cost < direct) ? 1 : 0;
        d.M = M;   // the convolution length, also for rings the register Bluestein takes
        d.bhat = d.bhat2 = d.chirp = -1;
        h.tw_n.push_back(d.n);
        h.tw_off.push_back(int(h.tw_total));
        h.tw_total += d.n;
        it = len_index.emplace(r.nph, int(h.descs.size())).first;
        h.descs.push_back(d);
        h.nmax_complex = std::max(h.nmax_complex, d.N);
      }
      h.fft[i] = it->second;
      const long long a = r.ofs, b = r.ofs + (long long)(r.nph - 1) * r.stride;
      const long long rlo = std::min(a, b), rhi = std::max(a, b) + 1;
      if (first) { lo = rlo; hi = rhi; first = false; }
      lo = std::min(lo, rlo);
      hi = std::max(hi, rhi);
      if (r.stride != 1) unit_stride = false;
      spans.push_back({rlo, rhi});
    }
  }
  SHT_REQUIRE(h.tw_total < (1ll << 31), "geometry too large (twiddle table)");
  // rings tile [lo,hi) exactly -> synthesis need not pre-load the map
  bool covered = unit_stride && !spans.empty();
  if (covered) {
    std::sort(spans.begin(), spans.end());
    long long cur = lo;
    for (auto &sp : spans) {
      if (sp.first != cur) { covered = false; break; }
      cur = sp.second;
    }
    covered = covered && cur == hi;
  }
  h.map_lo = lo;
  h.map_hi = hi;
  h.map_covered = covered;
  // pairs whose present rings all take the power-of-two register FFT with
  // the same length run there; the rest go to the size classes
  // (the same for the register Bluestein kernels, keyed by the convolution
  // length); a length whose buffer and phi0 slices exceed the shared memory
  // of a CTA stays in the size classes
  std::map<int, std::vector<int>> pw_lists, pb_lists;
  std::vector<char> is_pw(np, 0);   // 1: power-of-two pair, 2: register Bluestein pair
  auto fits = [&](int len) {
    return sizeof(double2) * pow2_ring_smem_entries(len, mmax) <= kRingSmemLimit;
  };
  for (int p = 0; p < np; ++p) {
    const int mm = std::min(mmax, h.mlim_sorted[p]);
    int N = -1, M = -1;
    for (int hh = 0; hh < 2; ++hh) {
      const int i = 2 * p + hh;
      if (h.nph[i] <= 0) continue;
      const int n = pow2_ring_length(h.nph[i], h.stride[i], mm);
      N = (N < 0 || N == n) ? n : 0;
      const int b = blue_ring_length(h.nph[i], h.descs[h.fft[i]]);
      M = (M < 0 || M == b) ? b : 0;
    }
    if (N > 0 && fits(N)) {
      pw_lists[N].push_back(p);
      is_pw[p] = 1;
    } else if (M > 0 && fits(M)) {
      pb_lists[M].push_back(p);
      is_pw[p] = 2;
    }
  }
  for (auto &kv : pw_lists) {
    h.pw_N.push_back(kv.first);
    h.pw_start.push_back(int(h.pw_pairs.size()));
    h.pw_count.push_back(int(kv.second.size()));
    h.pw_pairs.insert(h.pw_pairs.end(), kv.second.begin(), kv.second.end());
  }
  for (auto &kv : pb_lists) {
    h.pb_M.push_back(kv.first);
    h.pb_start.push_back(int(h.pb_pairs.size()));
    h.pb_count.push_back(int(kv.second.size()));
    h.pb_pairs.insert(h.pb_pairs.end(), kv.second.begin(), kv.second.end());
  }
  // FFT size classes (the last class is capped by shared memory)
  const int bounds[4] = {256, 1024, 4096, h.nmax_complex};
  std::vector<std::vector<int>> lists(4);
  for (int p = 0; p < np; ++p) {
    if (is_pw[p]) continue;
    int nmx = 0;
    for (int hh = 0; hh < 2; ++hh)
      if (h.nph[2 * p + hh] > 0) nmx = std::max(nmx, h.descs[h.fft[2 * p + hh]].N);
    int c = 0;
    while (c < 3 && nmx > bounds[c]) ++c;
    lists[c].push_back(p);
  }
  for (int c = 0; c < 4; ++c) {
    // shared memory: buffer A holds N+2 (Stockham) or M (Bluestein)
    // entries, buffer B N+2
    int bufA = 2, bufB = 2;
    for (int p : lists[c])
      for (int hh = 0; hh < 2; ++hh)
        if (h.nph[2 * p + hh] > 0) {
          const FftDesc &d = h.descs[h.fft[2 * p + hh]];
          bufA = std::max(bufA, d.blue ? std::max(d.M, d.N + 2) : d.N + 2);
          bufB = std::max(bufB, d.N + 2);
        }
    // whole blocks of 8 entries: the ring kernels swizzle indices inside them
    bufA = (bufA + 7) & ~7;
    bufB = (bufB + 7) & ~7;
    h.cls_N.push_back(std::max(bounds[c], 1));
    h.cls_bufA.push_back(bufA);
    h.cls_bufB.push_back(bufB);
    h.cls_start.push_back(int(h.cls_pairs.size()));
    h.cls_count.push_back(int(lists[c].size()));
    h.cls_pairs.insert(h.cls_pairs.end(), lists[c].begin(), lists[c].end());
    // classes whose buffers exceed shared memory run them in global scratch
  }
  // chirp transforms: the radix-4 order for Bluestein rings of the size
  // classes, the register-pass order for those of the register classes
  std::vector<char> use4(h.descs.size(), 0), use16(h.descs.size(), 0);
  for (int p = 0; p < np; ++p)
    for (int hh = 0; hh < 2; ++hh) {
      const int i = 2 * p + hh;
      if (h.nph[i] <= 0) continue;
      const FftDesc &d = h.descs[h.fft[i]];
      if (is_pw[p] == 0 && d.blue) use4[h.fft[i]] = 1;
      if (is_pw[p] == 2) use16[h.fft[i]] = 1;   // register Bluestein pairs
    }
  for (int i = 0; i < int(h.descs.size()); ++i) {
    FftDesc &d = h.descs[i];
    if (use4[i]) {
      d.bhat = h.bhat_total;
      h.bhat_total += d.M;
      h.blue_idx.push_back(i);
    }
    if (use16[i]) {
      d.bhat2 = h.bhat_total;
      h.bhat_total += d.M;
      d.chirp = h.chirp_total;
      h.chirp_total += d.N;
      h.blue2_idx.push_back(i);
    }
    if (use4[i] || use16[i]) h.P = std::max(h.P, d.M);
  }
  return h;
}

namespace {

// ---------------------------------------------------------------------------
// geometry plan
// ---------------------------------------------------------------------------
std::unique_ptr<GeomPlan> build_geom_plan(const sharp_geom_info *g, int lmax, int mmax, int spin,
                                          cudaStream_t st) {
  const GeomHost h = build_geom_host(g, lmax, mmax, spin);
  auto gp = std::make_unique<GeomPlan>();
  gp->key = g;
  gp->hash = hash_geom(g);
  gp->lmax = lmax;
  gp->mmax = mmax;
  gp->spin = spin;
  gp->npairs = h.npairs;
  gp->nphmax = h.nphmax;
  gp->nmax_complex = h.nmax_complex;
  gp->count_m = h.count_m;
  gp->order = h.order;
  gp->synth_items = h.synth_items;
  gp->synth_tile = h.synth_tile;
  gp->mixed_items = h.mixed_items;
  gp->P = h.P;
  gp->cls_N = h.cls_N;
  gp->cls_start = h.cls_start;
  gp->cls_count = h.cls_count;
  gp->cls_bufA = h.cls_bufA;
  gp->cls_bufB = h.cls_bufB;
  gp->map_lo = h.map_lo;
  gp->map_hi = h.map_hi;
  gp->map_covered = h.map_covered;
  gp->cls_pairs = dev_upload(h.cls_pairs, st);
  gp->pw_N = h.pw_N;
  gp->pw_start = h.pw_start;
  gp->pw_count = h.pw_count;
  gp->pw_pairs = dev_upload(h.pw_pairs, st);
  gp->pb_M = h.pb_M;
  gp->pb_start = h.pb_start;
  gp->pb_count = h.pb_count;
  gp->pb_pairs = dev_upload(h.pb_pairs, st);
  gp->cth = dev_upload(h.cth, st);
  gp->sth = dev_upload(h.sth, st);
  gp->mlim = dev_upload(h.mlim_sorted, st);
  gp->count = dev_upload(gp->count_m, st);
  gp->items = dev_upload(gp->synth_items, st);
  gp->mitems = dev_upload(gp->mixed_items, st);
  gp->phi0 = dev_upload(h.phi0, st);
  gp->weight = dev_upload(h.weight, st);
  gp->ofs = dev_upload(h.ofs, st);
  gp->nph = dev_upload(h.nph, st);
  gp->stride = dev_upload(h.stride, st);
  gp->fft = dev_upload(h.fft, st);
  gp->fdesc = dev_upload(h.descs, st);
  SHT_CUDA(cudaMalloc(&gp->twiddle, sizeof(double2) * std::max<long long>(h.tw_total, 1)));
  launch_twiddles(*gp, int(h.tw_total), h.tw_n, h.tw_off, st);
  SHT_CUDA(cudaMalloc(&gp->bhat, sizeof(double2) * std::max<long long>(h.bhat_total, 1)));
  SHT_CUDA(cudaMalloc(&gp->wpow2, sizeof(double2) * gp->P));
  SHT_CUDA(cudaMalloc(&gp->chirp, sizeof(double2) * std::max<long long>(h.chirp_total, 1)));
  launch_bluestein_setup(*gp, h, st);
  SHT_CUDA(cudaStreamSynchronize(st));
  return gp;
}

GeomPlan *get_geom_plan(const sharp_geom_info *g, int lmax, int mmax, int spin, cudaStream_t st) {
  const uint64_t h = hash_geom(g);
  auto &vec = g_geom_cache[g];
  for (auto &p : vec)
    if (p->hash == h && p->lmax == lmax && p->mmax == mmax && p->spin == spin) return p.get();
  // drop stale plans of this address (content changed)
  vec.erase(std::remove_if(vec.begin(), vec.end(), [&](auto &p) { return p->hash != h; }),
            vec.end());
  if (vec.size() >= 8) vec.erase(vec.begin());
  vec.push_back(build_geom_plan(g, lmax, mmax, spin, st));
  return vec.back().get();
}

// ---------------------------------------------------------------------------
// coefficient plan
// ---------------------------------------------------------------------------
// sqrt((2 mhi)! / ((mhi+mlo)! (mhi-mlo)!)) as mantissa * 2^exp
// (prefactor of the spin seed, libsharp/sharp_ylmgen_c.c:97-118).
void spin_prefactor(int lmax, int mmax, int s, std::vector<double> &mant, std::vector<int> &ex) {
  std::vector<double> fm(2 * lmax + 1);
  std::vector<int> fe(2 * lmax + 1);
  fm[0] = 1.0;
  fe[0] = 0;
  for (int k = 1; k <= 2 * lmax; ++k) {
    int e;
    fm[k] = std::frexp(fm[k - 1] * std::sqrt(double(k)), &e);
    fe[k] = fe[k - 1] + e;
  }
  mant.resize(mmax + 1);
  ex.resize(mmax + 1);
  for (int m = 0; m <= mmax; ++m) {
    const int mhi = std::max(m, s), mlo = std::min(m, s);
    int e;
    double v = std::frexp(fm[2 * mhi] / fm[mhi + mlo], &e);
    int E = e + fe[2 * mhi] - fe[mhi + mlo];
    v = std::frexp(v / fm[mhi - mlo], &e);
    E += e - fe[mhi - mlo];
    mant[m] = v;
    ex[m] = E;
  }
}

CoefPlan *get_coef_plan(int lmax, int mmax, int spin, cudaStream_t st) {
  for (auto &p : g_coef_cache)
    if (p->lmax == lmax && p->mmax == mmax && p->spin == spin) return p.get();
  auto cp = std::make_unique<CoefPlan>();
  cp->lmax = lmax;
  cp->mmax = mmax;
  cp->spin = spin;
  cp->moff.resize(mmax + 2);
  long long off = 0;
  for (int m = 0; m <= mmax; ++m) {
    cp->moff[m] = off;
    off += (lmax - m + 1) + kPad;
  }
  cp->moff[mmax + 1] = off;
  cp->total = off;
  cp->d_moff = dev_upload(cp->moff, st);
  SHT_CUDA(cudaMalloc(&cp->alpha, sizeof(double) * off));
  SHT_CUDA(cudaMalloc(&cp->cfac, sizeof(double) * off));
  if (spin > 0) {
    SHT_CUDA(cudaMalloc(&cp->beta, sizeof(double) * off));
    std::vector<double> mant;
    std::vector<int> ex;
    spin_prefactor(lmax, mmax, spin, mant, ex);
    cp->seed = dev_upload(mant, st);
    cp->seed_exp = dev_upload(ex, st);
  } else {
    std::vector<double> mfac(mmax + 1);
    mfac[0] = 0.2820947917738781434740397257803862929220;  // 1/sqrt(4 pi)
    for (int m = 1; m <= mmax; ++m) mfac[m] = mfac[m - 1] * std::sqrt((2 * m + 1.) / (2 * m));
    cp->seed = dev_upload(mfac, st);
  }
  launch_coef_tables(*cp, st);
  SHT_CUDA(cudaStreamSynchronize(st));
  if (g_coef_cache.size() >= 6) g_coef_cache.erase(g_coef_cache.begin());
  g_coef_cache.push_back(std::move(cp));
  return g_coef_cache.back().get();
}

// ---------------------------------------------------------------------------
// a_lm plan
// ---------------------------------------------------------------------------
AlmPlan *get_alm_plan(const sharp_alm_info *a, int mmax, cudaStream_t st) {
  const uint64_t h = hash_alm(a);
  auto it = g_alm_cache.find(a);
  if (it != g_alm_cache.end() && it->second->hash == h) return it->second.get();
  auto ap = std::make_unique<AlmPlan>();
  ap->key = a;
  ap->hash = h;
  ap->lmax = a->lmax;
  ap->mmax = mmax;
  ap->packed = (a->flags & SHARP_PACKED) != 0;
  ap->stride = a->stride;
  std::vector<long long> mv(mmax + 1, 0);
  long long lo = 0, hi = 0, nslots = 0;
  bool first = true;
  for (int mi = 0; mi < a->nm; ++mi) {
    const int m = a->mval[mi];
    mv[m] = a->mvstart[mi];
    for (int l = m; l <= a->lmax; l += std::max(1, a->lmax - m)) {
      // first and last l bound the (monotone) index range of this m
      long long i0, i1;
      if (ap->packed && m == 0) {
        i0 = i1 = a->mvstart[mi] + (long long)l * a->stride;
      } else if (ap->packed) {
        i0 = a->mvstart[mi] + 2ll * l * a->stride;
        i1 = i0 + 1;
      } else {
        i0 = i1 = a->mvstart[mi] + (long long)l * a->stride;
      }
      const long long mn = std::min(i0, i1), mx = std::max(i0, i1) + 1;
      if (first) { lo = mn; hi = mx; first = false; }
      lo = std::min(lo, mn);
      hi = std::max(hi, mx);
      if (l == a->lmax) break;
    }
    nslots += (long long)(a->lmax - m + 1) * ((ap->packed && m != 0) ? 2 : 1);
  }
  ap->lo = lo;
  ap->hi = hi;
  ap->covered = (std::llabs(a->stride) == 1) && (nslots == hi - lo);
  ap->mvstart = dev_upload(mv, st);
  SHT_CUDA(cudaStreamSynchronize(st));
  auto *raw = ap.get();
  if (g_alm_cache.size() >= 64) g_alm_cache.clear();
  g_alm_cache[a] = std::move(ap);
  return raw;
}

// ---------------------------------------------------------------------------
// per-device library stream
// ---------------------------------------------------------------------------
cudaStream_t library_stream() {
  static std::map<int, cudaStream_t> streams;
  int dev = 0;
  SHT_CUDA(cudaGetDevice(&dev));
  auto it = streams.find(dev);
  if (it != streams.end()) return it->second;
  cudaStream_t s;
  SHT_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  streams[dev] = s;
  return s;
}

// Error word of the tensor-core kernels: pinned, mapped host memory the
// kernels store a nonzero value into when a bounded wait gives up.  Read
// without synchronisation: a host-pointer call checks it after its final
// synchronisation, a device-pointer call finds a failure of an earlier call
// at its start.
int *tc_error_word(int **dev_view) {
  static int *host = nullptr;
  static std::map<int, int *> views;
  if (!host) {
    SHT_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&host), sizeof(int), cudaHostAllocMapped |
                           cudaHostAllocPortable));
    *reinterpret_cast<volatile int *>(host) = 0;
  }
  int dev = 0;
  SHT_CUDA(cudaGetDevice(&dev));
  auto it = views.find(dev);
  if (it == views.end()) {
    int *d = nullptr;
    SHT_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void **>(&d), host, 0));
    it = views.emplace(dev, d).first;
  }
  if (dev_view) *dev_view = it->second;
  return host;
}

void check_tc_error() {
  volatile int *w = tc_error_word(nullptr);
  if (*w) {
    *w = 0;
    fail(__FILE__, __LINE__, "a tensor-core transform gave up waiting on the device (SHARP_MIXED)");
  }
}

struct DevBuf {
  void *p = nullptr;
  cudaStream_t st = nullptr;
  DevBuf() = default;
  DevBuf(size_t bytes, cudaStream_t s) : st(s) {
    if (bytes) SHT_CUDA(::sht::ws_alloc(&p, bytes, s));
  }
  ~DevBuf() {
    if (p) cudaFreeAsync(p, st);
  }
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  template <typename T>
  T *as() const { return static_cast<T *>(p); }
};

double wall_now() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// ---------------------------------------------------------------------------
// the job
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Pass-width tuner, the counterpart of the reference's nv oracle
// (libsharp/sharp.c:890-965, which times its SIMD vector counts on first
// use): the FP64 Legendre kernels take 1, 2 or 4 transforms per pass (spin s
// and deriv1: 1 or 2); wider passes share one recurrence, narrower ones keep
// more CTAs per SM, and which wins depends on the geometry, lmax and spin.
// The first job of a shape with several transforms times each width once on
// its own buffers (after one untimed run of it; one host synchronisation per
// width) and the fastest is kept for the process, the default width unless
// another is more than 3% faster.  Jobs whose flags carry a vector-count hint (the low bits,
// SHARP_NVMAX, as the reference's nv), jobs on a stream that is being
// captured, and all jobs when SHARP_B200_TUNE=0 keep the default widths;
// SHARP_B200_TUNE_LOG prints each decision with its timings to stderr.
// ---------------------------------------------------------------------------
struct TuneKey {
  uint64_t geom;
  int lmax, mmax, spin, type, ntrans, pass;   // pass: 0 synthesis, 1 analysis
  bool operator<(const TuneKey &o) const {
    return std::tie(geom, lmax, mmax, spin, type, ntrans, pass) <
           std::tie(o.geom, o.lmax, o.mmax, o.spin, o.type, o.ntrans, o.pass);
  }
};
std::mutex g_tune_mutex;
std::map<TuneKey, int> g_tuned;

bool tuner_on(int flags, cudaStream_t st) {
  static const bool env_on = [] {
    const char *e = getenv("SHARP_B200_TUNE");
    return !(e && e[0] == '0');
  }();
  if (!env_on || (flags & SHARP_NVMAX) != 0) return false;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  return cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone;
}

// run(w) enqueues every pass of the job with width w on st; reset() undoes
// what the timing runs accumulated.  Returns the width to use.
int tuned_width(const TuneKey &key, int wmax, int wdefault, const std::function<void(int)> &run,
                const std::function<void()> &reset, cudaStream_t st) {
  std::lock_guard<std::mutex> lk(g_tune_mutex);
  auto it = g_tuned.find(key);
  if (it != g_tuned.end()) return it->second;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  SHT_CUDA(cudaEventCreate(&e0));
  SHT_CUDA(cudaEventCreate(&e1));
  std::vector<std::pair<int, float>> times;
  for (int w = 1; w <= wmax; w *= 2) {
    run(w);   // untimed: first launch of the width's kernels, first touch of the buffers
    SHT_CUDA(cudaEventRecord(e0, st));
    run(w);
    SHT_CUDA(cudaEventRecord(e1, st));
    SHT_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    SHT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    times.push_back({w, ms});
  }
  SHT_CUDA(cudaEventDestroy(e0));
  SHT_CUDA(cudaEventDestroy(e1));
  reset();
  float tdef = 0.f;
  for (auto &t : times)
    if (t.first == wdefault) tdef = t.second;
  int best = wdefault;
  float tbest = tdef;
  for (auto &t : times)
    if (t.second < tbest && t.second < 0.97f * tdef) {
      best = t.first;
      tbest = t.second;
    }
  g_tuned[key] = best;
  static const bool log = getenv("SHARP_B200_TUNE_LOG") != nullptr;
  if (log) {
    std::fprintf(stderr, "sharp_b200 tuner: %s spin %d lmax %d ntrans %d:",
                 key.pass ? "analysis" : "synthesis", key.spin, key.lmax, key.ntrans);
    for (auto &t : times) std::fprintf(stderr, " width %d %.3f ms", t.first, t.second);
    std::fprintf(stderr, " -> %d\n", best);
  }
  return best;
}

void execute_impl(sharp_jobtype type_in, int spin, void *alm, void *map,
                  const sharp_geom_info *ginfo, const sharp_alm_info *ainfo, int ntrans,
                  int flags, bool device_ptrs, cudaStream_t user_stream, double *time,
                  unsigned long long *opcnt) {
  const double t0 = wall_now();
  int type = int(type_in);
  SHT_REQUIRE(type >= 0 && type <= 4, "bad job type");
  SHT_REQUIRE(ginfo != nullptr && ainfo != nullptr, "null geometry or alm info");
  SHT_REQUIRE(ntrans > 0 && ntrans <= kMaxTrans, "bad number of simultaneous transforms");
  if (flags & SHARP_ADJOINT) {
    // transpose of the named type (Y <-> Yt, YtW <-> WY)
    static const int adj[5] = {SHARP_WY, SHARP_Yt, SHARP_Y, SHARP_YtW, -1};
    SHT_REQUIRE(adj[type] >= 0, "SHARP_ADJOINT is not defined for SHARP_ALM2MAP_DERIV1");
    type = adj[type];
    flags &= ~int(SHARP_ADJOINT);
  }
  // sharp_build_job_common, libsharp/sharp.c:840-867
  if (type == SHARP_ALM2MAP_DERIV1) spin = 1;
  if (type == SHARP_MAP2ALM) flags |= SHARP_USE_WEIGHTS;
  if (type == SHARP_Yt) type = SHARP_MAP2ALM;
  if (type == SHARP_WY) {
    type = SHARP_ALM2MAP;
    flags |= SHARP_USE_WEIGHTS;
  }
  SHT_REQUIRE(spin >= 0 && spin <= ainfo->lmax, "bad spin");
  SHT_REQUIRE((flags & kAccumulate) != kAccumulate,
              "SHARP_ADD and SHARP_SUBTRACT exclude each other");
  SHT_REQUIRE(!(flags & SHARP_MIXED) || (type == SHARP_ALM2MAP && spin == 0) ||
                  type == SHARP_MAP2ALM || type == SHARP_ALM2MAP,
              "SHARP_MIXED applies to alm2map and map2alm jobs");
  // all m from 0 to nm-1 exactly once (sharp_get_mmax, sharp.c:238-251)
  const int nm = ainfo->nm;
  {
    std::vector<char> seen(std::max(nm, 1), 0);
    for (int i = 0; i < nm; ++i) {
      const int mv = ainfo->mval[i];
      SHT_REQUIRE(mv >= 0 && mv < nm, "not all m values are present");
      SHT_REQUIRE(!seen[mv], "duplicate m value");
      seen[mv] = 1;
    }
  }
  const int mmax = nm - 1;
  SHT_REQUIRE(mmax <= ainfo->lmax, "incorrect l_max: must be >= m_max");
  const bool deriv = type == SHARP_ALM2MAP_DERIV1;
  JobDesc job{};
  job.type = type;
  job.spin = spin;
  job.nmaps = (deriv || spin > 0) ? 2 : 1;
  job.nalm = deriv ? 1 : (spin > 0 ? 2 : 1);
  job.ntrans = ntrans;
  job.flags = flags;
  job.lmax = ainfo->lmax;
  job.mmax = mmax;
  job.dp = (flags & SHARP_DP) != 0;
  const bool analysis = type == SHARP_MAP2ALM;
  const bool no_fft = (flags & SHARP_NO_FFT) != 0;
  if (no_fft)
    for (int i = 0; i < ginfo->npairs; ++i) {
      SHT_REQUIRE(ginfo->pair[i].r1.nph == mmax + 1, "bad ring size");
      SHT_REQUIRE(ginfo->pair[i].r2.nph < 0 || ginfo->pair[i].r2.nph == mmax + 1, "bad ring size");
    }

  std::lock_guard<std::mutex> lk(g_cache_mutex);
  if (flags & SHARP_MIXED) check_tc_error();
  cudaStream_t st = device_ptrs ? user_stream : library_stream();
  GeomPlan *gp = get_geom_plan(ginfo, job.lmax, mmax, spin, st);
  CoefPlan *cp = get_coef_plan(job.lmax, mmax, spin, st);
  AlmPlan *ap = get_alm_plan(ainfo, mmax, st);

  const int nalmptr = ntrans * job.nalm;
  const int nmapptr = ntrans * job.nmaps;
  const int ncA = nalmptr;
  const int ncm = nmapptr;
  void **alm_in = static_cast<void **>(alm);
  void **map_in = static_cast<void **>(map);

  // norm_l (libsharp/sharp_ylmgen_c.c:200-232)
  std::vector<double> norm(job.lmax + 1, 1.0);
  if (deriv) {
    for (int l = 0; l <= job.lmax; ++l)
      norm[l] = (l < 1) ? 0. : 0.5 * std::sqrt(l * (l + 1.) * (2 * l + 1.) / (4 * M_PI));
  } else if (spin > 0) {
    double spinsign = -1.0;
    if (spin & 1) spinsign = -spinsign;
    for (int l = 0; l <= job.lmax; ++l)
      norm[l] = (l < spin) ? 0. : spinsign * 0.5 * std::sqrt((2 * l + 1) / (4 * M_PI));
  }
  DevBuf d_norm(sizeof(double) * norm.size(), st);
  SHT_CUDA(cudaMemcpyAsync(d_norm.p, norm.data(), sizeof(double) * norm.size(),
                           cudaMemcpyHostToDevice, st));

  // device views of the user arrays
  const size_t esz_map = (job.dp ? 8 : 4) * (no_fft ? 2 : 1);
  const size_t esz_alm = (job.dp ? 8 : 4) * (ap->packed ? 1 : 2);
  const long long map_n = gp->map_hi - gp->map_lo;
  const long long alm_n = ap->hi - ap->lo;
  std::vector<void *> dmap(nmapptr), dalm(nalmptr);
  std::vector<std::unique_ptr<DevBuf>> owned;
  long long map_lo = 0, alm_lo = 0;
  if (device_ptrs) {
    for (int i = 0; i < nmapptr; ++i) dmap[i] = map_in[i];
    for (int i = 0; i < nalmptr; ++i) dalm[i] = alm_in[i];
  } else {
    map_lo = gp->map_lo;
    alm_lo = ap->lo;
    const bool load_maps = analysis || (flags & kAccumulate) || !gp->map_covered;
    const bool load_alm = !analysis || (flags & kAccumulate) || !ap->covered;
    for (int i = 0; i < nmapptr; ++i) {
      owned.emplace_back(new DevBuf(esz_map * map_n, st));
      dmap[i] = owned.back()->p;
      if (load_maps && map_n > 0)
        SHT_CUDA(cudaMemcpyAsync(dmap[i], static_cast<char *>(map_in[i]) + esz_map * map_lo,
                                 esz_map * map_n, cudaMemcpyHostToDevice, st));
    }
    for (int i = 0; i < nalmptr; ++i) {
      owned.emplace_back(new DevBuf(esz_alm * alm_n, st));
      dalm[i] = owned.back()->p;
      if (load_alm && alm_n > 0)
        SHT_CUDA(cudaMemcpyAsync(dalm[i], static_cast<char *>(alm_in[i]) + esz_alm * alm_lo,
                                 esz_alm * alm_n, cudaMemcpyHostToDevice, st));
    }
  }
  DevBuf d_mapptr(sizeof(void *) * nmapptr, st), d_almptr(sizeof(void *) * nalmptr, st);
  SHT_CUDA(cudaMemcpyAsync(d_mapptr.p, dmap.data(), sizeof(void *) * nmapptr,
                           cudaMemcpyHostToDevice, st));
  SHT_CUDA(cudaMemcpyAsync(d_almptr.p, dalm.data(), sizeof(void *) * nalmptr,
                           cudaMemcpyHostToDevice, st));

  const size_t phase_bytes = sizeof(double2) * 2 * size_t(mmax + 1) * gp->npairs * ncm;
  DevBuf d_phase(phase_bytes, st);
  double2 *phase = d_phase.as<double2>();
  const int ntmax_synth = (spin == 0 && !deriv) ? 4 : 2;
  // FP64 analysis: one transform per launch is fastest per transform (the
  // per-thread phase factors of several transforms cost occupancy): at Nside
  // 2048 / lmax 4096, spin 0 takes 14.1 ms at 1, 15.2 ms each at 4; spin 2
  // takes 44.9 ms at 1, 54.1 ms each at 2.
  const int ntmax_anal = 1;
  auto group = [&](int left, int ntmax) {
    int nt = 1;
    while (nt * 2 <= ntmax && nt * 2 <= left) nt *= 2;
    return nt;
  };

  if (!analysis) {
    DevBuf d_A(sizeof(double2) * size_t(cp->total) * ncA, st);
    launch_stage_alm(job, *ap, alm_lo, *cp, d_norm.as<double>(),
                     reinterpret_cast<void *const *>(d_almptr.p), nalmptr, d_A.as<double2>(), ncA,
                     st);
    if ((flags & SHARP_MIXED) && mixed_synth_supported(job)) {
      int *d_err = nullptr;
      tc_error_word(&d_err);
      launch_mixed_synth(job, *gp, *cp, d_A.as<double2>(), ncA, phase, ncm, d_err, st);
    } else {
      auto passes = [&](int width) {
        for (int t0 = 0; t0 < ntrans;) {
          const int nt = group(ntrans - t0, width);
          launch_legendre_synth(job, *gp, *cp, d_A.as<double2>(), ncA, t0 * job.nalm, nt,
                                phase, ncm, t0 * job.nmaps, st);
          t0 += nt;
        }
      };
      int width = ntmax_synth;
      if (ntrans >= 2 && tuner_on(flags, st))
        // synthesis passes overwrite the phase rows, so the timing runs leave nothing behind
        width = tuned_width(TuneKey{gp->hash, job.lmax, mmax, spin, type, ntrans, 0},
                            ntmax_synth, ntmax_synth, passes, [] {}, st);
      passes(width);
    }
    if (no_fft)
      launch_phase2ring_direct(job, *gp, map_lo, phase, ncm,
                               reinterpret_cast<void *const *>(d_mapptr.p), nmapptr, st);
    else
      launch_phase2ring(job, *gp, map_lo, phase, ncm, reinterpret_cast<void *const *>(d_mapptr.p),
                        nmapptr, st);
    if (!device_ptrs && map_n > 0)
      for (int i = 0; i < nmapptr; ++i)
        SHT_CUDA(cudaMemcpyAsync(static_cast<char *>(map_in[i]) + esz_map * map_lo, dmap[i],
                                 esz_map * map_n, cudaMemcpyDeviceToHost, st));
  } else {
    if (no_fft)
      launch_ring2phase_direct(job, *gp, map_lo,
                               reinterpret_cast<const void *const *>(d_mapptr.p), nmapptr, phase,
                               ncm, st);
    else
      launch_ring2phase(job, *gp, map_lo, reinterpret_cast<const void *const *>(d_mapptr.p),
                        nmapptr, phase, ncm, st);
    DevBuf d_Aout(sizeof(double2) * size_t(cp->total) * ncA, st);
    SHT_CUDA(cudaMemsetAsync(d_Aout.p, 0, sizeof(double2) * size_t(cp->total) * ncA, st));
    if ((flags & SHARP_MIXED) && mixed_anal_supported(job)) {
      int *d_err = nullptr;
      tc_error_word(&d_err);
      launch_mixed_anal(job, *gp, *cp, phase, ncm, d_Aout.as<double2>(), ncA, d_err, st);
    } else {
      auto passes = [&](int width) {
        for (int t0 = 0; t0 < ntrans;) {
          const int nt = group(ntrans - t0, width);
          launch_legendre_anal(job, *gp, *cp, phase, ncm, t0 * job.nmaps, nt,
                               d_Aout.as<double>(), ncA, t0 * job.nalm, st);
          t0 += nt;
        }
      };
      int width = ntmax_anal;
      if (ntrans >= 2 && tuner_on(flags, st)) {
        // analysis passes accumulate into Aout: cleared again after the timing runs
        auto clear = [&] {
          SHT_CUDA(cudaMemsetAsync(d_Aout.p, 0, sizeof(double2) * size_t(cp->total) * ncA, st));
        };
        width = tuned_width(TuneKey{gp->hash, job.lmax, mmax, spin, type, ntrans, 1},
                            spin == 0 ? 4 : 2, ntmax_anal, passes, clear, st);
      }
      passes(width);
    }
    launch_scatter_alm(job, *ap, alm_lo, *cp, d_norm.as<double>(), d_Aout.as<double>(), ncA,
                       reinterpret_cast<void *const *>(d_almptr.p), nalmptr, st);
    if (!device_ptrs && alm_n > 0)
      for (int i = 0; i < nalmptr; ++i)
        SHT_CUDA(cudaMemcpyAsync(static_cast<char *>(alm_in[i]) + esz_alm * alm_lo, dalm[i],
                                 esz_alm * alm_n, cudaMemcpyDeviceToHost, st));
  }
  if (!device_ptrs) {
    SHT_CUDA(cudaStreamSynchronize(st));
    if (flags & SHARP_MIXED) check_tc_error();
  }
  owned.clear();

  if (opcnt) {
    // per (l, m, pair) weight the reference counts (sharp_core_inc2.c:173,442,585)
    const unsigned long long c = (spin == 0 && !deriv) ? 4 + 4ull * ntrans
                                 : deriv ? 12 + 8ull * ntrans : 12 + 16ull * ntrans;
    unsigned long long tot = 0;
    for (int m = 0; m <= mmax; ++m) {
      const int l0 = (spin == 0) ? m : std::max(m, spin);
      if (l0 <= job.lmax) tot += (unsigned long long)gp->count_m[m] * (job.lmax - l0 + 1);
    }
    *opcnt = tot * c;
  }
  if (time) *time = wall_now() - t0;
}

// ---------------------------------------------------------------------------
// Host-array jobs with several transforms: the transforms run in pieces so
// that the host->device copies of piece k+1 and the device->host copies of
// piece k-1 overlap the compute of piece k (three streams, event-ordered).
// Each piece is an ordinary device-pointer job on window buffers; every
// transform's arithmetic is that of the single-call path, so the results
// are the same.  Returns false (nothing done) where the plain path applies.
// ---------------------------------------------------------------------------
// Library streams of the current device: 0 and 1 carry the host-array
// copies, 2 .. 2 + kBatchLanes - 1 the concurrent groups of a batch.
cudaStream_t copy_stream(int which) {
  static std::map<std::pair<int, int>, cudaStream_t> streams;
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  int dev = 0;
  SHT_CUDA(cudaGetDevice(&dev));
  auto key = std::make_pair(dev, which);
  auto it = streams.find(key);
  if (it != streams.end()) return it->second;
  cudaStream_t s;
  SHT_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  streams[key] = s;
  return s;
}

// A host-array job the pipelined path can take (checked like execute_impl
// would; anything else goes through execute_impl, which reports the error).
bool pipelinable(sharp_jobtype type, int spin, const void *alm, const void *map,
                 const sharp_geom_info *ginfo, const sharp_alm_info *ainfo, int ntrans,
                 int flags) {
  if (type != SHARP_ALM2MAP && type != SHARP_MAP2ALM) return false;
  if (flags & (SHARP_ADJOINT | SHARP_NO_FFT)) return false;
  if ((flags & kAccumulate) == kAccumulate) return false;
  if (!ginfo || !ainfo || !alm || !map || ntrans < 1 || ntrans > kMaxTrans) return false;
  if (spin < 0 || spin > ainfo->lmax || ainfo->nm < 1 || ainfo->nm - 1 > ainfo->lmax) return false;
  // every m exactly once (otherwise the plain path reports the error)
  std::vector<char> seen(ainfo->nm, 0);
  for (int i = 0; i < ainfo->nm; ++i) {
    const int mv = ainfo->mval[i];
    if (mv < 0 || mv >= ainfo->nm || seen[mv]) return false;
    seen[mv] = 1;
  }
  return true;
}

struct HostJob {
  sharp_jobtype type;
  int spin;
  void *alm, *map;
  const sharp_geom_info *ginfo;
  const sharp_alm_info *ainfo;
  int ntrans, flags;
};

// Runs host-array jobs as one sequence of pieces (see above): the copies of
// consecutive pieces overlap the compute across job boundaries too, so a
// list of jobs has one fill and one drain.  Every job must satisfy
// pipelinable().  A job may read host arrays that an earlier job of the
// list writes (a round trip: alm2map, then map2alm of its maps): the input
// copy of such bytes waits for the output copy of the piece that wrote
// them, so the data passes through host memory in order while the other
// pieces keep the copy engines and the GPU busy.  (Writes after reads and
// after writes are ordered already: every output copy follows the compute
// of its piece, which follows all earlier input copies, on one output
// stream.)  *opcnt receives the summed operation count of the jobs.
void execute_pipelined_jobs(const std::vector<HostJob> &jobs, unsigned long long *opcnt) {
  cudaStream_t cs = library_stream();
  cudaStream_t sin = copy_stream(0), sout = copy_stream(1);
  // window buffers of one piece, released on the output stream after its copies
  struct Piece {
    std::vector<void *> dmap, dalm;
    cudaEvent_t in_done = nullptr, compute_done = nullptr, out_done = nullptr;
  };
  std::vector<Piece> pieces;
  // host byte ranges written by the output copies so far: [lo, hi), piece
  struct Written {
    uintptr_t lo, hi;
    int piece;
  };
  std::vector<Written> written;
  // makes the input stream wait for the last output copy that wrote any of
  // [src, src + bytes)
  auto order_after_writes = [&](const void *src, size_t bytes) {
    const uintptr_t lo = reinterpret_cast<uintptr_t>(src), hi = lo + bytes;
    int last = -1;
    for (const Written &w : written)
      if (w.lo < hi && lo < w.hi) last = std::max(last, w.piece);
    if (last >= 0) SHT_CUDA(cudaStreamWaitEvent(sin, pieces[last].out_done, 0));
  };
  auto release = [&]() {
    for (auto &pc : pieces) {
      for (void *p : pc.dmap) if (p) cudaFreeAsync(p, sout);
      for (void *p : pc.dalm) if (p) cudaFreeAsync(p, sout);
      if (pc.in_done) cudaEventDestroy(pc.in_done);
      if (pc.compute_done) cudaEventDestroy(pc.compute_done);
      if (pc.out_done) cudaEventDestroy(pc.out_done);
    }
    pieces.clear();
  };
  unsigned long long total_ops = 0;
  bool any_mixed = false;
  try {
    for (const HostJob &jb : jobs) {
      const sharp_jobtype type = jb.type;
      const int spin = jb.spin, ntrans = jb.ntrans, flags = jb.flags;
      const sharp_geom_info *ginfo = jb.ginfo;
      const sharp_alm_info *ainfo = jb.ainfo;
      any_mixed = any_mixed || (flags & SHARP_MIXED);
      const bool analysis = type == SHARP_MAP2ALM;
      // piece size: the transforms one launch of the batched kernels takes
      const int piece = spin > 0 ? 3 : (analysis ? 6 : 4);
      const int ncomp = spin > 0 ? 2 : 1;       // maps and a_lm per transform
      const bool dp = (flags & SHARP_DP) != 0;
      long long map_lo, map_hi, alm_lo, alm_hi;
      bool map_covered, alm_covered, packed;
      {
        std::lock_guard<std::mutex> lk(g_cache_mutex);
        const int mmax = ainfo->nm - 1;
        GeomPlan *gp = get_geom_plan(ginfo, ainfo->lmax, mmax, spin, cs);
        AlmPlan *ap = get_alm_plan(ainfo, mmax, cs);
        map_lo = gp->map_lo; map_hi = gp->map_hi; map_covered = gp->map_covered;
        alm_lo = ap->lo; alm_hi = ap->hi; alm_covered = ap->covered; packed = ap->packed;
      }
      const size_t esz_map = dp ? 8 : 4, esz_alm = (dp ? 8 : 4) * (packed ? 1 : 2);
      const long long map_n = map_hi - map_lo, alm_n = alm_hi - alm_lo;
      const bool load_maps = analysis || (flags & kAccumulate) || !map_covered;
      const bool load_alm = !analysis || (flags & kAccumulate) || !alm_covered;
      void **alm_in = static_cast<void **>(jb.alm);
      void **map_in = static_cast<void **>(jb.map);
      unsigned long long first_ops = 0;
      for (int t0p = 0; t0p < ntrans; t0p += piece) {
        const int nt = std::min(piece, ntrans - t0p);
        pieces.emplace_back();
        Piece &pc = pieces.back();
        pc.dmap.assign(size_t(nt) * ncomp, nullptr);
        pc.dalm.assign(size_t(nt) * ncomp, nullptr);
        SHT_CUDA(cudaEventCreateWithFlags(&pc.in_done, cudaEventDisableTiming));
        SHT_CUDA(cudaEventCreateWithFlags(&pc.compute_done, cudaEventDisableTiming));
        SHT_CUDA(cudaEventCreateWithFlags(&pc.out_done, cudaEventDisableTiming));
        const int this_piece = int(pieces.size()) - 1;
        // inputs of the piece: host -> device on the input stream
        for (int i = 0; i < nt * ncomp; ++i) {
          const int gi = t0p * ncomp + i;
          SHT_CUDA(::sht::ws_alloc(&pc.dmap[i], esz_map * std::max<long long>(map_n, 1), sin));
          SHT_CUDA(::sht::ws_alloc(&pc.dalm[i], esz_alm * std::max<long long>(alm_n, 1), sin));
          if (load_maps && map_n > 0) {
            const char *src = static_cast<char *>(map_in[gi]) + esz_map * map_lo;
            order_after_writes(src, esz_map * map_n);
            SHT_CUDA(cudaMemcpyAsync(pc.dmap[i], src, esz_map * map_n, cudaMemcpyHostToDevice,
                                     sin));
          }
          if (load_alm && alm_n > 0) {
            const char *src = static_cast<char *>(alm_in[gi]) + esz_alm * alm_lo;
            order_after_writes(src, esz_alm * alm_n);
            SHT_CUDA(cudaMemcpyAsync(pc.dalm[i], src, esz_alm * alm_n, cudaMemcpyHostToDevice,
                                     sin));
          }
        }
        SHT_CUDA(cudaEventRecord(pc.in_done, sin));
        // compute on the library stream: a device-pointer job whose array
        // bases are placed so that element lo sits at the start of each window
        SHT_CUDA(cudaStreamWaitEvent(cs, pc.in_done, 0));
        std::vector<void *> bm(nt * ncomp), ba(nt * ncomp);
        for (int i = 0; i < nt * ncomp; ++i) {
          bm[i] = static_cast<char *>(pc.dmap[i]) - esz_map * map_lo;
          ba[i] = static_cast<char *>(pc.dalm[i]) - esz_alm * alm_lo;
        }
        unsigned long long oc = 0;
        execute_impl(type, spin, ba.data(), bm.data(), ginfo, ainfo, nt, flags, true, cs,
                     nullptr, &oc);
        if (t0p == 0) first_ops = oc;
        SHT_CUDA(cudaEventRecord(pc.compute_done, cs));
        // outputs of the piece: device -> host on the output stream
        SHT_CUDA(cudaStreamWaitEvent(sout, pc.compute_done, 0));
        for (int i = 0; i < nt * ncomp; ++i) {
          const int gi = t0p * ncomp + i;
          char *dst = nullptr;
          size_t bytes = 0;
          if (analysis) {
            if (alm_n > 0) {
              dst = static_cast<char *>(alm_in[gi]) + esz_alm * alm_lo;
              bytes = esz_alm * alm_n;
              SHT_CUDA(cudaMemcpyAsync(dst, pc.dalm[i], bytes, cudaMemcpyDeviceToHost, sout));
            }
          } else if (map_n > 0) {
            dst = static_cast<char *>(map_in[gi]) + esz_map * map_lo;
            bytes = esz_map * map_n;
            SHT_CUDA(cudaMemcpyAsync(dst, pc.dmap[i], bytes, cudaMemcpyDeviceToHost, sout));
          }
          if (bytes)
            written.push_back(Written{reinterpret_cast<uintptr_t>(dst),
                                      reinterpret_cast<uintptr_t>(dst) + bytes, this_piece});
        }
        SHT_CUDA(cudaEventRecord(pc.out_done, sout));
      }
      // the count of one call with all transforms (per-triple weight of
      // sharp_core_inc2.c:173,442): the pieces share the triples
      const int n0 = std::min(piece, ntrans);
      const unsigned long long c0 = spin == 0 ? 4 + 4ull * n0 : 12 + 16ull * n0;
      const unsigned long long c = spin == 0 ? 4 + 4ull * ntrans : 12 + 16ull * ntrans;
      total_ops += (first_ops / c0) * c;
    }
    release();
    SHT_CUDA(cudaStreamSynchronize(sout));
    SHT_CUDA(cudaStreamSynchronize(cs));
    if (any_mixed) check_tc_error();
  } catch (const Failure &) {
    release();
    cudaStreamSynchronize(sout);
    cudaStreamSynchronize(cs);
    throw;
  }
  if (opcnt) *opcnt = total_ops;
}

// sharp_execute on host arrays: jobs of several transforms go through the
// pipelined path; returns false (nothing done) where the plain path applies.
bool execute_pipelined(sharp_jobtype type, int spin, void *alm, void *map,
                       const sharp_geom_info *ginfo, const sharp_alm_info *ainfo, int ntrans,
                       int flags, double *time, unsigned long long *opcnt) {
  if (!pipelinable(type, spin, alm, map, ginfo, ainfo, ntrans, flags)) return false;
  const int piece = spin > 0 ? 3 : (type == SHARP_MAP2ALM ? 6 : 4);
  if (ntrans <= piece) return false;
  const double t0 = wall_now();
  execute_pipelined_jobs({HostJob{type, spin, alm, map, ginfo, ainfo, ntrans, flags}}, opcnt);
  if (time) *time = wall_now() - t0;
  return true;
}

bool guarded(const std::function<void()> &fn) {
  try {
    fn();
    return true;
  } catch (const Failure &) {
    // message already recorded; non-aborting mode returns to the caller
    return false;
  }
}

// Host byte range [lo, hi) that one array of a job spans (maps: the ring
// pixels; a_lm: the layout's entries), from the geometry and a_lm structs.
std::pair<uintptr_t, uintptr_t> host_span(const void *base, const sharp_b200_job &j, bool maps) {
  const size_t ereal = (j.flags & SHARP_DP) ? 8 : 4;
  long long lo = 0, hi = 0;
  bool first = true;
  auto take = [&](long long a, long long b) {
    const long long mn = std::min(a, b), mx = std::max(a, b) + 1;
    if (first) { lo = mn; hi = mx; first = false; }
    lo = std::min(lo, mn);
    hi = std::max(hi, mx);
  };
  size_t esz = ereal;
  if (maps) {
    const sharp_geom_info *g = j.geom_info;
    for (int p = 0; p < g->npairs; ++p)
      for (int h = 0; h < 2; ++h) {
        const sharp_ringinfo &r = h ? g->pair[p].r2 : g->pair[p].r1;
        if (r.nph > 0) take(r.ofs, r.ofs + (long long)(r.nph - 1) * r.stride);
      }
  } else {
    const sharp_alm_info *a = j.alm_info;
    const bool packed = (a->flags & SHARP_PACKED) != 0;
    esz = packed ? ereal : 2 * ereal;
    for (int mi = 0; mi < a->nm; ++mi) {
      const int m = a->mval[mi];
      if (m > a->lmax) continue;
      const long long s = a->stride, e = packed && m != 0 ? 2 : 1;
      const long long i0 = a->mvstart[mi] + e * m * s, i1 = a->mvstart[mi] + e * a->lmax * s;
      take(i0, i1);
      take(i0 + e - 1, i1 + e - 1);   // the imaginary entries of a packed layout
    }
  }
  const uintptr_t b = reinterpret_cast<uintptr_t>(base);
  return {b + uintptr_t(lo * (long long)esz), b + uintptr_t(hi * (long long)esz)};
}

// Batch of jobs: jobs with the same type, spin, flags, geometry and a_lm
// objects are merged (their pointer arrays concatenated in order) into jobs
// of at most kMaxTrans transforms; each merged job runs through
// execute_impl.  With host arrays a job may read what an earlier job writes:
// such batches merge only consecutive jobs, so that no job moves ahead of
// one it depends on.  Returns the number of merged jobs.
struct BatchGroup {
  const sharp_b200_job *first;
  std::vector<void *> alm, map;
  int ntrans = 0;
};

// The merged groups of a batch, in order; group_of (if given) receives each
// job's group index.  Host work only.
std::vector<BatchGroup> group_batch(const sharp_b200_job *jobs, int njobs, bool device_ptrs,
                                    std::vector<int> *group_of) {
  SHT_REQUIRE(njobs >= 0 && (jobs != nullptr || njobs == 0), "bad job list");
  std::vector<BatchGroup> groups;
  // pointers per transform before the type remap (sharp.c:855-856)
  auto counts = [](const sharp_b200_job &j, int &na, int &nm) {
    const bool deriv = j.type == SHARP_ALM2MAP_DERIV1;
    na = deriv ? 1 : (j.spin > 0 ? 2 : 1);
    nm = (deriv || j.spin > 0) ? 2 : 1;
  };
  for (int i = 0; i < njobs; ++i) {
    const sharp_b200_job &j = jobs[i];
    SHT_REQUIRE(j.ntrans > 0 && j.ntrans <= kMaxTrans, "bad number of simultaneous transforms");
    SHT_REQUIRE(j.alm != nullptr && j.map != nullptr, "null alm or map pointer array");
    SHT_REQUIRE(j.geom_info != nullptr && j.alm_info != nullptr, "null geometry or a_lm info");
  }
  // host arrays: does any job read bytes that another job writes?
  bool dependent = false;
  if (!device_ptrs) {
    struct Span {
      uintptr_t lo, hi;
      int job;
    };
    std::vector<Span> reads, writes;
    for (int i = 0; i < njobs; ++i) {
      const sharp_b200_job &j = jobs[i];
      int na, nm;
      counts(j, na, nm);
      const bool to_alm = j.type == SHARP_MAP2ALM || j.type == SHARP_Yt;
      void *const *pa = static_cast<void *const *>(j.alm);
      void *const *pm = static_cast<void *const *>(j.map);
      for (int t = 0; t < j.ntrans * na; ++t) {
        if (!pa[t]) continue;
        const auto sp = host_span(pa[t], j, false);
        (to_alm ? writes : reads).push_back(Span{sp.first, sp.second, i});
      }
      for (int t = 0; t < j.ntrans * nm; ++t) {
        if (!pm[t]) continue;
        const auto sp = host_span(pm[t], j, true);
        (to_alm ? reads : writes).push_back(Span{sp.first, sp.second, i});
      }
    }
    for (const Span &r : reads) {
      for (const Span &w : writes)
        if (r.job != w.job && r.lo < w.hi && w.lo < r.hi) {
          dependent = true;
          break;
        }
      if (dependent) break;
    }
  }
  if (group_of) group_of->assign(njobs, -1);
  for (int i = 0; i < njobs; ++i) {
    const sharp_b200_job &j = jobs[i];
    int na, nm;
    counts(j, na, nm);
    // independent jobs: any earlier group; a host batch with dependences:
    // the last group only, so that merging never moves a job ahead of one
    // it depends on
    int gi = -1;
    for (size_t k = dependent ? (groups.empty() ? 0 : groups.size() - 1) : 0;
         k < groups.size(); ++k) {
      const BatchGroup &c = groups[k];
      const sharp_b200_job &f = *c.first;
      if (f.type == j.type && f.spin == j.spin && f.flags == j.flags &&
          f.geom_info == j.geom_info && f.alm_info == j.alm_info &&
          c.ntrans + j.ntrans <= kMaxTrans) {
        gi = int(k);
        break;
      }
    }
    if (gi < 0) {
      groups.push_back(BatchGroup{&j, {}, {}, 0});
      gi = int(groups.size()) - 1;
    }
    BatchGroup *g = &groups[gi];
    void *const *pa = static_cast<void *const *>(j.alm);
    void *const *pm = static_cast<void *const *>(j.map);
    g->alm.insert(g->alm.end(), pa, pa + size_t(j.ntrans) * na);
    g->map.insert(g->map.end(), pm, pm + size_t(j.ntrans) * nm);
    g->ntrans += j.ntrans;
    if (group_of) (*group_of)[i] = gi;
  }
  return groups;
}

int execute_batch_impl(const sharp_b200_job *jobs, int njobs, bool device_ptrs,
                       cudaStream_t stream, unsigned long long *opcnt) {
  std::vector<BatchGroup> groups = group_batch(jobs, njobs, device_ptrs, nullptr);
  unsigned long long tot = 0;
  // host arrays: every merged group through one pipelined sequence of pieces
  // (one fill and one drain for the batch) where each group allows it
  bool pipe = !device_ptrs && !groups.empty();
  for (auto &g : groups)
    pipe = pipe && pipelinable(g.first->type, g.first->spin, g.alm.data(), g.map.data(),
                               g.first->geom_info, g.first->alm_info, g.ntrans, g.first->flags);
  if (pipe) {
    std::vector<HostJob> hj;
    for (auto &g : groups)
      hj.push_back(HostJob{g.first->type, g.first->spin, g.alm.data(), g.map.data(),
                           g.first->geom_info, g.first->alm_info, g.ntrans, g.first->flags});
    execute_pipelined_jobs(hj, &tot);
  } else if (device_ptrs && groups.size() > 1) {
    // device arrays: the merged groups run side by side on up to kBatchLanes
    // library streams (forked from and joined back to the caller's stream),
    // so groups of uneven size fill the GPU together; largest groups first,
    // each to the least loaded lane.  The groups write disjoint outputs.
    constexpr int kBatchLanes = 4;
    const int lanes = std::min<int>(kBatchLanes, int(groups.size()));
    std::vector<int> order(groups.size());
    std::iota(order.begin(), order.end(), 0);
    auto cost = [&](int i) {
      const sharp_b200_job &f = *groups[i].first;
      const double l1 = f.alm_info->lmax + 1.0;
      return double(groups[i].ntrans) * l1 * l1 * (f.spin > 0 ? 3.0 : 1.0);
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
    std::vector<double> load(lanes, 0.0);
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join(lanes, nullptr);
    SHT_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    for (auto &e : join) SHT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    SHT_CUDA(cudaEventRecord(fork, stream));
    for (int i = 0; i < lanes; ++i) SHT_CUDA(cudaStreamWaitEvent(copy_stream(2 + i), fork, 0));
    try {
      for (int gi : order) {
        const int lane = int(std::min_element(load.begin(), load.end()) - load.begin());
        load[lane] += cost(gi);
        BatchGroup &g = groups[gi];
        unsigned long long oc = 0;
        execute_impl(g.first->type, g.first->spin, g.alm.data(), g.map.data(),
                     g.first->geom_info, g.first->alm_info, g.ntrans, g.first->flags, true,
                     copy_stream(2 + lane), nullptr, &oc);
        tot += oc;
      }
    } catch (const Failure &) {
      // join what was enqueued before reporting
      for (int i = 0; i < lanes; ++i) {
        cudaEventRecord(join[i], copy_stream(2 + i));
        cudaStreamWaitEvent(stream, join[i], 0);
      }
      cudaEventDestroy(fork);
      for (auto &e : join) cudaEventDestroy(e);
      throw;
    }
    for (int i = 0; i < lanes; ++i) {
      SHT_CUDA(cudaEventRecord(join[i], copy_stream(2 + i)));
      SHT_CUDA(cudaStreamWaitEvent(stream, join[i], 0));
    }
    SHT_CUDA(cudaEventDestroy(fork));
    for (auto &e : join) SHT_CUDA(cudaEventDestroy(e));
  } else {
    for (auto &g : groups) {
      unsigned long long oc = 0;
      execute_impl(g.first->type, g.first->spin, g.alm.data(), g.map.data(), g.first->geom_info,
                   g.first->alm_info, g.ntrans, g.first->flags, device_ptrs, stream, nullptr, &oc);
      tot += oc;
    }
  }
  if (opcnt) *opcnt = tot;
  return int(groups.size());
}

}  // namespace

GeomPlan::~GeomPlan() {
  dev_free(cth); dev_free(sth); dev_free(mlim); dev_free(count); dev_free(items);
  dev_free(mitems);
  dev_free(phi0); dev_free(weight); dev_free(ofs); dev_free(nph); dev_free(stride);
  dev_free(fft); dev_free(fdesc); dev_free(twiddle); dev_free(cls_pairs); dev_free(pw_pairs);
  dev_free(pb_pairs);
  dev_free(bhat); dev_free(wpow2); dev_free(chirp);
}
CoefPlan::~CoefPlan() {
  dev_free(d_moff); dev_free(alpha); dev_free(beta); dev_free(cfac); dev_free(seed);
  dev_free(seed_exp);
  dev_free(mx_coef);
}
AlmPlan::~AlmPlan() { dev_free(mvstart); }

}  // namespace sht

extern "C" {

void sharp_execute(sharp_jobtype type, int spin, void *alm, void *map,
                   const sharp_geom_info *geom_info, const sharp_alm_info *alm_info, int ntrans,
                   int flags, double *time, unsigned long long *opcnt) {
  sht::guarded([&] {
    if (!sht::execute_pipelined(type, spin, alm, map, geom_info, alm_info, ntrans, flags, time,
                                opcnt))
      sht::execute_impl(type, spin, alm, map, geom_info, alm_info, ntrans, flags, false, nullptr,
                        time, opcnt);
  });
}

void sharp_b200_execute_device(sharp_jobtype type, int spin, void *alm, void *map,
                               const sharp_geom_info *geom_info, const sharp_alm_info *alm_info,
                               int ntrans, int flags, void *stream, double *time,
                               unsigned long long *opcnt) {
  sht::guarded([&] {
    sht::execute_impl(type, spin, alm, map, geom_info, alm_info, ntrans, flags, true,
                      static_cast<cudaStream_t>(stream), time, opcnt);
  });
}

int sharp_b200_batch_groups(const sharp_b200_job *jobs, int njobs, int device_ptrs,
                            int *group_of_job) {
  int n = -1;
  sht::guarded([&] {
    std::vector<int> of;
    n = int(sht::group_batch(jobs, njobs, device_ptrs != 0, &of).size());
    if (group_of_job) std::copy(of.begin(), of.end(), group_of_job);
  });
  return n;
}

int sharp_b200_execute_batch(const sharp_b200_job *jobs, int njobs, int device_ptrs,
                             void *stream, unsigned long long *opcnt) {
  int n = -1;
  sht::guarded([&] {
    n = sht::execute_batch_impl(jobs, njobs, device_ptrs != 0,
                                static_cast<cudaStream_t>(stream), opcnt);
  });
  return n;
}

void sharp_b200_forget_geometry(const sharp_geom_info *info) {
  std::lock_guard<std::mutex> lk(sht::g_cache_mutex);
  sht::g_geom_cache.erase(info);
}

void sharp_b200_release_cache(void) {
  std::lock_guard<std::mutex> lk(sht::g_cache_mutex);
  sht::g_geom_cache.clear();
  sht::g_coef_cache.clear();
  sht::g_alm_cache.clear();
  // workspace freed in stream order is unused once the device is idle
  cudaDeviceSynchronize();
  sht::ws_trim();
}

int sharp_b200_check_device_errors(void *stream) {
  int rc = -1;
  sht::guarded([&] {
    SHT_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    sht::check_tc_error();
    rc = 0;
  });
  return rc;
}

int sharp_b200_workspace_bytes(unsigned long long *reserved, unsigned long long *used) {
  if (reserved) *reserved = 0;
  if (used) *used = 0;
  return sht::ws_bytes(reserved, used) ? 0 : -1;
}

}  // extern "C"
