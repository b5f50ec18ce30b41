// Allocation-free spin-0 synthesis (sharp_b200_alm2map_noalloc).
//
// Some callers cannot call cudaMalloc at the time they need a transform: the
// GPU memory of their process belongs to another allocator (a framework's
// caching pool, a fixed arena reserved at start-up) or they run under a
// policy that forbids allocation once initialised.  This entry point serves
// them: every device buffer the transform needs (geometry and recurrence
// tables, FFT twiddles, staged a_lm, phase array) is carved out of one
// file-scope __device__ array of kNoAllocScratchBytes, which every GPU that
// loads the library holds until process exit.  The caller passes the a_lm
// and the map as device pointers.  No cudaMalloc, cudaFree or allocating
// library routine is called, so no plan is cached either: the tables are
// rebuilt on every call.
//
// The symbol address of the array is looked up once per device, on the first
// call made with that device current (cudaGetSymbolAddress); that first call
// should come before any stream capture.  All calls share the one array:
// calls that overlap on the GPU (different streams, or host threads calling
// concurrently) race on it and must be serialised by the caller.  Each call
// rewrites every part of the array it reads before reading it, so the
// contents left by an earlier call are never used.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <vector>

#include "sht_device.h"

namespace sht {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mutex;
void *g_scratch_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch for the current device (looked up once
// per device, with that device current).
void *scratch_base() {
  int dev = 0;
  SHT_CUDA(cudaGetDevice(&dev));
  SHT_REQUIRE(dev >= 0 && dev < kMaxDevices, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mutex);
  if (!g_scratch_addr[dev]) {
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    SHT_CUDA(e);
    g_scratch_addr[dev] = ptr;
  }
  return g_scratch_addr[dev];
}

// Bump layout of the scratch array (256-byte aligned pieces).
struct Layout {
  size_t used = 0;
  template <typename T>
  size_t take(size_t count) {
    const size_t off = used;
    used += (sizeof(T) * std::max<size_t>(count, 1) + 255) & ~size_t(255);
    return off;
  }
};

std::vector<int> factors(int N) {
  std::vector<int> r;
  int n = N;
  while (n % 4 == 0) { r.push_back(4); n /= 4; }
  while (n % 2 == 0) { r.push_back(2); n /= 2; }
  for (int p = 3; n > 1; p += 2)
    while (n % p == 0) { r.push_back(p); n /= p; }
  return r;
}

int alm2map_noalloc(const sharp_geom_info *g, const sharp_alm_info *a, const void *alm,
                    void *map, cudaStream_t st) {
  SHT_REQUIRE(g != nullptr && a != nullptr && alm != nullptr && map != nullptr,
              "null argument");
  SHT_REQUIRE(!(a->flags & SHARP_PACKED), "SHARP_PACKED a_lm are not supported here");
  const int nm = a->nm, lmax = a->lmax, mmax = nm - 1;
  {
    std::vector<char> seen(std::max(nm, 1), 0);
    for (int i = 0; i < nm; ++i) {
      const int mv = a->mval[i];
      SHT_REQUIRE(mv >= 0 && mv < nm, "not all m values are present");
      SHT_REQUIRE(!seen[mv], "duplicate m value");
      seen[mv] = 1;
    }
  }
  SHT_REQUIRE(mmax <= lmax, "incorrect l_max: must be >= m_max");

  // ---- host tables: pairs in decreasing mlim order -------------------------
  const int np = g->npairs;
  std::vector<int> mlim(np), order(np);
  for (int i = 0; i < np; ++i) mlim[i] = get_mlim(lmax, 0, g->pair[i].r1.sth, g->pair[i].r1.cth);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return mlim[x] > mlim[y]; });
  std::vector<int> count(mmax + 1, 0), hist(mmax + 1, 0);
  for (int i = 0; i < np; ++i)
    if (mlim[i] >= 0) hist[std::min(mlim[i], mmax)] += 1;
  for (int m = mmax, run = 0; m >= 0; --m) count[m] = (run += hist[m]);
  const int tile = 256;
  std::vector<int2> items;
  for (int m = 0; m <= mmax; ++m)
    for (int t = 0; t * tile < count[m]; ++t) items.push_back({m, t});

  std::vector<double> cth(np), sth(np), phi0(2 * np), weight(2 * np);
  std::vector<int> mls(np), nph(2 * np), stride(2 * np), fft(2 * np, 0);
  std::vector<long long> ofs(2 * np);
  std::map<int, int> len_index;
  std::vector<FftDesc> descs;
  std::vector<int> tw_n, tw_off, blue_idx;
  long long tw_total = 0, bhat_total = 0;
  int P = 2;
  for (int p = 0; p < np; ++p) {
    const sharp_ringpair &pr = g->pair[order[p]];
    cth[p] = pr.r1.cth;
    sth[p] = pr.r1.sth;
    mls[p] = mlim[order[p]];
    for (int h = 0; h < 2; ++h) {
      const sharp_ringinfo &r = h ? pr.r2 : pr.r1;
      const int i = 2 * p + h;
      const bool present = (h == 0) || r.nph > 0;
      nph[i] = present ? r.nph : -1;
      phi0[i] = present ? r.phi0 : 0.0;
      weight[i] = present ? r.weight : 0.0;
      ofs[i] = present ? r.ofs : 0;
      stride[i] = present ? r.stride : 1;
      if (!present || r.nph <= 0) continue;
      auto it = len_index.find(r.nph);
      if (it == len_index.end()) {
        FftDesc d{};
        d.n = r.nph;
        d.N = (r.nph & 1) ? r.nph : r.nph / 2;
        d.tw = int(tw_total);
        const auto rad = factors(d.N);
        SHT_REQUIRE(int(rad.size()) <= kMaxRadices, "ring length has too many factors");
        d.nrad = int(rad.size());
        for (int k = 0; k < d.nrad; ++k) d.rad[k] = rad[k];
        long long direct = 0;
        for (int rr : rad) direct += (rr > 5) ? rr : 1;
        direct *= d.N;
        int M = 1, lg = 0;
        while (M < 2 * d.N - 1) { M <<= 1; ++lg; }
        d.blue = (d.N > 16 && 2ll * ((long long)M * lg + 2ll * d.N) < direct) ? 1 : 0;
        d.M = d.blue ? M : 0;
        d.bhat = 0;
        if (d.blue) {
          d.bhat = bhat_total;
          bhat_total += M;
          P = std::max(P, M);
          blue_idx.push_back(int(descs.size()));
        }
        tw_n.push_back(d.n);
        tw_off.push_back(int(tw_total));
        tw_total += d.n;
        it = len_index.emplace(r.nph, int(descs.size())).first;
        descs.push_back(d);
      }
      fft[i] = it->second;
    }
  }
  // FFT size classes
  const int bounds[4] = {256, 1024, 4096, 1 << 30};
  std::vector<std::vector<int>> lists(4);
  for (int p = 0; p < np; ++p) {
    int nmx = 0;
    for (int h = 0; h < 2; ++h)
      if (nph[2 * p + h] > 0) nmx = std::max(nmx, descs[fft[2 * p + h]].N);
    int c = 0;
    while (c < 3 && nmx > bounds[c]) ++c;
    lists[c].push_back(p);
  }
  std::vector<int> flat, cls_N, cls_start, cls_count, cls_bufA, cls_bufB;
  int nmax_all = 1;
  for (const FftDesc &d : descs) nmax_all = std::max(nmax_all, d.N);
  for (int c = 0; c < 4; ++c) {
    int bufA = 2, bufB = 2, nmaxc = 1;
    for (int p : lists[c])
      for (int h = 0; h < 2; ++h)
        if (nph[2 * p + h] > 0) {
          const FftDesc &d = descs[fft[2 * p + h]];
          bufA = std::max(bufA, d.blue ? std::max(d.M, d.N + 2) : d.N + 2);
          bufB = std::max(bufB, d.N + 2);
          nmaxc = std::max(nmaxc, d.N);
        }
    cls_N.push_back(std::min(bounds[c], std::max(nmaxc, 1)));
    bufA = (bufA + 7) & ~7;   // whole blocks of 8 (swizzled in the ring kernels)
    bufB = (bufB + 7) & ~7;
    cls_bufA.push_back(bufA);
    cls_bufB.push_back(bufB);
    cls_start.push_back(int(flat.size()));
    cls_count.push_back(int(lists[c].size()));
    flat.insert(flat.end(), lists[c].begin(), lists[c].end());
    SHT_REQUIRE(sizeof(double2) * ring_fft_smem_entries(bufA, bufB, mmax, nmax_all, P) <=
                    227 * 1024,
                "ring length exceeds the shared-memory FFT limit");
  }
  // recurrence tables
  std::vector<long long> moff(mmax + 2);
  long long off = 0;
  for (int m = 0; m <= mmax; ++m) {
    moff[m] = off;
    off += (lmax - m + 1) + kPad;
  }
  moff[mmax + 1] = off;
  std::vector<double> mfac(mmax + 1);
  mfac[0] = 0.2820947917738781434740397257803862929220;  // 1/sqrt(4 pi)
  for (int m = 1; m <= mmax; ++m) mfac[m] = mfac[m - 1] * std::sqrt((2 * m + 1.) / (2 * m));
  std::vector<long long> mvstart(mmax + 1, 0);
  for (int mi = 0; mi < nm; ++mi) mvstart[a->mval[mi]] = a->mvstart[mi];
  std::vector<double> norm(lmax + 1, 1.0);

  // ---- scratch layout --------------------------------------------------------
  Layout L;
  const size_t o_cth = L.take<double>(np), o_sth = L.take<double>(np);
  const size_t o_mlim = L.take<int>(np), o_count = L.take<int>(mmax + 1);
  const size_t o_items = L.take<int2>(items.size());
  const size_t o_phi0 = L.take<double>(2 * np), o_weight = L.take<double>(2 * np);
  const size_t o_ofs = L.take<long long>(2 * np);
  const size_t o_nph = L.take<int>(2 * np), o_stride = L.take<int>(2 * np);
  const size_t o_fft = L.take<int>(2 * np);
  const size_t o_fdesc = L.take<FftDesc>(descs.size());
  const size_t o_cls = L.take<int>(flat.size());
  const size_t o_twn = L.take<int>(tw_n.size()), o_twoff = L.take<int>(tw_off.size());
  const size_t o_blue = L.take<int>(blue_idx.size());
  const size_t o_tw = L.take<double2>(tw_total);
  const size_t o_wp = L.take<double2>(P);
  const size_t o_bhat = L.take<double2>(bhat_total);
  const size_t o_moff = L.take<long long>(mmax + 2);
  const size_t o_alpha = L.take<double>(off), o_cfac = L.take<double>(off);
  const size_t o_mfac = L.take<double>(mmax + 1);
  const size_t o_mvs = L.take<long long>(mmax + 1);
  const size_t o_norm = L.take<double>(lmax + 1);
  const size_t o_ptr = L.take<void *>(2);
  const size_t o_pw = L.take<int>(2);
  const size_t o_A = L.take<double2>(off);
  const size_t o_phase = L.take<double2>(size_t(2) * (mmax + 1) * std::max(np, 1));
  if (L.used > kNoAllocScratchBytes) {
    record_error("sharp_b200_alm2map_noalloc: this geometry and lmax need " +
                 std::to_string(L.used >> 20) + " MiB of scratch, above the fixed " +
                 std::to_string(kNoAllocScratchBytes >> 20) +
                 " MiB of the allocation-free path; use sharp_b200_execute_device instead");
    return -1;
  }
  auto *base = static_cast<unsigned char *>(scratch_base());
  auto at = [&](size_t o) { return static_cast<void *>(base + o); };
  auto put = [&](size_t o, const void *src, size_t bytes) {
    if (bytes) SHT_CUDA(cudaMemcpyAsync(at(o), src, bytes, cudaMemcpyHostToDevice, st));
  };
  put(o_cth, cth.data(), sizeof(double) * np);
  put(o_sth, sth.data(), sizeof(double) * np);
  put(o_mlim, mls.data(), sizeof(int) * np);
  put(o_count, count.data(), sizeof(int) * (mmax + 1));
  put(o_items, items.data(), sizeof(int2) * items.size());
  put(o_phi0, phi0.data(), sizeof(double) * 2 * np);
  put(o_weight, weight.data(), sizeof(double) * 2 * np);
  put(o_ofs, ofs.data(), sizeof(long long) * 2 * np);
  put(o_nph, nph.data(), sizeof(int) * 2 * np);
  put(o_stride, stride.data(), sizeof(int) * 2 * np);
  put(o_fft, fft.data(), sizeof(int) * 2 * np);
  put(o_fdesc, descs.data(), sizeof(FftDesc) * descs.size());
  put(o_cls, flat.data(), sizeof(int) * flat.size());
  put(o_twn, tw_n.data(), sizeof(int) * tw_n.size());
  put(o_twoff, tw_off.data(), sizeof(int) * tw_off.size());
  put(o_blue, blue_idx.data(), sizeof(int) * blue_idx.size());
  put(o_moff, moff.data(), sizeof(long long) * (mmax + 2));
  put(o_mfac, mfac.data(), sizeof(double) * (mmax + 1));
  put(o_mvs, mvstart.data(), sizeof(long long) * (mmax + 1));
  put(o_norm, norm.data(), sizeof(double) * (lmax + 1));
  const void *ptrs[2] = {alm, map};
  put(o_ptr, ptrs, sizeof(ptrs));

  // ---- non-owning plan views over the scratch array --------------------------
  GeomPlan gp;
  CoefPlan cp;
  AlmPlan ap;
  struct Release {  // the views must not free scratch pieces
    GeomPlan &g;
    CoefPlan &c;
    AlmPlan &a;
    ~Release() {
      g.cth = g.sth = nullptr; g.mlim = g.count = nullptr; g.items = nullptr;
      g.phi0 = g.weight = nullptr; g.ofs = nullptr; g.nph = g.stride = g.fft = nullptr;
      g.fdesc = nullptr; g.twiddle = g.bhat = g.wpow2 = nullptr; g.cls_pairs = nullptr;
      c.d_moff = nullptr; c.alpha = c.beta = c.cfac = c.seed = nullptr; c.seed_exp = nullptr;
      a.mvstart = nullptr;
    }
  } release{gp, cp, ap};
  gp.lmax = lmax; gp.mmax = mmax; gp.spin = 0; gp.npairs = np; gp.nphmax = g->nphmax;
  gp.nmax_complex = nmax_all;
  gp.count_m = count; gp.synth_items = items; gp.synth_tile = tile;
  gp.cth = static_cast<double *>(at(o_cth)); gp.sth = static_cast<double *>(at(o_sth));
  gp.mlim = static_cast<int *>(at(o_mlim)); gp.count = static_cast<int *>(at(o_count));
  gp.items = static_cast<int2 *>(at(o_items));
  gp.phi0 = static_cast<double *>(at(o_phi0)); gp.weight = static_cast<double *>(at(o_weight));
  gp.ofs = static_cast<long long *>(at(o_ofs));
  gp.nph = static_cast<int *>(at(o_nph)); gp.stride = static_cast<int *>(at(o_stride));
  gp.fft = static_cast<int *>(at(o_fft)); gp.fdesc = static_cast<FftDesc *>(at(o_fdesc));
  gp.twiddle = static_cast<double2 *>(at(o_tw)); gp.wpow2 = static_cast<double2 *>(at(o_wp));
  gp.bhat = static_cast<double2 *>(at(o_bhat)); gp.P = P;
  gp.cls_N = cls_N; gp.cls_start = cls_start; gp.cls_count = cls_count;
  gp.cls_bufA = cls_bufA; gp.cls_bufB = cls_bufB;
  gp.cls_pairs = static_cast<int *>(at(o_cls));
  cp.lmax = lmax; cp.mmax = mmax; cp.spin = 0; cp.total = off; cp.moff = moff;
  cp.d_moff = static_cast<long long *>(at(o_moff));
  cp.alpha = static_cast<double *>(at(o_alpha)); cp.cfac = static_cast<double *>(at(o_cfac));
  cp.seed = static_cast<double *>(at(o_mfac));
  ap.lmax = lmax; ap.mmax = mmax; ap.packed = false; ap.stride = a->stride;
  ap.mvstart = static_cast<long long *>(at(o_mvs));

  JobDesc job{};
  job.type = SHARP_ALM2MAP; job.spin = 0; job.nmaps = 1; job.nalm = 1; job.ntrans = 1;
  job.flags = SHARP_DP; job.lmax = lmax; job.mmax = mmax; job.dp = true;

  // ---- the transform ---------------------------------------------------------
  launch_twiddles_preplaced(gp.twiddle, static_cast<int *>(at(o_twn)),
                            static_cast<int *>(at(o_twoff)), int(tw_n.size()), st);
  // power-of-two table exp(-2 pi i j/P) of the Bluestein passes
  const int pw[2] = {P, 0};  // length, offset
  put(o_pw, pw, sizeof(pw));
  launch_twiddles_preplaced(gp.wpow2, static_cast<int *>(at(o_pw)),
                            static_cast<int *>(at(o_pw)) + 1, 1, st);
  launch_bluestein_setup_preplaced(gp, static_cast<int *>(at(o_blue)), int(blue_idx.size()), st);
  launch_coef_tables(cp, st);
  auto *ptr_dev = static_cast<void *const *>(at(o_ptr));
  launch_stage_alm(job, ap, 0, cp, static_cast<double *>(at(o_norm)), ptr_dev, 1,
                   static_cast<double2 *>(at(o_A)), 1, st);
  launch_legendre_synth(job, gp, cp, static_cast<double2 *>(at(o_A)), 1, 0, 1,
                        static_cast<double2 *>(at(o_phase)), 1, 0, st);
  launch_phase2ring(job, gp, 0, static_cast<double2 *>(at(o_phase)), 1, ptr_dev + 1, 1, st);
  return 0;
}

}  // namespace
}  // namespace sht

extern "C" int sharp_b200_alm2map_noalloc(const sharp_geom_info *geom_info,
                                          const sharp_alm_info *alm_info, const void *alm,
                                          void *map, void *stream) {
  try {
    return sht::alm2map_noalloc(geom_info, alm_info, alm, map,
                                static_cast<cudaStream_t>(stream));
  } catch (const sht::Failure &) {
    return -1;
  }
}
