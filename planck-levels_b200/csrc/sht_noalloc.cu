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
// call made with that device current (cudaGetSymbolAddress).  All calls share
// the one array:
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

  // ---- host tables (the same builder as the cached plans) --------------------
  const GeomHost h = build_geom_host(g, lmax, mmax, 0);
  const int np = h.npairs;
  // every size class must run its FFT buffers in shared memory: the
  // global-scratch variant of the ring kernels allocates workspace
  for (int c = 0; c < int(h.cls_N.size()); ++c)
    if (h.cls_count[c] > 0 &&
        sizeof(double2) * ring_fft_smem_entries(h.cls_bufA[c], h.cls_bufB[c], mmax,
                                                h.nmax_complex, h.P) > 227 * 1024) {
      record_error("sharp_b200_alm2map_noalloc: ring lengths above the shared-memory FFT "
                   "limit need workspace; use sharp_b200_execute_device instead");
      return -1;
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
  const size_t o_items = L.take<int2>(h.synth_items.size());
  const size_t o_phi0 = L.take<double>(2 * np), o_weight = L.take<double>(2 * np);
  const size_t o_ofs = L.take<long long>(2 * np);
  const size_t o_nph = L.take<int>(2 * np), o_stride = L.take<int>(2 * np);
  const size_t o_fft = L.take<int>(2 * np);
  const size_t o_fdesc = L.take<FftDesc>(h.descs.size());
  const size_t o_cls = L.take<int>(h.cls_pairs.size());
  const size_t o_pwp = L.take<int>(h.pw_pairs.size());
  const size_t o_twn = L.take<int>(h.tw_n.size()), o_twoff = L.take<int>(h.tw_off.size());
  const size_t o_blue = L.take<int>(h.blue_idx.size());
  const size_t o_blue2 = L.take<int>(h.blue2_idx.size());
  const size_t o_pbp = L.take<int>(h.pb_pairs.size());
  const size_t o_tw = L.take<double2>(h.tw_total);
  const size_t o_wp = L.take<double2>(h.P);
  const size_t o_bhat = L.take<double2>(h.bhat_total);
  const size_t o_chirp = L.take<double2>(h.chirp_total);
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
  put(o_cth, h.cth.data(), sizeof(double) * np);
  put(o_sth, h.sth.data(), sizeof(double) * np);
  put(o_mlim, h.mlim_sorted.data(), sizeof(int) * np);
  put(o_count, h.count_m.data(), sizeof(int) * (mmax + 1));
  put(o_items, h.synth_items.data(), sizeof(int2) * h.synth_items.size());
  put(o_phi0, h.phi0.data(), sizeof(double) * 2 * np);
  put(o_weight, h.weight.data(), sizeof(double) * 2 * np);
  put(o_ofs, h.ofs.data(), sizeof(long long) * 2 * np);
  put(o_nph, h.nph.data(), sizeof(int) * 2 * np);
  put(o_stride, h.stride.data(), sizeof(int) * 2 * np);
  put(o_fft, h.fft.data(), sizeof(int) * 2 * np);
  put(o_fdesc, h.descs.data(), sizeof(FftDesc) * h.descs.size());
  put(o_cls, h.cls_pairs.data(), sizeof(int) * h.cls_pairs.size());
  put(o_pwp, h.pw_pairs.data(), sizeof(int) * h.pw_pairs.size());
  put(o_twn, h.tw_n.data(), sizeof(int) * h.tw_n.size());
  put(o_twoff, h.tw_off.data(), sizeof(int) * h.tw_off.size());
  put(o_blue, h.blue_idx.data(), sizeof(int) * h.blue_idx.size());
  put(o_blue2, h.blue2_idx.data(), sizeof(int) * h.blue2_idx.size());
  put(o_pbp, h.pb_pairs.data(), sizeof(int) * h.pb_pairs.size());
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
      g.fdesc = nullptr; g.twiddle = g.bhat = g.wpow2 = g.chirp = nullptr; g.cls_pairs = nullptr;
      g.pw_pairs = nullptr; g.pb_pairs = nullptr;
      c.d_moff = nullptr; c.alpha = c.beta = c.cfac = c.seed = nullptr; c.seed_exp = nullptr;
      a.mvstart = nullptr;
    }
  } release{gp, cp, ap};
  gp.lmax = lmax; gp.mmax = mmax; gp.spin = 0; gp.npairs = np; gp.nphmax = h.nphmax;
  gp.nmax_complex = h.nmax_complex;
  gp.count_m = h.count_m; gp.synth_items = h.synth_items; gp.synth_tile = h.synth_tile;
  gp.cth = static_cast<double *>(at(o_cth)); gp.sth = static_cast<double *>(at(o_sth));
  gp.mlim = static_cast<int *>(at(o_mlim)); gp.count = static_cast<int *>(at(o_count));
  gp.items = static_cast<int2 *>(at(o_items));
  gp.phi0 = static_cast<double *>(at(o_phi0)); gp.weight = static_cast<double *>(at(o_weight));
  gp.ofs = static_cast<long long *>(at(o_ofs));
  gp.nph = static_cast<int *>(at(o_nph)); gp.stride = static_cast<int *>(at(o_stride));
  gp.fft = static_cast<int *>(at(o_fft)); gp.fdesc = static_cast<FftDesc *>(at(o_fdesc));
  gp.twiddle = static_cast<double2 *>(at(o_tw)); gp.wpow2 = static_cast<double2 *>(at(o_wp));
  gp.bhat = static_cast<double2 *>(at(o_bhat)); gp.P = h.P;
  gp.chirp = static_cast<double2 *>(at(o_chirp));
  gp.cls_N = h.cls_N; gp.cls_start = h.cls_start; gp.cls_count = h.cls_count;
  gp.cls_bufA = h.cls_bufA; gp.cls_bufB = h.cls_bufB;
  gp.cls_pairs = static_cast<int *>(at(o_cls));
  gp.pw_N = h.pw_N; gp.pw_start = h.pw_start; gp.pw_count = h.pw_count;
  gp.pw_pairs = static_cast<int *>(at(o_pwp));
  gp.pb_M = h.pb_M; gp.pb_start = h.pb_start; gp.pb_count = h.pb_count;
  gp.pb_pairs = static_cast<int *>(at(o_pbp));
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
                            static_cast<int *>(at(o_twoff)), int(h.tw_n.size()), st);
  // power-of-two table exp(-2 pi i j/P) of the Bluestein passes
  const int pw[2] = {h.P, 0};  // length, offset
  put(o_pw, pw, sizeof(pw));
  launch_twiddles_preplaced(gp.wpow2, static_cast<int *>(at(o_pw)),
                            static_cast<int *>(at(o_pw)) + 1, 1, st);
  launch_bluestein_setup_preplaced(gp, static_cast<int *>(at(o_blue)), int(h.blue_idx.size()),
                                   static_cast<int *>(at(o_blue2)), int(h.blue2_idx.size()),
                                   st);
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
