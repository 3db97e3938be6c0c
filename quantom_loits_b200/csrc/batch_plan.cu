// batch_plan.cu -- host side of the batched sampler: plans, workspace layout,
// launches (persistent and one-launch-per-density), CDF export, quantiles.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include <cuda_runtime.h>

#include "batch_kernels.cuh"

namespace loits_dev {
template <int TPB, int R, bool kLarge>
__global__ void batch_forward_kernel(BatchArgs a);
template <int TPB, int R, bool kLarge, bool kFix>
__global__ void batch_backward_kernel(BatchArgs a, double* grho);
__global__ void batch_cdf_export_kernel(const float4* rec, int64_t n, double* cdf);
__global__ void batch_quantile_kernel(const float4* rec, const uint32_t* guide, int m, int G,
                                      bool count_all, const float* u, int64_t n, float* x,
                                      int32_t* intervals);
}  // namespace loits_dev

// template definitions: batch_kernels_impl.cuh, instantiated in batch_inst_*.cu

using namespace loits_dev;

namespace {

constexpr size_t kAlign = 256;
size_t align_up(size_t v, size_t a = kAlign) { return (v + a - 1) / a * a; }

struct Layout {
  size_t status, tickets_fwd, dflags, cdf_ready, cdf_scanned, fin_done, cflag, tile_state;  // zeroed by forward
  size_t tickets_bwd, chunks_done, lfin_done, lflag, gcdf;                        // zeroed by backward
  size_t rec, invd, gl, gpk, norm, kstar, cagg, cinc, cmax, tile_prefix, warp_off, stage, partials,
      grho;
  size_t lagg, linc, lgn;
  size_t fwd_zero_lo, fwd_zero_hi, bwd_zero_lo, bwd_zero_hi, total;
};

}  // namespace

struct loits_batch_plan {
  int64_t nd = 0;
  std::vector<int64_t> koff, nev;
  int64_t nmax = 0, capacity = 0, total_knots = 0, max_g = 0, small_max_g = 0, dbase = 0;
  loits_batch_config cfg{};
  int tpb = 256, r = 4, scan_knots = 8;
  int32_t n_tiles = 0, n_cdf = 0, n_fin = 0, n_chunks = 0, last_nonempty = -1;
  int32_t gcap = 0, mcap = 0, tiles_per_chunk = 1, n_lfin = 0, m_cap_b = 2;
  int32_t lbits_f = 0, lbits_b = 0;  // coarse large-density guide bits in shared memory
  bool fix_small = false;             // backward slot sized for fixed-point sums of gcap knots
  bool fix_used = false;              // backward variant with the fixed-point small path
  int32_t win_n = 0, bwd_guide_off = 0;  // backward: large-density window, guide offset
  int32_t fwin_n = 0, fwd_guide_off = 0;  // forward: large-density window, guide offset
  bool has_large = false;  // densities above the shared-memory limit
  int64_t total_partials = 0, total_guide = 0, total_pk = 0, total_gc = 0;
  std::vector<int32_t> tile_first, cdf_first, fin_first, chunk_first, rowfill_lo, gbits;
  std::vector<int32_t> tile_r, scan_k;  // per density: blocks per thread per tile, CDF width
  std::vector<int32_t> tile_owner, cdf_owner, chunk_owner;  // density of each item
  std::vector<int64_t> part_off, goff, pkoff, gc_off;
  std::vector<int32_t> lfin_first;
  void* dtab = nullptr;
  const int64_t *d_koff = nullptr, *d_nev = nullptr, *d_part_off = nullptr, *d_goff = nullptr,
                *d_pkoff = nullptr, *d_gc_off = nullptr;
  const int32_t* d_lfin_first = nullptr;
  const int32_t *d_tile_first = nullptr, *d_cdf_first = nullptr, *d_fin_first = nullptr,
                *d_chunk_first = nullptr, *d_rowfill_lo = nullptr, *d_gbits = nullptr,
                *d_tile_r = nullptr, *d_scan_k = nullptr, *d_tile_owner = nullptr,
                *d_cdf_owner = nullptr, *d_chunk_owner = nullptr;
  Layout lay{};
  size_t fwd_smem = 0, bwd_smem = 0;
  // dynamic shared memory already allowed for the kernels (histogram mode
  // launches with more; raised once, so that later launches -- and CUDA
  // graph captures -- make no attribute calls)
  mutable size_t fwd_smem_allowed = 0, bwd_smem_allowed = 0;
  int fwd_grid = 1, bwd_grid = 1, num_sms = 148;
};

namespace {

using FwdKernel = void (*)(BatchArgs);
using BwdKernel = void (*)(BatchArgs, double*);

template <int TPB, int R>
void pick(bool large, bool fix, FwdKernel& f, BwdKernel& b) {
  constexpr bool kFixOK = TPB >= 512;  // fixed-point paths: 512- and 1024-thread CTAs
  if (large) {
    f = batch_forward_kernel<TPB, R, true>;
    b = batch_backward_kernel<TPB, R, true, false>;
    if constexpr (kFixOK) if (fix) b = batch_backward_kernel<TPB, R, true, true>;
  } else {
    f = batch_forward_kernel<TPB, R, false>;
    b = batch_backward_kernel<TPB, R, false, false>;
    if constexpr (kFixOK) if (fix) b = batch_backward_kernel<TPB, R, false, true>;
  }
}

// Kernels of a launch geometry; `large`: the plan has densities above the
// shared-memory limit; `fix`: small densities that sum in fixed point (the
// backward variant with that path; 512- and 1024-thread CTAs).
bool kernels_for(int tpb, int r, bool large, FwdKernel& f, BwdKernel& b, bool fix = false) {
  if (tpb == 256) {
    switch (r) {
      case 2: pick<256, 2>(large, fix, f, b); return true;
      case 4: pick<256, 4>(large, fix, f, b); return true;
      case 8: pick<256, 8>(large, fix, f, b); return true;
      case 16: pick<256, 16>(large, fix, f, b); return true;
    }
  } else if (tpb == 512) {
    switch (r) {
      case 2: pick<512, 2>(large, fix, f, b); return true;
      case 4: pick<512, 4>(large, fix, f, b); return true;
      case 8: pick<512, 8>(large, fix, f, b); return true;
      case 16: pick<512, 16>(large, fix, f, b); return true;
    }
  } else if (tpb == 1024) {
    switch (r) {
      case 2: pick<1024, 2>(large, fix, f, b); return true;
      case 4: pick<1024, 4>(large, fix, f, b); return true;
      case 8: pick<1024, 8>(large, fix, f, b); return true;
      case 16: pick<1024, 16>(large, fix, f, b); return true;
    }
  }
  return false;
}

// Largest number of knots a sampling CTA holds in shared memory; densities
// with more knots are sampled from global memory.
constexpr int64_t kMaxSmemKnots = 8192;
// Largest density (knot indices are int32).
constexpr int64_t kMaxKnots = int64_t(1) << 28;
// A large density's guide has at most 2^18 buckets: where u is likely the
// knots are far apart in u, and the rarely hit buckets of the flat tails
// (holding many knots) are finished by a short search.
constexpr int kMaxLargeGuideBits = 18;
constexpr size_t kSmemLimit = 227 * 1024;

int default_blocks(int threads) { return threads == 1024 ? 8 : 16; }

// Guide buckets per knot of a small density, as log2: M >= 2^ratio G buckets
// where shared memory allows without lowering the CTAs an SM holds.  Finer
// buckets hold fewer knots, so fewer slots need more than one key compare
// (about 1 % of the benchmark densities' slots search with 4 G buckets,
// 3 % with 2 G), but cost more shared memory to copy per tile; 4 G measured
// fastest on the uniform and ragged benchmark batches.
constexpr int kDefaultGuideRatio = 2;
constexpr int kMaxGuideRatio = 6;
// Most guide bits a small density's packed guide takes in shared memory.
constexpr int kMaxSmallGuideBits = 15;

// Validates a configuration; threads == 0 (choose by occupancy) and
// blocks_per_item == 0 (default for the thread count) stay unresolved.
int resolve_config(const loits_batch_config* in, loits_batch_config& out) {
  out = in ? *in : loits_batch_config{};
  if (out.scan_knots == 0) out.scan_knots = 8;
  if (out.threads != 0 && out.threads != 256 && out.threads != 512 && out.threads != 1024)
    return LOITS_ERR_INVALID;
  if (out.blocks_per_item != 0 && out.blocks_per_item != 2 && out.blocks_per_item != 4 &&
      out.blocks_per_item != 8 && out.blocks_per_item != 16)
    return LOITS_ERR_INVALID;
  if (out.scan_knots < 1 || out.scan_knots > 64) return LOITS_ERR_INVALID;
  if (out.ctas_per_sm < 0 || out.ctas_per_sm > 32) return LOITS_ERR_INVALID;
  if (out.plain != 0 && out.plain != 1) return LOITS_ERR_INVALID;
  if (out.guide_ratio < 0 || out.guide_ratio > kMaxGuideRatio) return LOITS_ERR_INVALID;
  if (out.guide_ratio == 0) out.guide_ratio = kDefaultGuideRatio;
  if (out.wait_limit < 0 || out.withhold_tile < 0) return LOITS_ERR_INVALID;
  if (out.density_base < 0 || out.slot_stride < 0) return LOITS_ERR_INVALID;
  return LOITS_OK;
}

// Raise a kernel's dynamic shared-memory limit to at least `bytes`.  The
// limit is a property of the function shared by every plan, so it only ever
// grows: a plan built later with smaller densities must not lower it below
// what an earlier plan launches with.
bool allow_dynamic_smem(const void* fn, size_t bytes) {
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  cudaFuncAttributes now{};
  if (cudaFuncGetAttributes(&now, fn) != cudaSuccess) return false;
  if (static_cast<size_t>(now.maxDynamicSharedSizeBytes) >= bytes) return true;
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              static_cast<int>(bytes)) == cudaSuccess;
}

// Shared memory of the sampling kernels of (tpb, r) for small densities of at
// most max_g knots (gcap rounded to 4): the guide caps, the largest guide
// (mcap entries) and the dynamic bytes of the forward and backward CTAs.
struct SmemGeometry {
  int m_cap = 2;    // forward: log2 of the most guide buckets beside the records
  int m_cap_b = 2;  // backward: the same beside records, weights and gradients
  int lbits_f = 0;  // large densities: log2 of the coarse guide a forward CTA holds
  int lbits_b = 0;  // ... and a backward CTA
  bool fix_small = false;   // backward slot sized for fixed-point sums of gcap knots
  int32_t win_n = 0;        // backward: large densities' fixed-point window (intervals)
  int32_t bwd_guide_off = 0;  // backward: uint32 words before the guide
  int32_t fwin_n = 0;       // forward: large densities' window of records
  int32_t fwd_guide_off = 0;  // forward: uint32 words before the guide
  int32_t mcap = 0;
  size_t static_smem = 0, fwd = 0, bwd = 0;
};

// Shared memory of one SM, and what the driver reserves per resident CTA.
constexpr size_t kSmemPerSM = 228 * 1024;
constexpr size_t kSmemPerCtaReserved = 1024;

// Guide bits of a density of g knots: M = 2^m buckets, 2^ratio g <= M, at
// most 2^cap.
int guide_bits(int64_t g, int cap, int ratio) {
  int m = 2;
  while ((int64_t(1) << m) < (g << ratio) && m < cap) ++m;
  return m;
}

// large_g: knots of the largest density above the shared-memory limit (0: none).
int smem_geometry(int tpb, int r, int64_t large_g, int32_t gcap, int64_t max_g, int ratio,
                  SmemGeometry& g) {
  const bool large = large_g > 0;
  FwdKernel fk;
  BwdKernel bk;
  if (!kernels_for(tpb, r, large, fk, bk)) return LOITS_ERR_INVALID;
  cudaFuncAttributes fattr{}, battr{};
  if (cudaFuncGetAttributes(&fattr, fk) != cudaSuccess ||
      cudaFuncGetAttributes(&battr, bk) != cudaSuccess)
    return LOITS_ERR_CUDA;
  g.static_smem = std::max(fattr.sharedSizeBytes, battr.sharedSizeBytes);
  // a forward CTA holds per knot a record (16 bytes), a backward CTA also a
  // weight and a gradient slot (24 bytes); each beside the density's guide
  const size_t fwd_knots = static_cast<size_t>(gcap) * sizeof(float4);
  const size_t bwd_knots = static_cast<size_t>(gcap) * (sizeof(float4) + 2 * sizeof(float));
  if (bwd_knots + g.static_smem + 64 * sizeof(uint32_t) > kSmemLimit) return LOITS_ERR_UNSUPPORTED;
  // guide tables: M = 2^m buckets per density, 2G <= M < 4G, at most 2^14 and
  // at most what the forward's shared memory leaves beside the records (a
  // smaller guide only widens buckets: the search finishes them exactly).
  // The backward reads every 2^s-th count when its budget is smaller: the
  // same guide with 2^s-times wider buckets.
  // forward and backward CTAs hold a small density's packed guide (8 bytes
  // per bucket: the entry and the key its first compare needs)
  constexpr size_t kFwdEntry = sizeof(uint2), kBwdEntry = sizeof(uint2);
  auto cap_for = [&](size_t knot_bytes, int from, size_t entry) {
    int mc = from;
    while (mc > 2 && knot_bytes + g.static_smem + (size_t(1) << mc) * entry > kSmemLimit) --mc;
    return mc;
  };
  g.m_cap = cap_for(fwd_knots, kMaxSmallGuideBits, kFwdEntry);
  g.m_cap_b = cap_for(bwd_knots, kMaxSmallGuideBits, kBwdEntry);
  // guide bytes of `entries` buckets (8-byte entries, rounded up to 8 entries);
  // kept events are staged in global memory, not here
  auto gbytes = [](int32_t entries) { return static_cast<size_t>((entries + 7) & ~7) * sizeof(uint2); };
  auto fbytes = [&](int32_t entries) { return gbytes(entries); };
  // CTAs per SM that `bytes` of dynamic shared memory allow (at most the
  // register cap's 1280 / tpb)
  auto resident = [&](size_t bytes) {
    size_t c = static_cast<size_t>(std::max(1, 1280 / tpb));
    while (c > 1 && c * (bytes + g.static_smem + kSmemPerCtaReserved) > kSmemPerSM) --c;
    return c;
  };
  // the largest small density's guide: 2^ratio buckets per knot, unless that
  // holds fewer CTAs per SM than 2 buckets per knot would (in the forward
  // with records beside it; in the backward with records, weights and sums)
  const int m1 = guide_bits(max_g, g.m_cap, 1);
  int m = guide_bits(max_g, g.m_cap, ratio);
  while (m > m1 && resident(fwd_knots + fbytes(1 << m)) < resident(fwd_knots + fbytes(1 << m1))) --m;
  g.m_cap = m;  // every small density's guide takes at most this many bits
  g.mcap = static_cast<int32_t>(int64_t(1) << m);
  const int mb1 = std::min(g.m_cap_b, m1);
  int mb = std::min(g.m_cap_b, m);
  const size_t bwd_fix = static_cast<size_t>(gcap) * (sizeof(float4) + 5 * sizeof(float));
  while (mb > mb1 && resident(std::max(bwd_knots, tpb >= 512 ? bwd_fix : 0) + gbytes(1 << mb)) <
                         resident(std::max(bwd_knots, tpb >= 512 ? bwd_fix : 0) + gbytes(1 << mb1)))
    --mb;
  g.m_cap_b = mb;
  const int32_t mcap_b = std::min<int32_t>(g.mcap, int32_t(1) << g.m_cap_b);
  const size_t guide_f = fbytes(g.mcap);
  size_t guide_b = gbytes(mcap_b);
  // Backward small-density slot: records, weights and either fp32 grad-CDF
  // sums (4 bytes per knot) or the fixed-point sums A, B (16 bytes per
  // knot).  Fixed point is used when it costs neither residency nor guide
  // resolution (a coarser backward guide measured slower than the fp32 sums).
  size_t small_b = bwd_knots;
  {
    const size_t fix_knots = static_cast<size_t>(gcap) * (sizeof(float4) + 5 * sizeof(float));
    if (tpb >= 512 && fix_knots + guide_b + g.static_smem + 16 * 1024 <= kSmemLimit &&
        resident(fix_knots + guide_b) >= resident(bwd_knots + guide_b)) {
      g.fix_small = true;
      small_b = fix_knots;
    }
  }
  size_t before_guide = small_b;
  if (large) {
    // backward CTAs of large densities (records in global memory) read a
    // coarse copy of the guide (every 2^s-th count, 2^lbits + 1 uint32) from
    // shared memory and sum the most probable run of intervals (the window)
    // in fixed point where small densities keep their records; both sized
    // not to lower the residency the register cap allows and to leave room
    // for a histogram-mode cotangent (16 KB).  The forward reads the full
    // guide through L2 (lbits_f = 0), which measured faster than the coarser
    // buckets' longer searches.
    auto bytes = [](int b) { return ((size_t(1) << b) + 1 + 7) / 8 * 8 * sizeof(uint32_t); };
    const size_t ctas = resident(small_b + bytes(6));
    const size_t per_cta = std::min(kSmemPerSM / ctas - kSmemPerCtaReserved, kSmemLimit);
    const size_t avail = per_cta > g.static_smem + 16 * 1024 ? per_cta - g.static_smem - 16 * 1024 : 0;
    size_t win_bytes = std::min<size_t>(8192 * 16, avail / 2) / 4096 * 4096;
    if (win_bytes < 1024 * 16 || tpb < 512) win_bytes = 0;  // the kernels' fixed-point paths
    const size_t region = std::max(small_b, win_bytes);
    int lb = kMaxLargeGuideBits;
    while (lb > 6 && region + bytes(lb) > avail) --lb;
    g.lbits_f = 0;
    // a copy more than 16 times coarser than the largest guide costs more
    // search steps than it saves: the full guide is read in place instead
    // (and the window, found on the coarse copy, is not used)
    g.lbits_b = lb >= guide_bits(large_g, kMaxLargeGuideBits, 1) - 4 ? lb : 0;
    if (g.lbits_b > 0) {
      guide_b = std::max(guide_b, bytes(lb));
      g.win_n = static_cast<int32_t>(win_bytes / 16);
      before_guide = region;
    }
  }
  g.bwd_guide_off = static_cast<int32_t>((before_guide / sizeof(uint32_t) + 3) & ~size_t(3));
  // Forward CTAs of large densities (512/1024 threads): a coarse guide (at
  // most 2^14 buckets) and a window of up to 8192 records around the
  // density's most probable stretch in shared memory, where the slots that
  // fall in it are searched; the rest use the full guide through L2.  Sized
  // not to lower the residency the register cap allows, with room for a
  // histogram-mode tile (16 KB).
  size_t fwd_region = fwd_knots, guide_fl = guide_f;
  if (large && tpb >= 512) {
    auto bytes = [](int b) { return ((size_t(1) << b) + 1 + 7) / 8 * 8 * sizeof(uint32_t); };
    const size_t ctas = resident(fwd_knots + guide_f);
    const size_t per_cta = std::min(kSmemPerSM / ctas - kSmemPerCtaReserved, kSmemLimit);
    const size_t avail = per_cta > g.static_smem + 16 * 1024 ? per_cta - g.static_smem - 16 * 1024 : 0;
    int lb = 14;
    while (lb > 6 && bytes(lb) * 3 > avail) --lb;
    const size_t rest = avail > bytes(lb) ? avail - bytes(lb) : 0;
    const size_t w = std::min<size_t>(8192, rest / sizeof(float4) / 256 * 256);
    if (w >= 1024) {
      g.lbits_f = lb;
      g.fwin_n = static_cast<int32_t>(w);
      fwd_region = std::max(fwd_knots, w * sizeof(float4));
      guide_fl = std::max(guide_f, bytes(lb));
    }
  }
  g.fwd_guide_off = static_cast<int32_t>((fwd_region / sizeof(uint32_t) + 3) & ~size_t(3));
  g.fwd = static_cast<size_t>(g.fwd_guide_off) * sizeof(uint32_t) + guide_fl;
  g.bwd = static_cast<size_t>(g.bwd_guide_off) * sizeof(uint32_t) + guide_b;
  if (g.fwd + g.static_smem > kSmemLimit || g.bwd + g.static_smem > kSmemLimit)
    return LOITS_ERR_UNSUPPORTED;
  FwdKernel fk2;
  BwdKernel bk_fix;
  kernels_for(tpb, r, large, fk2, bk_fix, true);
  if (!allow_dynamic_smem(reinterpret_cast<const void*>(fk), g.fwd) ||
      !allow_dynamic_smem(reinterpret_cast<const void*>(bk), g.bwd) ||
      !allow_dynamic_smem(reinterpret_cast<const void*>(bk_fix), g.bwd))
    return LOITS_ERR_CUDA;
  return LOITS_OK;
}

// Resident CTAs per SM of the forward and backward kernels of (tpb, r).
void occupancy(int tpb, int r, bool large, const SmemGeometry& g, int& occ_f, int& occ_b) {
  FwdKernel fk;
  BwdKernel bk;
  occ_f = occ_b = 0;
  if (!kernels_for(tpb, r, large, fk, bk)) return;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_f, fk, tpb, g.fwd);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_b, bk, tpb, g.bwd);
}

// CTA size with the most resident threads per SM for both kernels (the
// smaller CTA on a tie: fewer threads wait at each tile barrier).
int choose_threads(int r_req, int64_t large_g, int32_t gcap, int64_t max_g, int ratio,
                   int& tpb_out) {
  int best = -1, best_tpb = 0, last_rc = LOITS_ERR_UNSUPPORTED;
  for (int tpb : {256, 512, 1024}) {
    const int r = r_req ? r_req : default_blocks(tpb);
    SmemGeometry g;
    const int rc = smem_geometry(tpb, r, large_g, gcap, max_g, ratio, g);
    if (rc != LOITS_OK) {
      last_rc = rc;
      continue;
    }
    int of = 0, ob = 0;
    occupancy(tpb, r, large_g > 0, g, of, ob);
    const int resident = tpb * std::min(of, ob);
    if (resident > best) {
      best = resident;
      best_tpb = tpb;
    }
  }
  if (best <= 0) return last_rc == LOITS_OK ? LOITS_ERR_UNSUPPORTED : last_rc;
  tpb_out = best_tpb;
  return LOITS_OK;
}

template <typename T>
T* carve(void* ws, size_t off) {
  return reinterpret_cast<T*>(static_cast<char*>(ws) + off);
}

BatchArgs base_args(const loits_batch_plan* p, void* ws) {
  BatchArgs a{};
  a.knot_off = p->d_koff;
  a.n_events = p->d_nev;
  a.tile_first = p->d_tile_first;
  a.tile_owner = p->d_tile_owner;
  a.cdf_owner = p->d_cdf_owner;
  a.chunk_owner = p->d_chunk_owner;
  a.cdf_first = p->d_cdf_first;
  a.fin_first = p->d_fin_first;
  a.chunk_first = p->d_chunk_first;
  a.part_off = p->d_part_off;
  a.rowfill_lo = p->d_rowfill_lo;
  a.goff = p->d_goff;
  a.pkoff = p->d_pkoff;
  a.gbits = p->d_gbits;
  a.gc_off = p->d_gc_off;
  a.lfin_first = p->d_lfin_first;
  a.mcap = p->mcap;
  a.gbits_cap = 30;  // forward: full guides (the backward lowers this)
  a.lguide_bits = p->lbits_f;
  a.fwin_n = p->fwin_n;
  a.fwd_guide_off = p->fwd_guide_off;
  a.nd = static_cast<int32_t>(p->nd);
  a.last_nonempty = p->last_nonempty;
  a.tiles_total = p->n_tiles;
  a.tile_r = p->d_tile_r;
  a.scan_k = p->d_scan_k;
  a.gcap = p->gcap;
  a.tiles_per_chunk = p->tiles_per_chunk;
  a.spin_limit = p->cfg.wait_limit > 0 ? static_cast<uint32_t>(p->cfg.wait_limit) : kSpinLimit;
  a.withhold_tile = p->cfg.withhold_tile - 1;
  a.nmax = p->nmax;
  a.dbase = p->dbase;
  const Layout& L = p->lay;
  a.rec = carve<float4>(ws, L.rec);
  a.invd = carve<float>(ws, L.invd);
  a.gl = carve<uint32_t>(ws, L.gl);
  a.gpk = carve<uint32_t>(ws, L.gpk);
  a.fin_done = carve<uint32_t>(ws, L.fin_done);
  a.norm = carve<double>(ws, L.norm);
  a.kstar = carve<int32_t>(ws, L.kstar);
  a.dflags = carve<uint32_t>(ws, L.dflags);
  a.cdf_ready = carve<uint32_t>(ws, L.cdf_ready);
  a.cdf_scanned = carve<uint32_t>(ws, L.cdf_scanned);
  a.cflag = carve<uint32_t>(ws, L.cflag);
  a.cagg = carve<double>(ws, L.cagg);
  a.cinc = carve<double>(ws, L.cinc);
  a.cmax = carve<double>(ws, L.cmax);
  a.tile_state = carve<unsigned long long>(ws, L.tile_state);
  a.tile_prefix = carve<int64_t>(ws, L.tile_prefix);
  a.warp_off = carve<int32_t>(ws, L.warp_off);
  a.stage_g = carve<float>(ws, L.stage);
  a.status = carve<int32_t>(ws, L.status);
  a.chunks_done = carve<uint32_t>(ws, L.chunks_done);
  a.gcdf = carve<float2>(ws, L.gcdf);
  a.lflag = carve<uint32_t>(ws, L.lflag);
  a.lagg = carve<double>(ws, L.lagg);
  a.linc = carve<double>(ws, L.linc);
  a.lgn = carve<double>(ws, L.lgn);
  a.lfin_done = carve<uint32_t>(ws, L.lfin_done);
  a.partials = carve<float>(ws, L.partials);
  return a;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

}  // namespace

extern "C" int loits_batch_plan_create(int64_t n_densities, const int64_t* knot_offsets,
                                       const int64_t* event_counts,
                                       const loits_batch_config* cfg, loits_batch_plan** out) {
  return loits_batch_plan_create_ex(n_densities, knot_offsets, event_counts, cfg, nullptr,
                                    nullptr, out);
}

extern "C" int loits_batch_plan_create_ex(int64_t n_densities, const int64_t* knot_offsets,
                                          const int64_t* event_counts,
                                          const loits_batch_config* cfg,
                                          const int32_t* blocks_per_density,
                                          const int32_t* scan_knots_per_density,
                                          loits_batch_plan** out) {
  if (!out) return LOITS_ERR_INVALID;
  *out = nullptr;
  if (n_densities < 1 || n_densities > (1 << 24) || !knot_offsets || !event_counts)
    return LOITS_ERR_INVALID;
  loits_batch_config c;
  int rc = resolve_config(cfg, c);
  if (rc != LOITS_OK) return rc;
  auto* p = new (std::nothrow) loits_batch_plan();
  if (!p) return LOITS_ERR_INVALID;
  p->nd = n_densities;
  p->scan_knots = c.scan_knots;
  p->koff.assign(knot_offsets, knot_offsets + n_densities + 1);
  p->nev.assign(event_counts, event_counts + n_densities);
  if (p->koff[0] != 0) { delete p; return LOITS_ERR_INVALID; }
  for (int64_t b = 0; b < n_densities; ++b) {
    const int64_t g = p->koff[b + 1] - p->koff[b];
    if (g < 2 || p->nev[b] < 0) { delete p; return LOITS_ERR_INVALID; }
    p->max_g = std::max(p->max_g, g);
    if (g <= kMaxSmemKnots) p->small_max_g = std::max(p->small_max_g, g);
    p->nmax = std::max(p->nmax, p->nev[b]);
    p->capacity += p->nev[b];
    if (p->nev[b] > 0) p->last_nonempty = static_cast<int32_t>(b);
  }
  p->total_knots = p->koff[n_densities];
  if (p->max_g > kMaxKnots) { delete p; return LOITS_ERR_UNSUPPORTED; }
  if (c.slot_stride > 0) {
    if (c.slot_stride < p->nmax) { delete p; return LOITS_ERR_INVALID; }
    p->nmax = c.slot_stride;
  }
  p->dbase = c.density_base;
  if (p->nmax > 0 && static_cast<double>(p->nmax) * static_cast<double>(n_densities + p->dbase) > 4.0e18) {
    delete p;
    return LOITS_ERR_UNSUPPORTED;
  }
  // knots a sampling CTA holds: the largest small density, rounded to a
  // multiple of 4 so that every shared-memory array after the records stays
  // 16-byte aligned (every large density has more knots than this)
  p->gcap = static_cast<int32_t>((std::max<int64_t>(p->small_max_g, 4) + 3) & ~int64_t(3));
  p->has_large = p->max_g > p->gcap;
  const int64_t large_g = p->has_large ? p->max_g : 0;
  // ---- launch geometry: the CTA size (by occupancy unless given)
  if (c.threads == 0) {
    int tpb = 0;
    rc = choose_threads(c.blocks_per_item, large_g, p->gcap, p->small_max_g, c.guide_ratio,
                        tpb);
    if (rc != LOITS_OK) { delete p; return rc; }
    c.threads = tpb;
  }
  if (c.blocks_per_item == 0) c.blocks_per_item = default_blocks(c.threads);
  p->cfg = c;
  p->tpb = c.threads;
  p->r = c.blocks_per_item;
  SmemGeometry sg;
  rc = smem_geometry(p->tpb, p->r, large_g, p->gcap, p->small_max_g, c.guide_ratio, sg);
  if (rc != LOITS_OK) { delete p; return rc; }
  // ---- per-density tile length (at most the launch's blocks per item) and
  // CDF scan width (1..64): the defaults, or the caller's tables
  p->tile_r.assign(n_densities, p->r);
  p->scan_k.assign(n_densities, p->scan_knots);
  for (int64_t b = 0; b < n_densities; ++b) {
    if (blocks_per_density) {
      if (blocks_per_density[b] < 1 || blocks_per_density[b] > p->r) { delete p; return LOITS_ERR_INVALID; }
      p->tile_r[b] = blocks_per_density[b];
    }
    if (scan_knots_per_density) {
      if (scan_knots_per_density[b] < 1 || scan_knots_per_density[b] > 64) {
        delete p;
        return LOITS_ERR_INVALID;
      }
      p->scan_k[b] = scan_knots_per_density[b];
    }
  }
  // ---- work items
  const int64_t blocks_per_tile = static_cast<int64_t>(p->tpb) * p->r;  // the longest tile
  p->tile_first.resize(n_densities + 1);
  p->cdf_first.resize(n_densities + 1);
  p->fin_first.resize(n_densities + 1);
  p->rowfill_lo.resize(n_densities);
  int64_t nt = 0, nc = 0, nf = 0;
  int32_t next_fill = 0;
  for (int64_t b = 0; b < n_densities; ++b) {
    p->tile_first[b] = static_cast<int32_t>(nt);
    p->cdf_first[b] = static_cast<int32_t>(nc);
    p->fin_first[b] = static_cast<int32_t>(nf);
    const int64_t g = p->koff[b + 1] - p->koff[b];
    const int64_t kt = static_cast<int64_t>(p->tpb) * p->scan_k[b];
    const int64_t tiles_c = (g + kt - 1) / kt;
    nc += tiles_c;
    if (tiles_c > 1) nf += tiles_c;
    const int64_t n = p->nev[b];
    if (n > 0) {
      const int64_t P0 = (p->dbase + b) * p->nmax;
      const int64_t nblk = ((P0 + n - 1) >> 2) - (P0 >> 2) + 1;
      // even out the density's tiles: keep the tile count its length cap
      // gives, with the fewest blocks per thread that still cover it, so
      // that a density smaller than one tile spreads over every warp of
      // the CTA instead of the first few
      const int64_t cap_bpt = static_cast<int64_t>(p->tpb) * p->tile_r[b];
      const int64_t tiles_b = (nblk + cap_bpt - 1) / cap_bpt;
      const int64_t per_tile = (nblk + tiles_b - 1) / tiles_b;
      p->tile_r[b] = static_cast<int32_t>((per_tile + p->tpb - 1) / p->tpb);
      const int64_t bpt = static_cast<int64_t>(p->tpb) * p->tile_r[b];
      nt += (nblk + bpt - 1) / bpt;
      p->rowfill_lo[b] = next_fill;
      next_fill = static_cast<int32_t>(b + 1);
    } else {
      p->rowfill_lo[b] = next_fill;
    }
  }
  if (nt > 0x7fffffff || nc > 0x7fffffff) { delete p; return LOITS_ERR_UNSUPPORTED; }
  p->tile_first[n_densities] = static_cast<int32_t>(nt);
  p->cdf_first[n_densities] = static_cast<int32_t>(nc);
  p->fin_first[n_densities] = static_cast<int32_t>(nf);
  p->n_tiles = static_cast<int32_t>(nt);
  p->n_cdf = static_cast<int32_t>(nc);
  p->n_fin = static_cast<int32_t>(nf);
  // guide tables: M + 1 uint32 counts per density, and for small densities
  // also M packed 8-byte entries (the copy the sampling CTAs load); a large
  // density's guide is capped by kMaxLargeGuideBits, not shared memory
  p->gbits.resize(n_densities);
  p->goff.resize(n_densities);
  p->pkoff.resize(n_densities);
  p->gc_off.resize(n_densities);
  p->lfin_first.resize(n_densities + 1);
  const int64_t lseg = static_cast<int64_t>(p->tpb) * 4;
  int64_t go = 0, pko = 0, gco = 0, nl = 0;
  for (int64_t b = 0; b < n_densities; ++b) {
    const int64_t g = p->koff[b + 1] - p->koff[b];
    const bool large = g > p->gcap;
    const int m = large ? guide_bits(g, kMaxLargeGuideBits, 1) : guide_bits(g, sg.m_cap, c.guide_ratio);
    p->gbits[b] = m;
    p->goff[b] = go;
    go += ((int64_t(1) << m) + 1 + 7) & ~int64_t(7);
    p->lfin_first[b] = static_cast<int32_t>(nl);
    if (large) {
      p->pkoff[b] = -1;
      p->gc_off[b] = gco;
      gco += g;
      nl += (g + lseg - 1) / lseg;
    } else {
      p->pkoff[b] = pko;
      pko += 2 * (((int64_t(1) << m) + 7) & ~int64_t(7));
      p->gc_off[b] = -1;
      p->mcap = std::max<int32_t>(p->mcap, static_cast<int32_t>(int64_t(1) << m));
    }
  }
  if (nl > 0x3fffffff) { delete p; return LOITS_ERR_UNSUPPORTED; }
  p->lfin_first[n_densities] = static_cast<int32_t>(nl);
  p->n_lfin = static_cast<int32_t>(nl);
  p->total_guide = go;
  p->total_pk = pko;
  p->total_gc = gco;
  p->m_cap_b = sg.m_cap_b;
  p->lbits_f = sg.lbits_f;
  p->lbits_b = sg.lbits_b;
  p->fix_small = sg.fix_small;
  p->win_n = sg.win_n;
  p->bwd_guide_off = sg.bwd_guide_off;
  p->fwin_n = sg.fwin_n;
  p->fwd_guide_off = sg.fwd_guide_off;
  // the backward variant with fixed-point sums, when some small density
  // takes that path (its 36 bytes per knot within the slot; see
  // vjp_chunk_item)
  if (p->tpb >= 512) {
    for (int64_t b = 0; b < n_densities && !p->fix_used; ++b) {
      const int64_t g = p->koff[b + 1] - p->koff[b];
      p->fix_used = g <= p->gcap && 36 * g <= 4 * static_cast<int64_t>(p->bwd_guide_off);
    }
  }
  p->fwd_smem = sg.fwd;
  p->fwd_smem_allowed = sg.fwd;
  p->bwd_smem_allowed = sg.bwd;
  p->bwd_smem = sg.bwd;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) { delete p; return LOITS_ERR_CUDA; }
  cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, dev);
  int occ_f = 0, occ_b = 0;
  occupancy(p->tpb, p->r, p->has_large, sg, occ_f, occ_b);
  if (occ_f < 1 || occ_b < 1) { delete p; return LOITS_ERR_UNSUPPORTED; }
  if (c.ctas_per_sm > 0) {
    occ_f = std::min(occ_f, static_cast<int>(c.ctas_per_sm));
    occ_b = std::min(occ_b, static_cast<int>(c.ctas_per_sm));
  }
  const int64_t tile_events = blocks_per_tile * 4;
  const int64_t items_f = nc + nf + nt;
  p->fwd_grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(items_f, int64_t(occ_f) * p->num_sms)));
  const int64_t resident_b = int64_t(occ_b) * p->num_sms;
  // backward chunks: ~4 per resident CTA keeps the last wave short; plans
  // with large densities (global atomics, no per-chunk shared histogram)
  // measured faster with ~2
  const int64_t target_chunks = std::max<int64_t>(1, (p->has_large ? 2 : 4) * resident_b);
  p->tiles_per_chunk = static_cast<int32_t>(std::max<int64_t>(1, nt / target_chunks));
  p->chunk_first.resize(n_densities + 1);
  p->part_off.resize(n_densities);
  int64_t nk = 0, po = 0;
  for (int64_t b = 0; b < n_densities; ++b) {
    p->chunk_first[b] = static_cast<int32_t>(nk);
    p->part_off[b] = po;
    const int64_t tiles_b = p->tile_first[b + 1] - p->tile_first[b];
    const int64_t ch = (tiles_b + p->tiles_per_chunk - 1) / p->tiles_per_chunk;
    nk += ch;
    po += ch * (p->koff[b + 1] - p->koff[b]);
  }
  p->chunk_first[n_densities] = static_cast<int32_t>(nk);
  p->n_chunks = static_cast<int32_t>(nk);
  // the density of every tile, CDF scan tile and chunk (one load per item
  // instead of a search of the first-item tables)
  auto owners = [&](const std::vector<int32_t>& first, std::vector<int32_t>& out) {
    out.assign(static_cast<size_t>(first.back()), 0);
    for (int64_t b = 0; b < n_densities; ++b)
      for (int32_t i = first[b]; i < first[b + 1]; ++i) out[i] = static_cast<int32_t>(b);
  };
  owners(p->tile_first, p->tile_owner);
  owners(p->cdf_first, p->cdf_owner);
  owners(p->chunk_first, p->chunk_owner);
  p->total_partials = po;
  const int64_t items_b = nk + n_densities + 2 * static_cast<int64_t>(p->n_lfin);
  p->bwd_grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(items_b, resident_b)));

  // ---- workspace layout
  Layout& L = p->lay;
  size_t o = 0;
  const size_t nd = static_cast<size_t>(n_densities);
  L.fwd_zero_lo = o;
  L.status = o; o += 16;
  L.tickets_fwd = o; o = align_up(o + (nd + 1) * 4, 16);
  L.dflags = o; o = align_up(o + nd * 4, 16);
  L.cdf_ready = o; o = align_up(o + nd * 4, 16);
  L.cdf_scanned = o; o = align_up(o + nd * 4, 16);
  L.fin_done = o; o = align_up(o + nd * 4, 16);
  L.cflag = o; o = align_up(o + static_cast<size_t>(nc) * 4, 16);
  L.tile_state = o; o = align_up(o + static_cast<size_t>(nt) * 8, 16);
  L.fwd_zero_hi = o;
  o = align_up(o);
  L.bwd_zero_lo = o;
  L.tickets_bwd = o; o = align_up(o + (nd + 1) * 4, 16);
  L.chunks_done = o; o = align_up(o + nd * 4, 16);
  L.lfin_done = o; o = align_up(o + nd * 4, 16);
  L.lflag = o; o = align_up(o + static_cast<size_t>(p->n_lfin) * 4, 16);
  L.gcdf = o; o = align_up(o + static_cast<size_t>(p->total_gc) * 8, 16);
  L.bwd_zero_hi = o;
  o = align_up(o);
  L.rec = o; o = align_up(o + static_cast<size_t>(p->total_knots) * 16);
  L.invd = o; o = align_up(o + static_cast<size_t>(p->total_knots) * 4);
  L.gl = o; o = align_up(o + static_cast<size_t>(p->total_guide) * 4);
  L.gpk = o; o = align_up(o + static_cast<size_t>(p->total_pk) * 4);
  L.lagg = o; o = align_up(o + static_cast<size_t>(p->n_lfin) * 8);
  L.linc = o; o = align_up(o + static_cast<size_t>(p->n_lfin) * 8);
  L.lgn = o; o = align_up(o + static_cast<size_t>(p->n_lfin) * 8);
  L.norm = o; o = align_up(o + nd * 8);
  L.kstar = o; o = align_up(o + nd * 4);
  L.cagg = o; o = align_up(o + static_cast<size_t>(nc) * 8);
  L.cinc = o; o = align_up(o + static_cast<size_t>(nc) * 8);
  L.cmax = o; o = align_up(o + static_cast<size_t>(nc) * 8);
  L.tile_prefix = o; o = align_up(o + static_cast<size_t>(nt + 1) * 8);  // + one past the end
  L.warp_off = o; o = align_up(o + static_cast<size_t>(nt) * (p->tpb / 32) * 4);
  L.stage = o; o = align_up(o + static_cast<size_t>(p->fwd_grid) * tile_events * 4);
  L.partials = o; o = align_up(o + static_cast<size_t>(po) * 4);
  L.grho = o; o = align_up(o + static_cast<size_t>(p->total_knots) * 8);
  L.total = o;

  // ---- device tables (one allocation owned by the plan)
  std::vector<char> host;
  auto push = [&host](const void* src, size_t bytes) {
    const size_t off = align_up(host.size(), 16);
    host.resize(off + bytes);
    if (bytes) std::memcpy(host.data() + off, src, bytes);
    return off;
  };
  const size_t o_koff = push(p->koff.data(), p->koff.size() * 8);
  const size_t o_nev = push(p->nev.data(), p->nev.size() * 8);
  const size_t o_part = push(p->part_off.data(), p->part_off.size() * 8);
  const size_t o_tf = push(p->tile_first.data(), p->tile_first.size() * 4);
  const size_t o_cf = push(p->cdf_first.data(), p->cdf_first.size() * 4);
  const size_t o_ff = push(p->fin_first.data(), p->fin_first.size() * 4);
  const size_t o_kf = push(p->chunk_first.data(), p->chunk_first.size() * 4);
  const size_t o_to = push(p->tile_owner.data(), p->tile_owner.size() * 4);
  const size_t o_co = push(p->cdf_owner.data(), p->cdf_owner.size() * 4);
  const size_t o_ko = push(p->chunk_owner.data(), p->chunk_owner.size() * 4);
  const size_t o_rf = push(p->rowfill_lo.data(), p->rowfill_lo.size() * 4);
  const size_t o_go = push(p->goff.data(), p->goff.size() * 8);
  const size_t o_gb = push(p->gbits.data(), p->gbits.size() * 4);
  const size_t o_pk = push(p->pkoff.data(), p->pkoff.size() * 8);
  const size_t o_gc = push(p->gc_off.data(), p->gc_off.size() * 8);
  const size_t o_lf = push(p->lfin_first.data(), p->lfin_first.size() * 4);
  const size_t o_tr = push(p->tile_r.data(), p->tile_r.size() * 4);
  const size_t o_sk = push(p->scan_k.data(), p->scan_k.size() * 4);
  if (cudaMalloc(&p->dtab, host.size()) != cudaSuccess) { delete p; return LOITS_ERR_CUDA; }
  if (cudaMemcpy(p->dtab, host.data(), host.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(p->dtab);
    delete p;
    return LOITS_ERR_CUDA;
  }
  char* d = static_cast<char*>(p->dtab);
  p->d_koff = reinterpret_cast<const int64_t*>(d + o_koff);
  p->d_nev = reinterpret_cast<const int64_t*>(d + o_nev);
  p->d_part_off = reinterpret_cast<const int64_t*>(d + o_part);
  p->d_tile_first = reinterpret_cast<const int32_t*>(d + o_tf);
  p->d_cdf_first = reinterpret_cast<const int32_t*>(d + o_cf);
  p->d_fin_first = reinterpret_cast<const int32_t*>(d + o_ff);
  p->d_chunk_first = reinterpret_cast<const int32_t*>(d + o_kf);
  p->d_tile_owner = reinterpret_cast<const int32_t*>(d + o_to);
  p->d_cdf_owner = reinterpret_cast<const int32_t*>(d + o_co);
  p->d_chunk_owner = reinterpret_cast<const int32_t*>(d + o_ko);
  p->d_rowfill_lo = reinterpret_cast<const int32_t*>(d + o_rf);
  p->d_goff = reinterpret_cast<const int64_t*>(d + o_go);
  p->d_gbits = reinterpret_cast<const int32_t*>(d + o_gb);
  p->d_pkoff = reinterpret_cast<const int64_t*>(d + o_pk);
  p->d_gc_off = reinterpret_cast<const int64_t*>(d + o_gc);
  p->d_lfin_first = reinterpret_cast<const int32_t*>(d + o_lf);
  p->d_tile_r = reinterpret_cast<const int32_t*>(d + o_tr);
  p->d_scan_k = reinterpret_cast<const int32_t*>(d + o_sk);
  *out = p;
  return LOITS_OK;
}

extern "C" void loits_batch_plan_destroy(loits_batch_plan* plan) {
  if (!plan) return;
  if (plan->dtab) cudaFree(plan->dtab);
  delete plan;
}

extern "C" int64_t loits_batch_capacity(const loits_batch_plan* p) { return p ? p->capacity : -1; }
extern "C" int64_t loits_batch_total_knots(const loits_batch_plan* p) {
  return p ? p->total_knots : -1;
}
extern "C" size_t loits_batch_workspace_bytes(const loits_batch_plan* p) {
  return p ? p->lay.total : 0;
}
extern "C" size_t loits_batch_status_offset(const loits_batch_plan* p) {
  return p ? p->lay.status : 0;
}
extern "C" int loits_batch_plan_config(const loits_batch_plan* p, loits_batch_config* cfg) {
  if (!p || !cfg) return LOITS_ERR_INVALID;
  *cfg = p->cfg;
  return LOITS_OK;
}

namespace {

// Forward launch(es) of a prepared argument block: one persistent launch, or
// one launch per density (plain form).
int launch_forward(const loits_batch_plan* p, BatchArgs& a, void* workspace, size_t smem,
                   cudaStream_t st) {
  const Layout& L = p->lay;
  if (cudaMemsetAsync(static_cast<char*>(workspace) + L.fwd_zero_lo, 0,
                      L.fwd_zero_hi - L.fwd_zero_lo, st) != cudaSuccess)
    return LOITS_ERR_CUDA;
  FwdKernel fk;
  BwdKernel bk;
  kernels_for(p->tpb, p->r, p->has_large, fk, bk);
  if (smem > p->fwd_smem_allowed) {
    if (!allow_dynamic_smem(reinterpret_cast<const void*>(fk), smem)) return LOITS_ERR_CUDA;
    p->fwd_smem_allowed = smem;
  }
  uint32_t* tickets = carve<uint32_t>(workspace, L.tickets_fwd);
  if (!p->cfg.plain) {
    a.c_lo = 0; a.c_hi = p->n_cdf;
    a.f_lo = 0; a.f_hi = p->n_fin;
    a.t_lo = 0; a.t_hi = p->n_tiles;
    a.d_lo = 0; a.d_hi = static_cast<int32_t>(p->nd);
    a.ticket = tickets + p->nd;
    fk<<<p->fwd_grid, p->tpb, smem, st>>>(a);
    return cudaGetLastError() == cudaSuccess ? LOITS_OK : LOITS_ERR_CUDA;
  }
  for (int64_t b = 0; b < p->nd; ++b) {
    a.c_lo = p->cdf_first[b]; a.c_hi = p->cdf_first[b + 1];
    a.f_lo = p->fin_first[b]; a.f_hi = p->fin_first[b + 1];
    a.t_lo = p->tile_first[b]; a.t_hi = p->tile_first[b + 1];
    a.d_lo = static_cast<int32_t>(b); a.d_hi = static_cast<int32_t>(b + 1);
    a.ticket = tickets + b;
    const int64_t items = (a.c_hi - a.c_lo) + (a.f_hi - a.f_lo) + (a.t_hi - a.t_lo);
    const int grid_b = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(items, p->fwd_grid)));
    fk<<<grid_b, p->tpb, smem, st>>>(a);
    if (cudaGetLastError() != cudaSuccess) return LOITS_ERR_CUDA;
  }
  return LOITS_OK;
}

int launch_backward(const loits_batch_plan* p, BatchArgs& a, void* workspace, size_t smem,
                    cudaStream_t st) {
  const Layout& L = p->lay;
  if (cudaMemsetAsync(static_cast<char*>(workspace) + L.bwd_zero_lo, 0,
                      L.bwd_zero_hi - L.bwd_zero_lo, st) != cudaSuccess)
    return LOITS_ERR_CUDA;
  a.gbits_cap = p->m_cap_b;
  a.lguide_bits = p->lbits_b;
  a.win_n = p->win_n;
  a.bwd_guide_off = p->bwd_guide_off;
  double* grho = carve<double>(workspace, L.grho);
  FwdKernel fk;
  BwdKernel bk;
  kernels_for(p->tpb, p->r, p->has_large, fk, bk, p->fix_used);
  if (smem > p->bwd_smem_allowed) {
    if (!allow_dynamic_smem(reinterpret_cast<const void*>(bk), smem)) return LOITS_ERR_CUDA;
    p->bwd_smem_allowed = smem;
  }
  uint32_t* tickets = carve<uint32_t>(workspace, L.tickets_bwd);
  if (!p->cfg.plain) {
    a.k_lo = 0; a.k_hi = p->n_chunks;
    a.d_lo = 0; a.d_hi = static_cast<int32_t>(p->nd);
    a.l_lo = 0; a.l_hi = p->n_lfin;
    a.ticket = tickets + p->nd;
    bk<<<p->bwd_grid, p->tpb, smem, st>>>(a, grho);
    return cudaGetLastError() == cudaSuccess ? LOITS_OK : LOITS_ERR_CUDA;
  }
  for (int64_t b = 0; b < p->nd; ++b) {
    a.k_lo = p->chunk_first[b]; a.k_hi = p->chunk_first[b + 1];
    a.d_lo = static_cast<int32_t>(b); a.d_hi = static_cast<int32_t>(b + 1);
    a.l_lo = p->lfin_first[b]; a.l_hi = p->lfin_first[b + 1];
    a.ticket = tickets + b;
    const int64_t items = (a.k_hi - a.k_lo) + 1 + 2 * (a.l_hi - a.l_lo);
    const int grid_b = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(items, p->bwd_grid)));
    bk<<<grid_b, p->tpb, smem, st>>>(a, grho);
    if (cudaGetLastError() != cudaSuccess) return LOITS_ERR_CUDA;
  }
  return LOITS_OK;
}

BatchArgs step_args(const loits_batch_plan* p, void* workspace, const float* grid,
                    const float* values, const float* x_cut, uint64_t seed, uint64_t sequence) {
  BatchArgs a = base_args(p, workspace);
  a.seed = seed;
  a.rk = philox_key(seed);
  a.stream_id = 2 * sequence;
  a.grid = grid;
  a.values = values;
  a.x_cut = x_cut;
  return a;
}

bool hist_range_ok(int32_t bins, float lo, float hi) {
  return bins >= 1 && bins <= kMaxHistBins && std::isfinite(lo) && std::isfinite(hi) && lo < hi;
}

}  // namespace

extern "C" int loits_batch_forward(const loits_batch_plan* p, const float* grid,
                                   const float* values, const float* x_cut, uint64_t seed,
                                   uint64_t sequence, float* events, int64_t* row_offsets,
                                   int32_t* intervals, void* workspace, void* stream) {
  if (!p || !grid || !values || !row_offsets || !workspace) return LOITS_ERR_INVALID;
  if (p->capacity > 0 && (!events || !aligned16(events))) return LOITS_ERR_INVALID;
  if (intervals && !aligned16(intervals)) return LOITS_ERR_INVALID;
  if (!aligned16(workspace)) return LOITS_ERR_INVALID;
  if (sequence > (UINT64_MAX - 1) / 2) return LOITS_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (p->n_tiles == 0 &&
      cudaMemsetAsync(row_offsets, 0, (p->nd + 1) * sizeof(int64_t), st) != cudaSuccess)
    return LOITS_ERR_CUDA;
  BatchArgs a = step_args(p, workspace, grid, values, x_cut, seed, sequence);
  a.events = events;
  a.row_offsets = row_offsets;
  a.intervals = intervals;
  return launch_forward(p, a, workspace, p->fwd_smem, st);
}

extern "C" int loits_batch_backward(const loits_batch_plan* p, const float* grid,
                                    const float* values, const float* x_cut, uint64_t seed,
                                    uint64_t sequence, const float* grad_events,
                                    float* grad_values, void* workspace, void* stream) {
  if (!p || !grid || !values || !grad_values || !workspace) return LOITS_ERR_INVALID;
  if (p->capacity > 0 && (!grad_events || !aligned16(grad_events))) return LOITS_ERR_INVALID;
  if (!aligned16(workspace)) return LOITS_ERR_INVALID;
  if (sequence > (UINT64_MAX - 1) / 2) return LOITS_ERR_INVALID;
  BatchArgs a = step_args(p, workspace, grid, values, x_cut, seed, sequence);
  a.grad = grad_events;
  a.grad_values = grad_values;
  return launch_backward(p, a, workspace, p->bwd_smem, static_cast<cudaStream_t>(stream));
}

extern "C" int loits_batch_forward_state(const loits_batch_plan* p, const float* grid,
                                         const float* values, const float* x_cut, uint64_t seed,
                                         uint64_t sequence, float* events, int64_t* row_offsets,
                                         int32_t* intervals, float* offsets, void* workspace,
                                         void* stream) {
  if (p && p->capacity > 0 && (!intervals || !offsets)) return LOITS_ERR_INVALID;
  if (!p || !grid || !values || !row_offsets || !workspace) return LOITS_ERR_INVALID;
  if (p->capacity > 0 && (!events || !aligned16(events) || !aligned16(intervals) ||
                          !aligned16(offsets)))
    return LOITS_ERR_INVALID;
  if (!aligned16(workspace)) return LOITS_ERR_INVALID;
  if (sequence > (UINT64_MAX - 1) / 2) return LOITS_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (p->n_tiles == 0 &&
      cudaMemsetAsync(row_offsets, 0, (p->nd + 1) * sizeof(int64_t), st) != cudaSuccess)
    return LOITS_ERR_CUDA;
  BatchArgs a = step_args(p, workspace, grid, values, x_cut, seed, sequence);
  a.events = events;
  a.row_offsets = row_offsets;
  a.intervals = intervals;
  a.offsets = offsets;
  return launch_forward(p, a, workspace, p->fwd_smem, st);
}

extern "C" int loits_batch_backward_state(const loits_batch_plan* p, const float* grid,
                                          const float* values, const float* x_cut,
                                          const int32_t* intervals, const float* offsets,
                                          const float* grad_events, float* grad_values,
                                          void* workspace, void* stream) {
  if (!p || !grid || !values || !grad_values || !workspace) return LOITS_ERR_INVALID;
  if (p->capacity > 0 && (!grad_events || !intervals || !offsets)) return LOITS_ERR_INVALID;
  if (!aligned16(workspace)) return LOITS_ERR_INVALID;
  BatchArgs a = step_args(p, workspace, grid, values, x_cut, 0, 0);
  a.grad = grad_events;
  a.grad_values = grad_values;
  a.st_intervals = intervals;
  a.st_offsets = offsets;
  return launch_backward(p, a, workspace, p->bwd_smem, static_cast<cudaStream_t>(stream));
}

namespace {

// Whether the densities of plan p can take their values from theory
// parameters: each CDF is one tile staged in shared memory (the tile load
// evaluates the theory) and sampled from shared memory.
bool theory_fits(const loits_batch_plan* p) {
  for (int64_t b = 0; b < p->nd; ++b) {
    const int64_t g = p->koff[b + 1] - p->koff[b];
    const int64_t kt = static_cast<int64_t>(p->tpb) * p->scan_k[b];
    if (g > p->gcap || g > kt || 8 * (g + 2) > 4 * static_cast<int64_t>(p->fwd_guide_off))
      return false;
  }
  return true;
}

int forward_hist(const loits_batch_plan* p, const float* grid, const float* values,
                 const float* theory, const float* x_cut, uint64_t seed, uint64_t sequence,
                 int32_t bins, float lo, float hi, float* hist, int64_t* kept, void* workspace,
                 const uint64_t* sequence_dev, void* stream) {
  if (!p || !grid || !(values || theory) || !hist || !kept || !workspace) return LOITS_ERR_INVALID;
  if (!hist_range_ok(bins, lo, hi) || !aligned16(workspace)) return LOITS_ERR_INVALID;
  if (sequence > (UINT64_MAX - 1) / 2) return LOITS_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(hist, 0, static_cast<size_t>(p->nd) * bins * sizeof(float), st) != cudaSuccess ||
      cudaMemsetAsync(kept, 0, static_cast<size_t>(p->nd) * sizeof(int64_t), st) != cudaSuccess)
    return LOITS_ERR_CUDA;
  BatchArgs a = step_args(p, workspace, grid, values, x_cut, seed, sequence);
  a.theory = theory;
  a.seq_dev = sequence_dev;
  a.hist = hist;
  a.kept = reinterpret_cast<unsigned long long*>(kept);
  a.hist_bins = bins;
  a.hist_lo = lo;
  a.hist_inv_h = static_cast<float>(bins / (static_cast<double>(hi) - lo));
  a.hist_smem_off = static_cast<int32_t>(p->fwd_smem / sizeof(float));
  int rep = 1;
  while (rep < 32 && 2 * rep * (bins + 1) * sizeof(float) <= static_cast<size_t>(kHistSmemBytes))
    rep *= 2;
  a.hist_rep = rep;
  // a copy takes at most tpb / rep lanes x r blocks x 4 slots of a tile, each
  // adding at most 2^shift to one bin: keep that below 2^32
  const int64_t per_copy = static_cast<int64_t>(p->tpb) * p->r * 4 / rep;
  int shift = 31;
  while (shift > 8 && (per_copy << shift) >= (int64_t(1) << 32)) --shift;
  a.hist_shift = shift;
  const size_t smem = p->fwd_smem + static_cast<size_t>(rep) * (bins + 1) * sizeof(float);
  return launch_forward(p, a, workspace, smem, st);
}

int backward_hist(const loits_batch_plan* p, const float* grid, const float* values,
                  const float* theory, const float* x_cut, uint64_t seed, uint64_t sequence,
                  int32_t bins, float lo, float hi, const float* grad_hist, float* grad_values,
                  float* grad_theory, void* workspace, const uint64_t* sequence_dev,
                  void* stream) {
  if (!p || !grid || !(values || theory) || !grad_hist || !(grad_values || grad_theory) ||
      !workspace)
    return LOITS_ERR_INVALID;
  if (!hist_range_ok(bins, lo, hi) || !aligned16(workspace)) return LOITS_ERR_INVALID;
  if (sequence > (UINT64_MAX - 1) / 2) return LOITS_ERR_INVALID;
  BatchArgs a = step_args(p, workspace, grid, values, x_cut, seed, sequence);
  a.theory = theory;
  a.seq_dev = sequence_dev;
  a.grad_hist = grad_hist;
  a.grad_values = grad_values;
  a.grad_theory = grad_theory;
  a.hist_bins = bins;
  a.hist_lo = lo;
  a.hist_inv_h = static_cast<float>(bins / (static_cast<double>(hi) - lo));
  a.hist_smem_off = static_cast<int32_t>(p->bwd_smem / sizeof(float));
  const size_t smem = p->bwd_smem + static_cast<size_t>(bins) * sizeof(float);
  return launch_backward(p, a, workspace, smem, static_cast<cudaStream_t>(stream));
}

}  // namespace

extern "C" int loits_batch_forward_hist(const loits_batch_plan* p, const float* grid,
                                        const float* values, const float* x_cut, uint64_t seed,
                                        uint64_t sequence, int32_t bins, float lo, float hi,
                                        float* hist, int64_t* kept, void* workspace,
                                        const uint64_t* sequence_dev, void* stream) {
  if (!values) return LOITS_ERR_INVALID;
  return forward_hist(p, grid, values, nullptr, x_cut, seed, sequence, bins, lo, hi, hist, kept,
                      workspace, sequence_dev, stream);
}

extern "C" int loits_batch_backward_hist(const loits_batch_plan* p, const float* grid,
                                         const float* values, const float* x_cut, uint64_t seed,
                                         uint64_t sequence, int32_t bins, float lo, float hi,
                                         const float* grad_hist, float* grad_values,
                                         void* workspace, const uint64_t* sequence_dev,
                                         void* stream) {
  if (!values || !grad_values) return LOITS_ERR_INVALID;
  return backward_hist(p, grid, values, nullptr, x_cut, seed, sequence, bins, lo, hi, grad_hist,
                       grad_values, nullptr, workspace, sequence_dev, stream);
}

extern "C" int loits_batch_forward_hist_powerlaw(const loits_batch_plan* p, const float* grid,
                                                 const float* params, const float* x_cut,
                                                 uint64_t seed, uint64_t sequence, int32_t bins,
                                                 float lo, float hi, float* hist, int64_t* kept,
                                                 void* workspace, const uint64_t* sequence_dev,
                                                 void* stream) {
  if (!p || !params) return LOITS_ERR_INVALID;
  if (!theory_fits(p)) return LOITS_ERR_UNSUPPORTED;
  return forward_hist(p, grid, nullptr, params, x_cut, seed, sequence, bins, lo, hi, hist, kept,
                      workspace, sequence_dev, stream);
}

extern "C" int loits_batch_backward_hist_powerlaw(const loits_batch_plan* p, const float* grid,
                                                  const float* params, const float* x_cut,
                                                  uint64_t seed, uint64_t sequence, int32_t bins,
                                                  float lo, float hi, const float* grad_hist,
                                                  float* grad_params, void* workspace,
                                                  const uint64_t* sequence_dev, void* stream) {
  if (!p || !params || !grad_params) return LOITS_ERR_INVALID;
  if (!theory_fits(p)) return LOITS_ERR_UNSUPPORTED;
  return backward_hist(p, grid, nullptr, params, x_cut, seed, sequence, bins, lo, hi, grad_hist,
                       nullptr, grad_params, workspace, sequence_dev, stream);
}

extern "C" int loits_batch_cdf(const loits_batch_plan* p, const void* workspace, double* cdf,
                               double* norm, void* stream) {
  if (!p || !workspace || !cdf) return LOITS_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const float4* rec = reinterpret_cast<const float4*>(static_cast<const char*>(workspace) + p->lay.rec);
  const int64_t n = p->total_knots;
  const int threads = 256;
  const int64_t grid = std::min<int64_t>((n + threads - 1) / threads, 148 * 32);
  batch_cdf_export_kernel<<<static_cast<int>(std::max<int64_t>(grid, 1)), threads, 0, st>>>(rec, n, cdf);
  if (cudaGetLastError() != cudaSuccess) return LOITS_ERR_CUDA;
  if (norm &&
      cudaMemcpyAsync(norm, static_cast<const char*>(workspace) + p->lay.norm,
                      p->nd * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return LOITS_ERR_CUDA;
  return LOITS_OK;
}

extern "C" int loits_batch_quantile(const loits_batch_plan* p, const void* workspace,
                                    int64_t density, const float* u, int64_t n, float* x,
                                    int32_t* intervals, void* stream) {
  if (!p || !workspace || density < 0 || density >= p->nd || n < 0 || (n > 0 && (!u || !x)))
    return LOITS_ERR_INVALID;
  if (n == 0) return LOITS_OK;
  // the non-decreasing flag lives on the device; read it (a 4-byte sync copy)
  uint32_t flags = 0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const char* ws = static_cast<const char*>(workspace);
  if (cudaMemcpyAsync(&flags, ws + p->lay.dflags + density * 4, 4, cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return LOITS_ERR_CUDA;
  const float4* rec = reinterpret_cast<const float4*>(ws + p->lay.rec) + p->koff[density];
  const uint32_t* guide = reinterpret_cast<const uint32_t*>(ws + p->lay.gl) + p->goff[density];
  const int G = static_cast<int>(p->koff[density + 1] - p->koff[density]);
  const int threads = 256;
  const int64_t grid = std::min<int64_t>((n + threads - 1) / threads, 148 * 32);
  batch_quantile_kernel<<<static_cast<int>(grid), threads, 0, st>>>(
      rec, guide, p->gbits[density], G, (flags & kNonMonotone) != 0, u, n, x, intervals);
  return cudaGetLastError() == cudaSuccess ? LOITS_OK : LOITS_ERR_CUDA;
}
