// lookback.cuh -- single-pass decoupled look-back prefix for ordered tiles.
//
// Tile t publishes its aggregate (kept-event count) as soon as it is known,
// then walks back over its predecessors, 32 at a time with one warp, until it
// meets an inclusive prefix; it then publishes its own inclusive prefix.
// Tiles are handed out in increasing order (an atomic ticket), so every tile a
// wait depends on is already held by a running CTA.  Each poll is bounded: a
// wait that runs out records LOITS_ERR_TIMEOUT, and the tile still publishes
// an inclusive prefix so that no successor waits on it.
#pragma once

#include "common.cuh"

namespace loits_dev {

constexpr unsigned long long kFlagAggregate = 1ull << 62;
constexpr unsigned long long kFlagInclusive = 2ull << 62;
constexpr unsigned long long kValueMask = (1ull << 62) - 1;

// Called by every lane of ONE warp.  Returns the exclusive prefix of `tile`.
// limit: polls of one predecessor before the wait gives up.  publish = false
// leaves the tile's own state unpublished, so that its successors' waits run
// out (a test of the bounded waits; never set in sampling).
__device__ __forceinline__ int64_t lookback_exclusive(unsigned long long* states, int64_t tile,
                                                      uint64_t count, int32_t* status,
                                                      uint32_t limit = kSpinLimit,
                                                      bool publish = true) {
  const int lane = threadIdx.x & 31;
  if (tile == 0) {
    if (lane == 0 && publish) st_release_u64(&states[0], kFlagInclusive | count);
    return 0;
  }
  if (lane == 0 && publish) st_release_u64(&states[tile], kFlagAggregate | count);
  uint64_t excl = 0;
  int64_t base = tile - 1;
  uint32_t polls = 0;
  bool timed_out = false;
  while (base >= 0) {
    const int64_t idx = base - lane;
    const unsigned long long s = idx >= 0 ? ld_acquire_u64(&states[idx]) : kFlagInclusive;
    const unsigned long long flag = s & ~kValueMask;
    if (__any_sync(0xffffffffu, flag == 0)) {
      if (++polls >= limit ||
          ((polls & 63u) == 0u && __any_sync(0xffffffffu, launch_timed_out(status)))) {
        timed_out = true;
        break;
      }
      spin_pause(polls);
      continue;
    }
    const unsigned inc = __ballot_sync(0xffffffffu, flag == kFlagInclusive);
    const int first = inc ? __ffs(inc) - 1 : 32;
    const uint64_t v = lane <= first ? (s & kValueMask) : 0;
    excl += warp_sum(v);
    if (inc) break;
    base -= 32;
  }
  if (timed_out && lane == 0) raise_status(status, LOITS_ERR_TIMEOUT);
  if (lane == 0 && publish)
    st_release_u64(&states[tile], kFlagInclusive | ((excl + count) & kValueMask));
  return static_cast<int64_t>(excl);
}

}  // namespace loits_dev
