// budget.cpp -- the per-device VRAM budget of the reference (source/budget.cpp:15-51),
// used here as the admission model of the serving loop.
//
//   budget   = min(floor(f * free), cap)
//   scratch  = fixed, else min(floor(0.15 * budget), 1 GiB)
//   backing  = budget - scratch - 64 MiB headroom, floored to 4 KiB (0 when that underflows)
//   slabs    = floor(backing / slab size)
//
// and the allocation-failure step: one midpoint move of f toward the 0.50 floor.
#include <algorithm>
#include <cstdint>

#include "ffb200.h"

namespace {

constexpr unsigned long long kGranularity = 4096;            // backing floor granularity
constexpr unsigned long long kHeadroom = 64ull << 20;        // always reserved
constexpr unsigned long long kAutoScratchCap = 1ull << 30;   // min(0.15 x budget, 1 GiB)
constexpr double kFloorFraction = 0.50;

}  // namespace

extern "C" int ffb_compute_budget(uint64_t freeBytes, double fraction, uint64_t capBytes,
                                  uint64_t scratchBytes, uint64_t slabBytes, FfbBudget* out)
{
    if (!out || !(fraction > 0.0) || fraction > 1.0) return -1;
    FfbBudget b{};
    b.fraction = fraction;
    b.freeQueried = freeBytes;
    b.freeUsed = static_cast<unsigned long long>(fraction * double(freeBytes));
    b.cap = capBytes ? capBytes : ~0ull;
    b.budget = std::min<unsigned long long>(b.freeUsed, b.cap);
    b.scratch = scratchBytes ? scratchBytes
                             : std::min(static_cast<unsigned long long>(0.15 * double(b.budget)),
                                        kAutoScratchCap);
    b.headroom = kHeadroom;
    unsigned long long backing = 0;
    if (b.budget > b.scratch) {
        const unsigned long long after = b.budget - b.scratch;
        if (after > b.headroom) backing = after - b.headroom;
    }
    backing -= backing % kGranularity;
    b.backing = backing;
    b.slabCount = slabBytes ? backing / slabBytes : 0;
    *out = b;
    return 0;
}

extern "C" int ffb_shrink_budget(uint64_t freeBytes, double fraction, uint64_t capBytes,
                                 uint64_t scratchBytes, uint64_t slabBytes, FfbBudget* out)
{
    const double next = fraction <= kFloorFraction ? kFloorFraction
                                                   : 0.5 * (fraction + kFloorFraction);
    return ffb_compute_budget(freeBytes, next, capBytes, scratchBytes, slabBytes, out);
}
