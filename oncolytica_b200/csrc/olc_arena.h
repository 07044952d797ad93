// Host-side range allocator for the serving pool's device arenas (field
// voxels, bin-table entries).  A simulation admitted to the pool takes one
// contiguous range of each arena; retiring it returns the ranges.  Free ranges
// are kept ordered by offset and merged with their neighbours on release;
// allocation is best fit (the smallest free range that holds the request,
// lowest offset on ties), which keeps large ranges whole for large members.
// No counterpart in the reference (one simulation per engine, buffers sized
// once at load).
#pragma once

#include <cstdint>
#include <iterator>
#include <map>

namespace olc {

class RangeArena {
public:
    static constexpr uint64_t NONE = ~0ull;

    void reset(uint64_t capacity) {
        cap_ = capacity;
        used_ = 0;
        free_.clear();
        taken_.clear();
        if (capacity) free_[0] = capacity;
    }

    uint64_t capacity() const { return cap_; }
    uint64_t used() const { return used_; }

    uint64_t largest_free() const {
        uint64_t best = 0;
        for (const auto& r : free_)
            if (r.second > best) best = r.second;
        return best;
    }

    // Offset of a range of `n` units whose start is a multiple of `align`
    // (a power of two), or NONE.  The alignment padding stays free.
    uint64_t alloc(uint64_t n, uint64_t align = 1) {
        if (n == 0) return NONE;
        auto best = free_.end();
        uint64_t best_start = 0, best_len = ~0ull;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            const uint64_t start = (it->first + align - 1) & ~(align - 1);
            const uint64_t pad = start - it->first;
            if (it->second < pad || it->second - pad < n) continue;
            if (it->second < best_len) {
                best = it;
                best_start = start;
                best_len = it->second;
            }
        }
        if (best == free_.end()) return NONE;
        const uint64_t off = best->first, len = best->second;
        free_.erase(best);
        if (best_start > off) free_[off] = best_start - off;
        const uint64_t end = best_start + n;
        if (off + len > end) free_[end] = off + len - end;
        used_ += n;
        taken_[best_start] = n;
        return best_start;
    }

    // Returns [off, off + n) to the free list; false unless it is exactly one
    // range that alloc() returned and that is still allocated (double free,
    // part of a range, out of range).
    bool release(uint64_t off, uint64_t n) {
        auto t = taken_.find(off);
        if (t == taken_.end() || t->second != n) return false;
        taken_.erase(t);
        auto next = free_.lower_bound(off);
        uint64_t start = off, len = n;
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                start = prev->first;
                len += prev->second;
                free_.erase(prev);
            }
        }
        if (next != free_.end() && next->first == off + n) {
            len += next->second;
            free_.erase(next);
        }
        free_[start] = len;
        used_ -= n;
        return true;
    }

    size_t free_ranges() const { return free_.size(); }

private:
    uint64_t cap_ = 0;
    uint64_t used_ = 0;
    std::map<uint64_t, uint64_t> free_;   // offset -> length of free ranges
    std::map<uint64_t, uint64_t> taken_;  // offset -> length of allocated ranges
};

}  // namespace olc
