// arena.hpp -- first-fit allocator over one device region, in 256-byte
// granules, coalescing free neighbours on release.  Host-only bookkeeping of
// offsets (no CUDA calls): the serving loop carves request operands out of
// its HBM region with it, under the server's lock.
#pragma once

#include <algorithm>
#include <cstddef>
#include <iterator>
#include <map>

namespace nttb {

constexpr size_t kGranule = 256;
inline size_t round_up(size_t x) { return (x + kGranule - 1) / kGranule * kGranule; }

class Arena {
   public:
    void init(size_t bytes) {
        size_ = bytes / kGranule * kGranule;
        free_.clear();
        used_ = peak_ = 0;
        if (size_) free_[0] = size_;
    }
    // lowest-offset free run that holds `bytes` (rounded up to a granule)
    bool alloc(size_t bytes, size_t* off) {
        bytes = round_up(bytes);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            const size_t o = it->first, rest = it->second - bytes;
            free_.erase(it);
            if (rest) free_[o + bytes] = rest;
            *off = o;
            used_ += bytes;
            peak_ = std::max(peak_, used_);
            return true;
        }
        return false;
    }
    // `off` and `bytes` exactly as one earlier alloc returned and was asked
    void release(size_t off, size_t bytes) {
        bytes = round_up(bytes);
        used_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    size_t size() const { return size_; }
    size_t used() const { return used_; }
    size_t peak() const { return peak_; }
    size_t free_runs() const { return free_.size(); }

   private:
    std::map<size_t, size_t> free_;  // offset -> length of each free run
    size_t size_ = 0, used_ = 0, peak_ = 0;
};

}  // namespace nttb
