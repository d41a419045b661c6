// Host-side range allocator of the serving loop's device pools (pure C++,
// no CUDA types, so the CPU tests compile it on its own).
#pragma once
#include <algorithm>
#include <iterator>
#include <map>

namespace nsb {

// First-fit free list over [0, capacity) with coalescing.
class RangeAllocator {
public:
    explicit RangeAllocator(long long capacity = 0) { reset(capacity); }
    void reset(long long capacity) {
        free_.clear();
        cap_ = capacity;
        used_ = 0;
        if (capacity > 0) free_[0] = capacity;
    }
    // Start of a free range of length n, or -1.
    long long allocate(long long n) {
        if (n <= 0) return -1;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            const long long start = it->first, len = it->second;
            free_.erase(it);
            if (len > n) free_[start + n] = len - n;
            used_ += n;
            return start;
        }
        return -1;
    }
    void release(long long start, long long n) {
        if (n <= 0) return;
        used_ -= n;
        auto next = free_.lower_bound(start);
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == start) {
                start = prev->first;
                n += prev->second;
                free_.erase(prev);
            }
        }
        next = free_.lower_bound(start);
        if (next != free_.end() && start + n == next->first) {
            n += next->second;
            free_.erase(next);
        }
        free_[start] = n;
    }
    long long used() const { return used_; }
    long long capacity() const { return cap_; }
    long long largest() const {
        long long m = 0;
        for (auto &kv : free_) m = std::max(m, kv.second);
        return m;
    }
    size_t fragments() const { return free_.size(); }

private:
    std::map<long long, long long> free_;
    long long cap_ = 0, used_ = 0;
};

}  // namespace nsb
