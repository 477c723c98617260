/*
 * lt_arena.h -- first-fit sub-allocator over one device allocation: the serving loop's
 * admission budget.  Host-only bookkeeping (offsets, no device access), so it is
 * unit-tested without a GPU.
 *
 * A request is admitted only when its output planes fit in the arena; it waits in the
 * queue otherwise, and its bytes return to the arena when its results have been copied
 * out.  Adjacent free ranges are merged on release.
 */
#pragma once
#include <cstddef>
#include <cstdint>
#include <iterator>
#include <map>

namespace lt {

class Arena {
public:
    static constexpr size_t kAlign = 256;
    static constexpr size_t kFail = ~(size_t)0;

    explicit Arena(size_t bytes = 0) { reset(bytes); }

    void reset(size_t bytes)
    {
        free_.clear();
        used_.clear();
        size_ = bytes / kAlign * kAlign;
        in_use_ = peak_ = 0;
        if (size_) free_[0] = size_;
    }

    static size_t round(size_t n) { return (n + kAlign - 1) / kAlign * kAlign; }

    /* Offset of a block of at least n bytes, or kFail. */
    size_t alloc(size_t n)
    {
        n = round(n ? n : 1);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            const size_t off = it->first, len = it->second;
            free_.erase(it);
            if (len > n) free_[off + n] = len - n;
            used_[off] = n;
            in_use_ += n;
            if (in_use_ > peak_) peak_ = in_use_;
            return off;
        }
        return kFail;
    }

    /* Return the block at `off`; false if no block starts there. */
    bool release(size_t off)
    {
        auto u = used_.find(off);
        if (u == used_.end()) return false;
        size_t len = u->second;
        used_.erase(u);
        in_use_ -= len;
        auto next = free_.lower_bound(off);
        if (next != free_.end() && off + len == next->first) {
            len += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                prev->second += len;
                return true;
            }
        }
        free_[off] = len;
        return true;
    }

    size_t size() const { return size_; }
    size_t in_use() const { return in_use_; }
    size_t peak() const { return peak_; }
    size_t largest_free() const
    {
        size_t m = 0;
        for (const auto &f : free_)
            if (f.second > m) m = f.second;
        return m;
    }
    size_t free_ranges() const { return free_.size(); }

private:
    std::map<size_t, size_t> free_; /* offset -> length */
    std::map<size_t, size_t> used_;
    size_t size_ = 0, in_use_ = 0, peak_ = 0;
};

} // namespace lt
