// sfd_cache.h -- a small keyed cache shared between threads.
//
// Entries are built once per key and read under the cache's lock: a reader
// copies what it needs out of the entry before the lock is released, so an
// insertion or eviction by another thread (which may move or destroy
// entries) can never leave a caller holding a pointer into the cache.
#pragma once

#include <cstddef>
#include <deque>
#include <mutex>
#include <utility>

namespace sfd {

template <class K, class V, std::size_t CAP>
class KeyedCache {
public:
    // Runs read(entry) under the lock on the entry of `key`, building it
    // first with build(entry) when absent; returns what read returns.  The
    // oldest entry is evicted when the cache holds CAP entries.
    template <class Build, class Read>
    auto with(const K &key, Build build, Read read) -> decltype(read(std::declval<const V &>()))
    {
        std::lock_guard<std::mutex> lk(mu_);
        for (auto &e : items_)
            if (e.first == key) return read(static_cast<const V &>(e.second));
        if (items_.size() >= CAP) items_.pop_front();
        items_.emplace_back(key, V{});
        build(items_.back().second);
        return read(static_cast<const V &>(items_.back().second));
    }
    std::size_t size()
    {
        std::lock_guard<std::mutex> lk(mu_);
        return items_.size();
    }

private:
    std::mutex mu_;
    std::deque<std::pair<K, V>> items_;
};

}  // namespace sfd
