// sfd_selftest.cpp -- host-only checks of the library's shared host state,
// callable without a GPU.
#include <atomic>
#include <cstdint>
#include <thread>
#include <vector>

#include "seiscl_b200.h"
#include "sfd_cache.h"

namespace {

// A value large enough that a torn or dangling copy shows: every word is a
// function of the key.
struct Payload {
    int64_t w[1024];
};

int64_t word(int key, int i) { return (int64_t)key * 1000003 + i; }

}  // namespace

// Hammers a KeyedCache of the kind that holds the TMA tensor maps from
// `nthreads` threads, `iters` lookups each over 3x more keys than the cache
// holds (so entries are evicted and rebuilt all the time), and checks every
// copied-out value.  Returns the number of bad copies (0 when the cache is
// sound).
extern "C" int64_t sfd_selftest_cache(int nthreads, int iters)
{
    if (nthreads <= 0 || iters <= 0) return SFD_ERR_ARG;
    sfd::KeyedCache<int, Payload, 16> cache;
    std::atomic<int64_t> bad{0};
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; t++)
        th.emplace_back([&, t] {
            uint32_t s = 2654435761u * (uint32_t)(t + 1);
            for (int it = 0; it < iters; it++) {
                s = s * 1664525u + 1013904223u;
                const int key = (int)(s >> 8) % 48;
                Payload out;
                cache.with(
                    key,
                    [&](Payload &p) {
                        for (int i = 0; i < 1024; i++) p.w[i] = word(key, i);
                    },
                    [&](const Payload &p) {
                        out = p;
                        return 0;
                    });
                for (int i = 0; i < 1024; i += 37)
                    if (out.w[i] != word(key, i)) {
                        bad++;
                        break;
                    }
            }
        });
    for (auto &x : th) x.join();
    if (cache.size() > 16) bad++;
    return bad.load();
}
