// Randomised check of lt::Arena (the serving loop's admission budget) against a
// byte-map model: blocks never overlap, stay inside the arena, and freeing every block
// merges the free list back into one range.  Prints "ok" on success.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "lt_arena.h"

int main(int argc, char **argv)
{
    const unsigned seed = argc > 1 ? (unsigned)atoi(argv[1]) : 1u;
    std::mt19937_64 rng(seed);
    const size_t size = 1 << 20;
    lt::Arena a(size);
    std::vector<unsigned char> owner(size, 0);
    std::vector<std::pair<size_t, size_t>> live;
    for (int step = 0; step < 20000; step++) {
        if (live.empty() || rng() % 3) {
            const size_t n = 1 + rng() % 40000;
            const size_t off = a.alloc(n);
            if (off == lt::Arena::kFail) {
                if (a.largest_free() >= lt::Arena::round(n)) { printf("alloc failed with room\n"); return 1; }
                continue;
            }
            const size_t len = lt::Arena::round(n);
            if (off % lt::Arena::kAlign || off + len > size) { printf("bad block\n"); return 1; }
            for (size_t i = off; i < off + len; i++) {
                if (owner[i]) { printf("overlap at %zu\n", i); return 1; }
                owner[i] = 1;
            }
            live.push_back({off, len});
        } else {
            const size_t k = rng() % live.size();
            const auto b = live[k];
            live[k] = live.back();
            live.pop_back();
            if (!a.release(b.first)) { printf("release failed\n"); return 1; }
            for (size_t i = b.first; i < b.first + b.second; i++) owner[i] = 0;
        }
        size_t used = 0;
        for (auto &b : live) used += b.second;
        if (used != a.in_use() || a.peak() > size) { printf("accounting\n"); return 1; }
    }
    if (a.release(12345)) { printf("released a block that does not exist\n"); return 1; }
    for (auto &b : live) a.release(b.first);
    if (a.in_use() != 0 || a.free_ranges() != 1 || a.largest_free() != size) { printf("no merge\n"); return 1; }
    printf("ok\n");
    return 0;
}
