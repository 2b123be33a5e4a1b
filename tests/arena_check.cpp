// CPU check of the serving loop's device-region allocator (csrc/arena.hpp)
// against a granule bitmap: every allocation lands at the lowest offset
// whose free run holds it, allocations never overlap, the used and peak
// counters follow, and releasing everything leaves one free run.
// Built and run by tests/test_host_cpp.py; prints "ok" and exits 0 on success.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "arena.hpp"

namespace {

int fails = 0;
void expect(bool c, const char* what, long a, long b) {
    if (!c && fails++ < 10) std::printf("FAIL %s (%ld vs %ld)\n", what, a, b);
}

// lowest granule index that starts a run of `g` free granules, or -1
long model_first_fit(const std::vector<char>& used, size_t g) {
    size_t run = 0;
    for (size_t i = 0; i < used.size(); i++) {
        run = used[i] ? 0 : run + 1;
        if (run == g) return (long)(i + 1 - g);
    }
    return -1;
}

}  // namespace

int main() {
    using nttb::Arena;
    using nttb::kGranule;
    std::mt19937_64 rng(20261204);
    for (int trial = 0; trial < 20; trial++) {
        const size_t granules = 64 + rng() % 960;
        Arena a;
        a.init(granules * kGranule + rng() % kGranule);  // a ragged size rounds down
        expect(a.size() == granules * kGranule, "size rounds down to granules", (long)a.size(), (long)granules);
        std::vector<char> used(granules, 0);
        struct Live { size_t off, bytes; };
        std::vector<Live> live;
        size_t in_use = 0, peak = 0;
        for (int step = 0; step < 4000; step++) {
            if (live.empty() || rng() % 100 < 55) {
                const size_t bytes = 1 + rng() % (kGranule * (1 + rng() % 48));
                const size_t g = (bytes + kGranule - 1) / kGranule;
                const long want = model_first_fit(used, g);
                size_t off = 0;
                const bool ok = a.alloc(bytes, &off);
                expect(ok == (want >= 0), "alloc succeeds exactly when a run fits", ok, want);
                if (!ok) continue;
                expect(off % kGranule == 0, "granule aligned", (long)off, 0);
                expect((long)(off / kGranule) == want, "first fit", (long)(off / kGranule), want);
                for (size_t i = off / kGranule; i < off / kGranule + g; i++) {
                    expect(!used[i], "no overlap", (long)i, 0);
                    used[i] = 1;
                }
                live.push_back({off, bytes});
                in_use += g * kGranule;
                peak = in_use > peak ? in_use : peak;
            } else {
                const size_t k = rng() % live.size();
                const Live l = live[k];
                live[k] = live.back();
                live.pop_back();
                a.release(l.off, l.bytes);
                const size_t g = (l.bytes + kGranule - 1) / kGranule;
                for (size_t i = l.off / kGranule; i < l.off / kGranule + g; i++) used[i] = 0;
                in_use -= g * kGranule;
            }
            expect(a.used() == in_use, "used bytes", (long)a.used(), (long)in_use);
            expect(a.peak() == peak, "peak bytes", (long)a.peak(), (long)peak);
        }
        for (const Live& l : live) a.release(l.off, l.bytes);
        expect(a.used() == 0, "all released", (long)a.used(), 0);
        expect(a.free_runs() == 1, "free runs coalesce into one", (long)a.free_runs(), 1);
        size_t off = 1;
        expect(a.alloc(a.size(), &off) && off == 0, "the whole region fits again", (long)off, 0);
    }
    Arena empty;
    empty.init(kGranule - 1);
    size_t off = 0;
    expect(empty.size() == 0 && !empty.alloc(1, &off), "a region under one granule holds nothing", 0, 0);
    if (fails) {
        std::printf("%d failures\n", fails);
        return 1;
    }
    std::printf("ok\n");
    return 0;
}
