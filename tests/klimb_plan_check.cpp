// CPU check of the K-limb pass plan (csrc/klimb_plan.hpp) for K = 2, 3, 11
// and every log_n up to 24: the passes cover the stages 0 .. log_n - 1 once
// and in order, every tile fits its launch (at most 48 KB of shared memory,
// no more elements than the transform has, logC <= s0 so that a pass's
// column chunks exist), and small transforms are a single tile.
// Built and run by tests/test_host_cpp.py; prints "ok" and exits 0 on success.
#include <cstdio>
#include <initializer_list>

#include "klimb_plan.hpp"

namespace {

int fails = 0;
void expect(bool c, const char* what, unsigned K, unsigned lg) {
    if (!c && fails++ < 20) std::printf("FAIL K=%u log_n=%u: %s\n", K, lg, what);
}

}  // namespace

int main() {
    constexpr unsigned long kSmem = 48 * 1024;
    for (unsigned K : {2u, 3u, 11u}) {
        for (unsigned lg = 1; lg <= 24; lg++) {
            const nttb::KlimbPlan P = nttb::klimb_plan(K, lg);
            const unsigned long n = 1ul << lg;
            expect(P.single_tile == (lg <= (K <= 3 ? 10u : 8u)), "single tile exactly for small transforms", K, lg);
            if (P.single_tile) {
                expect(n * K * 4 <= kSmem, "single tile fits shared memory", K, lg);
                expect(P.n_passes == 0, "no stage passes after a single tile", K, lg);
                continue;
            }
            expect(P.log_emax >= 6 && P.log_emax <= (K <= 3 ? 12u : 10u), "tile bound in range", K, lg);
            expect(P.n_passes >= 1 && P.n_passes <= 24, "pass count", K, lg);
            unsigned s0 = 0;
            for (unsigned i = 0; i < P.n_passes; i++) {
                const nttb::KlimbPass& q = P.pass[i];
                expect(q.s0 == s0, "passes are consecutive", K, lg);
                expect(q.r >= 1, "every pass runs a stage", K, lg);
                expect(i == 0 || q.r <= 8, "later passes run at most 8 stages", K, lg);
                expect(q.r <= P.log_emax, "stages per pass within the tile bound", K, lg);
                expect(q.logC <= q.s0, "column chunks exist", K, lg);
                const unsigned long E = 1ul << (q.r + q.logC);
                expect(E <= (1ul << P.log_emax), "tile within the bound", K, lg);
                expect(E * K * 4 <= kSmem, "tile fits shared memory", K, lg);
                expect(E <= n && n % E == 0, "whole tiles", K, lg);
                expect(E >= 2, "a tile holds a butterfly", K, lg);
                s0 += q.r;
            }
            expect(s0 == lg, "stages covered exactly once", K, lg);
            // tiles shrink only while a pass would otherwise have under 148 of them
            if (P.log_emax < (K <= 3 ? 12u : 10u) && P.log_emax > 6)
                expect((n >> P.log_emax) >= nttb::kKlimbTargetCtas && (n >> (P.log_emax + 1)) < nttb::kKlimbTargetCtas,
                       "tile bound is the largest with 148 tiles", K, lg);
        }
    }
    if (fails) {
        std::printf("%d failures\n", fails);
        return 1;
    }
    std::printf("ok\n");
    return 0;
}
