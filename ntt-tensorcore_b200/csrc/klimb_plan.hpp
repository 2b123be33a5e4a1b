// klimb_plan.hpp -- the pass plan of the K-limb forward transform
// (csrc/klimb.cu), host-only so that it can be checked on the CPU.
//
// A transform of 2^log_n elements runs either as one tile in one launch (the
// bit reversal fused into the loads), or as a tiled bit reversal followed by
// passes of radix-2 DIT stages: pass i runs stages s0 .. s0 + r - 1 on tiles
// of 2^(r + logC) elements (2^logC columns of 2^r-element groups, logC <= s0).
// Tiles hold at most 2^log_emax elements, 48 KB of shared memory at the
// largest; log_emax shrinks while a pass would have fewer than 148 tiles
// (small transforms are bound by the latency of their stage chains, so more,
// shorter tiles win), but not below 2^6.
#pragma once

#include <cstdint>

namespace nttb {

struct KlimbPass {
    uint32_t s0, r, logC;
};

struct KlimbPlan {
    bool single_tile = false;  // one launch, bit reversal fused
    uint32_t log_emax = 0;     // largest tile of the stage passes
    uint32_t n_passes = 0;
    KlimbPass pass[24];
};

constexpr uint32_t kKlimbTargetCtas = 148;

// K: limbs per element (2, 3 or 11); log_n <= 24
inline KlimbPlan klimb_plan(uint32_t K, uint32_t log_n) {
    KlimbPlan P;
    const uint32_t n = 1u << log_n;
    uint32_t log_emax = K <= 3 ? 12u : 10u;
    while (log_emax > 6 && (n >> log_emax) < kKlimbTargetCtas) log_emax--;
    P.log_emax = log_emax;
    // measured: K <= 3 up to 2^10, K = 11 up to 2^8 are fastest as one tile
    P.single_tile = log_n <= (K <= 3 ? 10u : 8u);
    if (P.single_tile) return P;
    uint32_t s0 = 0;
    while (s0 < log_n) {
        uint32_t r = log_n - s0, logC = 0;
        if (s0 == 0) {
            if (r > log_emax) r = log_emax;
        } else {
            if (r > 8) r = 8;
            if (r > log_emax) r = log_emax;
            logC = log_emax - r < s0 ? log_emax - r : s0;
        }
        P.pass[P.n_passes++] = {s0, r, logC};
        s0 += r;
    }
    return P;
}

}  // namespace nttb
