// engines.cu -- engine selection for 31-bit plans.
#include <cstdlib>
#include <cstring>

#include "../../include/ntt_b200.h"
#include "engines.hpp"

namespace nttb {

static int env_engine() {
    const char* e = std::getenv("NTT_B200_ENGINE");
    if (!e) return NTTB_ENGINE_AUTO;
    if (!std::strcmp(e, "scalar")) return NTTB_ENGINE_SCALAR;
    if (!std::strcmp(e, "dmma")) return NTTB_ENGINE_DMMA;
    if (!std::strcmp(e, "int8")) return NTTB_ENGINE_INT8;
    if (!std::strcmp(e, "tiles")) return NTTB_ENGINE_TILES;
    return NTTB_ENGINE_AUTO;
}

// The INT8 cluster kernel gives each (polynomial, limb) unit four SMs; AUTO
// takes it from kInt8MinUnits units on, below which the CUDA-core engine,
// which spreads one polynomial over the whole GPU, is faster (uint64 words at
// 2^16: 13 - 17 us for 1 - 4 polynomials against 21 us; 25 against 21 us for 8).
constexpr uint64_t kInt8MinUnits = 8;
// The batch queue's tensor tiles take sizes 2^17 .. 2^20 once a call holds
// 2^20 residues: single forward transforms of BabyBear words, CUDA events
// over 200 calls, tiles / CUDA-core engine in us: 1 x 2^20 26.4 / 33.8,
// 4 x 2^18 23.6 / 32.7, 4 x 2^20 51.2 / 81.9; below that the CUDA-core
// engine, which spreads a call over the whole GPU with less set-up, is as
// fast or faster (4 x 2^17 22.5 / 22.6, 1 x 2^19 24.4 / 22.5).
constexpr uint32_t kTilesMinLog = 17;
constexpr uint64_t kTilesMinResidues = 1ull << 20;

int auto_engine32(const Plan32& p, bool src_u64, uint64_t units) {
    if (int8_serves(p, src_u64) && units >= kInt8MinUnits) return NTTB_ENGINE_INT8;
    if (tiles_serve(p) && p.log_n >= kTilesMinLog && (units << p.log_n) >= kTilesMinResidues) return NTTB_ENGINE_TILES;
    return NTTB_ENGINE_SCALAR;
}

int run_transform32(Plan32& p, const void* src, void* dst, bool src_u64, uint32_t n_polys, bool inverse,
                    int engine, cudaStream_t s) {
    if (engine == NTTB_ENGINE_AUTO) engine = env_engine();
    if (engine == NTTB_ENGINE_AUTO) engine = auto_engine32(p, src_u64, (uint64_t)n_polys * p.n_limbs);
    switch (engine) {
        case NTTB_ENGINE_SCALAR:
            return scalar_transform32(p, src, dst, src_u64, n_polys, inverse, s);
        case NTTB_ENGINE_INT8:
            return int8_transform32(p, src, dst, src_u64, n_polys, inverse, s);
        case NTTB_ENGINE_DMMA:
            return dmma_transform32(p, src, dst, src_u64, n_polys, inverse, s);
        case NTTB_ENGINE_TILES:
            return tiles_transform32(p, src, dst, src_u64, n_polys, inverse, s);
        default:
            return 1;
    }
}

void engines_release32(Plan32* p) {
    int8_release(p);
    dmma_release(p);
    tiles_release(p);
}

}  // namespace nttb
