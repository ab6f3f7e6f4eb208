// Soft-path kernels for one precision (NWG_T: float or double) and one end mode (NWG_SOFT_AM:
// 0 Global, 1 Local, 2 semi-global ends), every compiled geometry.  One translation unit per
// (precision, mode) so the units compile in parallel.
#include "nwg_kernels.h"

namespace nwg {
namespace {
// SG: the semi-global ends (Global kernels, full DP), their own instantiations so the Global
// kernels test no end flag per cell
template <class T, bool AFF, bool LOC, bool TR, bool SG = false>
SoftFn pick(Geo g) {
    if (g.post) {
        if constexpr (!TR) {
            if (g.G == 32 && g.R == 4 && !g.band && g.mw <= 1)
                return &soft_kernel<T, AFF, LOC, false, 32, 4, false, false, SG, true>;
        }
        return nullptr;
    }
    if (g.band) return (g.G == 32 && g.R == 4 && g.mw <= 1) ? &soft_kernel<T, AFF, LOC, TR, 32, 4, false, true, SG> : nullptr;
    if (g.tile) {   // tiled long pairs: untracked, Global or Local
        if constexpr (!TR && !SG) {
            if (g.G == 32 && g.R == 4) return &soft_kernel<T, AFF, LOC, false, 32, 4, false, false, false, false, true>;
        }
        return nullptr;
    }
    if constexpr (!TR) {
        if (g.mw > 1) return (g.G == 32 && g.R == 4) ? &soft_kernel<T, AFF, LOC, false, 32, 4, true, false, SG> : nullptr;
    } else {
        if (g.mw > 1) return nullptr;
    }
#define NWG_S(GG, RR) if (g.G == GG && g.R == RR) return &soft_kernel<T, AFF, LOC, TR, GG, RR, false, false, SG>;
    NWG_S(1, 8) NWG_S(1, 16) NWG_S(1, 24) NWG_S(1, 32) NWG_S(32, 2) NWG_S(32, 4)
    NWG_S(16, 2) NWG_S(16, 4) NWG_S(8, 4) NWG_S(16, 8) NWG_S(32, 8)
#undef NWG_S
    return nullptr;
}
}  // namespace

SoftFn NWG_SOFT_FN(bool aff, bool tr, Geo g) {
    using T = NWG_T;
#if NWG_SOFT_AM == 2
    if (aff) return tr ? pick<T, true, false, true, true>(g) : pick<T, true, false, false, true>(g);
    return tr ? pick<T, false, false, true, true>(g) : pick<T, false, false, false, true>(g);
#else
    constexpr bool loc = NWG_SOFT_AM == 1;
    if (aff) return tr ? pick<T, true, loc, true>(g) : pick<T, true, loc, false>(g);
    return tr ? pick<T, false, loc, true>(g) : pick<T, false, loc, false>(g);
#endif
}
}  // namespace nwg
