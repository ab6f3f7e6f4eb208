// Hard-path kernels for one precision (NWG_T: float or double), every compiled geometry.
#include "nwg_kernels.h"

namespace nwg {
namespace {
template <class T, bool AFF, bool LOC, bool TR>
HardFn pick_band(Geo g) {
    if (g.G == 32 && g.R == 1) return &hard_fill_kernel<T, AFF, LOC, TR, 32, 1, true>;
    if (g.G == 32 && g.R == 2) return &hard_fill_kernel<T, AFF, LOC, TR, 32, 2, true>;
    return nullptr;
}
// semi-global ends: their own instantiations, so the Global fills carry none of their state
template <class T, bool AFF, bool TR>
HardFn pick_sg(Geo g) {
    if (g.band) {   // glocal ends, banded re-alignment
        if (g.G == 32 && g.R == 1) return &hard_fill_kernel<T, AFF, false, TR, 32, 1, true, true>;
        if (g.G == 32 && g.R == 2) return &hard_fill_kernel<T, AFF, false, TR, 32, 2, true, true>;
        return nullptr;
    }
    if (g.mw > 1 || g.tile) return nullptr;
#define NWG_H(GG, RR) if (g.G == GG && g.R == RR) return &hard_fill_kernel<T, AFF, false, TR, GG, RR, false, true>;
    NWG_H(1, 8) NWG_H(1, 16) NWG_H(1, 24) NWG_H(1, 32) NWG_H(32, 1) NWG_H(32, 2) NWG_H(32, 4) NWG_H(32, 8)
#undef NWG_H
    return nullptr;
}
template <class T, bool AFF, bool LOC, bool TR>
HardFn pick(Geo g) {
    if (g.band) return pick_band<T, AFF, LOC, TR>(g);
    if (g.tile) {
        if (g.G != 32 || g.R != 8) return nullptr;
        if (g.grid) return &hard_fill_kernel<T, AFF, LOC, TR, 32, 8, false, false, true, true>;
        return &hard_fill_kernel<T, AFF, LOC, TR, 32, 8, false, false, true>;
    }
    if (g.mw > 1) return nullptr;
#define NWG_H(GG, RR) if (g.G == GG && g.R == RR) return &hard_fill_kernel<T, AFF, LOC, TR, GG, RR>;
    NWG_H(1, 8) NWG_H(1, 16) NWG_H(1, 24) NWG_H(1, 32) NWG_H(32, 1) NWG_H(32, 2) NWG_H(32, 4) NWG_H(32, 8)
#undef NWG_H
    return nullptr;
}
}  // namespace

HardFn NWG_HARD_FN(bool aff, int am, bool tr, Geo g) {
    using T = NWG_T;
    const bool loc = am == 1;
    if (am == 2) {
        if (aff) return tr ? pick_sg<T, true, true>(g) : pick_sg<T, true, false>(g);
        return tr ? pick_sg<T, false, true>(g) : pick_sg<T, false, false>(g);
    }
    if (aff) {
        if (loc) return tr ? pick<T, true, true, true>(g) : pick<T, true, true, false>(g);
        return tr ? pick<T, true, false, true>(g) : pick<T, true, false, false>(g);
    }
    if (loc) return tr ? pick<T, false, true, true>(g) : pick<T, false, true, false>(g);
    return tr ? pick<T, false, false, true>(g) : pick<T, false, false, false>(g);
}
}  // namespace nwg
