// Kernel entry tables: the argument blocks and, per precision, the instantiated kernels for
// each (gap model, mode, tracked, geometry).  The kernels live in nwg_hard_inst.cu and
// nwg_soft_inst.cu (compiled once per precision), the host logic in nwg_capi.cu.
#pragma once
#include "nwg_common.cuh"
#include "nwg_hard.cuh"
#include "nwg_soft.cuh"

namespace nwg {
using HardFn = void (*)(const HardArgs);
using SoftFn = void (*)(const SoftArgs);
// mw > 1: that many warps per pair (soft); post: the posterior-guide kernels (32 x 4, full DP,
// untracked); tile: the hard fill over tiles of long pairs (32 x 8, a launch per anti-diagonal);
// grid (with tile): the grid traceback's walk, which refills the tiles its path crosses
struct Geo { int G, R; bool band = false; int mw = 0; bool post = false; bool tile = false; bool grid = false; };
// am: 0 Global, 1 Local, 2 semi-global ends (full DP, one warp or lane per pair)
HardFn hard_fn_f32(bool aff, int am, bool tr, Geo g);
HardFn hard_fn_f64(bool aff, int am, bool tr, Geo g);
// soft: one table per end mode (0 Global, 1 Local, 2 semi-global ends)
SoftFn soft_fn_f32_am0(bool aff, bool tr, Geo g);
SoftFn soft_fn_f32_am1(bool aff, bool tr, Geo g);
SoftFn soft_fn_f32_am2(bool aff, bool tr, Geo g);
SoftFn soft_fn_f64_am0(bool aff, bool tr, Geo g);
SoftFn soft_fn_f64_am1(bool aff, bool tr, Geo g);
SoftFn soft_fn_f64_am2(bool aff, bool tr, Geo g);
}  // namespace nwg
