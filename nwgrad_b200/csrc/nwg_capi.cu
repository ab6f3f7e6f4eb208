// nwgrad_b200: the C ABI (include/nwgrad_b200.h) over the sm_100a kernels.
//
// The store keeps a batch resident in HBM: codes and offsets uploaded once, parameters cast
// to the DP precision once per set_params, per-pair results (scores, end cells, guides,
// gradients) kept on the device until read.  nwg_run plans the batch once per problem shape
// (pairs sorted into length buckets, each bucket a launch of one kernel geometry: one lane
// per pair for short pairs, one warp per pair otherwise) and replays the plan on every call.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <tuple>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/nwgrad_b200.h"
#include "nwg_hb.h"
#include "nwg_kernels.h"
#include "nwg_walk.cuh"

namespace nwg {
// The traceback of pairs filled by several warps each: one thread per pair, after the fills.
__global__ void walk_kernel(const WalkArgs A) {
    const int64_t it = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (it >= A.n_items) return;
    walk_pair(A, A.order[it]);
}
}  // namespace nwg

namespace {

thread_local std::string g_err;

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define NWG_CUDA(call)                                                                     \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            throw Error(e_ == cudaErrorMemoryAllocation ? NWG_ENOMEM : NWG_ECUDA,          \
                        std::string(#call) + ": " + cudaGetErrorString(e_));               \
    } while (0)

// A device buffer that only grows, from the device's stream-ordered memory pool (which keeps
// freed memory for reuse: a batch built after another reuses its blocks without a cudaMalloc).
// With a stream, need() and release() free and allocate in that stream's order; without one
// they wait for the whole device first, so no launch on any stream still uses the old block.
struct DBuf {
    void* p = nullptr;
    size_t bytes = 0;
    void need(size_t n, cudaStream_t st = nullptr) {
        if (n <= bytes) return;
        if (!st) NWG_CUDA(cudaDeviceSynchronize());
        if (p) cudaFreeAsync(p, st);
        p = nullptr; bytes = 0;
        const size_t want = std::max<size_t>(n + n / 8, 256);
        NWG_CUDA(cudaMallocAsync(&p, want, st));
        if (!st) NWG_CUDA(cudaStreamSynchronize(nullptr));
        bytes = want;
    }
    void release(cudaStream_t st = nullptr) {
        if (!p) return;
        if (!st) cudaDeviceSynchronize();
        cudaFreeAsync(p, st);
        if (!st) cudaStreamSynchronize(nullptr);
        p = nullptr; bytes = 0;
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

// The pool keeps what it frees (no release threshold): repeated batches reuse device memory.
void keep_pool(int dev) {
    static bool done[64] = {};
    if (dev < 0 || dev >= 64 || done[dev]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = ~uint64_t(0);
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    done[dev] = true;
}

// ── reductions ────────────────────────────────────────────────────────────────
// The reference's blocked sum: block b sums w[p] * g[p][k] over its pairs in pair order from
// 0.0 (a product, then an add: no fused multiply-add), then the blocks are added in order.
template <bool W>
__global__ void blocked_partial_kernel(const double* __restrict__ g, const double* __restrict__ w,
                                       int64_t n_pairs, int64_t gs, int64_t block, double* part) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t b = blockIdx.y;
    if (k >= gs) return;
    const int64_t p0 = b * block, p1 = min(n_pairs, p0 + block);
    double acc = 0.0;
    // the adds stay in pair order; the loads run a batch ahead (two register batches), so
    // 2U loads are in flight while U are added
    constexpr int U = 16;
    double va[U], vb[U], wa[W ? U : 1], wb[W ? U : 1];
    auto load = [&](double (&v)[U], double (&ww)[W ? U : 1], int64_t q) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            v[u] = g[(q + u) * gs + k];
            if constexpr (W) ww[u] = w[q + u];
        }
    };
    const int64_t nfull = (p1 - p0) / U;
    if (nfull > 0) load(va, wa, p0);
    for (int64_t i = 0; i < nfull; ++i) {
        const int64_t q = p0 + i * U;
        if (i + 1 < nfull) load(vb, wb, q + U);
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if constexpr (W) acc = __dadd_rn(acc, __dmul_rn(wa[u], va[u]));
            else acc = __dadd_rn(acc, va[u]);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            va[u] = vb[u];
            if constexpr (W) wa[u] = wb[u];
        }
    }
    for (int64_t p = p0 + nfull * U; p < p1; ++p)
        acc = W ? __dadd_rn(acc, __dmul_rn(w[p], g[p * gs + k])) : __dadd_rn(acc, g[p * gs + k]);
    part[b * gs + k] = acc;
}
__global__ void blocked_total_kernel(const double* __restrict__ part, int64_t nblocks, int64_t gs,
                                     double* out) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= gs) return;
    double t = 0.0;
    for (int64_t b = 0; b < nblocks; ++b) t = __dadd_rn(t, part[b * gs + k]);
    out[k] = t;
}

// Tracked Global/Local: the column-0 border per DP row by runs of bitwise-equal extends
// (aligner.hpp:1986-2006), one thread per pair.
template <class T, bool AFF>
__global__ void bx0_kernel(const int64_t* oa, int64_t n_pairs, const uint16_t* tracks,
                           const T* gapsT, T* bx0) {
    const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= n_pairs) return;
    const int64_t ao = oa[p];
    const int m = int(oa[p + 1] - ao);
    const uint16_t* tk = tracks + ao;
    T* out = bx0 + ao + p;
    out[0] = T(0);
    if (m == 0) return;
    const T go = gapsT[4 * tk[0] + 2];
    T csum = T(0);
    int s = 1;
    T prev = T(0);
    for (int i = 1; i <= m; ++i) {
        const T ge = gapsT[4 * tk[i - 1] + 3];
        if (i > 1) {
            bool differ;
            if constexpr (sizeof(T) == 4) differ = __float_as_uint(float(ge)) != __float_as_uint(float(prev));
            else differ = __double_as_longlong(double(ge)) != __double_as_longlong(double(prev));
            if (differ) {
                csum = (s == 1) ? nwg::mul_rn(static_cast<T>(i - 1), prev)
                                : nwg::add_rn(csum, nwg::mul_rn(static_cast<T>(i - s), prev));
                s = i;
            }
        }
        if constexpr (AFF)
            out[i] = (s == 1) ? -nwg::add_rn(go, nwg::mul_rn(static_cast<T>(i), ge))
                              : -nwg::add_rn(go, nwg::add_rn(csum, nwg::mul_rn(static_cast<T>(i - s + 1), ge)));
        else
            out[i] = (s == 1) ? nwg::mul_rn(-static_cast<T>(i), ge)
                              : -nwg::add_rn(csum, nwg::mul_rn(static_cast<T>(i - s + 1), ge));
        prev = ge;
    }
}

__global__ void mark_status_kernel(const int32_t* order, int64_t n, int32_t* status, int32_t v) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < n) status[order[k]] = v;
}

int sm_count(int dev) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v > 0 ? v : 148;
}

// ── captured launch sequences ────────────────────────────────────────────────
// A kernel launch held for replay: the function, its shape and its one argument (the
// kernels take a single plain-data struct).
struct Launch {
    const void* fn = nullptr;
    unsigned grid = 0;
    int block = 0;
    size_t smem = 0;
    std::vector<unsigned char> arg;
};
template <class A>
Launch make_launch(const void* fn, unsigned grid, int block, size_t smem, const A& a) {
    Launch l;
    l.fn = fn; l.grid = grid; l.block = block; l.smem = smem;
    l.arg.resize(sizeof(A));
    std::memcpy(l.arg.data(), &a, sizeof(A));
    return l;
}

// One bucket sequence's CUDA graph: the launches of a plan (one per length bucket) captured
// once and replayed while the sequence -- functions, shapes and argument bytes, pointers
// included -- is unchanged.  set_params does not change it (the weights live in buffers that
// keep their address), a new batch or a grown scratch buffer does (a new capture).
struct GraphCache {
    std::vector<unsigned char> key;
    std::vector<unsigned char> seen;   // the last sequence launched directly (not yet captured)
    cudaGraphExec_t exec = nullptr;
    void reset() {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        key.clear();
        seen.clear();
    }
};

// ── kernel tables (instantiated in nwg_hard_inst.cu / nwg_soft_inst.cu) ─────────
using HardFn = nwg::HardFn;
using SoftFn = nwg::SoftFn;
using Geo = nwg::Geo;
template <class T> HardFn hard_fn_rt(bool aff, int am, bool tr, Geo g) {
    return sizeof(T) == 4 ? nwg::hard_fn_f32(aff, am, tr, g) : nwg::hard_fn_f64(aff, am, tr, g);
}
template <class T> SoftFn soft_fn_rt(bool aff, int am, bool tr, Geo g) {
    if (sizeof(T) == 4)
        return am == 2 ? nwg::soft_fn_f32_am2(aff, tr, g) : am == 1 ? nwg::soft_fn_f32_am1(aff, tr, g)
                                                          : nwg::soft_fn_f32_am0(aff, tr, g);
    return am == 2 ? nwg::soft_fn_f64_am2(aff, tr, g) : am == 1 ? nwg::soft_fn_f64_am1(aff, tr, g)
                                                      : nwg::soft_fn_f64_am0(aff, tr, g);
}

// The kernel geometries (lanes per pair G, rows per lane R) each path is instantiated for.
bool geo_available(bool soft, int G, int R) {
    if (G == 1) return R == 8 || R == 16 || R == 24 || R == 32;
    if (soft) return (G == 32 && (R == 2 || R == 4 || R == 8)) || (G == 16 && (R == 2 || R == 4 || R == 8)) || (G == 8 && R == 4);
    return G == 32 && (R == 1 || R == 2 || R == 4 || R == 8);
}

// Padded cells a geometry computes for an (m, n) problem over `rows` DP rows.
double geo_cost(Geo g, int rows, int n, int extra_cols) {
    const int GR = g.G * g.R;
    const int64_t stripes = (int64_t(rows) + GR - 1) / GR;
    return double(stripes * GR) * double(n + extra_cols + g.G - 1);
}

// The geometry for one pair: a lane per pair when the rows fit one lane (up to 32 rows);
// else (soft) the geometry of least measured cost x padded cells, (hard) the warp geometry
// that pads the fewest cells, weighing the shuffles of fewer rows per lane.
// lanes / rpl > 0 force the lanes per pair / rows per lane (the tuner's measurements).
Geo pick_geo(bool soft, int rows, int n, int lanes, int rpl, bool lane_ok) {
    if (lanes == 1 || (lanes == 0 && lane_ok && rows <= 32)) {
        int R = rpl;
        if (!R) R = rows <= 8 ? 8 : rows <= 16 ? 16 : rows <= 24 ? 24 : 32;
        return {1, R};
    }
    const int G = lanes > 1 ? lanes : 32;
    if (rpl) return {G, rpl};
    if (soft && lanes == 0) {
        // soft, untuned: the geometry of least predicted time = a measured cost per padded cell
        // (B200, float, the 100-500 residue batch; 32 x 4 = 1) x the pair's padded cells, so
        // short pairs take narrower stripes and fewer lanes
        struct C { int G, R; double cost; };
        static const C costs[] = {{32, 4, 1.00}, {32, 8, 1.02}, {16, 8, 1.18}, {16, 4, 1.35},
                                  {32, 2, 1.73}, {8, 4, 1.78}, {16, 2, 2.00}};
        Geo bestc{32, 4};
        double bt = 1e300;
        for (const C& k : costs) {
            const double t = k.cost * geo_cost(Geo{k.G, k.R}, rows, n, 1);
            if (t < bt) { bt = t; bestc = Geo{k.G, k.R}; }
        }
        return bestc;
    }
    Geo best{G, 4};
    double bc = 1e300;
    // hard: fewer rows per lane cost more shuffles and boundary moves per cell -- measured cost
    // per padded cell (B200, float, the 50-300 residue batch; 8 rows = 1)
    const int opts_h[] = {8, 4, 2, 1};
    const double cost_h[] = {1.00, 1.22, 1.35, 1.80};
    const int opts_s[] = {4, 2};
    const double cost_s[] = {1.00, 1.73};
    const int* opts = soft ? opts_s : opts_h;
    const double* cst = soft ? cost_s : cost_h;
    const int no = soft ? 2 : 4;
    for (int k = 0; k < no; ++k) {
        const Geo g{G, opts[k]};
        if (!geo_available(soft, g.G, g.R)) continue;
        const double c = geo_cost(g, rows, n, soft ? 1 : 0) * cst[k];
        if (c < bc) { bc = c; best = g; }
    }
    return best;
}

// Pairs of at least this many DP rows run with several warps per pair (a pipeline over the
// pair's stripes) instead of one: a long pair is then not a single warp's serial work.  The
// warps per pair grow with the pair's stripes (each warp keeps at least 3 stripes).
constexpr int kLongRows = 1536;
constexpr int kTileW = 256;   // columns per tile of a tiled long pair (a multiple of 8; soft: of 32)
int long_warps(int rows, int GR) {
    const int ns = (rows + GR - 1) / GR;
    return ns >= 64 ? 16 : ns >= 24 ? 8 : 4;
}

// Pairs are bucketed by geometry and by size class: the binary order of magnitude of the DP
// (rows x columns).  A bucket per doubling sizes its scratch stride close to its own pairs and
// lets the autotuner pick a geometry per class.
int size_class(int rows, int n) {
    const uint64_t cells = uint64_t(std::max(rows, 1)) * uint64_t(std::max(n, 1));
    return cells <= 1 ? 0 : 64 - __builtin_clzll(cells - 1);   // ceil(log2(cells))
}



struct Bucket {
    Geo geo;
    std::vector<int32_t> pairs;
    int64_t off = 0;           // into the store's order array
    int maxn = 0;
    int64_t max_soft_cells = 0;   // soft: max over pairs of nstripes * (n + G) * G * R
    int max_rows = 0;             // soft: DP rows (m + 1) of the bucket's tallest pair
};

struct Plan {
    bool valid = false;
    int key_soft = -1, key_lanes = -1, key_rows = -1, key_band = -1, key_hb = -1, key_one_warp = -1, key_grid = -1;
    int64_t n_planned = 0;           // pairs in the buckets (hard: those not split by Hirschberg)
    std::vector<Bucket> buckets;
    std::vector<int64_t> code_off;   // hard: per pair
    int64_t code_bytes = 0;
    int64_t n_stripes = 0;           // banded: stripes over all pairs
    DBuf order, dcode_off, stripe_base;
    // hard, tiled long pairs: the tiles (p, s, c) of every tiled pair grouped by anti-diagonal
    // s + c (diagonal d: items diag_off[d] .. diag_off[d + 1] - 1); per pair (by index) its row
    // and column buffer offsets and first tile slot, in elements
    // (soft: rows in columns, lane states, tiles and stripes; every stripe's partial too)
    std::vector<int32_t> tile_pairs;
    std::vector<int64_t> diag_off;
    int64_t tile_row_elems = 0, tile_col_elems = 0, n_tiles = 0, n_tile_stripes = 0;
    DBuf tile_items, tile_rowoff, tile_coloff, tile_slot, tile_plist, tile_count, tile_stripeoff, tile_nstripes;
    void reset() {
        order.release(); dcode_off.release(); stripe_base.release();
        tile_items.release(); tile_rowoff.release(); tile_coloff.release(); tile_slot.release();
        tile_plist.release(); tile_count.release(); tile_stripeoff.release(); tile_nstripes.release();
        valid = false; buckets.clear(); code_off.clear(); code_bytes = 0; n_stripes = 0;
        tile_pairs.clear(); diag_off.clear(); tile_row_elems = tile_col_elems = n_tiles = n_tile_stripes = 0;
    }
};

}  // namespace

struct nwg_store {
    int device = 0;
    int64_t n = 0;
    int nalpha = 0;
    bool tracked_seq = false;   // tracks were given
    int max_track = 0;          // the largest track / gap-track entry
    std::vector<int64_t> oa, ob;
    int64_t total_a = 0, total_b = 0;
    DBuf a, b, doa, dob, tracks, gtracks;
    // params
    int K = 0, N = 0;
    std::vector<double> mats, gaps;
    DBuf matf, gapf, matd, gapd;       // Viterbi precision casts
    DBuf bx0f, bx0d;                    // tracked column-0 borders
    DBuf tmatf, tgapf, tmatd, tgapd, tbx0f, tbx0d, tscore, tend;   // a guide snapshot's copies
    bool bx0f_ok = false, bx0d_ok = false;
    // results
    DBuf score, end, grad, guide, status, codes, scratch, part, red, moves, moves_off, path_info;
    DBuf trow, tcol, tbest, tcell;      // tiled long pairs: stripe rows, tile columns, Local tile bests
    DBuf tgrid;                         // grid traceback: one tile's codes per walking warp
    // soft tiles: per-warp tables, rows, lane states, Z parts and per-pair Z, stripe partials
    DBuf tl_table, tl_rowf, tl_rowb, tl_colf, tl_colb, tl_zpart, tl_zpair, tl_spart;
    int64_t gstride = 0;
    bool have_scores = false, have_grads = false, have_guides = false, have_paths = false;
    int last_grad_mode = 0, last_gm = -1, last_am = -1, last_prec = 0;
    Plan hard_plan, soft_plan, band_plan, soft_band_plan;
    // geometry per (soft, size class) chosen by the autotuner; plain: one fixed geometry
    std::map<std::pair<int, int>, std::pair<int, int>> geo_table;
    // per (soft, size class): measured cost per padded cell of each geometry; a pair of the
    // class runs with the geometry whose cost x the pair's padded cells is least
    struct GeoCost { int G, R; double ns_per_cell; };
    std::map<std::pair<int, int>, std::vector<GeoCost>> geo_costs;
    bool plain = false;
    int64_t scratch_budget = -1;   // bytes of soft scratch one call may hold (-1: from the device's memory)
    int64_t auto_budget = -1;      // that budget as first computed for this store, kept so later calls
                                   // decide concurrency (and scratch size) the same way
    int64_t ck_threshold = int64_t(16) << 20;     // soft: forward tables above this are checkpointed
    int spin_limit = nwg::kSpinLimit;             // several warps per pair: polls before a wait gives up
    // work-queue counters, two ints per launch of a call (soft launches from 0, hard fills from
    // kQueueHard); each launch leaves its pair at zero, so they are zeroed once
    static constexpr int kQueues = 4096, kQueueHard = 2048;
    DBuf wq;
    int* queue(int k, cudaStream_t st) {
        if (!wq.p) {
            wq.need(size_t(kQueues) * 2 * sizeof(int), st);
            NWG_CUDA(cudaMemsetAsync(wq.p, 0, wq.bytes, st));
        }
        if (k < 0 || k >= kQueues) throw Error(NWG_EINVAL, "too many launches in one call");
        return wq.as<int>() + 2 * k;
    }
    DBuf stripe_tab;
    DBuf hb_pairs;                      // the pairs a Hirschberg run splits
    std::vector<int32_t> h_status;
    // soft weights per precision (kept: a captured graph reads them at a fixed address)
    DBuf swf, sgwf, swd, sgwd;
    // captured bucket sequences, replayed on a private stream ordered after the caller's
    GraphCache g_soft[2], g_soft_band, g_hard[2], g_hard_band, g_soft_tile[2];
    bool use_graphs = true;
    cudaStream_t gstream = nullptr;
    cudaEvent_t gev_in = nullptr, gev_out = nullptr;
    // concurrent buckets: one private stream per bucket (up to kBucketStreams), fork / join events
    static constexpr int kBucketStreams = 8;
    cudaStream_t bstream[kBucketStreams] = {};
    cudaEvent_t bev_fork = nullptr, bev_join[kBucketStreams] = {};
    int64_t graph_captures = 0, graph_replays = 0, graph_failures = 0;
    // timing
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0;
    int64_t last_launches = 0;
    bool tracked() const { return tracked_seq || K > 1; }
};

namespace {

// Run a bucket sequence on `st`.  With graphs on (and a cache given), the sequence runs as a
// CUDA graph on the store's private stream, which waits for `st` before and makes `st` wait
// for it after: one graph launch in place of a launch per bucket, captured again only when
// the sequence changes.
void run_launches(nwg_store* s, GraphCache* gc, const std::vector<Launch>& L, cudaStream_t st,
                  bool concurrent = false, const std::vector<int>* lanes = nullptr) {
    if (L.empty()) return;
    s->last_launches += int64_t(L.size());
    concurrent = concurrent && L.size() > 1;
    if (concurrent && !s->bev_fork) {
        NWG_CUDA(cudaEventCreateWithFlags(&s->bev_fork, cudaEventDisableTiming));
        for (int k = 0; k < nwg_store::kBucketStreams; ++k) {
            NWG_CUDA(cudaStreamCreateWithFlags(&s->bstream[k], cudaStreamNonBlocking));
            NWG_CUDA(cudaEventCreateWithFlags(&s->bev_join[k], cudaEventDisableTiming));
        }
    }
    // the launches in order on `on`; concurrent: each on its own private stream, forked from and
    // joined back into `on` (so a capture on `on` records them as parallel branches)
    auto issue = [&](cudaStream_t on) -> cudaError_t {
        if (!concurrent) {
            for (const Launch& l : L) {
                void* args[] = {const_cast<unsigned char*>(l.arg.data())};
                const cudaError_t e = cudaLaunchKernel(l.fn, dim3(l.grid), dim3(unsigned(l.block)), args, l.smem, on);
                if (e != cudaSuccess) return e;
            }
            return cudaSuccess;
        }
        cudaError_t e = cudaEventRecord(s->bev_fork, on);
        if (e != cudaSuccess) return e;
        // launches of one lane run in order on one stream; lanes run at once
        auto lane_of = [&](size_t i) { return (lanes ? size_t((*lanes)[i]) : i) % size_t(nwg_store::kBucketStreams); };
        int ns = 0;
        for (size_t i = 0; i < L.size(); ++i) ns = std::max(ns, int(lane_of(i)) + 1);
        for (int k = 0; k < ns; ++k)
            if ((e = cudaStreamWaitEvent(s->bstream[k], s->bev_fork, 0)) != cudaSuccess) return e;
        for (size_t i = 0; i < L.size(); ++i) {
            const Launch& l = L[i];
            void* args[] = {const_cast<unsigned char*>(l.arg.data())};
            e = cudaLaunchKernel(l.fn, dim3(l.grid), dim3(unsigned(l.block)), args, l.smem, s->bstream[lane_of(i)]);
            if (e != cudaSuccess) return e;
        }
        for (int k = 0; k < ns; ++k) {
            if ((e = cudaEventRecord(s->bev_join[k], s->bstream[k])) != cudaSuccess) return e;
            if ((e = cudaStreamWaitEvent(on, s->bev_join[k], 0)) != cudaSuccess) return e;
        }
        return cudaSuccess;
    };
    auto launch_all = [&](cudaStream_t on) { NWG_CUDA(issue(on)); };
    if (!gc || !s->use_graphs) {
        launch_all(st);
        return;
    }
    std::vector<unsigned char> key;
    key.push_back(concurrent ? 1 : 0);
    if (concurrent && lanes)
        for (int v : *lanes) key.push_back(static_cast<unsigned char>(v & 0xff));
    for (const Launch& l : L) {
        const unsigned char* f = reinterpret_cast<const unsigned char*>(&l.fn);
        key.insert(key.end(), f, f + sizeof(l.fn));
        const int64_t shape[3] = {int64_t(l.grid), int64_t(l.block), int64_t(l.smem)};
        const unsigned char* sh = reinterpret_cast<const unsigned char*>(shape);
        key.insert(key.end(), sh, sh + sizeof(shape));
        key.insert(key.end(), l.arg.begin(), l.arg.end());
    }
    if (!s->gstream) {
        NWG_CUDA(cudaStreamCreateWithFlags(&s->gstream, cudaStreamNonBlocking));
        NWG_CUDA(cudaEventCreateWithFlags(&s->gev_in, cudaEventDisableTiming));
        NWG_CUDA(cudaEventCreateWithFlags(&s->gev_out, cudaEventDisableTiming));
    }
    // a sequence seen for the first time launches directly (a batch run once -- a new store
    // per batch -- never pays for a capture); the second time it is captured, then replayed
    if ((!gc->exec || key != gc->key) && key != gc->seen) {
        gc->seen = std::move(key);
        launch_all(st);
        return;
    }
    NWG_CUDA(cudaEventRecord(s->gev_in, st));
    NWG_CUDA(cudaStreamWaitEvent(s->gstream, s->gev_in, 0));
    if (!gc->exec || key != gc->key) {
        gc->reset();
        cudaGraph_t g = nullptr;
        NWG_CUDA(cudaStreamBeginCapture(s->gstream, cudaStreamCaptureModeThreadLocal));
        const cudaError_t le = issue(s->gstream);
        const cudaError_t ee = cudaStreamEndCapture(s->gstream, &g);
        cudaError_t ie = cudaErrorStreamCaptureInvalidated;
        if (le == cudaSuccess && ee == cudaSuccess && g) ie = cudaGraphInstantiate(&gc->exec, g, 0);
        if (g) cudaGraphDestroy(g);
        if (ie != cudaSuccess) {
            // a capture that another thread's call invalidated (or that failed to instantiate):
            // this call launches directly, the next one tries again
            cudaGetLastError();
            gc->exec = nullptr;
            gc->key.clear();
            s->graph_failures++;
            if (le != cudaSuccess && le != cudaErrorStreamCaptureInvalidated && le != cudaErrorStreamCaptureUnsupported)
                NWG_CUDA(le);
            launch_all(s->gstream);
            NWG_CUDA(cudaEventRecord(s->gev_out, s->gstream));
            NWG_CUDA(cudaStreamWaitEvent(st, s->gev_out, 0));
            return;
        }
        gc->key = std::move(key);
        s->graph_captures++;
    } else {
        s->graph_replays++;
    }
    NWG_CUDA(cudaGraphLaunch(gc->exec, s->gstream));
    NWG_CUDA(cudaEventRecord(s->gev_out, s->gstream));
    NWG_CUDA(cudaStreamWaitEvent(st, s->gev_out, 0));
}

// The scratch budget of one call: as set, else 60 % of what the device could give it (its free
// memory plus the scratch this store already holds), at least 24 GiB.
int64_t scratch_budget_of(nwg_store* s) {
    if (s->scratch_budget >= 0) return s->scratch_budget;
    if (s->auto_budget >= 0) return s->auto_budget;
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    // blocks the pool keeps from earlier batches are free for this one too (the device's free
    // memory does not count them)
    uint64_t reserved = 0, used = 0;
    cudaMemPool_t pool;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
    }
    const double idle = reserved > used ? double(reserved - used) : 0.0;
    s->auto_budget = std::max<int64_t>(int64_t(24) << 30, int64_t(0.6 * (double(fr) + idle + double(s->scratch.bytes))));
    return s->auto_budget;
}

void set_params_dev(nwg_store* s) {
    const size_t nm = s->mats.size(), ng = s->gaps.size();
    std::vector<float> mf(nm), gf(ng);
    for (size_t k = 0; k < nm; ++k) mf[k] = static_cast<float>(s->mats[k]);
    for (size_t k = 0; k < ng; ++k) gf[k] = static_cast<float>(s->gaps[k]);
    s->matf.need(nm * 4); s->gapf.need(ng * 4);
    s->matd.need(nm * 8); s->gapd.need(ng * 8);
    NWG_CUDA(cudaMemcpy(s->matf.p, mf.data(), nm * 4, cudaMemcpyHostToDevice));
    NWG_CUDA(cudaMemcpy(s->gapf.p, gf.data(), ng * 4, cudaMemcpyHostToDevice));
    NWG_CUDA(cudaMemcpy(s->matd.p, s->mats.data(), nm * 8, cudaMemcpyHostToDevice));
    NWG_CUDA(cudaMemcpy(s->gapd.p, s->gaps.data(), ng * 8, cudaMemcpyHostToDevice));
    s->bx0f_ok = s->bx0d_ok = false;
}

template <class T>
const T* ensure_bx0(nwg_store* s, bool aff, cudaStream_t st, bool& ok, DBuf& buf, const DBuf& gapsT) {
    if (!s->tracked()) return nullptr;
    const int64_t rows = s->total_a + s->n;
    buf.need(size_t(rows) * sizeof(T));
    if (!s->tracks.p) {
        // K > 1 without tracks: every row is set 0 -- the untracked closed forms apply, but the
        // kernels read the table: fill it the same way from an all-zero track.
        s->tracks.need(size_t(std::max<int64_t>(s->total_a, 1)) * 2);
        NWG_CUDA(cudaMemsetAsync(s->tracks.p, 0, size_t(std::max<int64_t>(s->total_a, 1)) * 2, st));
    }
    const int th = 128;
    const int64_t bl = (s->n + th - 1) / th;
    if (bl > 0) {
        if (aff) bx0_kernel<T, true><<<unsigned(bl), th, 0, st>>>(s->doa.as<int64_t>(), s->n, s->tracks.as<uint16_t>(), gapsT.as<T>(), buf.as<T>());
        else     bx0_kernel<T, false><<<unsigned(bl), th, 0, st>>>(s->doa.as<int64_t>(), s->n, s->tracks.as<uint16_t>(), gapsT.as<T>(), buf.as<T>());
        NWG_CUDA(cudaGetLastError());
        s->last_launches++;
    }
    ok = true;
    return buf.as<T>();
}

// hb_cut > 0 (hard, full DP): pairs longer than hb_cut rows are left out (Hirschberg runs them).
// one_warp (hard): no pair runs with several warps (the semi-global ends are one warp's).
// grid: the grid traceback for tiled pairs (no code table for them)
void build_plan(nwg_store* s, Plan& P, bool soft, int lanes, int rpl, int elem_bytes, bool band = false,
                int hb_cut = 0, bool one_warp = false, bool grid = false) {
    if (P.valid && P.key_soft == int(soft) && P.key_lanes == lanes && P.key_rows == rpl && P.key_band == int(band) &&
        P.key_hb == hb_cut && P.key_one_warp == int(one_warp) && P.key_grid == int(grid)) return;
    P.reset();
    P.key_soft = soft; P.key_lanes = lanes; P.key_rows = rpl; P.key_band = band; P.key_hb = hb_cut;
    P.key_one_warp = one_warp; P.key_grid = grid;
    const int64_t n = s->n;
    // one lane per pair keeps a K*N*N histogram per lane in shared memory (soft)
    const bool lane_ok_soft = int64_t(s->K) * s->N * s->N * elem_bytes * 32 <= 48 * 1024;
    std::vector<std::array<int, 3>> bkeys;   // the distinct geometries
    std::vector<int> btab;                   // per geometry and size class: its bucket (-1: none)
    // the tuner's choices per size class, looked up once
    constexpr int kClasses = 64;
    std::vector<const std::vector<nwg_store::GeoCost>*> cost_of(kClasses, nullptr);
    std::vector<std::pair<int, int>> table_of(kClasses, {0, 0});
    for (const auto& kv : s->geo_costs)
        if (kv.first.first == int(soft) && kv.first.second >= 0 && kv.first.second < kClasses) cost_of[kv.first.second] = &kv.second;
    for (const auto& kv : s->geo_table)
        if (kv.first.first == int(soft) && kv.first.second >= 0 && kv.first.second < kClasses) table_of[kv.first.second] = kv.second;
    for (int64_t p = 0; p < n; ++p) {
        const int m = int(s->oa[p + 1] - s->oa[p]), nb = int(s->ob[p + 1] - s->ob[p]);
        if (hb_cut > 0 && m > hb_cut) continue;
        const int rows = soft ? m + 1 : m;
        const int sc = size_class(rows, nb);
        Geo g = band ? (soft ? Geo{32, 4, true} : Geo{32, 2, true})
                     : pick_geo(soft, std::max(rows, 1), nb, lanes, rpl, soft ? lane_ok_soft : true);
        if (!band && !lanes && !rpl) {
            if (s->plain) g = Geo{32, 4};
            else if (soft && !s->tracked() && rows >= kLongRows && nb >= 256)
                // long pairs: tiles over the whole device; with semi-global ends, several warps
                g = one_warp ? Geo{32, 4, false, long_warps(rows, 128)} : Geo{32, 4, false, 0, false, true};
            else if (!soft && !one_warp && rows >= kLongRows && nb >= 256)
                g = Geo{32, 8, false, 0, false, true};   // long pairs: tiles over the whole device
            else if (sc < kClasses && cost_of[sc]) {
                double best = 1e300;
                for (const auto& gc : *cost_of[sc]) {
                    if (soft && gc.G == 1 && !lane_ok_soft) continue;
                    const double t = gc.ns_per_cell * geo_cost(Geo{gc.G, gc.R}, std::max(rows, 1), nb, soft ? 1 : 0);
                    if (t < best) { best = t; g = Geo{gc.G, gc.R}; }
                }
            } else if (sc < kClasses && table_of[sc].first > 0 && (!soft || table_of[sc].first > 1 || lane_ok_soft)) {
                g = Geo{table_of[sc].first, table_of[sc].second};
            }
        }
        // the bucket of (geometry, size class): the geometry's index among the few distinct ones
        // seen (a short search), then a table over size classes
        const int k1 = g.G, k2 = g.R * 100 + g.mw + (g.tile ? 50 : 0);
        int gi = -1;
        for (int q = 0; q < int(bkeys.size()); ++q)
            if (bkeys[q][0] == k1 && bkeys[q][1] == k2) { gi = q; break; }
        if (gi < 0) {
            gi = int(bkeys.size());
            bkeys.push_back({k1, k2, 0});
            btab.resize(bkeys.size() * kClasses, -1);
        }
        const int sci = std::min(sc, kClasses - 1);
        int bi = btab[size_t(gi) * kClasses + sci];
        if (bi < 0) {
            bi = int(P.buckets.size());
            btab[size_t(gi) * kClasses + sci] = bi;
            P.buckets.push_back(Bucket{g, {}, 0, 0, 0});
        }
        P.buckets[bi].pairs.push_back(int32_t(p));
    }
    // tiled buckets last: the pairs walked from a code table are then a prefix of the order
    std::stable_partition(P.buckets.begin(), P.buckets.end(), [](const Bucket& B) { return !B.geo.tile; });
    std::vector<int32_t> order;
    order.reserve(n);
    if (!soft) P.code_off.assign(n + 1, 0);
    std::vector<int64_t> cells_v(size_t(n) + 1);
    int64_t* const pair_cells = cells_v.data();
    for (int64_t q = 0; q < n; ++q) pair_cells[q] = (s->oa[q + 1] - s->oa[q]) * (s->ob[q + 1] - s->ob[q]);
    // longest first, to 1/64 of a doubling of the cells (a counting sort, stable: pair order
    // within a bin): the persistent groups, which take pairs in this order from their work
    // queue, then finish together
    constexpr int kSortBins = 64 * 64;
    auto sort_key = [](int64_t cells) -> int {
        if (cells <= 1) return 0;
        const uint64_t c = uint64_t(cells);
        const int e = 63 - __builtin_clzll(c);                       // floor(log2)
        const int frac = e >= 6 ? int((c >> (e - 6)) & 63) : int((c << (6 - e)) & 63);
        return std::min(kSortBins - 1, e * 64 + frac);
    };
    std::vector<int32_t> bin_count(kSortBins + 1), sorted;
    std::vector<int> keys;
    for (auto& B : P.buckets) {
        const size_t np = B.pairs.size();
        keys.resize(np);
        std::fill(bin_count.begin(), bin_count.end(), 0);
        for (size_t q = 0; q < np; ++q) { keys[q] = kSortBins - 1 - sort_key(pair_cells[B.pairs[q]]); ++bin_count[keys[q] + 1]; }
        for (int k = 0; k < kSortBins; ++k) bin_count[k + 1] += bin_count[k];
        sorted.resize(np);
        for (size_t q = 0; q < np; ++q) sorted[size_t(bin_count[keys[q]]++)] = B.pairs[q];
        B.pairs.swap(sorted);
        B.off = int64_t(order.size());
        for (int32_t p : B.pairs) {
            order.push_back(p);
            const int m = int(s->oa[p + 1] - s->oa[p]), nb = int(s->ob[p + 1] - s->ob[p]);
            B.maxn = std::max(B.maxn, nb);
            const int GR = B.geo.G * B.geo.R;
            if (soft) {
                const int64_t st = (m + 1 + GR - 1) / GR;
                B.max_soft_cells = std::max<int64_t>(B.max_soft_cells, st * (nb + B.geo.G) * GR);
                B.max_rows = std::max(B.max_rows, m + 1);
            }
        }
    }
    if (!soft) {
        // code tables: per pair nstripes * (n + G - 1) * G * R bytes, 16-byte aligned
        int64_t off = 0;
        for (auto& B : P.buckets)
            for (int32_t p : B.pairs) {
                const int m = int(s->oa[p + 1] - s->oa[p]), nb = int(s->ob[p + 1] - s->ob[p]);
                const int GR = B.geo.G * B.geo.R;
                const int64_t st = (m + GR - 1) / GR;
                P.code_off[p] = off;
                const bool table = m && nb && !(grid && B.geo.tile);
                const int64_t bytes = table ? st * (((nb + B.geo.G - 1) + 7) & ~int64_t(7)) * GR : 0;
                off += (bytes + 15) & ~int64_t(15);
            }
        P.code_bytes = std::max<int64_t>(off, 16);
    }
    // tiled pairs: stripes of G R rows x tiles of kTileW columns; the tile (s, c) needs
    // (s - 1, c) and (s, c - 1), both on the diagonal before its own.  Hard: rows 1..m and
    // columns 1..n, offsets in T; soft: rows 0..m and columns 0..n, offsets in columns, lane
    // states, tiles and stripes (the kernel scales them by its own state sizes)
    bool any_tile = false;
    for (auto& B : P.buckets) any_tile |= B.geo.tile && !B.pairs.empty();
    const size_t tn = any_tile ? size_t(n) + 1 : 0;   // per-pair tile offsets only when tiles exist
    std::vector<int64_t> roff(tn, 0), coff(tn, 0), toff(tn, 0), soff(tn, 0);
    std::vector<int32_t> tcount, scount;
    std::vector<std::vector<int32_t>> diags;
    for (auto& B : P.buckets) {
        if (!B.geo.tile) continue;
        const int GR = B.geo.G * B.geo.R;
        for (int32_t p : B.pairs) {
            const int m = int(s->oa[p + 1] - s->oa[p]), nb = int(s->ob[p + 1] - s->ob[p]);
            const int ns = soft ? (m + 1 + GR - 1) / GR : (m + GR - 1) / GR;
            const int nt = soft ? nb / kTileW + 1 : (nb + kTileW - 1) / kTileW;
            roff[p] = P.tile_row_elems; P.tile_row_elems += int64_t(ns) * (soft ? 1 : 3) * (nb + 1);
            coff[p] = P.tile_col_elems; P.tile_col_elems += int64_t(ns) * nt * (soft ? B.geo.G : 3 * GR);
            toff[p] = P.n_tiles; P.n_tiles += int64_t(ns) * nt;
            soff[p] = P.n_tile_stripes; P.n_tile_stripes += ns;
            P.tile_pairs.push_back(p);
            tcount.push_back(ns * nt);
            scount.push_back(ns);
            if (int(diags.size()) < ns + nt - 1) diags.resize(size_t(ns + nt - 1));
            for (int st = 0; st < ns; ++st)
                for (int c = 0; c < nt; ++c) {
                    auto& dv = diags[size_t(st + c)];
                    dv.push_back(p); dv.push_back(st); dv.push_back(c);
                }
        }
    }
    if (!P.tile_pairs.empty()) {
        std::vector<int32_t> items;
        items.reserve(size_t(P.n_tiles) * 3);
        P.diag_off.assign(1, 0);
        for (auto& dv : diags) {
            items.insert(items.end(), dv.begin(), dv.end());
            P.diag_off.push_back(int64_t(items.size() / 3));
        }
        auto up = [](DBuf& d, const void* h, size_t bytes) {
            d.need(bytes);
            NWG_CUDA(cudaMemcpy(d.p, h, bytes, cudaMemcpyHostToDevice));
        };
        up(P.tile_items, items.data(), items.size() * 4);
        up(P.tile_rowoff, roff.data(), roff.size() * 8);
        up(P.tile_coloff, coff.data(), coff.size() * 8);
        up(P.tile_slot, toff.data(), toff.size() * 8);
        up(P.tile_plist, P.tile_pairs.data(), P.tile_pairs.size() * 4);
        up(P.tile_count, tcount.data(), tcount.size() * 4);
        up(P.tile_stripeoff, soff.data(), soff.size() * 8);
        up(P.tile_nstripes, scount.data(), scount.size() * 4);
    }
    P.n_planned = int64_t(order.size());
    P.order.need(size_t(std::max<int64_t>(n, 1)) * 4);
    if (!order.empty()) NWG_CUDA(cudaMemcpy(P.order.p, order.data(), order.size() * 4, cudaMemcpyHostToDevice));
    if (!soft) {
        P.dcode_off.need(size_t(n + 1) * 8);
        NWG_CUDA(cudaMemcpy(P.dcode_off.p, P.code_off.data(), size_t(n + 1) * 8, cudaMemcpyHostToDevice));
    }
    if (band) {
        // per pair the index of its first stripe in the stripe table
        std::vector<int64_t> sb(size_t(n) + 1, 0);
        for (int64_t p = 0; p < n; ++p) {
            const int m = int(s->oa[p + 1] - s->oa[p]);
            sb[p + 1] = sb[p] + (m + 63) / 64;
        }
        P.n_stripes = sb[n];
        P.stripe_base.need(size_t(n + 1) * 8);
        NWG_CUDA(cudaMemcpy(P.stripe_base.p, sb.data(), size_t(n + 1) * 8, cudaMemcpyHostToDevice));
    }
    P.valid = true;
}

template <class T>
void run_hard(nwg_store* s, const nwg_job& J, cudaStream_t st, bool want_grad, bool want_guide) {
    const bool aff = J.gap_model == 1, loc = J.mode == 1, tr = s->tracked();
    const int ends = J.mode == 2 ? J.free_ends : 0;   // semi-global free ends (0: Global's)
    const bool band = J.band >= 0;
    // Hirschberg (untracked, full DP): pairs longer than the cutoff split (Local: by the
    // endpoint scans and their box)
    // (semi-global ends: glocal's only -- aligner.hpp:2323-2330, 4709, 5132; tracked, affine)
    const bool glocal_hb = J.mode == 2 && J.free_ends == 12 && (!tr || aff);
    const bool hb = !band && (J.mode != 2 || glocal_hb) && (J.traceback == 3 || J.traceback == 4);
    const int hb_cut = hb ? (J.hb_cutoff > 0 ? J.hb_cutoff : 512) : 0;
    std::vector<int32_t> hb_pairs;
    if (hb) {
        for (int64_t p = 0; p < s->n; ++p)
            if (s->oa[p + 1] - s->oa[p] > hb_cut) hb_pairs.push_back(int32_t(p));
        // non-negative penalties (hb_penalties_ok_, aligner.hpp:5747-5763): linear, the extends
        bool ok = true;
        for (int k = 0; k < s->K; ++k)
            ok = ok && s->gaps[4 * k + 1] >= 0.0 && s->gaps[4 * k + 3] >= 0.0 &&
                 (!aff || (s->gaps[4 * k] >= 0.0 && s->gaps[4 * k + 2] >= 0.0));
        if (!hb_pairs.empty() && !ok)
            throw Error(NWG_EINVAL, "nwgrad: traceback=\"hirschberg\" / \"hirschberg_pmax\" needs non-negative "
                                    "gap penalties (got a negative one); use traceback=\"pointers\" or \"auto\"");
    }
    // the grid traceback (aligner.hpp:89-100): tiled pairs keep rows and columns, not codes
    const bool grid = !band && ends == 0 && J.traceback == 5;
    Plan& P = band ? s->band_plan : s->hard_plan;
    build_plan(s, P, false, band ? 32 : J.lanes, band ? 2 : J.rows, sizeof(T), band, hb_cut, ends != 0, grid);
    s->codes.need(size_t(P.code_bytes), st);
    if (band) s->stripe_tab.need(size_t(std::max<int64_t>(P.n_stripes, 1)) * 16, st);
    const DBuf& matT = sizeof(T) == 4 ? s->matf : s->matd;
    const DBuf& gapT = sizeof(T) == 4 ? s->gapf : s->gapd;
    const T* bx0 = nullptr;
    if (tr) {
        if (sizeof(T) == 4) bx0 = reinterpret_cast<const T*>(ensure_bx0<float>(s, aff, st, s->bx0f_ok, s->bx0f, s->gapf));
        else bx0 = reinterpret_cast<const T*>(ensure_bx0<double>(s, aff, st, s->bx0d_ok, s->bx0d, s->gapd));
    }
    s->score.need(size_t(std::max<int64_t>(s->n, 1)) * 8, st);
    s->end.need(size_t(std::max<int64_t>(s->n, 1)) * 16, st);
    const int sms = sm_count(s->device);
    const size_t smem_base = (size_t(s->K) * s->N * s->N + 4 * size_t(s->K)) * sizeof(T);
    // scratch per slot: the stripe boundary row (one group per pair)
    auto bucket_shape = [&](const Bucket& B, int64_t& blocks, int64_t& slots, int64_t& stride) {
        const int gpb = 128 / B.geo.G;
        const int64_t items = int64_t(B.pairs.size());
        const int64_t row = 3 * (int64_t(B.maxn) + 1);
        if (B.geo.tile) {   // tiles: per-pair row and column buffers instead of scratch
            blocks = 0; slots = 0; stride = 0;
        } else {
            blocks = std::min<int64_t>((items + gpb - 1) / gpb, int64_t(sms) * 16);
            slots = blocks * gpb;
            stride = row;
        }
    };
    int64_t max_total = 1, sum_total = 0;
    bool any_tile = false;
    int nbk = 0;
    for (auto& B : P.buckets) {
        if (B.pairs.empty()) continue;
        int64_t bl, sl, sd;
        bucket_shape(B, bl, sl, sd);
        max_total = std::max(max_total, sl * sd);
        sum_total += (sl * sd * int64_t(sizeof(T)) + 255) & ~int64_t(255);
        any_tile |= B.geo.tile;
        ++nbk;
    }
    // tiles: the fills first, then one walk over every pair
    const bool sep_walk = any_tile;
    // otherwise the buckets' fills and walks run at once (bucket k's walk after its fill, each
    // bucket on its own stream and scratch part) when their scratch parts fit
    const bool concurrent = !sep_walk && nbk > 1 && sum_total <= scratch_budget_of(s);
    s->scratch.need(concurrent ? size_t(sum_total) : size_t(max_total) * sizeof(T), st);
    std::vector<Launch> fills;
    std::vector<nwg::HardArgs> fill_args;
    int64_t soff_b = 0;
    int nq = 0;   // work-queue counters used
    for (auto& B : P.buckets) {
        if (B.pairs.empty() || B.geo.tile) continue;
        HardFn fn = hard_fn_rt<T>(aff, ends ? 2 : (loc ? 1 : 0), tr, B.geo);
        if (!fn) throw Error(NWG_EINVAL, "no kernel for this geometry");
        const int hblock = 128;
        const size_t smem = smem_base;
        NWG_CUDA(nwg::allow_smem(reinterpret_cast<const void*>(fn), smem));
        nwg::HardArgs A{};
        A.a = s->a.as<uint8_t>(); A.oa = s->doa.as<int64_t>();
        A.b = s->b.as<uint8_t>(); A.ob = s->dob.as<int64_t>();
        A.tracks = tr ? s->tracks.as<uint16_t>() : nullptr;
        A.gtracks = tr ? s->gtracks.as<uint16_t>() : nullptr;
        A.bx0 = bx0;
        A.order = P.order.as<int32_t>() + B.off;
        A.n_items = int64_t(B.pairs.size());
        A.mat = matT.p; A.gaps = gapT.p; A.N = s->N; A.K = s->K;
        A.codes = s->codes.as<uint8_t>(); A.code_off = P.dcode_off.as<int64_t>();
        if (band) {
            A.guide = s->guide.as<int32_t>(); A.band = J.band;
            A.stripe_base = P.stripe_base.as<int64_t>(); A.stripe_tab = s->stripe_tab.as<int64_t>();
        }
        int64_t blocks, slots, stride;
        bucket_shape(B, blocks, slots, stride);
        A.scratch = concurrent ? static_cast<void*>(static_cast<unsigned char*>(s->scratch.p) + soff_b) : s->scratch.p;
        soff_b += (slots * stride * int64_t(sizeof(T)) + 255) & ~int64_t(255);
        A.scratch_stride = stride;
        A.score = s->score.as<double>(); A.end = s->end.as<int32_t>();
        A.ends = ends;
        A.queue = s->queue(nwg_store::kQueueHard + nq++, st);
        fills.push_back(make_launch(reinterpret_cast<const void*>(fn), unsigned(blocks), hblock, smem, A));
        fill_args.push_back(A);
    }
    if (any_tile) {
        // tiled long pairs: a launch per anti-diagonal of tiles over every tiled pair, each tile
        // one warp's item from the launch's work queue; the launches run in order on one stream,
        // so they share one queue (each leaves it at zero)
        const Geo tg{32, 8, false, 0, false, true};
        HardFn fn = hard_fn_rt<T>(aff, loc ? 1 : 0, tr, tg);
        if (!fn) throw Error(NWG_EINVAL, "no kernel for this geometry");
        NWG_CUDA(nwg::allow_smem(reinterpret_cast<const void*>(fn), smem_base));
        s->trow.need(size_t(std::max<int64_t>(P.tile_row_elems, 1)) * sizeof(T), st);
        s->tcol.need(size_t(std::max<int64_t>(P.tile_col_elems, 1)) * sizeof(T), st);
        if (loc) {
            s->tbest.need(size_t(std::max<int64_t>(P.n_tiles, 1)) * sizeof(T), st);
            s->tcell.need(size_t(std::max<int64_t>(P.n_tiles, 1)) * 12, st);
        }
        nwg::HardArgs A{};
        A.a = s->a.as<uint8_t>(); A.oa = s->doa.as<int64_t>();
        A.b = s->b.as<uint8_t>(); A.ob = s->dob.as<int64_t>();
        A.tracks = tr ? s->tracks.as<uint16_t>() : nullptr;
        A.gtracks = tr ? s->gtracks.as<uint16_t>() : nullptr;
        A.bx0 = bx0;
        A.mat = matT.p; A.gaps = gapT.p; A.N = s->N; A.K = s->K;
        A.codes = grid ? nullptr : s->codes.as<uint8_t>(); A.code_off = P.dcode_off.as<int64_t>();
        A.scratch = s->trow.p; A.scratch_stride = 0;
        A.score = s->score.as<double>(); A.end = s->end.as<int32_t>();
        A.queue = s->queue(nwg_store::kQueueHard + nq++, st);
        A.tile_w = kTileW;
        A.rowbuf = s->trow.p; A.rowbuf_off = P.tile_rowoff.as<int64_t>();
        A.colbuf = s->tcol.p; A.colbuf_off = P.tile_coloff.as<int64_t>();
        A.tbest = loc ? s->tbest.p : nullptr; A.tcell = loc ? s->tcell.as<int32_t>() : nullptr;
        A.tile_off = P.tile_slot.as<int64_t>();
        for (size_t d = 0; d + 1 < P.diag_off.size(); ++d) {
            const int64_t cnt = P.diag_off[d + 1] - P.diag_off[d];
            A.tiles = P.tile_items.as<int32_t>() + 3 * P.diag_off[d];
            A.n_items = cnt;
            const int64_t blocks = std::min<int64_t>((cnt + 3) / 4, int64_t(sms) * 16);
            fills.push_back(make_launch(reinterpret_cast<const void*>(fn), unsigned(blocks), 128, smem_base, A));
        }
        if (loc) {
            nwg::TileBestArgs TB{};
            TB.pairs = P.tile_plist.as<int32_t>(); TB.n_pairs = int64_t(P.tile_pairs.size());
            TB.tile_off = P.tile_slot.as<int64_t>(); TB.tiles_of = P.tile_count.as<int32_t>();
            TB.tbest = s->tbest.p; TB.tcell = s->tcell.as<int32_t>();
            TB.score = s->score.as<double>(); TB.end = s->end.as<int32_t>(); TB.layout = (32 << 8) | 8;
            fills.push_back(make_launch(reinterpret_cast<const void*>(&nwg::tile_best_kernel<T>),
                                        unsigned((TB.n_pairs + 127) / 128), 128, 0, TB));
        }
    }
    // traceback buffers: gradient, guide, path
    if (want_grad) {
        s->grad.need(size_t(s->n) * s->gstride * 8 + 8, st);
        NWG_CUDA(cudaMemsetAsync(s->grad.p, 0, size_t(s->n) * s->gstride * 8, st));
    }
    if (want_guide) s->guide.need(size_t(s->total_a + s->n) * 4 + 4, st);
    const bool keep = J.keep_paths != 0;
    if (keep) {
        std::vector<int64_t> mo(s->n + 1, 0);
        for (int64_t p = 0; p < s->n; ++p) mo[p + 1] = mo[p] + (s->oa[p + 1] - s->oa[p]) + (s->ob[p + 1] - s->ob[p]);
        s->moves.need(size_t(mo[s->n]) + 16);
        s->moves_off.need(size_t(s->n + 1) * 8);
        NWG_CUDA(cudaMemcpyAsync(s->moves_off.p, mo.data(), size_t(s->n + 1) * 8, cudaMemcpyHostToDevice, st));
        NWG_CUDA(cudaStreamSynchronize(st));
        s->path_info.need(size_t(s->n) * 12 + 12);
    }
    nwg::WalkArgs W{};
    W.a = s->a.as<uint8_t>(); W.oa = s->doa.as<int64_t>();
    W.b = s->b.as<uint8_t>(); W.ob = s->dob.as<int64_t>();
    W.tracks = tr ? s->tracks.as<uint16_t>() : nullptr;
    W.gtracks = tr ? s->gtracks.as<uint16_t>() : nullptr;
    W.order = P.order.as<int32_t>(); W.n_items = P.n_planned;
    W.stripe_base = band ? P.stripe_base.as<int64_t>() : nullptr;
    W.stripe_tab = band ? s->stripe_tab.as<int64_t>() : nullptr;
    W.N = s->N; W.K = s->K; W.affine = aff; W.local = loc; W.ends = ends;
    W.codes = s->codes.as<uint8_t>(); W.code_off = P.dcode_off.as<int64_t>();
    W.end = s->end.as<int32_t>();
    W.grad = want_grad ? s->grad.as<double>() : nullptr; W.gstride = s->gstride;
    W.guide = want_guide ? s->guide.as<int32_t>() : nullptr;
    W.moves = keep ? s->moves.as<uint8_t>() : nullptr;
    W.moves_off = keep ? s->moves_off.as<int64_t>() : nullptr;
    W.path_info = keep ? s->path_info.as<int32_t>() : nullptr;
    const Launch walk = make_launch(reinterpret_cast<const void*>(&nwg::walk_kernel),
                                    unsigned((P.n_planned + 127) / 128), 128, 0, W);
    // one captured sequence: the fills walk their own pairs, or (tiles) one walk launch over
    // every pair follows all the fills
    GraphCache* gc = band ? &s->g_hard_band : &s->g_hard[sizeof(T) == 4 ? 0 : 1];
    if (!sep_walk) {
        // a warp per pair: the fill walks its own pairs (the codes still in L2); a lane per pair
        // (many short pairs): a walk launch over the bucket's pairs after its fill.  The buckets
        // run at once when their scratch parts fit.
        std::vector<Launch> seq;
        std::vector<int> lanes;
        size_t k = 0;
        for (auto& B : P.buckets) {
            if (B.pairs.empty()) continue;
            const bool fuse = B.geo.G > 1;
            fill_args[k].walk_fused = fuse ? 1 : 0;
            fill_args[k].walk = W;
            std::memcpy(fills[k].arg.data(), &fill_args[k], sizeof(nwg::HardArgs));
            seq.push_back(fills[k]);
            lanes.push_back(int(k));
            if (!fuse) {
                nwg::WalkArgs Wb = W;
                Wb.order = P.order.as<int32_t>() + B.off;
                Wb.n_items = int64_t(B.pairs.size());
                seq.push_back(make_launch(reinterpret_cast<const void*>(&nwg::walk_kernel),
                                          unsigned((Wb.n_items + 127) / 128), 128, 0, Wb));
                lanes.push_back(int(k));
            }
            ++k;
        }
        run_launches(s, gc, seq, st, concurrent, &lanes);
    } else {
        const int64_t n_tiled = int64_t(P.tile_pairs.size());
        if (grid && n_tiled) {
            // a warp per tiled pair walks back, refilling the tiles its path crosses into its
            // own tile buffer; the pairs before them in the order walk their code tables
            const Geo gg{32, 8, false, 0, false, true, true};
            HardFn fn = hard_fn_rt<T>(aff, loc ? 1 : 0, tr, gg);
            if (!fn) throw Error(NWG_EINVAL, "no kernel for this geometry");
            NWG_CUDA(nwg::allow_smem(reinterpret_cast<const void*>(fn), smem_base));
            const int64_t blocks = std::min<int64_t>((n_tiled + 3) / 4, int64_t(sms) * 16);
            const int64_t stride = int64_t((kTileW + 32 - 1 + 7) & ~7) * 32 * 8;   // steps x lanes x rows
            s->tgrid.need(size_t(blocks * 4 * stride), st);
            nwg::HardArgs A{};
            A.a = s->a.as<uint8_t>(); A.oa = s->doa.as<int64_t>();
            A.b = s->b.as<uint8_t>(); A.ob = s->dob.as<int64_t>();
            A.tracks = tr ? s->tracks.as<uint16_t>() : nullptr;
            A.gtracks = tr ? s->gtracks.as<uint16_t>() : nullptr;
            A.bx0 = bx0;
            A.order = P.tile_plist.as<int32_t>(); A.n_items = n_tiled;
            A.mat = matT.p; A.gaps = gapT.p; A.N = s->N; A.K = s->K;
            A.codes = nullptr; A.code_off = P.dcode_off.as<int64_t>();
            A.scratch = s->tgrid.p; A.scratch_stride = stride;
            A.score = s->score.as<double>(); A.end = s->end.as<int32_t>();
            A.queue = s->queue(nwg_store::kQueueHard + nq++, st);
            A.tile_w = kTileW;
            A.rowbuf = s->trow.p; A.rowbuf_off = P.tile_rowoff.as<int64_t>();
            A.colbuf = s->tcol.p; A.colbuf_off = P.tile_coloff.as<int64_t>();
            A.walk = W;
            fills.push_back(make_launch(reinterpret_cast<const void*>(fn), unsigned(blocks), 128, smem_base, A));
            if (P.n_planned > n_tiled) {
                nwg::WalkArgs Wp = W;
                Wp.n_items = P.n_planned - n_tiled;
                fills.push_back(make_launch(reinterpret_cast<const void*>(&nwg::walk_kernel),
                                            unsigned((Wp.n_items + 127) / 128), 128, 0, Wp));
            }
        } else if (P.n_planned) {
            fills.push_back(walk);
        }
        run_launches(s, gc, fills, st);
    }
    if (!hb_pairs.empty()) {
        s->hb_pairs.need(hb_pairs.size() * 4, st);
        NWG_CUDA(cudaMemcpyAsync(s->hb_pairs.p, hb_pairs.data(), hb_pairs.size() * 4, cudaMemcpyHostToDevice, st));
        nwg::HbRun H{};
        H.a = s->a.as<uint8_t>(); H.b = s->b.as<uint8_t>();
        H.oa = s->doa.as<int64_t>(); H.ob = s->dob.as<int64_t>();
        H.pairs = s->hb_pairs.as<int32_t>();
        H.mat = matT.p; H.N = s->N;
        H.go_a = s->gaps[0]; H.ge_a = s->gaps[1]; H.go_b = s->gaps[2]; H.ge_b = s->gaps[3];
        H.score = s->score.as<double>(); H.end = s->end.as<int32_t>();
        H.grad = want_grad ? s->grad.as<double>() : nullptr; H.gstride = s->gstride;
        H.guide = want_guide ? s->guide.as<int32_t>() : nullptr;
        H.moves = keep ? s->moves.as<uint8_t>() : nullptr;
        H.moves_off = keep ? s->moves_off.as<int64_t>() : nullptr;
        H.path_info = keep ? s->path_info.as<int32_t>() : nullptr;
        H.h_pairs = hb_pairs.data(); H.n_pairs = int64_t(hb_pairs.size());
        H.h_oa = s->oa.data(); H.h_ob = s->ob.data();
        H.cutoff = hb_cut; H.pmax = J.traceback == 4; H.local = loc ? 1 : 0; H.linear = aff ? 0 : 1;
        H.glocal = J.mode == 2 ? 1 : 0;
        H.tile_budget = scratch_budget_of(s) / 2;
        H.K = s->K; H.gaps_t = gapT.p;
        if (tr) {   // tracked (the fill's border set-up gave every tracked store its tracks)
            H.tracks = s->tracks.as<uint16_t>();
            H.gtracks = s->gtracks.p ? s->gtracks.as<uint16_t>() : nullptr;
        }
        try {
            s->last_launches += nwg::hb_run(H, int(sizeof(T)), st, sms);
        } catch (const std::runtime_error& e) {
            throw Error(NWG_ECUDA, e.what());
        }
    }
}

template <class T>
void soft_weights(const nwg_store* s, const nwg_job& J, std::vector<T>& w, std::vector<T>& gw, bool& overflow) {
    const int N = s->N, K = s->K, wc = N + 1;
    const double invT = 1.0 / J.temperature;
    w.assign(size_t(K * N + 1) * wc, T(0));
    overflow = false;
    auto cvt = [&](double x) {
        const T v = static_cast<T>(x);
        if (!std::isfinite(double(v))) overflow = true;
        return v;
    };
    for (int r = 0; r < K * N; ++r)
        for (int c = 0; c < N; ++c) w[size_t(r) * wc + c] = cvt(std::exp(s->mats[size_t(r) * N + c] * invT));
    w[size_t(K * N) * wc + N] = T(1);   // the padding corner: carries the Global seed at (m, n)
    gw.assign(size_t(4) * K, T(0));
    for (int k = 0; k < K; ++k) {
        const double goa = s->gaps[4 * k], gea = s->gaps[4 * k + 1], gob = s->gaps[4 * k + 2], geb = s->gaps[4 * k + 3];
        if (J.gap_model == 1) {
            gw[4 * k + 0] = cvt(std::exp(-(goa + gea) * invT)); gw[4 * k + 1] = cvt(std::exp(-gea * invT));
            gw[4 * k + 2] = cvt(std::exp(-(gob + geb) * invT)); gw[4 * k + 3] = cvt(std::exp(-geb * invT));
        } else {
            gw[4 * k + 0] = gw[4 * k + 1] = cvt(std::exp(-gea * invT));
            gw[4 * k + 2] = gw[4 * k + 3] = cvt(std::exp(-geb * invT));
        }
    }
}

// One soft pass (precision T) over `subset` (all pairs when null).
// The soft pass over tiled long pairs (soft_kernel<..., TL>): a launch per anti-diagonal of
// tiles in the forward phase, Z per pair, a launch per anti-diagonal in reverse order in the
// backward phase (each tile recomputes its own forward table), then every pair's totals; one
// captured sequence, replayed while the plan and buffers stay.
template <class T>
void soft_tile_pass(nwg_store* s, const nwg_job& J, cudaStream_t st, const Plan& P, const DBuf& dw, const DBuf& dgw,
                    int renorm, bool loc, bool aff) {
    const Geo tg{32, 4, false, 0, false, true};
    SoftFn fn = soft_fn_rt<T>(aff, loc ? 1 : 0, false, tg);
    if (!fn) throw Error(NWG_EINVAL, "no soft kernel for this geometry");
    const int K = s->K, N = s->N, G = 32, R = 4, NV = aff ? 3 : 1, BW = aff ? 4 : 2, LS = NV * R + 1;
    const int block = 128, gpb = block / G;
    const size_t smem = nwg::soft_smem_bytes(K, N, G, R, block, int(sizeof(T)), false, false);
    if (smem > 227 * 1024) throw Error(NWG_EINVAL, "soft: the alphabet / parameter sets do not fit shared memory");
    NWG_CUDA(nwg::allow_smem(reinterpret_cast<const void*>(fn), smem));
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, block, smem);
    occ = std::max(occ, 1);
    const int sms = sm_count(s->device);
    // per warp: one tile's forward table (its steps x G lanes x NV R values) and exponents
    const int64_t steps = kTileW + G;
    const int64_t fwd_bytes = (steps * G * NV * R * int64_t(sizeof(T)) + 255) & ~int64_t(255);
    const int64_t exp_bytes = (steps * G * 4 + 255) & ~int64_t(255);
    const int64_t stride = fwd_bytes + exp_bytes;
    const int64_t max_blocks = int64_t(sms) * occ;
    const int64_t nt = int64_t(P.tile_pairs.size());
    s->tl_table.need(size_t(max_blocks * gpb * stride), st);
    s->tl_rowf.need(size_t(std::max<int64_t>(P.tile_row_elems, 1)) * BW * sizeof(T), st);
    s->tl_rowb.need(size_t(std::max<int64_t>(P.tile_row_elems, 1)) * BW * sizeof(T), st);
    s->tl_colf.need(size_t(std::max<int64_t>(P.tile_col_elems, 1)) * LS * sizeof(T), st);
    s->tl_colb.need(size_t(std::max<int64_t>(P.tile_col_elems, 1)) * LS * sizeof(T), st);
    s->tl_zpart.need(size_t(std::max<int64_t>(P.n_tiles, 1)) * 16, st);
    s->tl_zpair.need(size_t(std::max<int64_t>(s->n, 1)) * 16, st);
    const int64_t part_bytes = P.n_tile_stripes * (s->gstride + 1) * 8;
    s->tl_spart.need(size_t(std::max<int64_t>(part_bytes, 8)), st);
    NWG_CUDA(cudaMemsetAsync(s->tl_spart.p, 0, size_t(part_bytes), st));
    nwg::SoftArgs A{};
    A.a = s->a.as<uint8_t>(); A.oa = s->doa.as<int64_t>();
    A.b = s->b.as<uint8_t>(); A.ob = s->dob.as<int64_t>();
    A.w = dw.p; A.gw = dgw.p; A.N = N; A.K = K;
    A.scratch = s->tl_table.p; A.scratch_stride = stride; A.fwd_bytes = fwd_bytes;
    A.maxn = 0; A.ck = 1; A.max_stripes = 1; A.bnd_off = 0; A.warp_stride = 0;
    A.renorm_mask = renorm - 1;
    A.temperature = J.temperature;
    A.score = s->score.as<double>(); A.grad = s->grad.as<double>(); A.gstride = s->gstride;
    A.status = s->status.as<int32_t>();
    A.spin_limit = s->spin_limit;
    A.queue = s->queue(nwg_store::kQueueHard - 1, st);   // the tile launches run in order: one queue
    A.tile_w = kTileW;
    A.rowf = s->tl_rowf.p; A.rowb = s->tl_rowb.p; A.row_off = P.tile_rowoff.as<int64_t>();
    A.colf = s->tl_colf.p; A.colb = s->tl_colb.p; A.col_off = P.tile_coloff.as<int64_t>();
    A.zpart = s->tl_zpart.as<double>(); A.tile_off = P.tile_slot.as<int64_t>();
    A.zpair = s->tl_zpair.as<double>();
    A.spart = s->tl_spart.as<double>(); A.stripe_off = P.tile_stripeoff.as<int64_t>();
    std::vector<Launch> L;
    const size_t nd = P.diag_off.size() - 1;
    auto diag = [&](size_t d, int phase) {
        const int64_t cnt = P.diag_off[d + 1] - P.diag_off[d];
        A.tiles = P.tile_items.as<int32_t>() + 3 * P.diag_off[d];
        A.n_items = cnt;
        A.tl_phase = phase;
        const int64_t blocks = std::min<int64_t>((cnt + gpb - 1) / gpb, max_blocks);
        L.push_back(make_launch(reinterpret_cast<const void*>(fn), unsigned(blocks), block, smem, A));
    };
    for (size_t d = 0; d < nd; ++d) diag(d, 0);
    nwg::TileSoftArgs Z{};
    Z.pairs = P.tile_plist.as<int32_t>(); Z.n_pairs = nt;
    Z.tile_off = P.tile_slot.as<int64_t>(); Z.tiles_of = P.tile_count.as<int32_t>();
    Z.zpart = s->tl_zpart.as<double>(); Z.zpair = s->tl_zpair.as<double>();
    Z.stripe_off = P.tile_stripeoff.as<int64_t>(); Z.stripes_of = P.tile_nstripes.as<int32_t>();
    Z.spart = s->tl_spart.as<double>(); Z.gw = dgw.p;
    Z.status = s->status.as<int32_t>(); Z.score = s->score.as<double>(); Z.grad = s->grad.as<double>();
    Z.gstride = s->gstride; Z.K = K; Z.N = N; Z.local = loc ? 1 : 0; Z.affine = aff ? 1 : 0;
    Z.temperature = J.temperature;
    L.push_back(make_launch(reinterpret_cast<const void*>(&nwg::tile_z_kernel<T>), unsigned((nt + 127) / 128), 128, 0, Z));
    for (size_t d = nd; d-- > 0;) diag(d, 1);
    L.push_back(make_launch(reinterpret_cast<const void*>(&nwg::tile_finish_kernel<T>), unsigned(nt), 128, 0, Z));
    run_launches(s, &s->g_soft_tile[sizeof(T) == 4 ? 0 : 1], L, st);
}

template <class T>
void soft_pass(nwg_store* s, const nwg_job& J, cudaStream_t st, const std::vector<int32_t>* subset) {
    const bool aff = J.gap_model == 1, loc = J.mode == 1, tr = s->tracked();
    std::vector<T> w, gw;
    bool ovf;
    soft_weights<T>(s, J, w, gw, ovf);
    // renormalisation period: between renormalisations a lane's largest value grows by at most
    // 3 x the largest weight per step, from at most 2^(kLift + 1); keep it below 2^126 (float)
    // or 2^1022 (double)
    double wmax = 1.0;
    for (T v : w) wmax = std::max(wmax, double(v));
    for (T v : gw) wmax = std::max(wmax, double(v));
    const double per_step = std::log2(3.0 * wmax);
    const double room = (sizeof(T) == 4 ? 126.0 : 1022.0) - (nwg::kLift + 1);
    int renorm = int(std::floor(room / per_step));
    if (renorm < 1) ovf = true;
    int pw = 1;
    while (pw * 2 <= std::min(renorm, sizeof(T) == 4 ? 8 : 16)) pw *= 2;
    renorm = pw;
    // after the gap weights: the float32 lost-mass charge per unit of F^ + B^ (nwg_soft.cuh)
    gw.push_back(static_cast<T>(16.0 + 16.0 * std::min(wmax, 1e30)));
    // the weights go to buffers the store keeps (one per precision), so a captured sequence
    // reads this call's weights at the same address
    DBuf& dw = sizeof(T) == 4 ? s->swf : s->swd;
    DBuf& dgw = sizeof(T) == 4 ? s->sgwf : s->sgwd;
    dw.need(w.size() * sizeof(T), st); dgw.need(gw.size() * sizeof(T), st);
    NWG_CUDA(cudaMemcpyAsync(dw.p, w.data(), w.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    NWG_CUDA(cudaMemcpyAsync(dgw.p, gw.data(), gw.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    Plan local_plan;
    Plan* P;
    std::vector<int32_t> order;
    if (subset) {
        // a plan over the subset only (double reruns): one bucket per geometry
        P = &local_plan;
        std::map<std::tuple<int, int, int>, int> idx;
        const bool lane_ok = int64_t(s->K) * s->N * s->N * sizeof(T) * 32 <= 48 * 1024;
        for (int32_t p : *subset) {
            const int m = int(s->oa[p + 1] - s->oa[p]), nb = int(s->ob[p + 1] - s->ob[p]);
            const Geo g = J.band >= 0 ? Geo{32, 4, true}
                        : J.soft_post ? Geo{32, 4}
                        : pick_geo(true, m + 1, nb, J.lanes, J.rows, lane_ok);
            auto key = std::make_tuple(g.G, g.R, size_class(m + 1, nb));
            auto itb = idx.find(key);
            int bi;
            if (itb == idx.end()) { bi = int(P->buckets.size()); idx[key] = bi; P->buckets.push_back(Bucket{g, {}, 0, 0, 0}); }
            else bi = itb->second;
            P->buckets[bi].pairs.push_back(p);
        }
        for (auto& B : P->buckets) {
            B.off = int64_t(order.size());
            for (int32_t p : B.pairs) {
                order.push_back(p);
                const int m = int(s->oa[p + 1] - s->oa[p]), nb = int(s->ob[p + 1] - s->ob[p]);
                B.maxn = std::max(B.maxn, nb);
                const int GR = B.geo.G * B.geo.R;
                const int64_t stp = (m + 1 + GR - 1) / GR;
                B.max_soft_cells = std::max<int64_t>(B.max_soft_cells, stp * (nb + B.geo.G) * GR);
                B.max_rows = std::max(B.max_rows, m + 1);
            }
        }
    } else if (J.band >= 0) {
        P = &s->soft_band_plan;
        build_plan(s, *P, true, 32, 4, sizeof(T), true);
    } else {
        P = &s->soft_plan;
        // posterior guides: every pair at 32 x 4, one warp (the POST kernels)
        build_plan(s, *P, true, J.soft_post ? 32 : J.lanes, J.soft_post ? 4 : J.rows, sizeof(T), false, 0,
                   J.mode == 2 && J.free_ends != 0);
    }
    DBuf sub_order;
    struct Free1 { DBuf& a; cudaStream_t st; ~Free1() { a.release(st); } } fr1{sub_order, st};
    const int32_t* d_order = P->order.as<int32_t>();
    if (subset) {
        sub_order.need(order.size() * 4 + 4, st);
        NWG_CUDA(cudaMemcpyAsync(sub_order.p, order.data(), order.size() * 4, cudaMemcpyHostToDevice, st));
        d_order = sub_order.as<int32_t>();
    }
    const int sms = sm_count(s->device);
    const int NV = aff ? 3 : 1;
    const int64_t budget = scratch_budget_of(s);
    std::vector<Launch> launches;
    std::vector<nwg::SoftArgs> args;
    std::vector<int64_t> need;   // scratch bytes of each launch
    int64_t scratch_total = 0;
    for (auto& B : P->buckets) {
        if (B.pairs.empty() || B.geo.tile) continue;
        Geo gk = B.geo;
        gk.post = J.soft_post != 0;
        SoftFn fn = soft_fn_rt<T>(aff, (J.mode == 2 && J.free_ends) ? 2 : (loc ? 1 : 0), tr, gk);
        if (!fn) throw Error(NWG_EINVAL, "no soft kernel for this geometry");
        const int G = B.geo.G;
        const bool mw = B.geo.mw > 1;            // several warps per pair (long pairs)
        int block = mw ? 32 * B.geo.mw : 128;
        const int K = s->K, N = s->N;
        auto smem_for = [&](int blk) {
            return nwg::soft_smem_bytes(K, N, G, B.geo.R, blk, int(sizeof(T)), tr, mw);
        };
        while (!mw && block > 32 && smem_for(block) > 96 * 1024) block /= 2;
        while (mw && block > 128 && smem_for(block) > 227 * 1024) block /= 2;   // fewer warps per pair
        const size_t smem = smem_for(block);
        if (smem > 227 * 1024) throw Error(NWG_EINVAL, "soft: the alphabet / parameter sets do not fit shared memory");
        NWG_CUDA(nwg::allow_smem(reinterpret_cast<const void*>(fn), smem));
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, block, smem);
        occ = std::max(occ, 1);
        const int gpb = block / G;
        const int64_t items = int64_t(B.pairs.size());
        // checkpointed when a pair's whole forward table would be large: only stripe
        // boundaries are kept, each stripe's table is recomputed just before its backward
        const int64_t GRb = int64_t(G) * B.geo.R;
        const int64_t nb1 = int64_t(B.maxn) + 1;
        const int64_t max_stripes = (B.max_rows + GRb - 1) / GRb;
        const bool ck = mw || B.max_soft_cells * NV * int64_t(sizeof(T)) > s->ck_threshold;
        const int64_t tab_cells = ck ? (nb1 + G) * GRb : B.max_soft_cells;
        const int64_t fwd_bytes = ((tab_cells * NV * int64_t(sizeof(T))) + 255) & ~int64_t(255);
        const int64_t exp_bytes = ((tab_cells / B.geo.R) * 4 + 255) & ~int64_t(255);
        const int64_t nbrows = ck ? max_stripes : 1;
        const int64_t nbrows_b = mw ? max_stripes : 1;
        // boundary rows: per column M (X, Y) and the exponent, as a 2- or 4-vector of T
        const int64_t bnd_bytes = nb1 * (nbrows + nbrows_b) * (aff ? 4 : 2) * int64_t(sizeof(T));
        const int64_t warp_bytes = fwd_bytes + exp_bytes;
        // a slot: one group's table and boundary rows, or (several warps per pair) one block's
        const int64_t stride = (((mw ? gpb : 1) * warp_bytes + bnd_bytes) + 255) & ~int64_t(255);
        const int64_t per_block = mw ? stride : stride * gpb;
        // as many resident groups as fit the device (occupancy) and the scratch budget
        int64_t blocks = std::min<int64_t>(mw ? items : (items + gpb - 1) / gpb, int64_t(sms) * occ);
        blocks = std::max<int64_t>(1, std::min<int64_t>(blocks, budget / std::max<int64_t>(1, per_block)));
        const int64_t slots = mw ? blocks : blocks * gpb;
        scratch_total = std::max<int64_t>(scratch_total, slots * stride);
        nwg::SoftArgs A{};
        const int64_t bucket_need = (slots * stride + 255) & ~int64_t(255);
        A.a = s->a.as<uint8_t>(); A.oa = s->doa.as<int64_t>();
        A.b = s->b.as<uint8_t>(); A.ob = s->dob.as<int64_t>();
        A.tracks = tr ? s->tracks.as<uint16_t>() : nullptr;
        A.gtracks = tr ? s->gtracks.as<uint16_t>() : nullptr;
        A.order = d_order + B.off; A.n_items = items;
        A.w = dw.p; A.gw = dgw.p; A.N = N; A.K = K;
        A.scratch = nullptr; A.scratch_stride = stride; A.fwd_bytes = fwd_bytes;   // set below
        A.maxn = B.maxn; A.temperature = J.temperature;
        A.ck = ck; A.max_stripes = int(std::max<int64_t>(max_stripes, 1));
        A.warp_stride = mw ? warp_bytes : 0;
        A.guide = J.band >= 0 ? s->guide.as<int32_t>() : nullptr; A.band = J.band;
        A.bnd_off = (mw ? gpb : 1) * warp_bytes;
        A.renorm_mask = renorm - 1;
        A.ends = J.mode == 2 ? J.free_ends : 0;
        A.score = s->score.as<double>(); A.grad = s->grad.as<double>(); A.gstride = s->gstride;
        A.status = s->status.as<int32_t>();
        A.spin_limit = s->spin_limit;
        A.queue = s->queue(int(launches.size()), st);
        A.post = J.soft_post ? s->guide.as<int32_t>() : nullptr;
        if (ovf) {
            // a weight overflows T: every pair of this bucket is out of range in T
            mark_status_kernel<<<unsigned((items + 255) / 256), 256, 0, st>>>(A.order, items, A.status,
                                                                                nwg::kSoftWeights);
            NWG_CUDA(cudaGetLastError());
            s->last_launches++;
            continue;
        }
        launches.push_back(make_launch(reinterpret_cast<const void*>(fn), unsigned(blocks), block, smem, A));
        args.push_back(A);
        need.push_back(bucket_need);
    }
    if (!launches.empty()) {
        // the buckets run at once, each in its own part of the scratch, when their parts fit the
        // budget together (a bucket of a few large pairs then shares the device with the others
        // instead of running alone); else one after another in one shared part
        int64_t sum = 0;
        for (int64_t b : need) sum += b;
        const bool concurrent = launches.size() > 1 && sum <= budget;
        s->scratch.need(size_t(concurrent ? sum : scratch_total), st);
        int64_t off = 0;
        for (size_t k = 0; k < launches.size(); ++k) {
            args[k].scratch = static_cast<unsigned char*>(s->scratch.p) + (concurrent ? off : 0);
            off += need[k];
            std::memcpy(launches[k].arg.data(), &args[k], sizeof(nwg::SoftArgs));
        }
        GraphCache* gc = subset ? nullptr : J.band >= 0 ? &s->g_soft_band : &s->g_soft[sizeof(T) == 4 ? 0 : 1];
        run_launches(s, gc, launches, st, concurrent);
    }
    if (!subset && !P->tile_pairs.empty() && !ovf)
        soft_tile_pass<T>(s, J, st, *P, dw, dgw, renorm, loc, aff);
    else if (!subset && !P->tile_pairs.empty()) {
        mark_status_kernel<<<unsigned((P->tile_pairs.size() + 255) / 256), 256, 0, st>>>(
            P->tile_plist.as<int32_t>(), int64_t(P->tile_pairs.size()), s->status.as<int32_t>(), nwg::kSoftWeights);
        NWG_CUDA(cudaGetLastError());
    }
}

// The reason a soft pass refused a pair, from its status bits (the first that applies).
std::string soft_refusal_reason(int32_t why) {
    if (why & nwg::kSoftWeights) return "a substitution or gap weight exp(score / T) overflows";
    if (why & nwg::kSoftRange) return "a forward or backward value overflows";
    if (why & nwg::kSoftZ) return "the partition function Z is zero or out of range";
    if (why & nwg::kSoftScale) return "the forward and backward mass of a cell sit too far apart for the count scale";
    if (why & nwg::kSoftCounts) return "an expected count overflows";
    if (why & nwg::kSoftLoss) return "mass lost to underflow could move a posterior by more than 2^-24";
    return "out of range";
}

void run_soft(nwg_store* s, const nwg_job& J, cudaStream_t st) {
    s->score.need(size_t(std::max<int64_t>(s->n, 1)) * 8, st);
    s->grad.need(size_t(s->n) * s->gstride * 8 + 8, st);
    s->status.need(size_t(std::max<int64_t>(s->n, 1)) * 4, st);
    NWG_CUDA(cudaMemsetAsync(s->status.p, 0, size_t(std::max<int64_t>(s->n, 1)) * 4, st));
    const bool f32 = J.precision == 32 && !J.soft_double;
    if (f32) soft_pass<float>(s, J, st, nullptr);
    else soft_pass<double>(s, J, st, nullptr);
    s->h_status.assign(size_t(s->n), 0);
    if (s->n) NWG_CUDA(cudaMemcpyAsync(s->h_status.data(), s->status.p, size_t(s->n) * 4, cudaMemcpyDeviceToHost, st));
    NWG_CUDA(cudaStreamSynchronize(st));
    auto stall_check = [&](const std::vector<int32_t>& hs) {
        for (int64_t p = 0; p < s->n; ++p)
            if (hs[size_t(p)] & nwg::kSoftStall)
                throw Error(NWG_ECUDA, "nwgrad_b200: soft pass: a wait between the warps of pair " + std::to_string(p) +
                                       " ran out (the kernel gave up instead of hanging)");
    };
    stall_check(s->h_status);
    std::vector<int32_t> refused;
    for (int64_t p = 0; p < s->n; ++p)
        if (s->h_status[p]) refused.push_back(int32_t(p));
    if (refused.empty()) return;
    // pairs the float32 pass refused (out of range, or a lost-mass bound above tolerance) rerun
    // in double, as the reference's run_fwdbwd does (aligner.hpp:6554-6626); a pair the double
    // pass refuses too is an error naming the reason
    std::vector<int32_t> why(s->h_status.begin(), s->h_status.end());
    std::vector<int32_t> left = refused;
    if (f32) {
        soft_pass<double>(s, J, st, &left);
        std::vector<int32_t> hs(size_t(s->n));
        NWG_CUDA(cudaMemcpyAsync(hs.data(), s->status.p, size_t(s->n) * 4, cudaMemcpyDeviceToHost, st));
        NWG_CUDA(cudaStreamSynchronize(st));
        stall_check(hs);
        std::vector<int32_t> still;
        for (int32_t p : left)
            if (hs[size_t(p)]) { still.push_back(p); why[size_t(p)] = hs[size_t(p)]; }
        left.swap(still);
    }
    // per pair: 1 the float32 pass refused it (reran in double), 2 every pass refused it; the
    // first pass's kSoft* reason bits above bit 8
    for (int32_t p : refused) s->h_status[p] = (f32 ? 1 : 0) | (s->h_status[p] << 8);
    for (int32_t p : left) s->h_status[p] = 2 | (why[size_t(p)] << 8);
    if (!left.empty()) {
        const int32_t p = left.front();
        char buf[512];
        std::snprintf(buf, sizeof buf,
                      "nwgrad: soft path: pair %d (lengths %lld x %lld) does not fit the scaled "
                      "probability-space forward-backward in double precision: %s (typically a very low "
                      "temperature or extreme scores)",
                      p, (long long)(s->oa[p + 1] - s->oa[p]), (long long)(s->ob[p + 1] - s->ob[p]),
                      soft_refusal_reason(why[size_t(p)]).c_str());
        throw Error(NWG_ERANGE, buf);
    }
}

template <class F>
int guarded(F&& f) {
    try {
        f();
        return NWG_OK;
    } catch (const Error& e) {
        g_err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_err = e.what();
        return NWG_EINVAL;
    } catch (...) {
        g_err = "unknown error";
        return NWG_EINVAL;
    }
}

// Upload a batch of pairs into a store (new or reused: buffers only grow), dropping every
// result, guide and plan of the previous pairs; the parameters stay.
void load_pairs(nwg_store* s, const uint8_t* codes_a, const int64_t* off_a, const uint8_t* codes_b,
                const int64_t* off_b, int64_t n_pairs, const uint16_t* tracks, const uint16_t* gap_tracks,
                cudaStream_t st) {
    if (n_pairs < 0) throw Error(NWG_EINVAL, "bad n_pairs");
    const int nalpha = s->nalpha;
    s->n = n_pairs;
    s->oa.assign(off_a, off_a + n_pairs + 1);
    s->ob.assign(off_b, off_b + n_pairs + 1);
    s->total_a = s->oa[n_pairs] - s->oa[0];
    s->total_b = s->ob[n_pairs] - s->ob[0];
    for (int64_t p = 0; p < n_pairs; ++p) {
        if (s->oa[p + 1] < s->oa[p] || s->ob[p + 1] < s->ob[p]) throw Error(NWG_EINVAL, "offsets decrease");
        if (s->oa[p + 1] - s->oa[p] > (1 << 30) || s->ob[p + 1] - s->ob[p] > (1 << 30))
            throw Error(NWG_EINVAL, "sequence too long");
    }
    const int64_t a0 = s->oa[0], b0 = s->ob[0];
    for (auto& v : s->oa) v -= a0;
    for (auto& v : s->ob) v -= b0;
    // the largest code of each side (a branch-free loop the compiler vectorises; large inputs
    // in parallel chunks on host threads)
    auto max_code = [](const uint8_t* x, int64_t len) {
        auto run = [](const uint8_t* y, int64_t l) {
            uint8_t mx = 0;
            for (int64_t k = 0; k < l; ++k) mx = y[k] > mx ? y[k] : mx;
            return mx;
        };
        const int64_t kChunk = int64_t(4) << 20;
        const int nth = int(std::min<int64_t>(8, (len + kChunk - 1) / kChunk));
        if (nth <= 1) return int(run(x, len));
        std::vector<uint8_t> part(size_t(nth), 0);
        std::vector<std::thread> th;
        const int64_t step = (len + nth - 1) / nth;
        for (int t = 0; t < nth; ++t) {
            const int64_t lo = t * step, hi = std::min(len, lo + step);
            th.emplace_back([&, t, lo, hi] { part[size_t(t)] = lo < hi ? run(x + lo, hi - lo) : 0; });
        }
        for (auto& h : th) h.join();
        return int(*std::max_element(part.begin(), part.end()));
    };
    if (s->total_a && max_code(codes_a + a0, s->total_a) >= nalpha) throw Error(NWG_EINVAL, "code out of range in sequence A");
    if (s->total_b && max_code(codes_b + b0, s->total_b) >= nalpha) throw Error(NWG_EINVAL, "code out of range in sequence B");
    s->a.need(size_t(s->total_a) + 16, st);
    s->b.need(size_t(s->total_b) + 16, st);
    if (s->total_a) NWG_CUDA(cudaMemcpyAsync(s->a.p, codes_a + a0, size_t(s->total_a), cudaMemcpyHostToDevice, st));
    if (s->total_b) NWG_CUDA(cudaMemcpyAsync(s->b.p, codes_b + b0, size_t(s->total_b), cudaMemcpyHostToDevice, st));
    s->doa.need(size_t(n_pairs + 1) * 8, st);
    s->dob.need(size_t(n_pairs + 1) * 8, st);
    NWG_CUDA(cudaMemcpyAsync(s->doa.p, s->oa.data(), size_t(n_pairs + 1) * 8, cudaMemcpyHostToDevice, st));
    NWG_CUDA(cudaMemcpyAsync(s->dob.p, s->ob.data(), size_t(n_pairs + 1) * 8, cudaMemcpyHostToDevice, st));
    s->tracked_seq = false;
    s->max_track = 0;
    if (tracks) {
        s->tracked_seq = true;
        s->tracks.need(size_t(std::max<int64_t>(s->total_a, 1)) * 2);
        if (s->total_a) NWG_CUDA(cudaMemcpyAsync(s->tracks.p, tracks + a0, size_t(s->total_a) * 2, cudaMemcpyHostToDevice, st));
        for (int64_t k = 0; k < s->total_a; ++k) s->max_track = std::max<int>(s->max_track, tracks[a0 + k]);
    }
    if (gap_tracks) {
        s->tracked_seq = true;
        if (!tracks) {   // gap tracks alone: the track is all zero
            s->tracks.need(size_t(std::max<int64_t>(s->total_a, 1)) * 2);
            NWG_CUDA(cudaMemsetAsync(s->tracks.p, 0, size_t(std::max<int64_t>(s->total_a, 1)) * 2, st));
        }
        const int64_t rows = s->total_a + n_pairs;
        s->gtracks.need(size_t(rows) * 2);
        NWG_CUDA(cudaMemcpyAsync(s->gtracks.p, gap_tracks + a0, size_t(rows) * 2, cudaMemcpyHostToDevice, st));
        for (int64_t k = 0; k < rows; ++k) s->max_track = std::max<int>(s->max_track, gap_tracks[a0 + k]);
    }
    if (s->K && s->tracked_seq && s->max_track >= s->K)
        throw Error(NWG_EINVAL, "nwgrad: a track entry is not a parameter set");
    // the host buffers may be reused by the caller after this returns
    NWG_CUDA(cudaStreamSynchronize(st));
    s->hard_plan.reset(); s->soft_plan.reset(); s->band_plan.reset(); s->soft_band_plan.reset();
    s->have_scores = s->have_grads = s->have_guides = s->have_paths = false;
    s->h_status.clear();
}

}  // namespace

extern "C" {

const char* nwg_last_error(void) { return g_err.c_str(); }

int nwg_store_create(const uint8_t* codes_a, const int64_t* off_a, const uint8_t* codes_b,
                     const int64_t* off_b, int64_t n_pairs, int nalpha, const uint16_t* tracks,
                     const uint16_t* gap_tracks, int device, nwg_store** out) {
    return guarded([&] {
        if (!out) throw Error(NWG_EINVAL, "out is null");
        if (nalpha <= 0 || nalpha > 255) throw Error(NWG_EINVAL, "bad nalpha");
        auto s = std::make_unique<nwg_store>();
        s->device = device;
        NWG_CUDA(cudaSetDevice(device));
        s->nalpha = nalpha;
        keep_pool(device);
        NWG_CUDA(cudaEventCreate(&s->ev0));
        NWG_CUDA(cudaEventCreate(&s->ev1));
        load_pairs(s.get(), codes_a, off_a, codes_b, off_b, n_pairs, tracks, gap_tracks, nullptr);
        *out = s.release();
    });
}

int nwg_store_load(nwg_store* s, const uint8_t* codes_a, const int64_t* off_a, const uint8_t* codes_b,
                   const int64_t* off_b, int64_t n_pairs, const uint16_t* tracks, const uint16_t* gap_tracks,
                   void* stream) {
    return guarded([&] {
        if (!s) throw Error(NWG_EINVAL, "null store");
        NWG_CUDA(cudaSetDevice(s->device));
        load_pairs(s, codes_a, off_a, codes_b, off_b, n_pairs, tracks, gap_tracks, static_cast<cudaStream_t>(stream));
    });
}

int nwg_store_destroy(nwg_store* s) {
    return guarded([&] {
        if (!s) return;
        cudaSetDevice(s->device);
        s->hard_plan.reset(); s->soft_plan.reset(); s->band_plan.reset(); s->soft_band_plan.reset();
        s->auto_budget = -1;   // a new batch: the budget from the memory free now
        for (DBuf* b : {&s->a, &s->b, &s->doa, &s->dob, &s->tracks, &s->gtracks, &s->matf, &s->gapf, &s->matd,
                        &s->gapd, &s->bx0f, &s->bx0d, &s->score, &s->end, &s->grad, &s->guide, &s->status,
                        &s->stripe_tab, &s->codes, &s->scratch, &s->part, &s->red, &s->moves,
                        &s->moves_off, &s->path_info, &s->tmatf, &s->tgapf, &s->tmatd, &s->tgapd,
                        &s->tbx0f, &s->tbx0d, &s->tscore, &s->tend, &s->hb_pairs, &s->swf, &s->sgwf,
                        &s->swd, &s->sgwd, &s->wq, &s->trow, &s->tcol, &s->tbest, &s->tcell, &s->tgrid,
                        &s->tl_table, &s->tl_rowf, &s->tl_rowb, &s->tl_colf, &s->tl_colb, &s->tl_zpart,
                        &s->tl_zpair, &s->tl_spart})
            b->release();
        for (GraphCache* g : {&s->g_soft[0], &s->g_soft[1], &s->g_soft_band, &s->g_hard[0], &s->g_hard[1],
                              &s->g_hard_band, &s->g_soft_tile[0], &s->g_soft_tile[1]})
            g->reset();
        if (s->gstream) cudaStreamDestroy(s->gstream);
        for (int k = 0; k < nwg_store::kBucketStreams; ++k) {
            if (s->bstream[k]) cudaStreamDestroy(s->bstream[k]);
            if (s->bev_join[k]) cudaEventDestroy(s->bev_join[k]);
        }
        if (s->bev_fork) cudaEventDestroy(s->bev_fork);
        if (s->gev_in) cudaEventDestroy(s->gev_in);
        if (s->gev_out) cudaEventDestroy(s->gev_out);
        if (s->ev0) cudaEventDestroy(s->ev0);
        if (s->ev1) cudaEventDestroy(s->ev1);
        delete s;
    });
}

int nwg_params_set(nwg_store* s, const double* mats, const double* gaps, int K, int N) {
    return guarded([&] {
        if (!s || !mats || !gaps) throw Error(NWG_EINVAL, "null argument");
        if (K < 1 || N < 1 || N != s->nalpha) throw Error(NWG_EINVAL, "params: alphabet size does not match the store");
        if (s->K && (K != s->K)) throw Error(NWG_EINVAL, "set_params() cannot change the number of parameter sets");
        NWG_CUDA(cudaSetDevice(s->device));
        s->K = K; s->N = N;
        s->mats.assign(mats, mats + size_t(K) * N * N);
        s->gaps.assign(gaps, gaps + size_t(4) * K);
        s->gstride = int64_t(K) * N * N + 4 * int64_t(K);
        if (s->tracked_seq && s->max_track >= K)
            throw Error(NWG_EINVAL, "nwgrad: a track entry (" + std::to_string(s->max_track) +
                                        ") is not a parameter set (params has " + std::to_string(K) + ")");
        set_params_dev(s);
        s->have_scores = s->have_grads = s->have_paths = false;
    });
}

int nwg_run(nwg_store* s, const nwg_job* job, void* stream, double* total) {
    return guarded([&] {
        if (!s || !job) throw Error(NWG_EINVAL, "null argument");
        if (!s->K) throw Error(NWG_ESTATE, "params not set");
        const nwg_job J = *job;
        if (J.gap_model < 0 || J.gap_model > 1 || J.mode < 0 || J.mode > 2 || J.grad_mode < 0 || J.grad_mode > 2)
            throw Error(NWG_EINVAL, "bad job");
        if (J.mode == 2) {
            if (J.free_ends < 0 || J.free_ends > 15)
                throw Error(NWG_EINVAL, "nwgrad: free_ends must be a 4-bit flag set (0..15), got " + std::to_string(J.free_ends));
            if (J.band >= 0 && J.free_ends != 12)
                throw Error(NWG_EINVAL, "nwgrad: guide-banded alignment supports the semi-global ends of \"glocal\" "
                                        "only; align these free ends with the full DP");
        }
        if (J.precision != 32 && J.precision != 64) throw Error(NWG_EINVAL, "precision must be 32 or 64");
        if (J.band >= 0 && !s->have_guides) throw Error(NWG_ESTATE, "banded_grad() needs a guide; call score_and_grad() first");
        NWG_CUDA(cudaSetDevice(s->device));
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        s->last_launches = 0;
        NWG_CUDA(cudaEventRecord(s->ev0, st));
        s->have_scores = s->have_grads = s->have_paths = false;
        if (J.grad_mode == 2) {
            if (J.soft_post && (J.band >= 0 || s->tracked()))
                throw Error(NWG_EINVAL, "posterior guides: full DP, untracked batches");
            if (J.soft_post) s->guide.need(size_t(s->total_a + s->n) * 4 + 4, st);
            run_soft(s, J, st);
            if (J.soft_post) s->have_guides = true;
        } else {
            const bool grad = J.grad_mode == 1;
            if (J.precision == 32) run_hard<float>(s, J, st, grad, true);
            else run_hard<double>(s, J, st, grad, true);
            s->have_guides = true;
            s->have_paths = J.keep_paths != 0;
        }
        NWG_CUDA(cudaEventRecord(s->ev1, st));
        NWG_CUDA(cudaStreamSynchronize(st));
        float ms = 0;
        cudaEventElapsedTime(&ms, s->ev0, s->ev1);
        s->last_ms = ms;
        s->have_scores = true;
        s->have_grads = J.grad_mode != 0;
        s->last_grad_mode = J.grad_mode; s->last_gm = J.gap_model; s->last_am = J.mode; s->last_prec = J.precision;
        if (total) {
            std::vector<double> sc(size_t(s->n));
            if (s->n) NWG_CUDA(cudaMemcpy(sc.data(), s->score.p, size_t(s->n) * 8, cudaMemcpyDeviceToHost));
            double t = 0.0;
            for (double v : sc) t += v;
            *total = t;
        }
    });
}

int nwg_resolve_guides(nwg_store* s, const double* mats, const double* gaps, const nwg_job* job, void* stream) {
    return guarded([&] {
        if (!s || !job || !mats || !gaps) throw Error(NWG_EINVAL, "null argument");
        if (!s->K) throw Error(NWG_ESTATE, "params not set");
        NWG_CUDA(cudaSetDevice(s->device));
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        nwg_job J = *job;
        J.grad_mode = 0; J.keep_paths = 0; J.band = -1;
        // the snapshot's parameters and scratch results, swapped in for the hard fill
        std::vector<double> m0 = s->mats, g0 = s->gaps;
        s->mats.assign(mats, mats + m0.size());
        s->gaps.assign(gaps, gaps + g0.size());
        std::swap(s->matf, s->tmatf); std::swap(s->gapf, s->tgapf);
        std::swap(s->matd, s->tmatd); std::swap(s->gapd, s->tgapd);
        std::swap(s->bx0f, s->tbx0f); std::swap(s->bx0d, s->tbx0d);
        std::swap(s->score, s->tscore); std::swap(s->end, s->tend);
        auto restore = [&] {
            s->mats = m0; s->gaps = g0;
            std::swap(s->matf, s->tmatf); std::swap(s->gapf, s->tgapf);
            std::swap(s->matd, s->tmatd); std::swap(s->gapd, s->tgapd);
            std::swap(s->bx0f, s->tbx0f); std::swap(s->bx0d, s->tbx0d);
            std::swap(s->score, s->tscore); std::swap(s->end, s->tend);
        };
        try {
            set_params_dev(s);
            if (J.precision == 32) run_hard<float>(s, J, st, false, true);
            else run_hard<double>(s, J, st, false, true);
            NWG_CUDA(cudaStreamSynchronize(st));
        } catch (...) { restore(); throw; }
        restore();
        s->have_guides = true;
    });
}

int nwg_set_geometry(nwg_store* s, int soft, int size_class_, int lanes, int rows) {
    return guarded([&] {
        if (!s) throw Error(NWG_EINVAL, "null store");
        if (size_class_ < 0) {   // -1: forget every tuned geometry; -2: the plain fill
            s->geo_table.clear();
            s->geo_costs.clear();
            s->plain = size_class_ == -2;
        } else {
            if (!geo_available(soft != 0, lanes, rows)) throw Error(NWG_EINVAL, "no kernel for this geometry");
            s->geo_table[{soft ? 1 : 0, size_class_}] = {lanes, rows};
            s->geo_costs.erase({soft ? 1 : 0, size_class_});
            s->plain = false;
        }
        s->hard_plan.reset(); s->soft_plan.reset(); s->soft_band_plan.reset();
    });
}

int nwg_set_geometry_costs(nwg_store* s, int soft, int size_class_, int n, const int* lanes, const int* rows,
                           const double* ns_per_cell) {
    return guarded([&] {
        if (!s || n < 1 || !lanes || !rows || !ns_per_cell || size_class_ < 0) throw Error(NWG_EINVAL, "bad argument");
        std::vector<nwg_store::GeoCost> v;
        for (int k = 0; k < n; ++k) {
            if (!geo_available(soft != 0, lanes[k], rows[k])) throw Error(NWG_EINVAL, "no kernel for this geometry");
            if (!(ns_per_cell[k] > 0.0) || !std::isfinite(ns_per_cell[k])) throw Error(NWG_EINVAL, "costs must be positive");
            v.push_back({lanes[k], rows[k], ns_per_cell[k]});
        }
        s->geo_costs[{soft ? 1 : 0, size_class_}] = std::move(v);
        s->geo_table.erase({soft ? 1 : 0, size_class_});
        s->plain = false;
        s->hard_plan.reset(); s->soft_plan.reset(); s->soft_band_plan.reset();
    });
}

int nwg_set_memory(nwg_store* s, int64_t scratch_budget_bytes, int64_t checkpoint_bytes) {
    return guarded([&] {
        if (!s) throw Error(NWG_EINVAL, "null store");
        if (scratch_budget_bytes >= 0) s->scratch_budget = std::max<int64_t>(scratch_budget_bytes, 1);
        if (checkpoint_bytes >= 0) s->ck_threshold = checkpoint_bytes;
    });
}

int nwg_set_spin_limit(nwg_store* s, int polls) {
    return guarded([&] {
        if (!s) throw Error(NWG_EINVAL, "null store");
        if (polls < 1) throw Error(NWG_EINVAL, "spin limit must be at least 1 poll");
        s->spin_limit = polls;
    });
}

int nwg_scores(nwg_store* s, double* out) {
    return guarded([&] {
        if (!s->have_scores) throw Error(NWG_ESTATE, "scores not computed; call score_and_grad() first");
        if (s->n) NWG_CUDA(cudaMemcpy(out, s->score.p, size_t(s->n) * 8, cudaMemcpyDeviceToHost));
    });
}

int nwg_grads(nwg_store* s, double* out) {
    return guarded([&] {
        if (!s->have_grads) throw Error(NWG_ESTATE, "gradient not computed; call score_and_grad() or banded_grad() first");
        if (s->n) NWG_CUDA(cudaMemcpy(out, s->grad.p, size_t(s->n) * s->gstride * 8, cudaMemcpyDeviceToHost));
    });
}

int nwg_reduce(nwg_store* s, const double* w, double* out) {
    return guarded([&] {
        if (!s->have_grads) throw Error(NWG_ESTATE, "gradient not computed; call score_and_grad() or banded_grad() first");
        NWG_CUDA(cudaSetDevice(s->device));
        const int64_t gs = s->gstride, n = s->n;
        const int64_t B = 4096, nb = (n + B - 1) / B;
        if (n == 0) { for (int64_t k = 0; k < gs; ++k) out[k] = 0.0; return; }
        s->part.need(size_t(nb * gs) * 8);
        s->red.need(size_t(gs) * 8 + size_t(w ? n : 0) * 8);
        double* dw = nullptr;
        if (w) {
            dw = s->red.as<double>() + gs;
            NWG_CUDA(cudaMemcpy(dw, w, size_t(n) * 8, cudaMemcpyHostToDevice));
        }
        dim3 grid(unsigned((gs + 31) / 32), unsigned(nb));
        if (dw) blocked_partial_kernel<true><<<grid, 32>>>(s->grad.as<double>(), dw, n, gs, B, s->part.as<double>());
        else blocked_partial_kernel<false><<<grid, 32>>>(s->grad.as<double>(), dw, n, gs, B, s->part.as<double>());
        NWG_CUDA(cudaGetLastError());
        blocked_total_kernel<<<unsigned((gs + 127) / 128), 128>>>(s->part.as<double>(), nb, gs, s->red.as<double>());
        NWG_CUDA(cudaGetLastError());
        NWG_CUDA(cudaMemcpy(out, s->red.p, size_t(gs) * 8, cudaMemcpyDeviceToHost));
    });
}

int nwg_reduce_range(nwg_store* s, int64_t start, int64_t end, const double* w, double* out) {
    return guarded([&] {
        if (!s->have_grads) throw Error(NWG_ESTATE, "gradient not computed; call score_and_grad() or banded_grad() first");
        if (start < 0 || end > s->n || start > end) throw Error(NWG_EINVAL, "bad pair range");
        NWG_CUDA(cudaSetDevice(s->device));
        const int64_t gs = s->gstride, n = end - start;
        const int64_t B = 4096, nb = (n + B - 1) / B;
        if (n == 0) { for (int64_t k = 0; k < gs; ++k) out[k] = 0.0; return; }
        s->part.need(size_t(nb * gs) * 8);
        s->red.need(size_t(gs) * 8 + size_t(w ? n : 0) * 8);
        double* dw = nullptr;
        if (w) {
            dw = s->red.as<double>() + gs;
            NWG_CUDA(cudaMemcpy(dw, w, size_t(n) * 8, cudaMemcpyHostToDevice));
        }
        dim3 grid(unsigned((gs + 31) / 32), unsigned(nb));
        if (dw) blocked_partial_kernel<true><<<grid, 32>>>(s->grad.as<double>() + start * gs, dw, n, gs, B, s->part.as<double>());
        else blocked_partial_kernel<false><<<grid, 32>>>(s->grad.as<double>() + start * gs, dw, n, gs, B, s->part.as<double>());
        NWG_CUDA(cudaGetLastError());
        blocked_total_kernel<<<unsigned((gs + 127) / 128), 128>>>(s->part.as<double>(), nb, gs, s->red.as<double>());
        NWG_CUDA(cudaGetLastError());
        NWG_CUDA(cudaMemcpy(out, s->red.p, size_t(gs) * 8, cudaMemcpyDeviceToHost));
    });
}

int nwg_scores_range(nwg_store* s, int64_t start, int64_t end, double* out) {
    return guarded([&] {
        if (!s->have_scores) throw Error(NWG_ESTATE, "scores not computed; call score_and_grad() first");
        if (start < 0 || end > s->n || start > end) throw Error(NWG_EINVAL, "bad pair range");
        if (end > start) NWG_CUDA(cudaMemcpy(out, s->score.as<double>() + start, size_t(end - start) * 8, cudaMemcpyDeviceToHost));
    });
}

int nwg_guides(nwg_store* s, int32_t* out) {
    return guarded([&] {
        if (!s->have_guides) throw Error(NWG_ESTATE, "no guide: run score_and_grad() first");
        const size_t k = size_t(s->total_a + s->n);
        if (k) NWG_CUDA(cudaMemcpy(out, s->guide.p, k * 4, cudaMemcpyDeviceToHost));
    });
}

int nwg_set_guides(nwg_store* s, const int32_t* in) {
    return guarded([&] {
        const size_t k = size_t(s->total_a + s->n);
        s->guide.need(k * 4 + 4);
        if (k) NWG_CUDA(cudaMemcpy(s->guide.p, in, k * 4, cudaMemcpyHostToDevice));
        s->have_guides = true;
    });
}

int nwg_paths(nwg_store* s, int64_t* moves_off, uint8_t* moves, int64_t moves_cap, int32_t* path_info,
              int32_t* ends) {
    return guarded([&] {
        if (!s->have_paths) throw Error(NWG_ESTATE, "no stored path: score_and_grad(keep_paths=True) first");
        std::vector<int64_t> mo(s->n + 1, 0);
        for (int64_t p = 0; p < s->n; ++p) mo[p + 1] = mo[p] + (s->oa[p + 1] - s->oa[p]) + (s->ob[p + 1] - s->ob[p]);
        if (moves_off) std::memcpy(moves_off, mo.data(), size_t(s->n + 1) * 8);
        if (moves) {
            if (moves_cap < mo[s->n]) throw Error(NWG_EINVAL, "moves buffer too small");
            if (mo[s->n]) NWG_CUDA(cudaMemcpy(moves, s->moves.p, size_t(mo[s->n]), cudaMemcpyDeviceToHost));
        }
        if (path_info && s->n) NWG_CUDA(cudaMemcpy(path_info, s->path_info.p, size_t(s->n) * 12, cudaMemcpyDeviceToHost));
        if (ends && s->n) {
            std::vector<int32_t> e(size_t(s->n) * 4);
            NWG_CUDA(cudaMemcpy(e.data(), s->end.p, e.size() * 4, cudaMemcpyDeviceToHost));
            for (int64_t p = 0; p < s->n; ++p) { ends[2 * p] = e[4 * p]; ends[2 * p + 1] = e[4 * p + 1]; }
        }
    });
}

int nwg_status(nwg_store* s, int32_t* out) {
    return guarded([&] {
        for (int64_t p = 0; p < s->n; ++p) out[p] = p < int64_t(s->h_status.size()) ? s->h_status[p] : 0;
    });
}

int nwg_set_graphs(nwg_store* s, int enable) {
    return guarded([&] {
        if (!s) throw Error(NWG_EINVAL, "null argument");
        s->use_graphs = enable != 0;
    });
}

int nwg_graph_stats(nwg_store* s, int64_t* captures, int64_t* replays) {
    return guarded([&] {
        if (!s) throw Error(NWG_EINVAL, "null argument");
        if (captures) *captures = s->graph_captures;
        if (replays) *replays = s->graph_replays;
    });
}

int nwg_last_timing(nwg_store* s, double* ms, int64_t* launches) {
    return guarded([&] {
        if (ms) *ms = s->last_ms;
        if (launches) *launches = s->last_launches;
    });
}

}  // extern "C"
