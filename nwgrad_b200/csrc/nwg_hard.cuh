// Hard (Viterbi) path: the guide-free full fill with predecessor codes, and the traceback.
//
// Fill.  A group of G lanes owns one pair; DP rows are cut into stripes of G*R rows and
// lane g of the group owns rows [g*R, g*R + R) of the current stripe, its R cells of one
// column held in registers.  Lanes run skewed by one column (a wavefront): at step t lane
// g fills column j = t - g + 1, reading the row above from lane g-1 by a warp shuffle
// (lane 0: from the previous stripe's bottom row in scratch, or the row-0 border).  G = 1
// is the one-pair-per-lane ("inter-pair") kernel for short pairs; G = 32 one warp per pair.
//
// Every cell is the reference recurrence, expression for expression
// (aligner.hpp:3955-4071 affine, 3756-3860 linear): (v - go) - ge left-associated, >=
// tie-breaks in M > X > Y order, parameters cast to T once.  The evaluation order across cells
// differs, but each cell is a fixed expression of its three neighbours, so the tables are
// bit-identical.  Maxima use the hardware max (fmax): it returns the same value as the
// reference's std::max except for the sign of an exact zero (the parameters are finite, so no
// NaN arises), and the codes, end cells and gradients depend only on comparisons, which do
// not see that sign.
//
// Codes: one byte per cell, affine M | X << 2 | Y << 4, linear 0 diag / 1 up / 2 left with
// 3 = stop (Local, value <= 0).  Layout per pair, per stripe s (S8 = n + G - 1 steps rounded
// up to a multiple of 8):
//   byte s * S8 * G * R + ((t / 8 * G + g) * 8 + t % 8) * R + r,
// i.e. tiles of 8 steps x R rows per lane: the fill's per-step store is R bytes per lane, and
// the traceback, which mostly steps diagonally (t - 1, r - 1), reads one tile for several
// steps.  Border cells (row 0, column 0) are not stored: the walk knows them.
#pragma once
#include "nwg_common.cuh"
#include "nwg_walk.cuh"

namespace nwg {

struct HardArgs {
    const uint8_t* a; const int64_t* oa;       // codes of A, n_pairs + 1 offsets
    const uint8_t* b; const int64_t* ob;
    const uint16_t* tracks;                    // per residue of A (oa offsets), or null
    const uint16_t* gtracks;                   // per DP row (oa[p] + p offsets), or null
    const void* bx0;                           // tracked: column-0 border per row (oa[p] + p), T
    const int32_t* order;                      // the pairs of this launch
    int64_t n_items;
    const void* mat;                           // K*N*N in T
    const void* gaps;                          // K*4 in T
    int N, K;
    uint8_t* codes; const int64_t* code_off;   // per pair code table
    void* scratch; int64_t scratch_stride;     // per group slot: the stripe boundary row, 3*(n+1) T
    double* score;                             // per pair
    int32_t* end;                              // per pair: end_i, end_j, state, layout (G<<8|R)
    // guide-banded re-alignment (BAND kernels only)
    const int32_t* guide;                      // per pair m+1 at oa[p] + p
    int band;                                  // half-width
    const int64_t* stripe_base;                // per pair: first entry in stripe_tab
    int64_t* stripe_tab;                       // per stripe: code offset in the pair, first column
    // one warp per pair: lane 0 walks the pair's codes as soon as its fill is done
    int walk_fused;
    WalkArgs walk;
    // semi-global free ends (Global kernels, full DP, one warp or lane per pair): 1 a_begin
    // (column 0 a free start), 2 a_end (column n's cells ends), 4 b_begin (row 0 a free start),
    // 8 b_end (row m's cells ends); 0: Global's charged borders and end (m, n)
    int ends;
    int* queue;                                // this launch's work-queue counters (2 ints, zero at launch)
    // tiled long pairs (TL kernels): an item is one tile -- stripe s of pair p over columns
    // c W + 1 .. (c + 1) W -- and a launch holds one anti-diagonal (s + c) of every pair's tiles
    const int32_t* tiles;                      // per item: p, s, c
    int tile_w;                                // W, a multiple of 8
    void* rowbuf; const int64_t* rowbuf_off;   // per pair, per stripe its bottom row: (n + 1) x 3 T
    void* colbuf; const int64_t* colbuf_off;   // per pair, per stripe and tile its last column: G R x 3 T
    void* tbest; int32_t* tcell;               // Local: per tile its first row-major best and cell (i, j, state)
    const int64_t* tile_off;                   // per pair: its first tile's slot in tbest / tcell
};

// The band of DP row i around guide g (aligner.hpp:2644-2700): columns [jlo, jhi].
struct BandRows {
    const int32_t* g; int band, m, n; bool global;
    __device__ __forceinline__ int jlo(int i) const { return max(1, g[i] - band); }
    __device__ __forceinline__ int jhi(int i) const {
        if (global && i == m) return n;
        int hi = g[i] + band;
        if (i < m) hi = max(hi, g[i + 1] - 1 + band);
        return min(n, hi);
    }
};

template <class T> struct HardRowParams { T goa, gea, gob, geb; };

// Column-0 border of DP row i >= 1 (Global): untracked closed form or the tracked table.
template <class T, bool AFF, bool TR>
__device__ __forceinline__ T border_col0(const HardArgs& A, const T* bx0p, int i, T gob, T geb) {
    if constexpr (TR) return bx0p[i];
    else {
        if constexpr (AFF) return -add_rn(gob, mul_rn(static_cast<T>(i), geb));
        else return mul_rn(-static_cast<T>(i), geb);
    }
}

// The first of the maxima among end candidates offered in order (strict >), its state by
// M > X > Y (aligner.hpp:6160-6170, SgEnd).
template <class T> struct EndPick {
    T v; int i, j, st; bool any;
    __device__ __forceinline__ void init() { v = T(0); i = 0; j = 0; st = 0; any = false; }
    __device__ __forceinline__ void offer(int ci, int cj, T vm, T vx, T vy) {
        const T w = rmax3(vm, vx, vy);
        if (any && !(w > v)) return;
        v = w; i = ci; j = cj; any = true;
        st = (vm >= vx && vm >= vy) ? 0 : (vx >= vy ? 1 : 2);
    }
};

// SG: the semi-global ends of A.ends (Global fills only, full DP, a warp or lane per pair)
// TL: tiled long pairs (A.tiles): each item one stripe of one pair over one tile of columns; the
// tile's top row comes from the stripe above (rowbuf), its left column from the tile to its left
// (colbuf), and its codes go where the full fill would put them, so the walk reads them as usual
// (A.codes null: no codes -- the grid traceback's score-only pass, which keeps only the rows and
// columns).
// GW: the grid traceback (aligner.hpp:89-100, viterbi_affine_grid :5327) over those rows and
// columns: a warp per pair (A.order) walks back from the end cell, and each time the path enters
// a tile the warp fills that tile again, with codes, into its own tile buffer (A.scratch).  The
// refill starts from the same row and column values as the first pass, so its codes are the
// Pointers fill's, bit for bit; memory is the grid of rows and columns, not a code per cell.
template <class T, bool AFF, bool LOC, bool TR, int G, int R, bool BAND = false, bool SG = false, bool TL = false,
          bool GW = false>
__global__ void __launch_bounds__(128) hard_fill_kernel(const HardArgs A) {
    static_assert(!TL || (G == 32 && !BAND && !SG), "tiles: 32 lanes, full DP, Global or Local");
    static_assert(!GW || TL, "the grid walk refills tiles");
    static_assert(!SG || !LOC, "semi-global ends: Global fills, one warp or lane per pair");
    constexpr int GR = G * R;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smat = reinterpret_cast<T*>(smem_raw);
    const int nmat = A.K * A.N * A.N;
    T* sgap = smat + nmat;
    for (int k = threadIdx.x; k < nmat; k += blockDim.x) smat[k] = static_cast<const T*>(A.mat)[k];
    for (int k = threadIdx.x; k < 4 * A.K; k += blockDim.x) sgap[k] = static_cast<const T*>(A.gaps)[k];
    __syncthreads();

    const int lane = threadIdx.x % G;
    const int gpb = blockDim.x / G;
    const int gib = threadIdx.x / G;
    const int64_t slot = int64_t(blockIdx.x) * gpb + gib;
    unsigned gmask;
    if constexpr (G == 32) gmask = 0xffffffffu;
    else gmask = ((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1));
    T* const bnd0 = static_cast<T*>(A.scratch) + slot * A.scratch_stride;
    const int N = A.N;
    // the next item (pair, or tile) of this group from the launch's work queue, in the
    // longest-first order: a group that finishes early takes the next one
    auto next_item = [&]() -> int64_t {
        long long v = 0;
        if (lane == 0) v = wq_next(A.queue, int(gridDim.x) * gpb, A.n_items);
        if constexpr (G > 1) v = __shfl_sync(gmask, v, 0, G);
        return v;
    };
    for (int64_t it = next_item(); it < A.n_items; it = next_item()) {
        const int p = (TL && !GW) ? A.tiles[3 * it] : A.order[it];
        // TL: the item's stripe and tile (GW: those of the tile being refilled)
        int ts = (TL && !GW) ? A.tiles[3 * it + 1] : 0, tc = (TL && !GW) ? A.tiles[3 * it + 2] : 0;
        const int64_t ao = A.oa[p], bo = A.ob[p];
        const int m = int(A.oa[p + 1] - ao), n = int(A.ob[p + 1] - bo);
        const uint8_t* __restrict__ ap = A.a + ao;
        const uint8_t* __restrict__ bp = A.b + bo;
        const uint16_t* tk = TR ? A.tracks + ao : nullptr;
        const uint16_t* gk = (TR && A.gtracks) ? A.gtracks + ao + p : nullptr;
        const T* bx0p = TR ? static_cast<const T*>(A.bx0) + ao + p : nullptr;
        // set of DP row i: matches / gaps in B (tset, i >= 1), gaps in A (gset, i >= 0)
        auto tset = [&](int i) -> int { return TR ? int(tk[i - 1]) : 0; };
        auto gset = [&](int i) -> int {
            if constexpr (!TR) return 0;
            if (gk) return int(gk[i]);
            return i == 0 ? (m ? int(tk[0]) : 0) : int(tk[i - 1]);
        };
        const T goa0 = sgap[4 * gset(0) + 0], gea0 = sgap[4 * gset(0) + 1];
        const T ugob = sgap[2], ugeb = sgap[3], ugoa = sgap[0], ugea = sgap[1];
        const bool sg_r0 = SG && (A.ends & 4), sg_c0 = SG && (A.ends & 1);
        const bool sg_ec = SG && (A.ends & 2), sg_er = SG && (A.ends & 8);
        if (m == 0 || n == 0) {
            if (lane == 0) {
                T sc; int ei, ej, st;
                if (LOC) { sc = T(0); ei = 0; ej = 0; st = 0; }
                else if (SG) {
                    // semi-global: the border cells in the reference's order (column n of rows
                    // 0..m-1, then row m), each from its closed form
                    auto cell = [&](int ci, int cj, T& vm, T& vx, T& vy) {
                        vm = ninf<T>(); vx = ninf<T>(); vy = ninf<T>();
                        if (ci == 0 && (cj == 0 || sg_r0)) vm = T(0);
                        else if (ci == 0) {
                            if constexpr (AFF) vy = -add_rn(goa0, mul_rn(static_cast<T>(cj), gea0));
                            else vm = mul_rn(-static_cast<T>(cj), gea0);
                        } else if (sg_c0) vm = T(0);
                        else {
                            const T bc = border_col0<T, AFF, TR>(A, bx0p, ci, ugob, ugeb);
                            if constexpr (AFF) vx = bc; else vm = bc;
                        }
                    };
                    EndPick<T> e; e.init();
                    T vm, vx, vy;
                    if (sg_ec) for (int ci = 0; ci < m; ++ci) { cell(ci, n, vm, vx, vy); e.offer(ci, n, vm, vx, vy); }
                    for (int cj = sg_er ? 0 : n; cj <= n; ++cj) { cell(m, cj, vm, vx, vy); e.offer(m, cj, vm, vx, vy); }
                    sc = e.v; ei = e.i; ej = e.j; st = e.st;
                }
                else if (m == 0 && n == 0) { sc = T(0); ei = 0; ej = 0; st = 0; }
                else if (m == 0) {
                    sc = AFF ? -add_rn(goa0, mul_rn(static_cast<T>(n), gea0)) : mul_rn(-static_cast<T>(n), gea0);
                    ei = 0; ej = n; st = 2;
                } else {
                    const T gob = TR ? sgap[4 * tset(1) + 2] : ugob;
                    const T geb = TR ? sgap[4 * tset(m) + 3] : ugeb;
                    sc = border_col0<T, AFF, TR>(A, bx0p, m, gob, geb);
                    ei = m; ej = 0; st = AFF ? 1 : 0;
                }
                A.score[p] = static_cast<double>(sc);
                A.end[4 * p] = ei; A.end[4 * p + 1] = ej; A.end[4 * p + 2] = st;
                A.end[4 * p + 3] = (G << 8) | R;
                // an empty side: the walk runs the border (no codes read)
                if (!TL && A.walk_fused) walk_pair(A.walk, p);
            }
            continue;
        }
        uint8_t* __restrict__ codes = (TL && !A.codes) ? nullptr : A.codes + A.code_off[p];
        const int nstripes = (m + GR - 1) / GR;
        // the band (full DP: every column of every row; borders reach every row / column)
        BandRows bw{BAND ? A.guide + ao + p : nullptr, A.band, m, n, !LOC && !SG};   // glocal: row m's own band
        int brows = m, bcols = n;            // rows / columns whose border cells are charged
        if constexpr (BAND) {
            brows = 0;
            while (brows < m && bw.g[brows + 1] <= A.band) ++brows;
            bcols = bw.jhi(0);
        }
        int64_t soff = 0;                     // this stripe's code offset within the pair
        int pmin = 1, pmax = TL ? n : 0;      // the previous stripe's columns (TL: all of them)

        T bestv = T(0); int besti = 0, bestj = 0, bests = 0;   // Local: the first row-major max
        T endM = ninf<T>(), endX = ninf<T>(), endY = ninf<T>();
        // semi-global: the first max of row m (from column 0's border cell) and of column n's
        // rows 0..m-1 (from row 0's cell); the lane holding row m tracks the former
        EndPick<T> erow, ecol;
        erow.init(); ecol.init();
        if constexpr (SG) {
            T vm, vx, vy;
            if (sg_c0) { vm = T(0); vx = ninf<T>(); vy = ninf<T>(); }
            else {
                // banded: column 0's cell of row m is charged only within the border rows
                const T bc = (!BAND || m <= brows) ? border_col0<T, AFF, TR>(A, bx0p, m, ugob, ugeb) : ninf<T>();
                vm = AFF ? ninf<T>() : bc; vx = AFF ? bc : ninf<T>(); vy = ninf<T>();
            }
            erow.offer(m, 0, vm, vx, vy);
            if (sg_ec) {
                if (sg_r0) { vm = T(0); vy = ninf<T>(); }
                else if constexpr (AFF) { vm = ninf<T>(); vy = -add_rn(goa0, mul_rn(static_cast<T>(n), gea0)); }
                else { vm = mul_rn(-static_cast<T>(n), gea0); vy = ninf<T>(); }
                ecol.offer(0, n, vm, ninf<T>(), vy);
            }
        }

        T* const rows_p = TL ? static_cast<T*>(A.rowbuf) + A.rowbuf_off[p] : nullptr;
        T* const cols_p = TL ? static_cast<T*>(A.colbuf) + A.colbuf_off[p] : nullptr;
        const int ntc = TL ? (n + A.tile_w - 1) / A.tile_w : 1;   // TL: tiles per stripe
        // GW: the walker lives in lane 0; each pass of the loop below refills the tile holding the
        // next code the walk needs, then walks on until the path leaves it (other fills: one pass)
        Walker wk;
        uint8_t* const tilebuf = GW ? static_cast<uint8_t*>(A.scratch) + slot * A.scratch_stride : nullptr;
        auto tile_code = [&](int ci, int cj) -> uint32_t {
            const int w = ci - 1 - ts * GR, gg = w / R, rr = w - gg * R;
            const int t = cj - tc * A.tile_w - 1 + gg;
            return tilebuf[((int64_t(t >> 3) * G + gg) * 8 + (t & 7)) * R + rr];
        };
        if constexpr (GW) { if (lane == 0) wk.init(A.walk, p); }
        // a monotone path crosses at most nstripes + ntc - 1 tiles: the bound only guards the loop
        for (int pass = 0, more = 1; more && pass <= nstripes + ntc; ++pass) {
            more = 0;
            if constexpr (GW) {
                const int wi = __shfl_sync(gmask, wk.i, 0), wj = __shfl_sync(gmask, wk.j, 0);
                if (__shfl_sync(gmask, wk.done ? 1 : 0, 0)) break;
                more = 1;
                if (wi == 0 || wj == 0) {   // the rest is border moves: no codes
                    if (lane == 0) wk.run(tile_code, 1, 1);
                    continue;
                }
                ts = (wi - 1) / GR;
                tc = (wj - 1) / A.tile_w;
            }
        for (int s = TL ? ts : 0; s < (TL ? ts + 1 : nstripes); ++s) {
            // the previous stripe's bottom row (read) and this stripe's (written; one row in
            // place, except for tiles: a row per stripe)
            T* const bnd = TL ? rows_p + int64_t(s - 1) * 3 * (n + 1) : bnd0;
            T* const bnd_out = TL ? rows_p + int64_t(s) * 3 * (n + 1) : bnd0;
            const int i0 = s * GR + lane * R + 1;   // this lane's first DP row
            // the stripe's columns [cmin, cmax]: the union of its rows' bands (TL: the tile's)
            int cmin = TL ? tc * A.tile_w + 1 : 1, cmax = TL ? min(n, (tc + 1) * A.tile_w) : n;
            // TL: the column left of the tile, GR rows x 3 values, and this tile's last column
            const T* const lcol = TL && tc > 0 ? cols_p + (int64_t(s) * ntc + tc - 1) * 3 * GR : nullptr;
            T* const rcol = TL ? cols_p + (int64_t(s) * ntc + tc) * 3 * GR : nullptr;
            int rlo[BAND ? R : 1], rhi[BAND ? R : 1];
            if constexpr (BAND) {
                int lo = n + 1, hi = 0;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int i = i0 + r;
                    rlo[r] = i <= m ? bw.jlo(i) : n + 1;
                    rhi[r] = i <= m ? bw.jhi(i) : 0;
                    if (rlo[r] <= rhi[r]) { lo = min(lo, rlo[r]); hi = max(hi, rhi[r]); }
                }
                if constexpr (G > 1) {
#pragma unroll
                    for (int off = G / 2; off > 0; off >>= 1) {
                        lo = min(lo, __shfl_xor_sync(gmask, lo, off, G));
                        hi = max(hi, __shfl_xor_sync(gmask, hi, off, G));
                    }
                }
                cmin = lo; cmax = hi;
                if (lane == 0) {
                    A.stripe_tab[2 * (A.stripe_base[p] + s)] = soff;
                    A.stripe_tab[2 * (A.stripe_base[p] + s) + 1] = cmin;
                }
            }
            const int S = cmax >= cmin ? (cmax - cmin + 1) + G - 1 : 0;
            const int S8 = (S + 7) & ~7;
            int rowbase[R];
            T cM[R], cX[R], cY[R];
            HardRowParams<T> rp[TR ? R : 1];
            T rbest[LOC ? R : 1]; int rbj[LOC ? R : 1]; int rbs[LOC ? R : 1];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = i0 + r;
                const bool valid = i <= m;
                const int key = valid ? (TR ? tset(i) * N + ap[i - 1] : int(ap[i - 1])) : 0;
                rowbase[r] = key * N;
                if constexpr (TR) {
                    const int gs = valid ? gset(i) : 0, ts = valid ? tset(i) : 0;
                    rp[r].goa = sgap[4 * gs + 0]; rp[r].gea = sgap[4 * gs + 1];
                    rp[r].gob = sgap[4 * ts + 2]; rp[r].geb = sgap[4 * ts + 3];
                }
                // the cell left of the stripe's first column: column 0's border, or out of band
                // (TL: the tile to the left's last column, its own rows)
                if constexpr (LOC) { rbest[r] = T(0); rbj[r] = 0; rbs[r] = 0; }
                if (TL && cmin > 1) {
                    const int q = lane * R + r;
                    cM[r] = lcol[3 * q]; cX[r] = lcol[3 * q + 1]; cY[r] = lcol[3 * q + 2];
                    continue;
                }
                if constexpr (LOC) {
                    cM[r] = cmin == 1 ? T(0) : ninf<T>(); cX[r] = ninf<T>();
                } else if (sg_c0 && cmin == 1) {
                    cM[r] = T(0); cX[r] = ninf<T>();   // column 0 a free start
                } else {
                    cM[r] = ninf<T>();
                    cX[r] = (valid && cmin == 1 && i <= brows) ? border_col0<T, AFF, TR>(A, bx0p, i, ugob, ugeb) : ninf<T>();
                    if constexpr (!AFF) cM[r] = cX[r];   // linear: H lives in cM
                }
                cY[r] = ninf<T>();
            }
            // row 0 at column j (Global: the charged gap chain up to bcols; Local: free starts)
            auto row0 = [&](int j, T& vM, T& vX, T& vY) {
                vX = ninf<T>();
                if constexpr (LOC) { vM = T(0); vY = ninf<T>(); }
                else if (j == 0 || sg_r0) { vM = T(0); vY = ninf<T>(); }
                else if constexpr (AFF) {
                    vM = ninf<T>();
                    vY = j <= bcols ? -add_rn(goa0, mul_rn(static_cast<T>(j), gea0)) : ninf<T>();
                } else {
                    vM = j <= bcols ? mul_rn(-static_cast<T>(j), gea0) : ninf<T>(); vY = ninf<T>();
                }
            };
            // the row above this lane's first row, at column cmin - 1
            T dgM, dgX, dgY;
            {
                const int i = i0 - 1;
                if (cmin == 1) {
                    if (i == 0) { dgM = T(0); dgX = ninf<T>(); dgY = ninf<T>(); }
                    else if (LOC || sg_c0) { dgM = T(0); dgX = ninf<T>(); dgY = ninf<T>(); }
                    else {
                        dgX = i <= brows ? border_col0<T, AFF, TR>(A, bx0p, i, ugob, ugeb) : ninf<T>();
                        dgM = AFF ? ninf<T>() : dgX; dgY = ninf<T>();
                    }
                } else if (lane == 0 && s == 0) {
                    row0(cmin - 1, dgM, dgX, dgY);
                } else if (lane == 0 && cmin - 1 >= pmin && cmin - 1 <= pmax) {
                    dgM = bnd[3 * (cmin - 1)]; dgX = bnd[3 * (cmin - 1) + 1]; dgY = bnd[3 * (cmin - 1) + 2];
                } else if (TL && lane > 0) {   // the lane above's last row in the tile to the left
                    const int q = lane * R - 1;
                    dgM = lcol[3 * q]; dgX = lcol[3 * q + 1]; dgY = lcol[3 * q + 2];
                } else { dgM = ninf<T>(); dgX = ninf<T>(); dgY = ninf<T>(); }
            }
            T upM = ninf<T>(), upX = ninf<T>(), upY = ninf<T>();
            // TL: the tile's steps start (cmin - 1) steps into the stripe's full-width codes
            uint8_t* cs = GW ? tilebuf
                        : TL ? (codes ? codes + int64_t(s) * ((n + G - 1 + 7) & ~7) * GR + int64_t((cmin - 1) >> 3) * G * 8 * R
                                      : nullptr)
                             : codes + (BAND ? soff : int64_t(s) * S8 * GR);
            // lane 0: the row above one column ahead, so the load is in flight meanwhile
            T nuM = ninf<T>(), nuX = ninf<T>(), nuY = ninf<T>();
            auto fetch_up = [&](int jj) {
                if (lane == 0 && s > 0 && jj <= cmax) {
                    if (!BAND || (jj >= pmin && jj <= pmax)) { nuM = bnd[3 * jj]; nuX = bnd[3 * jj + 1]; nuY = bnd[3 * jj + 2]; }
                    else { nuM = ninf<T>(); nuX = ninf<T>(); nuY = ninf<T>(); }
                }
            };
            fetch_up(cmin);

            for (int t = 0; t < S; ++t) {
                const int j = cmin + t - lane;
                if (lane == 0 && j <= cmax) {
                    if (s == 0) row0(j, upM, upX, upY);
                    else { upM = nuM; upX = nuX; upY = nuY; fetch_up(j + 1); }
                }
                const bool active = (j >= cmin) && (j <= cmax);
                if (active) {
                    const int bj = bp[j - 1];
                    T pM = dgM, pX = dgX, pY = dgY;   // row above, column j-1
                    T qM = upM, qX = upX, qY = upY;   // row above, column j
                    uint32_t w[(R + 3) / 4];
#pragma unroll
                    for (int k = 0; k < (R + 3) / 4; ++k) w[k] = 0u;
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const T sub = smat[rowbase[r] + bj];
                        T go_a, ge_a, go_b, ge_b;
                        if constexpr (TR) { go_a = rp[r].goa; ge_a = rp[r].gea; go_b = rp[r].gob; ge_b = rp[r].geb; }
                        else { go_a = ugoa; ge_a = ugea; go_b = ugob; ge_b = ugeb; }
                        uint32_t code;
                        const bool inb = !BAND || (j >= rlo[BAND ? r : 0] && j <= rhi[BAND ? r : 0]);
                        if constexpr (AFF) {
                            T mv = hmax3(pM, pX, pY) + sub;
                            uint32_t km = pick3(pM, pX, pY);
                            const T ux = (qM - go_b) - ge_b, vx = qX - ge_b, wx = (qY - go_b) - ge_b;
                            const T xv = hmax3(ux, vx, wx);
                            const uint32_t kx = pick3(ux, vx, wx);
                            const T uy = (cM[r] - go_a) - ge_a, vy = (cX[r] - go_a) - ge_a, wy = cY[r] - ge_a;
                            const T yv = hmax3(uy, vy, wy);
                            const uint32_t ky = pick3(uy, vy, wy);
                            T xo = xv, yo = yv;
                            if constexpr (LOC) mv = hmax(mv, T(0));
                            if constexpr (BAND) {
                                if (!inb) { mv = ninf<T>(); xo = ninf<T>(); yo = ninf<T>(); }
                            }
                            if constexpr (LOC) {
                                km |= 3u * uint32_t(mv <= T(0));
                                const T v = hmax3(mv, xo, yo);
                                if (v > rbest[r]) {
                                    rbest[r] = v; rbj[r] = j;
                                    rbs[r] = (mv >= xo && mv >= yo) ? 0 : (xo >= yo ? 1 : 2);
                                }
                            }
                            pM = cM[r]; pX = cX[r]; pY = cY[r];
                            cM[r] = mv; cX[r] = xo; cY[r] = yo;
                            qM = mv; qX = xo; qY = yo;
                            code = km | (kx << 2) | (ky << 4);
                        } else {
                            const T d0 = pM + sub;
                            const T u = qM - ge_b;
                            const T tt = hmax(d0, u);
                            uint32_t c = uint32_t(d0 < u);
                            const T l = cM[r] - ge_a;
                            T v = hmax(tt, l);
                            c = (tt < l) ? 2u : c;
                            if constexpr (LOC) v = hmax(v, T(0));
                            if constexpr (BAND) { if (!inb) v = ninf<T>(); }
                            if constexpr (LOC) {
                                c |= 3u * uint32_t(v <= T(0));
                                if (v > rbest[r]) { rbest[r] = v; rbj[r] = j; }
                            }
                            pM = cM[r];
                            cM[r] = v;
                            qM = v;
                            code = c;
                        }
                        w[r >> 2] |= code << (8 * (r & 3));
                    }
                    // one coalesced store of this lane's R codes
                    uint8_t* dst = cs + ((int64_t(t >> 3) * G + lane) * 8 + (t & 7)) * R;
                    if (TL && !cs) {
                    } else if constexpr (R % 16 == 0) {
#pragma unroll
                        for (int k = 0; k < R / 16; ++k)
                            reinterpret_cast<uint4*>(dst)[k] = make_uint4(w[4 * k], w[4 * k + 1], w[4 * k + 2], w[4 * k + 3]);
                    } else if constexpr (R % 8 == 0) {
#pragma unroll
                        for (int k = 0; k < R / 8; ++k) reinterpret_cast<uint2*>(dst)[k] = make_uint2(w[2 * k], w[2 * k + 1]);
                    } else if constexpr (R % 4 == 0) {
#pragma unroll
                        for (int k = 0; k < R / 4; ++k) reinterpret_cast<uint32_t*>(dst)[k] = w[k];
                    } else {
#pragma unroll
                        for (int r = 0; r < R; ++r) dst[r] = uint8_t(w[r >> 2] >> (8 * (r & 3)));
                    }
                    dgM = upM; dgX = upX; dgY = upY;
                    if (SG && sg_er) {
                        const int zr = m - i0;
#pragma unroll
                        for (int r = 0; r < R; ++r)
                            if (r == zr) erow.offer(m, j, cM[r], AFF ? cX[r] : ninf<T>(), AFF ? cY[r] : ninf<T>());
                    }
                }
                // hand the bottom row to the next lane (and, from the last lane, to the next stripe)
                if constexpr (G > 1) {
                    const T sM = __shfl_up_sync(gmask, cM[R - 1], 1, G);
                    T sX = sM, sY = sM;
                    if constexpr (AFF) {
                        sX = __shfl_up_sync(gmask, cX[R - 1], 1, G);
                        sY = __shfl_up_sync(gmask, cY[R - 1], 1, G);
                    }
                    if (lane > 0) { upM = sM; upX = sX; upY = sY; }
                }
                if (!GW && lane == G - 1 && active && s + 1 < nstripes) {
                    bnd_out[3 * j] = cM[R - 1];
                    if constexpr (AFF) { bnd_out[3 * j + 1] = cX[R - 1]; bnd_out[3 * j + 2] = cY[R - 1]; }
                }
            }
            if constexpr (TL) {   // the tile's last column, for the tile to its right
                if (!GW && tc + 1 < ntc) {
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const int q = lane * R + r;
                        rcol[3 * q] = cM[r]; rcol[3 * q + 1] = cX[r]; rcol[3 * q + 2] = cY[r];
                    }
                }
            }
            if constexpr (!TL) { pmin = cmin; pmax = cmax; }   // tiles: the row above is whole
            soff += int64_t(S8) * GR;
            // the end cell (m, n): after the stripe each register holds column n (a banded
            // Global stripe holding row m always reaches column n)
            if constexpr (!LOC) {
                if (m >= i0 && m < i0 + R && (!TL || cmax == n)) {
#pragma unroll
                    for (int r = 0; r < R; ++r)
                        if (i0 + r == m) { endM = cM[r]; endX = cX[r]; endY = cY[r]; }
                }
                if (SG && sg_ec) {
                    // column n of this stripe's rows below m, first max in row order: this
                    // lane's, then the group's (the lowest row among equal maxima)
                    EndPick<T> lc; lc.init();
#pragma unroll
                    for (int r = 0; r < R; ++r)
                        if (i0 + r < m) lc.offer(i0 + r, n, cM[r], AFF ? cX[r] : ninf<T>(), AFF ? cY[r] : ninf<T>());
                    if constexpr (G > 1) {
#pragma unroll
                        for (int off = 1; off < G; off <<= 1) {
                            const T ov = __shfl_down_sync(gmask, lc.v, off, G);
                            const int oi = __shfl_down_sync(gmask, lc.i, off, G);
                            const int os = __shfl_down_sync(gmask, lc.st, off, G);
                            const bool oa = __shfl_down_sync(gmask, lc.any ? 1 : 0, off, G) != 0;
                            const bool take = (lane + off < G) && oa && (!lc.any || ov > lc.v);
                            if (take) { lc.v = ov; lc.i = oi; lc.st = os; lc.any = true; }
                        }
                    }
                    if (lc.any && (!ecol.any || lc.v > ecol.v)) { ecol.v = lc.v; ecol.i = lc.i; ecol.j = n; ecol.st = lc.st; ecol.any = true; }
                }
            } else {
                // this lane's first row-major best of the stripe, then the group's
                T lv = T(0); int li = 0, lj = 0, ls = 0;
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (i0 + r <= m && rbest[r] > lv) { lv = rbest[r]; li = i0 + r; lj = rbj[r]; ls = rbs[r]; }
                if constexpr (G > 1) {
#pragma unroll
                    for (int off = 1; off < G; off <<= 1) {
                        const T ov = __shfl_down_sync(gmask, lv, off, G);
                        const int oi = __shfl_down_sync(gmask, li, off, G);
                        const int oj = __shfl_down_sync(gmask, lj, off, G);
                        const int os = __shfl_down_sync(gmask, ls, off, G);
                        const bool take = (lane + off < G) && (ov > lv || (ov == lv && ov > T(0) && oi < li));
                        if (take) { lv = ov; li = oi; lj = oj; ls = os; }
                    }
                }
                if (lv > bestv) { bestv = lv; besti = li; bestj = lj; bests = ls; }
            }
            if constexpr (G > 1) __syncwarp(gmask);
        }
            if constexpr (GW) {   // walk on through the refilled tile
                if (lane == 0) wk.run(tile_code, ts * GR + 1, tc * A.tile_w + 1);
                __syncwarp(gmask);
            }
        }
        if constexpr (GW) {
            if (lane == 0) wk.finish();
            continue;
        }
        if constexpr (!LOC) {
            if constexpr (G > 1) {
                // the lane holding row m broadcasts its end values
                const int src = ((m - 1) % GR) / R;
                endM = __shfl_sync(gmask, endM, src, G);
                endX = __shfl_sync(gmask, endX, src, G);
                endY = __shfl_sync(gmask, endY, src, G);
            }
            if (SG && sg_er) {
                // row m's first max: held by the lane of row m
                const int src = ((m - 1) % GR) / R;
                if constexpr (G > 1) {
                    erow.v = __shfl_sync(gmask, erow.v, src, G);
                    erow.j = __shfl_sync(gmask, erow.j, src, G);
                    erow.st = __shfl_sync(gmask, erow.st, src, G);
                }
            }
            // TL: the tile holding (m, n) writes the pair's result
            const bool tl_end = !TL || (ts == nstripes - 1 && min(n, (tc + 1) * A.tile_w) == n);
            if (lane == 0 && tl_end) {
                T sc; int st, ei = m, ej = n;
                if constexpr (AFF) {
                    sc = rmax3(endM, endX, endY);
                    st = (endM >= endX && endM >= endY) ? 0 : (endX >= endY ? 1 : 2);
                } else { sc = endM; st = 0; }
                if constexpr (SG) {
                    // semi-global: column n's rows 0..m-1 were offered first, then row m
                    if (sg_er) { sc = erow.v; ej = erow.j; st = erow.st; }
                    if (sg_ec && ecol.any && !(sc > ecol.v)) { sc = ecol.v; ei = ecol.i; ej = n; st = ecol.st; }
                }
                A.score[p] = static_cast<double>(sc);
                A.end[4 * p] = ei; A.end[4 * p + 1] = ej; A.end[4 * p + 2] = st;
                A.end[4 * p + 3] = (G << 8) | R;
            }
        } else if (lane == 0) {
            if constexpr (TL) {   // this tile's first row-major best; a later pass picks the pair's
                const int64_t slot = A.tile_off[p] + int64_t(ts) * ntc + tc;
                static_cast<T*>(A.tbest)[slot] = bestv;
                A.tcell[3 * slot] = besti; A.tcell[3 * slot + 1] = bestj; A.tcell[3 * slot + 2] = bests;
            } else {
                A.score[p] = static_cast<double>(bestv);
                A.end[4 * p] = besti; A.end[4 * p + 1] = bestj; A.end[4 * p + 2] = bests;
                A.end[4 * p + 3] = (G << 8) | R;
            }
        }
        if constexpr (!TL) {
            // the traceback, while this pair's codes are still in L2: the group's codes and end
            // cell are visible to its lane 0 after the warp barrier; its other lanes go on with
            // their next pair's fill meanwhile
            if (A.walk_fused) {
                if constexpr (G > 1) __syncwarp(gmask);
                if (lane == 0) walk_pair(A.walk, p);
            }
        }
    }
}

// TL, Local: each pair's best over its tiles -- the first row-major maximum (the largest value,
// then the lowest row, then the lowest column; a tile's own best is its first) -- as the
// pair's score and end cell.  One thread per pair.
struct TileBestArgs {
    const int32_t* pairs; int64_t n_pairs;   // the tiled pairs
    const int64_t* tile_off;                 // per pair: its first tile's slot
    const int32_t* tiles_of;                 // per listed pair: its tiles
    const void* tbest; const int32_t* tcell;
    double* score; int32_t* end; int layout;
};
template <class T>
__global__ void tile_best_kernel(const TileBestArgs A) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= A.n_pairs) return;
    const int p = A.pairs[k];
    const T* tbest = static_cast<const T*>(A.tbest);
    T bv = T(0); int bi = 0, bj = 0, bs = 0;
    for (int t = 0; t < A.tiles_of[k]; ++t) {
        const int64_t q = A.tile_off[p] + t;
        const T v = tbest[q];
        const int vi = A.tcell[3 * q], vj = A.tcell[3 * q + 1];
        if (v > bv || (v == bv && v > T(0) && (vi < bi || (vi == bi && vj < bj)))) {
            bv = v; bi = vi; bj = vj; bs = A.tcell[3 * q + 2];
        }
    }
    A.score[p] = static_cast<double>(bv);
    A.end[4 * p] = bi; A.end[4 * p + 1] = bj; A.end[4 * p + 2] = bs; A.end[4 * p + 3] = A.layout;
}

}  // namespace nwg
