// Traceback: one thread walks a pair's predecessor codes, which the fill stored
// (nwg_hard.cuh), from the end cell back to the start.  walk_pair is called by the hard fill
// itself right after it filled a pair (while the codes are fresh in L2), or by walk_kernel
// (nwg_capi.cu) after the fills of pairs that several warps filled.
#pragma once
#include "nwg_common.cuh"

namespace nwg {

// ── Traceback: one thread per pair ────────────────────────────────────────────
struct WalkArgs {
    const uint8_t* a; const int64_t* oa;
    const uint8_t* b; const int64_t* ob;
    const uint16_t* tracks; const uint16_t* gtracks;
    const int32_t* order; int64_t n_items;
    int N, K;
    int affine, local;
    const uint8_t* codes; const int64_t* code_off;
    const int32_t* end;
    double* grad; int64_t gstride;     // per pair, zeroed here: K*N*N matrix stack + K*4 gaps
    int32_t* guide;                    // per pair m+1 at oa[p] + p, or null
    uint8_t* moves; const int64_t* moves_off;   // keep_paths: walk-order moves, or null
    int32_t* path_info;                // per pair: n_moves, start_i, start_j (or null)
    const int64_t* stripe_base;        // banded: per pair first entry of stripe_tab (else null)
    const int64_t* stripe_tab;
    int ends;                          // semi-global free ends: 1 column 0 a start, 4 row 0 a start
};

// Byte of cell (i, j) in the fill's tiled layout; banded fills record each stripe's code
// offset and first column in `tab` (null: the full DP, stripes of n + G - 1 steps from column 1).
__device__ __forceinline__ uint8_t code_at(const uint8_t* codes, int i, int j, int n, int G, int R,
                                           const int64_t* tab) {
    const int GR = G * R;
    const int s = (i - 1) / GR, w = (i - 1) % GR, g = w / R, r = w % R;
    int64_t base;
    int t;
    if (tab) { base = tab[2 * s]; t = j - int(tab[2 * s + 1]) + g; }
    else {
        const int S8 = (n + G - 1 + 7) & ~7;
        base = int64_t(s) * S8 * GR;
        t = j - 1 + g;
    }
    return codes[base + ((int64_t(t >> 3) * G + g) * 8 + (t & 7)) * R + r];
}

// The walk of one pair as a resumable state: `run` walks from the current cell while the codes
// it needs lie at rows >= ilo and columns >= jlo (the whole table: 1, 1), and stops where the
// next code lies outside (the grid walk then refills the tile holding it) or at the path's start.
struct Walker {
    const WalkArgs* A;
    int p, m, n, N, G, R;
    int64_t NN;
    const uint8_t* ap; const uint8_t* bp;
    const uint16_t* tk; const uint16_t* gk;
    double* g;
    int32_t* gj;
    uint8_t* mv;
    int64_t nm;
    int i, j, tbl;
    bool done;

    __device__ int tset(int ii) const { return tk ? int(tk[ii - 1]) : 0; }
    __device__ int gset(int ii) const {
        if (!tk) return 0;
        if (gk) return int(gk[ii]);
        return ii == 0 ? (m ? int(tk[0]) : 0) : int(tk[ii - 1]);
    }
    __device__ void init(const WalkArgs& W, int pair) {
        A = &W; p = pair;
        const int64_t ao = W.oa[p], bo = W.ob[p];
        m = int(W.oa[p + 1] - ao); n = int(W.ob[p + 1] - bo);
        ap = W.a + ao; bp = W.b + bo;
        tk = W.tracks ? W.tracks + ao : nullptr;
        gk = W.gtracks ? W.gtracks + ao + p : nullptr;
        N = W.N;
        NN = int64_t(W.K) * N * N;
        g = W.grad ? W.grad + W.gstride * p : nullptr;   // zeroed by the host
        const int lay = W.end[4 * p + 3];
        G = lay >> 8; R = lay & 0xff;
        gj = W.guide ? W.guide + ao + p : nullptr;
        if (gj) {
            for (int k = 0; k <= m; ++k) gj[k] = -1;
            gj[0] = 0; gj[m] = n;
        }
        i = W.end[4 * p]; j = W.end[4 * p + 1];
        tbl = W.end[4 * p + 2];
        if (gj) gj[i] = j;
        mv = W.moves ? W.moves + W.moves_off[p] : nullptr;
        nm = 0;
        done = false;
    }
    // one move out of (ii, jj): 0 M, 1 X (gap in B), 2 Y (gap in A)
    __device__ void emit(int s, int ii, int jj, bool open) {
        if (mv) mv[nm] = uint8_t(s);
        ++nm;
        if (s == 0) {
            if (g) g[int64_t(tset(ii) * N + ap[ii - 1]) * N + bp[jj - 1]] += 1.0;
            if (gj) gj[ii - 1] = jj - 1;
        } else if (s == 1) {
            if (g) {
                const int64_t o = NN + 4 * tset(ii);
                g[o + 3] -= 1.0;
                if (open) g[o + 2] -= 1.0;
            }
            if (gj) gj[ii - 1] = jj;
        } else {
            if (g) {
                const int64_t o = NN + 4 * gset(ii);
                g[o + 1] -= 1.0;
                if (open) g[o + 0] -= 1.0;
            }
        }
    }
    template <class CodeFn>
    __device__ void run(CodeFn code, int ilo, int jlo) {
        const bool local = A->local != 0;
        const int ends = A->ends;
        if (A->affine) {
            while (!done) {
                if (i == 0 && j == 0) { done = true; break; }
                uint32_t c;
                if (local) {
                    if (i > 0 && j > 0 && (i < ilo || j < jlo)) return;
                    c = (i == 0 || j == 0) ? 3u : code(i, j);
                    if (tbl == 0 && (c & 3u) == 3u) { done = true; break; }
                } else {
                    // a free start ends the walk on its border; a charged border is one gap run
                    if (i == 0) { if (!(ends & 4)) for (; j > 0; --j) emit(2, 0, j, j == 1); done = true; break; }
                    if (j == 0) { if (!(ends & 1)) for (; i > 0; --i) emit(1, i, 0, i == 1); done = true; break; }
                    if (i < ilo || j < jlo) return;
                    c = code(i, j);
                }
                if (i == 0) tbl = 2;
                else if (j == 0) tbl = 1;
                int prev;
                auto from_code = [](uint32_t cc) { return cc == 1u ? 1 : (cc == 2u ? 2 : 0); };
                if (tbl == 0) { prev = from_code(c & 3u); emit(0, i, j, false); --i; --j; }
                else if (tbl == 1) { prev = from_code((c >> 2) & 3u); emit(1, i, j, prev != 1); --i; }
                else { prev = from_code(c >> 4); emit(2, i, j, prev != 2); --j; }
                tbl = prev;
            }
        } else {
            while (!done) {
                if (i == 0 && j == 0) { done = true; break; }
                int k;
                if (i == 0) k = (local || (ends & 4)) ? 3 : 2;
                else if (j == 0) k = (local || (ends & 1)) ? 3 : 1;
                else {
                    if (i < ilo || j < jlo) return;
                    k = code(i, j);
                }
                if (k == 3) { done = true; break; }
                if (k == 0) { emit(0, i, j, false); --i; --j; }
                else if (k == 1) {
                    if (mv) mv[nm] = 1;
                    ++nm;
                    if (g) g[NN + 4 * tset(i) + 3] -= 1.0;
                    if (gj) gj[i - 1] = j;
                    --i;
                } else {
                    if (mv) mv[nm] = 2;
                    ++nm;
                    if (g) g[NN + 4 * gset(i) + 1] -= 1.0;
                    --j;
                }
            }
        }
    }
    __device__ void finish() {
        if (A->path_info) { A->path_info[3 * p] = int32_t(nm); A->path_info[3 * p + 1] = i; A->path_info[3 * p + 2] = j; }
        if (gj) {
            // interpolate the rows the path does not fix (aligner.hpp:2734-2749)
            const int L = m + 1;
            int lo = 0;
            while (lo < L) {
                if (gj[lo] < 0) { ++lo; continue; }
                int hi = lo + 1;
                while (hi < L && gj[hi] < 0) ++hi;
                if (hi == L) { for (int k = lo + 1; k < L; ++k) gj[k] = gj[lo]; break; }
                for (int k = lo + 1; k < hi; ++k) gj[k] = gj[lo] + (gj[hi] - gj[lo]) * (k - lo) / (hi - lo);
                lo = hi;
            }
        }
    }
};

static __device__ __noinline__ void walk_pair(const WalkArgs& A, const int p) {
    Walker w;
    w.init(A, p);
    const uint8_t* codes = A.codes + A.code_off[p];
    const int64_t* tab = A.stripe_tab ? A.stripe_tab + 2 * A.stripe_base[p] : nullptr;
    const int n = w.n, G = w.G, R = w.R;
    w.run([&](int i, int j) -> uint32_t { return code_at(codes, i, j, n, G, R, tab); }, 1, 1);
    w.finish();
}

}  // namespace nwg
