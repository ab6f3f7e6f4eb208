// Hirschberg re-alignment (affine Global and Local, untracked) on the GPU: linear memory for
// long pairs.
//
// The reference's recursion (aligner.hpp:4151-4560): a block (rows i0..i1, columns j0..j1,
// boundary states in_x / out_x) longer than the cutoff is split at row p = i0 + H/2; a
// forward sweep over rows (i0, p] and a reverse sweep over rows [p, i1) keep only their last
// rows; the join picks the first column of the strictly best sum (or an X run straddling the
// cut, one open refunded); the two halves recurse.  Blocks of at most `cutoff` rows are
// solved by a Pointers fill with the block's own borders and walked back.  The score is then
// replayed along the whole path in T, the gradient counted and the guide read off it.
//
// B200 layout: the recursion runs breadth first, one level at a time over every block of
// every pair, so each launch has all of a level's work.
//   * hb_sweep_kernel -- one thread block per half-sweep, a pipeline of NW warps over the
//     block's stripes (32 lanes x R rows each): warp w fills stripe round * NW + w two chunks
//     of 32 columns behind warp w - 1, whose bottom row it reads from a shared-memory ring;
//     the last warp's bottom row reaches the next round's first warp through a row buffer in
//     global memory.  One __syncthreads per chunk; no spin waits.
//   * hb_join_kernel -- one thread block per split block: the first best column.
//   * hb_base_kernel -- one warp per base block: the lane-strip Pointers fill into a
//     row-major code table, then lane 0 walks it.
//   * hb_replay_kernel -- one thread per pair: the base blocks' moves in path order.
// Cells use the reference's expressions ((v - go) - ge, max of three, the prefix-max carry's
// rounded multiply and add), so the path, score, gradient and guide are bit-identical.
//
// Local (viterbi_affine_hirschberg_local, aligner.hpp:4746-4790): hb_scan_kernel runs the
// forward clamped scan of each pair for its end cell (ie, je) -- none positive: the empty
// alignment -- then the reverse global-suffix scan over rows [0, ie), columns [0, je) for the
// start (is, js); the box A[is, ie) x B[js, je) then goes through the same recursion as a
// Global pair, and the replay starts at (is, js).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "nwg_common.cuh"
#include "nwg_hb.h"

namespace nwg {
namespace {

constexpr int kHbC = 32;             // steps per pipeline chunk
constexpr int kHbRing = 4 * kHbC;    // ring slots per warp boundary

struct SweepJob {
    int64_t a_base; int64_t b_base;  // row t >= 1 reads a[a_base + a_step (t - 1)]; column c >= 1 b[b_base + b_step (c - 1)]
    int a_step, b_step;
    int H, W, flag;
    int tiled;                       // swept by hb_tile_kernel (hb_sweep_kernel skips it)
    // tracked: row t >= 0 consumes DP row di = i_base + i_step t (its set; a reverse sweep's
    // gaps in A lie in row di - 1); the pair's m and track offsets (oa[p], oa[p] + p)
    int i_base, i_step, pm, pad2;
    int64_t tk_off, gk_off;
    int64_t out;                     // T offset of the last row: M, X, Y arrays of W + 1
    int64_t wrap;                    // T offset of the wrap row buffer (3 (W + 1))
};

struct BaseJob {
    int64_t a_base, b_base;          // row t >= 1 reads a[a_base + t - 1]; column c >= 1 b[b_base + c - 1]
    int H, W, in_x, out_x;
    int i0, pm;                      // tracked: the DP row of the block's row 0, the pair's m
    int64_t tk_off, gk_off;          // tracked: the pair's track offsets (oa[p], oa[p] + p)
    int64_t codes;                   // byte offset of the (H + 1) x (W + 1) code table
    int64_t bnd;                     // T offset of the stripe boundary row (3 (W + 1))
    int64_t moves;                   // byte offset of the moves (walk order, H + W at most)
};

struct ScanJob {
    int64_t a_base, b_base;          // row t >= 1 reads a[a_base + a_step (t - 1)]; column c >= 1 b[b_base + b_step (c - 1)]
    int a_step, b_step;
    int H, W, local;
    int glocal;                      // 1: the glocal end scan, 2: the glocal start scan (see hb_scan_kernel)
    int i_base, i_step, pm, pad2;    // tracked: as SweepJob's
    int64_t tk_off, gk_off;
};

template <class T> struct Gaps { T go_a, ge_a, go_b, ge_b; };

// Per-row affine parameters of a tracked pair (aligner.hpp:1848-1871, 1907-1910): DP row i's
// substitution set and the gap moves into it (a gap in B, its residue's set) and within it (a
// gap in A, its gap set); a reverse sweep's vertical move into row i is rewritten
// (hb_reverse_rows_): the open of row i + 1 (row m: its own) and its own extend plus the
// difference of the two opens.  tk null: untracked, the one set `u`.
template <class T>
struct AffRows {
    const uint16_t* tk; const uint16_t* gk; const T* gaps; Gaps<T> u;
    __device__ __forceinline__ int tset(int i) const { return int(tk[i - 1]); }
    __device__ __forceinline__ int gset(int i) const { return gk ? int(gk[i]) : (i == 0 ? int(tk[0]) : int(tk[i - 1])); }
    // the parameters of sweep row t consuming DP row di (rev: a reverse sweep), as one Gaps
    __device__ __forceinline__ Gaps<T> row(int di, bool rev, int m) const {
        if (!tk) return u;
        Gaps<T> g;
        const int ga = gset(rev ? di - 1 : di);
        g.go_a = gaps[4 * ga]; g.ge_a = gaps[4 * ga + 1];
        if (di >= 1 && di <= m) {
            const int tb = tset(di);
            const T ob = gaps[4 * tb + 2], eb = gaps[4 * tb + 3];
            if (rev) {
                const T on = di < m ? gaps[4 * tset(di + 1) + 2] : ob;
                g.go_b = on; g.ge_b = eb + (ob - on);
            } else {
                g.go_b = ob; g.ge_b = eb;
            }
        } else {
            g.go_b = u.go_b; g.ge_b = u.ge_b;
        }
        return g;
    }
    __device__ __forceinline__ int key(int di, int ac, int N) const { return tk ? (tset(di) * N + ac) * N : ac * N; }
    __device__ __forceinline__ AffRows at(int64_t tk_off, int64_t gk_off) const {
        AffRows r = *this;
        if (tk) { r.tk = tk + tk_off; r.gk = gk ? gk + gk_off : nullptr; }
        return r;
    }
};

// Per-row linear parameters of a tracked pair: the substitution row, the extend of a gap in B
// into DP row i (its residue's set) and of a gap in A within DP row i (its gap set).
template <class T>
struct LinRows {
    const uint16_t* tk; const uint16_t* gk; const T* gaps; int N;
    __device__ __forceinline__ int tset(int i) const { return int(tk[i - 1]); }
    __device__ __forceinline__ int gset(int i) const { return gk ? int(gk[i]) : (i == 0 ? int(tk[0]) : int(tk[i - 1])); }
    __device__ __forceinline__ T ga(int i) const { return gaps[4 * gset(i) + 1]; }
    __device__ __forceinline__ T gb(int i) const { return gaps[4 * tset(i) + 3]; }
};

template <class T>
__device__ __forceinline__ T chain_y(T lm, T lx, T ly, const Gaps<T>& g) {
    return hmax3((lm - g.go_a) - g.ge_a, (lx - g.go_a) - g.ge_a, ly - g.ge_a);
}
template <class T>
__device__ __forceinline__ T chain_x(T um, T ux, T uy, const Gaps<T>& g) {
    return hmax3((um - g.go_b) - g.ge_b, ux - g.ge_b, (uy - g.go_b) - g.ge_b);
}

// ── endpoint scan ─────────────────────────────────────────────────────────────
// hb_scan_scalar (aligner.hpp:4611-4698) over one block: `local`, the clamped recurrence with
// free starts on row 0 and column 0; else the global borders (row 0 the charged Y chain,
// column 0 the X chain).  The best cell is the first strictly larger max(M, X, Y) in
// row-major order from 0: each lane keeps the lexicographically least (row, column) among its
// largest cells, then the warp reduces with the same order.  Glocal (`glocal` 1 / 2, the
// unclamped recurrence): only the block's last row is a candidate, column 0 included, the
// first column of its maximum; 1 (the end scan) has row 0 a free start (M = 0, no Y) and
// the candidate max(M, X, Y); 2 (the start scan from the end cell, Global's borders) has as
// its last row DP row 0, which a path leaves by a diagonal or a vertical move only, so the
// candidate is max(M, X).  One warp per block: lanes own R
// rows of a 32R-row stripe, skewed by one column; the row above arrives by shuffle, lane 0's
// from the previous stripe's bottom row (a per-warp row in global memory) or row 0.
template <class T, bool PMAX, int R>
__global__ void __launch_bounds__(128) hb_scan_kernel(const uint8_t* __restrict__ a, const uint8_t* __restrict__ b,
                                                      const T* __restrict__ mat, int N, AffRows<T> AR, int K,
                                                      const ScanJob* __restrict__ jobs, int n_jobs, T* rows,
                                                      int64_t row_stride, int32_t* __restrict__ res) {
    extern __shared__ __align__(16) unsigned char hb_smem[];
    T* smat = reinterpret_cast<T*>(hb_smem);
    for (int k = threadIdx.x; k < K * N * N; k += blockDim.x) smat[k] = mat[k];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    const int64_t wg = int64_t(blockIdx.x) * wpb + (threadIdx.x >> 5);
    const int64_t nwarps = int64_t(gridDim.x) * wpb;
    T* bnd = rows + wg * row_stride;
    const T NI = ninf<T>();
    for (int64_t jb = wg; jb < n_jobs; jb += nwarps) {
        const ScanJob J = jobs[jb];
        const int H = J.H, W = J.W;
        const bool loc = J.local != 0;
        const int gl = J.glocal;
        const bool rev = J.a_step < 0;
        const AffRows<T> AJ = AR.at(J.tk_off, J.gk_off);
        const Gaps<T> g0 = AJ.row(J.i_base, rev, J.pm);   // the block's row 0 (its gaps in A)
        T bv = gl ? NI : T(0); int bi = 0, bj = 0;
        if (H > 0 && W > 0) {
            const int nst = (H + 32 * R - 1) / (32 * R);
            for (int s = 0; s < nst; ++s) {
                const int i0 = s * 32 * R + lane * R + 1;   // block row of this lane's first row
                int code[R];
                bool valid[R];
                Gaps<T> rg[R];
                T cM[R], cX[R], cY[R], P[R];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int i = i0 + r;
                    const int di = J.i_base + J.i_step * i;
                    valid[r] = i <= H;
                    code[r] = valid[r] ? AJ.key(di, int(a[J.a_base + int64_t(J.a_step) * (i - 1)]), N) : 0;
                    rg[r] = AJ.row(di, rev, J.pm);
                    cM[r] = NI; cX[r] = NI; cY[r] = NI; P[r] = NI;
                }
                T dgM = NI, dgX = NI, dgY = NI;       // row above, column c - 1
                T upM = NI, upX = NI, upY = NI;       // row above, column c
                T r0M = T(0), r0X = NI, r0Y = NI;     // row 0 at column c - 1 (lane 0, stripe 0)
                // lane 0, s > 0: the previous stripe's bottom row one column ahead
                T nuM = NI, nuX = NI, nuY = NI;
                if (lane == 0 && s > 0) { nuM = bnd[0]; nuX = bnd[1]; nuY = bnd[2]; }
                const int S = W + 32;
                for (int t = 0; t < S; ++t) {
                    const int c = t - lane;
                    if (lane == 0 && c <= W) {
                        if (s == 0) {
                            if (c == 0 || loc || gl == 1) { upM = T(0); upX = NI; upY = NI; }
                            else {
                                upM = NI; upX = NI;
                                upY = hmax((hmax(r0M, r0X) - g0.go_a) - g0.ge_a, r0Y - g0.ge_a);
                            }
                            r0M = upM; r0X = upX; r0Y = upY;
                        } else {
                            upM = nuM; upX = nuX; upY = nuY;
                            if (c < W) { nuM = bnd[4 * (c + 1)]; nuX = bnd[4 * (c + 1) + 1]; nuY = bnd[4 * (c + 1) + 2]; }
                        }
                    }
                    if (c >= 0 && c <= W) {
                        T qM = upM, qX = upX, qY = upY;
                        T pM = dgM, pX = dgX, pY = dgY;
                        const int bc = c >= 1 ? int(b[J.b_base + int64_t(J.b_step) * (c - 1)]) : 0;
#pragma unroll
                        for (int r = 0; r < R; ++r) {
                            const Gaps<T>& q = rg[r];
                            const T rmpc = (PMAX && c >= 1) ? mul_rn(static_cast<T>(c - 1), q.ge_a) : T(0);
                            T m, x, y;
                            x = hmax3((qM - q.go_b) - q.ge_b, qX - q.ge_b, (qY - q.go_b) - q.ge_b);
                            if (c == 0) {
                                m = loc ? T(0) : NI;
                                y = NI;
                                if constexpr (PMAX) P[r] = y - q.ge_a;
                                if (gl && i0 + r == H) {   // glocal: row H's column 0 is a candidate
                                    const T here = gl == 2 ? hmax(m, x) : hmax3(m, x, y);
                                    if (here > bv) { bv = here; bi = H; bj = 0; }
                                }
                            } else {
                                m = hmax3(pM, pX, pY) + smat[code[r] + bc];
                                if (loc) m = hmax(m, T(0));
                                if constexpr (PMAX) {
                                    const T gg = (hmax(cM[r], cX[r]) - q.go_a) - q.ge_a;
                                    P[r] = hmax(add_rn(gg, rmpc), P[r]);
                                    y = P[r] - rmpc;
                                } else {
                                    y = hmax3((cM[r] - q.go_a) - q.ge_a, (cX[r] - q.go_a) - q.ge_a, cY[r] - q.ge_a);
                                }
                                if (gl) {
                                    if (i0 + r == H) {
                                        const T here = gl == 2 ? hmax(m, x) : hmax3(m, x, y);
                                        if (here > bv) { bv = here; bi = H; bj = c; }
                                    }
                                } else if (valid[r]) {
                                    const T here = hmax3(m, x, y);
                                    const int i = i0 + r;
                                    if (here > bv || (here == bv && i < bi)) { bv = here; bi = i; bj = c; }
                                }
                            }
                            pM = cM[r]; pX = cX[r]; pY = cY[r];
                            cM[r] = m; cX[r] = x; cY[r] = y;
                            qM = m; qX = x; qY = y;
                        }
                        dgM = upM; dgX = upX; dgY = upY;
                    }
                    const T sM = __shfl_up_sync(0xffffffffu, cM[R - 1], 1);
                    const T sX = __shfl_up_sync(0xffffffffu, cX[R - 1], 1);
                    const T sY = __shfl_up_sync(0xffffffffu, cY[R - 1], 1);
                    if (lane > 0) { upM = sM; upX = sX; upY = sY; }
                    if (lane == 31 && c >= 0 && c <= W && s + 1 < nst) {
                        bnd[4 * c] = cM[R - 1]; bnd[4 * c + 1] = cX[R - 1]; bnd[4 * c + 2] = cY[R - 1];
                    }
                }
                __syncwarp();
            }
        }
        // the warp's best: largest value, then least row, then least column
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const T ov = __shfl_xor_sync(0xffffffffu, bv, off);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
            const int oj = __shfl_xor_sync(0xffffffffu, bj, off);
            if (ov > bv || (ov == bv && (oi < bi || (oi == bi && oj < bj)))) { bv = ov; bi = oi; bj = oj; }
        }
        if (lane == 0) { res[3 * jb] = (gl || bv > T(0)) ? 1 : 0; res[3 * jb + 1] = bi; res[3 * jb + 2] = bj; }
        __syncwarp();
    }
}

// ── sweep ─────────────────────────────────────────────────────────────────────
template <class T, bool PMAX, int R>
__global__ void __launch_bounds__(512) hb_sweep_kernel(const uint8_t* __restrict__ a, const uint8_t* __restrict__ b,
                                                       const T* __restrict__ mat, int N, AffRows<T> AR, int K,
                                                       const SweepJob* __restrict__ jobs, int n_jobs,
                                                       T* __restrict__ out, T* __restrict__ wrapbuf) {
    constexpr int G = 32, GR = G * R;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smat = reinterpret_cast<T*>(smem_raw);
    T* ring = smat + ((K * N * N + 3) & ~3);               // [NW][3][kHbRing]
    for (int k = threadIdx.x; k < K * N * N; k += blockDim.x) smat[k] = mat[k];
    __syncthreads();
    const int NW = blockDim.x / G;
    const int w = threadIdx.x / G, lane = threadIdx.x % G;
    T* myring = ring + size_t(w) * 3 * kHbRing;
    const T* inring = ring + size_t(w > 0 ? w - 1 : 0) * 3 * kHbRing;
    const T NI = ninf<T>();

    for (int jb = blockIdx.x; jb < n_jobs; jb += gridDim.x) {
        const SweepJob J = jobs[jb];
        if (J.tiled) continue;
        const int H = J.H, W = J.W;
        const int ns = (H + 1 + GR - 1) / GR;              // stripes over rows 0..H
        const int rounds = (ns + NW - 1) / NW;
        const int S = W + G;                               // steps: columns 0..W plus the skew
        int Ct = (S + kHbC - 1) / kHbC;
        Ct = max(Ct, 2 * NW);                              // a wrap row is read a round after it is written
        const int64_t chunks = int64_t(rounds) * Ct;
        const int64_t supers = chunks + 2 * (NW - 1);
        T* oM = out + J.out; T* oX = oM + (W + 1); T* oY = oX + (W + 1);
        T* wM = wrapbuf + J.wrap; T* wX = wM + (W + 1); T* wY = wX + (W + 1);

        int sn = 0, i0 = 0;
        int key[R];
        Gaps<T> rg[R];                                     // each row's gap parameters
        T cM[R], cX[R], cY[R], P[R];
        T dgM = NI, dgX = NI, dgY = NI, upM = NI, upX = NI, upY = NI;
        const AffRows<T> AJ = AR.at(J.tk_off, J.gk_off);
        for (int64_t K = 0; K < supers; ++K) {
            const int64_t v = K - 2 * w;
            if (v >= 0 && v < chunks) {
                const int round = int(v / Ct), chunk = int(v % Ct);
                if (chunk == 0) {                          // a new stripe for this warp
                    sn = round * NW + w;
                    i0 = sn * GR + lane * R;
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const int t = i0 + r;
                        const int di = J.i_base + J.i_step * t;
                        key[r] = (t >= 1 && t <= H) ? AJ.key(di, int(a[J.a_base + int64_t(J.a_step) * (t - 1)]), N) : 0;
                        rg[r] = AJ.row(di, J.a_step < 0, J.pm);
                        cM[r] = NI; cX[r] = NI; cY[r] = NI; P[r] = NI;
                    }
                    dgM = dgX = dgY = NI; upM = upX = upY = NI;
                }
                if (sn < ns) {
                    for (int tt = 0; tt < kHbC; ++tt) {
                        const int tau = chunk * kHbC + tt;
                        const int64_t vstep = v * kHbC + tt;
                        const int c = tau - lane;
                        if (lane == 0 && sn > 0 && c <= W) {
                            if (w > 0) {
                                const int sl = int(vstep % kHbRing);
                                upM = inring[sl]; upX = inring[kHbRing + sl]; upY = inring[2 * kHbRing + sl];
                            } else {
                                upM = wM[c]; upX = wX[c]; upY = wY[c];
                            }
                        }
                        const bool active = c >= 0 && c <= W;
                        if (active) {
                            const int bj = c >= 1 ? int(b[J.b_base + int64_t(J.b_step) * (c - 1)]) : 0;
                            T pM = dgM, pX = dgX, pY = dgY;      // row above, column c - 1
                            T qM = upM, qX = upX, qY = upY;      // row above, column c
#pragma unroll
                            for (int r = 0; r < R; ++r) {
                                const int t = i0 + r;
                                T mv, xv, yv;
                                if (t == 0) {
                                    if (c == 0) { mv = J.flag ? NI : T(0); xv = NI; yv = NI; }
                                    else { mv = NI; xv = NI; yv = chain_y(cM[r], cX[r], cY[r], rg[r]); }
                                } else if (c == 0) {
                                    mv = NI; yv = NI;
                                    xv = (t == 1 && J.flag) ? T(0) - rg[r].ge_b : chain_x(qM, qX, qY, rg[r]);
                                } else {
                                    mv = hmax3(pM, pX, pY) + smat[key[r] + bj];
                                    xv = chain_x(qM, qX, qY, rg[r]);
                                    if constexpr (PMAX) {
                                        const T g = (hmax(cM[r], cX[r]) - rg[r].go_a) - rg[r].ge_a;
                                        const T rm = mul_rn(static_cast<T>(c - 1), rg[r].ge_a);
                                        P[r] = hmax(add_rn(g, rm), P[r]);
                                        yv = P[r] - rm;
                                    } else {
                                        yv = chain_y(cM[r], cX[r], cY[r], rg[r]);
                                    }
                                }
                                pM = cM[r]; pX = cX[r]; pY = cY[r];
                                cM[r] = mv; cX[r] = xv; cY[r] = yv;
                                qM = mv; qX = xv; qY = yv;
                                if (t == H) { oM[c] = mv; oX[c] = xv; oY[c] = yv; }
                            }
                            dgM = upM; dgX = upX; dgY = upY;
                        }
                        const T sM = __shfl_up_sync(0xffffffffu, cM[R - 1], 1);
                        const T sX = __shfl_up_sync(0xffffffffu, cX[R - 1], 1);
                        const T sY = __shfl_up_sync(0xffffffffu, cY[R - 1], 1);
                        if (lane > 0) { upM = sM; upX = sX; upY = sY; }
                        if (lane == G - 1 && active && sn + 1 < ns) {
                            if (w + 1 < NW) {
                                const int sl = int((vstep - (G - 1)) % kHbRing);
                                myring[sl] = cM[R - 1]; myring[kHbRing + sl] = cX[R - 1]; myring[2 * kHbRing + sl] = cY[R - 1];
                            } else {
                                wM[c] = cM[R - 1]; wX[c] = cX[R - 1]; wY[c] = cY[R - 1];
                            }
                        }
                    }
                }
            }
            __syncthreads();
        }
    }
}

// ── tiled half-sweeps ─────────────────────────────────────────────────────────
// The large half-sweeps of a level (a top level of long pairs: one block of warps would hold
// one SM for most of the level) as tiles: stripe s (rows s GR .. s GR + GR - 1 of 0..H) over
// columns c Wt .. c Wt + Wt - 1 of 0..W, one warp per tile, a launch per anti-diagonal s + c
// of every tiled job's tiles.  The cells are hb_sweep_kernel's -- the same expressions, borders
// and flags -- so the last row is the same bits; the row above comes from the stripe above's
// bottom row (one row per stripe), the lanes' state at the column left of the tile (M, X, Y and
// the prefix-max carry of each row) from the tile to the left.
struct HbTileArgs {
    const SweepJob* jobs;
    const int32_t* tiles;            // per item: job, stripe, tile
    int64_t n_items;
    int tile_w;                      // a multiple of 32
    const int64_t* row_off;          // per job: T offset of its rows (ns x 3 (W + 1))
    const int64_t* col_off;          // per job: T offset of its lane states (ns x nt x 32 x 4R)
    int* queue;                      // the work queue shared by the level's tile launches
};
template <class T, bool PMAX, int R>
__global__ void __launch_bounds__(128) hb_tile_kernel(const uint8_t* __restrict__ a, const uint8_t* __restrict__ b,
                                                      const T* __restrict__ mat, int N, AffRows<T> AR, int K,
                                                      HbTileArgs A, T* __restrict__ out, T* __restrict__ rows,
                                                      T* __restrict__ cols) {
    constexpr int G = 32, GR = G * R, LSZ = 4 * R;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smat = reinterpret_cast<T*>(smem_raw);
    for (int k = threadIdx.x; k < K * N * N; k += blockDim.x) smat[k] = mat[k];
    __syncthreads();
    const int lane = threadIdx.x % G, gpb = blockDim.x / G;
    const T NI = ninf<T>();
    auto next_item = [&]() -> int64_t {
        long long v = 0;
        if (lane == 0) v = wq_next(A.queue, int(gridDim.x) * gpb, A.n_items);
        return __shfl_sync(0xffffffffu, v, 0);
    };
    for (int64_t it = next_item(); it < A.n_items; it = next_item()) {
        const int jb = A.tiles[3 * it], s = A.tiles[3 * it + 1], tc = A.tiles[3 * it + 2];
        const SweepJob J = A.jobs[jb];
        const int H = J.H, W = J.W;
        const int ns = (H + 1 + GR - 1) / GR, nt = W / A.tile_w + 1;
        const int c0 = tc * A.tile_w, c1 = min(W, c0 + A.tile_w - 1);
        T* oM = out + J.out; T* oX = oM + (W + 1); T* oY = oX + (W + 1);
        T* const rowp = rows + A.row_off[jb];
        T* const colp = cols + A.col_off[jb];
        const T* const above = rowp + int64_t(s - 1) * 3 * (W + 1);   // s > 0
        T* const below = rowp + int64_t(s) * 3 * (W + 1);
        const int i0 = s * GR + lane * R;
        const AffRows<T> AJ = AR.at(J.tk_off, J.gk_off);
        int key[R];
        Gaps<T> rg[R];
        T cM[R], cX[R], cY[R], P[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int t = i0 + r;
            const int di = J.i_base + J.i_step * t;
            key[r] = (t >= 1 && t <= H) ? AJ.key(di, int(a[J.a_base + int64_t(J.a_step) * (t - 1)]), N) : 0;
            rg[r] = AJ.row(di, J.a_step < 0, J.pm);
            cM[r] = NI; cX[r] = NI; cY[r] = NI; P[r] = NI;
        }
        T dgM = NI, dgX = NI, dgY = NI, upM = NI, upX = NI, upY = NI;
        if (tc > 0) {   // the state the tile to the left left at column c0 - 1
            const T* ls = colp + (int64_t(s) * nt + tc - 1) * G * LSZ;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                cM[r] = ls[lane * LSZ + 4 * r]; cX[r] = ls[lane * LSZ + 4 * r + 1];
                cY[r] = ls[lane * LSZ + 4 * r + 2]; P[r] = ls[lane * LSZ + 4 * r + 3];
            }
            if (lane > 0) {
                const T* q = ls + (lane - 1) * LSZ + 4 * (R - 1);
                dgM = q[0]; dgX = q[1]; dgY = q[2];
            } else if (s > 0) {
                dgM = above[3 * (c0 - 1)]; dgX = above[3 * (c0 - 1) + 1]; dgY = above[3 * (c0 - 1) + 2];
            }
        }
        T nuM = NI, nuX = NI, nuY = NI;   // lane 0: the row above one column ahead
        if (lane == 0 && s > 0) { nuM = above[3 * c0]; nuX = above[3 * c0 + 1]; nuY = above[3 * c0 + 2]; }
        const int S = (c1 - c0 + 1) + G - 1;
        for (int t = 0; t < S; ++t) {
            const int c = c0 + t - lane;
            if (lane == 0 && s > 0 && c <= c1) {
                upM = nuM; upX = nuX; upY = nuY;
                if (c < c1) { nuM = above[3 * (c + 1)]; nuX = above[3 * (c + 1) + 1]; nuY = above[3 * (c + 1) + 2]; }
            }
            const bool active = c >= c0 && c <= c1;
            if (active) {
                const int bj = c >= 1 ? int(b[J.b_base + int64_t(J.b_step) * (c - 1)]) : 0;
                T pM = dgM, pX = dgX, pY = dgY;      // row above, column c - 1
                T qM = upM, qX = upX, qY = upY;      // row above, column c
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int t2 = i0 + r;
                    T mv, xv, yv;
                    if (t2 == 0) {
                        if (c == 0) { mv = J.flag ? NI : T(0); xv = NI; yv = NI; }
                        else { mv = NI; xv = NI; yv = chain_y(cM[r], cX[r], cY[r], rg[r]); }
                    } else if (c == 0) {
                        mv = NI; yv = NI;
                        xv = (t2 == 1 && J.flag) ? T(0) - rg[r].ge_b : chain_x(qM, qX, qY, rg[r]);
                    } else {
                        mv = hmax3(pM, pX, pY) + smat[key[r] + bj];
                        xv = chain_x(qM, qX, qY, rg[r]);
                        if constexpr (PMAX) {
                            const T g = (hmax(cM[r], cX[r]) - rg[r].go_a) - rg[r].ge_a;
                            const T rm = mul_rn(static_cast<T>(c - 1), rg[r].ge_a);
                            P[r] = hmax(add_rn(g, rm), P[r]);
                            yv = P[r] - rm;
                        } else {
                            yv = chain_y(cM[r], cX[r], cY[r], rg[r]);
                        }
                    }
                    pM = cM[r]; pX = cX[r]; pY = cY[r];
                    cM[r] = mv; cX[r] = xv; cY[r] = yv;
                    qM = mv; qX = xv; qY = yv;
                    if (t2 == H) { oM[c] = mv; oX[c] = xv; oY[c] = yv; }
                }
                dgM = upM; dgX = upX; dgY = upY;
            }
            const T sM = __shfl_up_sync(0xffffffffu, cM[R - 1], 1);
            const T sX = __shfl_up_sync(0xffffffffu, cX[R - 1], 1);
            const T sY = __shfl_up_sync(0xffffffffu, cY[R - 1], 1);
            if (lane > 0) { upM = sM; upX = sX; upY = sY; }
            if (lane == G - 1 && active && s + 1 < ns) { below[3 * c] = cM[R - 1]; below[3 * c + 1] = cX[R - 1]; below[3 * c + 2] = cY[R - 1]; }
        }
        if (tc + 1 < nt) {   // this lane's state at the tile's last column
            T* ls = colp + (int64_t(s) * nt + tc) * G * LSZ + lane * LSZ;
#pragma unroll
            for (int r = 0; r < R; ++r) { ls[4 * r] = cM[r]; ls[4 * r + 1] = cX[r]; ls[4 * r + 2] = cY[r]; ls[4 * r + 3] = P[r]; }
        }
        __syncwarp();
    }
}

// ── join ──────────────────────────────────────────────────────────────────────
// Split block k: forward sweep 2k, reverse sweep 2k + 1.  res[2k] = column, res[2k+1] = span.
template <class T>
__global__ void hb_join_kernel(const SweepJob* __restrict__ jobs, int n_blocks, const T* __restrict__ out,
                               AffRows<T> AR, int32_t* __restrict__ res) {
    __shared__ T sv[256];
    __shared__ int sc[256], ss[256];
    const T NI = ninf<T>();
    for (int k = blockIdx.x; k < n_blocks; k += gridDim.x) {
        const SweepJob F = jobs[2 * k], Rv = jobs[2 * k + 1];
        const int W = F.W;
        // the open refunded to an X run straddling the cut: tracked, that of the first row
        // below it, DP row p + 1 (aligner.hpp:4497)
        const int p = F.i_base + F.H;
        const T go_b = AR.tk ? AR.at(F.tk_off, F.gk_off).row(p + 1, false, F.pm).go_b : AR.u.go_b;
        const T* FM = out + F.out; const T* FX = FM + (W + 1); const T* FY = FX + (W + 1);
        const T* rM = out + Rv.out; const T* rX = rM + (W + 1); const T* rY = rX + (W + 1);
        T best = NI; int bc = 0x7fffffff, bs = 0;
        for (int c = threadIdx.x; c <= W; c += blockDim.x) {
            const int d = W - c;
            const T f = hmax3(FM[c], FX[c], FY[c]);
            const T g = hmax3(rM[d], rX[d], rY[d]);
            T val = f + g;
            int sp = 0;
            if (FX[c] > NI && rX[d] > NI) {
                const T joined = (FX[c] + rX[d]) + go_b;
                if (joined > val) { val = joined; sp = 1; }
            }
            if (val > best) { best = val; bc = c; bs = sp; }
        }
        sv[threadIdx.x] = best; sc[threadIdx.x] = bc; ss[threadIdx.x] = bs;
        __syncthreads();
        for (int off = blockDim.x / 2; off > 0; off >>= 1) {
            if (threadIdx.x < off) {
                const T ov = sv[threadIdx.x + off];
                const int oc = sc[threadIdx.x + off];
                if (ov > sv[threadIdx.x] || (ov == sv[threadIdx.x] && oc < sc[threadIdx.x])) {
                    sv[threadIdx.x] = ov; sc[threadIdx.x] = oc; ss[threadIdx.x] = ss[threadIdx.x + off];
                }
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            const bool none = sc[0] == 0x7fffffff;
            res[2 * k] = none ? 0 : sc[0];
            res[2 * k + 1] = none ? 0 : ss[0];
        }
        __syncthreads();
    }
}

// ── base blocks ───────────────────────────────────────────────────────────────
template <class T>
__device__ __forceinline__ uint32_t pick_hb(T vm, T vx, T vy) {
    if (vm >= vx && vm >= vy) return 0u;
    return vx >= vy ? 1u : 2u;
}

template <class T, int R>
__global__ void __launch_bounds__(128) hb_base_kernel(const uint8_t* __restrict__ a, const uint8_t* __restrict__ b,
                                                      const T* __restrict__ mat, int N, AffRows<T> AR, int K,
                                                      const BaseJob* __restrict__ jobs, int n_jobs,
                                                      uint8_t* __restrict__ codes, T* __restrict__ bndbuf,
                                                      uint8_t* __restrict__ moves, int32_t* __restrict__ nmoves) {
    constexpr int G = 32, GR = G * R;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smat = reinterpret_cast<T*>(smem_raw);
    for (int k = threadIdx.x; k < K * N * N; k += blockDim.x) smat[k] = mat[k];
    __syncthreads();
    const int lane = threadIdx.x % G;
    const int wpb = blockDim.x / G;
    const T NI = ninf<T>();
    for (int jb = blockIdx.x * wpb + threadIdx.x / G; jb < n_jobs; jb += gridDim.x * wpb) {
        const BaseJob J = jobs[jb];
        const int H = J.H, W = J.W;
        const int64_t st = int64_t(W) + 1;
        uint8_t* D = codes + J.codes;
        T* bM = bndbuf + J.bnd; T* bX = bM + st; T* bY = bX + st;
        const int ns = (H + 1 + GR - 1) / GR;
        T eM = NI, eX = NI, eY = NI;                       // row H, column W (its owner lane)
        const AffRows<T> AJ = AR.at(J.tk_off, J.gk_off);
        for (int s = 0; s < ns; ++s) {
            const int i0 = s * GR + lane * R;
            int key[R];
            Gaps<T> rg[R];                                 // row t is DP row J.i0 + t
            T cM[R], cX[R], cY[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int t = i0 + r;
                key[r] = (t >= 1 && t <= H) ? AJ.key(J.i0 + t, int(a[J.a_base + t - 1]), N) : 0;
                rg[r] = AJ.row(J.i0 + t, false, J.pm);
                cM[r] = NI; cX[r] = NI; cY[r] = NI;
            }
            T dgM = NI, dgX = NI, dgY = NI, upM = NI, upX = NI, upY = NI;
            for (int tau = 0; tau < W + G; ++tau) {
                const int c = tau - lane;
                if (lane == 0 && s > 0 && c <= W) { upM = bM[c]; upX = bX[c]; upY = bY[c]; }
                const bool active = c >= 0 && c <= W;
                if (active) {
                    const int bj = c >= 1 ? int(b[J.b_base + c - 1]) : 0;
                    T pM = dgM, pX = dgX, pY = dgY;
                    T qM = upM, qX = upX, qY = upY;
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const int t = i0 + r;
                        T mv, xv, yv;
                        uint32_t code;
                        if (t == 0) {
                            if (c == 0) { mv = J.in_x ? NI : T(0); xv = NI; yv = NI; code = 3u | (3u << 2) | (3u << 4); }
                            else {
                                const Gaps<T>& q = rg[r];
                                const T uy = (cM[r] - q.go_a) - q.ge_a, vy = (cX[r] - q.go_a) - q.ge_a, wy = cY[r] - q.ge_a;
                                mv = NI; xv = NI; yv = hmax3(uy, vy, wy);
                                code = 3u | (3u << 2) | (pick_hb(uy, vy, wy) << 4);
                            }
                        } else if (c == 0) {
                            const Gaps<T>& q = rg[r];
                            const T ux = (qM - q.go_b) - q.ge_b, vx = qX - q.ge_b, wx = (qY - q.go_b) - q.ge_b;
                            mv = NI; yv = NI; xv = hmax3(ux, vx, wx);
                            code = 3u | (pick_hb(ux, vx, wx) << 2) | (3u << 4);
                            if (J.in_x && t == 1) { xv = T(0) - q.ge_b; code = 3u | (1u << 2) | (3u << 4); }
                        } else {
                            const Gaps<T>& q = rg[r];
                            const T ux = (qM - q.go_b) - q.ge_b, vx = qX - q.ge_b, wx = (qY - q.go_b) - q.ge_b;
                            const T uy = (cM[r] - q.go_a) - q.ge_a, vy = (cX[r] - q.go_a) - q.ge_a, wy = cY[r] - q.ge_a;
                            mv = hmax3(pM, pX, pY) + smat[key[r] + bj];
                            xv = hmax3(ux, vx, wx);
                            yv = hmax3(uy, vy, wy);
                            code = pick_hb(pM, pX, pY) | (pick_hb(ux, vx, wx) << 2) | (pick_hb(uy, vy, wy) << 4);
                        }
                        if (t <= H) D[int64_t(t) * st + c] = uint8_t(code);
                        pM = cM[r]; pX = cX[r]; pY = cY[r];
                        cM[r] = mv; cX[r] = xv; cY[r] = yv;
                        qM = mv; qX = xv; qY = yv;
                        if (t == H && c == W) { eM = mv; eX = xv; eY = yv; }
                    }
                    dgM = upM; dgX = upX; dgY = upY;
                }
                const T sM = __shfl_up_sync(0xffffffffu, cM[R - 1], 1);
                const T sX = __shfl_up_sync(0xffffffffu, cX[R - 1], 1);
                const T sY = __shfl_up_sync(0xffffffffu, cY[R - 1], 1);
                if (lane > 0) { upM = sM; upX = sX; upY = sY; }
                if (lane == G - 1 && active && s + 1 < ns) { bM[c] = cM[R - 1]; bX[c] = cX[R - 1]; bY[c] = cY[R - 1]; }
            }
            __syncwarp();
        }
        const int owner = (H % GR) / R;
        eM = __shfl_sync(0xffffffffu, eM, owner);
        eX = __shfl_sync(0xffffffffu, eX, owner);
        eY = __shfl_sync(0xffffffffu, eY, owner);
        __syncwarp();
        if (lane == 0) {
            uint8_t* mv = moves + J.moves;
            int r = H, c = W, k = 0;
            int tbl = J.out_x ? 1 : ((eM >= eX && eM >= eY) ? 0 : (eX >= eY ? 1 : 2));
            while ((r > 0 || c > 0) && r >= 0 && c >= 0 && k <= H + W) {
                const uint32_t p = D[int64_t(r) * st + c];
                uint32_t code;
                if (tbl == 0)      { code = p & 3u;        mv[k++] = 0; --r; --c; }
                else if (tbl == 1) { code = (p >> 2) & 3u; mv[k++] = 1; --r; }
                else               { code = p >> 4;        mv[k++] = 2; --c; }
                tbl = code == 1u ? 1 : (code == 2u ? 2 : 0);
            }
            nmoves[jb] = k;
        }
        __syncwarp();
    }
}

// ── replay ────────────────────────────────────────────────────────────────────
template <class T>
__global__ void hb_replay_kernel(const HbRun P, const BaseJob* __restrict__ jobs, const int64_t* __restrict__ first,
                                 const uint8_t* __restrict__ moves, const int32_t* __restrict__ nmoves, int n,
                                 const int32_t* __restrict__ boxes) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int p = P.pairs[k];
    const int64_t ao = P.oa[p], bo = P.ob[p];
    const int m = int(P.oa[p + 1] - ao), nb = int(P.ob[p + 1] - bo);
    const uint8_t* ap = P.a + ao;
    const uint8_t* bp = P.b + bo;
    const T* mat = static_cast<const T*>(P.mat);
    const int N = P.N;
    const T go_a = static_cast<T>(P.go_a), ge_a = static_cast<T>(P.ge_a);
    const T go_b = static_cast<T>(P.go_b), ge_b = static_cast<T>(P.ge_b);
    double* g = P.grad ? P.grad + P.gstride * p : nullptr;
    // tracked: each row's substitution set and gap costs (opens too, affine)
    const bool trk = P.tracks != nullptr;
    const LinRows<T> LR{P.tracks + (trk ? ao : 0), P.gtracks ? P.gtracks + ao + p : nullptr,
                        static_cast<const T*>(P.gaps_t), N};
    const int64_t NN = int64_t(trk ? P.K : 1) * N * N;
    int32_t* gj = P.guide ? P.guide + ao + p : nullptr;
    // Local and glocal: the path runs from its box's start (is, js) to its end (ie, je); Global:
    // (0, 0) to (m, n)
    const int is = boxes ? boxes[4 * k] : 0;
    int js = boxes ? boxes[4 * k + 1] : 0;
    const int ie = boxes ? boxes[4 * k + 2] : m, je = boxes ? boxes[4 * k + 3] : nb;
    int64_t total = 0;
    for (int64_t q = first[k]; q < first[k + 1]; ++q) total += nmoves[q];
    // glocal: the box's leading moves along row 0 are free, not glocal moves -- dropped, the
    // start moving right past them (aligner.hpp:4716-4718)
    int64_t lead = 0;
    if (P.glocal) {
        bool on = true;
        for (int64_t q = first[k]; q < first[k + 1] && on; ++q) {
            const uint8_t* mv = moves + jobs[q].moves;
            for (int e = nmoves[q] - 1; e >= 0; --e) {
                if (mv[e] != 2) { on = false; break; }
                ++lead;
            }
        }
        js += int(lead);
        total -= lead;
    }
    if (gj) { for (int q = 0; q <= m; ++q) gj[q] = -1; gj[0] = 0; gj[is] = js; }
    uint8_t* keep = P.moves ? P.moves + P.moves_off[p] : nullptr;
    T s = T(0);
    int i = is, j = js;
    int prev = 3;
    int64_t idx = 0, skip = lead;
    for (int64_t q = first[k]; q < first[k + 1]; ++q) {
        const uint8_t* mv = moves + jobs[q].moves;
        for (int e = nmoves[q] - 1; e >= 0; --e) {
            const int op = mv[e];
            if (skip > 0) { --skip; continue; }
            if (op == 0) {
                ++i; ++j;
                const int64_t cell = (int64_t(trk ? LR.tset(i) : 0) * N + ap[i - 1]) * N + bp[j - 1];
                s += mat[cell];
                if (g) g[cell] += 1.0;
                if (gj) gj[i] = j;
            } else if (op == 1) {
                ++i;
                const int64_t o = NN + 4 * int64_t(trk ? LR.tset(i) : 0);
                if (!P.linear && prev != 1) { s -= trk ? LR.gaps[o - NN + 2] : go_b; if (g) g[o + 2] -= 1.0; }
                s -= trk ? LR.gb(i) : ge_b;
                if (g) g[o + 3] -= 1.0;
                if (gj) gj[i] = j;
            } else {
                const int64_t o = NN + 4 * int64_t(trk ? LR.gset(i) : 0);
                if (!P.linear && prev != 2) { s -= trk ? LR.gaps[o - NN] : go_a; if (g) g[o + 0] -= 1.0; }
                s -= trk ? LR.ga(i) : ge_a;
                if (g) g[o + 1] -= 1.0;
                ++j;
            }
            if (keep) keep[total - 1 - idx] = uint8_t(op);   // walk order: end to start
            ++idx;
            prev = op;
        }
    }
    P.score[p] = static_cast<double>(s);
    P.end[4 * p] = ie; P.end[4 * p + 1] = je; P.end[4 * p + 2] = prev == 1 ? 1 : (prev == 2 ? 2 : 0);
    P.end[4 * p + 3] = 0;
    if (P.path_info) { P.path_info[3 * p] = int32_t(total); P.path_info[3 * p + 1] = is; P.path_info[3 * p + 2] = js; }
    if (gj) {
        gj[m] = nb;
        const int L = m + 1;
        int lo = 0;
        while (lo < L) {
            if (gj[lo] < 0) { ++lo; continue; }
            int hi = lo + 1;
            while (hi < L && gj[hi] < 0) ++hi;
            if (hi == L) { for (int q = lo + 1; q < L; ++q) gj[q] = gj[lo]; break; }
            for (int q = lo + 1; q < hi; ++q) gj[q] = gj[lo] + (gj[hi] - gj[lo]) * (q - lo) / (hi - lo);
            lo = hi;
        }
    }
}

// ── linear gaps ───────────────────────────────────────────────────────────────
// viterbi_linear_hirschberg (aligner.hpp:5020-5185): one state per cell,
// v = diag + s; u = up - ge_b; l = left - ge_a; v < u -> u; v < l -> l (ties: M, then X, then
// Y).  lhb_kernel, one warp per block (lanes own R rows of a 32R-row stripe, skewed by one
// column; the row above by shuffle, lane 0's from a per-warp row in global memory):
//   MODE 0 -- a half-sweep (lhb_sweep :4844-4913), Global borders, the last row out;
//   MODE 1 -- Local's forward clamped scan: the first strictly larger cell, row-major;
//   MODE 2 -- Local's global-suffix scan (mirrored): row 0 seeds the best in its own order
//             (columns from the last down, strict >), then rows in order, column 0 first.
struct LhbJob {
    int64_t a_base, b_base;          // row t >= 1 reads a[a_base + a_step (t - 1)]; column c >= 1 b[b_base + b_step (c - 1)]
    int a_step, b_step;
    int H, W;
    int64_t out;                     // MODE 0: T offset of the last row (W + 1)
    // tracked: row t >= 1 is DP row i = i_base + i_step t (its substitution set and the
    // extend of a gap into it); its gaps in A lie in DP row i (forward) or i - 1 (reverse:
    // the suffix from row i - 1), row 0's on row i_base (forward) or i_base - 1 (reverse)
    int i_base, i_step;
    int64_t tk_off, gk_off;
    int free0, pad;                  // MODE 0: row 0 a free start (0 at every column; glocal's end sweep)
};


template <class T, int R, int MODE>
__global__ void __launch_bounds__(128) lhb_kernel(const uint8_t* __restrict__ a, const uint8_t* __restrict__ b,
                                                  const T* __restrict__ mat, int N, int K, T ga_u, T gb_u,
                                                  const uint16_t* __restrict__ tracks, const uint16_t* __restrict__ gtracks,
                                                  const T* __restrict__ gaps_t,
                                                  const LhbJob* __restrict__ jobs, int n_jobs, T* rows,
                                                  int64_t row_stride, T* __restrict__ out,
                                                  int32_t* __restrict__ res) {
    extern __shared__ __align__(16) unsigned char hb_smem[];
    T* smat = reinterpret_cast<T*>(hb_smem);
    for (int k = threadIdx.x; k < K * N * N; k += blockDim.x) smat[k] = mat[k];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    const int64_t wg = int64_t(blockIdx.x) * wpb + (threadIdx.x >> 5);
    const int64_t nwarps = int64_t(gridDim.x) * wpb;
    T* bnd = rows + wg * row_stride;
    constexpr bool LOC = MODE == 1;
    for (int64_t jb = wg; jb < n_jobs; jb += nwarps) {
        const LhbJob J = jobs[jb];
        const int H = J.H, W = J.W;
        const bool trk = tracks != nullptr;
        const LinRows<T> LR{tracks + (trk ? J.tk_off : 0), gtracks ? gtracks + J.gk_off : nullptr, gaps_t, N};
        const int gshift = J.i_step < 0 ? 1 : 0;   // reverse: row i's gaps in A on row i - 1
        const T ga0 = trk ? LR.ga(J.i_base - gshift) : ga_u;
        T bv = T(0); int bi = 0, bj = 0;
        if constexpr (MODE == 2) {
            // row 0 (the end cell's row) seeds the best, its columns visited from W down: the
            // chain 0, -ga, -2ga, ... never rises (ga >= 0: Hirschberg needs non-negative
            // penalties), so the first largest is column 0, or column W when ga is 0
            bv = T(0); bi = 0; bj = (ga0 > T(0)) ? 0 : W;
        }
        if (MODE == 0 && H == 0) {   // no rows: row 0 is the last
            if (lane == 0) {
                T v = T(0);
                out[J.out] = v;
                for (int c = 1; c <= W; ++c) { if (!J.free0) v = v - ga0; out[J.out + c] = v; }
            }
        }
        if (H > 0) {
            const int nst = (H + 32 * R - 1) / (32 * R);
            const int lst = (H - 1) / (32 * R), llane = ((H - 1) % (32 * R)) / R, lrow = (H - 1) % R;
            for (int s = 0; s < nst; ++s) {
                const int i0 = s * 32 * R + lane * R + 1;
                int code[R];
                bool valid[R];
                T cur[R], rga[R], rgb[R];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int i = i0 + r;
                    valid[r] = i <= H;
                    const int ac = valid[r] ? int(a[J.a_base + int64_t(J.a_step) * (i - 1)]) : 0;
                    rga[r] = ga_u; rgb[r] = gb_u;
                    code[r] = ac * N;
                    if (trk && valid[r]) {
                        const int di = J.i_base + J.i_step * i;   // the DP row
                        code[r] = (LR.tset(di) * N + ac) * N;
                        rga[r] = LR.ga(di - gshift); rgb[r] = LR.gb(di);
                    }
                    cur[r] = T(0);
                }
                T dg = T(0), up = T(0);       // row above at column c - 1, c
                T r0 = T(0);                   // row 0 at column c - 1 (lane 0, stripe 0)
                T nu = T(0);
                if (lane == 0 && s > 0) nu = bnd[0];
                const int S = W + 32;
                for (int t = 0; t < S; ++t) {
                    const int c = t - lane;
                    if (lane == 0 && c <= W) {
                        if (s == 0) {
                            if (c == 0 || LOC || J.free0) up = T(0);
                            else up = r0 - ga0;
                            r0 = up;
                        } else {
                            up = nu;
                            if (c < W) nu = bnd[c + 1];
                        }
                    }
                    if (c >= 0 && c <= W) {
                        T q = up, pd = dg;
                        const int bc = c >= 1 ? int(b[J.b_base + int64_t(J.b_step) * (c - 1)]) : 0;
#pragma unroll
                        for (int r = 0; r < R; ++r) {
                            T v;
                            if (c == 0) {
                                v = LOC ? T(0) : q - rgb[r];
                            } else {
                                v = pd + smat[code[r] + bc];
                                const T u = q - rgb[r], l = cur[r] - rga[r];
                                if (v < u) v = u;
                                if (v < l) v = l;
                                if constexpr (LOC) v = (v < T(0)) ? T(0) : v;
                            }
                            if constexpr (MODE != 0) {
                                if (valid[r] && (MODE == 2 || c >= 1)) {
                                    const int i = i0 + r;
                                    if (v > bv || (v == bv && (i < bi || (i == bi && c < bj)))) { bv = v; bi = i; bj = c; }
                                }
                            }
                            if constexpr (MODE == 0) {
                                if (s == lst && lane == llane && r == lrow) out[J.out + c] = v;
                            }
                            pd = cur[r];
                            cur[r] = v;
                            q = v;
                        }
                        dg = up;
                    }
                    const T sv = __shfl_up_sync(0xffffffffu, cur[R - 1], 1);
                    if (lane > 0) up = sv;
                    if (lane == 31 && c >= 0 && c <= W && s + 1 < nst) bnd[c] = cur[R - 1];
                }
                __syncwarp();
            }
        }
        if constexpr (MODE != 0) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const T ov = __shfl_xor_sync(0xffffffffu, bv, off);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
                const int oj = __shfl_xor_sync(0xffffffffu, bj, off);
                if (ov > bv || (ov == bv && (oi < bi || (oi == bi && oj < bj)))) { bv = ov; bi = oi; bj = oj; }
            }
            if (lane == 0) { res[3 * jb] = bv > T(0) ? 1 : 0; res[3 * jb + 1] = bi; res[3 * jb + 2] = bj; }
        }
        __syncwarp();
    }
}

// Linear glocal endpoints (viterbi_linear_hirschberg, aligner.hpp:5132-5158), one thread per
// pair.  phase 0: the end column je, the first of the largest values of the free-row-0 sweep's
// row m (F, W + 1 values).  phase 1: the start column js -- the best path from (0, q) to
// (m, je) whose first move is a diagonal or a vertical one, R[d] being the reverse sweep's row
// 1 (from (1, je - d)); q = je first (down only), then q = je - 1 down to 0, strict >.
template <class T>
__global__ void lhb_glocal_pick_kernel(int phase, const LhbJob* __restrict__ jobs, int n_jobs, const T* __restrict__ out,
                                       const uint8_t* __restrict__ a, const uint8_t* __restrict__ b,
                                       const T* __restrict__ mat, int N, T gb1, int32_t* __restrict__ res) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_jobs) return;
    const LhbJob J = jobs[k];
    const T* F = out + J.out;
    if (phase == 0) {
        int je = 0;
        for (int c = 1; c <= J.W; ++c) if (F[c] > F[je]) je = c;
        res[k] = je;
        return;
    }
    // phase 1: J.a_base points at A's last residue (the reverse sweep), J.b_base at B[je - 1];
    // row 1's residue is A[0], column q + 1's is B[q]
    const int je = J.W;
    const int64_t a0 = J.a_base - (J.H);         // A[0]: the reverse sweep ran over A[1 .. m - 1]
    const int64_t b0 = J.b_base - (je - 1);      // B[0]
    const int ar = int(a[a0]) * N;
    T sbest = F[0] - gb1;
    int js = je;
    for (int q = je - 1; q >= 0; --q) {
        T v = F[je - q - 1] + mat[ar + int(b[b0 + q])];
        const T u = F[je - q] - gb1;
        if (v < u) v = u;
        if (v > sbest) { sbest = v; js = q; }
    }
    res[k] = js;
}

// The join of a linear split (lhb_solve :4999-5017): the first column of the strictly largest
// F[c] + R[W - c].  One thread block per split block.
template <class T>
__global__ void lhb_join_kernel(const LhbJob* __restrict__ jobs, int n_blocks, const T* __restrict__ out,
                                int32_t* __restrict__ res) {
    __shared__ T sv[256];
    __shared__ int sc[256];
    for (int q = blockIdx.x; q < n_blocks; q += gridDim.x) {
        const LhbJob& F = jobs[2 * q];
        const LhbJob& Rv = jobs[2 * q + 1];
        const int W = F.W;
        T best = ninf<T>(); int cb = 0;
        for (int c = threadIdx.x; c <= W; c += blockDim.x) {
            const T v = out[F.out + c] + out[Rv.out + (W - c)];
            if (v > best) { best = v; cb = c; }
        }
        sv[threadIdx.x] = best; sc[threadIdx.x] = cb;
        __syncthreads();
        for (int h = blockDim.x / 2; h > 0; h >>= 1) {
            if (threadIdx.x < h) {
                const T ov = sv[threadIdx.x + h]; const int oc = sc[threadIdx.x + h];
                if (ov > sv[threadIdx.x] || (ov == sv[threadIdx.x] && oc < sc[threadIdx.x])) {
                    sv[threadIdx.x] = ov; sc[threadIdx.x] = oc;
                }
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) res[q] = sc[0];
        __syncthreads();
    }
}

// Base block of a linear split (lhb_base :4917-4997): the Pointers fill of the box with the
// Global borders into a row-major code table, walked back from its corner by lane 0.
template <class T, int R>
__global__ void __launch_bounds__(128) lhb_base_kernel(const uint8_t* __restrict__ a, const uint8_t* __restrict__ b,
                                                       const T* __restrict__ mat, int N, int K, T ga_u, T gb_u,
                                                       const uint16_t* __restrict__ tracks,
                                                       const uint16_t* __restrict__ gtracks, const T* __restrict__ gaps_t,
                                                       const BaseJob* __restrict__ jobs, int n_jobs,
                                                       uint8_t* __restrict__ codes, T* __restrict__ bnds,
                                                       uint8_t* __restrict__ moves, int32_t* __restrict__ nmoves) {
    extern __shared__ __align__(16) unsigned char hb_smem[];
    T* smat = reinterpret_cast<T*>(hb_smem);
    for (int k = threadIdx.x; k < K * N * N; k += blockDim.x) smat[k] = mat[k];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (int64_t jb = int64_t(blockIdx.x) * wpb + (threadIdx.x >> 5); jb < n_jobs; jb += int64_t(gridDim.x) * wpb) {
        const BaseJob J = jobs[jb];
        const int H = J.H, W = J.W;
        const int64_t st = int64_t(W) + 1;
        const bool trk = tracks != nullptr;
        const LinRows<T> LR{tracks + (trk ? J.tk_off : 0), gtracks ? gtracks + J.gk_off : nullptr, gaps_t, N};
        const T ga0 = trk ? LR.ga(J.i0) : ga_u;
        uint8_t* D = codes + J.codes;
        T* bnd = bnds + J.bnd;
        if (lane == 0) { D[0] = 3; for (int c = 1; c <= W; ++c) D[c] = 2; }
        if (H > 0) {
            const int nst = (H + 32 * R - 1) / (32 * R);
            for (int s = 0; s < nst; ++s) {
                const int i0 = s * 32 * R + lane * R + 1;
                int code[R];
                T cur[R], rga[R], rgb[R];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int i = i0 + r;
                    const int ac = i <= H ? int(a[J.a_base + i - 1]) : 0;
                    code[r] = ac * N;
                    rga[r] = ga_u; rgb[r] = gb_u;
                    if (trk && i <= H) {
                        const int di = J.i0 + i;
                        code[r] = (LR.tset(di) * N + ac) * N;
                        rga[r] = LR.ga(di); rgb[r] = LR.gb(di);
                    }
                    cur[r] = T(0);
                }
                T dg = T(0), up = T(0), r0 = T(0), nu = T(0);
                if (lane == 0 && s > 0) nu = bnd[0];
                const int S = W + 32;
                for (int t = 0; t < S; ++t) {
                    const int c = t - lane;
                    if (lane == 0 && c <= W) {
                        if (s == 0) { up = c == 0 ? T(0) : r0 - ga0; r0 = up; }
                        else { up = nu; if (c < W) nu = bnd[c + 1]; }
                    }
                    if (c >= 0 && c <= W) {
                        T q = up, pd = dg;
                        const int bc = c >= 1 ? int(b[J.b_base + c - 1]) : 0;
#pragma unroll
                        for (int r = 0; r < R; ++r) {
                            const int i = i0 + r;
                            T v;
                            uint8_t k;
                            if (c == 0) { v = q - rgb[r]; k = 1; }
                            else {
                                v = pd + smat[code[r] + bc];
                                k = 0;
                                const T u = q - rgb[r], l = cur[r] - rga[r];
                                if (v < u) { v = u; k = 1; }
                                if (v < l) { v = l; k = 2; }
                            }
                            if (i <= H) D[int64_t(i) * st + c] = k;
                            pd = cur[r];
                            cur[r] = v;
                            q = v;
                        }
                        dg = up;
                    }
                    const T sv = __shfl_up_sync(0xffffffffu, cur[R - 1], 1);
                    if (lane > 0) up = sv;
                    if (lane == 31 && c >= 0 && c <= W && s + 1 < nst) bnd[c] = cur[R - 1];
                }
                __syncwarp();
            }
        }
        __syncwarp();
        if (lane == 0) {
            uint8_t* mv = moves + J.moves;
            int r = H, c = W, k = 0;
            while (r > 0 || c > 0) {
                const uint8_t op = D[int64_t(r) * st + c];
                mv[k++] = op;
                if (op == 0) { --r; --c; } else if (op == 1) --r; else --c;
            }
            nmoves[jb] = k;
        }
        __syncwarp();
    }
}

// ── host driver ───────────────────────────────────────────────────────────────
struct Blk { int k; int i0, i1, j0, j1; int in_x, out_x; };   // k: index into P.pairs

#define HB_CUDA(call)                                                                      \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// A device buffer for one run, from the stream-ordered pool.
struct Tmp {
    void* p = nullptr; cudaStream_t st;
    explicit Tmp(cudaStream_t s) : st(s) {}
    void* get(size_t n) {
        if (p) { cudaFreeAsync(p, st); p = nullptr; }
        HB_CUDA(cudaMallocAsync(&p, std::max<size_t>(n, 256), st));
        return p;
    }
    ~Tmp() { if (p) cudaFreeAsync(p, st); }
};

template <class T>
int64_t hb_run_t(const HbRun& P, cudaStream_t st, int sms) {
    const int n = int(P.n_pairs);
    if (n == 0) return 0;
    int64_t launches = 0;
    const Gaps<T> gp{static_cast<T>(P.go_a), static_cast<T>(P.ge_a), static_cast<T>(P.go_b), static_cast<T>(P.ge_b)};
    // tracked: every row's parameters from the tracks (K sets of K x N x N and K x 4 in T)
    const bool trk = P.tracks != nullptr;
    const int K = trk ? std::max(P.K, 1) : 1;
    const AffRows<T> AR{trk ? P.tracks : nullptr, trk ? P.gtracks : nullptr, static_cast<const T*>(P.gaps_t), gp};
    // a job's tracked fields: row t consumes DP row i_base + i_step t
    auto track = [&](auto& J, int p, int i_base, int i_step) {
        J.i_base = i_base; J.i_step = i_step; J.pm = int(P.h_oa[p + 1] - P.h_oa[p]);
        J.tk_off = P.h_oa[p]; J.gk_off = P.h_oa[p] + p;
    };
    std::vector<Blk> cur;
    cur.reserve(size_t(n));
    constexpr int R = 4;
    Tmp djobs(st), dout(st), dwrap(st), dres(st), dboxes(st);
    Tmp dtiles(st), droff(st), dcoff(st), dtrows(st), dtcols(st), dq(st);   // tiled half-sweeps
    std::vector<int32_t> boxes;
    if (!P.local && !P.glocal) {
        for (int k = 0; k < n; ++k) {
            const int p = P.h_pairs[k];
            cur.push_back(Blk{k, 0, int(P.h_oa[p + 1] - P.h_oa[p]), 0, int(P.h_ob[p + 1] - P.h_ob[p]), 0, 0});
        }
    } else {
        // Local: the forward clamped scan of every pair, then the reverse global-suffix scan of
        // the pairs with a positive best, give each pair's box.  Glocal
        // (viterbi_affine_hirschberg_glocal, aligner.hpp:4709-4745): the end scan's first best
        // column je of row m, then the start scan from (m, je) for the start column js of row
        // 0; the box A x B[js, je) (a pair without B: column 0).  Either box then runs as a
        // Global pair.
        boxes.assign(size_t(n) * 4, 0);
        const size_t mat_b = size_t((K * P.N * P.N + 3) & ~3) * sizeof(T);
        auto run_scans = [&](const std::vector<ScanJob>& sj, std::vector<int32_t>& out) {
            out.assign(sj.size() * 3, 0);
            if (sj.empty()) return;
            int maxw = 1;
            for (const ScanJob& x : sj) maxw = std::max(maxw, x.W);
            const int wpb = 4;
            const int grid = int(std::min<int64_t>((int64_t(sj.size()) + wpb - 1) / wpb, int64_t(sms) * 4));
            const int64_t stride = 4 * (int64_t(maxw) + 1);
            ScanJob* dj = static_cast<ScanJob*>(djobs.get(sj.size() * sizeof(ScanJob)));
            HB_CUDA(cudaMemcpyAsync(dj, sj.data(), sj.size() * sizeof(ScanJob), cudaMemcpyHostToDevice, st));
            T* rw = static_cast<T*>(dwrap.get(size_t(grid) * wpb * stride * sizeof(T)));
            int32_t* rs = static_cast<int32_t*>(dres.get(out.size() * sizeof(int32_t)));
            auto fn = P.pmax ? hb_scan_kernel<T, true, R> : hb_scan_kernel<T, false, R>;
            HB_CUDA(allow_smem(reinterpret_cast<const void*>(fn), mat_b));
            fn<<<grid, 32 * wpb, mat_b, st>>>(P.a, P.b, static_cast<const T*>(P.mat), P.N, AR, K, dj, int(sj.size()), rw,
                                              stride, rs);
            HB_CUDA(cudaGetLastError());
            launches++;
            HB_CUDA(cudaMemcpyAsync(out.data(), rs, out.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            HB_CUDA(cudaStreamSynchronize(st));
        };
        std::vector<ScanJob> scan_f;
        std::vector<int> fk;                      // the pair of each forward scan
        scan_f.reserve(size_t(n));
        for (int k = 0; k < n; ++k) {
            const int p = P.h_pairs[k];
            ScanJob J{};
            J.a_base = P.h_oa[p]; J.a_step = 1; J.b_base = P.h_ob[p]; J.b_step = 1;
            J.H = int(P.h_oa[p + 1] - P.h_oa[p]); J.W = int(P.h_ob[p + 1] - P.h_ob[p]);
            track(J, p, 0, 1);
            J.local = P.glocal ? 0 : 1; J.glocal = P.glocal ? 1 : 0;
            if (P.glocal && J.W == 0) continue;   // no B: the end is column 0
            scan_f.push_back(J);
            fk.push_back(k);
        }
        std::vector<int32_t> fr, rr;
        run_scans(scan_f, fr);
        std::vector<ScanJob> rev;
        std::vector<int> rk;
        std::vector<int> ends(size_t(n) * 2, 0);  // per pair: ie, je
        for (size_t q = 0; q < fk.size(); ++q) {
            const int k = fk[q];
            const int p = P.h_pairs[k];
            const int ie = fr[3 * q + 1], je = fr[3 * q + 2];
            ends[2 * size_t(k)] = ie; ends[2 * size_t(k) + 1] = je;
            ScanJob J{};
            if (P.glocal) {
                if (je == 0) continue;            // the end on column 0: the box is column 0
                J.H = ie; J.glocal = 2;
            } else {
                if (!fr[3 * q] || ie <= 0 || je <= 0) continue;   // no positive cell: empty
                J.H = ie;
            }
            J.a_base = P.h_oa[p] + ie - 1; J.a_step = -1; J.b_base = P.h_ob[p] + je - 1; J.b_step = -1;
            track(J, p, ie + 1, -1);
            J.W = je; J.local = 0;
            rev.push_back(J);
            rk.push_back(k);
        }
        run_scans(rev, rr);
        std::vector<int> starts(size_t(n) * 2, -1);   // per pair: is, js (-1: no box)
        for (size_t q = 0; q < rk.size(); ++q) {
            const int k = rk[q];
            starts[2 * size_t(k)] = ends[2 * size_t(k)] - rr[3 * q + 1];
            starts[2 * size_t(k) + 1] = ends[2 * size_t(k) + 1] - rr[3 * q + 2];
        }
        for (int k = 0; k < n; ++k) {
            const int p = P.h_pairs[k];
            int is = starts[2 * size_t(k)], js = starts[2 * size_t(k) + 1];
            int ie = ends[2 * size_t(k)], je = ends[2 * size_t(k) + 1];
            if (P.glocal) {
                ie = int(P.h_oa[p + 1] - P.h_oa[p]);   // the end row is m (also without B)
                if (is < 0) { is = 0; js = je; }      // the end on column 0
            } else if (is < 0) {
                continue;                              // Local, nothing positive: the empty alignment
            }
            boxes[4 * size_t(k)] = is; boxes[4 * size_t(k) + 1] = js;
            boxes[4 * size_t(k) + 2] = ie; boxes[4 * size_t(k) + 3] = je;
            cur.push_back(Blk{k, is, ie, js, je, 0, 0});
        }
    }
    const int NWmax = 16;
    const size_t ring_bytes_per_warp = size_t(3) * kHbRing * sizeof(T);
    const size_t mat_bytes = size_t((K * P.N * P.N + 3) & ~3) * sizeof(T);
    while (true) {
        std::vector<int> split;
        for (int q = 0; q < int(cur.size()); ++q)
            if (cur[q].i1 - cur[q].i0 > P.cutoff) split.push_back(q);
        if (split.empty()) break;
        // the level's half-sweeps, largest first for the grid-stride order
        std::vector<SweepJob> jobs(2 * split.size());
        int64_t out_off = 0, wrap_off = 0;
        int max_ns = 1;
        for (size_t s = 0; s < split.size(); ++s) {
            const Blk& B = cur[split[s]];
            const int p = P.h_pairs[B.k];
            const int mid = B.i0 + (B.i1 - B.i0) / 2, W = B.j1 - B.j0;
            SweepJob& F = jobs[2 * s];
            F.a_base = P.h_oa[p] + B.i0; F.a_step = 1; F.b_base = P.h_ob[p] + B.j0; F.b_step = 1;
            F.H = mid - B.i0; F.W = W; F.flag = B.in_x; F.tiled = 0;
            track(F, p, B.i0, 1);
            SweepJob& Rv = jobs[2 * s + 1];
            Rv.a_base = P.h_oa[p] + B.i1 - 1; Rv.a_step = -1; Rv.b_base = P.h_ob[p] + B.j1 - 1; Rv.b_step = -1;
            Rv.H = B.i1 - mid; Rv.W = W; Rv.flag = B.out_x; Rv.tiled = 0;
            track(Rv, p, B.i1 + 1, -1);
            for (SweepJob* x : {&F, &Rv}) {
                x->out = out_off; out_off += 3 * (int64_t(W) + 1);
                x->wrap = wrap_off; wrap_off += 3 * (int64_t(W) + 1);
                max_ns = std::max(max_ns, (x->H + 1 + 32 * R - 1) / (32 * R));
            }
        }
        // half-sweeps of at least kHbTileCells cells run as tiles over the whole device (a
        // block of warps would hold one SM for most of the level), within a memory budget
        // for their rows and lane states; the rest as one block each
        constexpr int64_t kHbTileCells = int64_t(8) << 20;
        constexpr int kHbTileW = 256;
        const int GRt = 32 * R;
        std::vector<int64_t> roff(jobs.size(), 0), coff(jobs.size(), 0);
        std::vector<std::vector<int32_t>> diags;
        int64_t row_elems = 0, col_elems = 0, n_tiles = 0;
        {
            const int64_t budget = P.tile_budget;
            for (size_t q = 0; q < jobs.size(); ++q) {
                SweepJob& x = jobs[q];
                if ((int64_t(x.H) + 1) * (int64_t(x.W) + 1) < kHbTileCells) continue;
                const int nsj = (x.H + 1 + GRt - 1) / GRt, ntj = x.W / kHbTileW + 1;
                const int64_t re = int64_t(nsj) * 3 * (x.W + 1), ce = int64_t(nsj) * ntj * 32 * 4 * R;
                if ((row_elems + re + col_elems + ce) * int64_t(sizeof(T)) > budget) continue;
                x.tiled = 1;
                roff[q] = row_elems; row_elems += re;
                coff[q] = col_elems; col_elems += ce;
                if (int(diags.size()) < nsj + ntj - 1) diags.resize(size_t(nsj + ntj - 1));
                for (int sj = 0; sj < nsj; ++sj)
                    for (int cj = 0; cj < ntj; ++cj) {
                        auto& dv = diags[size_t(sj + cj)];
                        dv.push_back(int32_t(q)); dv.push_back(sj); dv.push_back(cj);
                    }
                n_tiles += int64_t(nsj) * ntj;
            }
        }
        int NW = 1;
        while (NW < NWmax && NW < max_ns) NW *= 2;
        SweepJob* dj = static_cast<SweepJob*>(djobs.get(jobs.size() * sizeof(SweepJob)));
        HB_CUDA(cudaMemcpyAsync(dj, jobs.data(), jobs.size() * sizeof(SweepJob), cudaMemcpyHostToDevice, st));
        T* o = static_cast<T*>(dout.get(size_t(out_off) * sizeof(T)));
        T* wr = static_cast<T*>(dwrap.get(size_t(wrap_off) * sizeof(T)));
        const size_t smem = mat_bytes + NW * ring_bytes_per_warp;
        auto fn = P.pmax ? hb_sweep_kernel<T, true, R> : hb_sweep_kernel<T, false, R>;
        HB_CUDA(allow_smem(reinterpret_cast<const void*>(fn), smem));
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 32 * NW, smem);
        int64_t n_block = 0;
        for (const SweepJob& x : jobs) n_block += x.tiled ? 0 : 1;
        if (n_block) {
            const int grid = int(std::min<int64_t>(n_block, int64_t(sms) * std::max(occ, 1)));
            fn<<<grid, 32 * NW, smem, st>>>(P.a, P.b, static_cast<const T*>(P.mat), P.N, AR, K, dj, int(jobs.size()), o, wr);
            HB_CUDA(cudaGetLastError());
        }
        if (n_tiles) {
            std::vector<int32_t> items;
            items.reserve(size_t(n_tiles) * 3);
            std::vector<int64_t> doff(1, 0);
            for (auto& dv : diags) { items.insert(items.end(), dv.begin(), dv.end()); doff.push_back(int64_t(items.size() / 3)); }
            int32_t* ti = static_cast<int32_t*>(dtiles.get(items.size() * 4));
            HB_CUDA(cudaMemcpyAsync(ti, items.data(), items.size() * 4, cudaMemcpyHostToDevice, st));
            int64_t* ro = static_cast<int64_t*>(droff.get(roff.size() * 8));
            int64_t* co = static_cast<int64_t*>(dcoff.get(coff.size() * 8));
            HB_CUDA(cudaMemcpyAsync(ro, roff.data(), roff.size() * 8, cudaMemcpyHostToDevice, st));
            HB_CUDA(cudaMemcpyAsync(co, coff.data(), coff.size() * 8, cudaMemcpyHostToDevice, st));
            T* tr_rows = static_cast<T*>(dtrows.get(size_t(row_elems) * sizeof(T)));
            T* tr_cols = static_cast<T*>(dtcols.get(size_t(col_elems) * sizeof(T)));
            int* q2 = static_cast<int*>(dq.get(2 * sizeof(int)));
            HB_CUDA(cudaMemsetAsync(q2, 0, 2 * sizeof(int), st));
            auto tfn = P.pmax ? hb_tile_kernel<T, true, R> : hb_tile_kernel<T, false, R>;
            HB_CUDA(allow_smem(reinterpret_cast<const void*>(tfn), mat_bytes));
            int tocc = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&tocc, tfn, 128, mat_bytes);
            const int64_t tmax = int64_t(sms) * std::max(tocc, 1);
            HbTileArgs TA{};
            TA.jobs = dj; TA.tile_w = kHbTileW; TA.row_off = ro; TA.col_off = co; TA.queue = q2;
            for (size_t d = 0; d + 1 < doff.size(); ++d) {
                TA.tiles = ti + 3 * doff[d];
                TA.n_items = doff[d + 1] - doff[d];
                const unsigned tg = unsigned(std::min<int64_t>((TA.n_items + 3) / 4, tmax));
                tfn<<<tg, 128, mat_bytes, st>>>(P.a, P.b, static_cast<const T*>(P.mat), P.N, AR, K, TA, o, tr_rows, tr_cols);
                HB_CUDA(cudaGetLastError());
                launches++;
            }
        }
        int32_t* res = static_cast<int32_t*>(dres.get(split.size() * 2 * sizeof(int32_t)));
        const int jgrid = int(std::min<int64_t>(int64_t(split.size()), int64_t(sms) * 8));
        hb_join_kernel<T><<<jgrid, 256, 0, st>>>(dj, int(split.size()), o, AR, res);
        HB_CUDA(cudaGetLastError());
        launches += (n_block ? 1 : 0) + 1;   // the block sweep, the join
        std::vector<int32_t> h(split.size() * 2);
        HB_CUDA(cudaMemcpyAsync(h.data(), res, h.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        HB_CUDA(cudaStreamSynchronize(st));
        std::vector<Blk> next;
        next.reserve(cur.size() + split.size());
        size_t si = 0;
        for (int q = 0; q < int(cur.size()); ++q) {
            const Blk& B = cur[q];
            if (si < split.size() && split[si] == q) {
                const int mid = B.i0 + (B.i1 - B.i0) / 2;
                const int js = B.j0 + h[2 * si];
                const int span = h[2 * si + 1];
                next.push_back(Blk{B.k, B.i0, mid, B.j0, js, B.in_x, span});
                next.push_back(Blk{B.k, mid, B.i1, js, B.j1, span, B.out_x});
                ++si;
            } else {
                next.push_back(B);
            }
        }
        cur.swap(next);
    }
    // base blocks (path order per pair), then the replay
    std::vector<BaseJob> bj(cur.size());
    std::vector<int64_t> first(size_t(n) + 1, 0);
    int64_t code_off = 0, bnd_off = 0, mv_off = 0;
    for (size_t q = 0; q < cur.size(); ++q) {
        const Blk& B = cur[q];
        const int p = P.h_pairs[B.k];
        BaseJob& J = bj[q];
        J.a_base = P.h_oa[p] + B.i0; J.b_base = P.h_ob[p] + B.j0;
        J.H = B.i1 - B.i0; J.W = B.j1 - B.j0; J.in_x = B.in_x; J.out_x = B.out_x;
        J.i0 = B.i0; J.pm = int(P.h_oa[p + 1] - P.h_oa[p]);
        J.tk_off = P.h_oa[p]; J.gk_off = P.h_oa[p] + p;
        J.codes = code_off; code_off += ((int64_t(J.H) + 1) * (int64_t(J.W) + 1) + 15) & ~int64_t(15);
        J.bnd = bnd_off; bnd_off += 3 * (int64_t(J.W) + 1);
        J.moves = mv_off; mv_off += int64_t(J.H) + J.W + 1;
        first[size_t(B.k) + 1] = int64_t(q) + 1;
    }
    for (int k = 0; k < n; ++k) first[size_t(k) + 1] = std::max(first[size_t(k) + 1], first[size_t(k)]);
    Tmp dbj(st), dcodes(st), dbnd(st), dmv(st), dnm(st), dfirst(st);
    BaseJob* dB = static_cast<BaseJob*>(dbj.get(bj.size() * sizeof(BaseJob)));
    HB_CUDA(cudaMemcpyAsync(dB, bj.data(), bj.size() * sizeof(BaseJob), cudaMemcpyHostToDevice, st));
    uint8_t* cd = static_cast<uint8_t*>(dcodes.get(size_t(code_off)));
    T* bd = static_cast<T*>(dbnd.get(size_t(bnd_off) * sizeof(T)));
    uint8_t* mvd = static_cast<uint8_t*>(dmv.get(size_t(mv_off)));
    int32_t* nm = static_cast<int32_t*>(dnm.get(bj.size() * sizeof(int32_t)));
    int64_t* fd = static_cast<int64_t*>(dfirst.get(first.size() * sizeof(int64_t)));
    HB_CUDA(cudaMemcpyAsync(fd, first.data(), first.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    {
        const int wpb = 4;
        const int grid = int(std::min<int64_t>((int64_t(bj.size()) + wpb - 1) / wpb, int64_t(sms) * 8));
        if (grid > 0) {
            hb_base_kernel<T, R><<<grid, 32 * wpb, mat_bytes, st>>>(P.a, P.b, static_cast<const T*>(P.mat), P.N, AR, K,
                                                                   dB, int(bj.size()), cd, bd, mvd, nm);
            HB_CUDA(cudaGetLastError());
        }
        int32_t* bx = nullptr;
        if (P.local || P.glocal) {
            bx = static_cast<int32_t*>(dboxes.get(boxes.size() * sizeof(int32_t)));
            HB_CUDA(cudaMemcpyAsync(bx, boxes.data(), boxes.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st));
        }
        hb_replay_kernel<T><<<(n + 127) / 128, 128, 0, st>>>(P, dB, fd, mvd, nm, n, bx);
        HB_CUDA(cudaGetLastError());
        launches += 2;
    }
    HB_CUDA(cudaStreamSynchronize(st));
    return launches;
}

// Linear gaps: the same breadth-first recursion with lhb_kernel sweeps, lhb_join_kernel and
// lhb_base_kernel; Local first finds each pair's box with the two scans.
template <class T>
int64_t lhb_run_t(const HbRun& P, cudaStream_t st, int sms) {
    const int n = int(P.n_pairs);
    if (n == 0) return 0;
    int64_t launches = 0;
    constexpr int R = 4;
    const T ga = static_cast<T>(P.ge_a), gb = static_cast<T>(P.ge_b);
    const T* mat = static_cast<const T*>(P.mat);
    const bool trk = P.tracks != nullptr;
    const int K = trk ? std::max(P.K, 1) : 1;
    const T* gaps_t = static_cast<const T*>(P.gaps_t);
    const size_t mat_bytes = size_t((K * P.N * P.N + 3) & ~3) * sizeof(T);
    Tmp djobs(st), dout(st), drows(st), dres(st), dboxes(st);
    auto track_offs = [&](LhbJob& J, int p, int i_base, int i_step) {
        J.i_base = i_base; J.i_step = i_step;
        J.tk_off = P.h_oa[p]; J.gk_off = P.h_oa[p] + p;
    };
    const int wpb = 4;
    // one launch of lhb_kernel<MODE> over jobs (MODE 0: rows out; else results back to the host)
    auto launch = [&](int mode, const std::vector<LhbJob>& jobs, T* o, std::vector<int32_t>* res) {
        if (jobs.empty()) return;
        int maxw = 1;
        for (const LhbJob& x : jobs) maxw = std::max(maxw, x.W);
        const int grid = int(std::min<int64_t>((int64_t(jobs.size()) + wpb - 1) / wpb, int64_t(sms) * 4));
        const int64_t stride = int64_t(maxw) + 1;
        LhbJob* dj = static_cast<LhbJob*>(djobs.get(jobs.size() * sizeof(LhbJob)));
        HB_CUDA(cudaMemcpyAsync(dj, jobs.data(), jobs.size() * sizeof(LhbJob), cudaMemcpyHostToDevice, st));
        T* rw = static_cast<T*>(drows.get(size_t(grid) * wpb * stride * sizeof(T)));
        int32_t* rs = res ? static_cast<int32_t*>(dres.get(jobs.size() * 3 * sizeof(int32_t))) : nullptr;
        auto fn = mode == 0 ? lhb_kernel<T, R, 0> : mode == 1 ? lhb_kernel<T, R, 1> : lhb_kernel<T, R, 2>;
        HB_CUDA(allow_smem(reinterpret_cast<const void*>(fn), mat_bytes));
        fn<<<grid, 32 * wpb, mat_bytes, st>>>(P.a, P.b, mat, P.N, K, ga, gb, trk ? P.tracks : nullptr,
                                              trk ? P.gtracks : nullptr, gaps_t, dj, int(jobs.size()), rw, stride, o, rs);
        HB_CUDA(cudaGetLastError());
        launches++;
        if (res) {
            res->assign(jobs.size() * 3, 0);
            HB_CUDA(cudaMemcpyAsync(res->data(), rs, res->size() * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            HB_CUDA(cudaStreamSynchronize(st));
        }
    };
    std::vector<Blk> cur;
    std::vector<int32_t> boxes;
    if (P.glocal) {
        // glocal (aligner.hpp:5132-5158): the end column je from row m of a sweep with row 0 a
        // free start, the start column js from the reverse sweep over rows 2..m to row 1 and a
        // pick over row 0's columns; the box A x B[js, je) then runs as a Global pair
        boxes.assign(size_t(n) * 4, 0);
        auto pick = [&](int phase, const std::vector<LhbJob>& jobs, std::vector<int32_t>& res) {
            res.assign(jobs.size(), 0);
            if (jobs.empty()) return;
            int64_t out_off = 0;
            for (const LhbJob& x : jobs) out_off += int64_t(x.W) + 1;
            T* o = static_cast<T*>(dout.get(size_t(out_off) * sizeof(T)));
            launch(0, jobs, o, nullptr);
            int32_t* rs = static_cast<int32_t*>(dres.get(jobs.size() * sizeof(int32_t)));
            lhb_glocal_pick_kernel<T><<<unsigned((jobs.size() + 127) / 128), 128, 0, st>>>(
                phase, static_cast<const LhbJob*>(djobs.p), int(jobs.size()), o, P.a, P.b, mat, P.N, gb, rs);
            HB_CUDA(cudaGetLastError());
            launches++;
            HB_CUDA(cudaMemcpyAsync(res.data(), rs, res.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            HB_CUDA(cudaStreamSynchronize(st));
        };
        std::vector<LhbJob> jf;
        int64_t off = 0;
        for (int k = 0; k < n; ++k) {
            const int p = P.h_pairs[k];
            LhbJob J{};
            J.a_base = P.h_oa[p]; J.a_step = 1; J.b_base = P.h_ob[p]; J.b_step = 1;
            J.H = int(P.h_oa[p + 1] - P.h_oa[p]); J.W = int(P.h_ob[p + 1] - P.h_ob[p]);
            J.free0 = 1;
            track_offs(J, p, 0, 1);
            J.out = off; off += int64_t(J.W) + 1;
            jf.push_back(J);
        }
        std::vector<int32_t> je_of, js_of;
        pick(0, jf, je_of);
        std::vector<LhbJob> jr;
        std::vector<int> rk;
        off = 0;
        for (int k = 0; k < n; ++k) {
            const int p = P.h_pairs[k];
            const int m = int(P.h_oa[p + 1] - P.h_oa[p]), je = je_of[size_t(k)];
            if (je == 0 || m < 2) continue;   // js = je: the box is one column (or one row: the pick is the end's)
            LhbJob J{};
            J.a_base = P.h_oa[p] + m - 1; J.a_step = -1; J.b_base = P.h_ob[p] + je - 1; J.b_step = -1;
            J.H = m - 1; J.W = je;
            track_offs(J, p, m + 1, -1);
            J.out = off; off += int64_t(je) + 1;
            jr.push_back(J);
            rk.push_back(k);
        }
        pick(1, jr, js_of);
        std::vector<int> js_k(size_t(n), -1);
        for (size_t q = 0; q < rk.size(); ++q) js_k[size_t(rk[q])] = js_of[q];
        for (int k = 0; k < n; ++k) {
            const int p = P.h_pairs[k];
            const int m = int(P.h_oa[p + 1] - P.h_oa[p]), je = je_of[size_t(k)];
            const int js = js_k[size_t(k)] >= 0 ? js_k[size_t(k)] : je;
            boxes[4 * size_t(k)] = 0; boxes[4 * size_t(k) + 1] = js;
            boxes[4 * size_t(k) + 2] = m; boxes[4 * size_t(k) + 3] = je;
            cur.push_back(Blk{k, 0, m, js, je, 0, 0});
        }
    } else if (!P.local) {
        for (int k = 0; k < n; ++k) {
            const int p = P.h_pairs[k];
            cur.push_back(Blk{k, 0, int(P.h_oa[p + 1] - P.h_oa[p]), 0, int(P.h_ob[p + 1] - P.h_ob[p]), 0, 0});
        }
    } else {
        boxes.assign(size_t(n) * 4, 0);
        std::vector<LhbJob> jf;
        for (int k = 0; k < n; ++k) {
            const int p = P.h_pairs[k];
            LhbJob J{};
            J.a_base = P.h_oa[p]; J.a_step = 1; J.b_base = P.h_ob[p]; J.b_step = 1;
            J.H = int(P.h_oa[p + 1] - P.h_oa[p]); J.W = int(P.h_ob[p + 1] - P.h_ob[p]);
            track_offs(J, p, 0, 1);
            jf.push_back(J);
        }
        std::vector<int32_t> fr, rr;
        launch(1, jf, nullptr, &fr);
        std::vector<LhbJob> jr;
        std::vector<int> rk;
        for (int k = 0; k < n; ++k) {
            if (!fr[3 * k] || fr[3 * k + 1] <= 0 || fr[3 * k + 2] <= 0) continue;   // empty alignment
            const int p = P.h_pairs[k];
            const int ie = fr[3 * k + 1], je = fr[3 * k + 2];
            LhbJob J{};
            J.a_base = P.h_oa[p] + ie - 1; J.a_step = -1; J.b_base = P.h_ob[p] + je - 1; J.b_step = -1;
            J.H = ie; J.W = je;
            track_offs(J, p, ie + 1, -1);
            jr.push_back(J);
            rk.push_back(k);
        }
        launch(2, jr, nullptr, &rr);
        for (size_t q = 0; q < rk.size(); ++q) {
            const int k = rk[q];
            const int ie = fr[3 * k + 1], je = fr[3 * k + 2];
            const int is = ie - rr[3 * q + 1], js = je - rr[3 * q + 2];
            boxes[4 * size_t(k)] = is; boxes[4 * size_t(k) + 1] = js;
            boxes[4 * size_t(k) + 2] = ie; boxes[4 * size_t(k) + 3] = je;
            cur.push_back(Blk{k, is, ie, js, je, 0, 0});
        }
    }
    while (true) {
        std::vector<int> split;
        for (int q = 0; q < int(cur.size()); ++q)
            if (cur[q].i1 - cur[q].i0 > P.cutoff) split.push_back(q);
        if (split.empty()) break;
        std::vector<LhbJob> jobs(2 * split.size());
        int64_t out_off = 0;
        for (size_t s = 0; s < split.size(); ++s) {
            const Blk& B = cur[split[s]];
            const int p = P.h_pairs[B.k];
            const int mid = B.i0 + (B.i1 - B.i0) / 2, W = B.j1 - B.j0;
            LhbJob& F = jobs[2 * s];
            F.a_base = P.h_oa[p] + B.i0; F.a_step = 1; F.b_base = P.h_ob[p] + B.j0; F.b_step = 1;
            F.H = mid - B.i0; F.W = W;
            track_offs(F, p, B.i0, 1);
            LhbJob& Rv = jobs[2 * s + 1];
            Rv.a_base = P.h_oa[p] + B.i1 - 1; Rv.a_step = -1; Rv.b_base = P.h_ob[p] + B.j1 - 1; Rv.b_step = -1;
            Rv.H = B.i1 - mid; Rv.W = W;
            track_offs(Rv, p, B.i1 + 1, -1);
            F.out = out_off; out_off += int64_t(W) + 1;
            Rv.out = out_off; out_off += int64_t(W) + 1;
        }
        T* o = static_cast<T*>(dout.get(size_t(out_off) * sizeof(T)));
        launch(0, jobs, o, nullptr);
        // the join reads the jobs launch() left on the device
        int32_t* res = static_cast<int32_t*>(dres.get(split.size() * sizeof(int32_t)));
        const int jgrid = int(std::min<int64_t>(int64_t(split.size()), int64_t(sms) * 8));
        lhb_join_kernel<T><<<jgrid, 256, 0, st>>>(static_cast<const LhbJob*>(djobs.p), int(split.size()), o, res);
        HB_CUDA(cudaGetLastError());
        launches++;
        std::vector<int32_t> h(split.size());
        HB_CUDA(cudaMemcpyAsync(h.data(), res, h.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        HB_CUDA(cudaStreamSynchronize(st));
        std::vector<Blk> next;
        next.reserve(cur.size() + split.size());
        size_t si = 0;
        for (int q = 0; q < int(cur.size()); ++q) {
            const Blk& B = cur[q];
            if (si < split.size() && split[si] == q) {
                const int mid = B.i0 + (B.i1 - B.i0) / 2;
                const int js = B.j0 + h[si];
                next.push_back(Blk{B.k, B.i0, mid, B.j0, js, 0, 0});
                next.push_back(Blk{B.k, mid, B.i1, js, B.j1, 0, 0});
                ++si;
            } else {
                next.push_back(B);
            }
        }
        cur.swap(next);
    }
    std::vector<BaseJob> bj(cur.size());
    std::vector<int64_t> first(size_t(n) + 1, 0);
    int64_t code_off = 0, bnd_off = 0, mv_off = 0;
    for (size_t q = 0; q < cur.size(); ++q) {
        const Blk& B = cur[q];
        const int p = P.h_pairs[B.k];
        BaseJob& J = bj[q];
        J.a_base = P.h_oa[p] + B.i0; J.b_base = P.h_ob[p] + B.j0;
        J.H = B.i1 - B.i0; J.W = B.j1 - B.j0; J.in_x = 0; J.out_x = 0;
        J.i0 = B.i0; J.pm = int(P.h_oa[p + 1] - P.h_oa[p]); J.tk_off = P.h_oa[p]; J.gk_off = P.h_oa[p] + p;
        J.codes = code_off; code_off += ((int64_t(J.H) + 1) * (int64_t(J.W) + 1) + 15) & ~int64_t(15);
        J.bnd = bnd_off; bnd_off += int64_t(J.W) + 1;
        J.moves = mv_off; mv_off += int64_t(J.H) + J.W + 1;
        first[size_t(B.k) + 1] = int64_t(q) + 1;
    }
    for (int k = 0; k < n; ++k) first[size_t(k) + 1] = std::max(first[size_t(k) + 1], first[size_t(k)]);
    Tmp dbj(st), dcodes(st), dbnd(st), dmv(st), dnm(st), dfirst(st);
    BaseJob* dB = static_cast<BaseJob*>(dbj.get(bj.size() * sizeof(BaseJob)));
    if (!bj.empty()) HB_CUDA(cudaMemcpyAsync(dB, bj.data(), bj.size() * sizeof(BaseJob), cudaMemcpyHostToDevice, st));
    uint8_t* cd = static_cast<uint8_t*>(dcodes.get(size_t(code_off)));
    T* bd = static_cast<T*>(dbnd.get(size_t(bnd_off) * sizeof(T)));
    uint8_t* mvd = static_cast<uint8_t*>(dmv.get(size_t(mv_off)));
    int32_t* nm = static_cast<int32_t*>(dnm.get(bj.size() * sizeof(int32_t)));
    int64_t* fd = static_cast<int64_t*>(dfirst.get(first.size() * sizeof(int64_t)));
    HB_CUDA(cudaMemcpyAsync(fd, first.data(), first.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    const int grid = int(std::min<int64_t>((int64_t(bj.size()) + wpb - 1) / wpb, int64_t(sms) * 8));
    if (grid > 0) {
        HB_CUDA(allow_smem(reinterpret_cast<const void*>(lhb_base_kernel<T, R>), mat_bytes));
        lhb_base_kernel<T, R><<<grid, 32 * wpb, mat_bytes, st>>>(P.a, P.b, mat, P.N, K, ga, gb, trk ? P.tracks : nullptr,
                                                                 trk ? P.gtracks : nullptr, gaps_t, dB, int(bj.size()),
                                                                 cd, bd, mvd, nm);
        HB_CUDA(cudaGetLastError());
        launches++;
    }
    int32_t* bx = nullptr;
    if (P.local || P.glocal) {
        bx = static_cast<int32_t*>(dboxes.get(boxes.size() * sizeof(int32_t)));
        HB_CUDA(cudaMemcpyAsync(bx, boxes.data(), boxes.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    }
    hb_replay_kernel<T><<<(n + 127) / 128, 128, 0, st>>>(P, dB, fd, mvd, nm, n, bx);
    HB_CUDA(cudaGetLastError());
    launches++;
    HB_CUDA(cudaStreamSynchronize(st));
    return launches;
}

}  // namespace

int64_t hb_run(const HbRun& P, int elem_bytes, cudaStream_t st, int sms) {
    if (P.linear) return elem_bytes == 4 ? lhb_run_t<float>(P, st, sms) : lhb_run_t<double>(P, st, sms);
    return elem_bytes == 4 ? hb_run_t<float>(P, st, sms) : hb_run_t<double>(P, st, sms);
}

}  // namespace nwg
