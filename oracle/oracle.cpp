// CPU oracle for the SeqPairBatch alignment path -- TEST INFRASTRUCTURE ONLY.
//
// A plain restatement of the reference's scalar algorithms (michalsta/nwgrad,
// src/nwgrad/cpp/nwgrad/aligner.hpp), written from reading them, used by the test suite,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker.  The product
// (nwgrad_b200) never links or calls this file.
//
//   Viterbi, affine, Pointers codes ........ aligner.hpp:3955-4071 (viterbi_affine_ptr_impl)
//   Viterbi, linear, Pointers codes ........ aligner.hpp:3756-3860 (viterbi_linear_ptr_impl)
//   Local end cell (first row-major max) ... aligner.hpp:5975-5984 (local_row_best_)
//   semi-global ends (glocal, overlap, free_ends): free row 0 / column 0 starts, end cells
//   column n then row m, first strict max ..... aligner.hpp:3984-4071, 6100-6230 (SgEnd),
//                                            soft borders / ends / gap targets 6362-6430, 6309-6319
//   affine walk + hard gradient ............ aligner.hpp:2985-3056, 3177-3230
//   linear walk + hard gradient ............ aligner.hpp:2852-2900 (walk_linear_impl), 3886-3925
//   guide_j and its gap interpolation ...... aligner.hpp:3155-3160, 2734-2749
//   tracks: per-row sets, column-0 border by runs of equal extends ... aligner.hpp:1919-2007
//   banded rows (guide band) ............... aligner.hpp:2644-2700 (jlo/jhi/border_rows)
//   soft (log space) forward/backward ...... aligner.hpp:6231-6330 (linear), 6362-6524 (affine),
//                                            guide-banded too (jlo/jhi/jlo0/jhi0, 2644-2700)
//   soft temperature: theta/T, log Z * T ... aligner.hpp:6594-6626
//   blocked weighted sum of gradients ...... batch_engine.hpp:1788-1827
//   Hirschberg (exact and prefix-max carry)  aligner.hpp:4151-4560 (hb_fwd, hb_rev, hb_base,
//                                            hb_solve, score replay), 5191-5249 (grad, guide)
//
// Arithmetic follows the reference expression for expression (same association, same
// >= tie-breaks, parameters cast to T once), compiled with -ffp-contract=off, so hard
// results are bit-exact with the reference's float32 / float64 scalar path.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

namespace {

enum { kOpenA = 0, kExtendA = 1, kOpenB = 2, kExtendB = 3 };
enum Tbl : uint8_t { TM = 0, TX = 1, TY = 2 };

struct Model {
    int gm;            // 0 linear, 1 affine
    int am;            // 0 global, 1 local, 2 semi-global (free ends `sg`)
    int N, K;
    const double* mat;   // K*N*N
    const double* gaps;  // K*4
    int sg = 12;         // am 2: free ends, 1 a_begin (column 0 a start), 2 a_end (column n ends),
                         // 4 b_begin (row 0 a start), 8 b_end (row m ends); glocal is 12
    bool semi() const { return am == 2; }
    bool free_row0() const { return am == 1 || (am == 2 && (sg & 4)); }
    bool free_col0() const { return am == 2 && (sg & 1); }
    bool end_col() const { return am == 2 && (sg & 2); }
    bool end_row() const { return am == 2 && (sg & 8); }
};

// The semi-global end (aligner.hpp:6160-6170, SgEnd): candidates offered in order, the
// first of the maxima kept (strict >), its state by M > X > Y.
template <class T>
struct SgEnd {
    T best = T(0); int i = -1, j = 0; Tbl t = TM;
    void offer(int ci, int cj, T vm, T vx, T vy) {
        const T v = (vm < vx ? vx : vm) < vy ? vy : (vm < vx ? vx : vm);
        if (i >= 0 && !(v > best)) return;
        best = v; i = ci; j = cj;
        t = (vm >= vx && vm >= vy) ? TM : (vx >= vy ? TX : TY);
    }
};

template <class T> inline T ninf() { return -std::numeric_limits<T>::infinity(); }
// std::max semantics (first argument kept on ties): (a < b) ? b : a.
template <class T> inline T mx(T a, T b) { return (a < b) ? b : a; }
template <class T> inline T mx3(T a, T b, T c) { return mx(mx(a, b), c); }

// One pair's per-row parameters in T (aligner.hpp:1919-2007).  Untracked: the plain
// casts of set 0, and the closed-form borders.
template <class T>
struct Rows {
    int m = 0;
    bool tracked = false;
    std::vector<uint32_t> rs;                 // substitution row of DP row i (index i-1)
    std::vector<T> goa, gea, gob, geb, bx0;   // size m+1
    std::vector<uint16_t> trk, gtrk;          // sets (tracked)
};

template <class T, bool Linear>
void setup_rows(Rows<T>& R, const Model& M, const uint8_t* a, int m,
                const uint16_t* track, const uint16_t* gtrack, bool tracked) {
    R.m = m; R.tracked = tracked;
    R.rs.resize(m); R.goa.assign(m + 1, T(0)); R.gea.assign(m + 1, T(0));
    R.gob.assign(m + 1, T(0)); R.geb.assign(m + 1, T(0)); R.bx0.assign(m + 1, T(0));
    R.trk.assign(m, 0); R.gtrk.assign(m + 1, 0);
    if (track) for (int i = 0; i < m; ++i) R.trk[i] = track[i];
    if (gtrack) for (int i = 0; i <= m; ++i) R.gtrk[i] = gtrack[i];
    else {
        R.gtrk[0] = m ? R.trk[0] : 0;
        for (int i = 1; i <= m; ++i) R.gtrk[i] = R.trk[i - 1];
    }
    for (int i = 0; i < m; ++i) R.rs[i] = uint32_t(R.trk[i]) * uint32_t(M.N) + a[i];
    auto gap = [&](int k, int f) { return M.gaps[4 * k + f]; };
    for (int i = 0; i <= m; ++i) {
        R.goa[i] = static_cast<T>(gap(R.gtrk[i], kOpenA));
        R.gea[i] = static_cast<T>(gap(R.gtrk[i], kExtendA));
    }
    for (int i = 1; i <= m; ++i) {
        R.gob[i] = static_cast<T>(gap(R.trk[i - 1], kOpenB));
        R.geb[i] = static_cast<T>(gap(R.trk[i - 1], kExtendB));
    }
    if (!tracked) {
        // untracked closed forms (aligner.hpp:6015-6021, 3714-3715)
        const T go_b = static_cast<T>(gap(0, kOpenB)), ge_b = static_cast<T>(gap(0, kExtendB));
        for (int i = 1; i <= m; ++i)
            R.bx0[i] = Linear ? -static_cast<T>(i) * ge_b : -(go_b + static_cast<T>(i) * ge_b);
        return;
    }
    // tracked: runs of bitwise-equal extends (aligner.hpp:1986-2006)
    T csum = T(0);
    int s = 1;
    for (int i = 1; i <= m; ++i) {
        if (i > 1 && std::memcmp(&R.geb[i], &R.geb[i - 1], sizeof(T)) != 0) {
            csum = (s == 1) ? static_cast<T>(i - 1) * R.geb[i - 1]
                            : csum + static_cast<T>(i - s) * R.geb[i - 1];
            s = i;
        }
        const T ge = R.geb[i];
        if (Linear) {
            R.bx0[i] = (s == 1) ? -static_cast<T>(i) * ge : -(csum + static_cast<T>(i - s + 1) * ge);
        } else {
            const T go = R.gob[1];
            R.bx0[i] = (s == 1) ? -(go + static_cast<T>(i) * ge)
                                : -(go + (csum + static_cast<T>(i - s + 1) * ge));
        }
    }
}

// Guide band helpers (aligner.hpp:2644-2700).  band < 0: the full DP.
struct Band {
    int band = -1;
    const int32_t* g = nullptr;
    int m = 0, n = 0;
    bool global = true;
    bool full() const { return band < 0; }
    int jlo(int i) const { return full() ? 1 : std::max(1, g[i] - band); }
    int jhi(int i) const {
        if (full()) return n;
        if (global && i == m) return n;
        int hi = g[i] + band;
        if (i < m) hi = std::max(hi, g[i + 1] - 1 + band);
        return std::min(n, hi);
    }
    int jlo0(int i) const { return full() ? 0 : std::max(0, g[i] - band); }
    int jhi0(int i) const { return jhi(i); }
    int border_rows() const {
        if (full()) return m;
        int bi = 0;
        while (bi < m && g[bi + 1] <= band) ++bi;
        return bi;
    }
    int border_cols() const { return full() ? n : jhi(0); }
};

void fill_guide_gaps(std::vector<int32_t>& gj) {   // aligner.hpp:2734-2749
    const int n = static_cast<int>(gj.size());
    int lo = 0;
    while (lo < n) {
        if (gj[lo] < 0) { ++lo; continue; }
        int hi = lo + 1;
        while (hi < n && gj[hi] < 0) ++hi;
        if (hi == n) { for (int k = lo + 1; k < n; ++k) gj[k] = gj[lo]; break; }
        for (int k = lo + 1; k < hi; ++k) gj[k] = gj[lo] + (gj[hi] - gj[lo]) * (k - lo) / (hi - lo);
        lo = hi;
    }
}

// Output of one hard alignment.
struct HardOut {
    double score = 0;
    double* grad = nullptr;      // K*N*N + 4*K, accumulated (caller zeroes)
    int32_t* guide = nullptr;    // m+1
    uint8_t* moves = nullptr;    // walk order (end -> start): 0 M, 1 X (gap in B), 2 Y (gap in A)
    int64_t nmoves = 0;
    int64_t moves_cap = 0;       // Hirschberg: bytes of moves
    int32_t end_i = 0, end_j = 0, start_i = 0, start_j = 0;
};

template <class T>
struct GradSink {
    const Model& M; const Rows<T>& R; const uint8_t* a; const uint8_t* b; HardOut& o;
    std::vector<int32_t>* gj;
    int64_t cap;
    void move(uint8_t k) { if (o.moves && o.nmoves < cap) o.moves[o.nmoves] = k; ++o.nmoves; }
    double& gap(int i, int f) {
        const int set = (f == kOpenA || f == kExtendA) ? R.gtrk[i] : R.trk[i - 1];
        return o.grad[size_t(M.K) * M.N * M.N + 4 * size_t(set) + f];
    }
    void emit(Tbl s, int i, int j, bool open) {   // aligner.hpp:3203-3226
        move(static_cast<uint8_t>(s));
        if (s == TM) {
            if (o.grad) o.grad[size_t(R.rs[i - 1]) * M.N + b[j - 1]] += 1.0;
            if (gj) (*gj)[i - 1] = j - 1;
        } else if (s == TX) {
            if (o.grad) { gap(i, kExtendB) -= 1.0; if (open) gap(i, kOpenB) -= 1.0; }
            if (gj) (*gj)[i - 1] = j;
        } else {
            if (o.grad) { gap(i, kExtendA) -= 1.0; if (open) gap(i, kOpenA) -= 1.0; }
        }
    }
};

// ── Affine Viterbi with Pointers codes (full DP) ──────────────────────────────
// D[i*(n+1)+j] = M | X << 2 | Y << 4.  Returns the end cell and state.
template <class T>
void affine_fill(const Model& M, const Rows<T>& R, const uint8_t* b, int m, int n,
                 const T* matT, std::vector<uint8_t>& D, T& score, int& bi, int& bj, Tbl& bt) {
    const bool local = M.am == 1;
    const size_t st = size_t(n) + 1;
    D.assign(size_t(m + 1) * st, 0);
    std::vector<T> pM(st), pX(st), pY(st), cM(st), cX(st), cY(st);
    auto pick = [](T vm, T vx, T vy) -> uint8_t {
        const uint8_t kxy = vx >= vy ? 1 : 2;
        return vm >= mx(vx, vy) ? uint8_t(0) : kxy;
    };
    const T go_a0 = R.goa[0], ge_a0 = R.gea[0];
    const bool free0 = M.free_row0(), freec = M.free_col0();
    for (int j = 0; j <= n; ++j) {
        if (free0) { pM[j] = 0; pX[j] = ninf<T>(); pY[j] = ninf<T>(); }
        else {
            pM[j] = (j == 0) ? T(0) : ninf<T>();
            pX[j] = ninf<T>();
            pY[j] = (j == 0) ? ninf<T>() : -(go_a0 + static_cast<T>(j) * ge_a0);
        }
        D[j] = (j <= 1 || free0) ? 3 : (3 | 2 << 4);
    }
    SgEnd<T> sge;
    if (M.end_col() && m > 0) sge.offer(0, n, pM[n], pX[n], pY[n]);
    bi = 0; bj = 0; bt = TM;
    T best_local = T(0);
    for (int i = 1; i <= m; ++i) {
        const T go_a = R.goa[i], ge_a = R.gea[i], go_b = R.gob[i], ge_b = R.geb[i];
        const T* srow = matT + size_t(R.rs[i - 1]) * M.N;
        uint8_t* d = D.data() + size_t(i) * st;
        if (local) { cM[0] = 0; cX[0] = ninf<T>(); }
        else { cM[0] = ninf<T>(); cX[0] = R.bx0[i]; }
        cY[0] = ninf<T>();
        d[0] = (i <= 1) ? 3 : (3 | 1 << 2);
        if (freec) { cM[0] = 0; cX[0] = ninf<T>(); d[0] = 3; }
        T rowmax = T(0);
        for (int j = 1; j <= n; ++j) {
            const T dgM = pM[j - 1], dgX = pX[j - 1], dgY = pY[j - 1];
            T m_val = mx3(dgM, dgX, dgY) + srow[b[j - 1]];
            uint8_t km = pick(dgM, dgX, dgY);
            const T ux = (pM[j] - go_b) - ge_b, vx = pX[j] - ge_b, wx = (pY[j] - go_b) - ge_b;
            const T x_val = mx3(ux, vx, wx);
            const uint8_t kx = pick(ux, vx, wx);
            const T uy = (cM[j - 1] - go_a) - ge_a, vy = (cX[j - 1] - go_a) - ge_a, wy = cY[j - 1] - ge_a;
            const T y_val = mx3(uy, vy, wy);
            const uint8_t ky = pick(uy, vy, wy);
            if (local) {
                m_val = mx(m_val, T(0));
                rowmax = mx(rowmax, mx3(m_val, x_val, y_val));
                km = uint8_t(km | (3u * unsigned(m_val <= T(0))));
            }
            cM[j] = m_val; cX[j] = x_val; cY[j] = y_val;
            d[j] = uint8_t(km | kx << 2 | ky << 4);
        }
        if (local && rowmax > best_local) {
            int j = 1;
            while (!(mx3(cM[j], cX[j], cY[j]) == rowmax)) ++j;
            best_local = rowmax; bi = i; bj = j;
            const T vm = cM[j], vx = cX[j], vy = cY[j];
            bt = (vm >= vx && vm >= vy) ? TM : (vx >= vy ? TX : TY);
        }
        if (M.end_col() && i < m) sge.offer(i, n, cM[n], cX[n], cY[n]);
        std::swap(pM, cM); std::swap(pX, cX); std::swap(pY, cY);
    }
    if (M.semi()) {   // row m (every column with a free B end, else (m, n)), after column n's
        if (M.end_row()) { for (int j = 0; j <= n; ++j) sge.offer(m, j, pM[j], pX[j], pY[j]); }
        else sge.offer(m, n, pM[n], pX[n], pY[n]);
        score = sge.best; bi = sge.i; bj = sge.j; bt = sge.t;
    } else if (!local) {
        const T vm = pM[n], vx = pX[n], vy = pY[n];
        score = mx3(vm, vx, vy);
        bi = m; bj = n;
        bt = (vm >= vx && vm >= vy) ? TM : (vx >= vy ? TX : TY);
    } else {
        score = best_local;
    }
}

template <class T>
void affine_walk(const Model& M, const std::vector<uint8_t>& D, int n, int bi, int bj, Tbl bt,
                 GradSink<T>& sink) {
    const bool local = M.am == 1;
    const size_t st = size_t(n) + 1;
    auto from_code = [](unsigned c) { return c == 1 ? TX : (c == 2 ? TY : TM); };
    int i = bi, j = bj;
    Tbl tbl = bt;
    while (true) {
        if (i == 0 && j == 0) break;
        unsigned c = 0;
        if (local) {
            c = D[size_t(i) * st + j];
            if (tbl == TM && (c & 3) == 3) break;
        } else {
            if (i == 0) {
                if (M.free_row0()) break;   // row 0: a free start
                for (; j > 0; --j) sink.emit(TY, 0, j, j == 1);
                break;
            }
            if (j == 0) {
                if (M.free_col0()) break;   // column 0: a free start
                for (; i > 0; --i) sink.emit(TX, i, 0, i == 1);
                break;
            }
            c = D[size_t(i) * st + j];
        }
        if (i == 0) tbl = TY;
        else if (j == 0) tbl = TX;
        Tbl prev;
        if (tbl == TM) {
            prev = from_code(c & 3);
            sink.emit(TM, i, j, false);
            --i; --j;
        } else if (tbl == TX) {
            prev = from_code((c >> 2) & 3);
            sink.emit(TX, i, j, prev != TX);
            --i;
        } else {
            prev = from_code(c >> 4);
            sink.emit(TY, i, j, prev != TY);
            --j;
        }
        tbl = prev;
    }
    sink.o.start_i = i; sink.o.start_j = j;
}

// ── Linear Viterbi with Pointers codes (full DP) ──────────────────────────────
// Codes: 0 diagonal, 1 up (gap in B), 2 left (gap in A), 3 stop.
template <class T>
void linear_fill(const Model& M, const Rows<T>& R, const uint8_t* b, int m, int n,
                 const T* matT, std::vector<uint8_t>& D, T& score, int& bi, int& bj) {
    const bool local = M.am == 1;
    const size_t st = size_t(n) + 1;
    D.assign(size_t(m + 1) * st, 0);
    std::vector<T> prev(st), cur(st);
    const T ge_a0 = R.gea[0];
    const bool free0 = M.free_row0(), freec = M.free_col0();
    prev[0] = T(0); D[0] = 3;
    for (int j = 1; j <= n; ++j) {
        prev[j] = free0 ? T(0) : -static_cast<T>(j) * ge_a0;
        D[j] = free0 ? 3 : 2;
    }
    const T NI = ninf<T>();
    SgEnd<T> sge;
    if (M.end_col() && m > 0) sge.offer(0, n, prev[n], NI, NI);
    bi = 0; bj = 0;
    T best_local = T(0);
    for (int i = 1; i <= m; ++i) {
        uint8_t* d = D.data() + size_t(i) * st;
        const T* prow = matT + size_t(R.rs[i - 1]) * M.N;
        const T ge_a = R.gea[i], ge_b = R.geb[i];
        cur[0] = (local || freec) ? T(0) : R.bx0[i];
        d[0] = (local || freec) ? 3 : 1;
        for (int j = 1; j <= n; ++j) {
            const T d0 = prev[j - 1] + prow[b[j - 1]];
            const T u = prev[j] - ge_b;
            cur[j] = mx(d0, u);
            d[j] = uint8_t(d0 < u);
        }
        T left = cur[0];
        for (int j = 1; j <= n; ++j) {
            const T t = cur[j], l = left - ge_a;
            T v = mx(t, l);
            const int tl = t < l;
            uint8_t c = uint8_t(d[j] + tl * (2 - d[j]));
            if (local) {
                v = mx(v, T(0));
                c = uint8_t(c | (3u * unsigned(v <= T(0))));
                if (v > best_local) { best_local = v; bi = i; bj = j; }
            }
            cur[j] = v; d[j] = c;
            left = v;
        }
        if (M.end_col() && i < m) sge.offer(i, n, cur[n], NI, NI);
        std::swap(prev, cur);
    }
    if (M.semi()) {
        if (M.end_row()) { for (int j = 0; j <= n; ++j) sge.offer(m, j, prev[j], NI, NI); }
        else sge.offer(m, n, prev[n], NI, NI);
        score = sge.best; bi = sge.i; bj = sge.j;
        return;
    }
    score = local ? best_local : prev[n];
    if (!local) { bi = m; bj = n; }
}

template <class T>
void linear_walk(const std::vector<uint8_t>& D, int n, int bi, int bj, GradSink<T>& sink) {
    const size_t st = size_t(n) + 1;
    int i = bi, j = bj;
    while (true) {
        if (i == 0 && j == 0) break;
        const int k = D[size_t(i) * st + j];
        if (k == 3) break;
        // linear moves: gap fields are extends only (aligner.hpp:3886-3925)
        if (k == 0) { sink.emit(TM, i, j, false); --i; --j; }
        else if (k == 1) {
            sink.move(1);
            if (sink.o.grad) sink.gap(i, kExtendB) -= 1.0;
            if (sink.gj) (*sink.gj)[i - 1] = j;
            --i;
        } else {
            sink.move(2);
            if (sink.o.grad) sink.gap(i, kExtendA) -= 1.0;
            --j;
        }
    }
    sink.o.start_i = i; sink.o.start_j = j;
}

// ── Banded Viterbi (GuideBanded), score tables + re-derived walk ─────────────
// Affine: aligner.hpp:5991-6098 (the band restricts j to [jlo(i), jhi(i)], cells outside
// the band are -inf); walk re-derives predecessors from the tables (walk_affine_impl with
// Ptr = false).  Linear: viterbi_linear_impl + walk_linear_impl (H equality walk).
template <class T>
void banded_affine(const Model& M, const Rows<T>& R, const uint8_t* b, int m, int n,
                   const T* matT, const Band& B, GradSink<T>& sink, T& score) {
    const bool local = M.am == 1;
    const size_t st = size_t(n) + 1;
    std::vector<T> VM(size_t(m + 1) * st, ninf<T>()), VX(VM), VY(VM);
    auto at = [&](std::vector<T>& v, int i, int j) -> T& { return v[size_t(i) * st + j]; };
    if (!local) {
        at(VM, 0, 0) = T(0);
        const int bi = B.border_rows(), bj = B.border_cols();
        for (int i = 1; i <= bi; ++i) at(VX, i, 0) = R.bx0[i];
        if (M.free_row0()) { for (int j = 0; j <= n; ++j) at(VM, 0, j) = T(0); }   // glocal: a free start
        else for (int j = 1; j <= bj; ++j) at(VY, 0, j) = -(R.goa[0] + static_cast<T>(j) * R.gea[0]);
    } else {
        for (int i = 0; i <= m; ++i) at(VM, i, 0) = T(0);
        for (int j = 0; j <= n; ++j) at(VM, 0, j) = T(0);
    }
    int bi = 0, bj = 0; Tbl bt = TM;
    T best_local = T(0);
    for (int i = 1; i <= m; ++i) {
        const T go_a = R.goa[i], ge_a = R.gea[i], go_b = R.gob[i], ge_b = R.geb[i];
        const T* srow = matT + size_t(R.rs[i - 1]) * M.N;
        const int j0 = B.jlo(i), j1 = B.jhi(i);
        if (j0 > j1) continue;
        T lM = at(VM, i, j0 - 1), lX = at(VX, i, j0 - 1), lY = at(VY, i, j0 - 1);
        T rowmax = T(0);
        for (int j = j0; j <= j1; ++j) {
            const T diag = mx3(at(VM, i - 1, j - 1), at(VX, i - 1, j - 1), at(VY, i - 1, j - 1));
            T m_val = diag + srow[b[j - 1]];
            const T x_val = mx(((mx(at(VM, i - 1, j), at(VY, i - 1, j)) - go_b) - ge_b), at(VX, i - 1, j) - ge_b);
            const T y_val = mx(((mx(lM, lX) - go_a) - ge_a), lY - ge_a);
            if (local) { m_val = mx(m_val, T(0)); rowmax = mx(rowmax, mx3(m_val, x_val, y_val)); }
            at(VM, i, j) = m_val; at(VX, i, j) = x_val; at(VY, i, j) = y_val;
            lM = m_val; lX = x_val; lY = y_val;
        }
        if (local && rowmax > best_local) {
            int j = j0;
            while (!(mx3(at(VM, i, j), at(VX, i, j), at(VY, i, j)) == rowmax)) ++j;
            best_local = rowmax; bi = i; bj = j;
            const T vm = at(VM, i, j), vx = at(VX, i, j), vy = at(VY, i, j);
            bt = (vm >= vx && vm >= vy) ? TM : (vx >= vy ? TX : TY);
        }
    }
    if (M.semi()) {   // glocal: row m's first best column over its band (glocal_end_affine_)
        SgEnd<T> e;
        for (int j = B.jlo0(m); j <= B.jhi0(m); ++j) e.offer(m, j, at(VM, m, j), at(VX, m, j), at(VY, m, j));
        score = e.best; bi = e.i; bj = e.j; bt = e.t;
    } else if (!local) {
        const T vm = at(VM, m, n), vx = at(VX, m, n), vy = at(VY, m, n);
        score = mx3(vm, vx, vy);
        bi = m; bj = n;
        bt = (vm >= vx && vm >= vy) ? TM : (vx >= vy ? TX : TY);
    } else score = best_local;
    sink.o.end_i = bi; sink.o.end_j = bj;
    if (sink.gj) { auto& gj = *sink.gj; gj.assign(m + 1, -1); gj[0] = 0; gj[m] = n; gj[bi] = bj; }
    // walk, re-deriving predecessors (aligner.hpp:2985-3056, Ptr = false)
    auto argmax = [](T vm, T vx, T vy) { if (vm >= vx && vm >= vy) return TM; return vx >= vy ? TX : TY; };
    int i = bi, j = bj;
    Tbl tbl = bt;
    while (true) {
        if (i == 0 && j == 0) break;
        if (local) {
            if (tbl == TM && at(VM, i, j) <= T(0)) break;
        } else {
            if (i == 0 && M.free_row0()) break;
            if (i == 0) { for (; j > 0; --j) sink.emit(TY, 0, j, j == 1); break; }
            if (j == 0) { for (; i > 0; --i) sink.emit(TX, i, 0, i == 1); break; }
        }
        if (i == 0) tbl = TY;
        else if (j == 0) tbl = TX;
        Tbl prev;
        if (tbl == TM) {
            prev = argmax(at(VM, i - 1, j - 1), at(VX, i - 1, j - 1), at(VY, i - 1, j - 1));
            sink.emit(TM, i, j, false); --i; --j;
        } else if (tbl == TX) {
            const T go_b = R.gob[i], ge_b = R.geb[i];
            prev = argmax((at(VM, i - 1, j) - go_b) - ge_b, at(VX, i - 1, j) - ge_b, (at(VY, i - 1, j) - go_b) - ge_b);
            sink.emit(TX, i, j, prev != TX); --i;
        } else {
            const T go_a = R.goa[i], ge_a = R.gea[i];
            prev = argmax((at(VM, i, j - 1) - go_a) - ge_a, (at(VX, i, j - 1) - go_a) - ge_a, at(VY, i, j - 1) - ge_a);
            sink.emit(TY, i, j, prev != TY); --j;
        }
        tbl = prev;
    }
    sink.o.start_i = i; sink.o.start_j = j;
}

template <class T>
void banded_linear(const Model& M, const Rows<T>& R, const uint8_t* b, int m, int n,
                   const T* matT, const Band& B, GradSink<T>& sink, T& score) {
    const bool local = M.am == 1;
    const size_t st = size_t(n) + 1;
    std::vector<T> H(size_t(m + 1) * st, ninf<T>());
    auto at = [&](int i, int j) -> T& { return H[size_t(i) * st + j]; };
    // viterbi_linear_impl's banded_fill: -inf over the band's row spans (here everywhere).
    if (!local) {
        at(0, 0) = T(0);
        const int bi = B.border_rows(), bj = B.border_cols();
        for (int i = 1; i <= bi; ++i) at(i, 0) = R.bx0[i];
        if (M.free_row0()) { for (int j = 0; j <= n; ++j) at(0, j) = T(0); }   // glocal: a free start
        else for (int j = 1; j <= bj; ++j) at(0, j) = -static_cast<T>(j) * R.gea[0];
    } else {
        for (int i = 0; i <= m; ++i) at(i, 0) = T(0);
        for (int j = 0; j <= n; ++j) at(0, j) = T(0);
    }
    int bi = 0, bj = 0;
    T best_local = T(0);
    for (int i = 1; i <= m; ++i) {
        const T ge_b = R.geb[i], ge_a = R.gea[i];
        const T* srow = matT + size_t(R.rs[i - 1]) * M.N;
        const int j0 = B.jlo(i), j1 = B.jhi(i);
        T rowmax = T(0);
        for (int j = j0; j <= j1; ++j) {
            T v = mx3(at(i - 1, j - 1) + srow[b[j - 1]], at(i - 1, j) - ge_b, at(i, j - 1) - ge_a);
            if (local) { v = mx(v, T(0)); rowmax = mx(rowmax, v); }
            at(i, j) = v;
        }
        if (local && rowmax > best_local) {
            int j = j0;
            while (!(at(i, j) == rowmax)) ++j;
            best_local = rowmax; bi = i; bj = j;
        }
    }
    if (M.semi()) {   // glocal: row m's first best column over its band (glocal_end_linear_)
        SgEnd<T> e;
        for (int j = B.jlo0(m); j <= B.jhi0(m); ++j) e.offer(m, j, at(m, j), ninf<T>(), ninf<T>());
        score = e.best; bi = e.i; bj = e.j;
    } else {
        score = local ? best_local : at(m, n);
        if (!local) { bi = m; bj = n; }
    }
    sink.o.end_i = bi; sink.o.end_j = bj;
    if (sink.gj) {
        auto& gj = *sink.gj; gj.assign(m + 1, -1); gj[0] = 0; gj[m] = n;
        gj[M.am == 0 ? m : bi] = M.am == 0 ? n : bj;
    }
    int i = bi, j = bj;
    while (true) {
        if (i == 0 && j == 0) break;
        if (local && at(i, j) <= T(0)) break;
        if (i == 0 && M.free_row0()) break;
        int k;
        if (i > 0 && j > 0 && at(i, j) == at(i - 1, j - 1) + matT[size_t(R.rs[i - 1]) * M.N + b[j - 1]]) k = 0;
        else if (i > 0 && (j == 0 || at(i, j) == at(i - 1, j) - R.geb[i])) k = 1;
        else k = 2;
        if (k == 0) { sink.emit(TM, i, j, false); --i; --j; }
        else if (k == 1) {
            sink.move(1);
            if (sink.o.grad) sink.gap(i, kExtendB) -= 1.0;
            if (sink.gj) (*sink.gj)[i - 1] = j;
            --i;
        } else {
            sink.move(2);
            if (sink.o.grad) sink.gap(i, kExtendA) -= 1.0;
            --j;
        }
    }
    sink.o.start_i = i; sink.o.start_j = j;
}

template <class T>
int hard_one(const Model& M, const uint8_t* a, int m, const uint8_t* b, int n,
             const uint16_t* track, const uint16_t* gtrack, bool tracked,
             const int32_t* guide_in, int band, HardOut& o, int64_t moves_cap) {
    const bool linear = M.gm == 0;
    Rows<T> R;
    if (linear) setup_rows<T, true>(R, M, a, m, track, gtrack, tracked);
    else        setup_rows<T, false>(R, M, a, m, track, gtrack, tracked);
    std::vector<T> matT(size_t(M.K) * M.N * M.N);
    for (size_t k = 0; k < matT.size(); ++k) matT[k] = static_cast<T>(M.mat[k]);
    std::vector<int32_t> gj;
    GradSink<T> sink{M, R, a, b, o, o.guide ? &gj : nullptr, moves_cap};
    T score = T(0);
    if (band >= 0) {
        Band B; B.band = band; B.g = guide_in; B.m = m; B.n = n; B.global = M.am == 0;
        if (linear) banded_linear<T>(M, R, b, m, n, matT.data(), B, sink, score);
        else        banded_affine<T>(M, R, b, m, n, matT.data(), B, sink, score);
    } else {
        std::vector<uint8_t> D;
        int bi, bj;
        if (linear) {
            linear_fill<T>(M, R, b, m, n, matT.data(), D, score, bi, bj);
            o.end_i = bi; o.end_j = bj;
            if (o.guide) {
                gj.assign(m + 1, -1); gj[0] = 0; gj[m] = n;
                if (M.am == 0) gj[m] = n; else gj[bi] = bj;
            }
            linear_walk<T>(D, n, bi, bj, sink);
        } else {
            Tbl bt;
            affine_fill<T>(M, R, b, m, n, matT.data(), D, score, bi, bj, bt);
            o.end_i = bi; o.end_j = bj;
            if (o.guide) { gj.assign(m + 1, -1); gj[0] = 0; gj[m] = n; gj[bi] = bj; }
            affine_walk<T>(M, D, n, bi, bj, bt, sink);
        }
    }
    o.score = static_cast<double>(score);
    if (o.guide) {
        fill_guide_gaps(gj);
        std::memcpy(o.guide, gj.data(), sizeof(int32_t) * (m + 1));
    }
    return 0;
}

// ── Soft, log space, double (aligner.hpp:6231-6524) ──────────────────────────
inline double lse2(double a, double b) {
    const double NI = -std::numeric_limits<double>::infinity();
    if (a == NI) return b;
    if (b == NI) return a;
    if (a > b) return a + std::log1p(std::exp(b - a));
    return b + std::log1p(std::exp(a - b));
}
inline double lse3(double a, double b, double c) { return lse2(lse2(a, b), c); }

// Per-row double parameters of theta/T.
struct DRows {
    std::vector<double> goa, gea, gob, geb, bx0;
    std::vector<uint32_t> rs;
    std::vector<uint16_t> trk, gtrk;
};

void setup_drows(DRows& R, const Model& M, const uint8_t* a, int m, const uint16_t* track,
                 const uint16_t* gtrack, double invT, bool linear) {
    R.trk.assign(m, 0); R.gtrk.assign(m + 1, 0); R.rs.resize(m);
    if (track) for (int i = 0; i < m; ++i) R.trk[i] = track[i];
    if (gtrack) for (int i = 0; i <= m; ++i) R.gtrk[i] = gtrack[i];
    else { R.gtrk[0] = m ? R.trk[0] : 0; for (int i = 1; i <= m; ++i) R.gtrk[i] = R.trk[i - 1]; }
    for (int i = 0; i < m; ++i) R.rs[i] = uint32_t(R.trk[i]) * uint32_t(M.N) + a[i];
    R.goa.assign(m + 1, 0); R.gea.assign(m + 1, 0); R.gob.assign(m + 1, 0); R.geb.assign(m + 1, 0);
    R.bx0.assign(m + 1, 0);
    for (int i = 0; i <= m; ++i) {
        R.goa[i] = M.gaps[4 * R.gtrk[i] + kOpenA] * invT;
        R.gea[i] = M.gaps[4 * R.gtrk[i] + kExtendA] * invT;
    }
    for (int i = 1; i <= m; ++i) {
        R.gob[i] = M.gaps[4 * R.trk[i - 1] + kOpenB] * invT;
        R.geb[i] = M.gaps[4 * R.trk[i - 1] + kExtendB] * invT;
    }
    // column-0 border: the charged chain of gaps in B (exact sums)
    double s = 0;
    for (int i = 1; i <= m; ++i) {
        s += R.geb[i];
        R.bx0[i] = linear ? -s : -(R.gob[1] + s);
    }
}

struct SoftOut { double logz = 0; double* grad = nullptr; int32_t* post = nullptr; };

// soft_guide="posterior" (aligner.hpp:6776-6808, posterior_rows_log): per row i, the column of
// greatest EXIT mass over the row's band -- the cell's posterior less the mass moving on to
// (i, j+1) in row i (affine: the Y posterior at (i, j+1); linear: F(i,j) e_a B(i,j+1)) -- the
// first such column on ties; both in units of the row's largest cell posterior.  v(j) and y(j)
// are the two log-space terms at column j.  The rows then become a monotone guide.
template <class V, class Y>
void posterior_rows(int m, const Band& bd, int32_t* post, V&& v, Y&& y) {
    const double NI = -std::numeric_limits<double>::infinity();
    for (int i = 0; i <= m; ++i) {
        post[i] = 0;
        const int lo = bd.jlo0(i), hi = bd.jhi0(i);
        if (lo > hi) continue;
        double rmax = NI;
        for (int j = lo; j <= hi; ++j) rmax = std::max(rmax, v(i, j));
        double bv = -1.0;
        int bj = lo;
        for (int j = lo; j <= hi; ++j) {
            const double e = std::exp(v(i, j) - rmax) - std::exp((j < hi ? y(i, j) : NI) - rmax);
            if (e > bv) { bv = e; bj = j; }
        }
        post[i] = bj;
    }
    // posterior_guide (aligner.hpp:1466-1475): the rows as a guide, non-decreasing in [0, n]
    int run = 0;
    for (int i = 0; i <= m; ++i) { run = std::max(run, std::min(std::max(post[i], 0), bd.n)); post[i] = run; }
}

// Semi-global end cells, each once (aligner.hpp:6190-6196): row m's band (a free B end) or
// (m, n), then column n of rows 0..m-1 (a free A end).
template <class F>
void for_end_cells(const Model& M, int m, int n, const Band& bd, F&& f) {
    if (M.end_row()) { for (int j = bd.jlo0(m); j <= bd.jhi0(m); ++j) f(m, j); }
    else f(m, n);
    if (M.end_col()) for (int i = 0; i < m; ++i) f(i, n);
}
// The first row / column a gap move may target and be counted (aligner.hpp:6309-6319): a
// free start's border cells are constants, not the targets of gap moves.
int gap_min_j(const Model& M) { return M.am == 1 ? 1 : (M.free_col0() ? 1 : 0); }
int gap_min_i(const Model& M) { return M.am == 0 ? 0 : (M.am == 1 ? 1 : ((M.sg & 4) ? 1 : 0)); }

// Band bd (full when bd.band < 0): the guide-banded forward-backward (aligner.hpp:6362-6524
// with AlignBand::GuideBanded): forward cells j in [jlo(i), jhi(i)], borders limited to
// border_rows / border_cols (Global), Local log Z over [jlo0(i), jhi0(i)], backward sources
// and gradient sums over the band; cells outside it read -inf.
void soft_affine(const Model& M, const uint8_t* a, int m, const uint8_t* b, int n,
                 const uint16_t* track, const uint16_t* gtrack, double T, SoftOut& o, const Band& bd) {
    (void)a;
    const double NI = -std::numeric_limits<double>::infinity();
    const bool local = M.am == 1;
    const double invT = 1.0 / T;
    DRows R; setup_drows(R, M, a, m, track, gtrack, invT, false);
    const size_t st = size_t(n) + 1, cells = size_t(m + 1) * st;
    std::vector<double> FM(cells, NI), FX(cells, NI), FY(cells, NI);
    auto I = [&](int i, int j) { return size_t(i) * st + j; };
    auto sub = [&](int i, int j) { return M.mat[size_t(R.rs[i - 1]) * M.N + b[j - 1]] * invT; };
    if (!local) {
        FM[I(0, 0)] = 0.0;
        const int bi = bd.border_rows(), bj = bd.border_cols();
        for (int i = 1; i <= bi; ++i) FX[I(i, 0)] = R.bx0[i];
        if (M.free_row0()) { for (int j = 0; j <= n; ++j) FM[I(0, j)] = 0.0; }   // a free start
        else for (int j = 1; j <= bj; ++j) FY[I(0, j)] = -(R.goa[0] + double(j) * R.gea[0]);
        if (M.free_col0()) for (int i = 1; i <= m; ++i) { FM[I(i, 0)] = 0.0; FX[I(i, 0)] = NI; }
    } else {
        for (int i = 0; i <= m; ++i) FM[I(i, 0)] = 0.0;
        for (int j = 0; j <= n; ++j) FM[I(0, j)] = 0.0;
    }
    for (int i = 1; i <= m; ++i)
        for (int j = bd.jlo(i); j <= bd.jhi(i); ++j) {
            const double diag = lse3(FM[I(i - 1, j - 1)], FX[I(i - 1, j - 1)], FY[I(i - 1, j - 1)]);
            double mv = diag + sub(i, j);
            const double gob = R.gob[i], geb = R.geb[i], goa = R.goa[i], gea = R.gea[i];
            const double xv = lse3(FM[I(i - 1, j)] - gob - geb, FX[I(i - 1, j)] - geb, FY[I(i - 1, j)] - gob - geb);
            const double yv = lse3(FM[I(i, j - 1)] - goa - gea, FX[I(i, j - 1)] - goa - gea, FY[I(i, j - 1)] - gea);
            if (local) mv = lse2(mv, 0.0);
            FM[I(i, j)] = mv; FX[I(i, j)] = xv; FY[I(i, j)] = yv;
        }
    double lz;
    if (M.semi()) {   // the end cells (sg_for_end_cells_, aligner.hpp:6190-6196)
        lz = NI;
        for_end_cells(M, m, n, bd, [&](int i, int j) { lz = lse2(lz, lse3(FM[I(i, j)], FX[I(i, j)], FY[I(i, j)])); });
    } else if (!local) lz = lse3(FM[I(m, n)], FX[I(m, n)], FY[I(m, n)]);
    else {
        lz = NI;
        for (int i = 0; i <= m; ++i) for (int j = bd.jlo0(i); j <= bd.jhi0(i); ++j)
            lz = lse2(lz, lse3(FM[I(i, j)], FX[I(i, j)], FY[I(i, j)]));
    }
    std::vector<double> BM(cells, local ? 0.0 : NI), BX(BM), BY(BM);
    if (M.semi()) for_end_cells(M, m, n, bd, [&](int i, int j) { BM[I(i, j)] = 0; BX[I(i, j)] = 0; BY[I(i, j)] = 0; });
    else if (!local) { BM[I(m, n)] = 0; BX[I(m, n)] = 0; BY[I(m, n)] = 0; }
    for (int i = m; i >= 0; --i)
        for (int j = bd.jhi0(i); j >= bd.jlo0(i); --j) {
            const double bm = BM[I(i, j)], bx = BX[I(i, j)], by = BY[I(i, j)];
            if (bm != NI && i > 0 && j > 0) {
                const double c = bm + sub(i, j);
                BM[I(i - 1, j - 1)] = lse2(BM[I(i - 1, j - 1)], c);
                BX[I(i - 1, j - 1)] = lse2(BX[I(i - 1, j - 1)], c);
                BY[I(i - 1, j - 1)] = lse2(BY[I(i - 1, j - 1)], c);
            }
            if (bx != NI && i > 0) {
                const double gob = R.gob[i], geb = R.geb[i];
                BM[I(i - 1, j)] = lse2(BM[I(i - 1, j)], bx - gob - geb);
                BX[I(i - 1, j)] = lse2(BX[I(i - 1, j)], bx - geb);
                BY[I(i - 1, j)] = lse2(BY[I(i - 1, j)], bx - gob - geb);
            }
            if (by != NI && j > 0) {
                const double goa = R.goa[i], gea = R.gea[i];
                BM[I(i, j - 1)] = lse2(BM[I(i, j - 1)], by - goa - gea);
                BX[I(i, j - 1)] = lse2(BX[I(i, j - 1)], by - goa - gea);
                BY[I(i, j - 1)] = lse2(BY[I(i, j - 1)], by - gea);
            }
        }
    const size_t NN = size_t(M.K) * M.N * M.N;
    double* g = o.grad;
    auto gap = [&](int set, int f) -> double& { return g[NN + 4 * size_t(set) + f]; };
    const int gmin_j = gap_min_j(M), gmin_i = gap_min_i(M);
    for (int i = 1; i <= m; ++i)
        for (int j = bd.jlo(i); j <= bd.jhi(i); ++j) {
            const double bm = BM[I(i, j)];
            if (bm == NI) continue;
            const double pred = lse3(FM[I(i - 1, j - 1)], FX[I(i - 1, j - 1)], FY[I(i - 1, j - 1)]);
            g[size_t(R.rs[i - 1]) * M.N + b[j - 1]] += std::exp(pred + sub(i, j) + bm - lz);
        }
    for (int i = 1; i <= m; ++i)
        for (int j = bd.jlo0(i); j <= bd.jhi0(i); ++j) {
            const double fx = FX[I(i, j)], bx = BX[I(i, j)];
            if (fx == NI || bx == NI) continue;
            gap(R.trk[i - 1], kExtendB) -= std::exp(fx + bx - lz);
        }
    for (int i = 0; i <= m; ++i)
        for (int j = std::max(1, bd.jlo0(i)); j <= bd.jhi0(i); ++j) {
            const double fy = FY[I(i, j)], by = BY[I(i, j)];
            if (fy == NI || by == NI) continue;
            gap(R.gtrk[i], kExtendA) -= std::exp(fy + by - lz);
        }
    for (int i = 1; i <= m; ++i)
        for (int j = std::max(gmin_j, bd.jlo0(i)); j <= bd.jhi0(i); ++j) {
            const double bx = BX[I(i, j)];
            if (bx == NI) continue;
            const double lo = lse2(FM[I(i - 1, j)], FY[I(i - 1, j)]) - R.gob[i] - R.geb[i] + bx - lz;
            if (lo > -700) gap(R.trk[i - 1], kOpenB) -= std::exp(lo);
        }
    for (int i = gmin_i; i <= m; ++i)
        for (int j = std::max(1, bd.jlo0(i)); j <= bd.jhi0(i); ++j) {
            const double by = BY[I(i, j)];
            if (by == NI) continue;
            const double lo = lse2(FM[I(i, j - 1)], FX[I(i, j - 1)]) - R.goa[i] - R.gea[i] + by - lz;
            if (lo > -700) gap(R.gtrk[i], kOpenA) -= std::exp(lo);
        }
    if (o.post)
        posterior_rows(m, bd, o.post,
                       [&](int i, int j) { return lse3(FM[I(i, j)] + BM[I(i, j)], FX[I(i, j)] + BX[I(i, j)], FY[I(i, j)] + BY[I(i, j)]); },
                       [&](int i, int j) { return FY[I(i, j + 1)] + BY[I(i, j + 1)]; });
    o.logz = lz * T;
}

void soft_linear(const Model& M, const uint8_t* a, int m, const uint8_t* b, int n,
                 const uint16_t* track, const uint16_t* gtrack, double T, SoftOut& o, const Band& bd) {
    const double NI = -std::numeric_limits<double>::infinity();
    const bool local = M.am == 1;
    const double invT = 1.0 / T;
    DRows R; setup_drows(R, M, a, m, track, gtrack, invT, true);
    const size_t st = size_t(n) + 1, cells = size_t(m + 1) * st;
    std::vector<double> F(cells, NI), B(cells, local ? 0.0 : NI);
    auto I = [&](int i, int j) { return size_t(i) * st + j; };
    auto sub = [&](int i, int j) { return M.mat[size_t(R.rs[i - 1]) * M.N + b[j - 1]] * invT; };
    if (!local) {
        F[I(0, 0)] = 0.0;
        const int bi = bd.border_rows(), bj = bd.border_cols();
        for (int i = 1; i <= bi; ++i) F[I(i, 0)] = R.bx0[i];
        if (M.free_row0()) { for (int j = 0; j <= n; ++j) F[I(0, j)] = 0.0; }   // a free start
        else for (int j = 1; j <= bj; ++j) F[I(0, j)] = -double(j) * R.gea[0];
        if (M.free_col0()) for (int i = 1; i <= m; ++i) F[I(i, 0)] = 0.0;
    } else {
        for (int i = 0; i <= m; ++i) F[I(i, 0)] = 0.0;
        for (int j = 0; j <= n; ++j) F[I(0, j)] = 0.0;
    }
    for (int i = 1; i <= m; ++i)
        for (int j = bd.jlo(i); j <= bd.jhi(i); ++j) {
            double v = lse3(F[I(i - 1, j - 1)] + sub(i, j), F[I(i - 1, j)] - R.geb[i], F[I(i, j - 1)] - R.gea[i]);
            if (local) v = lse2(v, 0.0);
            F[I(i, j)] = v;
        }
    double lz;
    if (M.semi()) {
        lz = NI;
        for_end_cells(M, m, n, bd, [&](int i, int j) { lz = lse2(lz, F[I(i, j)]); });
    } else if (!local) lz = F[I(m, n)];
    else {
        lz = NI;
        for (int i = 0; i <= m; ++i) for (int j = bd.jlo0(i); j <= bd.jhi0(i); ++j) lz = lse2(lz, F[I(i, j)]);
    }
    if (M.semi()) for_end_cells(M, m, n, bd, [&](int i, int j) { B[I(i, j)] = 0.0; });
    else if (!local) B[I(m, n)] = 0.0;
    for (int i = m; i >= 0; --i)
        for (int j = bd.jhi0(i); j >= bd.jlo0(i); --j) {
            const double bv = B[I(i, j)];
            if (bv == NI) continue;
            if (i > 0 && j > 0) B[I(i - 1, j - 1)] = lse2(B[I(i - 1, j - 1)], bv + sub(i, j));
            if (i > 0) B[I(i - 1, j)] = lse2(B[I(i - 1, j)], bv - R.geb[i]);
            if (j > 0) B[I(i, j - 1)] = lse2(B[I(i, j - 1)], bv - R.gea[i]);
        }
    const size_t NN = size_t(M.K) * M.N * M.N;
    double* g = o.grad;
    auto gap = [&](int set, int f) -> double& { return g[NN + 4 * size_t(set) + f]; };
    const int gmin_j = gap_min_j(M), gmin_i = gap_min_i(M);
    for (int i = 1; i <= m; ++i)
        for (int j = bd.jlo(i); j <= bd.jhi(i); ++j) {
            const double bv = B[I(i, j)];
            if (bv == NI) continue;
            g[size_t(R.rs[i - 1]) * M.N + b[j - 1]] += std::exp(F[I(i - 1, j - 1)] + sub(i, j) + bv - lz);
        }
    for (int i = 1; i <= m; ++i)
        for (int j = std::max(gmin_j, bd.jlo0(i)); j <= bd.jhi0(i); ++j) {
            const double bv = B[I(i, j)], fv = F[I(i - 1, j)];
            if (bv == NI || fv == NI) continue;
            gap(R.trk[i - 1], kExtendB) -= std::exp(fv - R.geb[i] + bv - lz);
        }
    for (int i = gmin_i; i <= m; ++i)
        for (int j = std::max(1, bd.jlo0(i)); j <= bd.jhi0(i); ++j) {
            const double bv = B[I(i, j)], fv = F[I(i, j - 1)];
            if (bv == NI || fv == NI) continue;
            gap(R.gtrk[i], kExtendA) -= std::exp(fv - R.gea[i] + bv - lz);
        }
    if (o.post)
        posterior_rows(m, bd, o.post, [&](int i, int j) { return F[I(i, j)] + B[I(i, j)]; },
                       [&](int i, int j) { return F[I(i, j)] - R.gea[i] + B[I(i, j + 1)]; });
    o.logz = lz * T;
}

// ── Hirschberg, affine Global, untracked (aligner.hpp:4151-4560) ───────────────
// Divide and conquer: split the block's rows at p = i0 + H/2, sweep rows (i0, p] forward
// and [p, i1) backward keeping only the last row (hb_fwd :4151, hb_rev :4210), join at the
// first column of the strictly largest f + g, or an X run straddling the cut with one
// go_b refunded (hb_solve :4458-4518), recurse; blocks of at most `cutoff` rows are solved
// by a Pointers fill with the block's own borders (hb_base :4318-4400).  in_x / out_x: the
// block's path leaves its origin / enters its corner by a vertical move of an inherited
// run.  Pmax: the horizontal carry by the closed-form prefix max (hirschberg_pmax).  The
// score is replayed along the path in T (:4530-4552).
template <class T, bool Pmax>
struct Hb {
    int N; const T* blk; const uint8_t* a; const uint8_t* b; int cutoff;
    T go_a, ge_a, go_b, ge_b;
    std::vector<uint8_t> hops;                 // 0 M, 1 X (down), 2 Y (right), path order
    T sub(int r, int c) const { return blk[size_t(a[r - 1]) * N + b[c - 1]]; }   // 1-based

    // row 0 of a sweep block: the origin, then Y moves along it
    void row0(bool flag, int W, std::vector<T>& pM, std::vector<T>& pX, std::vector<T>& pY) const {
        pM[0] = flag ? ninf<T>() : T(0); pX[0] = ninf<T>(); pY[0] = ninf<T>();
        for (int c = 1; c <= W; ++c) {
            pM[c] = ninf<T>(); pX[c] = ninf<T>();
            pY[c] = mx3<T>((pM[c - 1] - go_a) - ge_a, (pX[c - 1] - go_a) - ge_a, pY[c - 1] - ge_a);
        }
    }
    // One sweep: H rows; sub_of(t, c) the substitution of swept row t (1..H), column c.
    template <class F>
    void sweep(int H, int W, bool flag, F sub_of, std::vector<T>& pM, std::vector<T>& pX,
               std::vector<T>& pY) const {
        std::vector<T> cM(W + 1), cX(W + 1), cY(W + 1), rmp(W + 1);
        if (Pmax) for (int k = 0; k <= W; ++k) rmp[k] = static_cast<T>(k) * ge_a;
        row0(flag, W, pM, pX, pY);
        for (int t = 1; t <= H; ++t) {
            cM[0] = ninf<T>();
            cX[0] = mx3<T>((pM[0] - go_b) - ge_b, pX[0] - ge_b, (pY[0] - go_b) - ge_b);
            if (flag && t == 1) cX[0] = T(0) - ge_b;
            cY[0] = ninf<T>();
            T P = cY[0] - ge_a;
            for (int c = 1; c <= W; ++c) {
                cM[c] = mx3<T>(pM[c - 1], pX[c - 1], pY[c - 1]) + sub_of(t, c);
                cX[c] = mx3<T>((pM[c] - go_b) - ge_b, pX[c] - ge_b, (pY[c] - go_b) - ge_b);
                if (Pmax) {
                    const T g = (mx<T>(cM[c - 1], cX[c - 1]) - go_a) - ge_a;
                    P = mx<T>(g + rmp[c - 1], P);
                    cY[c] = P - rmp[c - 1];
                } else {
                    cY[c] = mx3<T>((cM[c - 1] - go_a) - ge_a, (cX[c - 1] - go_a) - ge_a, cY[c - 1] - ge_a);
                }
            }
            std::swap(pM, cM); std::swap(pX, cX); std::swap(pY, cY);
        }
    }
    static uint8_t pick(T vm, T vx, T vy) {
        if (vm >= vx && vm >= vy) return 0;
        return (vx >= vy) ? 1 : 2;
    }
    void base(int i0, int i1, int j0, int j1, bool in_x, bool out_x) {
        const int H = i1 - i0, W = j1 - j0;
        if (H == 0 && W == 0) return;
        const size_t st = size_t(W) + 1;
        std::vector<uint8_t> D(size_t(H + 1) * st);
        std::vector<T> pM(st), pX(st), pY(st), cM(st), cX(st), cY(st);
        auto pack = [](unsigned km, unsigned kx, unsigned ky) { return uint8_t(km | kx << 2 | ky << 4); };
        pM[0] = in_x ? ninf<T>() : T(0); pX[0] = ninf<T>(); pY[0] = ninf<T>();
        D[0] = pack(3, 3, 3);
        for (int c = 1; c <= W; ++c) {
            pM[c] = ninf<T>(); pX[c] = ninf<T>();
            const T uy = (pM[c - 1] - go_a) - ge_a, vy = (pX[c - 1] - go_a) - ge_a, wy = pY[c - 1] - ge_a;
            pY[c] = mx3<T>(uy, vy, wy);
            D[c] = pack(3, 3, pick(uy, vy, wy));
        }
        for (int r = 1; r <= H; ++r) {
            const size_t rb = size_t(r) * st;
            const T ux0 = (pM[0] - go_b) - ge_b, vx0 = pX[0] - ge_b, wx0 = (pY[0] - go_b) - ge_b;
            cM[0] = ninf<T>(); cX[0] = mx3<T>(ux0, vx0, wx0); cY[0] = ninf<T>();
            D[rb] = pack(3, pick(ux0, vx0, wx0), 3);
            if (in_x && r == 1) { cX[0] = T(0) - ge_b; D[rb] = pack(3, 1, 3); }
            for (int c = 1; c <= W; ++c) {
                const T dgM = pM[c - 1], dgX = pX[c - 1], dgY = pY[c - 1];
                cM[c] = mx3<T>(dgM, dgX, dgY) + sub(i0 + r, j0 + c);
                const T ux = (pM[c] - go_b) - ge_b, vx = pX[c] - ge_b, wx = (pY[c] - go_b) - ge_b;
                cX[c] = mx3<T>(ux, vx, wx);
                const T uy = (cM[c - 1] - go_a) - ge_a, vy = (cX[c - 1] - go_a) - ge_a, wy = cY[c - 1] - ge_a;
                cY[c] = mx3<T>(uy, vy, wy);
                D[rb + c] = pack(pick(dgM, dgX, dgY), pick(ux, vx, wx), pick(uy, vy, wy));
            }
            std::swap(pM, cM); std::swap(pX, cX); std::swap(pY, cY);
        }
        int r = H, c = W;
        Tbl tbl;
        if (out_x) tbl = TX;
        else {
            const T vm = pM[W], vx = pX[W], vy = pY[W];
            tbl = (vm >= vx && vm >= vy) ? TM : ((vx >= vy) ? TX : TY);
        }
        const size_t first = hops.size();
        while (r > 0 || c > 0) {
            const uint8_t p = D[size_t(r) * st + size_t(c)];
            uint8_t code;
            if (tbl == TM)      { code = p & 3;        hops.push_back(0); --r; --c; }
            else if (tbl == TX) { code = (p >> 2) & 3; hops.push_back(1); --r; }
            else                { code = p >> 4;       hops.push_back(2); --c; }
            tbl = (code == 1) ? TX : (code == 2 ? TY : TM);
        }
        std::reverse(hops.begin() + std::ptrdiff_t(first), hops.end());
    }
    void solve(int i0, int i1, int j0, int j1, bool in_x, bool out_x) {
        const int H = i1 - i0, W = j1 - j0;
        if (H <= cutoff) { base(i0, i1, j0, j1, in_x, out_x); return; }
        const int p = i0 + H / 2;
        std::vector<T> FM(W + 1), FX(W + 1), FY(W + 1), rM(W + 1), rX(W + 1), rY(W + 1);
        // forward: swept row t is DP row i0 + t, column c pairs b[j0 + c - 1]
        sweep(p - i0, W, in_x, [&](int t, int cc) { return sub(i0 + t, j0 + cc); }, FM, FX, FY);
        // reverse: swept row t consumes a[i1 - t] (DP row i1 - t + 1), column d pairs b[j1 - d]
        sweep(i1 - p, W, out_x, [&](int t, int d) { return sub(i1 - t + 1, j1 - d + 1); }, rM, rX, rY);
        T best = ninf<T>();
        int cstar = 0;
        bool span = false;
        for (int cc = 0; cc <= W; ++cc) {
            const int d = W - cc;
            const T f = mx3<T>(FM[cc], FX[cc], FY[cc]);
            const T g = mx3<T>(rM[d], rX[d], rY[d]);
            const T plain = f + g;
            if (plain > best) { best = plain; cstar = cc; span = false; }
            if (FX[cc] > ninf<T>() && rX[d] > ninf<T>()) {
                const T joined = (FX[cc] + rX[d]) + go_b;
                if (joined > best) { best = joined; cstar = cc; span = true; }
            }
        }
        const int jstar = j0 + cstar;
        solve(i0, p, j0, jstar, in_x, span);
        solve(p, i1, jstar, j1, span, out_x);
    }
};

// One pair by Hirschberg when it splits (m > cutoff); else the Pointers path (aligner.hpp
// :1360, run_viterbi: a pair that never splits runs AS Pointers).  Guide in the recursion's
// convention: the column where the path enters each row (guide_j_affine_hb :5233-5249).
// The endpoint scan of Local Hirschberg (hb_scan_scalar, aligner.hpp:4611-4698) over rows
// [i0, i1), columns [j0, j1): forward (reverse = false) or from the far corner back; `local`:
// the clamped Smith-Waterman recurrence with free starts on row 0 and column 0, else the
// global borders (row 0 the charged Y chain, column 0 the X chain).  The best cell is the
// first strictly larger max(M, X, Y) in row-major scan order from 0 (topmost row, then
// leftmost column), in block coordinates (rows 1..H, columns 1..NC); (0, 0) with best 0
// when no cell is positive.  Pmax: the prefix-max horizontal carry.
template <class T>
void hb_scan(const T* blk, int N, const uint8_t* a, const uint8_t* b, T go_a, T ge_a, T go_b, T ge_b, bool pmax,
             bool local, bool reverse, int i0, int i1, int j0, int j1, T& best, int& bi, int& bj) {
    const int H = i1 - i0, NC = j1 - j0;
    best = T(0); bi = 0; bj = 0;
    if (H == 0 || NC == 0) return;
    const int a_start = reverse ? i1 - 1 : i0, a_step = reverse ? -1 : 1;
    const int b_start = reverse ? j1 - 1 : j0, b_step = reverse ? -1 : 1;
    std::vector<T> pM(NC + 1), pX(NC + 1), pY(NC + 1), cM(NC + 1), cX(NC + 1), cY(NC + 1), rmp(NC + 1);
    if (pmax) for (int k = 0; k < NC; ++k) rmp[k] = static_cast<T>(k) * ge_a;
    pM[0] = T(0); pX[0] = ninf<T>(); pY[0] = ninf<T>();
    for (int cc = 1; cc <= NC; ++cc) {
        if (local) { pM[cc] = T(0); pX[cc] = ninf<T>(); pY[cc] = ninf<T>(); }
        else {
            pM[cc] = ninf<T>(); pX[cc] = ninf<T>();
            pY[cc] = mx<T>((mx<T>(pM[cc - 1], pX[cc - 1]) - go_a) - ge_a, pY[cc - 1] - ge_a);
        }
    }
    T gbest = T(0); int gi = 0, gj = 0;
    for (int t = 0; t < H; ++t) {
        const int arow = a_start + t * a_step;
        cM[0] = local ? T(0) : ninf<T>();
        cX[0] = mx<T>(mx<T>((pM[0] - go_b) - ge_b, pX[0] - ge_b), (pY[0] - go_b) - ge_b);
        cY[0] = ninf<T>();
        T P = cY[0] - ge_a;
        for (int cc = 1; cc <= NC; ++cc) {
            const int bcol = b_start + (cc - 1) * b_step;
            T mv = mx3<T>(pM[cc - 1], pX[cc - 1], pY[cc - 1]) + blk[size_t(a[arow]) * N + b[bcol]];
            if (local) mv = mx<T>(mv, T(0));
            const T xv = mx<T>(mx<T>((pM[cc] - go_b) - ge_b, pX[cc] - ge_b), (pY[cc] - go_b) - ge_b);
            T yv;
            if (pmax) {
                const T g = (mx<T>(cM[cc - 1], cX[cc - 1]) - go_a) - ge_a;
                P = mx<T>(g + rmp[cc - 1], P);
                yv = P - rmp[cc - 1];
            } else {
                yv = mx<T>(mx<T>((cM[cc - 1] - go_a) - ge_a, (cX[cc - 1] - go_a) - ge_a), cY[cc - 1] - ge_a);
            }
            cM[cc] = mv; cX[cc] = xv; cY[cc] = yv;
            const T here = mx3<T>(mv, xv, yv);
            if (here > gbest) { gbest = here; gi = t + 1; gj = cc; }
        }
        std::swap(pM, cM); std::swap(pX, cX); std::swap(pY, cY);
    }
    best = gbest; bi = gi; bj = gj;
}

// The path's score in T, counts and guide, replayed from (i0, j0) (aligner.hpp:4530-4552,
// hard_fields :776-790, guide_j_affine_hb :5233-5249).
template <class T>
void hb_replay(const Model& M, const uint8_t* a, int m, const uint8_t* b, int n, const std::vector<uint8_t>& hops,
               const std::vector<T>& blk, T go_a, T ge_a, T go_b, T ge_b, int i0, int j0, int ie, int je, HardOut& o) {
    T s = T(0);
    int i = i0, j = j0;
    uint8_t prev = 3;
    std::vector<int32_t> gj(size_t(m) + 1, -1);
    gj[0] = 0;
    gj[i0] = j0;
    for (uint8_t op : hops) {
        if (op == 0) {
            ++i; ++j;
            s += blk[size_t(a[i - 1]) * M.N + b[j - 1]];
            if (o.grad) o.grad[size_t(a[i - 1]) * M.N + b[j - 1]] += 1.0;
            gj[i] = j;
        } else if (op == 1) {
            ++i;
            if (prev != 1) { s -= go_b; if (o.grad) o.grad[size_t(M.N) * M.N + kOpenB] -= 1.0; }
            s -= ge_b;
            if (o.grad) o.grad[size_t(M.N) * M.N + kExtendB] -= 1.0;
            gj[i] = j;
        } else {
            if (prev != 2) { s -= go_a; if (o.grad) o.grad[size_t(M.N) * M.N + kOpenA] -= 1.0; }
            s -= ge_a;
            if (o.grad) o.grad[size_t(M.N) * M.N + kExtendA] -= 1.0;
            ++j;
        }
        prev = op;
    }
    gj[m] = n;
    fill_guide_gaps(gj);
    if (o.guide) std::memcpy(o.guide, gj.data(), sizeof(int32_t) * (m + 1));
    if (o.moves) {
        const int64_t k = std::min<int64_t>(int64_t(hops.size()), o.moves_cap);
        for (int64_t q = 0; q < k; ++q) o.moves[q] = hops[q];
    }
    o.nmoves = int64_t(hops.size());
    o.score = static_cast<double>(s);
    o.end_i = ie; o.end_j = je; o.start_i = i0; o.start_j = j0;
}

// Local affine Hirschberg (viterbi_affine_hirschberg_local, aligner.hpp:4746-4790), for a
// pair longer than the cutoff (shorter ones run the Pointers path): the
// forward clamped scan gives the end cell (ie, je) and the score; none positive: the empty
// alignment (score 0 at (0, 0)).  Else the reverse global-suffix scan over rows [0, ie),
// columns [0, je) gives the start (is, js) = (ie - p, je - q); the box A[is, ie) x B[js, je)
// is solved globally by the recursion (short boxes by its base case) and the path replayed.
template <class T>
int hb_local_one(const Model& M, const uint8_t* a, int m, const uint8_t* b, int n, int cutoff, bool pmax,
                 HardOut& o) {
    // a pair of at most `cutoff` rows runs AS Pointers (hb_splits, aligner.hpp:137-141)
    if (m <= cutoff) return hard_one<T>(M, a, m, b, n, nullptr, nullptr, false, nullptr, -1, o, 0);
    std::vector<T> blk(size_t(M.N) * M.N);
    for (size_t k = 0; k < blk.size(); ++k) blk[k] = static_cast<T>(M.mat[k]);
    const T go_a = static_cast<T>(M.gaps[kOpenA]), ge_a = static_cast<T>(M.gaps[kExtendA]);
    const T go_b = static_cast<T>(M.gaps[kOpenB]), ge_b = static_cast<T>(M.gaps[kExtendB]);
    T sf; int ie, je;
    hb_scan<T>(blk.data(), M.N, a, b, go_a, ge_a, go_b, ge_b, pmax, true, false, 0, m, 0, n, sf, ie, je);
    std::vector<uint8_t> hops;
    if (!(sf > T(0)) || ie <= 0 || je <= 0) {
        hb_replay<T>(M, a, m, b, n, hops, blk, go_a, ge_a, go_b, ge_b, 0, 0, 0, 0, o);
        return 0;
    }
    T sr; int p, q;
    hb_scan<T>(blk.data(), M.N, a, b, go_a, ge_a, go_b, ge_b, pmax, false, true, 0, ie, 0, je, sr, p, q);
    const int is = ie - p, js = je - q;
    if (pmax) {
        Hb<T, true> h{M.N, blk.data(), a, b, cutoff, go_a, ge_a, go_b, ge_b, {}};
        h.solve(is, ie, js, je, false, false);
        hops.swap(h.hops);
    } else {
        Hb<T, false> h{M.N, blk.data(), a, b, cutoff, go_a, ge_a, go_b, ge_b, {}};
        h.solve(is, ie, js, je, false, false);
        hops.swap(h.hops);
    }
    hb_replay<T>(M, a, m, b, n, hops, blk, go_a, ge_a, go_b, ge_b, is, js, ie, je, o);
    return 0;
}

// Linear-gap Hirschberg (viterbi_linear_hirschberg, aligner.hpp:5020-5185): no gap state
// crosses a cut, so the join is the first column of the strictly largest F + R; sweeps
// (lhb_sweep :4844-4913) keep one row, borders the Global gap chains; base blocks of at most
// `cutoff` rows are Pointers fills of the box (lhb_base :4917-4997; ties: M, then X, then Y),
// walked back.  Local: the forward clamped scan for the end (first strictly larger cell,
// row-major), then the unclamped global-suffix scan over [0, ie) x [0, je) for the start
// (row ie first with its columns ascending, then rows upward, column je first in each, then
// columns downward; strict >), then the box solved as Global.
template <class T>
struct Lhb {
    int N; const T* blk; const uint8_t* b; int cutoff;
    const Rows<T>* R;                           // per DP row: substitution row, extends
    std::vector<uint8_t> hops;
    T sub(int i, int c) const { return blk[size_t(R->rs[i - 1]) * N + b[c - 1]]; }   // 1-based
    T ga(int i) const { return R->gea[i]; }    // gaps in A within DP row i
    T gb(int i) const { return R->geb[i]; }    // a gap in B into DP row i
    // lhb_sweep: forward, DP rows i0+1..i1 (gaps in A on row i); reverse (the mirror), DP rows
    // i1..i0+1 as the suffix from row i-1 (gaps in A on row i-1); row 0's chain on row i0 / i1
    void sweep(bool rev, int i0, int i1, int j0, int j1, std::vector<T>& row) const {
        const int W = j1 - j0;
        row.assign(size_t(W) + 1, T(0));
        const T g0 = ga(rev ? i1 : i0);
        for (int cc = 1; cc <= W; ++cc) row[cc] = row[cc - 1] - g0;
        for (int r = 1; r <= i1 - i0; ++r) {
            const int i = rev ? i1 - r + 1 : i0 + r;
            const T gea = ga(rev ? i - 1 : i), geb = gb(i);
            T diag = row[0];
            row[0] = row[0] - geb;
            T left = row[0];
            for (int cc = 1; cc <= W; ++cc) {
                const int bcol = rev ? j1 - cc : j0 + cc - 1;   // 0-based
                T v = diag + blk[size_t(R->rs[i - 1]) * N + b[bcol]];
                const T u = row[cc] - geb, l = left - gea;
                if (v < u) v = u;
                if (v < l) v = l;
                diag = row[cc];
                row[cc] = v;
                left = v;
            }
        }
    }
    void base(int i0, int i1, int j0, int j1) {
        const int H = i1 - i0, W = j1 - j0;
        const size_t st = size_t(W) + 1;
        std::vector<uint8_t> D(size_t(H + 1) * st);
        std::vector<T> prev(st), cur(st);
        prev[0] = T(0);
        const T g0 = ga(i0);
        for (int cc = 1; cc <= W; ++cc) { prev[cc] = prev[cc - 1] - g0; D[cc] = 2; }
        for (int r = 1; r <= H; ++r) {
            const T gea = ga(i0 + r), geb = gb(i0 + r);
            uint8_t* d = D.data() + size_t(r) * st;
            cur[0] = prev[0] - geb; d[0] = 1;
            T left = cur[0];
            for (int cc = 1; cc <= W; ++cc) {
                T v = prev[cc - 1] + sub(i0 + r, j0 + cc);
                uint8_t k = 0;
                const T u = prev[cc] - geb, l = left - gea;
                if (v < u) { v = u; k = 1; }
                if (v < l) { v = l; k = 2; }
                cur[cc] = v; d[cc] = k; left = v;
            }
            std::swap(prev, cur);
        }
        const size_t first = hops.size();
        int r = H, cc = W;
        while (r > 0 || cc > 0) {
            const uint8_t k = D[size_t(r) * st + size_t(cc)];
            hops.push_back(k);
            if (k == 0) { --r; --cc; } else if (k == 1) --r; else --cc;
        }
        std::reverse(hops.begin() + std::ptrdiff_t(first), hops.end());
    }
    void solve(int i0, int i1, int j0, int j1) {
        const int H = i1 - i0, W = j1 - j0;
        if (H <= cutoff) { base(i0, i1, j0, j1); return; }
        const int p = i0 + H / 2;
        std::vector<T> F, Rr;
        sweep(false, i0, p, j0, j1, F);
        sweep(true, p, i1, j0, j1, Rr);
        T best = ninf<T>();
        int cstar = 0;
        for (int cc = 0; cc <= W; ++cc) {
            const T v = F[cc] + Rr[W - cc];
            if (v > best) { best = v; cstar = cc; }
        }
        solve(i0, p, j0, j0 + cstar);
        solve(p, i1, j0 + cstar, j1);
    }
};

template <class T>
int lhb_one(const Model& M, const uint8_t* a, int m, const uint8_t* b, int n, const uint16_t* track,
            const uint16_t* gtrack, bool tracked, int cutoff, HardOut& o) {
    if (m <= cutoff) return hard_one<T>(M, a, m, b, n, track, gtrack, tracked, nullptr, -1, o, 0);
    Rows<T> R;
    setup_rows<T, true>(R, M, a, m, track, gtrack, tracked);
    std::vector<T> blk(size_t(M.K) * M.N * M.N);
    for (size_t k = 0; k < blk.size(); ++k) blk[k] = static_cast<T>(M.mat[k]);
    Lhb<T> h{M.N, blk.data(), b, cutoff, &R, {}};
    int is = 0, js = 0, ie = m, je = n;
    bool empty = false;
    if (M.am == 1) {
        std::vector<T> row(size_t(n) + 1, T(0));
        T best = T(0); ie = 0; je = 0;
        for (int i = 1; i <= m; ++i) {
            T diag = row[0];
            const T gea = h.ga(i), geb = h.gb(i);
            for (int j = 1; j <= n; ++j) {
                T v = diag + h.sub(i, j);
                const T u = row[j] - geb, l = row[j - 1] - gea;
                if (v < u) v = u;
                if (v < l) v = l;
                v = mx<T>(v, T(0));
                diag = row[j];
                row[j] = v;
                if (v > best) { best = v; ie = i; je = j; }
            }
        }
        if (!(best > T(0))) { empty = true; ie = 0; je = 0; }
        else {
            std::vector<T> g(size_t(je) + 1);
            g[je] = T(0);
            const T g0 = h.ga(ie);
            for (int q = je - 1; q >= 0; --q) g[q] = g[q + 1] - g0;
            T sbest = g[0]; is = ie; js = 0;
            for (int q = 0; q <= je; ++q) if (g[q] > sbest) { sbest = g[q]; js = q; }
            for (int pi = ie - 1; pi >= 0; --pi) {
                const T gea = h.ga(pi), geb = h.gb(pi + 1);
                T diag = g[je];
                g[je] = g[je] - geb;
                if (g[je] > sbest) { sbest = g[je]; is = pi; js = je; }
                for (int q = je - 1; q >= 0; --q) {
                    T v = diag + h.sub(pi + 1, q + 1);
                    const T u = g[q] - geb, l = g[q + 1] - gea;
                    if (v < u) v = u;
                    if (v < l) v = l;
                    diag = g[q];
                    g[q] = v;
                    if (v > sbest) { sbest = v; is = pi; js = q; }
                }
            }
        }
    }
    if (!empty) h.solve(is, ie, js, je);
    // replay: score in T, counts, guide (guide_j_affine_hb :5233-5249, gap-model free)
    const size_t NN = size_t(M.K) * M.N * M.N;
    T s = T(0);
    int i = is, j = js;
    std::vector<int32_t> gj(size_t(m) + 1, -1);
    gj[0] = 0;
    gj[is] = js;
    for (uint8_t op : h.hops) {
        if (op == 0) {
            ++i; ++j;
            s += h.sub(i, j);
            if (o.grad) o.grad[size_t(R.rs[i - 1]) * M.N + b[j - 1]] += 1.0;
            gj[i] = j;
        } else if (op == 1) {
            ++i;
            s -= h.gb(i);
            if (o.grad) o.grad[NN + 4 * size_t(R.trk[i - 1]) + kExtendB] -= 1.0;
            gj[i] = j;
        } else {
            s -= h.ga(i);
            if (o.grad) o.grad[NN + 4 * size_t(R.gtrk[i]) + kExtendA] -= 1.0;
            ++j;
        }
    }
    gj[m] = n;
    fill_guide_gaps(gj);
    if (o.guide) std::memcpy(o.guide, gj.data(), sizeof(int32_t) * (m + 1));
    if (o.moves) {
        const int64_t k = std::min<int64_t>(int64_t(h.hops.size()), o.moves_cap);
        for (int64_t q = 0; q < k; ++q) o.moves[q] = h.hops[q];
    }
    o.nmoves = int64_t(h.hops.size());
    o.score = static_cast<double>(s);
    o.end_i = ie; o.end_j = je; o.start_i = is; o.start_j = js;
    return 0;
}

template <class T>
int hb_one(const Model& M, const uint8_t* a, int m, const uint8_t* b, int n, int cutoff, bool pmax,
           HardOut& o) {
    if (m <= cutoff) return hard_one<T>(M, a, m, b, n, nullptr, nullptr, false, nullptr, -1, o, 0);
    std::vector<T> blk(size_t(M.N) * M.N);
    for (size_t k = 0; k < blk.size(); ++k) blk[k] = static_cast<T>(M.mat[k]);
    const T go_a = static_cast<T>(M.gaps[kOpenA]), ge_a = static_cast<T>(M.gaps[kExtendA]);
    const T go_b = static_cast<T>(M.gaps[kOpenB]), ge_b = static_cast<T>(M.gaps[kExtendB]);
    std::vector<uint8_t> hops;
    if (pmax) {
        Hb<T, true> h{M.N, blk.data(), a, b, cutoff, go_a, ge_a, go_b, ge_b, {}};
        h.solve(0, m, 0, n, false, false);
        hops.swap(h.hops);
    } else {
        Hb<T, false> h{M.N, blk.data(), a, b, cutoff, go_a, ge_a, go_b, ge_b, {}};
        h.solve(0, m, 0, n, false, false);
        hops.swap(h.hops);
    }
    T s = T(0);
    int i = 0, j = 0;
    uint8_t prev = 3;
    std::vector<int32_t> gj(size_t(m) + 1, -1);
    gj[0] = 0;
    for (uint8_t op : hops) {
        if (op == 0) {
            ++i; ++j;
            s += blk[size_t(a[i - 1]) * M.N + b[j - 1]];
            if (o.grad) o.grad[size_t(a[i - 1]) * M.N + b[j - 1]] += 1.0;
            gj[i] = j;
        } else if (op == 1) {
            ++i;
            if (prev != 1) { s -= go_b; if (o.grad) o.grad[size_t(M.N) * M.N + kOpenB] -= 1.0; }
            s -= ge_b;
            if (o.grad) o.grad[size_t(M.N) * M.N + kExtendB] -= 1.0;
            gj[i] = j;
        } else {
            if (prev != 2) { s -= go_a; if (o.grad) o.grad[size_t(M.N) * M.N + kOpenA] -= 1.0; }
            s -= ge_a;
            if (o.grad) o.grad[size_t(M.N) * M.N + kExtendA] -= 1.0;
            ++j;
        }
        prev = op;
    }
    gj[m] = n;
    fill_guide_gaps(gj);
    if (o.guide) std::memcpy(o.guide, gj.data(), sizeof(int32_t) * (m + 1));
    if (o.moves) {
        const int64_t k = std::min<int64_t>(int64_t(hops.size()), o.moves_cap);
        for (int64_t q = 0; q < k; ++q) o.moves[q] = hops[q];
    }
    o.nmoves = int64_t(hops.size());
    o.score = static_cast<double>(s);
    o.end_i = m; o.end_j = n; o.start_i = 0; o.start_j = 0;
    return 0;
}


}  // namespace

// ── C ABI for the test suite (ctypes) ─────────────────────────────────────────
extern "C" {

// A batch of pairs.  a / b: concatenated codes, oa / ob: n_pairs + 1 offsets.
// tracks: concatenated per-residue sets of A (oa offsets) or null; gtracks: per DP row
// (oa[p] + p offsets, m + 1 each) or null.  tracked: whether the batch is tracked (tracks
// given or K > 1).  grads: n_pairs * (K*N*N + 4*K), zeroed here.  guides: (oa[p] + p)
// offsets, m + 1 each, or null.  moves (optional): per pair moves_cap bytes, walk order.
// band >= 0 with guides_in: the guide-banded DP.  prec: 32 float, 64 double.
int orc_hard_batch(int prec, int gm, int am, int N, int K, const double* mat, const double* gaps,
                   const uint8_t* a, const int64_t* oa, const uint8_t* b, const int64_t* ob,
                   int64_t n_pairs, const uint16_t* tracks, const uint16_t* gtracks, int tracked,
                   const int32_t* guides_in, int band,
                   double* scores, double* grads, int32_t* guides,
                   uint8_t* moves, int64_t moves_cap, int64_t* nmoves, int32_t* ends, int free_ends) {
    Model M{gm, am, N, K, mat, gaps, free_ends};
    const size_t gs = size_t(K) * N * N + 4 * size_t(K);
    for (int64_t p = 0; p < n_pairs; ++p) {
        const int m = int(oa[p + 1] - oa[p]), n = int(ob[p + 1] - ob[p]);
        HardOut o;
        o.grad = grads ? grads + gs * p : nullptr;
        if (o.grad) std::fill(o.grad, o.grad + gs, 0.0);
        o.guide = guides ? guides + oa[p] + p : nullptr;
        o.moves = moves ? moves + moves_cap * p : nullptr;
        const uint16_t* tk = tracks ? tracks + oa[p] : nullptr;
        const uint16_t* gk = gtracks ? gtracks + oa[p] + p : nullptr;
        const int32_t* gi = guides_in ? guides_in + oa[p] + p : nullptr;
        if (prec == 32)
            hard_one<float>(M, a + oa[p], m, b + ob[p], n, tk, gk, tracked != 0, gi, band, o, moves_cap);
        else
            hard_one<double>(M, a + oa[p], m, b + ob[p], n, tk, gk, tracked != 0, gi, band, o, moves_cap);
        scores[p] = o.score;
        if (nmoves) nmoves[p] = o.nmoves;
        if (ends) {
            ends[4 * p] = o.end_i; ends[4 * p + 1] = o.end_j;
            ends[4 * p + 2] = o.start_i; ends[4 * p + 3] = o.start_j;
        }
    }
    return 0;
}

// Soft gradient in log space, double, at temperature T: scores = T * log Z(theta/T),
// grads = expected counts under theta/T (gap fields negative).
// guides_in (oa[p] + p offsets, m + 1 each) with band >= 0: the guide-banded forward-backward.
int orc_soft_batch(int gm, int am, int N, int K, const double* mat, const double* gaps,
                   const uint8_t* a, const int64_t* oa, const uint8_t* b, const int64_t* ob,
                   int64_t n_pairs, const uint16_t* tracks, const uint16_t* gtracks,
                   double temperature, double* scores, double* grads, const int32_t* guides_in, int band,
                   int free_ends, int32_t* post_out) {
    Model M{gm, am, N, K, mat, gaps, free_ends};
    const size_t gs = size_t(K) * N * N + 4 * size_t(K);
    for (int64_t p = 0; p < n_pairs; ++p) {
        const int m = int(oa[p + 1] - oa[p]), n = int(ob[p + 1] - ob[p]);
        SoftOut o;
        o.grad = grads + gs * p;
        std::fill(o.grad, o.grad + gs, 0.0);
        o.post = post_out ? post_out + oa[p] + p : nullptr;
        const uint16_t* tk = tracks ? tracks + oa[p] : nullptr;
        const uint16_t* gk = gtracks ? gtracks + oa[p] + p : nullptr;
        Band bd; bd.m = m; bd.n = n; bd.global = am == 0;
        if (guides_in && band >= 0) { bd.band = band; bd.g = guides_in + oa[p] + p; }
        if (gm == 0) soft_linear(M, a + oa[p], m, b + ob[p], n, tk, gk, temperature, o, bd);
        else         soft_affine(M, a + oa[p], m, b + ob[p], n, tk, gk, temperature, o, bd);
        scores[p] = o.logz;
    }
    return 0;
}

// Hirschberg (affine Global, untracked, K = 1): pairs longer than `cutoff` rows split,
// the rest run the Pointers path.  pmax: the closed-form horizontal carry.  Outputs as
// orc_hard_batch (moves in path order, start to end).
int orc_hb_batch(int prec, int pmax, int cutoff, int N, const double* mat, const double* gaps,
                 const uint8_t* a, const int64_t* oa, const uint8_t* b, const int64_t* ob, int64_t n_pairs,
                 double* scores, double* grads, int32_t* guides, uint8_t* moves, int64_t moves_cap,
                 int64_t* nmoves, int local, int32_t* ends, int linear, int K, const uint16_t* tracks,
                 const uint16_t* gtracks) {
    K = std::max(K, 1);
    Model M{linear ? 0 : 1, local ? 1 : 0, N, K, mat, gaps};
    const bool tracked = tracks != nullptr || gtracks != nullptr || K > 1;
    const size_t gs = size_t(K) * N * N + 4 * size_t(K);
    for (int64_t p = 0; p < n_pairs; ++p) {
        const int m = int(oa[p + 1] - oa[p]), n = int(ob[p + 1] - ob[p]);
        HardOut o;
        o.grad = grads ? grads + gs * p : nullptr;
        if (o.grad) std::fill(o.grad, o.grad + gs, 0.0);
        o.guide = guides ? guides + oa[p] + p : nullptr;
        o.moves = moves ? moves + moves_cap * p : nullptr;
        o.moves_cap = moves_cap;
        if (linear) {
            const uint16_t* tk = tracks ? tracks + oa[p] : nullptr;
            const uint16_t* gk = gtracks ? gtracks + oa[p] + p : nullptr;
            if (prec == 32) lhb_one<float>(M, a + oa[p], m, b + ob[p], n, tk, gk, tracked, cutoff, o);
            else            lhb_one<double>(M, a + oa[p], m, b + ob[p], n, tk, gk, tracked, cutoff, o);
        } else if (local) {
            if (prec == 32) hb_local_one<float>(M, a + oa[p], m, b + ob[p], n, cutoff, pmax != 0, o);
            else            hb_local_one<double>(M, a + oa[p], m, b + ob[p], n, cutoff, pmax != 0, o);
        } else {
            if (prec == 32) hb_one<float>(M, a + oa[p], m, b + ob[p], n, cutoff, pmax != 0, o);
            else            hb_one<double>(M, a + oa[p], m, b + ob[p], n, cutoff, pmax != 0, o);
        }
        scores[p] = o.score;
        if (nmoves) nmoves[p] = o.nmoves;
        if (ends) { ends[4 * p] = o.start_i; ends[4 * p + 1] = o.start_j; ends[4 * p + 2] = o.end_i; ends[4 * p + 3] = o.end_j; }
    }
    return 0;
}

// sum_p w[p] * g[p] in blocks of 4096 pairs: each block from 0.0 in pair order, then the
// blocks in order (batch_engine.hpp:1788-1827).  w null: weights of one.
int orc_blocked_sum(const double* g, int64_t n_pairs, int64_t gs, const double* w, double* out) {
    const int64_t B = 4096;
    for (int64_t k = 0; k < gs; ++k) out[k] = 0.0;
    std::vector<double> acc(gs);
    for (int64_t b0 = 0; b0 < n_pairs; b0 += B) {
        std::fill(acc.begin(), acc.end(), 0.0);
        const int64_t e = std::min(n_pairs, b0 + B);
        for (int64_t p = b0; p < e; ++p)
            for (int64_t k = 0; k < gs; ++k) {
                const double v = w ? w[p] * g[p * gs + k] : g[p * gs + k];
                acc[k] += v;
            }
        for (int64_t k = 0; k < gs; ++k) out[k] += acc[k];
    }
    return 0;
}

}  // extern "C"
