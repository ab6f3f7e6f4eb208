// Soft path: scaled-probability forward-backward with the expected counts fused into the
// backward pass.
//
// Definition (the reference's log-space recurrences, aligner.hpp:6231-6524, in probability
// space): forward F over DP rows 0..m and columns 0..n with M(0,0) = 1 (Global) or a free
// start of weight 1 at every M cell (Local); X(i,j) = (M + Y)(i-1,j) o_b(i) + X(i-1,j) e_b(i),
// Y(i,j) = (M + X)(i,j-1) o_a(i) + Y(i,j-1) e_a(i), M(i,j) = (M+X+Y)(i-1,j-1) w(a_i, b_j),
// with o = exp(-(go+ge)/T), e = exp(-ge/T), w = exp(s/T); Local has no gap move into a border
// cell.  Z = (M+X+Y)(m,n) (Global) or the sum over every cell (Local); backward B the mirror
// recurrence seeded with 1 at (m,n) (Global) or at every cell (Local).  The expected count
// of a transition out of cell c into c' is F(c) trans B(c') / Z, so the backward pass, which
// forms exactly the products trans * B(c') to build B(c), adds F(c) times them to the counts.
// Linear gaps are the one-state case (o = e).
//
// Layout: the hard kernel's lane strips (nwg_hard.cuh), here over rows 0..m and columns
// 0..n.  Range: every lane keeps its own power-of-two exponent, renormalised after each
// step so its largest value lies in [1, 2); values crossing lanes are converted by exact
// power-of-two factors.  The forward values of every cell (3 per cell, scaled, plus one
// exponent per lane step) go to a per-group scratch table that the backward pass reads in
// reverse.  A value that overflows or turns NaN marks the pair refused; the host reruns
// refused pairs in double precision.  Sums of exponentials and the gradient's gap fields
// accumulate in double; substitution counts in a per-group shared-memory histogram.
#pragma once
#include "nwg_common.cuh"

namespace nwg {

struct SoftArgs {
    const uint8_t* a; const int64_t* oa;
    const uint8_t* b; const int64_t* ob;
    const uint16_t* tracks; const uint16_t* gtracks;
    const int32_t* order; int64_t n_items;
    const void* w;       // weights, (K*N + 1) rows x (N + 1) columns in T; row K*N and column N are 0
    const void* gw;      // per set: o_a, e_a, o_b, e_b in T
    int N, K;
    void* scratch; int64_t scratch_stride;   // bytes per group slot
    int64_t fwd_bytes;                       // bytes of the forward table within a slot
    int maxn;                                // columns (n) the boundary rows are sized for
    double temperature;
    double* score; double* grad; int64_t gstride;
    int32_t* status;                         // per pair: 0 ok, 1 refused (out of range)
};

// Double accumulator with its own binary exponent: value = m * 2^e.
struct XAcc {
    double m; int e;
    __device__ __forceinline__ void init() { m = 0.0; e = -100000; }
    __device__ __forceinline__ void add(double x, int ex) {
        if (!(x > 0.0)) return;
        if (m == 0.0) { m = x; e = ex; return; }
        if (ex > e) { m = m * pow2i<double>(e - ex) + x; e = ex; }
        else m += x * pow2i<double>(ex - e);
    }
};

template <class T, bool AFF, bool LOC, bool TR, int G, int R>
__global__ void __launch_bounds__(128) soft_kernel(const SoftArgs A) {
    constexpr int GR = G * R;
    constexpr int NV = AFF ? 3 : 1;          // values per cell
    const int N = A.N, K = A.K;
    const int wcols = N + 1;
    const int nw = (K * N + 1) * wcols;
    const int gpb = blockDim.x / G;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sw = reinterpret_cast<T*>(smem_raw);
    T* sgw = sw + nw;
    // per group: the substitution-count histogram (K*N*N T) and tracked gap sums (4K double)
    const int hsz = K * N * N;
    unsigned char* after = reinterpret_cast<unsigned char*>(sgw + 4 * K);
    after = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(after) + 15) & ~uintptr_t(15));
    double* sgap_all = reinterpret_cast<double*>(after);
    T* hist_all = reinterpret_cast<T*>(sgap_all + (TR ? 4 * K * gpb : 0));
    for (int k = threadIdx.x; k < nw; k += blockDim.x) sw[k] = static_cast<const T*>(A.w)[k];
    for (int k = threadIdx.x; k < 4 * K; k += blockDim.x) sgw[k] = static_cast<const T*>(A.gw)[k];

    const int lane = threadIdx.x % G;
    const int gib = threadIdx.x / G;
    const int64_t slot = int64_t(blockIdx.x) * gpb + gib;
    T* hist = hist_all + int64_t(gib) * hsz;
    double* sgap = sgap_all + 4 * K * gib;
    for (int k = lane; k < hsz; k += G) hist[k] = T(0);
    if (TR) for (int k = lane; k < 4 * K; k += G) sgap[k] = 0.0;
    __syncthreads();

    unsigned gmask;
    if constexpr (G == 32) gmask = 0xffffffffu;
    else gmask = ((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1));

    unsigned char* sbase = static_cast<unsigned char*>(A.scratch) + slot * A.scratch_stride;
    T* fwd = reinterpret_cast<T*>(sbase);
    int* fexp = reinterpret_cast<int*>(sbase + A.fwd_bytes);
    // boundary rows: forward (values, exponent) and backward, (maxn + 1) columns each
    const int64_t nb = int64_t(A.maxn) + 1;
    unsigned char* bb = sbase + A.scratch_stride - nb * (2 * NV * sizeof(T) + 2 * sizeof(int));
    T* fbnd = reinterpret_cast<T*>(bb);
    T* bbnd = fbnd + NV * nb;
    int* fbndE = reinterpret_cast<int*>(bbnd + NV * nb);
    int* bbndE = fbndE + nb;

    for (int64_t it = slot; it < A.n_items; it += int64_t(gridDim.x) * gpb) {
        const int p = A.order[it];
        const int64_t ao = A.oa[p], bo = A.ob[p];
        const int m = int(A.oa[p + 1] - ao), n = int(A.ob[p + 1] - bo);
        const uint8_t* __restrict__ ap = A.a + ao;
        const uint8_t* __restrict__ bp = A.b + bo;
        const uint16_t* tk = TR ? A.tracks + ao : nullptr;
        const uint16_t* gk = (TR && A.gtracks) ? A.gtracks + ao + p : nullptr;
        auto tset = [&](int i) -> int { return TR ? int(tk[i - 1]) : 0; };
        auto gset = [&](int i) -> int {
            if constexpr (!TR) return 0;
            if (gk) return int(gk[i]);
            return i == 0 ? (m ? int(tk[0]) : 0) : int(tk[i - 1]);
        };
        const int rows = m + 1;                 // DP rows 0..m
        const int nstripes = (rows + GR - 1) / GR;
        const int S = n + G;                    // steps: columns 0..n plus the skew
        const T one = T(1);
        bool bad = false;

        // ── forward ──────────────────────────────────────────────────────────
        XAcc zacc; zacc.init();                 // Local: the sum over every cell
        T zM = T(0), zX = T(0), zY = T(0); int zE = 0;   // Global: (m, n)
        for (int s = 0; s < nstripes; ++s) {
            const int i0 = s * GR + lane * R;   // this lane's first DP row (0-based rows incl. row 0)
            int key[R];
            T roa[R], rea[R], rob[R], reb[R];
            T cM[R], cX[R], cY[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = i0 + r;
                const bool valid = i <= m;
                key[r] = (valid && i >= 1) ? (tset(i) * N + ap[i - 1]) * wcols : K * N * wcols;
                const int gs = valid ? gset(i) : 0;
                const int ts = (valid && i >= 1) ? tset(i) : 0;
                roa[r] = sgw[4 * gs + 0]; rea[r] = sgw[4 * gs + 1];
                rob[r] = sgw[4 * ts + 2]; reb[r] = sgw[4 * ts + 3];
                cM[r] = T(0); cX[r] = T(0); cY[r] = T(0);
            }
            int E = 0;
            T lone = one;                         // 2^-E
            T dgM = T(0), dgX = T(0), dgY = T(0); // row above, column j-1 (column -1: 0)
            T upM = T(0), upX = T(0), upY = T(0);
            T* fs = fwd + int64_t(s) * S * G * (NV * R);
            int* fe = fexp + int64_t(s) * S * G;
            for (int t = 0; t < S; ++t) {
                const int j = t - lane;           // column 0..n
                if (lane == 0 && j <= n) {
                    if (s == 0) { upM = T(0); upX = T(0); upY = T(0); }
                    else {
                        const int eb = fbndE[j];
                        const int d = eb - E;
                        if (d > 100) {   // keep the incoming values in range: rescale own state down
                            const T f = pow2i<T>(100 - d);
#pragma unroll
                            for (int r = 0; r < R; ++r) { cM[r] *= f; cX[r] *= f; cY[r] *= f; }
                            dgM *= f; dgX *= f; dgY *= f;
                            E = eb - 100; lone = pow2i<T>(-E);
                        }
                        const T f = pow2i<T>(eb - E);
                        upM = fbnd[NV * j] * f;
                        if constexpr (AFF) { upX = fbnd[NV * j + 1] * f; upY = fbnd[NV * j + 2] * f; }
                    }
                }
                const bool active = (j >= 0) && (j <= n);
                if (active) {
                    const int bj = j >= 1 ? int(bp[j - 1]) : N;   // column 0: the zero column
                    T pM = dgM, pX = dgX, pY = dgY;
                    T qM = upM, qX = upX, qY = upY;
                    T mx = T(0);
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const int i = i0 + r;
                        const T wv = sw[key[r] + bj];
                        T fm, fx = T(0), fy = T(0);
                        if constexpr (AFF) {
                            fm = (pM + pX + pY) * wv;
                            fx = (qM + qY) * rob[r] + qX * reb[r];
                            fy = (cM[r] + cX[r]) * roa[r] + cY[r] * rea[r];
                            if constexpr (LOC) {
                                fm += lone;
                                if (j == 0) fx = T(0);
                                if (i == 0) fy = T(0);
                            } else {
                                if (i == 0 && j == 0) fm = lone;
                            }
                        } else {
                            fm = pM * wv + qM * reb[r] + cM[r] * rea[r];
                            if constexpr (LOC) {
                                if (i == 0 || j == 0) fm = T(0);
                                fm += lone;
                            } else {
                                if (i == 0 && j == 0) fm = lone;
                            }
                        }
                        if (i > m) { fm = T(0); fx = T(0); fy = T(0); }
                        pM = cM[r]; pX = cX[r]; pY = cY[r];
                        cM[r] = fm; cX[r] = fx; cY[r] = fy;
                        qM = fm; qX = fx; qY = fy;
                        mx = rmax(mx, rmax3(fm, fx, fy));
                    }
                    dgM = upM; dgX = upX; dgY = upY;
                    // renormalise: the lane's largest value into [1, 2)
                    if (!is_finite(mx)) bad = true;
                    else if (mx > T(0)) {
                        int e = ilog2(mx);
                        if (e < -120) e = -120;
                        if (e != 0) {
                            const T f = pow2i<T>(-e);
#pragma unroll
                            for (int r = 0; r < R; ++r) { cM[r] *= f; cX[r] *= f; cY[r] *= f; }
                            dgM *= f; dgX *= f; dgY *= f;
                            E += e; lone = pow2i<T>(-E);
                        }
                    }
                    // store the column for the backward pass
                    T* dst = fs + (int64_t(t) * G + lane) * (NV * R);
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        dst[NV * r] = cM[r];
                        if constexpr (AFF) { dst[NV * r + 1] = cX[r]; dst[NV * r + 2] = cY[r]; }
                    }
                    fe[int64_t(t) * G + lane] = E;
                    if constexpr (LOC) {
                        T cs = T(0);
#pragma unroll
                        for (int r = 0; r < R; ++r) cs += (cM[r] + cX[r]) + cY[r];
                        zacc.add(static_cast<double>(cs), E);
                    }
                }
                if constexpr (G > 1) {
                    const T sM = __shfl_up_sync(gmask, cM[R - 1], 1, G);
                    T sX = sM, sY = sM;
                    if constexpr (AFF) {
                        sX = __shfl_up_sync(gmask, cX[R - 1], 1, G);
                        sY = __shfl_up_sync(gmask, cY[R - 1], 1, G);
                    }
                    const int sE = __shfl_up_sync(gmask, E, 1, G);
                    if (lane > 0) {
                        int d = sE - E;
                        if (d > 100) {
                            const T f = pow2i<T>(100 - d);
#pragma unroll
                            for (int r = 0; r < R; ++r) { cM[r] *= f; cX[r] *= f; cY[r] *= f; }
                            dgM *= f; dgX *= f; dgY *= f;
                            E = sE - 100; lone = pow2i<T>(-E);
                            d = 100;
                        }
                        const T f = pow2i<T>(d);
                        upM = sM * f; upX = sX * f; upY = sY * f;
                    }
                }
                if (lane == G - 1 && active && s + 1 < nstripes) {
                    fbnd[NV * j] = cM[R - 1];
                    if constexpr (AFF) { fbnd[NV * j + 1] = cX[R - 1]; fbnd[NV * j + 2] = cY[R - 1]; }
                    fbndE[j] = E;
                }
            }
            if constexpr (!LOC) {
                if (m >= i0 && m < i0 + R) {
#pragma unroll
                    for (int r = 0; r < R; ++r)
                        if (i0 + r == m) { zM = cM[r]; zX = cX[r]; zY = cY[r]; zE = E; }
                }
            }
            if constexpr (G > 1) __syncwarp(gmask);
        }
        // Z = zhat * 2^EZ with zhat in [1, 2)
        double zm; int ze;
        if constexpr (LOC) {
            if constexpr (G > 1) {
#pragma unroll
                for (int off = 1; off < G; off <<= 1) {
                    const double om = __shfl_xor_sync(gmask, zacc.m, off, G);
                    const int oe = __shfl_xor_sync(gmask, zacc.e, off, G);
                    zacc.add(om, oe);
                }
            }
            zm = zacc.m; ze = zacc.e;
            if constexpr (G > 1) {   // one value for the whole group (lanes summed in different orders)
                zm = __shfl_sync(gmask, zm, 0, G);
                ze = __shfl_sync(gmask, ze, 0, G);
            }
        } else {
            zm = static_cast<double>((zM + zX) + zY); ze = zE;
            if constexpr (G > 1) {
                const int src = (m % GR) / R;
                zm = __shfl_sync(gmask, zm, src, G);
                ze = __shfl_sync(gmask, ze, src, G);
            }
        }
        if constexpr (G > 1) bad = __any_sync(gmask, bad);
        if (!(zm > 0.0) || !(zm < 1e300) || bad) {
            if (lane == 0) { A.status[p] = 1; A.score[p] = 0.0; }
            continue;
        }
        const int EZ = ze + ilog2(zm);
        const double zhat = zm * pow2i<double>(ze - EZ);
        const double invz = 1.0 / zhat;

        // ── backward, fused with the expected counts ─────────────────────────
        double ga_o = 0, ga_e = 0, gb_o = 0, gb_e = 0;   // untracked gap sums (scaled counts)
        for (int s = nstripes - 1; s >= 0; --s) {
            const int i0 = s * GR + lane * R;
            int keyd[R], hrow[R];
            T roa[R], rea[R], rob[R], reb[R];      // rob/reb: the row BELOW (i+1)
            int gsr[R], tsd[R];
            T bM[R], bX[R], bY[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = i0 + r;
                const bool valid = i <= m;
                const int gs = valid ? gset(i) : 0;
                const int td = (i + 1 <= m) ? tset(i + 1) : 0;
                gsr[r] = gs; tsd[r] = td;
                const int kd = (i + 1 <= m) ? (td * N + ap[i]) : K * N;
                keyd[r] = kd * wcols;
                hrow[r] = kd * N;
                roa[r] = sgw[4 * gs + 0]; rea[r] = sgw[4 * gs + 1];
                rob[r] = sgw[4 * td + 2]; reb[r] = sgw[4 * td + 3];
                bM[r] = T(0); bX[r] = T(0); bY[r] = T(0);
            }
            int EB = 0;
            T lone = one;
            T dgM = T(0);                             // row below, column j+1 (BM only)
            T dnM = T(0), dnX = T(0), dnY = T(0);     // row below, column j
            const T* fs = fwd + int64_t(s) * S * G * (NV * R);
            const int* fe = fexp + int64_t(s) * S * G;
            for (int t = 0; t < S; ++t) {
                const int j = n - t + (G - 1 - lane);     // column n..0
                if (lane == G - 1 && j >= 0) {
                    if (s == nstripes - 1) { dnM = T(0); dnX = T(0); dnY = T(0); }
                    else {
                        const int eb = bbndE[j];
                        int d = eb - EB;
                        if (d > 100) {
                            const T f = pow2i<T>(100 - d);
#pragma unroll
                            for (int r = 0; r < R; ++r) { bM[r] *= f; bX[r] *= f; bY[r] *= f; }
                            dgM *= f;
                            EB = eb - 100; lone = pow2i<T>(-EB);
                            d = 100;
                        }
                        const T f = pow2i<T>(d);
                        dnM = bbnd[NV * j] * f;
                        if constexpr (AFF) { dnX = bbnd[NV * j + 1] * f; dnY = bbnd[NV * j + 2] * f; }
                        else { dnX = dnM; dnY = dnM; }
                    }
                }
                const bool active = (j >= 0) && (j <= n);
                if (active) {
                    const int bj1 = j < n ? int(bp[j]) : N;   // b code of column j+1
                    const T* src = fs + (int64_t(j + lane) * G + lane) * (NV * R);
                    const int EF = fe[int64_t(j + lane) * G + lane];
                    T dM = dgM;                  // row below, column j+1
                    T xM = dnM, xX = dnX, xY = dnY;   // row below, column j
                    T sgo_a = T(0), sge_a = T(0), sgo_b = T(0), sge_b = T(0);
                    // scale of this step's products: 2^(EF + EB - EZ) / zhat
                    const double facd = pow2i<double>(EF + EB - EZ) * invz;
                    const T fac = static_cast<T>(facd);
                    if (!is_finite(fac)) bad = true;
                    T mx = T(0);
#pragma unroll
                    for (int r = R - 1; r >= 0; --r) {
                        const int i = i0 + r;
                        const T wv = sw[keyd[r] + bj1];
                        const T fm = src[NV * r];
                        T fx = T(0), fy = T(0);
                        if constexpr (AFF) { fx = src[NV * r + 1]; fy = src[NV * r + 2]; }
                        const T D = wv * dM;
                        T nM, nX, nY;
                        if constexpr (AFF) {
                            T tX = rob[r] * xX, eX = reb[r] * xX;
                            T tY = roa[r] * bY[r], eY = rea[r] * bY[r];
                            if constexpr (LOC) {
                                if (j == 0) { tX = T(0); eX = T(0); }
                                if (i == 0) { tY = T(0); eY = T(0); }
                            }
                            nM = D + tX + tY; nX = D + eX + tY; nY = D + tX + eY;
                            if constexpr (LOC) { nM += lone; nX += lone; nY += lone; }
                            else if (i == m && j == n) { nM = lone; nX = lone; nY = lone; }
                            // counts of the moves out of (i, j)
                            const T fsum = (fm + fx) + fy;
                            if (i < m && j < n) {
                                const T c = fsum * D * fac;
                                atomicAdd(&hist[hrow[r] + bj1], c);
                            }
                            const T oX = (fm + fy) * tX, xx = fx * eX;
                            const T oY = (fm + fx) * tY, yy = fy * eY;
                            if constexpr (TR) {
                                if (i < m) {
                                    const double ob = static_cast<double>(oX) * facd;
                                    atomicAdd(&sgap[4 * tsd[r] + 2], ob);
                                    atomicAdd(&sgap[4 * tsd[r] + 3], ob + static_cast<double>(xx) * facd);
                                }
                                if (i <= m) {
                                    const double oa = static_cast<double>(oY) * facd;
                                    atomicAdd(&sgap[4 * gsr[r] + 0], oa);
                                    atomicAdd(&sgap[4 * gsr[r] + 1], oa + static_cast<double>(yy) * facd);
                                }
                            } else {
                                if (i < m) { sgo_b += oX; sge_b += oX + xx; }
                                if (i <= m) { sgo_a += oY; sge_a += oY + yy; }
                            }
                        } else {
                            T tX = reb[r] * xM;
                            T tY = rea[r] * bM[r];
                            if constexpr (LOC) {
                                if (j == 0) tX = T(0);
                                if (i == 0) tY = T(0);
                            }
                            nM = D + tX + tY;
                            if constexpr (LOC) nM += lone;
                            else if (i == m && j == n) nM = lone;
                            nX = nM; nY = nM;
                            if (i < m && j < n) atomicAdd(&hist[hrow[r] + bj1], fm * D * fac);
                            if constexpr (TR) {
                                if (i < m) atomicAdd(&sgap[4 * tsd[r] + 3], static_cast<double>(fm * tX) * facd);
                                if (i <= m) atomicAdd(&sgap[4 * gsr[r] + 1], static_cast<double>(fm * tY) * facd);
                            } else {
                                if (i < m) sge_b += fm * tX;
                                if (i <= m) sge_a += fm * tY;
                            }
                        }
                        if (i > m) { nM = T(0); nX = T(0); nY = T(0); }
                        dM = bM[r];
                        bM[r] = nM; bX[r] = nX; bY[r] = nY;
                        xM = nM; xX = nX; xY = nY;
                        mx = rmax(mx, rmax3(nM, nX, nY));
                    }
                    if constexpr (!TR) {
                        ga_o += static_cast<double>(sgo_a) * facd; ga_e += static_cast<double>(sge_a) * facd;
                        gb_o += static_cast<double>(sgo_b) * facd; gb_e += static_cast<double>(sge_b) * facd;
                    }
                    dgM = dnM;
                    if (!is_finite(mx)) bad = true;
                    else if (mx > T(0)) {
                        int e = ilog2(mx);
                        if (e < -120) e = -120;
                        if (e != 0) {
                            const T f = pow2i<T>(-e);
#pragma unroll
                            for (int r = 0; r < R; ++r) { bM[r] *= f; bX[r] *= f; bY[r] *= f; }
                            dgM *= f;
                            EB += e; lone = pow2i<T>(-EB);
                        }
                    }
                }
                if constexpr (G > 1) {
                    const T sM = __shfl_down_sync(gmask, bM[0], 1, G);
                    T sX = sM, sY = sM;
                    if constexpr (AFF) {
                        sX = __shfl_down_sync(gmask, bX[0], 1, G);
                        sY = __shfl_down_sync(gmask, bY[0], 1, G);
                    }
                    const int sE = __shfl_down_sync(gmask, EB, 1, G);
                    if (lane < G - 1) {
                        int d = sE - EB;
                        if (d > 100) {
                            const T f = pow2i<T>(100 - d);
#pragma unroll
                            for (int r = 0; r < R; ++r) { bM[r] *= f; bX[r] *= f; bY[r] *= f; }
                            dgM *= f;
                            EB = sE - 100; lone = pow2i<T>(-EB);
                            d = 100;
                        }
                        const T f = pow2i<T>(d);
                        dnM = sM * f; dnX = sX * f; dnY = sY * f;
                    }
                }
                if (lane == 0 && active && s > 0) {
                    bbnd[NV * j] = bM[0];
                    if constexpr (AFF) { bbnd[NV * j + 1] = bX[0]; bbnd[NV * j + 2] = bY[0]; }
                    bbndE[j] = EB;
                }
            }
            if constexpr (G > 1) __syncwarp(gmask);
        }
        if constexpr (G > 1) bad = __any_sync(gmask, bad);
        // reduce the untracked gap sums over the group and write the pair's results
        if constexpr (!TR && G > 1) {
#pragma unroll
            for (int off = G / 2; off > 0; off >>= 1) {
                ga_o += __shfl_xor_sync(gmask, ga_o, off, G);
                ga_e += __shfl_xor_sync(gmask, ga_e, off, G);
                gb_o += __shfl_xor_sync(gmask, gb_o, off, G);
                gb_e += __shfl_xor_sync(gmask, gb_e, off, G);
            }
        }
        if constexpr (G > 1) __syncwarp(gmask);
        double* g = A.grad + A.gstride * p;
        const int64_t NN = int64_t(K) * N * N;
        if (bad) {
            if (lane == 0) { A.status[p] = 1; A.score[p] = 0.0; }
        } else {
            for (int k = lane; k < hsz; k += G) g[k] = static_cast<double>(hist[k]);
            if constexpr (TR) {
                for (int k = lane; k < 4 * K; k += G) g[NN + k] = -sgap[k];
            } else {
                for (int k = lane; k < 4 * K; k += G) g[NN + k] = 0.0;
                if (lane == 0) {
                    g[NN + 0] = -ga_o; g[NN + 1] = -ga_e; g[NN + 2] = -gb_o; g[NN + 3] = -gb_e;
                }
            }
            if (lane == 0) {
                A.status[p] = 0;
                A.score[p] = A.temperature * (log(zhat) + double(EZ) * 0.69314718055994530942);
            }
        }
        if constexpr (G > 1) __syncwarp(gmask);
        for (int k = lane; k < hsz; k += G) hist[k] = T(0);
        if (TR) for (int k = lane; k < 4 * K; k += G) sgap[k] = 0.0;
        if constexpr (G > 1) __syncwarp(gmask);
    }
}

}  // namespace nwg
