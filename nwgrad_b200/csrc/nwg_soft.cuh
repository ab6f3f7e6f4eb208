// Soft path: scaled-probability forward-backward with the expected counts fused into the
// backward pass.
//
// Definition (the reference's log-space recurrences, aligner.hpp:6231-6524, in probability
// space): forward F over DP rows 0..m and columns 0..n with M(0,0) = 1 (Global) or a free
// start of weight 1 at every M cell (Local); X(i,j) = (M + Y)(i-1,j) o_b(i) + X(i-1,j) e_b(i),
// Y(i,j) = (M + X)(i,j-1) o_a(i) + Y(i,j-1) e_a(i), M(i,j) = (M+X+Y)(i-1,j-1) w(a_i, b_j),
// with o = exp(-(go+ge)/T), e = exp(-ge/T), w = exp(s/T); Local has no gap move into a border
// cell.  Z = (M+X+Y)(m,n) (Global) or the sum over every cell (Local); backward B the mirror
// recurrence seeded with 1 at (m,n) (Global) or at every cell (Local).  Semi-global ends
// (`ends`, Global kernels): free starts of weight 1 on row 0 / column 0, and Z and the seeds
// over the end cells.  The expected count
// of a transition out of cell c into c' is F(c) trans B(c') / Z, so the backward pass, which
// forms exactly the products trans * B(c') to build B(c), adds F(c) times them to the counts.
// Linear gaps are the one-state case (o = e).
//
// Layout: the hard kernel's lane strips (nwg_hard.cuh), here over rows 0..m and columns
// 0..n.  Range: every lane keeps its own power-of-two exponent and renormalises its values
// every `renorm` steps (the host picks the period so that no value can overflow in
// between: growth per step is at most 3 * the largest weight); values crossing lanes are
// converted by exact power-of-two factors.  The forward values of every cell (3 per cell,
// scaled, plus one exponent per lane step) go to a per-group scratch table that the backward
// pass reads in reverse.  Checkpointed (long pairs): the forward pass keeps only each
// stripe's bottom row; the backward pass recomputes one stripe's table from the row above it
// just before it walks that stripe, so the table holds one stripe (twice the forward work,
// a table ~nstripes times smaller).  A value that overflows or turns NaN marks the pair refused; the
// host reruns refused pairs in double precision.
//
// Accumulation: each lane keeps its rows' substitution counts in shared memory, laid out
// [b][lane][row] so one step's R rows update one contiguous R-vector (one 128-bit load and
// store for R = 4) without conflicts; they are folded into the pair's histogram at the end
// of every stripe.  Gap counts (untracked) accumulate in T per lane and stripe and per pair in
// double; tracked gap counts per parameter set in shared memory (double).  log Z is formed in
// double; the per-step scale factor 2^(E_F + E_B - E_Z) / Z is an exact power of two times
// 1 / zhat in T.
#pragma once
#include "nwg_common.cuh"

namespace nwg {

struct SoftArgs {
    const uint8_t* a; const int64_t* oa;
    const uint8_t* b; const int64_t* ob;
    const uint16_t* tracks; const uint16_t* gtracks;
    const int32_t* order; int64_t n_items;
    const void* w;       // weights, (K*N + 1) rows x (N + 1) columns in T; row K*N and column N
                         // are 0 but for w[K*N][N] = 1, which carries the Global corner seed
    const void* gw;      // per set: o_a, e_a, o_b, e_b in T; then the float32 lost-mass charge per
                         // unit of F^ + B^ (16 + 16 wmax), so a parameter step changes no argument
    int N, K;
    void* scratch; int64_t scratch_stride;   // bytes per group slot
    int64_t fwd_bytes;                       // bytes of the forward table within a slot
    int maxn;                                // columns (n) the boundary rows are sized for
    int ck;                                  // checkpointed: keep every stripe's bottom row in the
                                             // forward pass, recompute a stripe's table before its
                                             // backward (the table then holds one stripe)
    int max_stripes;                         // ck: stripes the boundary rows are sized for
    int64_t bnd_off;                         // bytes from a slot's start to its boundary rows
    int64_t warp_stride;                     // several warps per pair: bytes of one warp's table
                                             // and exponents (each warp recomputes its stripes)
    const int32_t* guide;                    // banded: per pair m + 1 guide columns at oa[p] + p
    int band;                                // banded: half-width
    int renorm_mask;                         // renormalise when (step & renorm_mask) == 0
    int ends;                                // Global kernels, full DP: semi-global free ends, 1 a_begin
                                             // (column 0 a free start), 2 a_end (column n's cells
                                             // ends), 4 b_begin (row 0 a free start), 8 b_end (row m's
                                             // cells ends); 0: Global's borders and end (m, n)
    double temperature;
    double* score; double* grad; int64_t gstride;
    int32_t* status;                         // per pair: 0 ok, else kSoft* bits (why it was refused)
    int spin_limit;                          // several warps per pair: polls before a wait gives up
    int* queue;                              // this launch's work-queue counters (2 ints, zero at launch)
    int32_t* post;                           // POST kernels: per pair m + 1 posterior guide columns at oa[p] + p
    // tiled long pairs (TL kernels): an item is one tile -- stripe s of pair p over columns
    // c W .. c W + W - 1 -- and a launch holds one anti-diagonal s + c of every pair's tiles, in
    // the forward phase (0) or, in reverse diagonal order, the backward phase (1)
    const int32_t* tiles;                    // per item: p, s, c
    int tile_w;                              // W, a multiple of 32
    int tl_phase;
    void* rowf; void* rowb;                  // per pair, per stripe: the forward bottom row and the
    const int64_t* row_off;                  // backward top row, (n + 1) x BW T; offset per pair in
                                             // columns (x BW: T)
    void* colf; void* colb;                  // per pair, per (stripe, tile): every lane's forward state
    const int64_t* col_off;                  // at the tile's last column / backward state at its first
                                             // (G x (NV R + 1) T, the exponent as T's bits); offset per
                                             // pair in lane states (x (NV R + 1): T)
    double* zpart; const int64_t* tile_off;  // Local: per tile its part of Z (m, e); offset per pair in tiles
    double* zpair;                           // per pair: Z as (m, e) once the forward phase is done
    double* spart; const int64_t* stripe_off;   // per pair, per stripe: its counts (gstride doubles)
                                                // and lost-mass charge (1 more), added tile by tile;
                                                // offset per pair in stripes
};

// Per-pair status bits of a soft pass: a refused pair's score and counts are not written and
// the host reruns it (float32 -> double).
constexpr int32_t kSoftRange = 1;    // a forward or backward value left T's range
constexpr int32_t kSoftZ = 2;        // Z is zero or out of range
constexpr int32_t kSoftScale = 4;    // a count's scale factor 2^(E_F + E_B - E_Z) / Z overflowed T
constexpr int32_t kSoftCounts = 8;   // a count left T's range
constexpr int32_t kSoftLoss = 16;    // float32: mass lost to underflow could move a posterior by > 2^-24
constexpr int32_t kSoftWeights = 32; // (host) a weight overflows T
constexpr int32_t kSoftStall = 64;   // several warps per pair: a wait ran out (the call fails)

// A lane receiving values whose largest lies more than 2^kLift above its own scale moves its
// own state down instead: incoming values then land below 2^(kLift + 1), which bounds the
// renormalisation period the host picks (nwg_capi.cu).
constexpr int kLift = 32;

// The exponent of a lane whose values are all zero: it carries no scale, so a neighbour
// receiving its zeros keeps its own exponent, and the lane itself takes the scale of the
// first non-zero values it receives (a zero lane with a stale exponent once pulled the
// neighbouring lane's state down to zero, or flushed the values it received).
constexpr int kEmpty = -(1 << 28);

// Float32 lost-mass bound.  With subnormals kept (no FTZ), a rounding whose result falls
// below FLT_MIN errs by at most 2^-150 in the lane's units; an error in a value that a weight
// then multiplies grows by that weight (at most wmax, the largest of the exp'd scores and gap
// weights), and mass lost at a cell moves a posterior (and Z) by at most that mass times
// B(c) / Z.  So, with fac = 2^(E_F + E_B - E_Z) / Z, the backward pass charges per lane and
// step fac * (loss_w * (sum F^ + sum B^) + 16 R) -- loss_w = 16 + 16 wmax roundings per state
// and cell, transfers and rescales included, 16 per row for the count products -- in units of
// 2^-150.  Where 2^(E_F + E_B - E_Z) falls below the normal range, the step's F^ move down
// into it (fac stays normal) and the step charges its B^ once more for the F^ that rounded on
// the way.  A pair whose charge exceeds kLossMax (damage 2^-24) is refused.
constexpr float kLossMax = 0x1p126f;

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

template <class T> __device__ __forceinline__ T tmax(T a, T b);
template <> __device__ __forceinline__ float tmax<float>(float a, float b) { return fmaxf(a, b); }
template <> __device__ __forceinline__ double tmax<double>(double a, double b) { return fmax(a, b); }

// Vector load / store of n values of T (n a multiple of 4 floats or 2 doubles when possible).
template <class T, int NV>
__device__ __forceinline__ void vstore(T* dst, const T (&v)[NV]) {
    if constexpr (sizeof(T) == 4 && NV % 4 == 0) {
#pragma unroll
        for (int k = 0; k < NV / 4; ++k)
            reinterpret_cast<float4*>(dst)[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
    } else if constexpr (sizeof(T) == 8 && NV % 2 == 0) {
#pragma unroll
        for (int k = 0; k < NV / 2; ++k)
            reinterpret_cast<double2*>(dst)[k] = make_double2(v[2 * k], v[2 * k + 1]);
    } else if constexpr (sizeof(T) == 4 && NV == 2) {
        *reinterpret_cast<float2*>(dst) = make_float2(v[0], v[1]);
    } else {
#pragma unroll
        for (int k = 0; k < NV; ++k) dst[k] = v[k];
    }
}
// The forward table: written once and read once much later -- stores stream past the caches
// (evict first), loads take the read-only path.
template <class T, int NV>
__device__ __forceinline__ void vstore_stream(T* dst, const T (&v)[NV]) {
    if constexpr (sizeof(T) == 4 && NV % 4 == 0) {
#pragma unroll
        for (int k = 0; k < NV / 4; ++k)
            __stcs(reinterpret_cast<float4*>(dst) + k, make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]));
    } else if constexpr (sizeof(T) == 8 && NV % 2 == 0) {
#pragma unroll
        for (int k = 0; k < NV / 2; ++k) __stcs(reinterpret_cast<double2*>(dst) + k, make_double2(v[2 * k], v[2 * k + 1]));
    } else {
#pragma unroll
        for (int k = 0; k < NV; ++k) __stcs(dst + k, v[k]);
    }
}
template <class T, int NV>
__device__ __forceinline__ void vload_ro(T (&v)[NV], const T* src) {
    if constexpr (sizeof(T) == 4 && NV % 4 == 0) {
#pragma unroll
        for (int k = 0; k < NV / 4; ++k) {
            const float4 q = __ldg(reinterpret_cast<const float4*>(src) + k);
            v[4 * k] = q.x; v[4 * k + 1] = q.y; v[4 * k + 2] = q.z; v[4 * k + 3] = q.w;
        }
    } else if constexpr (sizeof(T) == 8 && NV % 2 == 0) {
#pragma unroll
        for (int k = 0; k < NV / 2; ++k) {
            const double2 q = __ldg(reinterpret_cast<const double2*>(src) + k);
            v[2 * k] = q.x; v[2 * k + 1] = q.y;
        }
    } else {
#pragma unroll
        for (int k = 0; k < NV; ++k) v[k] = __ldg(src + k);
    }
}
template <class T, int NV>
__device__ __forceinline__ void vload(T (&v)[NV], const T* src) {
    if constexpr (sizeof(T) == 4 && NV % 4 == 0) {
#pragma unroll
        for (int k = 0; k < NV / 4; ++k) {
            const float4 q = reinterpret_cast<const float4*>(src)[k];
            v[4 * k] = q.x; v[4 * k + 1] = q.y; v[4 * k + 2] = q.z; v[4 * k + 3] = q.w;
        }
    } else if constexpr (sizeof(T) == 8 && NV % 2 == 0) {
#pragma unroll
        for (int k = 0; k < NV / 2; ++k) {
            const double2 q = reinterpret_cast<const double2*>(src)[k];
            v[2 * k] = q.x; v[2 * k + 1] = q.y;
        }
    } else if constexpr (sizeof(T) == 4 && NV == 2) {
        const float2 q = *reinterpret_cast<const float2*>(src);
        v[0] = q.x; v[1] = q.y;
    } else {
#pragma unroll
        for (int k = 0; k < NV; ++k) v[k] = src[k];
    }
}

// A boundary-row column: M (X, Y) and the lane exponent, the exponent carried as T's bits.
__device__ __forceinline__ float exp_bits(int e, float) { return __int_as_float(e); }
__device__ __forceinline__ double exp_bits(int e, double) { return __longlong_as_double(static_cast<long long>(e)); }
__device__ __forceinline__ int bits_exp(float v) { return __float_as_int(v); }
__device__ __forceinline__ int bits_exp(double v) { return static_cast<int>(__double_as_longlong(v)); }

// Bytes of dynamic shared memory the soft kernel needs for a block of `block` threads.
__host__ __device__ inline size_t soft_smem_bytes(int K, int N, int G, int R, int block, int tsize, bool tracked,
                                                  bool multiwarp = false) {
    const int gpb = block / G;
    size_t b = size_t((K * N + 1) * (N + 1) + 4 * K) * tsize;
    b = (b + 15) & ~size_t(15);
    b += size_t(N + 1) * G * R * tsize * gpb;              // per-lane substitution counts
    if (G > 1) b += size_t(K) * N * N * tsize * gpb;        // per-group histogram
    b = (b + 15) & ~size_t(15);
    b += size_t(block) * 2 * 4 * tsize;                    // per-group boundary staging (write, read)
    if (tracked) b += size_t(4) * K * 8 * block;            // per-lane tracked gap sums
    if (multiwarp) b += size_t(gpb) * 8 * 8 + size_t(gpb) * 4 + 16;   // per-warp partials, progress
    return b;
}

// Several warps per pair (long pairs): warp w fills stripes w, w + NW, ... and waits, every 32
// steps, until the warp filling the stripe above (below, in the backward pass) has published
// enough progress.  The wait is bounded: past SoftArgs::spin_limit polls (kSpinLimit unless
// the store sets another) the pair is marked failed (kSoftStall) and every warp finishes the
// pass without waiting further.
constexpr int kSpinLimit = 1 << 22;

// The backward pass reads the forward table one lane-step row (G lanes x R rows x 3 values)
// per step, in reverse; the row kPrefetchSteps steps ahead is asked into L2 meanwhile, so the
// register prefetch one step ahead finds it there instead of waiting on HBM.
#ifndef NWG_SOFT_PREFETCH_STEPS
#define NWG_SOFT_PREFETCH_STEPS 4
#endif
constexpr int kPrefetchSteps = NWG_SOFT_PREFETCH_STEPS;

// BAND: the guide-banded forward-backward (aligner.hpp:6231-6524 with AlignBand::GuideBanded):
// cells outside the band are zero -- forward cells of row i >= 1 outside [jlo(i), jhi(i)],
// Global border cells past border_rows / border_cols, backward cells outside [jlo0(i), jhi0(i)];
// Local log Z sums the band only.  Zero cells neither receive nor pass on probability, which is
// what the reference's band-limited tables compute.  Each stripe sweeps only the union of its
// rows' bands (band_cols), so a pass costs about (128 + 2 x bandwidth) columns per stripe.
// POST: soft_guide="posterior" (aligner.hpp:6776-6808, 1466-1475): the backward pass also keeps,
// per row, the column of greatest exit mass -- the cell's posterior less the posterior of moving
// on to (i, j+1) within the row (affine: the Y posterior there; linear: F e_a B(i, j+1)), the
// first such column on ties -- and the pair's guide is their running maximum over the rows.
// TL: tiled long pairs (SoftArgs::tiles, one phase per launch).  Forward: the tile's lanes start
// from the tile to the left's saved last column and the row above from the stripe above's bottom
// row; the tile leaves its own bottom row and last column, and its part of Z.  Backward (tiles in
// reverse diagonal order): the tile recomputes its forward table from the same inputs (the same
// bits), starts from the tile to the right's saved first column and the row below from the
// stripe below's top row, and adds its counts into its stripe's partial; tile_z_kernel and
// tile_finish_kernel form Z and each pair's totals between and after the phases.
template <class T, bool AFF, bool LOC, bool TR, int G, int R, bool MW = false, bool BAND = false, bool SG = false,
          bool POST = false, bool TL = false>
__global__ void __launch_bounds__(MW ? 512 : 128, (POST ? 3 : MW ? 1 : (G > 1 ? (R >= 8 ? 2 : 4) : 1)))
soft_kernel(const SoftArgs A) {
    static_assert(!POST || (G == 32 && R == 4 && !MW && !BAND && !TR), "posterior guides: 32 x 4, untracked, full DP");
    static_assert(!TL || (G == 32 && !MW && !BAND && !SG && !TR && !POST), "tiles: 32 lanes, untracked, full DP, Global or Local");
    static_assert(!MW || (G == 32 && !TR), "several warps per pair: 32 lanes, untracked");
    static_assert(!BAND || (G == 32 && !MW), "banded: 32 lanes, one warp per pair");
    static_assert(!SG || !LOC, "semi-global ends: Global kernels");
    constexpr int GR = G * R;
    constexpr bool kCount = sizeof(T) == 4;  // float32 charges its lost mass (double's is ~2^-900)
    constexpr int NV = AFF ? 3 : 1;          // values per cell
    constexpr int CV = NV * R;               // values per lane column
    constexpr int BW = AFF ? 4 : 2;          // boundary-row values per column: M (X, Y), exponent
    const int N = A.N, K = A.K;
    const int wcols = N + 1;
    const int nw = (K * N + 1) * wcols;
    const int gpb = blockDim.x / G;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sw = reinterpret_cast<T*>(smem_raw);
    T* sgw = sw + nw;
    unsigned char* after = reinterpret_cast<unsigned char*>(sgw + 4 * K);
    after = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(after) + 15) & ~uintptr_t(15));
    T* macc_all = reinterpret_cast<T*>(after);
    T* hist_all = macc_all + size_t(N + 1) * GR * gpb;
    T* stage_all = reinterpret_cast<T*>(
        (reinterpret_cast<uintptr_t>(hist_all + (G > 1 ? size_t(K) * N * N * gpb : 0)) + 15) & ~uintptr_t(15));
    double* tg_all = reinterpret_cast<double*>(stage_all + size_t(blockDim.x) * 2 * 4);
    double* cpart = tg_all + (TR ? size_t(4) * K * blockDim.x : 0);        // MW: [warp][8] partials
    volatile int* prog = reinterpret_cast<volatile int*>(cpart + (MW ? 8 * gpb : 0));   // MW: per warp
    for (int k = threadIdx.x; k < nw; k += blockDim.x) sw[k] = static_cast<const T*>(A.w)[k];
    for (int k = threadIdx.x; k < 4 * K; k += blockDim.x) sgw[k] = static_cast<const T*>(A.gw)[k];

    const int lane = threadIdx.x % G;
    const int gib = threadIdx.x / G;
    const int64_t slot = MW ? int64_t(blockIdx.x) : int64_t(blockIdx.x) * gpb + gib;
    const int NWp = MW ? gpb : 1;                            // warps per pair
    T* macc = macc_all + size_t(N + 1) * GR * gib;          // [b][lane][r]
    T* hist = hist_all + size_t(K) * N * N * gib;
    // boundary rows pass through shared memory G columns at a time: the producing lane stages
    // its column every step and the group writes the G columns as one coalesced row segment;
    // the consuming lane reads a staged segment the group loaded one segment ahead
    T* stw = stage_all + size_t(gib) * G * 2 * 4;            // [G][BW] produced columns
    T* str = stw + G * 4;                                    // [G][BW] columns to consume
    double* tg = tg_all + size_t(4) * K * threadIdx.x;        // tracked gap sums of this lane
    for (int k = lane; k < (N + 1) * GR; k += G) macc[k] = T(0);
    if constexpr (G > 1) for (int k = lane; k < K * N * N; k += G) hist[k] = T(0);
    if constexpr (TR) for (int k = 0; k < 4 * K; ++k) tg[k] = 0.0;
    __syncthreads();

    unsigned gmask;
    if constexpr (G == 32) gmask = 0xffffffffu;
    else gmask = ((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1));
    const int rmask = A.renorm_mask;

    unsigned char* sbase = static_cast<unsigned char*>(A.scratch) + slot * A.scratch_stride;
    T* fwd = reinterpret_cast<T*>(sbase + (MW ? gib * A.warp_stride : 0));
    int* fexp = reinterpret_cast<int*>(reinterpret_cast<unsigned char*>(fwd) + A.fwd_bytes);
    const int64_t nb = int64_t(A.maxn) + 1;
    const bool ck = MW || TL || A.ck != 0;
    const int nbrows = ck ? A.max_stripes : 1;              // forward boundary rows kept
    const int nbrows_b = MW ? A.max_stripes : 1;            // backward boundary rows kept
    unsigned char* bb = sbase + A.bnd_off;
    T* fbnd = reinterpret_cast<T*>(bb);                      // [nbrows][nb][BW]
    T* bbnd = fbnd + BW * nb * nbrows;                       // [nbrows_b][nb][BW]
    const int pw = (gib + NWp - 1) % NWp;                    // MW: the warp of the neighbouring stripe
    // MW: wait until the neighbouring stripe's warp has published `target` (bounded)
    bool stalled = false;
    auto wait_for = [&](int target) {
        if constexpr (MW) {
            int k = 0;
            while (!stalled && prog[pw] < target) {
                if (++k > A.spin_limit) stalled = true;
                else __nanosleep(64);
            }
            __syncwarp();
            __threadfence_block();
        }
    };
    auto publish = [&](int v) {
        if constexpr (MW) {
            __syncwarp();
            __threadfence_block();
            if (lane == 0) prog[gib] = v;
        }
    };
    // untracked: the one set's gap weights
    const T oa0 = sgw[0], ea0 = sgw[1], ob0 = sgw[2], eb0 = sgw[3];
    const T loss_w = static_cast<const T*>(A.gw)[4 * K];
    // the largest exact power of two one factor of a transfer may take (incoming values can
    // lie more than that above a lane's scale only when they are at most 2^kLift in its units)
    constexpr int kExpHi = sizeof(T) == 4 ? 126 : 1022;

    // the next pair of this group (a block, for several warps per pair) from the launch's work
    // queue, in the longest-first order: a group that finishes early takes the next pair
    __shared__ long long s_next;
    auto next_item = [&]() -> int64_t {
        if constexpr (MW) {
            __syncthreads();
            if (threadIdx.x == 0) s_next = wq_next(A.queue, int(gridDim.x), A.n_items);
            __syncthreads();
            return s_next;
        } else {
            long long v = 0;
            if (lane == 0) v = wq_next(A.queue, int(gridDim.x) * gpb, A.n_items);
            if constexpr (G > 1) v = __shfl_sync(gmask, v, 0, G);
            return v;
        }
    };
    for (int64_t it = next_item(); it < A.n_items; it = next_item()) {
        const int p = TL ? A.tiles[3 * it] : A.order[it];
        const int ts = TL ? A.tiles[3 * it + 1] : 0, tc = TL ? A.tiles[3 * it + 2] : 0;   // TL: stripe, tile
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
        // banded: the band of row i (aligner.hpp:2644-2700) and the charged borders
        const int32_t* gd = BAND ? A.guide + ao + p : nullptr;
        const int bw = A.band;
        auto jlo_of = [&](int i) { return max(1, gd[i] - bw); };
        auto jlo0_of = [&](int i) { return max(0, gd[i] - bw); };
        auto jhi_of = [&](int i) {
            if (!LOC && !SG && i == m) return n;   // glocal: row m's own band
            int hi = gd[i] + bw;
            if (i < m) hi = max(hi, gd[i + 1] - 1 + bw);
            return min(n, hi);
        };
        int brows = m, bcols = n;
        if constexpr (BAND) {
            // border rows: the leading rows 1.. whose guide is within the band of column 0
            brows = m;
            for (int base = 1; base <= m; base += G) {
                const int i = base + lane;
                const unsigned over = __ballot_sync(gmask, i <= m && gd[i] > bw);
                if (over) { brows = base + __ffs(over) - 2; break; }
            }
            bcols = jhi_of(0);
        }
        // the columns [tc0f, tc1f] a stripe sweeps (TL: the tile's) and its steps, its columns
        // plus the skew; a banded stripe sweeps fewer (band_cols), within the same table stride
        const int tc0f = TL ? tc * A.tile_w : 0, tc1f = TL ? min(n, tc0f + A.tile_w - 1) : n;
        const int ntc = TL ? n / A.tile_w + 1 : 1;   // TL: tiles per stripe (columns 0..n)
        const int Sf = tc1f - tc0f + G;
        const int SP = Sf + 1;                  // MW: progress key per stripe
        // banded: the columns of stripe s, the union of its rows' bands with the first rounded
        // down to a multiple of G (the forward pass stages the row above in G-aligned
        // segments).  Both passes' cells of rows >= 1 outside a row's band are zero, so the
        // sweep skips them; a column left of the union is out of band for all of the stripe's
        // rows, and where the union starts at column 1 the rounding takes in column 0 (its Local
        // start weights feed column 1).  Stripe 0 starts at column 0: row 0's cells are the
        // origin and its gap run (Global) or start weights at every column (Local, glocal), and
        // row 1 reads them left of its band.  A neighbouring stripe's row outside its own
        // columns reads as zero.
        auto band_cols = [&](const int s, int& lo, int& hi) {
            int l = n + 1, h = -1;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = s * GR + lane * R + r;
                if (i <= m) { l = min(l, jlo0_of(i)); h = max(h, jhi_of(i)); }
            }
            l = __reduce_min_sync(gmask, l);
            h = __reduce_max_sync(gmask, h);
            lo = s == 0 ? 0 : l & ~(G - 1);
            hi = h;
        };
        // TL: this pair's rows (stride n + 1), per-tile lane states and per-stripe partials
        T* const rowf_p = TL ? static_cast<T*>(A.rowf) + A.row_off[p] * BW : nullptr;
        T* const rowb_p = TL ? static_cast<T*>(A.rowb) + A.row_off[p] * BW : nullptr;
        constexpr int LS = NV * R + 1;          // TL: one lane's saved state (values, exponent)
        T* const colf_p = TL ? static_cast<T*>(A.colf) + A.col_off[p] * LS : nullptr;
        T* const colb_p = TL ? static_cast<T*>(A.colb) + A.col_off[p] * LS : nullptr;
        int why = 0;                            // kSoft* bits: why this pair is refused
        // semi-global ends (aligner.hpp:6362-6430): free starts on row 0 / column 0, Z over the
        // end cells (row m or (m, n), then column n of rows 0..m-1), the backward seeded with 1
        // at each; gap moves into a free start's border cells are not moves (6309-6319)
        const bool sg_r0 = SG && (A.ends & 4), sg_c0 = SG && (A.ends & 1);
        const bool sg_ec = SG && (A.ends & 2), sg_er = SG && (A.ends & 8);
        const bool zsg = SG && A.ends != 0;
        if constexpr (MW) {
            if (lane == 0) prog[gib] = -1;
            __syncthreads();
        }

        // ── forward ──────────────────────────────────────────────────────────
        XAcc zacc; zacc.init();                 // Local: the sum over every cell
        T zM = T(0), zX = T(0), zY = T(0); int zE = 0;   // Global: (m, n)
        // One stripe of the forward pass.  pass1: the first pass (Z, boundary rows; the table
        // too unless checkpointed); else the recompute of a checkpointed stripe's table, which
        // repeats the first pass's arithmetic from the same boundary row: the same bits.
        auto fwd_stripe = [&](const int s, const bool pass1) {
            const int i0 = s * GR + lane * R;   // this lane's first DP row (rows 0..m)
            // a lane wholly below row m (the last stripe's padding) keeps no table: its backward
            // values are zero, so its forward values are never needed
            const bool store_table = (!ck || !pass1) && i0 <= m;
            int tc0 = tc0f, tc1 = tc1f;
            int plo = 0, phi = -1;              // banded: the columns the stripe above swept
            if constexpr (BAND) {
                band_cols(s, tc0, tc1);
                if (s > 0) band_cols(s - 1, plo, phi);
            }
            const int S = tc1 - tc0 + G;
            T* const fb_in = TL ? rowf_p + int64_t(s - 1) * BW * (n + 1) : fbnd + (ck ? int64_t(s - 1) * BW * nb : 0);
            T* const fb_out = TL ? rowf_p + int64_t(s) * BW * (n + 1) : fbnd + (ck ? int64_t(s) * BW * nb : 0);
            int key[R];
            T roa[TR ? R : 1], rea[TR ? R : 1], rob[TR ? R : 1], reb[TR ? R : 1];
            T vmask[R];
            T cM[R], cX[R], cY[R];
            int blo[BAND ? R : 1], bhi[BAND ? R : 1], blo0[BAND ? R : 1];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = i0 + r;
                const bool valid = i <= m;
                if constexpr (BAND) {
                    blo[r] = valid ? jlo_of(i) : n + 1;
                    bhi[r] = valid ? jhi_of(i) : -1;
                    blo0[r] = valid ? jlo0_of(i) : n + 1;
                }
                vmask[r] = valid ? T(1) : T(0);
                key[r] = (valid && i >= 1) ? (tset(i) * N + ap[i - 1]) * wcols : K * N * wcols;
                if constexpr (TR) {
                    const int gs = valid ? gset(i) : 0;
                    const int ts = (valid && i >= 1) ? tset(i) : 0;
                    roa[r] = sgw[4 * gs + 0]; rea[r] = sgw[4 * gs + 1];
                    rob[r] = sgw[4 * ts + 2]; reb[r] = sgw[4 * ts + 3];
                }
                cM[r] = T(0); cX[r] = T(0); cY[r] = T(0);
            }
            // a lane holding a start cell begins at exponent 0 (its start weight is 1); the
            // others begin empty and take the scale of the first values they receive.
            // Lanes that add a start weight at every step (Local; row 0 a free start) keep
            // their exponent when their values vanish (band masks), so that weight stays finite.
            const bool keep_e = LOC || (sg_r0 && s == 0 && lane == 0);
            int E = (LOC || sg_c0 || (s == 0 && lane == 0)) ? 0 : kEmpty;
            T lone = pow2s<T>(-E);                // 2^-E: a free start's weight in lane units
            T zpart = T(0);                       // Local: the cells' sum since the last renorm
            T dgM = T(0), dgX = T(0), dgY = T(0); // row above, column j-1
            T upM = T(0), upX = T(0), upY = T(0); // row above, column j
            T* fs = fwd + (ck ? 0 : int64_t(s) * Sf * G * CV);
            int* fe = fexp + (ck ? 0 : int64_t(s) * Sf * G);
            int nbj = tc0 > 0 ? int(bp[tc0 - 1]) : N;   // the first column's b code (column 0: none)
            // TL: this lane's state at the column left of the tile, as the tile to the left left it
            const T* const lst = (TL && tc > 0) ? colf_p + (int64_t(s) * ntc + tc - 1) * G * LS : nullptr;
            if (TL && tc > 0) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    cM[r] = lst[lane * LS + NV * r];
                    if constexpr (AFF) { cX[r] = lst[lane * LS + NV * r + 1]; cY[r] = lst[lane * LS + NV * r + 2]; }
                }
                E = bits_exp(lst[lane * LS + LS - 1]);
                lone = pow2s<T>(-E);
            }
            // the row above (the previous stripe's bottom row): one lane per pair reads it one
            // column ahead; a group loads it G columns at a time, one segment ahead (rb), into
            // the staging row lane 0 reads
            T rb[BW];
#pragma unroll
            for (int k = 0; k < BW; ++k) rb[k] = T(0);
            auto load_seg = [&](int c0) {   // group: columns c0 .. c0 + G - 1 into rb
                const int c = c0 + lane;
                if (BAND && (c < plo || c > phi)) {   // not swept above: zero, no scale
#pragma unroll
                    for (int k = 0; k < BW - 1; ++k) rb[k] = T(0);
                    rb[BW - 1] = exp_bits(kEmpty, T(0));
                } else if (c <= tc1) {
                    vload<T, BW>(rb, fb_in + int64_t(c) * BW);
                }
            };
            auto stage_seg = [&]() {        // group: rb into the staging row
                __syncwarp(gmask);
                vstore<T, BW>(str + lane * 4, rb);
                __syncwarp(gmask);
            };
            // MW: the stripe above has written column c by its step c + 2G - 2 (a segment is
            // written once complete); the group reads columns up to t + 2G within step t
            const bool waits = MW && pass1 && s > 0;
            if (waits) wait_for((s - 1) * SP + min(S, 4 * G + 1));
            // the next column's row-above values (lane 0: the previous stripe's bottom row; the
            // other lanes: the lane above's bottom row) into this lane's units
            auto take_up = [&](const T iM, const T iX, const T iY, const int iE) {
                int d = iE - E;
                if (d > kLift) {   // keep the incoming values in range: move own state down
                    const T mi = AFF ? tmax(iM, tmax(iX, iY)) : iM;
                    if (!(mi > T(0))) {   // zeros: nothing to align to
                        upM = T(0); upX = T(0); upY = T(0);
                        return;
                    }
                    // the incoming largest value lands at 2^kLift (an empty lane: at 1), by
                    // its own magnitude, not its sender's exponent -- a sender between its
                    // rescales can hold values far above 1, and lifts down a chain of empty
                    // lanes would compound
                    const int de = d + ilog2(mi);
                    const int tgt = E == kEmpty ? 0 : kLift;
                    if (de > tgt) {
                        const int sh = tgt - de;
#pragma unroll
                        for (int r = 0; r < R; ++r) { cM[r] = scale_down(cM[r], sh); cX[r] = scale_down(cX[r], sh); cY[r] = scale_down(cY[r], sh); }
                        dgM = scale_down(dgM, sh); dgX = scale_down(dgX, sh); dgY = scale_down(dgY, sh);
                        zpart = scale_down(zpart, sh);
                        E -= sh; lone = pow2s<T>(-E); d += sh;
                    }
                    if (d > kExpHi) {   // small values far above this lane's scale: 2^d in two factors
                        const T f1 = pow2i<T>(d - kExpHi), f2 = pow2i<T>(kExpHi);
                        upM = (iM * f1) * f2;
                        if constexpr (AFF) { upX = (iX * f1) * f2; upY = (iY * f1) * f2; }
                        return;
                    }
                }
                if (d >= (sizeof(T) == 4 ? -126 : -1022)) {
                    const T f = pow2i<T>(d);
                    upM = iM * f;
                    if constexpr (AFF) { upX = iX * f; upY = iY * f; }
                } else {
                    upM = scale_down(iM, d);
                    if constexpr (AFF) { upX = scale_down(iX, d); upY = scale_down(iY, d); }
                }
            };
            if (TL && tc > 0) {
                // the row above at the column left of the tile, into this lane's units: lane 0 from
                // the stripe above's bottom row, the others from the lane above's saved last row
                T v[BW];
                if (lane == 0) {
                    if (s > 0) vload<T, BW>(v, fb_in + int64_t(tc0 - 1) * BW);
                } else {
#pragma unroll
                    for (int k = 0; k < NV; ++k) v[k] = lst[(lane - 1) * LS + NV * (R - 1) + k];
                    v[BW - 1] = lst[(lane - 1) * LS + LS - 1];
                }
                if (lane > 0 || s > 0) {
                    take_up(v[0], AFF ? v[1] : T(0), AFF ? v[2] : T(0), bits_exp(v[BW - 1]));
                    dgM = upM; dgX = upX; dgY = upY;
                    upM = T(0); upX = T(0); upY = T(0);
                }
            }
            if constexpr (BAND) {
                // the row above at the column left of the stripe's first: lane 0 from the stripe
                // above's bottom row (the other lanes' rows above are out of band there)
                if (s > 0 && tc0 > 0 && lane == 0 && tc0 - 1 >= plo && tc0 - 1 <= phi) {
                    T v[BW];
                    vload<T, BW>(v, fb_in + int64_t(tc0 - 1) * BW);
                    take_up(v[0], AFF ? v[1] : T(0), AFF ? v[2] : T(0), bits_exp(v[BW - 1]));
                    dgM = upM; dgX = upX; dgY = upY;
                    upM = T(0); upX = T(0); upY = T(0);
                }
            }
            if (s > 0) {
                if constexpr (G == 1) {
                    load_seg(0);
                    take_up(rb[0], AFF ? rb[1] : T(0), AFF ? rb[2] : T(0), bits_exp(rb[BW - 1]));
                    load_seg(1);
                } else {
                    load_seg(tc0);
                    stage_seg();
                    load_seg(tc0 + G);
                    if (lane == 0) {
                        T v[BW];
                        vload<T, BW>(v, str);
                        take_up(v[0], AFF ? v[1] : T(0), AFF ? v[2] : T(0), bits_exp(v[BW - 1]));
                    }
                }
            }
            for (int t = 0; t < S; ++t) {
                const int j = tc0 + t - lane;     // column tc0..tc1 (the full DP: 0..n)
                if (waits && t > 0 && (t & 31) == 0) wait_for((s - 1) * SP + min(S, t + 4 * G + 1));
                if (MW && pass1 && t > 0 && (t & 7) == 0) publish(s * SP + t);   // steps 0 .. t-1 done
                const bool active = (j >= tc0) && (j <= tc1);
                if (active) {
                    const int bj = nbj;                   // column 0: the zero column
                    nbj = j < n ? int(bp[j]) : N;         // the next column's code, one step ahead
                    T pM = dgM, pX = dgX, pY = dgY;
                    T qM = upM, qX = upX, qY = upY;
                    const bool c0free = sg_c0 && j == 0;      // column 0 a free start
                    const bool jn = j == n, ecn = sg_ec && j == n;
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const int i = i0 + r;
                        const T wv = sw[key[r] + bj];
                        const T o_a = TR ? roa[r] : oa0, e_a = TR ? rea[r] : ea0;
                        const T o_b = TR ? rob[r] : ob0, e_b = TR ? reb[r] : eb0;
                        T fm, fx = T(0), fy = T(0);
                        if constexpr (AFF) {
                            fm = ((pM + pX) + pY) * wv;
                            fx = fmaf_t(qM + qY, o_b, qX * e_b);
                            fy = fmaf_t(cM[r] + cX[r], o_a, cY[r] * e_a);
                            // row 0 is only ever a lane's first row (r == 0): the test vanishes for r > 0
                            if constexpr (LOC) {
                                fm += lone;
                                if (j == 0) fx = T(0);
                                if (r == 0 && i == 0) fy = T(0);
                            } else {
                                if (r == 0 && i == 0 && (j == 0 || sg_r0)) { fm = lone; fy = T(0); }
                                if (c0free && i >= 1 && i <= m) { fm = lone; fx = T(0); }
                            }
                        } else {
                            fm = fmaf_t(pM, wv, fmaf_t(qM, e_b, cM[r] * e_a));
                            if constexpr (LOC) {
                                if ((r == 0 && i == 0) || j == 0) fm = T(0);
                                fm += lone;
                            } else {
                                if (r == 0 && i == 0 && (j == 0 || sg_r0)) fm = lone;
                                if (c0free && i >= 1 && i <= m) fm = lone;
                            }
                        }
                        if constexpr (BAND) {
                            if (i >= 1 && j >= 1) {
                                if (j < blo[r] || j > bhi[r]) { fm = T(0); fx = T(0); fy = T(0); }
                            } else if constexpr (!LOC) {
                                // the charged borders (linear keeps them in M)
                                if (i == 0 && j > bcols && !sg_r0) { fy = T(0); if constexpr (!AFF) fm = T(0); }
                                if (j == 0 && i > brows) { fx = T(0); if constexpr (!AFF) fm = T(0); }
                            }
                        }
                        pM = cM[r]; pX = cX[r]; pY = cY[r];
                        cM[r] = fm; cX[r] = fx; cY[r] = fy;
                        qM = fm; qX = fx; qY = fy;
                        if constexpr (LOC) {
                            T zm_ = vmask[r];
                            if constexpr (BAND) zm_ = (j >= blo0[r] && j <= bhi[r]) ? zm_ : T(0);
                            zpart = fmaf_t(zm_, (fm + fx) + fy, zpart);
                        } else if (zsg) {
                            const bool e = (i == m) ? (jn || sg_er) : (ecn && i < m);
                            if (e) zpart += (fm + fx) + fy;
                        }
                    }
                    dgM = upM; dgX = upX; dgY = upY;
                    if ((t & rmask) == 0 || j == tc1) {
                        // renormalise: the lane's largest value into [1, 2)
                        T mx = T(0);
#pragma unroll
                        for (int r = 0; r < R; ++r) mx = tmax(mx, tmax(cM[r], tmax(cX[r], cY[r])));
                        if (!is_finite(mx)) why |= kSoftRange;
                        else if (mx > T(0)) {
                            int e = ilog2(mx);
                            if (e < -120) e = -120;
                            if ((LOC || zsg) && pass1) zacc.add(static_cast<double>(zpart), E);
                            zpart = T(0);
                            if (e != 0) {
                                const T f = pow2i<T>(-e);
#pragma unroll
                                for (int r = 0; r < R; ++r) { cM[r] *= f; cX[r] *= f; cY[r] *= f; }
                                dgM *= f; dgX *= f; dgY *= f;
                                E += e; lone = pow2s<T>(-E);
                            }
                        } else if (!keep_e && !(dgM > T(0) || dgX > T(0) || dgY > T(0))) {
                            // nothing left to scale: the next values set the exponent
                            if ((LOC || zsg) && pass1) zacc.add(static_cast<double>(zpart), E);
                            zpart = T(0);
                            E = kEmpty;
                        }
                    }
                    // store the column for the backward pass
                    if (store_table) {
                        T v[CV];
#pragma unroll
                        for (int r = 0; r < R; ++r) {
                            v[NV * r] = cM[r];
                            if constexpr (AFF) { v[NV * r + 1] = cX[r]; v[NV * r + 2] = cY[r]; }
                        }
                        vstore_stream<T, CV>(fs + (int64_t(t) * G + lane) * CV, v);
                        __stcs(fe + int64_t(t) * G + lane, E);
                    }
                }
                // this stripe's bottom row (lane G-1's column t - G + 1) for the stripe below
                if (pass1 && s + 1 < nstripes) {
                    const int c = tc0 + t - (G - 1);
                    T v[BW];
                    v[0] = cM[R - 1];
                    if constexpr (AFF) { v[1] = cX[R - 1]; v[2] = cY[R - 1]; }
                    v[BW - 1] = exp_bits(E, T(0));
                    if constexpr (G == 1) {
                        if (c >= 0) vstore<T, BW>(fb_out + int64_t(c) * BW, v);
                    } else {
                        if (lane == G - 1 && c >= tc0) vstore<T, BW>(stw + (c & (G - 1)) * 4, v);
                        if (c >= tc0 && ((c & (G - 1)) == G - 1 || c == tc1)) {   // a full segment (or the last)
                            __syncwarp(gmask);
                            const int cc = c - (c & (G - 1)) + lane;
                            if (cc <= c) {
                                T w[BW];
                                vload<T, BW>(w, stw + lane * 4);
                                vstore<T, BW>(fb_out + int64_t(cc) * BW, w);
                            }
                            __syncwarp(gmask);
                        }
                    }
                }
                // the row above of the next step's column: one exponent alignment for every lane
                if constexpr (G > 1) {
                    const T sM = __shfl_up_sync(gmask, cM[R - 1], 1, G);
                    T sX = sM, sY = sM;
                    if constexpr (AFF) {
                        sX = __shfl_up_sync(gmask, cX[R - 1], 1, G);
                        sY = __shfl_up_sync(gmask, cY[R - 1], 1, G);
                    }
                    const int sE = __shfl_up_sync(gmask, E, 1, G);
                    const int cn = tc0 + t + 1;           // lane 0's next column
                    if (s > 0 && cn <= tc1 && (cn & (G - 1)) == 0) {   // a new segment: stage it, load the next
                        stage_seg();
                        load_seg(cn + G);
                    }
                    const bool top = lane == 0;
                    T v[BW];
                    vload<T, BW>(v, str + (cn & (G - 1)) * 4);
                    // only for a column this lane still computes: a finished lane keeps its
                    // state (row m's values are Z), an idle one its empty exponent
                    const int jn1 = tc0 + t + 1 - lane;
                    if (jn1 >= tc0 && jn1 <= tc1 && (!top || s > 0))
                        take_up(top ? v[0] : sM, top ? (AFF ? v[1] : T(0)) : sX, top ? (AFF ? v[2] : T(0)) : sY,
                                top ? bits_exp(v[BW - 1]) : sE);
                } else {
                    if (s > 0 && j < n) {
                        take_up(rb[0], AFF ? rb[1] : T(0), AFF ? rb[2] : T(0), bits_exp(rb[BW - 1]));
                        load_seg(j + 2);
                    }
                }
            }
            if (MW && pass1) publish(s * SP + S);
            if (TL && pass1 && tc + 1 < ntc) {   // this lane's state at the tile's last column
                T* const dst = colf_p + (int64_t(s) * ntc + tc) * G * LS + lane * LS;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    dst[NV * r] = cM[r];
                    if constexpr (AFF) { dst[NV * r + 1] = cX[r]; dst[NV * r + 2] = cY[r]; }
                }
                dst[LS - 1] = exp_bits(E, T(0));
            }
            if (pass1) {
                if (LOC || zsg) zacc.add(static_cast<double>(zpart), E);
                if constexpr (!LOC) {
                    if (m >= i0 && m < i0 + R && tc1 == n) {
#pragma unroll
                        for (int r = 0; r < R; ++r)
                            if (i0 + r == m) { zM = cM[r]; zX = cX[r]; zY = cY[r]; zE = E; }
                    }
                }
            }
            if constexpr (G > 1) __syncwarp(gmask);
        };
        if constexpr (TL) { if (A.tl_phase == 0) fwd_stripe(ts, true); }
        else for (int s = MW ? gib : 0; s < nstripes; s += NWp) fwd_stripe(s, true);
        // Z = zhat * 2^EZ with zhat in [1, 2)
        double zm; int ze;
        if (LOC || zsg) {
            if constexpr (G > 1) {
#pragma unroll
                for (int off = 1; off < G; off <<= 1) {
                    const double om = __shfl_xor_sync(gmask, zacc.m, off, G);
                    const int oe = __shfl_xor_sync(gmask, zacc.e, off, G);
                    zacc.add(om, oe);
                }
                zacc.m = __shfl_sync(gmask, zacc.m, 0, G);
                zacc.e = __shfl_sync(gmask, zacc.e, 0, G);
            }
            zm = zacc.m; ze = zacc.e;
        } else {
            zm = static_cast<double>((zM + zX) + zY); ze = zE;
            if constexpr (G > 1) {
                const int src = (m % GR) / R;
                zm = __shfl_sync(gmask, zm, src, G);
                ze = __shfl_sync(gmask, ze, src, G);
            }
        }
        if constexpr (G > 1) why = __reduce_or_sync(gmask, why);
        if constexpr (TL) {
            if (A.tl_phase == 0) {
                // the tile's part of Z (Local), or Z itself from the tile holding (m, n)
                if (lane == 0) {
                    if (LOC) {
                        const int64_t q = A.tile_off[p] + int64_t(ts) * ntc + tc;
                        A.zpart[2 * q] = zm; A.zpart[2 * q + 1] = double(ze);
                    } else if (ts == nstripes - 1 && tc1f == n) {
                        A.zpair[2 * p] = zm; A.zpair[2 * p + 1] = double(ze);
                    }
                    if (why) atomicOr(A.status + p, why);
                }
                continue;
            }
            // backward: the pair's Z (tile_z_kernel); a refused pair's tiles do nothing
            zm = A.zpair[2 * p]; ze = int(A.zpair[2 * p + 1]);
            if (A.status[p] != 0) continue;
        }
        if constexpr (MW) {
            // every warp's part of Z: Global, the warp holding row m; Local, the sum in warp order
            stalled = __any_sync(gmask, stalled);
            if (lane == 0) {
                cpart[8 * gib + 0] = zm; cpart[8 * gib + 1] = double(ze);
                cpart[8 * gib + 2] = double(why); cpart[8 * gib + 3] = stalled ? 1.0 : 0.0;
            }
            __syncthreads();
            bool anystall = false;
            if (LOC || zsg) {
                XAcc za; za.init();
                for (int w = 0; w < NWp; ++w) za.add(cpart[8 * w], int(cpart[8 * w + 1]));
                zm = za.m; ze = za.e;
            } else {
                const int ow = (nstripes - 1) % NWp;
                zm = cpart[8 * ow]; ze = int(cpart[8 * ow + 1]);
            }
            for (int w = 0; w < NWp; ++w) { why |= int(cpart[8 * w + 2]); anystall |= cpart[8 * w + 3] != 0.0; }
            stalled = anystall;
            if (lane == 0) prog[gib] = -1;
            __syncthreads();
            if (stalled) {
                if (threadIdx.x == 0) { A.status[p] = kSoftStall; A.score[p] = 0.0; }
                stalled = false;
                continue;
            }
        }
        if (!(zm > 0.0) || !(zm < 1e300)) why |= kSoftZ;
        if (why) {
            if (lane == 0 && (!MW || gib == 0)) { A.status[p] = why; A.score[p] = 0.0; }
            continue;
        }
        const int EZ = ze + ilog2(zm);
        const double zhat = zm * pow2i<double>(ze - EZ);
        const double invz = 1.0 / zhat;
        const T invzT = static_cast<T>(invz);

        // ── backward, fused with the expected counts ─────────────────────────
        double ga_o = 0, ga_x = 0, gb_o = 0, gb_x = 0;   // untracked: opens and extend-only moves
        T lacc = T(0);                                   // float32: this lane's lost-mass charge
        bool cnt_nf = false;                             // one lane per pair: a count not finite
        if constexpr (G == 1) {
            double* g1 = A.grad + A.gstride * p;
            for (int k = 0; k < K * N * N; ++k) g1[k] = 0.0;
        }
        for (int s = TL ? ts : nstripes - 1 - (MW ? gib : 0); s >= (TL ? ts : 0); s -= NWp) {
            if (ck) fwd_stripe(s, false);       // this stripe's forward table, from its checkpoint
            int tc0 = tc0f, tc1 = tc1f;
            int nlo = 0, nhi = -1;              // banded: the columns the stripe below swept
            if constexpr (BAND) {
                band_cols(s, tc0, tc1);
                if (s < nstripes - 1) band_cols(s + 1, nlo, nhi);
            }
            const int S = tc1 - tc0 + G;
            // this stripe's row below (read) and its own top row (written): MW keeps one per stripe
            T* const bb_in = TL ? rowb_p + int64_t(s + 1) * BW * (n + 1) : bbnd + (MW ? int64_t(s + 1) * BW * nb : 0);
            T* const bb_out = TL ? rowb_p + int64_t(s) * BW * (n + 1) : bbnd + (MW ? int64_t(s) * BW * nb : 0);
            const int bkey = nstripes - 1 - s;   // MW: progress keys grow as the pass goes up
            const int i0 = s * GR + lane * R;
            int keyd[R], krow[R];
            T roa[TR ? R : 1], rea[TR ? R : 1], rob[TR ? R : 1], reb[TR ? R : 1];   // rob/reb: row i+1
            int gsr[TR ? R : 1], tsd[TR ? R : 1];
            T vmask[R];
            T bM[R], bX[R], bY[R];
            int bblo0[BAND ? R : 1], bbhi[BAND ? R : 1];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = i0 + r;
                const bool valid = i <= m;
                if constexpr (BAND) {
                    bblo0[r] = valid ? jlo0_of(i) : n + 1;
                    bbhi[r] = valid ? jhi_of(i) : -1;
                }
                vmask[r] = valid ? T(1) : T(0);
                const int td = (i + 1 <= m) ? tset(i + 1) : 0;
                const int kd = (i + 1 <= m) ? (td * N + ap[i]) : K * N;
                keyd[r] = kd * wcols;
                krow[r] = kd;
                if constexpr (TR) {
                    const int gs = valid ? gset(i) : 0;
                    gsr[r] = gs; tsd[r] = td;
                    roa[r] = sgw[4 * gs + 0]; rea[r] = sgw[4 * gs + 1];
                    rob[r] = sgw[4 * td + 2]; reb[r] = sgw[4 * td + 3];
                }
                bM[r] = T(0); bX[r] = T(0); bY[r] = T(0);
            }
            // a lane holding an end cell at its first column (row m's lane; Local every lane;
            // column n ends every lane with rows) begins at exponent 0, the others empty
            const bool holds_m = i0 <= m && m < i0 + R;
            const bool keep_b = LOC || (sg_er && holds_m);
            int EB = (LOC || holds_m || (sg_ec && i0 <= m)) ? 0 : kEmpty;
            T lone = pow2s<T>(-EB);
            T sgb_o = T(0), sga_o = T(0), sgb_x = T(0), sga_x = T(0);   // untracked: this stripe's gap sums
            // POST: per row the best exit mass so far (columns n down to j), its column, and the
            // Y posterior of the column to the right
            T pbest[POST ? R : 1], pyr[POST ? R : 1];
            int pcol[POST ? R : 1];
#pragma unroll
            for (int r = 0; r < (POST ? R : 1); ++r) { pbest[r] = T(-1); pyr[r] = T(0); pcol[r] = 0; }
            T dgM = T(0);                             // row below, column j+1 (BM only)
            // Global affine: the seed B = 1 at (m, n) enters every state through the diagonal
            // term, as B_M(m+1, n+1) = 1 with the padding weight w[K*N][N] = 1 (the cell and
            // everything else it reaches in the padding are zero), so no cell tests for it
            if constexpr (AFF && !LOC) {
                if (s == nstripes - 1 && tc1 == n) {
                    const int rc = m - i0;
#pragma unroll
                    for (int r = 1; r < R; ++r) bM[r] = (r == rc + 1) ? T(1) : bM[r];
                    if (rc == R - 1) dgM = T(1);
                }
            }
            T dnM = T(0), dnX = T(0), dnY = T(0);     // row below, column j
            // TL: this lane's state at the column right of the tile, as the tile to the right left it
            const T* const rst = (TL && tc1 < n) ? colb_p + (int64_t(s) * ntc + tc + 1) * G * LS : nullptr;
            if (TL && tc1 < n) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    bM[r] = rst[lane * LS + NV * r];
                    if constexpr (AFF) { bX[r] = rst[lane * LS + NV * r + 1]; bY[r] = rst[lane * LS + NV * r + 2]; }
                    else { bX[r] = bM[r]; bY[r] = bM[r]; }
                }
                EB = bits_exp(rst[lane * LS + LS - 1]);
                lone = pow2s<T>(-EB);
            }
            const T* fs = fwd + (ck ? 0 : int64_t(s) * Sf * G * CV);
            const int* fe = fexp + (ck ? 0 : int64_t(s) * Sf * G);
            // a lane wholly below row m has no table (its backward values are zero): it reads
            // zeros and scales by zero
            const bool lane_rows = i0 <= m;
            T nf[CV];
#pragma unroll
            for (int k = 0; k < CV; ++k) nf[k] = T(0);
            int nEF = 0, nbj = N;
            bool have_next = false;
            // the row below (the next stripe's top row), by distance d = n - column from the
            // right end: as in the forward pass, one lane per pair reads it one column ahead, a
            // group G columns at a time, one segment ahead (rb), through the staging row
            T rb[BW];
#pragma unroll
            for (int k = 0; k < BW; ++k) rb[k] = T(0);
            auto load_seg = [&](int d0) {   // group: distances d0 .. d0 + G - 1 into rb
                const int c = tc1 - d0 - lane;
                if (BAND && (c < nlo || c > nhi)) {   // not swept below: zero, no scale
#pragma unroll
                    for (int k = 0; k < BW - 1; ++k) rb[k] = T(0);
                    rb[BW - 1] = exp_bits(kEmpty, T(0));
                } else if (d0 + lane <= tc1 - tc0) {
                    vload<T, BW>(rb, bb_in + int64_t(c) * BW);
                }
            };
            auto stage_seg = [&]() {
                __syncwarp(gmask);
                vstore<T, BW>(str + lane * 4, rb);
                __syncwarp(gmask);
            };
            // MW: the stripe below has written distance d by its step d + 2G - 2 (a segment is
            // written once complete); the group reads distances up to t + 2G within step t
            const bool bwaits = MW && s < nstripes - 1;
            if (bwaits) wait_for((bkey - 1) * SP + min(S, 4 * G + 1));
            // the next column's row-below values (lane G-1: the next stripe's top row; the other
            // lanes: the lane below's top row) into this lane's units
            auto take_dn = [&](const T iM, const T iX, const T iY, const int iE) {
                int d = iE - EB;
                if (d > kLift) {
                    const T mi = AFF ? tmax(iM, tmax(iX, iY)) : iM;
                    if (!(mi > T(0))) {   // zeros: nothing to align to
                        dnM = T(0); dnX = T(0); dnY = T(0);
                        return;
                    }
                    const int de = d + ilog2(mi);   // as in the forward pass
                    const int tgt = EB == kEmpty ? 0 : kLift;
                    if (de > tgt) {
                        const int sh = tgt - de;
#pragma unroll
                        for (int r = 0; r < R; ++r) { bM[r] = scale_down(bM[r], sh); bX[r] = scale_down(bX[r], sh); bY[r] = scale_down(bY[r], sh); }
                        dgM = scale_down(dgM, sh);
                        EB -= sh; lone = pow2s<T>(-EB); d += sh;
                    }
                    if (d > kExpHi) {   // as in the forward pass
                        const T f1 = pow2i<T>(d - kExpHi), f2 = pow2i<T>(kExpHi);
                        dnM = (iM * f1) * f2;
                        if constexpr (AFF) { dnX = (iX * f1) * f2; dnY = (iY * f1) * f2; }
                        else { dnX = dnM; dnY = dnM; }
                        return;
                    }
                }
                if (d >= (sizeof(T) == 4 ? -126 : -1022)) {
                    const T f = pow2i<T>(d);
                    dnM = iM * f;
                    if constexpr (AFF) { dnX = iX * f; dnY = iY * f; }
                } else {
                    dnM = scale_down(iM, d);
                    if constexpr (AFF) { dnX = scale_down(iX, d); dnY = scale_down(iY, d); }
                }
                if constexpr (!AFF) { dnX = dnM; dnY = dnM; }
            };
            if (TL && tc1 < n) {
                // the row below at the column right of the tile (its M enters the diagonal term),
                // into this lane's units: lane G-1 from the stripe below's top row, the others from
                // the lane below's saved first row
                T v[BW];
                if (lane == G - 1) {
                    if (s < nstripes - 1) vload<T, BW>(v, bb_in + int64_t(tc1 + 1) * BW);
                } else {
#pragma unroll
                    for (int k = 0; k < NV; ++k) v[k] = rst[(lane + 1) * LS + k];
                    v[BW - 1] = rst[(lane + 1) * LS + LS - 1];
                }
                if (lane < G - 1 || s < nstripes - 1) {
                    take_dn(v[0], AFF ? v[1] : T(0), AFF ? v[2] : T(0), bits_exp(v[BW - 1]));
                    dgM = dnM;
                    dnM = T(0); dnX = T(0); dnY = T(0);
                }
            }
            if constexpr (BAND) {
                // the row below at the column right of the stripe's last: lane G-1 from the
                // stripe below's top row (the other lanes' rows below are out of band there)
                if (s < nstripes - 1 && tc1 < n && lane == G - 1 && tc1 + 1 >= nlo && tc1 + 1 <= nhi) {
                    T v[BW];
                    vload<T, BW>(v, bb_in + int64_t(tc1 + 1) * BW);
                    take_dn(v[0], AFF ? v[1] : T(0), AFF ? v[2] : T(0), bits_exp(v[BW - 1]));
                    dgM = dnM;
                    dnM = T(0); dnX = T(0); dnY = T(0);
                }
            }
            if (s < nstripes - 1) {
                if constexpr (G == 1) {
                    load_seg(0);
                    take_dn(rb[0], AFF ? rb[1] : T(0), AFF ? rb[2] : T(0), bits_exp(rb[BW - 1]));
                    load_seg(1);
                } else {
                    load_seg(0);
                    stage_seg();
                    load_seg(G);
                    if (lane == G - 1) {
                        T v[BW];
                        vload<T, BW>(v, str);
                        take_dn(v[0], AFF ? v[1] : T(0), AFF ? v[2] : T(0), bits_exp(v[BW - 1]));
                    }
                }
            }
            for (int t = 0; t < S; ++t) {
                const int j = tc1 - t + (G - 1 - lane);   // column tc1..tc0 (the full DP: n..0)
                if constexpr (kPrefetchSteps > 0) {
                    // every lane reads table row j - tc0 + lane at step t: the row kPrefetchSteps
                    // steps ahead goes to L2 now
                    const int u = tc1 - tc0 + G - 1 - t - kPrefetchSteps;
                    if (lane == 0 && u >= 0) {
                        prefetch_l2_bulk(fs + int64_t(u) * G * CV, unsigned(G * CV * sizeof(T)));
                        if constexpr ((G * sizeof(int)) % 16 == 0) prefetch_l2_bulk(fe + int64_t(u) * G, unsigned(G * sizeof(int)));
                        else prefetch_l2(fe + int64_t(u) * G);
                    }
                }
                if (bwaits && t > 0 && (t & 31) == 0) wait_for((bkey - 1) * SP + min(S, t + 4 * G + 1));
                if (MW && t > 0 && (t & 7) == 0) publish(bkey * SP + t);
                const bool active = (j >= tc0) && (j <= tc1);
                if (active) {
                    // this column's forward values were loaded one step ahead (or now, on
                    // the lane's first step); issue the next column's loads before the math
                    if (!have_next) {
                        if (lane_rows) {
                            vload_ro<T, CV>(nf, fs + (int64_t(j - tc0 + lane) * G + lane) * CV);
                            nEF = __ldg(fe + int64_t(j - tc0 + lane) * G + lane);
                        }
                        nbj = j < n ? int(bp[j]) : N;
                    }
                    T f[CV];
#pragma unroll
                    for (int k = 0; k < CV; ++k) f[k] = nf[k];
                    const int EF = nEF;
                    const int bj1 = nbj;              // b code of column j+1 (N: none)
                    have_next = j > tc0;
                    if (have_next) {
                        if (lane_rows) {
                            vload_ro<T, CV>(nf, fs + (int64_t(j - 1 - tc0 + lane) * G + lane) * CV);
                            nEF = __ldg(fe + int64_t(j - 1 - tc0 + lane) * G + lane);
                        }
                        nbj = int(bp[j - 1]);
                    }
                    // scale of this step's products: 2^(E_F + E_B - E_Z) / zhat (an exact power of
                    // two times 1 / zhat rounded to T).  Both lanes may hold values far above 1
                    // between renormalisations, so where that power falls below T's normal range
                    // F^ B^ itself can leave it (a posterior of 1 at 2^-130: F^ 2^63, B^ 2^67);
                    // this step's F^ then move down by the difference and the factor stays
                    // normal, so that no product overflows and none is dropped
                    int efac = EF + EB - EZ;
                    constexpr int kFacLo = sizeof(T) == 4 ? -126 : -1022;
                    const bool fdown = efac < kFacLo;
                    if (__builtin_expect(fdown, 0)) {
                        // 2^(efac - kFacLo) in two factors: a normal one, then the rest with
                        // gradual underflow (each F^ rounds at most twice, by 2^-150 each)
                        const int a = efac - kFacLo, h1 = max(a, kFacLo);
                        const T s1 = pow2i<T>(h1), s2 = pow2s<T>(a - h1);
#pragma unroll
                        for (int k = 0; k < CV; ++k) f[k] = (f[k] * s1) * s2;
                        efac = kFacLo;
                    }
                    const double facd = (TR && lane_rows) ? pow2i<double>(efac) * invz : 0.0;
                    const T fac = TR ? static_cast<T>(facd) : lane_rows ? pow2i<T>(efac) * invzT : T(0);
                    if (!is_finite(fac)) why |= kSoftScale;
                    T SF = T(0), SB = T(0);           // float32: this step's F^ and B^ sums (lost mass)
                    T dM = dgM;                       // row below, column j+1
                    T xM = dnM, xX = dnX, xY = dnY;   // row below, column j
                    T so_b = T(0), sx_b = T(0), so_a = T(0), sx_a = T(0);
                    T mc[R];
                    const bool noX = (LOC || sg_c0) && j == 0;   // Local / a free column 0: no gap move into it
                    const bool ecn = sg_ec && j == n;
#pragma unroll
                    for (int r = R - 1; r >= 0; --r) {
                        const int i = i0 + r;
                        const T wv = sw[keyd[r] + bj1];
                        const T fm = f[NV * r];
                        const T o_a = TR ? roa[r] : oa0, e_a = TR ? rea[r] : ea0;
                        const T o_b = TR ? rob[r] : ob0, e_b = TR ? reb[r] : eb0;
                        const T D = wv * dM;
                        T nM, nX, nY;
                        if constexpr (AFF) {
                            const T fx = f[NV * r + 1], fy = f[NV * r + 2];
                            // B keeps the gap moves into a free start's border cells (down column
                            // 0, along row 0) that the forward pass never takes, as the reference's
                            // backward does (they carry no forward mass, but the posterior guide
                            // reads those cells' B); the counts leave them out (aligner.hpp:6309-6319)
                            const T dXb = xX, rYb = bY[r];              // BX(i+1, j), BY(i, j+1)
                            const T dX = noX ? T(0) : dXb;
                            const T rY = ((LOC || sg_r0) && r == 0 && i == 0) ? T(0) : rYb;
                            nM = fmaf_t(o_a, rYb, fmaf_t(o_b, dXb, D));
                            nX = fmaf_t(o_a, rYb, fmaf_t(e_b, dXb, D));
                            nY = fmaf_t(e_a, rYb, fmaf_t(o_b, dXb, D));
                            if constexpr (LOC) {
                                nM = fmaf_t(vmask[r], lone, nM);
                                nX = fmaf_t(vmask[r], lone, nX);
                                nY = fmaf_t(vmask[r], lone, nY);
                            } else if (zsg) {   // the end cells besides (m, n), which the padding seeds
                                const bool e = (i == m) ? (sg_er && j < n) : (ecn && i < m);
                                if (e) { nM += lone; nX += lone; nY += lone; }
                            }
                            const T fmy = fm + fy, fmx = fm + fx;
                            const T fsum = fmy + fx;
                            mc[r] = fsum * D;
                            if constexpr (kCount) SF = fmaf_t(vmask[r], fsum, SF);
                            if constexpr (TR) {
                                const double ob_c = static_cast<double>(fmy * o_b * dX) * facd;
                                const double eb_c = static_cast<double>(fx * e_b * dX) * facd;
                                const double oa_c = static_cast<double>(fmx * o_a * rY) * facd;
                                const double ea_c = static_cast<double>(fy * e_a * rY) * facd;
                                double* gb = tg + 4 * tsd[r];
                                double* ga = tg + 4 * gsr[r];
                                gb[2] += ob_c; gb[3] += ob_c + eb_c;
                                ga[0] += oa_c; ga[1] += oa_c + ea_c;
                            } else {
                                so_b = fmaf_t(fmy, dX, so_b); sx_b = fmaf_t(fx, dX, sx_b);
                                so_a = fmaf_t(fmx, rY, so_a); sx_a = fmaf_t(fy, rY, sx_a);
                            }
                        } else {
                            const T dXb = xM, rYb = bM[r];              // as in the affine case
                            const T dX = noX ? T(0) : dXb;
                            const T rY = ((LOC || sg_r0) && r == 0 && i == 0) ? T(0) : rYb;
                            nM = fmaf_t(e_a, rYb, fmaf_t(e_b, dXb, D));
                            if constexpr (LOC) nM = fmaf_t(vmask[r], lone, nM);
                            else if (i == m && j == n) nM = lone;
                            else if (zsg) {
                                const bool e = (i == m) ? sg_er : (ecn && i < m);
                                if (e) nM += lone;
                            }
                            nX = nM; nY = nM;
                            mc[r] = fm * D;
                            if constexpr (kCount) SF = fmaf_t(vmask[r], fm, SF);
                            if constexpr (TR) {
                                tg[4 * tsd[r] + 3] += static_cast<double>(fm * e_b * dX) * facd;
                                tg[4 * gsr[r] + 1] += static_cast<double>(fm * e_a * rY) * facd;
                            } else {
                                sx_b = fmaf_t(fm, dX, sx_b);
                                sx_a = fmaf_t(fm, rY, sx_a);
                            }
                        }
                        if constexpr (BAND) {
                            if (j < bblo0[r] || j > bbhi[r]) { nM = T(0); nX = T(0); nY = T(0); }
                        }
                        if constexpr (kCount) SB += AFF ? (nM + nX) + nY : nM;
                        if constexpr (POST) {
                            // scanning columns downwards, >= keeps the first (smallest) column of the max
                            T ex;
                            if constexpr (AFF) {
                                const T cp = fmaf_t(f[NV * r], nM, fmaf_t(f[NV * r + 1], nX, f[NV * r + 2] * nY)) * fac;
                                ex = cp - pyr[r];
                                pyr[r] = f[NV * r + 2] * nY * fac;
                            } else {
                                const T e_a = ea0;
                                ex = f[NV * r] * (nM - e_a * bM[r]) * fac;
                            }
                            if (ex >= pbest[r]) { pbest[r] = ex; pcol[r] = j; }
                        }
                        dM = bM[r];
                        bM[r] = nM; bX[r] = nX; bY[r] = nY;
                        xM = nM; xX = nX; xY = nY;
                    }
                    // substitution counts of this column: one R-vector read-modify-write
                    {
                        T* dst = macc + (size_t(bj1) * G + lane) * R;
                        T cur[R];
                        vload<T, R>(cur, dst);
#pragma unroll
                        for (int r = 0; r < R; ++r) cur[r] = fmaf_t(mc[r], fac, cur[r]);
                        vstore<T, R>(dst, cur);
                    }
                    if constexpr (!TR) {
                        if constexpr (AFF) {
                            sgb_o = fmaf_t(so_b, fac, sgb_o);
                            sga_o = fmaf_t(so_a, fac, sga_o);
                        }
                        sgb_x = fmaf_t(sx_b, fac, sgb_x);
                        sga_x = fmaf_t(sx_a, fac, sga_x);
                    }
                    if constexpr (kCount) {
                        // the lost-mass charge of this lane-step in units of 2^-150 (the factor is
                        // normal: a step whose F^ moved down charges its B^ twice, for the F^ that
                        // rounded into the subnormal range on the way); fac scales the sums first,
                        // so that a large F^ + B^ times loss_w stays in range
                        if (lane_rows) {
                            const T sb = fdown ? SB + SB : SB;
                            lacc = fmaf_t(fac * (SF + sb), loss_w, fmaf_t(fac, T(16 * R), lacc));
                        }
                    }
                    dgM = dnM;
                    if ((t & rmask) == 0 || j == tc0) {
                        T mx = T(0);
#pragma unroll
                        for (int r = 0; r < R; ++r) mx = tmax(mx, tmax(bM[r], tmax(bX[r], bY[r])));
                        if (!is_finite(mx)) why |= kSoftRange;
                        else if (mx > T(0)) {
                            int e = ilog2(mx);
                            if (e < -120) e = -120;
                            if (e != 0) {
                                const T fsc = pow2i<T>(-e);
#pragma unroll
                                for (int r = 0; r < R; ++r) { bM[r] *= fsc; bX[r] *= fsc; bY[r] *= fsc; }
                                dgM *= fsc;
                                EB += e; lone = pow2s<T>(-EB);
                            }
                        } else if (!keep_b && !(dgM > T(0))) {
                            EB = kEmpty;   // nothing left to scale: the next values set the exponent
                        }
                    }
                }
                // this stripe's top row (lane 0's distance t - G + 1) for the stripe above
                if (s > 0) {
                    const int d = t - (G - 1);
                    T v[BW];
                    v[0] = bM[0];
                    if constexpr (AFF) { v[1] = bX[0]; v[2] = bY[0]; }
                    v[BW - 1] = exp_bits(EB, T(0));
                    if constexpr (G == 1) {
                        if (d >= 0) vstore<T, BW>(bb_out + int64_t(n - d) * BW, v);
                    } else {
                        if (lane == 0 && d >= 0) vstore<T, BW>(stw + (d & (G - 1)) * 4, v);
                        if (d >= 0 && ((d & (G - 1)) == G - 1 || d == tc1 - tc0)) {   // a full segment (or the last)
                            __syncwarp(gmask);
                            const int dd = d - (d & (G - 1)) + lane;
                            if (dd <= d) {
                                T w[BW];
                                vload<T, BW>(w, stw + lane * 4);
                                vstore<T, BW>(bb_out + int64_t(tc1 - dd) * BW, w);
                            }
                            __syncwarp(gmask);
                        }
                    }
                }
                // the row below of the next step's column: one exponent alignment for every lane
                if constexpr (G > 1) {
                    const T sM = __shfl_down_sync(gmask, bM[0], 1, G);
                    T sX = sM, sY = sM;
                    if constexpr (AFF) {
                        sX = __shfl_down_sync(gmask, bX[0], 1, G);
                        sY = __shfl_down_sync(gmask, bY[0], 1, G);
                    }
                    const int sE = __shfl_down_sync(gmask, EB, 1, G);
                    const int dn = t + 1;                 // lane G-1's next distance
                    if (s < nstripes - 1 && dn <= tc1 - tc0 && (dn & (G - 1)) == 0) {   // a new segment
                        stage_seg();
                        load_seg(dn + G);
                    }
                    const bool bot = lane == G - 1;
                    T v[BW];
                    vload<T, BW>(v, str + (dn & (G - 1)) * 4);
                    const int jn1 = tc1 - (t + 1) + (G - 1 - lane);   // this lane's next column
                    if (jn1 >= tc0 && jn1 <= tc1 && (!bot || s < nstripes - 1))
                        take_dn(bot ? v[0] : sM, bot ? (AFF ? v[1] : T(0)) : sX, bot ? (AFF ? v[2] : T(0)) : sY,
                                bot ? bits_exp(v[BW - 1]) : sE);
                } else {
                    if (s < nstripes - 1 && j > 0) {
                        take_dn(rb[0], AFF ? rb[1] : T(0), AFF ? rb[2] : T(0), bits_exp(rb[BW - 1]));
                        load_seg(n - j + 2);
                    }
                }
            }
            if constexpr (MW) publish(bkey * SP + S);
            if (TL && tc > 0) {   // this lane's state at the tile's first column, for the tile to its left
                T* const dst = colb_p + (int64_t(s) * ntc + tc) * G * LS + lane * LS;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    dst[NV * r] = bM[r];
                    if constexpr (AFF) { dst[NV * r + 1] = bX[r]; dst[NV * r + 2] = bY[r]; }
                }
                dst[LS - 1] = exp_bits(EB, T(0));
            }
            if constexpr (POST) {   // this stripe's rows are complete: their columns
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (i0 + r <= m) A.post[ao + p + i0 + r] = pcol[r];
            }
            if constexpr (!TR) {   // the stripe's gap sums into the pair's (double)
                gb_o += static_cast<double>(sgb_o); ga_o += static_cast<double>(sga_o);
                gb_x += static_cast<double>(sgb_x); ga_x += static_cast<double>(sga_x);
            }
            // fold this stripe's per-lane substitution counts into the pair's histogram (one
            // lane per pair: straight into the pair's gradient, zeroed before the pass)
            if constexpr (G == 1) {
                double* g1 = A.grad + A.gstride * p;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if (krow[r] >= K * N) continue;
                    for (int c = 0; c < N; ++c) {
                        T& v = macc[(size_t(c) * G + lane) * R + r];
                        if (v != T(0)) { g1[krow[r] * N + c] += static_cast<double>(v); cnt_nf |= !is_finite(v); }
                        v = T(0);
                    }
                }
            }
            if constexpr (G > 1) {
                // lane c adds column c of every (lane, row) accumulator, in (lane, row) order:
                // the sum's order (and bits) never depends on scheduling, and the group's lanes
                // work on distinct histogram entries at once
                __syncwarp(gmask);
                for (int l = 0; l < G; ++l) {
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const int kr = __shfl_sync(gmask, krow[r], l, G);
                        if (kr < K * N) {
                            for (int c = lane; c < N; c += G) {
                                T& v = macc[(size_t(c) * G + l) * R + r];
                                hist[kr * N + c] += v;
                                v = T(0);
                            }
                        }
                    }
                }
                __syncwarp(gmask);
            }
        }
        if constexpr (POST) {   // the rows' columns as a guide: non-decreasing, in [0, n]
            __syncwarp(gmask);
            if (lane == 0) {
                int32_t* gp = A.post + ao + p;
                int run = 0;
                for (int i = 0; i <= m; ++i) { run = max(run, min(max(gp[i], 0), n)); gp[i] = run; }
            }
            __syncwarp(gmask);
        }
        if constexpr (kCount) {
            // the group's lost-mass charge (every lane's, in any order: a bound, not a result)
            if constexpr (G > 1) {
#pragma unroll
                for (int off = G / 2; off > 0; off >>= 1) lacc += __shfl_xor_sync(gmask, lacc, off, G);
            }
        }
        if constexpr (!TR && G > 1) {
#pragma unroll
            for (int off = G / 2; off > 0; off >>= 1) {
                ga_o += __shfl_xor_sync(gmask, ga_o, off, G);
                ga_x += __shfl_xor_sync(gmask, ga_x, off, G);
                gb_o += __shfl_xor_sync(gmask, gb_o, off, G);
                gb_x += __shfl_xor_sync(gmask, gb_x, off, G);
            }
        }
        if constexpr (TL) {
            // the tile's counts into its stripe's partial (the stripe's tiles run one launch after
            // another, right to left: a fixed order), its gap sums and lost-mass charge after them
            const int64_t NNt = int64_t(K) * N * N;
            double* sp = A.spart + (A.stripe_off[p] + ts) * (A.gstride + 1);
            __syncwarp(gmask);
            for (int k = lane; k < K * N * N; k += G) { sp[k] += static_cast<double>(hist[k]); hist[k] = T(0); }
            if (lane == 0) {
                sp[NNt + 0] += ga_o; sp[NNt + 1] += ga_x; sp[NNt + 2] += gb_o; sp[NNt + 3] += gb_x;
                if constexpr (kCount) sp[A.gstride] += static_cast<double>(lacc);
            }
            why = __reduce_or_sync(gmask, why);
            if (why && lane == 0) atomicOr(A.status + p, why);
            __syncwarp(gmask);
            continue;
        }
        double* g = A.grad + A.gstride * p;
        const int64_t NN = int64_t(K) * N * N;
        // counts that left the range of T (a scale factor that overflowed where a product with
        // it was zero) refuse the pair like any other overflow: the host reruns it in double
        {
            bool nf = false;
            if constexpr (G > 1) { for (int k = lane; k < K * N * N; k += G) nf |= !is_finite(hist[k]); }
            else nf |= cnt_nf;
            if constexpr (!TR) nf |= !(is_finite(ga_o) && is_finite(ga_x) && is_finite(gb_o) && is_finite(gb_x));
            else { for (int k = 0; k < 4 * K; ++k) nf |= !is_finite(tg[k]); }
            if (nf) why |= kSoftCounts;
            if constexpr (G > 1) why = __reduce_or_sync(gmask, why);
        }
        if constexpr (MW) {
            // the pair's totals: every warp's histogram and gap sums, added in warp order
            stalled = __any_sync(gmask, stalled);
            if (lane == 0) {
                cpart[8 * gib + 0] = ga_o; cpart[8 * gib + 1] = ga_x;
                cpart[8 * gib + 2] = gb_o; cpart[8 * gib + 3] = gb_x;
                cpart[8 * gib + 4] = double(why); cpart[8 * gib + 5] = stalled ? 1.0 : 0.0;
                cpart[8 * gib + 6] = kCount ? static_cast<double>(lacc) : 0.0;
            }
            __syncthreads();
            double to_a = 0, tx_a = 0, to_b = 0, tx_b = 0, tl = 0;
            bool anystall = false;
            for (int w = 0; w < NWp; ++w) {
                to_a += cpart[8 * w + 0]; tx_a += cpart[8 * w + 1];
                to_b += cpart[8 * w + 2]; tx_b += cpart[8 * w + 3];
                why |= int(cpart[8 * w + 4]); anystall |= cpart[8 * w + 5] != 0.0;
                tl += cpart[8 * w + 6];
            }
            if (kCount && !(tl <= double(kLossMax))) why |= kSoftLoss;
            if (anystall || why) {
                if (threadIdx.x == 0) { A.status[p] = anystall ? kSoftStall : why; A.score[p] = 0.0; }
            } else {
                for (int k = threadIdx.x; k < K * N * N; k += blockDim.x) {
                    double v = 0.0;
                    for (int w = 0; w < NWp; ++w) v += static_cast<double>(hist_all[size_t(K) * N * N * w + k]);
                    g[k] = v;
                }
                if (threadIdx.x == 0) {
                    const double cga_o = AFF ? static_cast<double>(oa0) * to_a : 0.0;
                    const double cgb_o = AFF ? static_cast<double>(ob0) * to_b : 0.0;
                    g[NN + 0] = 0.0 - cga_o;
                    g[NN + 1] = 0.0 - (cga_o + static_cast<double>(ea0) * tx_a);
                    g[NN + 2] = 0.0 - cgb_o;
                    g[NN + 3] = 0.0 - (cgb_o + static_cast<double>(eb0) * tx_b);
                    A.status[p] = 0;
                    A.score[p] = A.temperature * (log(zhat) + double(EZ) * 0.69314718055994530942);
                }
            }
            stalled = false;
            __syncthreads();
        } else if (why || (kCount && !(lacc <= kLossMax))) {
            if (lane == 0) { A.status[p] = why | ((kCount && !(lacc <= kLossMax)) ? kSoftLoss : 0); A.score[p] = 0.0; }
        } else {
            if constexpr (G > 1)
                for (int k = lane; k < K * N * N; k += G) g[k] = static_cast<double>(hist[k]);
            if constexpr (TR) {
                for (int k = lane; k < 4 * K; k += G) g[NN + k] = 0.0;
                if constexpr (G > 1) __syncwarp(gmask);
                for (int k = 0; k < 4 * K; ++k) {
                    double v = tg[k];
                    if constexpr (G > 1) {
#pragma unroll
                        for (int off = G / 2; off > 0; off >>= 1) v += __shfl_xor_sync(gmask, v, off, G);
                    }
                    if (lane == 0) g[NN + k] = 0.0 - v;
                }
            } else {
                for (int k = lane; k < 4 * K; k += G) g[NN + k] = 0.0;
                if constexpr (G > 1) __syncwarp(gmask);
                if (lane == 0) {
                    // opens carry o = exp(-(go+ge)/T); an opening move also extends
                    const double cga_o = AFF ? static_cast<double>(oa0) * ga_o : 0.0;
                    const double cgb_o = AFF ? static_cast<double>(ob0) * gb_o : 0.0;
                    g[NN + 0] = 0.0 - cga_o;
                    g[NN + 1] = 0.0 - (cga_o + static_cast<double>(ea0) * ga_x);
                    g[NN + 2] = 0.0 - cgb_o;
                    g[NN + 3] = 0.0 - (cgb_o + static_cast<double>(eb0) * gb_x);
                }
            }
            if (lane == 0) {
                A.status[p] = 0;
                A.score[p] = A.temperature * (log(zhat) + double(EZ) * 0.69314718055994530942);
            }
        }
        if constexpr (G > 1) {
            __syncwarp(gmask);
            for (int k = lane; k < K * N * N; k += G) hist[k] = T(0);
        }
        if constexpr (TR) for (int k = 0; k < 4 * K; ++k) tg[k] = 0.0;
        if constexpr (G > 1) __syncwarp(gmask);
    }
}

// TL: per tiled pair, between the phases, Z (Local: the tiles' parts in tile order) and its
// range check; after the backward phase, the pair's counts (its stripes' partials in stripe
// order), score and status -- what the untiled kernel writes at the end of a pair.
struct TileSoftArgs {
    const int32_t* pairs; int64_t n_pairs;   // the tiled pairs
    const int64_t* tile_off; const int32_t* tiles_of;      // per pair / per listed pair
    const double* zpart; double* zpair;
    const int64_t* stripe_off; const int32_t* stripes_of;  // per pair / per listed pair
    const double* spart;
    const void* gw;                          // the pass's gap weights o_a, e_a, o_b, e_b in T
    int32_t* status; double* score; double* grad; int64_t gstride;
    int K, N, local, affine;
    double temperature;
};
template <class T>
__global__ void tile_z_kernel(const TileSoftArgs A) {   // one thread per pair
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= A.n_pairs) return;
    const int p = A.pairs[k];
    if (A.local) {
        XAcc za; za.init();
        for (int t = 0; t < A.tiles_of[k]; ++t) {
            const int64_t q = A.tile_off[p] + t;
            za.add(A.zpart[2 * q], int(A.zpart[2 * q + 1]));
        }
        A.zpair[2 * p] = za.m; A.zpair[2 * p + 1] = double(za.e);
    }
    const double zm = A.zpair[2 * p];
    if (!(zm > 0.0) || !(zm < 1e300)) A.status[p] |= kSoftZ;
}
template <class T>
__global__ void tile_finish_kernel(const TileSoftArgs A) {   // one block per pair
    const int64_t k = blockIdx.x;
    if (k >= A.n_pairs) return;
    const int p = A.pairs[k];
    const int ns = A.stripes_of[k];
    const int64_t NN = int64_t(A.K) * A.N * A.N;
    const int64_t rs = A.gstride + 1;
    const double* sp = A.spart + A.stripe_off[p] * rs;
    double* g = A.grad + A.gstride * p;
    const int32_t st0 = A.status[p];
    __shared__ int s_bad;
    if (threadIdx.x == 0) s_bad = 0;
    __syncthreads();
    if (st0 == 0) {
        for (int64_t q = threadIdx.x; q < NN; q += blockDim.x) {
            double v = 0.0;
            for (int s = 0; s < ns; ++s) v += sp[s * rs + q];
            if (!is_finite(v)) s_bad = 1;
            g[q] = v;
        }
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    int32_t why = st0;
    if (why == 0) {
        double ga_o = 0, ga_x = 0, gb_o = 0, gb_x = 0, tl = 0;
        for (int s = 0; s < ns; ++s) {
            const double* q = sp + s * rs + NN;
            ga_o += q[0]; ga_x += q[1]; gb_o += q[2]; gb_x += q[3];
            tl += sp[s * rs + A.gstride];
        }
        if (s_bad || !(is_finite(ga_o) && is_finite(ga_x) && is_finite(gb_o) && is_finite(gb_x))) why |= kSoftCounts;
        if (sizeof(T) == 4 && !(tl <= double(kLossMax))) why |= kSoftLoss;
        if (why == 0) {
            const T* gw = static_cast<const T*>(A.gw);
            // opens carry o = exp(-(go+ge)/T); an opening move also extends
            const double cga_o = A.affine ? static_cast<double>(gw[0]) * ga_o : 0.0;
            const double cgb_o = A.affine ? static_cast<double>(gw[2]) * gb_o : 0.0;
            g[NN + 0] = 0.0 - cga_o;
            g[NN + 1] = 0.0 - (cga_o + static_cast<double>(gw[1]) * ga_x);
            g[NN + 2] = 0.0 - cgb_o;
            g[NN + 3] = 0.0 - (cgb_o + static_cast<double>(gw[3]) * gb_x);
            const double zm = A.zpair[2 * p];
            const int ze = int(A.zpair[2 * p + 1]);
            const int EZ = ze + ilog2(zm);
            const double zhat = zm * pow2i<double>(ze - EZ);
            A.status[p] = 0;
            A.score[p] = A.temperature * (log(zhat) + double(EZ) * 0.69314718055994530942);
            return;
        }
    }
    A.status[p] = why;
    A.score[p] = 0.0;
}

}  // namespace nwg
