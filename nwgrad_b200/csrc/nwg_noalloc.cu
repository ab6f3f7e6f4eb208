// nwg_scores_noalloc: Viterbi scores of a batch without any device allocation.
//
// Who needs it: a host program that hands this library device memory it manages itself --
// a framework with its own caching allocator or a fixed per-plugin memory budget -- and
// does not let libraries call cudaMalloc (which also synchronises the device and can fail
// under that budget).  Such a caller allocates the inputs and the output; everything else
// this entry point needs lives in memory the library reserves when it is loaded.
//
// What it runs: the score-only form of the hard fill (the lane-strip wavefront of
// nwg_hard.cuh: one warp per pair, 4 rows per lane, float32, untracked), global or local,
// linear or affine.  Pairs longer than one stripe (128 rows of A) hand each stripe's bottom
// row to the next through a scratch row per warp; those rows are carved out of one
// file-scope device array of kScratchBytes (24 MiB), which every GPU that loads the library
// holds until the process exits.  Limits: sequence B of at most kMaxColumns (2047) residues,
// A of at most kMaxRows.  The scores are bit-identical to nwg_run's (same expressions, same
// order).  The substitution matrix and gap costs travel in the kernel's argument block (by
// value), so a call copies nothing from host memory.
//
// Calls share the scratch array: calls whose kernels overlap on the GPU (other streams, other
// host threads) race and give wrong scores; serialise them.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/nwgrad_b200.h"
#include "nwg_common.cuh"

namespace {

constexpr int kWarpsPerBlock = 4;
constexpr int kBlocks = 256;
constexpr int kSlots = kWarpsPerBlock * kBlocks;              // one scratch row per warp
constexpr int kMaxColumns = 2047;                             // columns of B a scratch row holds
constexpr size_t kRowFloats = 3 * (size_t(kMaxColumns) + 1);  // M, X, Y per column 0..n
constexpr size_t kScratchBytes = size_t(kSlots) * kRowFloats * sizeof(float);   // 24 MiB
constexpr int kMaxAlpha = 32;
constexpr int64_t kMaxRows = (int64_t(1) << 31) - 256;        // A: rows stay in int with the stripe padding
constexpr int R = 4;     // rows per lane
constexpr int G = 32;    // lanes per pair

static __device__ __align__(256) float g_noalloc_scratch[kSlots * kRowFloats];

// The call's parameters, passed by value in the launch's argument block (4112 bytes; kernels
// take up to 32 KB of arguments on sm_70 and later with CUDA 12.1+): the N*N matrix, then the
// four gap costs (open_a, extend_a, open_b, extend_b), float.
struct NoallocParams {
    float v[kMaxAlpha * kMaxAlpha + 4];
};

thread_local std::string g_err_na;
std::mutex g_mu;
float* g_scratch_ptr[64] = {};   // per device: g_noalloc_scratch's device address

template <bool AFF, bool LOC>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
score_fill_noalloc_kernel(const uint8_t* __restrict__ ca, const int64_t* __restrict__ oa,
                          const uint8_t* __restrict__ cb, const int64_t* __restrict__ ob,
                          int64_t n_pairs, int N, float* scratch, double* scores, const NoallocParams P) {
    using T = float;
    constexpr int GR = G * R;
    __shared__ T smat[kMaxAlpha * kMaxAlpha];
    for (int k = threadIdx.x; k < N * N; k += blockDim.x) smat[k] = P.v[k];
    __syncthreads();
    const T go_a = P.v[N * N + 0], ge_a = P.v[N * N + 1];
    const T go_b = P.v[N * N + 2], ge_b = P.v[N * N + 3];
    const int lane = threadIdx.x & 31;
    const int64_t slot = int64_t(blockIdx.x) * kWarpsPerBlock + threadIdx.x / 32;
    T* bnd = scratch + slot * kRowFloats;
    for (int64_t p = slot; p < n_pairs; p += int64_t(gridDim.x) * kWarpsPerBlock) {
        const int64_t ao = oa[p], bo = ob[p];
        const int64_t m64 = oa[p + 1] - ao, n64 = ob[p + 1] - bo;
        // a pair over the limits (the caller understated max_len_b, or A is over kMaxRows)
        // is not computed: its score is NaN
        const bool over = n64 > kMaxColumns || m64 > kMaxRows || m64 < 0 || n64 < 0;
        const int m = over ? 0 : int(m64), n = over ? 0 : int(n64);
        const uint8_t* ap = ca + ao;
        const uint8_t* bp = cb + bo;
        if (m == 0 || n == 0) {
            if (lane == 0) {
                double sc = 0.0;
                if (over) sc = __longlong_as_double(0x7ff8000000000000ll);   // NaN: over the limits
                else if (!LOC && m == 0 && n > 0)
                    sc = AFF ? -nwg::add_rn(go_a, nwg::mul_rn(T(n), ge_a)) : nwg::mul_rn(-T(n), ge_a);
                else if (!LOC && n == 0 && m > 0)
                    sc = AFF ? -nwg::add_rn(go_b, nwg::mul_rn(T(m), ge_b)) : nwg::mul_rn(-T(m), ge_b);
                scores[p] = sc;
            }
            continue;
        }
        const int nstripes = (m + GR - 1) / GR;
        const int S = n + G - 1;
        T bestv = T(0);
        T endM = nwg::ninf<T>(), endX = nwg::ninf<T>(), endY = nwg::ninf<T>();
        for (int s = 0; s < nstripes; ++s) {
            const int i0 = s * GR + lane * R + 1;
            int rowbase[R];
            T cM[R], cX[R], cY[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = i0 + r;
                const bool valid = i <= m;
                rowbase[r] = valid ? int(ap[i - 1]) * N : 0;
                if (LOC) { cM[r] = T(0); cX[r] = nwg::ninf<T>(); }
                else {
                    cX[r] = valid ? (AFF ? -nwg::add_rn(go_b, nwg::mul_rn(T(i), ge_b)) : nwg::mul_rn(-T(i), ge_b))
                                  : nwg::ninf<T>();
                    cM[r] = AFF ? nwg::ninf<T>() : cX[r];
                }
                cY[r] = nwg::ninf<T>();
            }
            T dgM, dgX, dgY;
            {
                const int i = i0 - 1;
                if (i == 0 || LOC) { dgM = T(0); dgX = nwg::ninf<T>(); dgY = nwg::ninf<T>(); }
                else {
                    dgX = AFF ? -nwg::add_rn(go_b, nwg::mul_rn(T(i), ge_b)) : nwg::mul_rn(-T(i), ge_b);
                    dgM = AFF ? nwg::ninf<T>() : dgX; dgY = nwg::ninf<T>();
                }
            }
            T upM = nwg::ninf<T>(), upX = nwg::ninf<T>(), upY = nwg::ninf<T>();
            for (int t = 0; t < S; ++t) {
                const int j = t - lane + 1;
                if (lane == 0 && j <= n) {
                    if (s == 0) {
                        if (LOC) { upM = T(0); upX = nwg::ninf<T>(); upY = nwg::ninf<T>(); }
                        else if (AFF) { upM = nwg::ninf<T>(); upX = nwg::ninf<T>(); upY = -nwg::add_rn(go_a, nwg::mul_rn(T(j), ge_a)); }
                        else upM = nwg::mul_rn(-T(j), ge_a);
                    } else {
                        upM = bnd[3 * j]; upX = bnd[3 * j + 1]; upY = bnd[3 * j + 2];
                    }
                }
                const bool active = j >= 1 && j <= n;
                if (active) {
                    const int bj = bp[j - 1];
                    T pM = dgM, pX = dgX, pY = dgY, qM = upM, qX = upX, qY = upY;
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const T sub = smat[rowbase[r] + bj];
                        if (AFF) {
                            T mv = nwg::rmax3(pM, pX, pY) + sub;
                            const T xv = nwg::rmax3((qM - go_b) - ge_b, qX - ge_b, (qY - go_b) - ge_b);
                            const T yv = nwg::rmax3((cM[r] - go_a) - ge_a, (cX[r] - go_a) - ge_a, cY[r] - ge_a);
                            if (LOC) {
                                mv = nwg::rmax(mv, T(0));
                                if (i0 + r <= m) bestv = nwg::rmax(bestv, nwg::rmax3(mv, xv, yv));
                            }
                            pM = cM[r]; pX = cX[r]; pY = cY[r];
                            cM[r] = mv; cX[r] = xv; cY[r] = yv;
                            qM = mv; qX = xv; qY = yv;
                        } else {
                            T v = nwg::rmax(nwg::rmax(pM + sub, qM - ge_b), cM[r] - ge_a);
                            if (LOC) {
                                v = nwg::rmax(v, T(0));
                                if (i0 + r <= m) bestv = nwg::rmax(bestv, v);
                            }
                            pM = cM[r];
                            cM[r] = v; qM = v;
                        }
                    }
                    dgM = upM; dgX = upX; dgY = upY;
                }
                const T sM = __shfl_up_sync(0xffffffffu, cM[R - 1], 1);
                const T sX = __shfl_up_sync(0xffffffffu, cX[R - 1], 1);
                const T sY = __shfl_up_sync(0xffffffffu, cY[R - 1], 1);
                if (lane > 0) { upM = sM; upX = sX; upY = sY; }
                if (lane == G - 1 && active && s + 1 < nstripes) {
                    bnd[3 * j] = cM[R - 1]; bnd[3 * j + 1] = cX[R - 1]; bnd[3 * j + 2] = cY[R - 1];
                }
            }
            if (!LOC && m >= i0 && m < i0 + R) {
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (i0 + r == m) { endM = cM[r]; endX = cX[r]; endY = cY[r]; }
            }
            __syncwarp();
        }
        if (LOC) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) bestv = nwg::rmax(bestv, __shfl_xor_sync(0xffffffffu, bestv, off));
            if (lane == 0) scores[p] = double(bestv);
        } else {
            const int src = ((m - 1) % GR) / R;
            endM = __shfl_sync(0xffffffffu, endM, src);
            endX = __shfl_sync(0xffffffffu, endX, src);
            endY = __shfl_sync(0xffffffffu, endY, src);
            if (lane == 0) scores[p] = AFF ? double(nwg::rmax3(endM, endX, endY)) : double(endM);
        }
    }
}

int fail(int code, const std::string& msg) { g_err_na = msg; return code; }

}  // namespace

extern "C" {

const char* nwg_noalloc_last_error(void) { return g_err_na.c_str(); }

int nwg_scores_noalloc(const uint8_t* codes_a, const int64_t* off_a, const uint8_t* codes_b,
                       const int64_t* off_b, int64_t n_pairs, int max_len_b, int nalpha,
                       const double* mat, const double* gaps, int gap_model, int mode,
                       double* scores, void* stream) {
    if (n_pairs < 0 || nalpha < 1 || nalpha > kMaxAlpha || !mat || !gaps || (n_pairs && (!codes_a || !off_a || !codes_b || !off_b || !scores)))
        return fail(NWG_EINVAL, "nwg_scores_noalloc: bad argument (alphabet size 1..32, non-null pointers)");
    if (max_len_b < 0 || max_len_b > kMaxColumns)
        return fail(NWG_EINVAL, "nwg_scores_noalloc: sequence B longer than " + std::to_string(kMaxColumns) +
                                    " residues (the reserved scratch's limit); use nwg_run");
    if (gap_model < 0 || gap_model > 1 || mode < 0 || mode > 1)
        return fail(NWG_EINVAL, "nwg_scores_noalloc: gap_model and mode must be 0 or 1");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) return fail(NWG_ECUDA, "nwg_scores_noalloc: no current device");
    float* scratch;
    {
        // set-up, once per device, with that device current: the array's device address
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_scratch_ptr[dev]) {
            void* ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess || !ptr)
                return fail(NWG_ECUDA, std::string("nwg_scores_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_scratch_ptr[dev] = static_cast<float*>(ptr);
        }
        scratch = g_scratch_ptr[dev];
    }
    NoallocParams P{};
    for (int k = 0; k < nalpha * nalpha; ++k) P.v[k] = static_cast<float>(mat[k]);
    for (int k = 0; k < 4; ++k) P.v[nalpha * nalpha + k] = static_cast<float>(gaps[k]);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (n_pairs == 0) return NWG_OK;
    const dim3 grid(kBlocks), block(kWarpsPerBlock * 32);
    if (gap_model == 1) {
        if (mode == 1) score_fill_noalloc_kernel<true, true><<<grid, block, 0, st>>>(codes_a, off_a, codes_b, off_b, n_pairs, nalpha, scratch, scores, P);
        else score_fill_noalloc_kernel<true, false><<<grid, block, 0, st>>>(codes_a, off_a, codes_b, off_b, n_pairs, nalpha, scratch, scores, P);
    } else {
        if (mode == 1) score_fill_noalloc_kernel<false, true><<<grid, block, 0, st>>>(codes_a, off_a, codes_b, off_b, n_pairs, nalpha, scratch, scores, P);
        else score_fill_noalloc_kernel<false, false><<<grid, block, 0, st>>>(codes_a, off_a, codes_b, off_b, n_pairs, nalpha, scratch, scores, P);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(NWG_ECUDA, std::string("nwg_scores_noalloc: launch: ") + cudaGetErrorString(e));
    return NWG_OK;
}

}  // extern "C"
