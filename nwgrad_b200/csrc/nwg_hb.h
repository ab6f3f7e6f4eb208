// Hirschberg re-alignment on the GPU (nwg_hb.cu): the host driver's interface.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace nwg {

// One Hirschberg run over a set of pairs (affine or linear, Global or Local, untracked, one
// parameter set).
struct HbRun {
    // device
    const uint8_t* a; const uint8_t* b;        // the store's codes
    const int64_t* oa; const int64_t* ob;      // the store's offsets
    const int32_t* pairs;                      // the pairs to run
    const void* mat; int N;                    // N x N in T
    double go_a, ge_a, go_b, ge_b;             // cast to T as the reference does
    double* score; int32_t* end;               // per pair
    double* grad; int64_t gstride;             // per pair, zeroed by the caller (or null)
    int32_t* guide;                            // per pair m + 1 at oa[p] + p (or null)
    uint8_t* moves; const int64_t* moves_off;  // keep_paths: walk-order moves (or null)
    int32_t* path_info;                        // per pair n_moves, start_i, start_j (or null)
    // host
    const int32_t* h_pairs; int64_t n_pairs;
    const int64_t* h_oa; const int64_t* h_ob;
    int cutoff;                                // rows at which blocks stop splitting (>= 1)
    int pmax;                                  // the closed-form prefix-max horizontal carry
    int local;                                 // Local: endpoint scans, then the box's global solve
    int glocal;                                // glocal ends (row 0 a free start, row m's cells ends):
                                               // the glocal endpoint scans, then the box's global solve
    int linear;                                // linear gaps (one state; pmax does not apply)
    // linear, tracked: K sets (mat K x N x N, gaps_t K x 4 in T), per residue of A its set,
    // per DP row its gap set (oa[p] + p offsets; null: the residue's set)
    int K;
    const void* gaps_t;
    const uint16_t* tracks; const uint16_t* gtracks;
    int64_t tile_budget;                       // bytes the tiled half-sweeps' rows and lane states may hold
};

// Runs P on stream st (synchronising it); returns the number of kernel launches.  Throws
// std::runtime_error on a CUDA error.
int64_t hb_run(const HbRun& P, int elem_bytes, cudaStream_t st, int sms);

}  // namespace nwg
