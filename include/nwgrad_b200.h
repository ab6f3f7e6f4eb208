/* nwgrad_b200 -- C ABI of the B200 SeqPairBatch alignment path.
 *
 * One opaque store holds a batch of sequence pairs resident on one GPU (encoded codes,
 * offsets, tracks), its parameters and its per-pair results; every entry point takes plain
 * pointers and sizes and returns a status (0 = NWG_OK).  No C++ exception crosses this
 * boundary; nwg_last_error() describes the last failure on the calling thread.
 *
 * Each entry point replaces one call of the reference's batch engine
 * (michalsta/nwgrad, src/nwgrad/cpp/nwgrad/batch_engine.hpp), cited beside it.
 */
#ifndef NWGRAD_B200_H
#define NWGRAD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    NWG_OK = 0,
    NWG_EINVAL = 1,    /* bad argument (a foreign code, a track entry out of range, ...) -> ValueError */
    NWG_ECUDA = 2,     /* a CUDA call failed */
    NWG_ENOMEM = 3,    /* device memory exhausted */
    NWG_ESTATE = 4,    /* results not computed / no guide -> RuntimeError */
    NWG_ERANGE = 5     /* soft path: a pair does not fit the scaled forward-backward -> ValueError */
};

typedef struct nwg_store nwg_store;

typedef struct nwg_job {
    int gap_model;     /* 0 linear, 1 affine */
    int mode;          /* 0 global, 1 local, 2 semi-global (free_ends) */
    int grad_mode;     /* 0 none (score only), 1 hard, 2 soft */
    int precision;     /* 32 float32 DP, 64 float64 DP */
    int band;          /* -1: full DP; >= 1: guide-banded re-alignment of this half-width */
    int keep_paths;    /* hard: also keep every pair's path (moves) */
    double temperature;/* soft: T > 0 */
    int soft_double;   /* soft, precision 32: 0 float32 pass first (refused pairs rerun in double), 1 double only */
    int lanes;         /* 0 auto; else lanes per pair (1 or 32) for every pair (tuning) */
    int rows;          /* 0 auto; else rows per lane (tuning) */
    int traceback;     /* hard, affine Global, untracked: 3 hirschberg, 4 hirschberg_pmax (pairs
                          longer than hb_cutoff rows split); 5 grid (full DP, Global or Local:
                          pairs of 1536+ rows and 256+ columns keep a grid of rows and columns
                          and refill the tiles their path crosses, the Pointers result bit for
                          bit); anything else the Pointers path */
    int hb_cutoff;     /* Hirschberg base-case rows (>= 1; 0: 512) */
    int free_ends;     /* mode 2 (semi-global, the reference's AlignMode::Glocal with kSgFree*
                          bits, simd_levels.hpp:170-182): 1 a_begin (column 0 a free start),
                          2 a_end (column n's cells ends), 4 b_begin (row 0 a free start),
                          8 b_end (row m's cells ends); "glocal" is 12, "overlap" 15.  Traceback
                          Pointers; banded re-alignment with 12 only (aligner.hpp:2222-2231) */
    int soft_post;     /* soft, full DP, untracked: 1 also leave every pair's posterior guide
                          (soft_guide="posterior", aligner.hpp:6776-6808, 1466-1475) for
                          nwg_guides and a later banded run */
} nwg_job;

/* Last error message of the calling thread ("" if none). */
const char* nwg_last_error(void);

/* Build a store: upload n_pairs pairs (codes of A and B, concatenated, with n_pairs + 1
 * int64 offsets each), every code < nalpha.  tracks: per residue of A (off_a offsets) or
 * NULL; gap_tracks: per DP row, m + 1 per pair at off_a[p] + p, or NULL.  The host buffers
 * may be reused once the call returns.  Codes in pinned host memory (cudaHostAlloc, a torch
 * pin_memory tensor) upload at DMA speed; pageable ones go through the driver's staging (a
 * store of 60 MB of codes: about 9.5 ms from pageable buffers, about 6 ms from pinned ones on
 * a B200 host, the rest being the code check and the offsets).
 * Replaces BatchEngine's constructor (batch_engine.hpp:284-350). */
int nwg_store_create(const uint8_t* codes_a, const int64_t* off_a, const uint8_t* codes_b,
                     const int64_t* off_b, int64_t n_pairs, int nalpha, const uint16_t* tracks,
                     const uint16_t* gap_tracks, int device, nwg_store** out);
int nwg_store_destroy(nwg_store* s);

/* Replace a store's pairs (same alphabet), reusing its device buffers (they only grow): every
 * result, guide and plan of the previous pairs is dropped, the parameters stay.  The serving
 * loop's way to run one batch after another without reallocating.  No direct counterpart in
 * the reference (a batch there is built once); the equivalent of constructing a new batch. */
int nwg_store_load(nwg_store* s, const uint8_t* codes_a, const int64_t* off_a, const uint8_t* codes_b,
                   const int64_t* off_b, int64_t n_pairs, const uint16_t* tracks,
                   const uint16_t* gap_tracks, void* stream);

/* Parameters: K stacked N x N matrices (row-major) and K x 4 gaps (open_a, extend_a,
 * open_b, extend_b), copied.  Invalidates results, keeps guides.
 * Replaces BatchEngine::set_params (batch_engine.hpp:597-606). */
int nwg_params_set(nwg_store* s, const double* mats, const double* gaps, int K, int N);

/* Align every pair: scores, guides and (grad_mode 1/2) per-pair gradients, cached in the
 * store; *total = the sum of scores in pair order.  job->band >= 1 re-aligns inside a band
 * around each pair's stored guide.  stream: a cudaStream_t (NULL = the default stream).
 * Replaces BatchEngine::score_and_grad (batch_engine.hpp:615-629) and banded_grad (:633-653). */
int nwg_run(nwg_store* s, const nwg_job* job, void* stream, double* total);

/* Kernel geometry: pairs of a size class (max(20, ceil(log2(rows * columns)))) run with `lanes`
 * lanes per pair and `rows` DP rows per lane from now on (soft != 0: the soft path, else the
 * hard fill).  size_class -1 forgets every such choice (the planner picks per pair);
 * size_class -2 selects the plain fill (one fixed geometry, 32 lanes x 4 rows, for every
 * pair).  Results do not depend on the geometry.  No counterpart in the reference (its
 * kernel / fill choice is a CPU ISA dispatch). */
int nwg_set_geometry(nwg_store* s, int soft, int size_class, int lanes, int rows);

/* Kernel geometry by cost model: each pair of the size class runs with the geometry (lanes[k],
 * rows[k]) that minimises ns_per_cell[k] x the pair's padded cells (whole stripes of
 * lanes x rows DP rows, columns plus the lanes' skew) -- the autotuner's measured cost per
 * padded cell, so pairs whose rows fill stripes badly under one geometry take another.
 * Replaces a single geometry set for the class.  No counterpart in the reference. */
int nwg_set_geometry_costs(nwg_store* s, int soft, int size_class, int n, const int* lanes, const int* rows,
                           const double* ns_per_cell);

/* Device memory of soft runs: scratch_budget_bytes caps the forward tables one call holds
 * (fewer pairs run at once when they are large); a pair whose whole forward table would be
 * above checkpoint_bytes keeps only its stripe boundaries and recomputes each stripe just
 * before that stripe's backward (results are bit-identical either way).  A value < 0 keeps the
 * current setting (defaults: 60 % of the device memory free at the call -- the device's free
 * memory, the blocks the memory pool keeps idle and the store's own scratch -- at least 24 GiB;
 * and 16 MiB).  No counterpart in the reference (its CPU
 * path keeps a whole table per thread). */
int nwg_set_memory(nwg_store* s, int64_t scratch_budget_bytes, int64_t checkpoint_bytes);

/* Soft long pairs run with several warps per pair that wait on one another's progress; each wait
 * polls at most `polls` times (default 4194304, about a quarter second at the poll interval),
 * then the kernel marks the pair, finishes without waiting further and the call fails with
 * NWG_ECUDA ("a wait ... ran out") instead of hanging.  The store stays usable.  polls < 1 is
 * refused.  No counterpart in the reference (its CPU threads never wait on one another inside a
 * pair). */
int nwg_set_spin_limit(nwg_store* s, int polls);

/* Per-pair scores (n_pairs doubles).  Replaces BatchEngine::scores (batch_engine.hpp:689). */
int nwg_scores(nwg_store* s, double* out);

/* Per-pair gradients, n_pairs x (K*N*N + 4K) doubles: the K matrices then K x 4 gaps.
 * Replaces BatchEngine::grads_into (batch_engine.hpp:722-746). */
int nwg_grads(nwg_store* s, double* out);

/* sum_p w[p] * grad_p (w NULL: plain sum) into out (K*N*N + 4K doubles), in fixed blocks of
 * 4096 pairs: each block in pair order, the blocks in order -- the reference's order, so
 * bit-identical for identical per-pair gradients.
 * Replaces BatchEngine::weighted_grad / compute_grad (batch_engine.hpp:703-718, 1788-1827). */
int nwg_reduce(nwg_store* s, const double* w, double* out);

/* The reduction and scores of nwg_reduce / nwg_scores over the pairs [start, end) only, the
 * blocks of 4096 counted from start: a request's own gradient inside a served batch is the
 * same bits as when that request is a batch by itself.  (weighted_grad / scores over a view.) */
int nwg_reduce_range(nwg_store* s, int64_t start, int64_t end, const double* w, double* out);
int nwg_scores_range(nwg_store* s, int64_t start, int64_t end, double* out);

/* Guides (guide_j: m + 1 ints per pair at off_a[p] + p), read and written.
 * Replace SeqPair::guide_j (seq_pair_batch.hpp:236) and the guide a banded call bands around. */
int nwg_guides(nwg_store* s, int32_t* out);
int nwg_set_guides(nwg_store* s, const int32_t* in);

/* Compute every pair's guide under the given parameters (a snapshot: the params a soft
 * pass scored) with the hard fill, leaving the store's parameters and results untouched.
 * Replaces the deferred-guide resolution of the soft path (batch_soft_defer.inl:1-60, 241). */
int nwg_resolve_guides(nwg_store* s, const double* mats, const double* gaps, const nwg_job* job,
                       void* stream);

/* Kept paths (job.keep_paths): per pair the walk-order moves (0 M, 1 gap in B, 2 gap in A),
 * concatenated at the offsets given by path_info; path_info: n_pairs x 3 int32 = number of
 * moves, start_i, start_j; ends: n_pairs x 2 = end_i, end_j.
 * Replaces the stored path of BatchEngine (batch_engine.hpp:515-590). */
int nwg_paths(nwg_store* s, int64_t* moves_off, uint8_t* moves, int64_t moves_cap,
              int32_t* path_info, int32_t* ends);

/* Per-pair status of the last run: 0 ok, 1 refused by the float32 soft pass and rerun in
 * double, 2 out of range in double too.  Mirrors the kF32Refused flag (batch_engine.hpp:1285). */
int nwg_status(nwg_store* s, int32_t* out);

/* Device time (ms) of the last nwg_run's kernels and how many kernels it launched. */
int nwg_last_timing(nwg_store* s, double* ms, int64_t* launches);

/* Captured bucket sequences (no counterpart in the reference).  With graphs on (the default)
 * nwg_run runs a plan's per-bucket launches as one CUDA graph, captured on the first call and
 * replayed while the launches (kernels, shapes, arguments) are unchanged -- across set_params
 * steps, for one.  Results are the same either way.  nwg_graph_stats counts captures and
 * replays since the store was made. */
int nwg_set_graphs(nwg_store* s, int enable);
int nwg_graph_stats(nwg_store* s, int64_t* captures, int64_t* replays);

/* ── Serving: continuous batching (no counterpart in the reference, a CPU library with
 * no request loop; each request's results equal those of SeqPairBatch.score_and_grad +
 * compute_grad on its pairs alone, batch_engine.hpp:615, 714) ──────────────────────────
 * A server owns `workers` threads, each with a reusable store and stream.  Requests (host
 * codes + offsets, one parameter snapshot each: the params current at submit) queue on
 * submit; a free worker batches the queue's head requests within max_batch_pairs and the
 * server-wide hbm_budget_bytes (estimated from DP sizes), aligns them with `job`, and hands
 * every request its own scores and summed gradient (K*N*N + 4K doubles, the same bits as the
 * request aligned alone).  Batches of different workers run concurrently on the GPU. */
typedef struct nwg_server nwg_server;
int nwg_server_create(int device, const nwg_job* job, int nalpha, const double* mats, const double* gaps,
                      int K, int workers, int64_t hbm_budget_bytes, int64_t max_batch_pairs,
                      nwg_server** out);
int nwg_server_set_params(nwg_server* s, const double* mats, const double* gaps, int K);
int nwg_server_submit(nwg_server* s, const uint8_t* codes_a, const int64_t* off_a, const uint8_t* codes_b,
                      const int64_t* off_b, int64_t n_pairs, int64_t* ticket);
/* Block until the request is done; scores: n_pairs doubles; grad: K*N*N + 4K (grad_mode != 0). */
int nwg_server_wait(nwg_server* s, int64_t ticket, double* scores, double* grad, double* latency_ms);
/* Latency p50 / p99 (ms) of completed requests, throughput since the first submit. */
int nwg_server_stats(nwg_server* s, double* p50_ms, double* p99_ms, double* gcups, int64_t* done,
                     int64_t* batches);
/* Device time of the completed batches (CUDA events around each batch's run, on its worker's
 * stream): busy_ms the union of the intervals, sum_ms the sum of their lengths -- sum / busy > 1
 * means batches of different workers were on the device at the same time. */
int nwg_server_device_stats(nwg_server* s, double* busy_ms, double* sum_ms, int64_t* batches);
int nwg_server_destroy(nwg_server* s);
const char* nwg_server_last_error(void);

/* Viterbi scores of n_pairs pairs WITHOUT any device allocation (no counterpart in the
 * reference: it is a CPU library).  For callers whose host framework owns all device memory
 * (its own caching allocator or a fixed per-plugin budget) and forbids cudaMalloc, which also
 * synchronises the device.  All pointers but mat / gaps are device pointers the caller
 * allocated: codes and int64 offsets as nwg_store_create takes them, scores (n_pairs doubles)
 * the output.  mat (nalpha x nalpha, nalpha <= 32) and gaps (4) are host doubles.  The
 * float32 score-only fill of nwg_run (bit-identical scores), one parameter set, untracked.
 * Scratch comes from a 24 MiB array every GPU that loads the library reserves until exit;
 * limits: B at most 2047 residues (max_len_b states the batch's longest B; larger: NWG_EINVAL)
 * and A at most 2^31 - 256.  The offsets live on the device, so the call cannot check each
 * pair: a pair over either limit (max_len_b understated) gets a NaN score and the call still
 * returns NWG_OK.  The parameters travel by value in the kernel launch (no host copy).
 * The first call on a device looks the array up (cudaGetSymbolAddress) -- make it before any
 * stream capture.  Calls share that array: calls whose kernels overlap on the GPU race.
 * Errors: nwg_noalloc_last_error(). */
int nwg_scores_noalloc(const uint8_t* codes_a, const int64_t* off_a, const uint8_t* codes_b,
                       const int64_t* off_b, int64_t n_pairs, int max_len_b, int nalpha,
                       const double* mat, const double* gaps, int gap_model, int mode,
                       double* scores, void* stream);
const char* nwg_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* NWGRAD_B200_H */
