// Serving: a continuous-batching request loop over the store API.
//
// Requests (each a small batch of pairs: codes + offsets on the host) are queued on submit.
// W worker threads each own a store, reused from batch to batch (nwg_store_load), and a
// non-blocking CUDA stream.  A free worker takes the queue's head requests that share one
// parameter snapshot, as many as its pair and memory budgets admit (memory is estimated from
// the pairs' DP sizes and charged against one server-wide HBM budget until the batch ends),
// concatenates them into one batch, aligns it, and reads each request's scores and summed
// gradient back over the request's own pair range (nwg_scores_range / nwg_reduce_range), so
// a request's results are the same bits alone or in any mix.  Requests that arrive while
// others run are admitted as soon as a worker and memory free up; the workers' batches run
// concurrently on the device.  Latency = result ready - submit, per request.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/nwgrad_b200.h"

namespace {

using Clock = std::chrono::steady_clock;
thread_local std::string g_serr;

struct Params {
    std::vector<double> mats, gaps;
    int K = 1, N = 0;
    int64_t version = 0;
};

struct Request {
    int64_t id = 0;
    std::vector<uint8_t> a, b;
    std::vector<int64_t> oa, ob;   // rebased to 0
    int64_t n_pairs = 0;
    double cells = 0, bytes = 0;
    std::shared_ptr<const Params> params;
    Clock::time_point t_submit, t_done;
    // results
    std::vector<double> scores, grad;
    bool done = false;
    int status = 0;
    std::string err;
};

}  // namespace

struct nwg_server {
    int device = 0;
    nwg_job job{};
    int nalpha = 0;
    int64_t budget = 0;            // bytes of device memory the in-flight batches may hold
    int64_t scratch_share = 0;     // soft: bytes of forward tables one worker's batch may hold
    int64_t max_batch_pairs = 0;
    std::shared_ptr<const Params> params;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Request>> pending;
    std::unordered_map<int64_t, std::shared_ptr<Request>> live;
    int64_t next_id = 1;
    int64_t in_flight_bytes = 0;
    bool stop = false;
    std::vector<std::thread> workers;
    // statistics
    std::vector<double> latencies_ms;
    double cells_done = 0;
    int64_t batches = 0;
    // device intervals of the batches (ms from ev_ref): how much the workers' batches overlap
    cudaEvent_t ev_ref = nullptr;
    std::vector<std::pair<double, double>> dev_iv;
    Clock::time_point t0;
    bool started = false;
};

namespace {

// Device bytes a request's pairs hold while aligned: codes and per-pair results, plus the
// code table (hard) or the forward table (soft) of its largest pairs.
double request_bytes(const nwg_job& J, const std::vector<int64_t>& oa, const std::vector<int64_t>& ob, int N, int K) {
    double b = 0;
    const int64_t n = int64_t(oa.size()) - 1;
    for (int64_t p = 0; p < n; ++p) {
        const double m = double(oa[p + 1] - oa[p]), nn = double(ob[p + 1] - ob[p]);
        b += m + nn + 64 + 8.0 * (double(K) * N * N + 4 * K) + 4 * (m + 1);
        // hard: the code table (1 byte a cell); soft: the forward tables live in the worker's
        // scratch, which has its own cap (the budget's share of one worker)
        if (J.grad_mode != 2) b += 1.2 * (m + 64) * (nn + 40);
    }
    return b;
}

void run_batch(nwg_server* S, nwg_store*& store, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1,
               std::vector<std::shared_ptr<Request>>& reqs) {
    // concatenate the requests' pairs
    std::vector<uint8_t> a, b;
    std::vector<int64_t> oa{0}, ob{0};
    std::vector<int64_t> first;
    for (auto& r : reqs) {
        first.push_back(int64_t(oa.size()) - 1);
        for (int64_t p = 0; p < r->n_pairs; ++p) {
            oa.push_back(oa.back() + (r->oa[p + 1] - r->oa[p]));
            ob.push_back(ob.back() + (r->ob[p + 1] - r->ob[p]));
        }
        a.insert(a.end(), r->a.begin(), r->a.end());
        b.insert(b.end(), r->b.begin(), r->b.end());
    }
    first.push_back(int64_t(oa.size()) - 1);
    const int64_t n = int64_t(oa.size()) - 1;
    if (a.empty()) a.push_back(0);
    if (b.empty()) b.push_back(0);
    const Params& P = *reqs.front()->params;
    int rc = NWG_OK;
    std::string err;
    auto ck = [&](int r) { if (r != NWG_OK && rc == NWG_OK) { rc = r; err = nwg_last_error(); } return r == NWG_OK; };
    if (!store) {
        if (!ck(nwg_store_create(a.data(), oa.data(), b.data(), ob.data(), n, S->nalpha, nullptr, nullptr, S->device, &store)))
            store = nullptr;
        else {
            ck(nwg_set_memory(store, S->scratch_share, -1));
            // every served batch is a new plan: a captured sequence would never replay, and a
            // capture must not overlap the other workers' synchronising calls
            ck(nwg_set_graphs(store, 0));
        }
    } else {
        ck(nwg_store_load(store, a.data(), oa.data(), b.data(), ob.data(), n, nullptr, nullptr, st));
    }
    double total = 0;
    if (rc == NWG_OK) ck(nwg_params_set(store, P.mats.data(), P.gaps.data(), P.K, P.N));
    cudaEventRecord(e0, st);
    if (rc == NWG_OK) ck(nwg_run(store, &S->job, st, &total));
    cudaEventRecord(e1, st);
    const int64_t gs = int64_t(P.K) * P.N * P.N + 4 * P.K;
    for (size_t k = 0; k < reqs.size(); ++k) {
        auto& r = reqs[k];
        r->scores.assign(size_t(r->n_pairs), 0.0);
        r->grad.assign(S->job.grad_mode ? size_t(gs) : 0, 0.0);
        if (rc == NWG_OK && r->n_pairs) ck(nwg_scores_range(store, first[k], first[k + 1], r->scores.data()));
        if (rc == NWG_OK && S->job.grad_mode && r->n_pairs)
            ck(nwg_reduce_range(store, first[k], first[k + 1], nullptr, r->grad.data()));
    }
    float ms0 = 0, ms1 = 0;
    const bool timed = cudaEventSynchronize(e1) == cudaSuccess && S->ev_ref &&
                       cudaEventElapsedTime(&ms0, S->ev_ref, e0) == cudaSuccess &&
                       cudaEventElapsedTime(&ms1, S->ev_ref, e1) == cudaSuccess;
    const auto now = Clock::now();
    std::lock_guard<std::mutex> lk(S->mu);
    if (timed) S->dev_iv.emplace_back(double(ms0), double(ms1));
    for (auto& r : reqs) {
        r->status = rc;
        r->err = err;
        r->t_done = now;
        r->done = true;
        S->latencies_ms.push_back(std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count());
        S->cells_done += r->cells;
    }
    S->batches++;
    S->cv_done.notify_all();
}

void worker_main(nwg_server* S) {
    cudaSetDevice(S->device);
    cudaStream_t st = nullptr;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    nwg_store* store = nullptr;
    while (true) {
        std::vector<std::shared_ptr<Request>> take;
        double bytes = 0;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_work.wait(lk, [&] {
                if (S->stop) return true;
                if (S->pending.empty()) return false;
                // admit the head request when it fits the memory left (or nothing else is in flight)
                const double hb = S->pending.front()->bytes;
                return S->in_flight_bytes == 0 || S->in_flight_bytes + hb <= S->budget;
            });
            if (S->stop && S->pending.empty()) break;
            if (S->pending.empty()) continue;
            const Params* pv = S->pending.front()->params.get();
            int64_t pairs = 0;
            while (!S->pending.empty()) {
                auto& r = S->pending.front();
                if (r->params.get() != pv) break;                       // one parameter snapshot per batch
                if (!take.empty() && pairs + r->n_pairs > S->max_batch_pairs) break;
                if (!take.empty() && S->in_flight_bytes + bytes + r->bytes > S->budget) break;
                pairs += r->n_pairs;
                bytes += r->bytes;
                take.push_back(r);
                S->pending.pop_front();
            }
            S->in_flight_bytes += int64_t(bytes);
        }
        run_batch(S, store, st, e0, e1, take);
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->in_flight_bytes -= int64_t(bytes);
        }
        S->cv_work.notify_all();
    }
    if (store) nwg_store_destroy(store);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
}

template <class F>
int sguard(F&& f) {
    try { return f(); }
    catch (const std::exception& e) { g_serr = e.what(); return NWG_EINVAL; }
    catch (...) { g_serr = "unknown error"; return NWG_EINVAL; }
}

}  // namespace

extern "C" {

const char* nwg_server_last_error(void) { return g_serr.c_str(); }

int nwg_server_create(int device, const nwg_job* job, int nalpha, const double* mats, const double* gaps,
                      int K, int workers, int64_t hbm_budget_bytes, int64_t max_batch_pairs, nwg_server** out) {
    return sguard([&]() -> int {
        if (!job || !mats || !gaps || !out || nalpha < 1 || K < 1 || workers < 1)
            { g_serr = "nwg_server_create: bad argument"; return NWG_EINVAL; }
        if (job->band >= 0) { g_serr = "nwg_server_create: a server runs full alignments (band -1)"; return NWG_EINVAL; }
        auto S = std::make_unique<nwg_server>();
        S->device = device;
        S->job = *job;
        S->nalpha = nalpha;
        S->budget = hbm_budget_bytes > 0 ? hbm_budget_bytes : (int64_t(32) << 30);
        S->max_batch_pairs = max_batch_pairs > 0 ? max_batch_pairs : 65536;
        // half the budget for the workers' forward tables, the rest for the batches themselves
        S->scratch_share = std::max<int64_t>(S->budget / (2 * int64_t(workers)), int64_t(64) << 20);
        auto P = std::make_shared<Params>();
        P->K = K; P->N = nalpha;
        P->mats.assign(mats, mats + size_t(K) * nalpha * nalpha);
        P->gaps.assign(gaps, gaps + size_t(4) * K);
        S->params = P;
        S->t0 = Clock::now();
        cudaSetDevice(device);
        if (cudaEventCreate(&S->ev_ref) == cudaSuccess) {
            cudaEventRecord(S->ev_ref, nullptr);
            cudaEventSynchronize(S->ev_ref);
        } else {
            S->ev_ref = nullptr;
        }
        nwg_server* raw = S.get();
        for (int w = 0; w < workers; ++w) S->workers.emplace_back(worker_main, raw);
        *out = S.release();
        return NWG_OK;
    });
}

int nwg_server_set_params(nwg_server* S, const double* mats, const double* gaps, int K) {
    return sguard([&]() -> int {
        if (!S || !mats || !gaps) { g_serr = "null argument"; return NWG_EINVAL; }
        std::lock_guard<std::mutex> lk(S->mu);
        if (K != S->params->K) { g_serr = "set_params() cannot change the number of parameter sets"; return NWG_EINVAL; }
        auto P = std::make_shared<Params>(*S->params);
        P->mats.assign(mats, mats + size_t(K) * S->nalpha * S->nalpha);
        P->gaps.assign(gaps, gaps + size_t(4) * K);
        P->version = S->params->version + 1;
        S->params = P;
        return NWG_OK;
    });
}

int nwg_server_submit(nwg_server* S, const uint8_t* codes_a, const int64_t* off_a, const uint8_t* codes_b,
                      const int64_t* off_b, int64_t n_pairs, int64_t* ticket) {
    return sguard([&]() -> int {
        if (!S || !ticket || n_pairs < 0) { g_serr = "bad argument"; return NWG_EINVAL; }
        auto r = std::make_shared<Request>();
        r->t_submit = Clock::now();
        r->n_pairs = n_pairs;
        r->oa.resize(size_t(n_pairs) + 1);
        r->ob.resize(size_t(n_pairs) + 1);
        for (int64_t p = 0; p <= n_pairs; ++p) { r->oa[p] = off_a[p] - off_a[0]; r->ob[p] = off_b[p] - off_b[0]; }
        r->a.assign(codes_a + off_a[0], codes_a + off_a[n_pairs]);
        r->b.assign(codes_b + off_b[0], codes_b + off_b[n_pairs]);
        for (uint8_t c : r->a) if (c >= S->nalpha) { g_serr = "code out of range in sequence A"; return NWG_EINVAL; }
        for (uint8_t c : r->b) if (c >= S->nalpha) { g_serr = "code out of range in sequence B"; return NWG_EINVAL; }
        for (int64_t p = 0; p < n_pairs; ++p) r->cells += double(r->oa[p + 1] - r->oa[p]) * double(r->ob[p + 1] - r->ob[p]);
        {
            std::lock_guard<std::mutex> lk(S->mu);
            r->params = S->params;
            r->bytes = request_bytes(S->job, r->oa, r->ob, S->nalpha, S->params->K);
            r->id = S->next_id++;
            if (!S->started) { S->t0 = r->t_submit; S->started = true; }
            S->live[r->id] = r;
            S->pending.push_back(r);
            *ticket = r->id;
        }
        S->cv_work.notify_one();
        return NWG_OK;
    });
}

int nwg_server_wait(nwg_server* S, int64_t ticket, double* scores, double* grad, double* latency_ms) {
    return sguard([&]() -> int {
        std::shared_ptr<Request> r;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            auto it = S->live.find(ticket);
            if (it == S->live.end()) { g_serr = "unknown ticket"; return NWG_EINVAL; }
            r = it->second;
            S->cv_done.wait(lk, [&] { return r->done; });
            S->live.erase(it);
        }
        if (r->status != NWG_OK) { g_serr = r->err; return r->status; }
        if (scores) std::memcpy(scores, r->scores.data(), r->scores.size() * sizeof(double));
        if (grad && !r->grad.empty()) std::memcpy(grad, r->grad.data(), r->grad.size() * sizeof(double));
        if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
        return NWG_OK;
    });
}

// Latency quantiles of the requests completed so far (nearest rank), throughput over the
// time since the first submit, and counts.
int nwg_server_stats(nwg_server* S, double* p50_ms, double* p99_ms, double* gcups, int64_t* done, int64_t* batches) {
    return sguard([&]() -> int {
        std::lock_guard<std::mutex> lk(S->mu);
        std::vector<double> v = S->latencies_ms;
        std::sort(v.begin(), v.end());
        auto q = [&](double f) {
            if (v.empty()) return 0.0;
            size_t k = size_t(std::ceil(f * double(v.size()))) ;
            k = std::min(v.size(), std::max<size_t>(k, 1)) - 1;
            return v[k];
        };
        if (p50_ms) *p50_ms = q(0.50);
        if (p99_ms) *p99_ms = q(0.99);
        const double secs = std::chrono::duration<double>(Clock::now() - S->t0).count();
        if (gcups) *gcups = secs > 0 ? S->cells_done / secs / 1e9 : 0.0;
        if (done) *done = int64_t(v.size());
        if (batches) *batches = S->batches;
        return NWG_OK;
    });
}

// Device time of the completed batches: the union of their intervals (the device was busy
// with at least one batch) and the sum of their lengths; sum / union > 1 means batches of
// different workers ran on the device at the same time.
int nwg_server_device_stats(nwg_server* S, double* busy_ms, double* sum_ms, int64_t* batches) {
    return sguard([&]() -> int {
        std::vector<std::pair<double, double>> iv;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            iv = S->dev_iv;
        }
        std::sort(iv.begin(), iv.end());
        double uni = 0, sum = 0, cs = 0, ce = -1;
        for (auto& x : iv) {
            sum += x.second - x.first;
            if (x.first > ce) { if (ce > cs) uni += ce - cs; cs = x.first; ce = x.second; }
            else ce = std::max(ce, x.second);
        }
        if (ce > cs) uni += ce - cs;
        if (busy_ms) *busy_ms = uni;
        if (sum_ms) *sum_ms = sum;
        if (batches) *batches = int64_t(iv.size());
        return NWG_OK;
    });
}

int nwg_server_destroy(nwg_server* S) {
    return sguard([&]() -> int {
        if (!S) return NWG_OK;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->stop = true;
        }
        S->cv_work.notify_all();
        for (auto& t : S->workers) t.join();
        if (S->ev_ref) cudaEventDestroy(S->ev_ref);
        delete S;
        return NWG_OK;
    });
}

}  // extern "C"
