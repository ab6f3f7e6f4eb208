// C-ABI driver over the REFERENCE implementation (michalsta/nwgrad's header-only C++),
// TEST INFRASTRUCTURE ONLY: compiled by oracle/Makefile from the reference sources into
// oracle/_ref/ (never committed), to pin the CPU restatement in oracle.cpp and to time
// the reference's own CPU batch path as the baseline.  Nothing here is product code.
//
// Calls the reference's public C++ API only: SeqPairBatchT<T> (seq_pair_batch.hpp) with
// its constructor, score_and_grad / nwgrad_soft_score_and_grad, set_params, banded_grad,
// scores, grads_into, compute_grad, and the batch settings.
#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <string_view>
#include <vector>

#include "nwgrad/seq_pair_batch.hpp"
#include "nwgrad/batch_soft_defer.inl"

namespace {

thread_local std::string g_err;

struct Problem {
    int prec, gm, am, grad_mode, N, K;
    const double* mat;
    const double* gaps;
    const char* alphabet;
    int64_t n_pairs;
    const char* a; const int64_t* oa;
    const char* b; const int64_t* ob;
    const uint16_t* tracks; const uint16_t* gtracks;
    int traceback;   // 0 auto 1 pointers 2 scores 3 hirschberg 4 hirschberg_pmax 5 grid
    int kernel;      // -2 auto, -1 scalar
    int n_threads;
    double temperature;
    int soft_impl;   // 0 scaled 1 scaled_or_log 2 log
    int soft_f32;    // float32 batch: float32 soft pass first
    int hb_cutoff;
    int inter_fill;  // fill="interpair"
    int free_ends;   // am 2 (semi-global): kSgFree* bits (1 a_begin, 2 a_end, 4 b_begin, 8 b_end)
    int soft_guide;  // 0 eager, 1 lazy, 2 posterior
};

TracebackMode tb_of(int t) {
    switch (t) {
        case 1: return TracebackMode::Pointers;
        case 2: return TracebackMode::Scores;
        case 3: return TracebackMode::Hirschberg;
        case 4: return TracebackMode::HirschbergPmax;
        case 5: return TracebackMode::Grid;
        default: return TracebackMode::Default;
    }
}

AlignParams make_params(const Problem& P) {
    const Alphabet& al = Alphabet::get(P.alphabet);
    SubstMatrix sm(P.mat, al, P.K);
    return AlignParams(sm, P.gaps);
}

template <class T>
struct Run {
    std::vector<std::string_view> sa, sb;
    std::vector<size_t> toff, goff;
    std::unique_ptr<SeqPairBatchT<T>> batch;

    explicit Run(const Problem& P) {
        sa.resize(P.n_pairs); sb.resize(P.n_pairs);
        for (int64_t p = 0; p < P.n_pairs; ++p) {
            sa[p] = std::string_view(P.a + P.oa[p], size_t(P.oa[p + 1] - P.oa[p]));
            sb[p] = std::string_view(P.b + P.ob[p], size_t(P.ob[p + 1] - P.ob[p]));
        }
        PairTracks tk, gk;
        if (P.tracks) {
            toff.resize(P.n_pairs + 1);
            for (int64_t p = 0; p <= P.n_pairs; ++p) toff[p] = size_t(P.oa[p]);
            tk = PairTracks(P.tracks, toff.data(), size_t(P.n_pairs));
        }
        if (P.gtracks) {
            goff.resize(P.n_pairs + 1);
            for (int64_t p = 0; p <= P.n_pairs; ++p) goff[p] = size_t(P.oa[p] + p);
            gk = PairTracks(P.gtracks, goff.data(), size_t(P.n_pairs));
        }
        const GradMode gd = P.grad_mode == 0 ? GradMode::None : P.grad_mode == 1 ? GradMode::Hard : GradMode::Soft;
        batch = std::make_unique<SeqPairBatchT<T>>(
            sa, sb, make_params(P), P.gm == 0 ? GapModel::Linear : GapModel::Affine,
            P.am == 0 ? AlignMode::Global : P.am == 1 ? AlignMode::Local : AlignMode::Glocal, gd, P.n_threads, tb_of(P.traceback),
            P.kernel, tk, gk);
        if (P.grad_mode == 2) {
            batch->set_soft_temperature(P.temperature);
            batch->set_soft_impl(P.soft_impl == 2 ? SoftImpl::Log
                                 : P.soft_impl == 1 ? SoftImpl::ScaledOrLog : SoftImpl::Scaled);
            batch->set_soft_f32(P.soft_f32 != 0);
            batch->set_soft_guide(P.soft_guide == 1, P.soft_guide == 2);
        }
        if (P.am == 2) batch->set_free_ends(P.free_ends);
        if (P.hb_cutoff > 0) batch->set_hb_cutoff(P.hb_cutoff);
        batch->set_fill(false, P.inter_fill != 0);
    }
    double score_and_grad() {
        if (batch->grad_mode() == GradMode::Soft) return nwgrad_soft_score_and_grad(*batch, false);
        return batch->score_and_grad(false);
    }
    double banded(int bw) {
        if (batch->grad_mode() == GradMode::Soft) return nwgrad_soft_banded_grad(*batch, bw, false);
        return batch->banded_grad(bw, false);
    }
    void outputs(const Problem& P, double* scores, double* grads, int32_t* guides) {
        if (scores) {
            const std::vector<double> s = batch->scores();
            std::memcpy(scores, s.data(), s.size() * sizeof(double));
        }
        if (grads && P.grad_mode != 0) {
            const size_t nn = size_t(P.N) * P.N, K = size_t(P.K), n = size_t(P.n_pairs);
            std::vector<double> mats(n * K * nn), gp(n * K * 4);
            batch->grads_into(mats.data(), gp.data());
            const size_t gs = K * nn + 4 * K;
            for (size_t p = 0; p < n; ++p) {
                std::memcpy(grads + p * gs, mats.data() + p * K * nn, K * nn * sizeof(double));
                std::memcpy(grads + p * gs + K * nn, gp.data() + p * K * 4, K * 4 * sizeof(double));
            }
        }
        if (guides) {
            for (int64_t p = 0; p < P.n_pairs; ++p) {
                auto sp = (*batch)[size_t(p)];
                std::vector<int> g = sp.guide_j();
                for (size_t k = 0; k < g.size(); ++k) guides[P.oa[p] + p + int64_t(k)] = g[k];
            }
        }
    }
};

template <class F>
int guarded(F&& f) {
    try { f(); return 0; }
    catch (const std::exception& e) { g_err = e.what(); return 1; }
    catch (...) { g_err = "unknown exception"; return 1; }
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

// One score_and_grad() over the batch; per-pair scores, grads (K*N*N + 4*K each), guides
// (m + 1 each, at oa[p] + p).  band >= 0: then set_params(params2) + banded_grad(band) and
// the outputs are the banded ones.  total: the call's returned sum.
int ref_run(const Problem* P, const double* mat2, const double* gaps2, int band,
            double* scores, double* grads, int32_t* guides, double* total) {
    return guarded([&] {
        auto go = [&](auto tag) {
            using T = decltype(tag);
            Run<T> r(*P);
            double s = r.score_and_grad();
            if (band >= 0) {
                Problem Q = *P;
                Q.mat = mat2; Q.gaps = gaps2;
                r.batch->set_params(make_params(Q));
                s = r.banded(band);
            }
            if (total) *total = s;
            r.outputs(*P, scores, grads, guides);
        };
        if (P->prec == 32) go(float{}); else go(double{});
    });
}

// The CPU-baseline timing: construct once (untimed), `warmup` untimed passes, then `reps`
// timed passes of score_and_grad() + compute_grad(); returns every pass's seconds.
int ref_time(const Problem* P, int warmup, int reps, double* secs, double* total) {
    return guarded([&] {
        auto go = [&](auto tag) {
            using T = decltype(tag);
            Run<T> r(*P);
            for (int w = 0; w < warmup; ++w) { r.score_and_grad(); if (P->grad_mode) (void)r.batch->compute_grad(); }
            for (int k = 0; k < reps; ++k) {
                const auto t0 = std::chrono::steady_clock::now();
                const double s = r.score_and_grad();
                if (P->grad_mode) (void)r.batch->compute_grad();
                secs[k] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
                if (total) *total = s;
            }
        };
        if (P->prec == 32) go(float{}); else go(double{});
    });
}

// Resolved worker count and the SIMD level the reference dispatched to.
int ref_info(int n_threads, int* resolved, char* isa, int isa_cap) {
    return guarded([&] {
        BatchSettings s;
        s.set_n_threads(n_threads);
        *resolved = s.n_threads;
        const std::string lv = get_isa_level();
        std::snprintf(isa, size_t(isa_cap), "%s", lv.c_str());
    });
}

}  // extern "C"
