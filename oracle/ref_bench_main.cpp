// Timing executable over the reference driver (ref_driver.cpp), TEST/BENCH INFRASTRUCTURE:
// bench.py's CPU-baseline leg runs the reference's SIMD batch path in this separate process
// (the reference's vectorised kernels fault when they run inside a Python process that has
// numpy loaded, so they are kept out of it).
//
//   nwref_bench <problem file>
//
// Problem file (little-endian): int32 prec, gm, am, grad_mode, N, K, n_threads, warmup, reps,
// kernel, free_ends; int64 n_pairs; int32 alphabet length, alphabet bytes; K*N*N doubles; K*4 doubles;
// (n_pairs + 1) int64 offsets of A, then the A characters; the same for B.
// Prints one JSON line: {"secs": [...], "total": T, "threads": n, "isa": "..."}.
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

struct Problem {
    int prec, gm, am, grad_mode, N, K;
    const double* mat; const double* gaps; const char* alphabet; int64_t n_pairs;
    const char* a; const int64_t* oa; const char* b; const int64_t* ob;
    const uint16_t* tracks; const uint16_t* gtracks;
    int traceback, kernel, n_threads; double temperature; int soft_impl, soft_f32, hb_cutoff, inter_fill;
    int free_ends;
};
extern "C" int ref_time(const Problem* P, int warmup, int reps, double* secs, double* total);
extern "C" int ref_info(int n_threads, int* resolved, char* isa, int isa_cap);
extern "C" const char* ref_last_error();

template <class T> static T rd(std::ifstream& f) { T v; f.read(reinterpret_cast<char*>(&v), sizeof v); return v; }

int main(int argc, char** argv) {
    if (argc < 2) { std::fprintf(stderr, "usage: nwref_bench <problem file>\n"); return 2; }
    std::ifstream f(argv[1], std::ios::binary);
    if (!f) { std::fprintf(stderr, "cannot open %s\n", argv[1]); return 2; }
    int h[11];
    for (int& x : h) x = rd<int32_t>(f);
    const int64_t n = rd<int64_t>(f);
    const int al = rd<int32_t>(f);
    std::string alpha(size_t(al), '\0');
    f.read(&alpha[0], al);
    const int N = h[4], K = h[5];
    std::vector<double> mat(size_t(K) * N * N), gaps(size_t(4) * K);
    f.read(reinterpret_cast<char*>(mat.data()), std::streamsize(mat.size() * 8));
    f.read(reinterpret_cast<char*>(gaps.data()), std::streamsize(gaps.size() * 8));
    std::vector<int64_t> oa(size_t(n) + 1), ob(size_t(n) + 1);
    f.read(reinterpret_cast<char*>(oa.data()), std::streamsize(oa.size() * 8));
    std::string A(size_t(oa.back()), '\0');
    f.read(&A[0], std::streamsize(A.size()));
    f.read(reinterpret_cast<char*>(ob.data()), std::streamsize(ob.size() * 8));
    std::string B(size_t(ob.back()), '\0');
    f.read(&B[0], std::streamsize(B.size()));
    if (!f) { std::fprintf(stderr, "truncated problem file\n"); return 2; }
    Problem P{h[0], h[1], h[2], h[3], N, K, mat.data(), gaps.data(), alpha.c_str(), n,
              A.c_str(), oa.data(), B.c_str(), ob.data(), nullptr, nullptr,
              0, h[9], h[6], 1.0, 0, 1, 0, 1, h[10]};
    const int reps = h[8];
    std::vector<double> secs(static_cast<size_t>(reps));
    double total = 0;
    if (ref_time(&P, h[7], reps, secs.data(), &total)) {
        std::fprintf(stderr, "reference error: %s\n", ref_last_error());
        return 1;
    }
    int thr = 0;
    char isa[64] = {0};
    ref_info(h[6], &thr, isa, 64);
    std::printf("{\"secs\": [");
    for (int k = 0; k < reps; ++k) std::printf("%s%.9f", k ? ", " : "", secs[size_t(k)]);
    std::printf("], \"total\": %.17g, \"threads\": %d, \"isa\": \"%s\"}\n", total, thr, isa);
    return 0;
}
