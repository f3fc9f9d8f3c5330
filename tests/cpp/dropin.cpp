// Drives the C++ drop-ins of include/apxb200.hpp the way the reference's
// call sites drive cuda_sptrsv and cuda_pcg (preconditioner.h:247-284,
// src/solve.cpp:687-729), on a system read from a binary file:
//   u32 n, u32 m, u32 sddm, u64 nnz_f, u32 colptr[n+1], u32 rowidx[nnz_f], f32 vals[nnz_f],
//   u32 perm[n], u32 n_rounds, u64 rounds[n_rounds],
//   u64 nnz_a, i32 a_colptr[n+1], i32 a_rowidx[nnz_a], f64 a_vals[nnz_a], f64 b[n], f64 y[m]
// and writes: f64 sweep[m] (solve_LLt of y), f64 x[n], i32 iters, f64 residual.
// Exit status: 0 ok, 2 a drop-in threw (message on stderr), 1 bad input.
#include <cstdio>
#include <fstream>
#include <vector>

#include "apxb200.hpp"

namespace {

struct csc {   // the reference's sparse_csc surface
    uint32_t n = 0;
    std::vector<uint32_t> outer, inner;
    std::vector<float> vals;
    uint32_t rows() const { return n; }
    const uint32_t* outerIndexPtr() const { return outer.data(); }
    const uint32_t* innerIndexPtr() const { return inner.data(); }
    const float* valuePtr() const { return vals.data(); }
};

struct spmat {   // Eigen::SparseMatrix<double> surface
    int n = 0;
    std::vector<int> outer, inner;
    std::vector<double> vals;
    int rows() const { return n; }
    long nonZeros() const { return static_cast<long>(vals.size()); }
    const int* outerIndexPtr() const { return outer.data(); }
    const int* innerIndexPtr() const { return inner.data(); }
    const double* valuePtr() const { return vals.data(); }
};

struct vec {     // Eigen::VectorXd surface
    std::vector<double> v;
    long size() const { return static_cast<long>(v.size()); }
    void resize(long k) { v.resize(static_cast<size_t>(k)); }
    const double* data() const { return v.data(); }
    double* data() { return v.data(); }
};

struct precond {   // apx_cholesky with the one accessor cuda_pcg needs
    apxb::cuda_sptrsv trsv;
    apxb_factor* trsv_handle() const { return trsv.handle(); }
};

template <class T>
bool rd(std::ifstream& f, T* p, size_t k) {
    return static_cast<bool>(f.read(reinterpret_cast<char*>(p), static_cast<std::streamsize>(sizeof(T) * k)));
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) { std::fprintf(stderr, "usage: dropin <in.bin> <out.bin>\n"); return 1; }
    std::ifstream f(argv[1], std::ios::binary);
    uint32_t n = 0, m = 0, sddm = 0, n_rounds = 0;
    uint64_t nnz_f = 0, nnz_a = 0;
    csc L;
    spmat A;
    std::vector<uint32_t> perm;
    std::vector<uint64_t> rounds;
    vec b, x;
    std::vector<double> y;
    bool ok = rd(f, &n, 1) && rd(f, &m, 1) && rd(f, &sddm, 1) && rd(f, &nnz_f, 1);
    if (ok) {
        L.n = n; L.outer.resize(n + 1); L.inner.resize(nnz_f); L.vals.resize(nnz_f); perm.resize(n);
        ok = rd(f, L.outer.data(), n + 1) && rd(f, L.inner.data(), nnz_f) && rd(f, L.vals.data(), nnz_f) &&
             rd(f, perm.data(), n) && rd(f, &n_rounds, 1);
    }
    if (ok) { rounds.resize(n_rounds); ok = rd(f, rounds.data(), n_rounds) && rd(f, &nnz_a, 1); }
    if (ok) {
        A.n = static_cast<int>(n); A.outer.resize(n + 1); A.inner.resize(nnz_a); A.vals.resize(nnz_a);
        b.resize(n); y.resize(m);
        ok = rd(f, A.outer.data(), n + 1) && rd(f, A.inner.data(), nnz_a) && rd(f, A.vals.data(), nnz_a) &&
             rd(f, b.data(), n) && rd(f, y.data(), m);
    }
    if (!ok) { std::fprintf(stderr, "dropin: short input\n"); return 1; }
    try {
        precond P;
        std::vector<uint32_t> bounds{0};
        for (uint64_t r : rounds) bounds.push_back(bounds.back() + static_cast<uint32_t>(r));
        P.trsv.set_round_bounds(bounds);
        P.trsv.setup(L, m);
        std::vector<double> sweep(m);
        P.trsv.solve_LLt(y.data(), sweep.data());
        apxb::cuda_pcg pcg;
        pcg.setup(A, perm);
        int iters = 0;
        double res = 0.0;
        pcg.solve(P, b, x, 1e-8, 500, iters, res, sddm == 0);
        std::ofstream o(argv[2], std::ios::binary);
        o.write(reinterpret_cast<const char*>(sweep.data()), static_cast<std::streamsize>(8 * m));
        o.write(reinterpret_cast<const char*>(x.data()), static_cast<std::streamsize>(8 * n));
        const int32_t it32 = iters;
        o.write(reinterpret_cast<const char*>(&it32), 4);
        o.write(reinterpret_cast<const char*>(&res), 8);
    } catch (const std::exception& ex) {
        std::fprintf(stderr, "%s\n", ex.what());
        return 2;
    }
    return 0;
}
