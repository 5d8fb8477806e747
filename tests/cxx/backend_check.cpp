// Drives include/qa_cuda_backend.hpp -- the CUDABackend a maintainer adds to
// qanneal -- from C++ against qanneal's own classes (DenseIsing, SparseIsing,
// AnnealSchedule, SQASchedule and the result structs, compiled from the
// reference sources), so the C ABI's C++ usability is exercised: struct
// layouts, extern "C", ownership and error mapping.  Test infrastructure.
//
// usage: backend_check <case.bin> <result.bin>
// case.bin (little-endian): int32 mode (0 SA, 1 SQA, 2 SQA-PT), kind (0 dense,
// 1 sparse), n, P, K, steps, spb, wls, reads, m, rungs; uint64 seed; h[n];
// dense: J[n*n], sparse: m x (int64 i, int64 j, double w); SA/SQA: betas[steps]
// (and gammas[steps]); SQA-PT: betas[rungs], gammas[rungs].
// result.bin: per read the best energy, the best spins (int8[n]) and the
// trace (SA/SQA: energy_trace[steps]; SQA-PT: final_energies[rungs] then
// average_energy_trace[steps]); then the host energy of read 0's best state
// computed through the backend's per-flip interface.
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "qa_cuda_backend.hpp"

namespace {
template <class T>
void rd(FILE *f, T *p, size_t n) {
    if (n && std::fread(p, sizeof(T), n, f) != n) throw std::runtime_error("short case file");
}
template <class T>
void wr(FILE *f, const T *p, size_t n) {
    if (n) std::fwrite(p, sizeof(T), n, f);
}
}  // namespace

int main(int argc, char **argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s case.bin result.bin\n", argv[0]);
        return 2;
    }
    try {
        FILE *f = std::fopen(argv[1], "rb");
        if (!f) throw std::runtime_error("cannot open the case file");
        int32_t hd[11];
        rd(f, hd, 11);
        const int mode = hd[0], kind = hd[1], n = hd[2], P = hd[3], K = hd[4], steps = hd[5], spb = hd[6],
                  wls = hd[7], reads = hd[8], m = hd[9], rungs = hd[10];
        uint64_t seed;
        rd(f, &seed, 1);
        std::vector<double> h(n);
        rd(f, h.data(), n);
        std::shared_ptr<const qanneal::Hamiltonian> ham;
        if (kind == 0) {
            std::vector<double> J((size_t)n * n);
            rd(f, J.data(), J.size());
            ham = std::make_shared<qanneal::DenseIsing>(h, J, (size_t)n);
        } else {
            std::vector<qanneal::SparseEdge> e(m);
            for (int k = 0; k < m; ++k) {
                int64_t ij[2];
                double w;
                rd(f, ij, 2);
                rd(f, &w, 1);
                e[k] = qanneal::SparseEdge{(size_t)ij[0], (size_t)ij[1], w};
            }
            ham = std::make_shared<qanneal::SparseIsing>(h, e, (size_t)n);
        }
        const int nb = mode == 2 ? rungs : steps;
        std::vector<double> betas(nb), gammas(nb);
        rd(f, betas.data(), nb);
        if (mode != 0) rd(f, gammas.data(), nb);
        std::fclose(f);

        qa_cuda::CUDABackend backend(ham);
        if (backend.kind() != qanneal::BackendKind::CUDA || backend.size() != (size_t)n)
            throw std::runtime_error("backend identity");
        FILE *o = std::fopen(argv[2], "wb");
        if (!o) throw std::runtime_error("cannot open the result file");
        std::vector<int8_t> first;
        if (mode == 0) {
            qanneal::AnnealSchedule sched;
            sched.betas = betas;
            auto res = qa_cuda::sa_run(backend, sched, spb, reads, seed);
            for (auto &r : res) {
                wr(o, &r.best_energy, 1);
                wr(o, r.best_state.spins.data(), n);
                wr(o, r.energy_trace.data(), r.energy_trace.size());
            }
            first = res[0].best_state.spins;
        } else if (mode == 1) {
            auto sched = qanneal::SQASchedule::from_vectors(betas, gammas);
            auto res = qa_cuda::sqa_run(backend, sched, P, K, spb, wls, 0, 0, reads, seed);
            for (auto &r : res) {
                wr(o, &r.best_energy, 1);
                wr(o, r.best_state.spins.data(), n);
                wr(o, r.energy_trace.data(), r.energy_trace.size());
            }
            first = res[0].best_state.spins;
        } else {
            auto res = qa_cuda::sqapt_run(backend, betas, gammas, P, spb, wls, steps, 2, 0, reads, seed);
            for (auto &r : res) {
                wr(o, &r.best_energy, 1);
                wr(o, r.best_state.spins.data(), n);
                wr(o, r.final_energies.data(), r.final_energies.size());
                wr(o, r.average_energy_trace.data(), r.average_energy_trace.size());
            }
            first = res[0].best_state.spins;
        }
        const double e0 = backend.energy(first.data(), first.size());
        wr(o, &e0, 1);
        std::fclose(o);
        // an argument error crosses as std::invalid_argument
        try {
            qanneal::AnnealSchedule bad;
            bad.betas = {1.0};
            qa_cuda::sa_run(backend, bad, 0, 1, 1);
            std::fprintf(stderr, "sweeps_per_beta = 0 was accepted\n");
            return 1;
        } catch (const std::invalid_argument &) {
        }
    } catch (const std::exception &ex) {
        std::fprintf(stderr, "backend_check: %s\n", ex.what());
        return 1;
    }
    return 0;
}
