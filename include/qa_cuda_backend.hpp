/*
 * qa_cuda_backend.hpp -- the reference-side C++ binding of libqa_gpu.so.
 *
 * What a maintainer adds to qanneal to make backend "cuda" real: a Backend
 * (include/qanneal/backend.hpp:39-53, whose make_backend throws "CUDA backend
 * stub" today, backend.hpp:97-102) that owns a device copy of the model, and
 * whole-run dispatch functions that the annealers' run() would call when
 * backend_->kind() == BackendKind::CUDA, returning qanneal's own result
 * structs (AnnealResult, SQAResult, SQAParallelTemperingResult).  Per-flip
 * Backend calls stay on the host model: a per-flip call cannot cross to a
 * device, so whole runs do.
 *
 * Header-only C++17.  Compile with qanneal's include directory and this
 * repository's include/ on the include path; link libqa_gpu.so and qanneal's
 * core library.  Read r of a batched call equals set_seed(seed + r); run(...).
 */
#ifndef QA_CUDA_BACKEND_HPP
#define QA_CUDA_BACKEND_HPP

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "qa_gpu.h"
#include "qanneal/annealer.hpp"
#include "qanneal/backend.hpp"
#include "qanneal/dense_ising.hpp"
#include "qanneal/schedule.hpp"
#include "qanneal/sparse_ising.hpp"
#include "qanneal/sqa_annealer.hpp"
#include "qanneal/sqa_parallel_tempering.hpp"
#include "qanneal/sqa_schedule.hpp"

namespace qa_cuda {

// Status codes to qanneal's exceptions: argument errors are
// std::invalid_argument (ValueError in Python), the rest std::runtime_error.
inline void check(int rc) {
    if (rc == QA_OK) return;
    char msg[1024];
    qa_last_error(msg, sizeof msg);
    if (rc == QA_ERR_ARG) throw std::invalid_argument(msg);
    throw std::runtime_error(std::string("qa_gpu: ") + msg);
}

class CUDABackend final : public qanneal::Backend {
public:
    // Dense and sparse models through their public accessors.
    explicit CUDABackend(std::shared_ptr<const qanneal::Hamiltonian> ham, int device = 0) : ham_(std::move(ham)) {
        if (!ham_) throw std::invalid_argument("CUDABackend requires a Hamiltonian.");
        check(qa_create(&ctx_, device));
        try {
            if (auto *d = dynamic_cast<const qanneal::DenseIsing *>(ham_.get())) {
                check(qa_problem_dense(ctx_, (int)d->size(), d->h().data(), d->J().data(), d->constant(), &prob_));
            } else if (auto *s = dynamic_cast<const qanneal::SparseIsing *>(ham_.get())) {
                const auto &e = s->edges();
                std::vector<int64_t> ei(e.size()), ej(e.size());
                std::vector<double> w(e.size());
                for (size_t k = 0; k < e.size(); ++k) {
                    ei[k] = (int64_t)e[k].i;
                    ej[k] = (int64_t)e[k].j;
                    w[k] = e[k].value;
                }
                check(qa_problem_sparse(ctx_, (int)s->size(), s->h().data(), (int)e.size(), ei.data(), ej.data(),
                                        w.data(), s->constant(), &prob_));
            } else {
                throw std::invalid_argument(
                    "CUDABackend: a HigherOrderIsing keeps its consolidated terms private; use the constructor "
                    "that takes them");
            }
        } catch (...) {
            release();
            throw;
        }
    }

    // A higher-order model from its consolidated terms (degree >= 2, strictly
    // increasing variables per term, the degree-1 part folded into h and the
    // constant into c, as HigherOrderIsing's constructor leaves them,
    // higher_order_ising.cpp:10-90); ham serves the per-flip host calls.
    CUDABackend(std::shared_ptr<const qanneal::Hamiltonian> ham, const std::vector<double> &h,
                const std::vector<int64_t> &term_ptr, const std::vector<int32_t> &term_vars,
                const std::vector<double> &coeff, double c, int device = 0)
        : ham_(std::move(ham)) {
        if (!ham_) throw std::invalid_argument("CUDABackend requires a Hamiltonian.");
        check(qa_create(&ctx_, device));
        try {
            check(qa_problem_hubo(ctx_, (int)ham_->size(), h.data(), (int)coeff.size(), term_ptr.data(),
                                  term_vars.data(), coeff.data(), c, &prob_));
        } catch (...) {
            release();
            throw;
        }
    }

    CUDABackend(const CUDABackend &) = delete;
    CUDABackend &operator=(const CUDABackend &) = delete;
    ~CUDABackend() override { release(); }

    qanneal::BackendKind kind() const override { return qanneal::BackendKind::CUDA; }
    std::size_t size() const override { return ham_->size(); }
    double energy(const int8_t *spins, std::size_t n) const override { return ham_->energy(spins, n); }
    double delta_energy(const int8_t *spins, std::size_t n, std::size_t flip) const override {
        return ham_->delta_energy(spins, n, flip);
    }
    void compute_local_fields(const int8_t *spins, std::size_t n, double *fields) const override {
        ham_->compute_local_fields(spins, n, fields);
    }
    void update_local_fields_after_flip(double *fields, const int8_t *new_spins, std::size_t n, std::size_t flip,
                                        int8_t old_spin) const override {
        ham_->update_local_fields_after_flip(fields, new_spins, n, flip, old_spin);
    }

    qa_ctx *context() const { return ctx_; }
    const qa_problem *problem() const { return prob_; }

private:
    void release() {
        if (prob_) qa_problem_free(prob_);
        if (ctx_) qa_destroy(ctx_);
        prob_ = nullptr;
        ctx_ = nullptr;
    }
    std::shared_ptr<const qanneal::Hamiltonian> ham_;
    qa_ctx *ctx_ = nullptr;
    qa_problem *prob_ = nullptr;
};

// Annealer::run (annealer.cpp:33-75) for `reads` reads in one launch.
inline std::vector<qanneal::AnnealResult> sa_run(const CUDABackend &b, const qanneal::AnnealSchedule &schedule,
                                                 std::size_t sweeps_per_beta, int reads, uint64_t seed) {
    const int n = (int)b.size(), steps = (int)schedule.size();
    std::vector<int8_t> spins((size_t)reads * n);
    std::vector<double> best(reads), trace((size_t)reads * steps);
    qa_sa_params p{schedule.betas.data(), steps, (int)sweeps_per_beta, reads, seed};
    qa_run_out o{spins.data(), best.data(), trace.data()};
    const qa_problem *pp = b.problem();
    check(qa_sa_run(b.context(), &pp, 1, &p, &o, nullptr));
    std::vector<qanneal::AnnealResult> out(reads);
    for (int r = 0; r < reads; ++r) {
        out[r].best_state.spins.assign(spins.begin() + (size_t)r * n, spins.begin() + (size_t)(r + 1) * n);
        out[r].best_energy = best[r];
        out[r].energy_trace.assign(trace.begin() + (size_t)r * steps, trace.begin() + (size_t)(r + 1) * steps);
    }
    return out;
}

// SQAAnnealer::run (sqa_annealer.cpp:87-477) for `reads` reads in one launch.
inline std::vector<qanneal::SQAResult> sqa_run(const CUDABackend &b, const qanneal::SQASchedule &schedule,
                                               std::size_t trotter_slices, std::size_t replicas,
                                               std::size_t sweeps_per_beta, std::size_t worldline_sweeps,
                                               std::size_t cluster_sweeps, std::size_t continuous_time_slices,
                                               int reads, uint64_t seed) {
    const int n = (int)b.size(), steps = (int)schedule.size();
    std::vector<int8_t> spins((size_t)reads * n);
    std::vector<double> best(reads), trace((size_t)reads * steps);
    qa_sqa_params p{schedule.betas.data(), schedule.gammas.data(), steps, (int)trotter_slices, (int)replicas,
                    (int)sweeps_per_beta, (int)worldline_sweeps, (int)cluster_sweeps,
                    (int)continuous_time_slices, reads, seed};
    qa_run_out o{spins.data(), best.data(), trace.data()};
    const qa_problem *pp = b.problem();
    check(qa_sqa_run(b.context(), &pp, 1, &p, &o, nullptr));
    std::vector<qanneal::SQAResult> out(reads);
    for (int r = 0; r < reads; ++r) {
        out[r].best_state.spins.assign(spins.begin() + (size_t)r * n, spins.begin() + (size_t)(r + 1) * n);
        out[r].best_energy = best[r];
        out[r].energy_trace.assign(trace.begin() + (size_t)r * steps, trace.begin() + (size_t)(r + 1) * steps);
    }
    return out;
}

// SQAParallelTemperingAnnealer::run (sqa_parallel_tempering.cpp:81-346).
inline std::vector<qanneal::SQAParallelTemperingResult> sqapt_run(
    const CUDABackend &b, const std::vector<double> &betas, const std::vector<double> &gammas,
    std::size_t trotter_slices, std::size_t sweeps_per_step, std::size_t worldline_sweeps, std::size_t steps,
    std::size_t swap_interval, std::size_t cluster_sweeps, int reads, uint64_t seed) {
    const int n = (int)b.size(), R = (int)betas.size(), S = (int)steps;
    if (gammas.size() != betas.size()) throw std::invalid_argument("betas/gammas length mismatch.");
    std::vector<int8_t> spins((size_t)reads * n), fspins((size_t)reads * R * n);
    std::vector<double> best(reads), fE((size_t)reads * R), avg((size_t)reads * S), swp((size_t)reads * S);
    qa_sqapt_params p{betas.data(), gammas.data(), R, (int)trotter_slices, (int)sweeps_per_step,
                      (int)worldline_sweeps, S, (int)swap_interval, (int)cluster_sweeps, 0, reads, seed};
    qa_sqapt_out o{spins.data(), best.data(), fspins.data(), fE.data(), avg.data(), swp.data()};
    const qa_problem *pp = b.problem();
    check(qa_sqapt_run(b.context(), &pp, 1, &p, &o, nullptr));
    std::vector<qanneal::SQAParallelTemperingResult> out(reads);
    for (int r = 0; r < reads; ++r) {
        auto &x = out[r];
        x.best_state.spins.assign(spins.begin() + (size_t)r * n, spins.begin() + (size_t)(r + 1) * n);
        x.best_energy = best[r];
        for (int k = 0; k < R; ++k) {
            qanneal::State st;
            const size_t o0 = ((size_t)r * R + k) * n;
            st.spins.assign(fspins.begin() + o0, fspins.begin() + o0 + n);
            x.final_states.push_back(std::move(st));
            x.final_energies.push_back(fE[(size_t)r * R + k]);
        }
        x.average_energy_trace.assign(avg.begin() + (size_t)r * S, avg.begin() + (size_t)(r + 1) * S);
        x.swap_acceptance_trace.assign(swp.begin() + (size_t)r * S, swp.begin() + (size_t)(r + 1) * S);
    }
    return out;
}

}  // namespace qa_cuda

#endif  // QA_CUDA_BACKEND_HPP
