// ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A C-ABI driver over the UNMODIFIED qanneal classes, compiled together with
// qanneal's own sources by oracle/Makefile into oracle/_ref/libqanneal_ref.so.
// It is used for two things only: (1) golden vectors and statistical parity
// checks in tests/, (2) the timed CPU baseline ("kind": "reference") in
// bench.py.  Nothing in the product links it.
//
// Every entry point calls the public qanneal API exactly as python/bindings.cpp
// does (make_backend(CPU, ham) + the annealer class + set_seed + run*).
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

#include "qanneal/annealer.hpp"
#include "qanneal/parallel_tempering.hpp"
#include "qanneal/replica_annealer.hpp"
#include "qanneal/backend.hpp"
#include "qanneal/dense_ising.hpp"
#include "qanneal/higher_order_ising.hpp"
#include "qanneal/qubo.hpp"
#include "qanneal/sparse_ising.hpp"
#include "qanneal/sqa_annealer.hpp"
#include "qanneal/sqa_chi_annealer.hpp"
#include "qanneal/sqa_parallel_tempering.hpp"

using namespace qanneal;

namespace {
struct RefModel {
    std::shared_ptr<Hamiltonian> ham;
    HigherOrderIsing *hubo = nullptr;
};
thread_local char g_err[512];
template <class F> int guarded(F &&f) {
    try {
        f();
        return 0;
    } catch (const std::exception &e) {
        std::snprintf(g_err, sizeof(g_err), "%s", e.what());
        return -1;
    }
}
}  // namespace

extern "C" {

const char *ref_last_error() { return g_err; }

void *ref_dense_new(int n, const double *h, const double *J, double c) {
    RefModel *m = nullptr;
    guarded([&] {
        auto ham = std::make_shared<DenseIsing>(std::vector<double>(h, h + n),
                                                std::vector<double>(J, J + (size_t)n * n), (size_t)n, c);
        m = new RefModel{ham, nullptr};
    });
    return m;
}

void *ref_sparse_new(int n, const double *h, int m_edges, const int64_t *ei, const int64_t *ej,
                     const double *w, double c) {
    RefModel *m = nullptr;
    guarded([&] {
        std::vector<SparseEdge> edges;
        for (int e = 0; e < m_edges; ++e) edges.push_back({(size_t)ei[e], (size_t)ej[e], w[e]});
        auto ham = std::make_shared<SparseIsing>(std::vector<double>(h, h + n), edges, (size_t)n, c);
        m = new RefModel{ham, nullptr};
    });
    return m;
}

void *ref_hubo_new(int n, int nraw, const int64_t *rptr, const int64_t *rvars, const double *rcoef, double c) {
    RefModel *m = nullptr;
    guarded([&] {
        std::vector<HigherOrderIsing::RawTerm> raw;
        for (int t = 0; t < nraw; ++t) {
            std::vector<size_t> v;
            for (int64_t k = rptr[t]; k < rptr[t + 1]; ++k) v.push_back((size_t)rvars[k]);
            raw.push_back({v, rcoef[t]});
        }
        auto ham = std::make_shared<HigherOrderIsing>((size_t)n, raw, c);
        m = new RefModel{ham, ham.get()};
    });
    return m;
}

// QUBO(Q).to_ising() (qubo.cpp:33-69): writes h[n], J[n*n], c.
int ref_qubo_to_ising(int n, const double *Q, double *h, double *J, double *c) {
    return guarded([&] {
        QUBO q(std::vector<double>(Q, Q + (size_t)n * n), (size_t)n);
        DenseIsing d = q.to_ising();
        std::memcpy(h, d.h().data(), sizeof(double) * n);
        std::memcpy(J, d.J().data(), sizeof(double) * (size_t)n * n);
        *c = d.constant();
    });
}

void ref_model_free(void *p) { delete static_cast<RefModel *>(p); }

int ref_hubo_info(void *p, int *num_terms, int *max_degree, double *constant, double *h) {
    auto *m = static_cast<RefModel *>(p);
    if (!m->hubo) return -1;
    *num_terms = (int)m->hubo->num_terms();
    *max_degree = (int)m->hubo->max_degree();
    *constant = m->hubo->constant();
    const auto &hv = m->hubo->h();
    std::memcpy(h, hv.data(), sizeof(double) * hv.size());
    return 0;
}

double ref_energy(void *p, const int8_t *s, int n) {
    double e = 0.0;
    guarded([&] { e = static_cast<RefModel *>(p)->ham->energy(s, (size_t)n); });
    return e;
}

double ref_delta_energy(void *p, const int8_t *s, int n, int flip) {
    double e = 0.0;
    guarded([&] { e = static_cast<RefModel *>(p)->ham->delta_energy(s, (size_t)n, (size_t)flip); });
    return e;
}

int ref_fields(void *p, const int8_t *s, int n, double *f) {
    return guarded([&] { static_cast<RefModel *>(p)->ham->compute_local_fields(s, (size_t)n, f); });
}

int ref_update_fields(void *p, double *f, const int8_t *new_s, int n, int flip, int old_spin) {
    return guarded([&] {
        static_cast<RefModel *>(p)->ham->update_local_fields_after_flip(f, new_s, (size_t)n, (size_t)flip,
                                                                        (int8_t)old_spin);
    });
}

// Annealer::run, one read (annealer.cpp:33-75).
int ref_sa_run(void *p, const double *betas, int steps, int spb, uint64_t seed, int8_t *best_spins,
               double *best_E, double *trace) {
    return guarded([&] {
        auto *m = static_cast<RefModel *>(p);
        AnnealSchedule sched;
        sched.betas.assign(betas, betas + steps);
        Annealer a(make_backend(BackendKind::CPU, m->ham), sched);
        a.set_seed(seed);
        AnnealResult r = a.run((size_t)spb);
        std::memcpy(best_spins, r.best_state.spins.data(), r.best_state.size());
        *best_E = r.best_energy;
        if (trace) std::memcpy(trace, r.energy_trace.data(), sizeof(double) * r.energy_trace.size());
    });
}

// SQAAnnealer::run, one read (sqa_annealer.cpp:87-477).
int ref_sqa_run(void *p, const double *betas, const double *gammas, int steps, int P, int K, int spb, int wls,
                uint64_t seed, int8_t *best_spins, double *best_E, double *trace, int cls) {
    return guarded([&] {
        auto *m = static_cast<RefModel *>(p);
        auto sched = SQASchedule::from_vectors(std::vector<double>(betas, betas + steps),
                                               std::vector<double>(gammas, gammas + steps));
        SQAAnnealer a(make_backend(BackendKind::CPU, m->ham), sched, (size_t)P, (size_t)K);
        a.set_seed(seed);
        SQAResult r = a.run((size_t)spb, (size_t)wls, (size_t)cls);
        std::memcpy(best_spins, r.best_state.spins.data(), r.best_state.size());
        *best_E = r.best_energy;
        if (trace) std::memcpy(trace, r.energy_trace.data(), sizeof(double) * r.energy_trace.size());
    });
}

// ParallelTemperingAnnealer::run (parallel_tempering.cpp:36-122).
int ref_pt_run(void *p, const double *betas, int R, int spb, int steps, int swap_interval, uint64_t seed,
               int8_t *best_spins, double *best_E, double *final_E, double *avg_trace, double *swap_trace) {
    return guarded([&] {
        auto *m = static_cast<RefModel *>(p);
        ParallelTemperingAnnealer a(make_backend(BackendKind::CPU, m->ham), std::vector<double>(betas, betas + R));
        a.set_seed(seed);
        auto r = a.run((size_t)spb, (size_t)steps, (size_t)swap_interval);
        std::memcpy(best_spins, r.best_state.spins.data(), r.best_state.size());
        *best_E = r.best_energy;
        if (final_E) std::memcpy(final_E, r.final_energies.data(), sizeof(double) * r.final_energies.size());
        if (avg_trace) std::memcpy(avg_trace, r.average_energy_trace.data(), sizeof(double) * steps);
        if (swap_trace) std::memcpy(swap_trace, r.swap_acceptance_trace.data(), sizeof(double) * steps);
    });
}

// ReplicaAnnealer::run (replica_annealer.cpp:46-142): global best and the average traces.
int ref_replica_run(void *p, const double *betas, int steps, int spb, int R, uint64_t seed, double *best_E,
                    double *avg_energy, double *avg_mag) {
    return guarded([&] {
        auto *m = static_cast<RefModel *>(p);
        AnnealSchedule sched;
        sched.betas.assign(betas, betas + steps);
        ReplicaAnnealer a(make_backend(BackendKind::CPU, m->ham), sched, (size_t)R);
        a.set_seed(seed);
        auto r = a.run((size_t)spb);
        *best_E = r.global_best_energy;
        std::memcpy(avg_energy, r.average_energy_trace.data(), sizeof(double) * steps);
        std::memcpy(avg_mag, r.average_magnetization_trace.data(), sizeof(double) * steps);
    });
}

// SQAAnnealer::run_optimal, one read (sqa_annealer.cpp:499-952).
int ref_sqa_opt_run(void *p, int P, int K, double beta, double js, double je, double eps_tilde, double alpha,
                    int num_steps, int spb, int wls, int cls, int probes, int csweeps, double ramp_fraction,
                    double ramp_start, uint64_t seed, double *best_E, double *trace, double *jtrace, double *chitrace,
                    double *scalars) {
    return guarded([&] {
        auto *m = static_cast<RefModel *>(p);
        SQAAnnealer a(make_backend(BackendKind::CPU, m->ham), SQASchedule::from_vectors({1.0}, {1.0}), (size_t)P,
                      (size_t)K);
        a.set_seed(seed);
        SQAResult r = a.run_optimal(beta, js, je, eps_tilde, alpha, (size_t)num_steps, (size_t)spb, (size_t)wls,
                                    (size_t)cls, (size_t)probes, (size_t)csweeps, "", ramp_fraction, ramp_start);
        *best_E = r.best_energy;
        std::memcpy(trace, r.energy_trace.data(), sizeof(double) * num_steps);
        std::memcpy(jtrace, r.j_perp_trace.data(), sizeof(double) * num_steps);
        std::memcpy(chitrace, r.chi_B_trace.data(), sizeof(double) * num_steps);
        scalars[0] = r.calibrated_eps_tilde;
        scalars[1] = r.j_perp_start;
        scalars[2] = r.resolved_j_perp_end;
        scalars[3] = r.final_j_perp;
    });
}

// SQAParallelTemperingAnnealer::run, one read (sqa_parallel_tempering.cpp:81-346).
int ref_sqapt_run(void *p, const double *betas, const double *gammas, int R, int P, int spb, int wls, int steps,
                  int swap_interval, uint64_t seed, int8_t *best_spins, double *best_E, double *final_E,
                  double *avg_trace, double *swap_trace, int cls) {
    return guarded([&] {
        auto *m = static_cast<RefModel *>(p);
        SQAParallelTemperingAnnealer a(make_backend(BackendKind::CPU, m->ham), std::vector<double>(betas, betas + R),
                                       std::vector<double>(gammas, gammas + R), (size_t)P);
        a.set_seed(seed);
        auto r = a.run((size_t)spb, (size_t)wls, (size_t)steps, (size_t)swap_interval, (size_t)cls);
        std::memcpy(best_spins, r.best_state.spins.data(), r.best_state.size());
        *best_E = r.best_energy;
        if (final_E) std::memcpy(final_E, r.final_energies.data(), sizeof(double) * r.final_energies.size());
        if (avg_trace) std::memcpy(avg_trace, r.average_energy_trace.data(), sizeof(double) * steps);
        if (swap_trace) std::memcpy(swap_trace, r.swap_acceptance_trace.data(), sizeof(double) * steps);
    });
}

// SQAParallelTemperingAnnealer::run_optimal, one read (sqa_parallel_tempering.cpp:348-882).
int ref_sqapt_opt_run(void *p, const double *betas, const double *gammas, int R, int P, int spb, int wls, int cls,
                      int steps, int swap_interval, double eps_tilde, double alpha, double je, int probes,
                      int csweeps, uint64_t seed, double *best_E, double *final_E, double *avg_trace,
                      double *swap_trace, double *jtrace, double *chitrace, double *scalars) {
    return guarded([&] {
        auto *m = static_cast<RefModel *>(p);
        SQAParallelTemperingAnnealer a(make_backend(BackendKind::CPU, m->ham), std::vector<double>(betas, betas + R),
                                       std::vector<double>(gammas, gammas + R), (size_t)P);
        a.set_seed(seed);
        auto r = a.run_optimal((size_t)steps, (size_t)spb, (size_t)wls, eps_tilde, alpha, je, (size_t)cls,
                               (size_t)swap_interval, 0, (size_t)probes, (size_t)csweeps, "");
        *best_E = r.best_energy;
        std::memcpy(final_E, r.final_energies.data(), sizeof(double) * r.final_energies.size());
        std::memcpy(avg_trace, r.average_energy_trace.data(), sizeof(double) * steps);
        std::memcpy(swap_trace, r.swap_acceptance_trace.data(), sizeof(double) * steps);
        std::memcpy(jtrace, r.j_perp_trace.data(), sizeof(double) * steps);
        std::memcpy(chitrace, r.chi_B_trace.data(), sizeof(double) * steps);
        scalars[0] = r.calibrated_eps_tilde;
        scalars[1] = r.j_perp_start;
        scalars[2] = r.resolved_j_perp_end;
        scalars[3] = r.final_j_perp;
    });
}

// SQAChiAnnealer::run_chi, one read (sqa_chi_annealer.cpp:146-438).
int ref_chi_run(void *p, int P, int K, double beta, double gamma_start, double gamma_end, int num_steps, int spb,
                int scan_points, int scan_sweeps, int scan_burn, double chi_floor_fraction, double driver_A0,
                double beta_ramp_fraction, double beta_ramp_start, uint64_t seed, int8_t *best_spins,
                double *best_E, double *scan_s, double *scan_gamma, double *scan_chi, double *beta_sched,
                double *gamma_sched, double *s_sched, double *trace, double *scalars /* s*,g*,jp*,floor,A0 */) {
    return guarded([&] {
        auto *m = static_cast<RefModel *>(p);
        SQAChiAnnealer a(make_backend(BackendKind::CPU, m->ham), (size_t)P, (size_t)K);
        a.set_seed(seed);
        SQAChiResult r = a.run_chi(beta, gamma_start, gamma_end, (size_t)num_steps, (size_t)spb, (size_t)scan_points,
                                   (size_t)scan_sweeps, (size_t)scan_burn, chi_floor_fraction, driver_A0,
                                   beta_ramp_fraction, beta_ramp_start);
        std::memcpy(best_spins, r.best_state.spins.data(), r.best_state.size());
        *best_E = r.best_energy;
        auto cp = [](double *dst, const std::vector<double> &v) {
            if (dst) std::memcpy(dst, v.data(), sizeof(double) * v.size());
        };
        cp(scan_s, r.scan_s); cp(scan_gamma, r.scan_gamma); cp(scan_chi, r.scan_chi_B);
        cp(beta_sched, r.beta_schedule); cp(gamma_sched, r.gamma_schedule); cp(s_sched, r.s_schedule);
        cp(trace, r.energy_trace);
        if (scalars) {
            scalars[0] = r.s_star; scalars[1] = r.gamma_star; scalars[2] = r.j_perp_star;
            scalars[3] = r.chi_floor; scalars[4] = r.driver_A0;
        }
    });
}

// Many independent reads spread over host threads, one annealer per thread
// (the reference's own process-per-read practice).  method: 0 = SA, 1 = SQA.
// Read r uses set_seed(seed + r), as solve() does (solver.py:679-681).
int ref_batch_run(void *p, int method, const double *betas, const double *gammas, int steps, int P, int K, int spb,
                  int wls, int reads, uint64_t seed, int threads, double *best_E) {
    auto *m = static_cast<RefModel *>(p);
    std::atomic<int> next{0};
    std::atomic<int> fail{0};
    auto worker = [&] {
        for (;;) {
            int r = next.fetch_add(1);
            if (r >= reads) break;
            try {
                if (method == 0) {
                    AnnealSchedule sched;
                    sched.betas.assign(betas, betas + steps);
                    Annealer a(make_backend(BackendKind::CPU, m->ham), sched);
                    a.set_seed(seed + (uint64_t)r);
                    best_E[r] = a.run((size_t)spb).best_energy;
                } else {
                    auto sched = SQASchedule::from_vectors(std::vector<double>(betas, betas + steps),
                                                           std::vector<double>(gammas, gammas + steps));
                    SQAAnnealer a(make_backend(BackendKind::CPU, m->ham), sched, (size_t)P, (size_t)K);
                    a.set_seed(seed + (uint64_t)r);
                    best_E[r] = a.run((size_t)spb, (size_t)wls).best_energy;
                }
            } catch (const std::exception &e) {
                std::snprintf(g_err, sizeof(g_err), "%s", e.what());
                fail = 1;
            }
        }
    };
    threads = std::max(1, std::min(threads, reads));
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
    for (auto &t : pool) t.join();
    return fail ? -1 : 0;
}

}  // extern "C"
