// qa_capi.cu -- host side of libqa_gpu.so: contexts, problem upload, and the
// run entry points declared in include/qa_gpu.h.  Each entry point batches all
// reads (and all problems of the call) into single kernel launches.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <new>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "qa_gpu.h"
#include "qa_kernels.cuh"
#include "qa_chi.cuh"
#include "qa_mlp.cuh"
#include "qa_sparse.cuh"
#include "qa_tc.cuh"
#include "qa_pm1.cuh"
#include "qa_pt.cuh"
#include "qa_ingest.cuh"

using namespace qa;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

// The error word the sweep kernels leave in counters[4]: a bounded wait of
// the slice pipeline that ran out (the outputs of that call are void).
int check_device_error(const unsigned long long *cnt) {
    if (cnt[4] & QA_DEV_ERR_TIMEOUT)
        return fail(QA_ERR_TIMEOUT, "a sweep kernel's bounded wait for its slice pipeline ran out; the run's "
                                    "outputs are void");
    return QA_OK;
}

#define QA_CK(call)                                                                                   \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) {                                                                      \
            return fail(e_ == cudaErrorMemoryAllocation ? QA_ERR_OOM : QA_ERR_CUDA,                   \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                          \
        }                                                                                             \
    } while (0)

#define QA_TRY(expr)                  \
    do {                              \
        int rc_ = (expr);             \
        if (rc_ != QA_OK) return rc_; \
    } while (0)

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
};

// Device blocks of freed problems, kept for the next problem of about the
// same size (a model rebuilt per call then costs no cudaMalloc / cudaFree).
// Shared by a context and its problems, so it outlives whichever goes last.
struct BlockPool {
    int device = 0;
    std::mutex mu;
    std::vector<std::pair<size_t, void *>> free_blocks;
    size_t pooled = 0;
    static constexpr size_t kCap = (size_t)1 << 30;
    ~BlockPool() {
        cudaSetDevice(device);
        for (auto &b : free_blocks) cudaFree(b.second);
    }
    void *take(size_t bytes, size_t *got) {
        std::lock_guard<std::mutex> lk(mu);
        int best = -1;
        for (int k = 0; k < (int)free_blocks.size(); ++k) {
            const size_t c = free_blocks[k].first;
            if (c >= bytes && c <= 2 * bytes + ((size_t)1 << 20) && (best < 0 || c < free_blocks[best].first)) best = k;
        }
        if (best < 0) return nullptr;
        void *p = free_blocks[best].second;
        *got = free_blocks[best].first;
        pooled -= *got;
        free_blocks.erase(free_blocks.begin() + best);
        return p;
    }
    void give(void *p, size_t bytes) {
        std::lock_guard<std::mutex> lk(mu);
        if (pooled + bytes > kCap) {
            cudaFree(p);
            return;
        }
        free_blocks.push_back({bytes, p});
        pooled += bytes;
    }
};

}  // namespace

namespace qa {
// Lets the other translation units of the library report through qa_last_error().
int set_last_error(int code, const char *msg) {
    g_err = msg;
    return code;
}
}  // namespace qa

// Host staging of problem arrays, reused across problems (grown, never
// shrunk): pinned, so the one copy of a problem block is a direct DMA that
// overlaps the host.  `sent` marks the end of the last copy out of it; the
// buffer is rewritten only after that copy has completed.  If pinned memory
// cannot be had it falls back to pageable memory (copies then stage
// synchronously).
struct HostStage {
    unsigned char *p = nullptr;
    size_t n = 0, cap = 0;
    bool pinned = false, pending = false;
    cudaEvent_t sent = nullptr;
    size_t size() const { return n; }
    bool empty() const { return n == 0; }
    unsigned char *data() { return p; }
    void clear() { n = 0; }
    void wait() {
        if (pending) cudaEventSynchronize(sent);
        pending = false;
    }
    void resize(size_t m) {
        if (m > cap) {
            wait();
            const size_t want = std::max(m, cap * 3 / 2);
            unsigned char *q = nullptr;
            const bool pin = cudaHostAlloc(reinterpret_cast<void **>(&q), want, cudaHostAllocDefault) == cudaSuccess;
            if (!pin) {
                cudaGetLastError();  // clear the allocation error; pageable memory still works
                q = static_cast<unsigned char *>(std::malloc(want));
                if (!q) throw std::bad_alloc();
            }
            if (n) std::memcpy(q, p, n);
            release();
            p = q;
            cap = want;
            pinned = pin;
        }
        n = m;
    }
    void release() {
        wait();
        if (p) {
            if (pinned) cudaFreeHost(p);
            else std::free(p);
        }
        p = nullptr;
        cap = 0;
    }
};

struct qa_ctx {
    int device = 0;
    std::shared_ptr<BlockPool> pool;
    HostStage stage;  // host staging of problem arrays, reused across problems
    HostStage down;   // pinned landing buffer for a run's large results (used within one call)
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    int smem_optin = 0;
    int sms = 0;             // streaming multiprocessors of the device
    double drift_tol = 0.0;  // > 0: field-drift check after SA / SQA / SQA-PT runs
    int update_order = QA_ORDER_REFERENCE;  // SQA / SQA-PT sweep order (qa_set_update_order)
    qa_tuning tune{0, -1, -1, 0, 0};        // launch-shape overrides (qa_set_tuning); all automatic
    // side streams for the rotated ring launches (run_rings_rotated) and their events
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> side_ev;
    // the dynamic shared memory each ring kernel is opted in to (a function attribute)
    std::vector<std::pair<const void *, size_t>> smem_attr;
    static constexpr int kWsSlots = 48;
    DevBuf ws[kWsSlots];
};

struct qa_mlp {
    qa_ctx *ctx = nullptr;
    std::vector<int> dims;
    long long nparams = 0, nw16 = 0;
    std::vector<long long> woff, boff, w16off;
    float *W = nullptr, *g = nullptr, *mo = nullptr, *vo = nullptr;  // masters, grads, Adam moments
    __nv_bfloat16 *W16 = nullptr;
    long long *wmap = nullptr;
    int cap_B = 0;
    std::vector<long long> aoff;  // per-layer activation offsets for the current batch
    float *acts = nullptr, *dacts = nullptr, *T = nullptr, *rowloss = nullptr;
    int step = 0;
};

struct qa_problem {
    qa_ctx *ctx = nullptr;
    int kind = 0, n = 0, nw = 0, T = 0, m = 0;
    // dense couplings as int8 rows for the tensor-core field init (built on
    // first use when every coupling is an integer in [-127, 127])
    int tc_int8 = -1;  // -1 unknown, 0 no, 1 yes
    int8_t *J8 = nullptr;
    int tc_ldj = 0;
    double c = 0.0;
    std::vector<void *> allocs;
    ProbDev dev{};
    // arrays staged on the host (the context's buffer) while the problem is
    // built, then sent with one copy into one device block; fix = (offset,
    // device pointer to patch)
    std::vector<std::pair<size_t, const void **>> fix;
    // arrays the device fills after the block exists: (bytes, pointer to patch)
    std::vector<std::pair<size_t, const void **>> resv;
    std::shared_ptr<BlockPool> pool;  // where the block goes back
    void *block = nullptr;
    size_t block_bytes = 0;
};

namespace {

enum WsSlot { W_PROBS, W_RINGS, W_SPINS, W_FIELDS, W_A, W_T4, W_SUM, W_BESTE, W_BESTSTEP, W_BITS, W_CNT, W_EXACT,
              W_PROBOF, W_MIN, W_BOND, W_MAG, W_SLOT, W_RIN, W_BSLOT, W_FBITS, W_AVG, W_SWP, W_BPJP, W_JP,
              W_BSAMP, W_SSAVE, W_FSAVE, W_CBESTE, W_CBSTEP, W_CBITS, W_CBOND, W_FLAG, W_QSTAGE,
              W_TRB, W_TRE, W_TREB, W_TREE, W_RSPIN, W_DRIFT, W_ORDER, W_OSCR, W_COUNT };
static_assert(W_COUNT <= qa_ctx::kWsSlots, "qa_ctx::ws has a slot per WsSlot");

int ws_get(qa_ctx *ctx, int slot, size_t bytes, void **out) {
    DevBuf &b = ctx->ws[slot];
    if (bytes == 0) bytes = 16;
    if (b.cap < bytes) {
        if (b.p) cudaFree(b.p);
        b.p = nullptr;
        b.cap = 0;
        size_t want = std::max(bytes, b.cap * 3 / 2);
        QA_CK(cudaMalloc(&b.p, want));
        b.cap = want;
    }
    *out = b.p;
    return QA_OK;
}

// Space for `count` T in the staging buffer, to be filled before the next
// staging call (which may move the buffer); *dev is set by finish_problem.
template <class T>
T *stage_array(qa_problem *P, size_t count, const T **dev) {
    HostStage &st = P->ctx->stage;
    if (P->fix.empty()) {  // first array of this problem: the previous block's copy must be done
        st.wait();
        st.clear();
    }
    const size_t off = (st.size() + 255) & ~(size_t)255;
    st.resize(off + std::max<size_t>(count * sizeof(T), 16));
    P->fix.push_back({off, reinterpret_cast<const void **>(dev)});
    return reinterpret_cast<T *>(st.data() + off);
}

// Space in the problem's device block for an array the device writes itself.
template <class T>
void reserve_array(qa_problem *P, size_t count, const T **dev) {
    P->resv.push_back({std::max<size_t>(count * sizeof(T), 16), reinterpret_cast<const void **>(dev)});
}

template <class T>
int upload(qa_problem *P, const T *host, size_t count, const T **dev) {
    T *dst = stage_array(P, count, dev);
    if (count) std::memcpy(dst, host, count * sizeof(T));
    return QA_OK;
}

int begin(qa_ctx *ctx) {
    if (!ctx) return fail(QA_ERR_ARG, "null context");
    QA_CK(cudaSetDevice(ctx->device));
    return QA_OK;
}

// Sends the staged arrays (one allocation, one copy; the reserved arrays follow
// them in the block, uncopied) and sets the scalars.
int finish_problem(qa_problem *P) {
    P->dev.kind = P->kind;
    P->dev.n = P->n;
    P->dev.nw = P->nw;
    P->dev.T = P->T;
    P->dev.m = P->m;
    P->dev.c = P->c;
    HostStage &st = P->ctx->stage;
    if (P->fix.empty()) st.clear();  // nothing staged for this problem
    std::vector<size_t> roff;
    size_t end = st.size();
    for (auto &r : P->resv) {
        end = (end + 255) & ~(size_t)255;
        roff.push_back(end);
        end += r.first;
    }
    const size_t bytes = std::max<size_t>(end, 16);
    P->pool = P->ctx->pool;
    size_t got = 0;
    void *d = P->pool->take(bytes, &got);
    if (!d) {
        const cudaError_t e = cudaMalloc(&d, bytes);
        if (e != cudaSuccess) {
            st.clear();
            P->fix.clear();
            return fail(e == cudaErrorMemoryAllocation ? QA_ERR_OOM : QA_ERR_CUDA, cudaGetErrorString(e));
        }
        got = bytes;
    }
    P->block = d;
    P->block_bytes = got;
    // on the context's stream (non-blocking): every later use of the block,
    // the device-side derivations first, is ordered after the copy; a
    // pageable source is staged before the call returns, so the buffer is free
    cudaError_t e =
        st.empty() ? cudaSuccess : cudaMemcpyAsync(d, st.data(), st.size(), cudaMemcpyHostToDevice, P->ctx->stream);
    if (e == cudaSuccess && !st.empty()) {
        e = cudaEventRecord(st.sent, P->ctx->stream);
        st.pending = e == cudaSuccess;
    }
    st.clear();
    if (e != cudaSuccess) {
        P->fix.clear();
        P->resv.clear();
        return fail(QA_ERR_CUDA, cudaGetErrorString(e));
    }
    for (auto &f : P->fix) *f.second = static_cast<unsigned char *>(d) + f.first;
    for (size_t k = 0; k < P->resv.size(); ++k) *P->resv[k].second = static_cast<unsigned char *>(d) + roff[k];
    P->fix.clear();
    P->resv.clear();
    return QA_OK;
}


int common_h(qa_problem *P, const double *h) {
    std::vector<float> h32(P->n);
    for (int i = 0; i < P->n; ++i) h32[i] = (float)h[i];
    QA_TRY(upload(P, h32.data(), h32.size(), &P->dev.h32));
    QA_TRY(upload(P, h, (size_t)P->n, &P->dev.h64));
    return QA_OK;
}

double trotter_coupling(double beta, double gamma, int P) {
    // sqa_annealer.cpp:66-70
    const double x = std::max(beta * gamma / (double)P, 1e-12);
    return 0.5 * std::log(1.0 / std::tanh(x));
}

std::vector<uint32_t> dummy;

void unpack_bits(const uint32_t *bits, int n, int8_t *out) {
    for (int i = 0; i < n; ++i) out[i] = ((bits[i >> 5] >> (i & 31)) & 1u) ? 1 : -1;
}

int check_batch(const qa_problem *const *probs, int np, int *kind, int *n_max) {
    if (!probs || np <= 0) return fail(QA_ERR_ARG, "at least one problem is required.");
    *kind = probs[0] ? probs[0]->kind : -1;
    *n_max = 0;
    for (int i = 0; i < np; ++i) {
        if (!probs[i]) return fail(QA_ERR_ARG, "null problem.");
        if (probs[i]->kind != *kind) return fail(QA_ERR_ARG, "all problems of one call must be of the same model kind.");
        *n_max = std::max(*n_max, probs[i]->n);
    }
    return QA_OK;
}

template <class F>
void dispatch_kind(int kind, F &&f) {
    if (kind == K_DENSE) f(std::integral_constant<int, K_DENSE>());
    else if (kind == K_SPARSE) f(std::integral_constant<int, K_SPARSE>());
    else f(std::integral_constant<int, K_HUBO>());
}

// Ring layout shared by the SA and ring launches.
struct Layout {
    std::vector<RingDev> rings;
    long long spin_words = 0, field_floats = 0;
    int nw_max = 1;
};

// Rings ordered (problem, read, [scan point,] replica).  With points > 0 every
// (read, point) probe gets its own K rings, schedule row `point` and the
// domain-tag extension point << 8 (the chi pilot).
void build_rings(Layout &L, const qa_problem *const *probs, int np, int reads, int K, int P, uint64_t seed,
                 int points = 0) {
    L.rings.clear();
    L.spin_words = L.field_floats = 0;
    L.nw_max = 1;
    for (int p = 0; p < np; ++p) L.nw_max = std::max(L.nw_max, probs[p]->nw);
    const int npt = points > 0 ? points : 1;
    for (int p = 0; p < np; ++p)
        for (int r = 0; r < reads; ++r)
            for (int m = 0; m < npt; ++m)
                for (int k = 0; k < K; ++k) {
                    RingDev R{};
                    R.prob = p;
                    R.out = p * reads + r;
                    R.k = k;
                    R.sched = points > 0 ? m : 0;
                    R.tag_extra = points > 0 ? (uint32_t)m << 8 : 0u;
                    R.key = seed + (uint64_t)r;
                    R.spin_off = L.spin_words;
                    R.field_off = L.field_floats;
                    L.spin_words += (long long)P * probs[p]->nw;
                    L.field_floats += (long long)P * pm1_npad(probs[p]->n);  // rows padded for ring_pm1_kernel
                    L.rings.push_back(R);
                }
}

double chi_s_to_gamma(double A0, double s) {
    s = std::min(std::max(s, 1e-10), 1.0 - 1e-10);
    return A0 * (1.0 - s) / s;
}

// Stage 2 of run_chi (sqa_chi_annealer.cpp:283-387), float64, same operation
// order: the chi_B peak, floor, 4096-point trapezoid CDF of
// w(s) = max(chi_B(s), floor), its inverse at uniform targets, the beta ramp.
// scalars = {s*, Gamma*, J_perp*, floor}.
void chi_schedule(int Pts, const double *xs, const double *gs, const double *ys, double beta, double gamma_start,
                  double gamma_end, double A0, int slices, int num_steps, double floor_fraction, double ramp_fraction,
                  double ramp_start, double *betas, double *gammas, double *s_sched, double *scalars) {
    const int peak = (int)(std::max_element(ys, ys + Pts) - ys);
    scalars[0] = xs[peak];
    scalars[1] = gs[peak];
    scalars[2] = trotter_coupling(beta, gs[peak], slices);
    const double max_chi = ys[peak];
    const bool degenerate = !(max_chi > 0.0) || !std::isfinite(max_chi);
    if (degenerate)
        std::fprintf(stderr, "[qlatanneal_b200 chi] WARNING: chi_B scan is flat/non-finite; "
                             "falling back to a linear-in-s schedule.\n");
    const double floor_ = degenerate ? 1.0 : std::max(floor_fraction * max_chi, 1e-12);
    scalars[3] = floor_;
    const double s_lo = A0 / (A0 + gamma_start), s_hi = A0 / (A0 + gamma_end);
    auto chi_weight = [&](double s) {
        double chi;
        if (s <= xs[0]) chi = ys[0];
        else if (s >= xs[Pts - 1]) chi = ys[Pts - 1];
        else {
            int hi = 1;
            while (hi < Pts && xs[hi] < s) ++hi;
            const int lo = hi - 1;
            const double t = (s - xs[lo]) / (xs[hi] - xs[lo]);
            chi = ys[lo] + t * (ys[hi] - ys[lo]);
        }
        return std::max(chi, floor_);
    };
    int n1 = 0;
    if (ramp_fraction > 0.0) {
        n1 = (int)(size_t)(ramp_fraction * (double)num_steps);
        if (n1 > num_steps - 2) n1 = num_steps - 2;
    }
    const int n2 = num_steps - n1;
    const int GRID = 4096;
    const double hs = (s_hi - s_lo) / (double)GRID;
    std::vector<double> cdf(GRID + 2, 0.0);
    double w_left = chi_weight(s_lo);
    for (int k = 1; k <= GRID; ++k) {
        const double sk = s_lo + (double)k * hs;
        const double w_right = chi_weight(sk);
        cdf[k] = cdf[k - 1] + 0.5 * (w_left + w_right) * hs;
        w_left = w_right;
    }
    const double cdf_end = cdf[GRID];
    for (int s = 0; s < num_steps; ++s) {
        betas[s] = beta;
        gammas[s] = gamma_start;
        s_sched[s] = s_lo;
    }
    for (int step = 0; step < n1; ++step) {
        const double frac = n1 > 1 ? (double)step / (double)(n1 - 1) : 1.0;
        betas[step] = ramp_start + (beta - ramp_start) * frac;
    }
    int cell = 0;
    for (int t = 0; t < n2; ++t) {
        const double target = cdf_end > 0.0 ? ((double)t / (double)(n2 - 1)) * cdf_end : 0.0;
        while (cell < GRID && cdf[cell + 1] < target) ++cell;
        const double c0 = cdf[cell], c1 = cdf[cell + 1];
        const double frac = c1 > c0 ? (target - c0) / (c1 - c0) : 0.0;
        const double s_t = s_lo + ((double)cell + frac) * hs;
        s_sched[n1 + t] = s_t;
        gammas[n1 + t] = std::min(std::max(chi_s_to_gamma(A0, s_t), gamma_end), gamma_start);
    }
}

int upload_common(qa_ctx *ctx, const qa_problem *const *probs, int np, const Layout &L, ProbDev **d_probs,
                  RingDev **d_rings, uint32_t **d_spins, float **d_fields) {
    std::vector<ProbDev> pd(np);
    for (int p = 0; p < np; ++p) pd[p] = probs[p]->dev;
    void *v;
    QA_TRY(ws_get(ctx, W_PROBS, sizeof(ProbDev) * np, &v));
    *d_probs = static_cast<ProbDev *>(v);
    QA_CK(cudaMemcpyAsync(*d_probs, pd.data(), sizeof(ProbDev) * np, cudaMemcpyHostToDevice, ctx->stream));
    QA_TRY(ws_get(ctx, W_RINGS, sizeof(RingDev) * L.rings.size(), &v));
    *d_rings = static_cast<RingDev *>(v);
    QA_CK(cudaMemcpyAsync(*d_rings, L.rings.data(), sizeof(RingDev) * L.rings.size(), cudaMemcpyHostToDevice,
                          ctx->stream));
    QA_TRY(ws_get(ctx, W_SPINS, sizeof(uint32_t) * L.spin_words, &v));
    *d_spins = static_cast<uint32_t *>(v);
    QA_TRY(ws_get(ctx, W_FIELDS, sizeof(float) * L.field_floats, &v));
    *d_fields = static_cast<float *>(v);
    return QA_OK;
}

// Whether a dense problem's couplings are integers in [-127, 127]; if so its
// int8 rows for the tensor-core field init are built (once per problem).
int tc_prepare(qa_ctx *ctx, qa_problem *P) {
    if (P->tc_int8 >= 0) return QA_OK;
    P->tc_int8 = 0;
    if (P->kind != K_DENSE || !P->dev.J32) return QA_OK;
    const int n = P->n;
    int *d_ok = nullptr;
    QA_CK(cudaMallocAsync(reinterpret_cast<void **>(&d_ok), sizeof(int), ctx->stream));
    const int one = 1;
    QA_CK(cudaMemcpyAsync(d_ok, &one, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    tc_int8_check_kernel<<<256, 256, 0, ctx->stream>>>(P->dev.J32, (long long)n * n, d_ok);
    QA_CK(cudaGetLastError());
    int ok = 0;
    QA_CK(cudaMemcpyAsync(&ok, d_ok, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaStreamSynchronize(ctx->stream));
    QA_CK(cudaFreeAsync(d_ok, ctx->stream));
    if (!ok) return QA_OK;
    const int ldj = (n + TC_K - 1) / TC_K * TC_K, rows = (n + TC_N - 1) / TC_N * TC_N;
    void *d = nullptr;
    QA_CK(cudaMalloc(&d, (size_t)rows * ldj));
    P->allocs.push_back(d);
    P->J8 = static_cast<int8_t *>(d);
    P->tc_ldj = ldj;
    tc_pack_couplings_kernel<<<256, 256, 0, ctx->stream>>>(P->dev.J32, n, ldj, rows, P->J8);
    QA_CK(cudaGetLastError());
    P->tc_int8 = 1;
    return QA_OK;
}

// The initial fields of every cell of dense problems with int8-exact
// couplings on the tensor cores (tc_fields_kernel), one launch per problem
// over its rings (rings are ordered by problem).  *done = false when some
// problem does not qualify (the caller then runs the float64 init).
int tc_init_fields(qa_ctx *ctx, const qa_problem *const *probs, int np, const Layout &L, const RingDev *d_rings,
                   uint32_t *d_spins, float *d_fields, int P, unsigned long long *err, bool *done) {
    *done = false;
    if (std::getenv("QA_DISABLE_TC_INIT")) return QA_OK;
    for (int p = 0; p < np; ++p) {
        QA_TRY(tc_prepare(ctx, const_cast<qa_problem *>(probs[p])));
        if (probs[p]->tc_int8 != 1) return QA_OK;
    }
    int r0 = 0;
    for (int p = 0; p < np; ++p) {
        int cnt = 0;
        while (r0 + cnt < (int)L.rings.size() && L.rings[r0 + cnt].prob == p) ++cnt;
        if (cnt == 0) continue;
        TcFieldParams tp{};
        tp.rings = d_rings + r0;
        tp.spins = d_spins;
        tp.fields = d_fields;
        tp.J8 = probs[p]->J8;
        tp.ldj = probs[p]->tc_ldj;
        tp.n = probs[p]->n;
        tp.nw = probs[p]->nw;
        tp.P = P;
        tp.n_cells = cnt * P;
        tp.err = err;
        const dim3 grid((tp.n_cells + TC_M - 1) / TC_M, (tp.n + TC_N - 1) / TC_N);
        tc_fields_kernel<<<grid, 128, 0, ctx->stream>>>(tp);
        QA_CK(cudaGetLastError());
        r0 += cnt;
    }
    *done = true;
    return QA_OK;
}

int init_state(qa_ctx *ctx, int kind, const ProbDev *d_probs, const RingDev *d_rings, int n_rings, uint32_t *d_spins,
               float *d_fields, int P, int n_max, int nw_max, uint32_t tag, bool with_fields = true,
               const qa_problem *const *probs = nullptr, int np = 0, const Layout *L = nullptr,
               unsigned long long *err = nullptr) {
    init_spins_kernel<<<dim3(n_rings, P), 128, 0, ctx->stream>>>(d_probs, d_rings, d_spins, P, tag, nw_max);
    QA_CK(cudaGetLastError());
    if (!with_fields) return QA_OK;
    if (kind == K_DENSE && probs && L && err) {
        bool done = false;
        QA_TRY(tc_init_fields(ctx, probs, np, *L, d_rings, d_spins, d_fields, P, err, &done));
        if (done) return QA_OK;
    }
    const int zb = std::max(1, std::min(64, (n_max + 127) / 128));
    int rc = QA_OK;
    dispatch_kind(kind, [&](auto K) {
        init_fields_kernel<decltype(K)::value><<<dim3(n_rings, P, zb), 128, nw_max * 4, ctx->stream>>>(
            d_probs, d_rings, d_spins, d_fields, P);
        if (cudaGetLastError() != cudaSuccess) rc = fail(QA_ERR_CUDA, "init_fields_kernel launch failed");
    });
    return rc;
}

int exact_energies(qa_ctx *ctx, int kind, const ProbDev *d_probs, const Layout &L, const uint32_t *d_bits,
                   double *d_exact) {
    std::vector<int> prob_of(L.rings.size());
    for (size_t i = 0; i < L.rings.size(); ++i) prob_of[i] = L.rings[i].prob;
    void *v;
    QA_TRY(ws_get(ctx, W_PROBOF, sizeof(int) * prob_of.size(), &v));
    int *d_pof = static_cast<int *>(v);
    QA_CK(cudaMemcpyAsync(d_pof, prob_of.data(), sizeof(int) * prob_of.size(), cudaMemcpyHostToDevice, ctx->stream));
    int rc = QA_OK;
    dispatch_kind(kind, [&](auto K) {
        exact_energy_kernel<decltype(K)::value><<<(unsigned)L.rings.size(), 32, L.nw_max * 4, ctx->stream>>>(
            d_probs, d_pof, d_bits, L.nw_max, d_exact, (int)L.rings.size());
        if (cudaGetLastError() != cudaSuccess) rc = fail(QA_ERR_CUDA, "exact_energy_kernel launch failed");
    });
    return rc;
}

// Which ring kernel a batch runs on, and with what launch shape.
struct RingPlan {
    bool pm1 = false;     // ring_pm1_kernel
    bool sparse = false;  // ring_sparse_kernel
    bool own_fields() const { return pm1 || sparse; }  // no field cache to initialise
    int gbytes = 4;       // pm1: bytes per field (4 int32, 2 int16)
    bool jw_smem = true;  // pm1: J bits in shared memory
    bool ref_order = false;  // qanneal's update order (else the parity checkerboard)
    bool order_global = false;  // ring_kernel: order rows read in global memory (too large for shared)
    int n_max = 0;        // largest model of the batch
    int W = 1;
    size_t smem = 0;
    int smem_fields = 1;
};

// Dense +-1 batches run the bit-packed kernel, in the first of these forms
// whose ring fits in shared memory: J bits + int32 fields, J bits + int16
// fields, int16 fields with J read from L2.  P <= 64 (worldlines are 64-bit
// columns) and n <= 2048.  Anything else runs ring_kernel.
int plan_rings(qa_ctx *ctx, const qa_problem *const *probs, int np, int kind, int P, int n_max, RingPlan *pl,
               bool clusters = false, bool ref_order = false) {
    pl->W = std::max(1, std::min(32, (P + 1) / 2));
    if (ctx->tune.warps_per_ring > 0) pl->W = std::max(1, std::min({32, P, ctx->tune.warps_per_ring}));
    pl->ref_order = ref_order;
    pl->n_max = n_max;
    if (ref_order && n_max > QA_ORDER_MAX_N)
        return fail(QA_ERR_ARG, "the shuffled update order supports at most 65536 spins per model.");
    // cluster moves are in ring_kernel only
    pl->pm1 = !clusters && kind == K_DENSE && P <= 64 && n_max <= 2048 && !std::getenv("QA_DISABLE_PM1");
    for (int p = 0; p < np && pl->pm1; ++p) pl->pm1 = probs[p]->dev.Jw != nullptr;
    if (pl->pm1) {
        const size_t cap = (size_t)ctx->smem_optin;
        const bool int32_only = std::getenv("QA_PM1_INT32_ONLY") != nullptr;
        // qanneal's order, n <= 512: int16 fields with the J bits read through
        // L1 first; the resolve loop's J reads at random visiting positions
        // conflict in shared memory and hit in L1 (n=512 P=32: 2-4% faster,
        // n=256 P=16 the same)
        const int form = ctx->tune.field_form >= 0 ? ctx->tune.field_form : (ref_order && n_max <= 512 ? 2 : -1);
        if (form == 0 && pm1_smem_bytes(P, n_max, 4, true, ref_order) <= cap) {
            pl->gbytes = 4; pl->jw_smem = true;
        } else if (form == 1 && !int32_only && pm1_smem_bytes(P, n_max, 2, true, ref_order) <= cap) {
            pl->gbytes = 2; pl->jw_smem = true;
        } else if (form == 2 && !int32_only && pm1_smem_bytes(P, n_max, 2, false, ref_order) <= cap) {
            pl->gbytes = 2; pl->jw_smem = false;
        } else if (pm1_smem_bytes(P, n_max, 4, true, ref_order) <= cap) {
            pl->gbytes = 4; pl->jw_smem = true;
        } else if (!int32_only && pm1_smem_bytes(P, n_max, 2, true, ref_order) <= cap) {
            pl->gbytes = 2; pl->jw_smem = true;
        } else if (!int32_only && pm1_smem_bytes(P, n_max, 2, false, ref_order) <= cap) {
            pl->gbytes = 2; pl->jw_smem = false;
        } else {
            pl->pm1 = false;
        }
    }
    if (pl->pm1) {
        pl->smem = pm1_smem_bytes(P, n_max, pl->gbytes, pl->jw_smem, ref_order);
        pl->smem_fields = 0;
        // qanneal's order pipelines the slices: one warp per slice shortens
        // each warp's share of the wavefront.  Taken where it costs no
        // resident ring: P <= 16 (512 threads), or a ring whose shared memory
        // leaves one CTA per SM anyway (measured: n=256/2048 P=16 and n=1024
        // P=32 8-26% faster, n=512 P=32 at two rings per SM 2-13% slower)
        if (ref_order && ctx->tune.warps_per_ring <= 0 && P <= 32 &&
            (P <= 16 || 2 * pl->smem > (size_t)ctx->smem_optin))
            pl->W = P;
        return QA_OK;
    }
    // sparse integer couplings: fields on demand, worldline sums from bits
    pl->sparse = !clusters && kind == K_SPARSE && P <= 64 &&
                 sparse_smem_bytes(P, n_max, ref_order) <= (size_t)ctx->smem_optin &&
                 !std::getenv("QA_DISABLE_SPARSE_INT");
    for (int p = 0; p < np && pl->sparse; ++p) pl->sparse = probs[p]->dev.spcv != nullptr;
    if (pl->sparse) {
        pl->smem = sparse_smem_bytes(P, n_max, ref_order);
        pl->smem_fields = 0;
        return QA_OK;
    }
    // generic kernel in qanneal's order: one warp per slice for P <= 16, as
    // for the +-1 kernel (HUBO n=1024 P=16: 11.5% faster)
    if (ref_order && ctx->tune.warps_per_ring <= 0 && P <= 16) pl->W = P;
    // fields in shared memory where they fit (up to 200 KB), the order rows
    // too, else the order rows read in global memory first
    const size_t fcap = (size_t)std::min(ctx->smem_optin, 200 * 1024), cap = (size_t)ctx->smem_optin;
    bool placed = false;
    for (int form = 0; form < 4 && !placed; ++form) {
        const bool fields = form == 0 || form == 1, ord_smem = form == 0 || form == 2;
        if (!ref_order && !ord_smem) continue;
        const size_t b = ring_smem_bytes(P, n_max, pl->W, fields, ref_order, ord_smem);
        if (b <= (fields ? fcap : cap)) {
            pl->smem = b;
            pl->smem_fields = fields ? 1 : 0;
            pl->order_global = ref_order && !ord_smem;
            placed = true;
        }
    }
    if (!placed) pl->smem = ring_smem_bytes(P, n_max, pl->W, false, ref_order, false);
    if (pl->smem > (size_t)ctx->smem_optin) return fail(QA_ERR_ARG, "ring state does not fit in shared memory.");
    return QA_OK;
}

// One launch of the planned ring kernel over steps [rp.step0, rp.step1).
// Opt kernel kern in to smem bytes of dynamic shared memory (above the
// default 48 KB), once per size increase rather than before every launch.
// The attribute belongs to the function on the device, which other contexts
// share: it is only ever raised (to the larger of the request and its current
// value), so what a context has recorded stays a lower bound.
static int opt_in_smem(qa_ctx *ctx, const void *kern, size_t smem) {
    if (smem <= 48 * 1024) return QA_OK;
    std::pair<const void *, size_t> *rec = nullptr;
    for (auto &e : ctx->smem_attr)
        if (e.first == kern) rec = &e;
    if (rec && rec->second >= smem) return QA_OK;
    cudaFuncAttributes fa{};
    QA_CK(cudaFuncGetAttributes(&fa, kern));
    size_t now = (size_t)std::max(fa.maxDynamicSharedSizeBytes, 0);
    if (now < smem) {
        QA_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        now = smem;
    }
    if (rec)
        rec->second = now;
    else
        ctx->smem_attr.emplace_back(kern, now);
    return QA_OK;
}

// qanneal's order: the ring kernels take the visiting orders of their sweeps
// from rows that order_fill_kernel writes before each launch.  Rows a step:
// the slice, cluster (ring_kernel only) and worldline sweeps.  All rows of a
// run's rings for the steps of one launch live in the W_ORDER workspace, at
// most kOrderBudget bytes: longer whole-grid launches are split into chunks of
// steps, rotated runs shorten their launches.
constexpr size_t kOrderBudget = (size_t)256 << 20;

static int ord_rows_per_step(const RingPlan &pl, const RingParams &rp) {
    return rp.spb + (pl.pm1 || pl.sparse ? 0 : rp.cls) + rp.wls;
}

// Steps of one launch whose rows for nr rings fit the budget.
static int ord_chunk_steps(const RingPlan &pl, const RingParams &rp, int nr, int steps) {
    const size_t per = (size_t)ord_rows_per_step(pl, rp) * ord_row_bytes(pl.n_max) * (size_t)std::max(nr, 1);
    const size_t fit = per ? kOrderBudget / per : (size_t)steps;
    return (int)std::max<size_t>(1, std::min<size_t>(fit, (size_t)std::max(steps, 1)));
}

// The rows buffer of nr rings x `steps` steps into rp (ring b at b * ord_ring).
static int ord_buffer(qa_ctx *ctx, const RingPlan &pl, RingParams *rp, int nr, int steps) {
    rp->ord_per_step = ord_rows_per_step(pl, *rp);
    rp->ord_stride = ord_row_entries(pl.n_max);
    rp->ord_ring = (long long)std::max(steps, 1) * std::max(rp->ord_per_step, 1) * rp->ord_stride;
    void *v;
    QA_TRY(ws_get(ctx, W_ORDER, sizeof(OrdT) * (size_t)rp->ord_ring * (size_t)std::max(nr, 1), &v));
    rp->ordg = static_cast<OrdT *>(v);
    return QA_OK;
}

// The rows of one launch (rp.step0 .. rp.step1 of rings rp.rings[0 .. n_rings)).
// The keys and counters of a row in shared memory where they fit, else in
// the W_OSCR workspace (used only by launches on the context stream).
static int fill_orders(qa_ctx *ctx, const RingPlan &pl, const RingParams &rp, int n_rings, cudaStream_t strm) {
    const long long total = (long long)(rp.step1 - rp.step0) * rp.ord_per_step * n_rings;
    if (total <= 0) return QA_OK;
    const size_t need = order_fill_bytes(pl.n_max);
    const int with_cls = pl.pm1 || pl.sparse ? 0 : 1;
    if (need <= (size_t)ctx->smem_optin) {
        const int grid = (int)std::min<long long>(total, (long long)ctx->sms * 8);
        QA_TRY(opt_in_smem(ctx, (const void *)order_fill_kernel, need));
        order_fill_kernel<<<grid, 256, need, strm>>>(rp, n_rings, with_cls, nullptr, 0);
    } else {
        if (strm != ctx->stream) return fail(QA_ERR_ARG, "order rows of this size need whole-grid launches");
        const int grid = (int)std::min<long long>(total, (long long)ctx->sms);
        void *v;
        QA_TRY(ws_get(ctx, W_OSCR, need * (size_t)grid, &v));
        order_fill_kernel<<<grid, 256, 0, strm>>>(rp, n_rings, with_cls, static_cast<unsigned char *>(v),
                                                  (long long)need);
    }
    QA_CK(cudaGetLastError());
    return QA_OK;
}

int launch_rings(qa_ctx *ctx, int kind, const RingPlan &pl, RingParams rp, int n_rings,
                 cudaStream_t stream = nullptr) {
    cudaStream_t strm = stream ? stream : ctx->stream;
    rp.W = pl.W;
    rp.smem_fields = pl.smem_fields;
    rp.ref_order = pl.ref_order ? 1 : 0;
    rp.ord_in_smem = pl.order_global ? 0 : 1;
    if (pl.ref_order && !rp.ordg) {
        // a whole-grid launch (context stream): the rows of chunks of steps,
        // each chunk's launch after its rows
        const int steps = rp.step1 - rp.step0, chunk = ord_chunk_steps(pl, rp, n_rings, steps);
        QA_TRY(ord_buffer(ctx, pl, &rp, n_rings, std::min(chunk, std::max(steps, 1))));
        for (int c0 = rp.step0; c0 < rp.step1 || c0 == rp.step0; c0 += chunk) {
            RingParams r2 = rp;
            r2.step0 = c0;
            r2.step1 = std::min(rp.step1, c0 + chunk);
            if (c0 > rp.step0) {
                r2.init_fields = 0;
                r2.init_scan = 0;
                if (r2.bsamp) r2.bsamp += (size_t)(c0 - rp.step0) * (rp.spb + rp.cls);
            }
            QA_TRY(launch_rings(ctx, kind, pl, r2, n_rings, strm));  // fills r2's rows first
            if (r2.step1 >= rp.step1) break;
        }
        return QA_OK;
    }
    if (pl.ref_order) {
        rp.ord_per_step = ord_rows_per_step(pl, rp);
        QA_TRY(fill_orders(ctx, pl, rp, n_rings, strm));
    }
    if (pl.pm1) {
        auto kern = pl.gbytes == 4 ? ring_pm1_kernel<int, true>
                                   : (pl.jw_smem ? ring_pm1_kernel<short, true> : ring_pm1_kernel<short, false>);
        QA_TRY(opt_in_smem(ctx, (const void *)kern, pl.smem));
        kern<<<n_rings, 32 * pl.W, pl.smem, strm>>>(rp);
        QA_CK(cudaGetLastError());
        return QA_OK;
    }
    if (pl.sparse) {
        QA_TRY(opt_in_smem(ctx, (const void *)ring_sparse_kernel, pl.smem));
        ring_sparse_kernel<<<n_rings, 32 * pl.W, pl.smem, strm>>>(rp);
        QA_CK(cudaGetLastError());
        return QA_OK;
    }
    int rc = QA_OK;
    dispatch_kind(kind, [&](auto Kd) {
        auto kern = ring_kernel<decltype(Kd)::value>;
        if (opt_in_smem(ctx, (const void *)kern, pl.smem) != QA_OK) {
            rc = QA_ERR_CUDA;
            return;
        }
        kern<<<n_rings, 32 * pl.W, pl.smem, strm>>>(rp);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = fail(QA_ERR_CUDA, std::string("ring_kernel launch: ") + cudaGetErrorString(e));
    });
    return rc;
}

template <class T>
int ws_array(qa_ctx *ctx, int slot, size_t count, T **out) {
    void *v;
    QA_TRY(ws_get(ctx, slot, sizeof(T) * count, &v));
    *out = static_cast<T *>(v);
    return QA_OK;
}

// Ring groups of a rotated run (run_rings_rotated): groups of G rings, one
// stream each, at most 128 streams.
struct RotPlan {
    int G, streams;
};
static RotPlan rot_plan(qa_ctx *ctx, int nr) {
    RotPlan r;
    r.G = std::max(2, (nr + 127) / 128);
    if (ctx->tune.rot_group > 0) r.G = std::max(ctx->tune.rot_group, (nr + 127) / 128);  // at most 128 streams
    r.streams = (nr + r.G - 1) / r.G;
    return r;
}
// Steps per rotated launch: the tuned length, else `auto_steps`.
static int rot_seg(qa_ctx *ctx, int auto_steps, int range) {
    const int s = ctx->tune.rot_steps > 0 ? ctx->tune.rot_steps : auto_steps;
    return std::max(1, std::min(s, std::max(1, range)));
}
// SQA: launches of 25..100 steps (an eighth of the run)
static int sqa_rot_seg(qa_ctx *ctx, int steps) {
    return rot_seg(ctx, std::max(25, std::min(100, steps / 8)), steps);
}

// Whether nr rings are worth rotating: more rings than SMs, and whole-grid
// launches would leave more than 3% of the resident slots idle.  With w the
// number of waves (rings over resident CTAs per SM times SMs), the last of
// ceil(w) waves is part-empty: the idle fraction is (ceil(w) - w) / ceil(w).
// For many full waves that is small and the extra launches cost more than the
// balance gains (an 8-instance sparse set of 8192 rings ran 1.7% slower).
// QA_WHOLE_GRID set: never (one launch over all rings per segment).
static bool rotation_pays(qa_ctx *ctx, int kind, const RingPlan &pl, int nr) {
    if (nr <= ctx->sms || std::getenv("QA_WHOLE_GRID") || ctx->tune.rotate == 0) return false;
    // order rows whose keys do not fit in shared memory are filled on the context stream only
    if (pl.ref_order && order_fill_bytes(pl.n_max) > (size_t)ctx->smem_optin) return false;
    if (ctx->tune.rotate == 1) return true;
    const int threads = 32 * pl.W;
    const void *kern = nullptr;
    if (pl.pm1)
        kern = pl.gbytes == 4 ? (const void *)ring_pm1_kernel<int, true>
                              : (pl.jw_smem ? (const void *)ring_pm1_kernel<short, true>
                                            : (const void *)ring_pm1_kernel<short, false>);
    else if (pl.sparse)
        kern = (const void *)ring_sparse_kernel;
    else
        dispatch_kind(kind, [&](auto Kd) { kern = (const void *)ring_kernel<decltype(Kd)::value>; });
    if (opt_in_smem(ctx, kern, pl.smem) != QA_OK) return false;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, pl.smem) != cudaSuccess || per_sm < 1)
        return false;
    const double w = (double)nr / ((double)per_sm * ctx->sms), full = std::ceil(w);
    return (full - w) / full > 0.03;
}

// The parameters of a launch over rings g0, g0 + 1, ...: every per-ring array
// the ring kernels index by block (ring records, best and final states, slot,
// samples) advanced to ring g0.  Sweep traces are indexed by grid position
// and are not offset: rotated runs carry none.
static RingParams ring_offset(RingParams r, int g0) {
    r.rings += g0;
    if (r.slot) r.slot += g0;
    r.best_E += g0;
    r.best_step += g0;
    if (r.best_slot) r.best_slot += g0;
    r.best_bits += (size_t)g0 * r.nw_max;
    if (r.final_bits) r.final_bits += (size_t)g0 * r.nw_max;
    if (r.ring_sum) r.ring_sum += (size_t)g0 * r.rec_stride;
    if (r.ring_min) r.ring_min += (size_t)g0 * r.rec_stride;
    if (r.ring_bond) r.ring_bond += (size_t)g0 * r.rec_stride;
    if (r.mag) r.mag += (size_t)g0 * r.steps_total * r.spb;
    if (r.bsamp) r.bsamp += (size_t)g0 * r.bstride;
    if (r.ordg) r.ordg += (size_t)g0 * r.ord_ring;
    return r;
}

// Instance sets of uneven size.  A whole-grid launch sizes every CTA's shared
// memory for the largest model, which can cost the smaller models resident
// rings.  Instead each model's rings run in launches of their own, with the
// plan of that model alone, side by side on the context's side streams
// (forked from and joined into the context stream, like the rotated launches);
// the kernels, keys and per-ring records are those of the whole-grid launch,
// so the results are the same bit for bit.
struct ModelRun {
    RingPlan pl;
    int g0 = 0, nr = 0;  // the model's rings: g0 .. g0 + nr - 1
};

// The per-model plans of a set, or an empty list where they would not pay:
// one model, or no model whose own ring needs 80% of the set's shared memory
// or less.  A model whose own plan picks another kernel keeps the set's.
static int plan_models(qa_ctx *ctx, const qa_problem *const *probs, int np, int kind, int P, const RingPlan &set_pl,
                       int nr, bool clusters, bool ref_order, std::vector<ModelRun> *out) {
    out->clear();
    if (np < 2 || nr % np) return QA_OK;
    std::vector<ModelRun> mr(np);
    bool pays = false;
    for (int m = 0; m < np; ++m) {
        QA_TRY(plan_rings(ctx, probs + m, 1, kind, P, probs[m]->n, &mr[m].pl, clusters, ref_order));
        if (mr[m].pl.pm1 != set_pl.pm1 || mr[m].pl.sparse != set_pl.sparse) mr[m].pl = set_pl;
        mr[m].g0 = m * (nr / np);
        mr[m].nr = nr / np;
        pays = pays || 5 * mr[m].pl.smem <= 4 * set_pl.smem;
    }
    if (pays) *out = std::move(mr);
    return QA_OK;
}

static int ensure_side_streams(qa_ctx *ctx, int count) {
    while ((int)ctx->side.size() < count) {
        cudaStream_t x;
        cudaEvent_t e;
        QA_CK(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
        ctx->side.push_back(x);
        QA_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ctx->side_ev.push_back(e);
    }
    return QA_OK;
}

// Steps [s_begin, s_end) of every model of a set, each model on its own
// side stream (at most 128; models beyond share them), in launches of at most
// 256 steps.  qanneal's order: model m's visiting orders at its own row
// stride, the rows of all models for one launch's steps in the W_ORDER
// workspace (at most 1 GB: fewer steps per launch when they would not fit).
static int run_models(qa_ctx *ctx, int kind, const std::vector<ModelRun> &mr, const RingParams &rp, int s_begin,
                      int s_end, int *launches) {
    const int nm = (int)mr.size(), streams = std::min(nm, 128);
    int chunk = std::max(1, std::min(256, s_end - s_begin));
    const bool ordered = mr[0].pl.ref_order;
    OrdT *rows = nullptr;
    if (ordered) {
        size_t per_step = 0;
        for (const auto &m : mr) per_step += (size_t)m.nr * ord_rows_per_step(m.pl, rp) * ord_row_bytes(m.pl.n_max);
        if (per_step) chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)chunk, (4 * kOrderBudget) / per_step));
        void *v;
        QA_TRY(ws_get(ctx, W_ORDER, std::max<size_t>(per_step * (size_t)chunk, 16), &v));
        rows = static_cast<OrdT *>(v);
    }
    QA_TRY(ensure_side_streams(ctx, streams));
    QA_CK(cudaEventRecord(ctx->side_ev[0], ctx->stream));
    for (int k = 0; k < streams; ++k) QA_CK(cudaStreamWaitEvent(ctx->side[k], ctx->side_ev[0], 0));
    int n = 0, rc = QA_OK;
    for (int c0 = s_begin; c0 < s_end && rc == QA_OK; c0 += chunk) {
        const int c1 = std::min(s_end, c0 + chunk);
        size_t off = 0;  // entries
        for (int m = 0; m < nm && rc == QA_OK; ++m) {
            RingParams r2 = ring_offset(rp, mr[m].g0);
            if (r2.bsamp) r2.bsamp += (size_t)(c0 - s_begin) * (rp.spb + rp.cls);  // indexed from step0
            r2.step0 = c0;
            r2.step1 = c1;
            r2.init_fields = rp.init_fields && c0 == s_begin;
            r2.init_scan = rp.init_scan && c0 == s_begin;
            if (ordered) {
                r2.ord_per_step = ord_rows_per_step(mr[m].pl, rp);
                r2.ord_stride = ord_row_entries(mr[m].pl.n_max);
                r2.ord_ring = (long long)(c1 - c0) * std::max(r2.ord_per_step, 1) * r2.ord_stride;
                r2.ordg = rows + off;
                off += (size_t)mr[m].nr * (size_t)r2.ord_ring;
            }
            rc = launch_rings(ctx, kind, mr[m].pl, r2, mr[m].nr, ctx->side[m % streams]);
            if (rc == QA_OK) ++n;
        }
    }
    // join, also after a failed launch
    for (int k = 0; k < streams; ++k) {
        cudaError_t e1 = cudaEventRecord(ctx->side_ev[k], ctx->side[k]);
        cudaError_t e2 = e1 == cudaSuccess ? cudaStreamWaitEvent(ctx->stream, ctx->side_ev[k], 0) : e1;
        if (e2 != cudaSuccess && rc == QA_OK)
            rc = fail(QA_ERR_CUDA, std::string("per-model launches, join: ") + cudaGetErrorString(e2));
    }
    *launches = n;
    return rc;
}

// Steps [s_begin, s_end) of every ring as independent chains of short
// launches: groups of G rings, each group on its own stream, one launch per
// seg steps.  When the rings outnumber the SMs but do not fill whole waves,
// some SMs hold more rings than others (or a second wave runs part-empty); a
// group that ran on a lightly loaded SM finishes its launch early and its next
// launch takes whatever slot is free, so rings move between SMs at launch
// boundaries and all finish together, instead of SMs idling while the loaded
// ones finish.  Each ring keeps its key, counters and records, so the results
// are those of whole-grid launches.  rp's init_scan / init_fields apply to
// the first launch.  Forks from and joins into the context stream; returns
// the number of launches in *launches.
static int run_rings_rotated(qa_ctx *ctx, int kind, const RingPlan &pl, const RingParams &rp, int nr, int s_begin,
                             int s_end, int seg, int *launches) {
    if (rp.tr_bits || rp.tr_E || rp.tr_end_bits || rp.tr_end_E || rp.ring_spin)
        return fail(QA_ERR_ARG, "rotated ring launches carry no sweep traces");
    const RotPlan rt = rot_plan(ctx, nr);
    RingParams base = rp;
    if (pl.ref_order) {
        // every ring's rows of one launch; shorter launches where they would not fit
        seg = std::min(seg, ord_chunk_steps(pl, rp, nr, seg));
        QA_TRY(ord_buffer(ctx, pl, &base, nr, seg));
    }
    while ((int)ctx->side.size() < rt.streams) {
        cudaStream_t x;
        cudaEvent_t e;
        QA_CK(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
        ctx->side.push_back(x);
        QA_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ctx->side_ev.push_back(e);
    }
    // fork: every side stream starts after the context stream's work so far
    QA_CK(cudaEventRecord(ctx->side_ev[0], ctx->stream));
    for (int k = 0; k < rt.streams; ++k) QA_CK(cudaStreamWaitEvent(ctx->side[k], ctx->side_ev[0], 0));
    int n = 0, rc = QA_OK;
    for (int s0 = s_begin; s0 < s_end && rc == QA_OK; s0 += seg) {  // segment-major issue keeps the streams in step
        for (int k = 0; k < rt.streams; ++k) {
            RingParams r2 = ring_offset(base, k * rt.G);
            if (r2.bsamp) r2.bsamp += (size_t)(s0 - s_begin) * (rp.spb + rp.cls);  // indexed from step0
            r2.step0 = s0;
            r2.step1 = std::min(s_end, s0 + seg);
            r2.init_fields = rp.init_fields && s0 == s_begin;
            r2.init_scan = rp.init_scan && s0 == s_begin;
            rc = launch_rings(ctx, kind, pl, r2, std::min(rt.G, nr - k * rt.G), ctx->side[k]);
            if (rc != QA_OK) break;
            ++n;
        }
    }
    // join, also after a failed launch: the context stream must wait for
    // whatever the side streams already hold before its next workspace write
    for (int k = 0; k < rt.streams; ++k) {
        cudaError_t e1 = cudaEventRecord(ctx->side_ev[k], ctx->side[k]);
        cudaError_t e2 = e1 == cudaSuccess ? cudaStreamWaitEvent(ctx->stream, ctx->side_ev[k], 0) : e1;
        if (e2 != cudaSuccess && rc == QA_OK)
            rc = fail(QA_ERR_CUDA, std::string("rotated launches, join: ") + cudaGetErrorString(e2));
    }
    *launches = n;
    return rc;
}

// Batch buffers of an MLP (grown on demand) and the inputs/targets copied in.
int mlp_prepare(qa_mlp *m, int B, const float *X, const float *T) {
    const int L = (int)m->dims.size() - 1;
    if (B > m->cap_B) {
        for (float **p : {&m->acts, &m->dacts, &m->T, &m->rowloss})
            if (*p) { cudaFree(*p); *p = nullptr; }
        long long per_row = 0;
        for (int d : m->dims) per_row += d;
        QA_CK(cudaMalloc(&m->acts, sizeof(float) * per_row * B));
        QA_CK(cudaMalloc(&m->dacts, sizeof(float) * per_row * B));
        QA_CK(cudaMalloc(&m->T, sizeof(float) * (size_t)B * (m->dims[L] / 2)));
        QA_CK(cudaMalloc(&m->rowloss, sizeof(float) * B));
        m->cap_B = B;
    }
    m->aoff.assign(L + 1, 0);
    for (int l = 1; l <= L; ++l) m->aoff[l] = m->aoff[l - 1] + (long long)B * m->dims[l - 1];
    QA_CK(cudaMemcpyAsync(m->acts, X, sizeof(float) * (size_t)B * m->dims[0], cudaMemcpyHostToDevice, m->ctx->stream));
    if (T)
        QA_CK(cudaMemcpyAsync(m->T, T, sizeof(float) * (size_t)B * (m->dims[L] / 2), cudaMemcpyHostToDevice,
                              m->ctx->stream));
    return QA_OK;
}

int mlp_forward_dev(qa_mlp *m, int B) {
    const int L = (int)m->dims.size() - 1;
    for (int l = 0; l < L; ++l) {
        const int K = m->dims[l], N = m->dims[l + 1];
        mlp_fwd_kernel<<<(B * N + 127) / 128, 128, 0, m->ctx->stream>>>(m->acts + m->aoff[l], B, K,
                                                                        m->W16 + m->w16off[l], m->W + m->boff[l],
                                                                        m->acts + m->aoff[l + 1], N, l + 1 < L);
        QA_CK(cudaGetLastError());
    }
    return QA_OK;
}

// Loss and gradients (into m->g) of the last forward pass.
int mlp_backward_dev(qa_mlp *m, int B, float *loss) {
    const int L = (int)m->dims.size() - 1, M = m->dims[L] / 2;
    mlp_loss_kernel<<<B, 128, 0, m->ctx->stream>>>(m->acts + m->aoff[L], m->T, B, M, m->dacts + m->aoff[L],
                                                  m->rowloss);
    QA_CK(cudaGetLastError());
    for (int l = L - 1; l >= 0; --l) {
        const int K = m->dims[l], N = m->dims[l + 1];
        mlp_bwd_weight_kernel<<<(K * N + N + 127) / 128, 128, 0, m->ctx->stream>>>(
            m->acts + m->aoff[l], m->dacts + m->aoff[l + 1], B, K, N, m->g + m->woff[l], m->g + m->boff[l]);
        QA_CK(cudaGetLastError());
        if (l > 0) {
            mlp_bwd_input_kernel<<<(B * K + 127) / 128, 128, 0, m->ctx->stream>>>(
                m->dacts + m->aoff[l + 1], m->W16 + m->w16off[l], m->acts + m->aoff[l], B, K, N, m->dacts + m->aoff[l]);
            QA_CK(cudaGetLastError());
        }
    }
    if (loss) {
        std::vector<float> rl(B);
        QA_CK(cudaMemcpyAsync(rl.data(), m->rowloss, sizeof(float) * B, cudaMemcpyDeviceToHost, m->ctx->stream));
        QA_CK(cudaStreamSynchronize(m->ctx->stream));
        double s = 0.0;
        for (float x : rl) s += x;
        *loss = (float)(s / ((double)B * M));
    }
    return QA_OK;
}

}  // namespace

// ====================================================================== API
extern "C" {

const char *qa_version(void) { return "qlatanneal-b200 0.1.0 (qanneal 2.0 sweep engine, sm_100a)"; }

int qa_last_error(char *buf, size_t len) {
    if (!buf || len == 0) return QA_ERR_ARG;
    std::snprintf(buf, len, "%s", g_err.c_str());
    return QA_OK;
}

int qa_device_count(int *count) {
    if (!count) return fail(QA_ERR_ARG, "null count");
    QA_CK(cudaGetDeviceCount(count));
    return QA_OK;
}

int qa_create(qa_ctx **out, int device) {
    if (!out) return fail(QA_ERR_ARG, "null output pointer");
    *out = nullptr;
    int cnt = 0;
    QA_CK(cudaGetDeviceCount(&cnt));
    if (device < 0 || device >= cnt) return fail(QA_ERR_ARG, "device index out of range");
    QA_CK(cudaSetDevice(device));
    qa_ctx *ctx = new qa_ctx();
    ctx->device = device;
    ctx->pool = std::make_shared<BlockPool>();
    ctx->pool->device = device;
    cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    for (int i = 0; i < 4 && e == cudaSuccess; ++i) e = cudaEventCreate(&ctx->ev[i]);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->stage.sent, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) {
        qa_destroy(ctx);
        return fail(QA_ERR_CUDA, std::string("context setup: ") + cudaGetErrorString(e));
    }
    *out = ctx;
    return QA_OK;
}

int qa_destroy(qa_ctx *ctx) {
    if (!ctx) return QA_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto &b : ctx->ws)
        if (b.p) cudaFree(b.p);
    for (auto &e : ctx->ev)
        if (e) cudaEventDestroy(e);
    for (auto &x : ctx->side) cudaStreamDestroy(x);
    for (auto &x : ctx->side_ev) cudaEventDestroy(x);
    ctx->stage.release();
    ctx->down.release();
    if (ctx->stage.sent) cudaEventDestroy(ctx->stage.sent);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return QA_OK;
}

int qa_problem_free(qa_problem *p) {
    if (!p) return QA_OK;
    if (p->pool) cudaSetDevice(p->pool->device);
    for (void *d : p->allocs) cudaFree(d);
    if (p->block) p->pool->give(p->block, p->block_bytes);
    delete p;
    return QA_OK;
}

int qa_problem_size(const qa_problem *p, int *n) {
    if (!p || !n) return fail(QA_ERR_ARG, "null argument");
    *n = p->n;
    return QA_OK;
}

// The device-derived dense arrays (J32, and Jw when every upper coupling is
// +-1) from the J64 already in the block; one flag read back decides Jw.
static int derive_dense(qa_problem *P) {
    qa_ctx *ctx = P->ctx;
    const int n = P->n, nw = (n + 31) / 32, np = pm1_npad(n);
    int *d_flag;
    QA_TRY(ws_array(ctx, W_FLAG, 1, &d_flag));
    QA_CK(cudaMemsetAsync(d_flag, 0, sizeof(int), ctx->stream));
    QA_CK(cudaMemsetAsync(const_cast<uint32_t *>(P->dev.Jw), 0, sizeof(uint32_t) * (size_t)nw * np, ctx->stream));
    dense_derive_kernel<<<dim3(nw, nw), dim3(kIngestTile, 8), 0, ctx->stream>>>(
        P->dev.J64, n, const_cast<float *>(P->dev.J32), const_cast<uint32_t *>(P->dev.Jw), np, d_flag);
    QA_CK(cudaGetLastError());
    int not_pm1 = 0;
    QA_CK(cudaMemcpyAsync(&not_pm1, d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaStreamSynchronize(ctx->stream));
    if (not_pm1) P->dev.Jw = nullptr;
    return QA_OK;
}

int qa_problem_dense(qa_ctx *ctx, int n, const double *h, const double *J, double c, qa_problem **out) {
    QA_TRY(begin(ctx));
    if (!out) return fail(QA_ERR_ARG, "null output pointer");
    *out = nullptr;
    if (n <= 0) return fail(QA_ERR_ARG, "DenseIsing size must be > 0.");
    if (!h || !J) return fail(QA_ERR_ARG, "DenseIsing h/J must not be null.");
    qa_problem *P = new qa_problem();
    P->ctx = ctx;
    P->kind = K_DENSE;
    P->n = n;
    P->nw = (n + 31) / 32;
    P->c = c;
    // J64 as given; the float32 mirror of its upper triangle (DenseIsing::energy
    // reads i < j) and the +-1 bit rows are derived on the device
    int rc = common_h(P, h);
    if (rc == QA_OK) rc = upload(P, J, (size_t)n * n, &P->dev.J64);
    if (rc == QA_OK) {
        reserve_array(P, (size_t)n * n, &P->dev.J32);
        reserve_array(P, (size_t)P->nw * pm1_npad(n), &P->dev.Jw);
        rc = finish_problem(P);
    }
    if (rc == QA_OK) rc = derive_dense(P);
    if (rc != QA_OK) {
        qa_problem_free(P);
        return rc;
    }
    *out = P;
    return QA_OK;
}

int qa_problem_qubo(qa_ctx *ctx, int n, const double *Q, double *h_out, double *c_out, qa_problem **out) {
    QA_TRY(begin(ctx));
    if (!out) return fail(QA_ERR_ARG, "null output pointer");
    *out = nullptr;
    if (n <= 0) return fail(QA_ERR_ARG, "QUBO size must be > 0.");
    if (!Q) return fail(QA_ERR_ARG, "QUBO matrix must not be null.");
    qa_problem *P = new qa_problem();
    P->ctx = ctx;
    P->kind = K_DENSE;
    P->n = n;
    P->nw = (n + 31) / 32;
    reserve_array(P, (size_t)n, &P->dev.h32);
    reserve_array(P, (size_t)n, &P->dev.h64);
    reserve_array(P, (size_t)n * n, &P->dev.J64);
    reserve_array(P, (size_t)n * n, &P->dev.J32);
    reserve_array(P, (size_t)P->nw * pm1_npad(n), &P->dev.Jw);
    int rc = finish_problem(P);
    double *d_Q = nullptr;
    if (rc == QA_OK) rc = ws_array(ctx, W_QSTAGE, (size_t)n * n, &d_Q);
    if (rc == QA_OK) {
        const cudaError_t e = cudaMemcpyAsync(d_Q, Q, sizeof(double) * (size_t)n * n, cudaMemcpyHostToDevice,
                                              ctx->stream);
        if (e != cudaSuccess) rc = fail(QA_ERR_CUDA, cudaGetErrorString(e));
    }
    if (rc == QA_OK) {
        qubo_rows_kernel<<<(n + kIngestTile - 1) / kIngestTile, dim3(kIngestTile, 8), 0, ctx->stream>>>(
            d_Q, n, const_cast<double *>(P->dev.J64), const_cast<double *>(P->dev.h64),
            const_cast<float *>(P->dev.h32));
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = fail(QA_ERR_CUDA, cudaGetErrorString(e));
    }
    if (rc == QA_OK) {
        // c = sum_i (W[i][i]/4 + sum_j W[i][j]/4), the single running sum of
        // qubo.cpp:57-66, on the host while the device builds the arrays
        double c = 0.0;
        for (int i = 0; i < n; ++i) {
            const double *qi = Q + (size_t)i * n;
            const double wii = 0.5 * (qi[i] + qi[i]);
            c += 0.25 * wii;
            for (int j = 0; j < n; ++j) {
                const double w = 0.5 * (qi[j] + Q[(size_t)j * n + i]);
                c += 0.25 * w;
            }
        }
        P->c = P->dev.c = c;
        if (c_out) *c_out = c;
        rc = derive_dense(P);
    }
    if (rc == QA_OK && h_out) {
        cudaError_t e = cudaMemcpyAsync(h_out, P->dev.h64, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = fail(QA_ERR_CUDA, cudaGetErrorString(e));
    }
    if (rc != QA_OK) {
        qa_problem_free(P);
        return rc;
    }
    *out = P;
    return QA_OK;
}

int qa_problem_sparse(qa_ctx *ctx, int n, const double *h, int m, const int64_t *ei, const int64_t *ej,
                      const double *w, double c, qa_problem **out) {
    QA_TRY(begin(ctx));
    if (!out) return fail(QA_ERR_ARG, "null output pointer");
    *out = nullptr;
    if (n <= 0) return fail(QA_ERR_ARG, "SparseIsing size must be > 0.");
    if (!h || m < 0 || (m > 0 && (!ei || !ej || !w))) return fail(QA_ERR_ARG, "SparseIsing arrays must not be null.");
    for (int e = 0; e < m; ++e) {
        if (ei[e] < 0 || ej[e] < 0 || ei[e] >= n || ej[e] >= n)
            return fail(QA_ERR_ARG, "SparseIsing edge index out of range.");
        if (ei[e] == ej[e]) return fail(QA_ERR_ARG, "SparseIsing self-edge not allowed.");
    }
    // adjacency in insertion order (sparse_ising.cpp:35-41); entries of one
    // neighbour merged in float64 in that order; rows sorted by neighbour.
    std::vector<std::vector<std::pair<int, double>>> adj(n);
    for (int e = 0; e < m; ++e) {
        adj[ei[e]].push_back({(int)ej[e], w[e]});
        adj[ej[e]].push_back({(int)ei[e], w[e]});
    }
    std::vector<int> rowptr(n + 1, 0), col;
    std::vector<float> val;
    for (int i = 0; i < n; ++i) {
        auto &a = adj[i];
        std::stable_sort(a.begin(), a.end(), [](const auto &x, const auto &y) { return x.first < y.first; });
        rowptr[i] = (int)col.size();
        size_t k = 0;
        while (k < a.size()) {
            double acc = 0.0;
            size_t kk = k;
            while (kk < a.size() && a[kk].first == a[k].first) acc += a[kk++].second;
            col.push_back(a[k].first);
            val.push_back((float)acc);
            k = kk;
        }
    }
    rowptr[n] = (int)col.size();
    // integer couplings (merged): (column, value) pairs for ring_sparse_kernel;
    // every field then stays an exact integer (|g| <= 2^24 checked per row)
    bool integer = true;
    for (int i = 0; i < n && integer; ++i) {
        double tot = 0.0;
        for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) {
            const double v = (double)val[e];
            integer = integer && v == std::nearbyint(v) && std::fabs(v) <= 32767.0;
            tot += std::fabs(v);
        }
        integer = integer && tot < 16777216.0;
    }
    std::vector<int2> spcv;
    if (integer) {
        spcv.resize(col.size());
        for (size_t e = 0; e < col.size(); ++e) spcv[e] = make_int2(col[e], (int)val[e]);
    }
    // the same rows as 16-byte records where every row fits one: at most 4
    // neighbours, values in [-127, 127], columns below 65536
    bool slab = integer && n < 65536;
    for (int i = 0; i < n && slab; ++i) {
        slab = rowptr[i + 1] - rowptr[i] <= 4;
        for (int e = rowptr[i]; e < rowptr[i + 1] && slab; ++e) slab = std::fabs((double)val[e]) <= 127.0;
    }
    std::vector<uint4> spslab;
    if (slab) {
        spslab.assign(n, make_uint4(0u, 0u, 0u, 0u));
        for (int i = 0; i < n; ++i) {
            uint32_t c4[4] = {0u, 0u, 0u, 0u}, v4 = 0u;
            for (int e = rowptr[i], k = 0; e < rowptr[i + 1]; ++e, ++k) {
                c4[k] = (uint32_t)col[e];
                v4 |= ((uint32_t)(int)val[e] & 0xFFu) << (8 * k);
            }
            spslab[i] = make_uint4(c4[0] | (c4[1] << 16), c4[2] | (c4[3] << 16), v4, 0u);
        }
    }
    std::vector<int> e_i(m), e_j(m);
    for (int e = 0; e < m; ++e) { e_i[e] = (int)ei[e]; e_j[e] = (int)ej[e]; }
    qa_problem *P = new qa_problem();
    P->ctx = ctx;
    P->kind = K_SPARSE;
    P->n = n;
    P->nw = (n + 31) / 32;
    P->m = m;
    P->c = c;
    int rc = common_h(P, h);
    if (rc == QA_OK) rc = upload(P, rowptr.data(), rowptr.size(), &P->dev.rowptr);
    if (rc == QA_OK) rc = upload(P, col.data(), col.size(), &P->dev.col);
    if (rc == QA_OK) rc = upload(P, val.data(), val.size(), &P->dev.val32);
    if (rc == QA_OK) rc = upload(P, e_i.data(), e_i.size(), &P->dev.ei);
    if (rc == QA_OK) rc = upload(P, e_j.data(), e_j.size(), &P->dev.ej);
    if (rc == QA_OK) rc = upload(P, w, (size_t)m, &P->dev.ew);
    if (rc == QA_OK && integer) rc = upload(P, spcv.data(), spcv.size(), &P->dev.spcv);
    if (rc == QA_OK && slab) rc = upload(P, spslab.data(), spslab.size(), &P->dev.spslab);
    if (rc != QA_OK) {
        qa_problem_free(P);
        return rc;
    }
    rc = finish_problem(P);
    if (rc != QA_OK) {
        qa_problem_free(P);
        return rc;
    }
    *out = P;
    return QA_OK;
}

int qa_problem_hubo(qa_ctx *ctx, int n, const double *h, int n_terms, const int64_t *term_ptr,
                    const int32_t *term_vars, const double *coeff, double c, qa_problem **out) {
    QA_TRY(begin(ctx));
    if (!out) return fail(QA_ERR_ARG, "null output pointer");
    *out = nullptr;
    if (n <= 0) return fail(QA_ERR_ARG, "HigherOrderIsing size must be > 0.");
    if (!h || n_terms < 0 || (n_terms > 0 && (!term_ptr || !term_vars || !coeff)))
        return fail(QA_ERR_ARG, "HigherOrderIsing arrays must not be null.");
    std::vector<int> tptr(n_terms + 1, 0), tvars;
    for (int t = 0; t < n_terms; ++t) {
        const int64_t a = term_ptr[t], b = term_ptr[t + 1];
        if (b - a < 2) return fail(QA_ERR_ARG, "HigherOrderIsing terms must have degree >= 2 (fold lower degrees).");
        for (int64_t k = a; k < b; ++k) {
            if (term_vars[k] < 0 || term_vars[k] >= n)
                return fail(QA_ERR_ARG, "HigherOrderIsing term variable index out of range.");
            if (k > a && term_vars[k] <= term_vars[k - 1])
                return fail(QA_ERR_ARG, "HigherOrderIsing term variables must be strictly increasing.");
            tvars.push_back(term_vars[k]);
        }
        tptr[t + 1] = (int)tvars.size();
    }
    std::vector<int> incptr(n + 1, 0);
    for (int v : tvars) incptr[v + 1]++;
    for (int i = 0; i < n; ++i) incptr[i + 1] += incptr[i];
    std::vector<int> incterm(tvars.size()), fillc(n, 0);
    for (int t = 0; t < n_terms; ++t)
        for (int k = tptr[t]; k < tptr[t + 1]; ++k) incterm[incptr[tvars[k]] + fillc[tvars[k]]++] = t;
    std::vector<float> c32(n_terms);
    for (int t = 0; t < n_terms; ++t) c32[t] = (float)coeff[t];
    // flip updates grouped by target (terms of degree <= 4 only)
    bool small_terms = true;
    for (int t = 0; t < n_terms && small_terms; ++t) small_terms = tptr[t + 1] - tptr[t] <= 4;
    std::vector<int> upd_ptr, upd_run;
    std::vector<int4> upd_rec;
    if (small_terms) {
        upd_ptr.assign(n + 1, 0);
        struct U { int v, t, w1, w2; };
        std::vector<U> u;
        for (int j = 0; j < n; ++j) {
            u.clear();
            for (int q = incptr[j]; q < incptr[j + 1]; ++q) {
                const int t = incterm[q];
                for (int k = tptr[t]; k < tptr[t + 1]; ++k) {
                    const int v = tvars[k];
                    if (v == j) continue;
                    int w[2] = {-1, -1}, nw_ = 0;
                    for (int k2 = tptr[t]; k2 < tptr[t + 1]; ++k2)
                        if (tvars[k2] != j && tvars[k2] != v) w[nw_++] = tvars[k2];
                    u.push_back({v, t, w[0], w[1]});
                }
            }
            std::stable_sort(u.begin(), u.end(), [](const U &a, const U &b) { return a.v != b.v ? a.v < b.v : a.t < b.t; });
            for (size_t k = 0; k < u.size(); ++k) {
                if (k == 0 || u[k].v != u[k - 1].v) upd_run.push_back((int)upd_rec.size());
                const float two = 2.0f * c32[u[k].t];
                int bits;
                std::memcpy(&bits, &two, 4);
                upd_rec.push_back(make_int4(u[k].v, u[k].w1, u[k].w2, bits));
            }
            upd_ptr[j + 1] = (int)upd_run.size();
        }
        upd_run.push_back((int)upd_rec.size());
    }
    qa_problem *P = new qa_problem();
    P->ctx = ctx;
    P->kind = K_HUBO;
    P->n = n;
    P->nw = (n + 31) / 32;
    P->T = n_terms;
    P->c = c;
    int rc = common_h(P, h);
    if (rc == QA_OK) rc = upload(P, tptr.data(), tptr.size(), &P->dev.tptr);
    if (rc == QA_OK) rc = upload(P, tvars.data(), tvars.size(), &P->dev.tvars);
    if (rc == QA_OK) rc = upload(P, incptr.data(), incptr.size(), &P->dev.incptr);
    if (rc == QA_OK) rc = upload(P, incterm.data(), incterm.size(), &P->dev.incterm);
    if (rc == QA_OK) rc = upload(P, c32.data(), c32.size(), &P->dev.coef32);
    if (rc == QA_OK) rc = upload(P, coeff, (size_t)n_terms, &P->dev.coef64);
    if (rc == QA_OK && small_terms) {
        rc = upload(P, upd_ptr.data(), upd_ptr.size(), &P->dev.upd_ptr);
        if (rc == QA_OK) rc = upload(P, upd_run.data(), upd_run.size(), &P->dev.upd_run);
        if (rc == QA_OK) rc = upload(P, upd_rec.data(), upd_rec.size(), &P->dev.upd_rec);
        // one 16-byte record per term for the per-step energy scan
        std::vector<int4> trec(std::max(n_terms, 1), make_int4(-1, -1, -1, -1));
        for (int t = 0; t < n_terms; ++t) {
            int v[4] = {-1, -1, -1, -1};
            for (int k = tptr[t]; k < tptr[t + 1]; ++k) v[k - tptr[t]] = tvars[k];
            trec[t] = make_int4(v[0], v[1], v[2], v[3]);
        }
        if (rc == QA_OK) rc = upload(P, trec.data(), trec.size(), &P->dev.trec);
    }
    if (rc != QA_OK) {
        qa_problem_free(P);
        return rc;
    }
    rc = finish_problem(P);
    if (rc != QA_OK) {
        qa_problem_free(P);
        return rc;
    }
    *out = P;
    return QA_OK;
}

// ---------------------------------------------------------------------- drift check
int qa_set_drift_check(qa_ctx *ctx, double tolerance) {
    if (!ctx) return fail(QA_ERR_ARG, "null context");
    ctx->drift_tol = tolerance > 0.0 ? tolerance : 0.0;
    return QA_OK;
}

int qa_set_tuning(qa_ctx *ctx, const qa_tuning *t) {
    if (!ctx) return fail(QA_ERR_ARG, "null context");
    if (!t) {
        ctx->tune = qa_tuning{0, -1, -1, 0, 0};
        return QA_OK;
    }
    if (t->warps_per_ring < 0 || t->warps_per_ring > 32 || t->field_form < -1 || t->field_form > 2 ||
        t->rotate < -1 || t->rotate > 1 || t->rot_steps < 0 || t->rot_group < 0)
        return fail(QA_ERR_ARG, "qa_set_tuning: a field out of range.");
    ctx->tune = *t;
    return QA_OK;
}

int qa_get_tuning(const qa_ctx *ctx, qa_tuning *t) {
    if (!ctx || !t) return fail(QA_ERR_ARG, "null argument");
    *t = ctx->tune;
    return QA_OK;
}

int qa_set_update_order(qa_ctx *ctx, int order) {
    if (!ctx) return fail(QA_ERR_ARG, "null context");
    if (order != QA_ORDER_REFERENCE && order != QA_ORDER_CHECKERBOARD)
        return fail(QA_ERR_ARG, "update order must be QA_ORDER_REFERENCE or QA_ORDER_CHECKERBOARD.");
    ctx->update_order = order;
    return QA_OK;
}

int qa_get_update_order(const qa_ctx *ctx, int *order) {
    if (!ctx || !order) return fail(QA_ERR_ARG, "null argument");
    *order = ctx->update_order;
    return QA_OK;
}

// After a run on float32 field caches (field rows of ring r at
// fields + field_off, stride n): the drift check when the context has one.
// Sets stats->max_field_drift; QA_ERR_DRIFT above the tolerance.
static int check_drift(qa_ctx *ctx, bool float_fields, int kind, const ProbDev *d_probs, const RingDev *d_rings,
                       int nr, const uint32_t *d_spins, const float *d_fields, int P, int n_max, int nw_max,
                       qa_stats *stats) {
    if (stats) stats->max_field_drift = 0.0;
    if (!(ctx->drift_tol > 0.0) || !float_fields) return QA_OK;
    unsigned long long *d_max;
    QA_TRY(ws_array(ctx, W_DRIFT, 1, &d_max));
    QA_CK(cudaMemsetAsync(d_max, 0, sizeof(unsigned long long), ctx->stream));
    const int zb = std::max(1, std::min(64, (n_max + 127) / 128));
    int rc = QA_OK;
    dispatch_kind(kind, [&](auto K) {
        field_drift_kernel<decltype(K)::value><<<dim3(nr, P, zb), 128, nw_max * 4, ctx->stream>>>(
            d_probs, d_rings, d_spins, d_fields, P, d_max);
        if (cudaGetLastError() != cudaSuccess) rc = fail(QA_ERR_CUDA, "field_drift_kernel launch failed");
    });
    QA_TRY(rc);
    unsigned long long bits = 0;
    QA_CK(cudaMemcpyAsync(&bits, d_max, sizeof(bits), cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaStreamSynchronize(ctx->stream));
    double d;
    std::memcpy(&d, &bits, sizeof(d));
    if (stats) stats->max_field_drift = d;
    if (d > ctx->drift_tol) {
        char msg[160];
        std::snprintf(msg, sizeof(msg), "incremental local fields drifted by %.3g from a float64 recompute (tolerance %.3g)",
                      d, ctx->drift_tol);
        return fail(QA_ERR_DRIFT, msg);
    }
    return QA_OK;
}

// ---------------------------------------------------------------------- SA
// SA reads (qa_sa_run) and SA replicas (qa_replica_run, which adds the
// magnetisation trace and the step of each replica's best).
static int sa_impl(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, const qa_sa_params *prm,
                   qa_run_out *outs, qa_stats *stats, double *const *mag_out, int32_t *const *bstep_out,
                   const qa_sa_trace *traces = nullptr) {
    QA_TRY(begin(ctx));
    if (!prm) return fail(QA_ERR_ARG, "null params");
    const int stride = traces && n_problems > 0 ? traces[0].stride : 1;
    if (traces)
        for (int p = 0; p < n_problems; ++p)
            if (traces[p].stride != stride || stride < 1)
                return fail(QA_ERR_ARG, "trace stride must be >= 1 and the same for every problem.");
    if (prm->steps <= 0 || !prm->betas) return fail(QA_ERR_ARG, "Schedule must contain at least one beta.");
    if (prm->sweeps_per_beta <= 0) return fail(QA_ERR_ARG, "sweeps_per_beta must be > 0.");
    if (prm->reads <= 0) return fail(QA_ERR_ARG, "reads must be > 0.");
    for (int s = 0; s < prm->steps; ++s)
        if (!(prm->betas[s] >= 0.0)) return fail(QA_ERR_ARG, "betas must be >= 0.");
    int kind, n_max;
    QA_TRY(check_batch(problems, n_problems, &kind, &n_max));
    Layout L;
    build_rings(L, problems, n_problems, prm->reads, 1, 1, prm->seed);
    const int nr = (int)L.rings.size();
    ProbDev *d_probs;
    RingDev *d_rings;
    uint32_t *d_spins;
    float *d_fields;
    QA_TRY(upload_common(ctx, problems, n_problems, L, &d_probs, &d_rings, &d_spins, &d_fields));
    std::vector<float> A(prm->steps);
    for (int s = 0; s < prm->steps; ++s) A[s] = (float)(2.0 * prm->betas[s]);  // B = 2 beta
    void *v;
    QA_TRY(ws_get(ctx, W_A, sizeof(float) * A.size(), &v));
    float *d_A = static_cast<float *>(v);
    QA_CK(cudaMemcpyAsync(d_A, A.data(), sizeof(float) * A.size(), cudaMemcpyHostToDevice, ctx->stream));
    QA_TRY(ws_get(ctx, W_SUM, sizeof(double) * (size_t)nr * prm->steps, &v));
    double *d_trace = static_cast<double *>(v);
    QA_TRY(ws_get(ctx, W_BESTE, sizeof(double) * nr, &v));
    double *d_best = static_cast<double *>(v);
    QA_TRY(ws_get(ctx, W_BITS, sizeof(uint32_t) * (size_t)nr * L.nw_max, &v));
    uint32_t *d_bits = static_cast<uint32_t *>(v);
    QA_TRY(ws_get(ctx, W_CNT, sizeof(unsigned long long) * 5, &v));
    unsigned long long *d_cnt = static_cast<unsigned long long *>(v);
    QA_TRY(ws_get(ctx, W_EXACT, sizeof(double) * nr, &v));
    double *d_exact = static_cast<double *>(v);
    QA_CK(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long) * 5, ctx->stream));
    double *d_mag = nullptr;
    int *d_bstep = nullptr;
    bool want_mag = mag_out != nullptr, want_states = false, want_end = false;
    for (int p = 0; traces && p < n_problems; ++p) {
        want_mag = want_mag || traces[p].magnetization;
        want_states = want_states || traces[p].states || traces[p].energies;
        want_end = want_end || traces[p].step_states;
    }
    if (want_mag) {
        QA_TRY(ws_get(ctx, W_MAG, sizeof(double) * (size_t)nr * prm->steps, &v));
        d_mag = static_cast<double *>(v);
    }
    if (mag_out) {
        QA_TRY(ws_get(ctx, W_BESTSTEP, sizeof(int) * nr, &v));
        d_bstep = static_cast<int *>(v);
    }
    const int rps = (prm->sweeps_per_beta + stride - 1) / stride;
    const size_t n_rec = (size_t)nr * prm->steps * rps;
    const size_t n_end = want_end ? (size_t)nr * prm->steps : 0;
    uint32_t *d_trb = nullptr, *d_treb = nullptr;
    double *d_tre = nullptr;
    if ((want_states ? n_rec * ((size_t)L.nw_max * 4 + 8) : 0) + n_end * L.nw_max * 4 > ((size_t)4 << 30))
        return fail(QA_ERR_ARG, "sweep trace over 4 GiB: raise the stride or trace fewer reads.");
    if (want_states) {
        QA_TRY(ws_array(ctx, W_TRB, n_rec * L.nw_max, &d_trb));
        QA_TRY(ws_array(ctx, W_TRE, n_rec, &d_tre));
    }
    if (want_end) QA_TRY(ws_array(ctx, W_TREB, n_end * L.nw_max, &d_treb));

    // dense +-1 couplings: bits and int32 fields in shared memory (fields built in-kernel);
    // traced runs take the generic kernel, which gives the same results
    bool pm1 = kind == K_DENSE && !traces && sa_pm1_smem_bytes(n_max) <= (size_t)ctx->smem_optin &&
               !std::getenv("QA_DISABLE_PM1");
    for (int p = 0; p < n_problems && pm1; ++p) pm1 = problems[p]->dev.Jw != nullptr;
    QA_CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    QA_TRY(init_state(ctx, kind, d_probs, d_rings, nr, d_spins, d_fields, 1, n_max, L.nw_max, DOM_INIT, !pm1));
    const int nwp = (L.nw_max + 3) & ~3, np4 = (n_max + 3) & ~3;
    size_t smem = (size_t)nwp * 4 + (size_t)np4 * 4;
    int smem_fields = (smem + (size_t)n_max * 4) <= (size_t)std::min(ctx->smem_optin, 160 * 1024) ? 1 : 0;
    if (smem_fields) smem += (size_t)n_max * 4;
    SAParams sp{};
    sp.probs = d_probs; sp.rings = d_rings; sp.spins = d_spins; sp.fields = d_fields; sp.B = d_A;
    sp.steps = prm->steps; sp.spb = prm->sweeps_per_beta; sp.smem_fields = smem_fields;
    sp.trace = d_trace; sp.best_E = d_best; sp.best_bits = d_bits; sp.nw_max = L.nw_max; sp.counters = d_cnt;
    sp.mag_trace = d_mag; sp.best_step = d_bstep;
    sp.tr_bits = d_trb; sp.tr_E = d_tre; sp.tr_end_bits = d_treb; sp.tr_stride = stride; sp.tr_rps = rps;
    QA_CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    int rc = QA_OK;
    if (pm1) {
        const size_t sm1 = sa_pm1_smem_bytes(n_max);
        if (sm1 > 48 * 1024)
            QA_CK(cudaFuncSetAttribute(sa_pm1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1));
        sa_pm1_kernel<<<nr, 32, sm1, ctx->stream>>>(sp);
        QA_CK(cudaGetLastError());
    } else {
        dispatch_kind(kind, [&](auto K) {
            auto kern = sa_kernel<decltype(K)::value>;
            if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            kern<<<nr, 32, smem, ctx->stream>>>(sp);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) rc = fail(QA_ERR_CUDA, std::string("sa_kernel launch: ") + cudaGetErrorString(e));
        });
    }
    QA_TRY(rc);
    QA_CK(cudaEventRecord(ctx->ev[2], ctx->stream));
    QA_TRY(exact_energies(ctx, kind, d_probs, L, d_bits, d_exact));
    QA_CK(cudaEventRecord(ctx->ev[3], ctx->stream));

    std::vector<double> trace((size_t)nr * prm->steps), exact(nr);
    std::vector<uint32_t> bits((size_t)nr * L.nw_max);
    unsigned long long cnt[5];
    QA_CK(cudaMemcpyAsync(trace.data(), d_trace, sizeof(double) * trace.size(), cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(exact.data(), d_exact, sizeof(double) * nr, cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(bits.data(), d_bits, sizeof(uint32_t) * bits.size(), cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(cnt, d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, ctx->stream));
    std::vector<double> mag(want_mag ? (size_t)nr * prm->steps : 0);
    std::vector<int> bst(mag_out ? nr : 0);
    if (want_mag)
        QA_CK(cudaMemcpyAsync(mag.data(), d_mag, sizeof(double) * mag.size(), cudaMemcpyDeviceToHost, ctx->stream));
    if (mag_out)
        QA_CK(cudaMemcpyAsync(bst.data(), d_bstep, sizeof(int) * nr, cudaMemcpyDeviceToHost, ctx->stream));
    std::vector<uint32_t> trb(want_states ? n_rec * L.nw_max : 0);
    std::vector<double> tre(want_states ? n_rec : 0);
    if (want_states) {
        QA_CK(cudaMemcpyAsync(trb.data(), d_trb, sizeof(uint32_t) * trb.size(), cudaMemcpyDeviceToHost, ctx->stream));
        QA_CK(cudaMemcpyAsync(tre.data(), d_tre, sizeof(double) * tre.size(), cudaMemcpyDeviceToHost, ctx->stream));
    }
    std::vector<uint32_t> treb(n_end * L.nw_max);
    if (want_end)
        QA_CK(cudaMemcpyAsync(treb.data(), d_treb, sizeof(uint32_t) * treb.size(), cudaMemcpyDeviceToHost,
                              ctx->stream));
    QA_CK(cudaStreamSynchronize(ctx->stream));
    for (int i = 0; i < nr; ++i) {
        const RingDev &R = L.rings[i];
        const int p = R.prob, r = R.out - p * prm->reads, n = problems[p]->n;
        qa_run_out &o = outs[p];
        if (o.best_spins) unpack_bits(bits.data() + (size_t)i * L.nw_max, n, o.best_spins + (size_t)r * n);
        if (o.best_energy) o.best_energy[r] = exact[i];
        if (o.energy_trace)
            std::memcpy(o.energy_trace + (size_t)r * prm->steps, trace.data() + (size_t)i * prm->steps,
                        sizeof(double) * prm->steps);
        if (mag_out && mag_out[p])
            std::memcpy(mag_out[p] + (size_t)r * prm->steps, mag.data() + (size_t)i * prm->steps,
                        sizeof(double) * prm->steps);
        if (bstep_out && bstep_out[p]) bstep_out[p][r] = bst[i];
        if (traces) {
            const qa_sa_trace &t = traces[p];
            const size_t per = (size_t)prm->steps * rps;
            if (t.magnetization)
                std::memcpy(t.magnetization + (size_t)r * prm->steps, mag.data() + (size_t)i * prm->steps,
                            sizeof(double) * prm->steps);
            if (t.energies) std::memcpy(t.energies + (size_t)r * per, tre.data() + (size_t)i * per, sizeof(double) * per);
            if (t.states)
                for (size_t k = 0; k < per; ++k)
                    unpack_bits(trb.data() + ((size_t)i * per + k) * L.nw_max, n, t.states + ((size_t)r * per + k) * n);
            if (t.step_states)
                for (int st = 0; st < prm->steps; ++st)
                    unpack_bits(treb.data() + ((size_t)i * prm->steps + st) * L.nw_max, n,
                                t.step_states + ((size_t)r * prm->steps + st) * n);
        }
    }
    if (stats) {
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, ctx->ev[1], ctx->ev[2]);
        cudaEventElapsedTime(&b, ctx->ev[0], ctx->ev[3]);
        stats->slice_attempts = (int64_t)cnt[0];
        stats->slice_accepts = (int64_t)cnt[1];
        stats->worldline_attempts = stats->worldline_accepts = 0;
        stats->sweep_ms = a;
        stats->total_ms = b;
        stats->max_field_drift = 0.0;
        stats->launches = pm1 ? 3 : 4;
        stats->sweep_launches = 1;
        stats->h2d_bytes = (int64_t)(sizeof(ProbDev) * n_problems + sizeof(RingDev) * nr + sizeof(float) * A.size() +
                                     sizeof(int) * nr);
        stats->d2h_bytes = (int64_t)(sizeof(double) * trace.size() + sizeof(double) * nr +
                                     sizeof(uint32_t) * bits.size() + sizeof(cnt));
    }
    QA_TRY(check_drift(ctx, !pm1, kind, d_probs, d_rings, nr, d_spins, d_fields, 1, n_max, L.nw_max, stats));
    return QA_OK;
}

int qa_sa_run(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, const qa_sa_params *prm,
              qa_run_out *outs, qa_stats *stats) {
    return sa_impl(ctx, problems, n_problems, prm, outs, stats, nullptr, nullptr);
}

int qa_sa_trace_run(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, const qa_sa_params *prm,
                    const qa_sa_trace *traces, qa_run_out *outs, qa_stats *stats) {
    if (!traces) return fail(QA_ERR_ARG, "null traces");
    return sa_impl(ctx, problems, n_problems, prm, outs, stats, nullptr, nullptr, traces);
}

int qa_replica_run(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, const qa_sa_params *prm,
                   qa_replica_out *outs, qa_stats *stats) {
    if (!outs || n_problems <= 0) return fail(QA_ERR_ARG, "null outputs or empty batch");
    if (prm && prm->reads <= 0) return fail(QA_ERR_ARG, "replicas must be > 0.");
    std::vector<qa_run_out> ro(n_problems);
    std::vector<double *> mag(n_problems);
    std::vector<int32_t *> bst(n_problems);
    for (int p = 0; p < n_problems; ++p) {
        ro[p] = qa_run_out{outs[p].best_spins, outs[p].best_energy, outs[p].energy_trace};
        mag[p] = outs[p].magnetization_trace;
        bst[p] = outs[p].best_step;
    }
    return sa_impl(ctx, problems, n_problems, prm, ro.data(), stats, mag.data(), bst.data());
}

// ---------------------------------------------------------------------- SQA
// SQA reads (qa_sqa_run); with traces, the observer form (qa_sqa_trace_run):
// the generic ring kernel also writes the sweep trace.
static int sqa_impl(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, const qa_sqa_params *prm,
                    qa_run_out *outs, qa_stats *stats, const qa_sqa_trace *traces) {
    QA_TRY(begin(ctx));
    if (!prm) return fail(QA_ERR_ARG, "null params");
    const int stride = traces && n_problems > 0 ? traces[0].stride : 1;
    if (traces)
        for (int p = 0; p < n_problems; ++p)
            if (traces[p].stride != stride || stride < 1)
                return fail(QA_ERR_ARG, "trace stride must be >= 1 and the same for every problem.");
    if (prm->steps <= 0 || !prm->betas || !prm->gammas) return fail(QA_ERR_ARG, "SQA schedule must contain betas.");
    if (prm->trotter_slices <= 0) return fail(QA_ERR_ARG, "trotter_slices must be > 0.");
    if (prm->replicas <= 0) return fail(QA_ERR_ARG, "replicas must be > 0.");
    if (prm->sweeps_per_beta < 0 || prm->worldline_sweeps < 0 || prm->cluster_sweeps < 0)
        return fail(QA_ERR_ARG, "sweep counts must be >= 0.");
    if (prm->sweeps_per_beta == 0 && prm->worldline_sweeps == 0 && prm->cluster_sweeps == 0)
        return fail(QA_ERR_ARG,
                    "At least one of sweeps_per_beta, worldline_sweeps, or cluster_sweeps must be > 0.");
    if (prm->reads <= 0) return fail(QA_ERR_ARG, "reads must be > 0.");
    int kind, n_max;
    QA_TRY(check_batch(problems, n_problems, &kind, &n_max));
    const int P = (prm->continuous_time_slices > 0 && prm->continuous_time_slices > prm->trotter_slices)
                      ? prm->continuous_time_slices
                      : prm->trotter_slices;
    const int K = prm->replicas, steps = prm->steps;
    if (prm->cluster_sweeps > 0 && P > 64)
        return fail(QA_ERR_UNSUPPORTED, "cluster_sweeps > 0 runs with at most 64 Trotter slices on the GPU.");
    Layout L;
    build_rings(L, problems, n_problems, prm->reads, K, P, prm->seed);
    const int nr = (int)L.rings.size();
    ProbDev *d_probs;
    RingDev *d_rings;
    uint32_t *d_spins;
    float *d_fields;
    QA_TRY(upload_common(ctx, problems, n_problems, L, &d_probs, &d_rings, &d_spins, &d_fields));
    std::vector<float> A(steps), T4(steps);
    for (int s = 0; s < steps; ++s) {
        const double bs = prm->betas[s] / (double)P;
        A[s] = (float)(2.0 * bs);  // B = 2 beta / P
        T4[s] = (float)(4.0 * trotter_coupling(prm->betas[s], prm->gammas[s], P));
    }
    void *v;
    QA_TRY(ws_get(ctx, W_A, sizeof(float) * steps, &v));
    float *d_A = static_cast<float *>(v);
    QA_TRY(ws_get(ctx, W_T4, sizeof(float) * steps, &v));
    float *d_T4 = static_cast<float *>(v);
    QA_CK(cudaMemcpyAsync(d_A, A.data(), sizeof(float) * steps, cudaMemcpyHostToDevice, ctx->stream));
    QA_CK(cudaMemcpyAsync(d_T4, T4.data(), sizeof(float) * steps, cudaMemcpyHostToDevice, ctx->stream));
    std::vector<float> JP(steps);  // join probability of the cluster moves (sqa_annealer.cpp:158)
    for (int s = 0; s < steps; ++s)
        JP[s] = (float)(1.0 - std::exp(-2.0 * trotter_coupling(prm->betas[s], prm->gammas[s], P)));
    QA_TRY(ws_get(ctx, W_JP, sizeof(float) * steps, &v));
    float *d_JP = static_cast<float *>(v);
    QA_CK(cudaMemcpyAsync(d_JP, JP.data(), sizeof(float) * steps, cudaMemcpyHostToDevice, ctx->stream));
    QA_TRY(ws_get(ctx, W_SUM, sizeof(double) * (size_t)nr * steps, &v));
    double *d_sum = static_cast<double *>(v);
    QA_TRY(ws_get(ctx, W_BESTE, sizeof(double) * nr, &v));
    double *d_best = static_cast<double *>(v);
    QA_TRY(ws_get(ctx, W_BESTSTEP, sizeof(int) * nr, &v));
    int *d_bstep = static_cast<int *>(v);
    QA_TRY(ws_get(ctx, W_BITS, sizeof(uint32_t) * (size_t)nr * L.nw_max, &v));
    uint32_t *d_bits = static_cast<uint32_t *>(v);
    QA_TRY(ws_get(ctx, W_CNT, sizeof(unsigned long long) * 5, &v));
    unsigned long long *d_cnt = static_cast<unsigned long long *>(v);
    QA_TRY(ws_get(ctx, W_EXACT, sizeof(double) * nr, &v));
    double *d_exact = static_cast<double *>(v);
    QA_CK(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long) * 5, ctx->stream));
    {
        std::vector<double> inf(nr, INFINITY);
        std::vector<int> neg(nr, -1);
        QA_CK(cudaMemcpyAsync(d_best, inf.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_bstep, neg.data(), sizeof(int) * nr, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaStreamSynchronize(ctx->stream));
    }

    // sweep traces (observers): the generic ring kernel writes them
    bool tr_rec = false, tr_end = false, tr_mag = false;
    for (int p = 0; traces && p < n_problems; ++p) {
        tr_rec = tr_rec || traces[p].ring_states || traces[p].ring_energies;
        tr_end = tr_end || traces[p].step_states || traces[p].step_energies;
        tr_mag = tr_mag || traces[p].magnetization;
    }
    const int rps = (prm->sweeps_per_beta + stride - 1) / stride + (prm->cluster_sweeps + stride - 1) / stride +
                    (prm->worldline_sweeps + stride - 1) / stride;
    const size_t n_rec = tr_rec ? (size_t)nr * steps * rps : 0, n_end = tr_end ? (size_t)nr * (steps + 1) : 0;
    if ((n_rec + n_end) * (size_t)P * ((size_t)L.nw_max * 4 + 8) > ((size_t)4 << 30))
        return fail(QA_ERR_ARG, "sweep trace over 4 GiB: raise the stride or trace fewer reads.");
    uint32_t *d_trb = nullptr, *d_treb = nullptr;
    double *d_tre = nullptr, *d_tree = nullptr;
    long long *d_rspin = nullptr;
    if (tr_rec) {
        QA_TRY(ws_array(ctx, W_TRB, n_rec * P * L.nw_max, &d_trb));
        QA_TRY(ws_array(ctx, W_TRE, n_rec * P, &d_tre));
    }
    if (tr_end) {
        QA_TRY(ws_array(ctx, W_TREB, n_end * P * L.nw_max, &d_treb));
        QA_TRY(ws_array(ctx, W_TREE, n_end * P, &d_tree));
    }
    if (tr_mag) QA_TRY(ws_array(ctx, W_RSPIN, (size_t)nr * steps, &d_rspin));

    QA_CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    RingPlan pl;
    QA_TRY(plan_rings(ctx, problems, n_problems, kind, P, n_max, &pl, prm->cluster_sweeps > 0 || traces,
                      ctx->update_order == QA_ORDER_REFERENCE));
    // dense +-1 couplings: the bit-packed kernel builds its fields in-kernel
    QA_TRY(init_state(ctx, kind, d_probs, d_rings, nr, d_spins, d_fields, P, n_max, L.nw_max, DOM_INIT, !pl.own_fields(),
                      problems, n_problems, &L, d_cnt + 4));
    RingParams rp{};
    rp.probs = d_probs; rp.rings = d_rings; rp.spins = d_spins; rp.fields = d_fields;
    rp.P = P; rp.steps_total = steps; rp.spb = prm->sweeps_per_beta; rp.wls = prm->worldline_sweeps;
    rp.slice_tag = DOM_SLICE; rp.slot = nullptr; rp.B = d_A; rp.T4 = d_T4; rp.per_slot_sched = 0;
    rp.cls = prm->cluster_sweeps; rp.JP = d_JP;
    rp.ring_sum = d_sum; rp.ring_min = nullptr; rp.ring_bond = nullptr;
    rp.best_E = d_best; rp.best_step = d_bstep; rp.best_bits = d_bits; rp.nw_max = L.nw_max; rp.mag = nullptr;
    rp.counters = d_cnt;
    rp.rec_base = 0;
    rp.rec_stride = steps;
    rp.tr_bits = d_trb; rp.tr_E = d_tre; rp.tr_end_bits = d_treb; rp.tr_end_E = d_tree; rp.ring_spin = d_rspin;
    rp.tr_stride = stride; rp.tr_rps = rps;
    QA_CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    const int seg = 256;
    int n_seg = (steps + seg - 1) / seg;
    // rotated launches where whole-grid ones would leave slots idle (a traced
    // run's records are indexed by the position in a whole-grid launch, so
    // those stay whole)
    std::vector<ModelRun> mr;  // an instance set of uneven size: per-model launches
    const bool rotate = !traces && steps >= 200 && rotation_pays(ctx, kind, pl, nr);
    if (!traces && !rotate)
        QA_TRY(plan_models(ctx, problems, n_problems, kind, P, pl, nr, prm->cluster_sweeps > 0,
                           ctx->update_order == QA_ORDER_REFERENCE, &mr));
    if (rotate) {
        rp.init_fields = 1;
        QA_TRY(run_rings_rotated(ctx, kind, pl, rp, nr, 0, steps, sqa_rot_seg(ctx, steps), &n_seg));
    } else if (!mr.empty()) {
        rp.init_fields = 1;
        QA_TRY(run_models(ctx, kind, mr, rp, 0, steps, &n_seg));
    } else {
        for (int s0 = 0; s0 < steps; s0 += seg) {
            rp.step0 = s0;
            rp.step1 = std::min(steps, s0 + seg);
            rp.init_fields = s0 == 0;
            QA_TRY(launch_rings(ctx, kind, pl, rp, nr));
        }
    }
    QA_CK(cudaEventRecord(ctx->ev[2], ctx->stream));
    QA_TRY(exact_energies(ctx, kind, d_probs, L, d_bits, d_exact));
    QA_CK(cudaEventRecord(ctx->ev[3], ctx->stream));

    // the per-step ring sums (the largest result) land in the pinned buffer
    ctx->down.resize(sizeof(double) * (size_t)nr * steps);
    const double *sums = reinterpret_cast<const double *>(ctx->down.data());
    std::vector<double> bestE(nr), exact(nr);
    std::vector<int> bstep(nr);
    std::vector<uint32_t> bits((size_t)nr * L.nw_max);
    unsigned long long cnt[5];
    QA_CK(cudaMemcpyAsync(ctx->down.data(), d_sum, sizeof(double) * (size_t)nr * steps, cudaMemcpyDeviceToHost,
                          ctx->stream));
    QA_CK(cudaMemcpyAsync(bestE.data(), d_best, sizeof(double) * nr, cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(bstep.data(), d_bstep, sizeof(int) * nr, cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(exact.data(), d_exact, sizeof(double) * nr, cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(bits.data(), d_bits, sizeof(uint32_t) * bits.size(), cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(cnt, d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, ctx->stream));
    std::vector<uint32_t> trb(n_rec * P * L.nw_max), treb(n_end * P * L.nw_max);
    std::vector<double> tre(n_rec * P), tree(n_end * P);
    std::vector<long long> rspin(tr_mag ? (size_t)nr * steps : 0);
    if (tr_rec) {
        QA_CK(cudaMemcpyAsync(trb.data(), d_trb, sizeof(uint32_t) * trb.size(), cudaMemcpyDeviceToHost, ctx->stream));
        QA_CK(cudaMemcpyAsync(tre.data(), d_tre, sizeof(double) * tre.size(), cudaMemcpyDeviceToHost, ctx->stream));
    }
    if (tr_end) {
        QA_CK(cudaMemcpyAsync(treb.data(), d_treb, sizeof(uint32_t) * treb.size(), cudaMemcpyDeviceToHost,
                              ctx->stream));
        QA_CK(cudaMemcpyAsync(tree.data(), d_tree, sizeof(double) * tree.size(), cudaMemcpyDeviceToHost, ctx->stream));
    }
    if (tr_mag)
        QA_CK(cudaMemcpyAsync(rspin.data(), d_rspin, sizeof(long long) * rspin.size(), cudaMemcpyDeviceToHost,
                              ctx->stream));
    QA_CK(cudaStreamSynchronize(ctx->stream));
    QA_TRY(check_device_error(cnt));
    for (int p = 0; traces && p < n_problems; ++p) {
        const qa_sqa_trace &t = traces[p];
        const int n = problems[p]->n;
        for (int r = 0; r < prm->reads; ++r) {
            const int base = (p * prm->reads + r) * K;  // ring of (read, replica 0)
            const size_t per_rec = (size_t)steps * rps, per_end = (size_t)steps + 1;
            for (int k = 0; k < K; ++k) {
                const size_t ring = (size_t)base + k, orow = (size_t)r * K + k;
                for (size_t e = 0; e < per_rec && (t.ring_states || t.ring_energies); ++e) {
                    const size_t src = ring * per_rec + e, dst = orow * per_rec + e;
                    for (int sl = 0; sl < P; ++sl) {
                        if (t.ring_states)
                            unpack_bits(trb.data() + (src * P + sl) * L.nw_max, n, t.ring_states + (dst * P + sl) * n);
                        if (t.ring_energies) t.ring_energies[dst * P + sl] = tre[src * P + sl];
                    }
                }
                for (size_t e = 0; e < per_end && (t.step_states || t.step_energies); ++e) {
                    const size_t src = ring * per_end + e, dst = orow * per_end + e;
                    for (int sl = 0; sl < P; ++sl) {
                        if (t.step_states)
                            unpack_bits(treb.data() + (src * P + sl) * L.nw_max, n, t.step_states + (dst * P + sl) * n);
                        if (t.step_energies) t.step_energies[dst * P + sl] = tree[src * P + sl];
                    }
                }
            }
            if (t.magnetization)
                for (int st = 0; st < steps; ++st) {
                    long long m = 0;
                    for (int k = 0; k < K; ++k) m += rspin[(size_t)(base + k) * steps + st];
                    t.magnetization[(size_t)r * steps + st] = (double)m / ((double)K * P * n);
                }
        }
    }

    // per read: trace = (sum_k sum_t E) / (K*P); best ring = min energy, then
    // earliest step, then lowest replica (the (step, replica, slice) scan
    // order of sqa_annealer.cpp:455-469)
    for (int p = 0; p < n_problems; ++p) {
        const int n = problems[p]->n;
        qa_run_out &o = outs[p];
        // a power-of-two K*P: the product with its exact reciprocal is the
        // correctly rounded quotient, without a division per entry
        const int kp = K * P;
        const bool kp_pow2 = (kp & (kp - 1)) == 0;
        const double kp_inv = 1.0 / (double)kp;
        for (int r = 0; r < prm->reads; ++r) {
            const int base = (p * prm->reads + r) * K;
            if (o.energy_trace)
                for (int s = 0; s < steps; ++s) {
                    double tot = 0.0;
                    for (int k = 0; k < K; ++k) tot += sums[(size_t)(base + k) * steps + s];
                    o.energy_trace[(size_t)r * steps + s] = kp_pow2 ? tot * kp_inv : tot / (double)kp;
                }
            int kb = 0;
            for (int k = 1; k < K; ++k) {
                const int a = base + k, b = base + kb;
                if (bestE[a] < bestE[b] || (bestE[a] == bestE[b] && bstep[a] < bstep[b])) kb = k;
            }
            const int ib = base + kb;
            if (o.best_spins) unpack_bits(bits.data() + (size_t)ib * L.nw_max, n, o.best_spins + (size_t)r * n);
            if (o.best_energy) o.best_energy[r] = exact[ib];
        }
    }
    if (stats) {
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, ctx->ev[1], ctx->ev[2]);
        cudaEventElapsedTime(&b, ctx->ev[0], ctx->ev[3]);
        stats->slice_attempts = (int64_t)cnt[0];
        stats->slice_accepts = (int64_t)cnt[1];
        stats->worldline_attempts = (int64_t)cnt[2];
        stats->worldline_accepts = (int64_t)cnt[3];
        stats->sweep_ms = a;
        stats->total_ms = b;
        stats->max_field_drift = 0.0;
        stats->sweep_launches = n_seg;
        stats->launches = (pl.own_fields() ? 2 : 3) + n_seg;
        stats->h2d_bytes = (int64_t)(sizeof(ProbDev) * n_problems + sizeof(RingDev) * nr + 2 * sizeof(float) * steps +
                                     (sizeof(double) + sizeof(int)) * nr + sizeof(int) * nr);
        stats->d2h_bytes = (int64_t)(sizeof(double) * (size_t)nr * steps + (2 * sizeof(double) + sizeof(int)) * nr +
                                     sizeof(uint32_t) * bits.size() + sizeof(cnt));
    }
    QA_TRY(check_drift(ctx, !pl.own_fields(), kind, d_probs, d_rings, nr, d_spins, d_fields, P, n_max, L.nw_max,
                       stats));
    return QA_OK;
}

int qa_sqa_run(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, const qa_sqa_params *prm,
               qa_run_out *outs, qa_stats *stats) {
    return sqa_impl(ctx, problems, n_problems, prm, outs, stats, nullptr);
}

int qa_sqa_trace_run(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, const qa_sqa_params *prm,
                     const qa_sqa_trace *traces, qa_run_out *outs, qa_stats *stats) {
    if (!traces) return fail(QA_ERR_ARG, "null traces");
    return sqa_impl(ctx, problems, n_problems, prm, outs, stats, traces);
}

// ---------------------------------------------------------------------- SQA run_optimal
namespace {

// chi_B = Var(B) over one step's bond-sum samples of a read's K rings
// (sqa_annealer.cpp:711-739); last_bond: the first ring's bond sum after the
// step (the one-sample fallback).
double opt_chi_raw(const long long *samp, int K, int ns, size_t ring_stride, long long last_bond, double nM) {
    double bs = 0.0, b2 = 0.0;
    long long total = 0;
    for (int k = 0; k < K; ++k)
        for (int j = 0; j < ns; ++j) {
            const double b = (double)samp[(size_t)k * ring_stride + j];
            bs += b;
            b2 += b * b;
            ++total;
        }
    double var;
    if (total >= 2) {
        const double bm = bs / (double)total, b2m = b2 / (double)total;
        var = b2m - bm * bm;
    } else {
        const double ba = (double)last_bond / nM;
        var = nM * (1.0 - ba * ba);
    }
    if (K == 1 && ns > 0) {
        const double ba = (double)samp[ns - 1] / nM;
        var = std::max(var, nM * (1.0 - ba * ba));
    }
    return var;
}

double opt_profile(const std::vector<double> &pj, const std::vector<double> &pc, double J) {
    const size_t M = pj.size();
    if (M == 0) return -1.0;
    if (J <= pj.front()) return pc.front();
    if (J >= pj.back()) return pc.back();
    size_t hi = 1;
    while (hi < M && pj[hi] < J) ++hi;
    const size_t lo = hi - 1;
    const double t = (J - pj[lo]) / (pj[hi] - pj[lo]);
    return pc[lo] + t * (pc[hi] - pc[lo]);
}

// The calibrated J_perp trajectory: step t of nt sits where
// G(J) = int_js^J max(chi(J'), min_chi)^alpha dJ' (trapezoids on a 4096 grid)
// reaches t/(nt-1) of G(je) (sqa_annealer.cpp:895-920,
// sqa_parallel_tempering.cpp:768-794).
std::vector<double> opt_trajectory(const std::vector<double> &pj, const std::vector<double> &pc, double js, double je,
                                   double min_chi, double alpha, int nt) {
    const int GRID = 4096;
    const double h = (je - js) / (double)GRID;
    std::vector<double> G(GRID + 1, 0.0), jt(nt);
    double prev = std::pow(std::max(opt_profile(pj, pc, js), min_chi), alpha);
    for (int k = 1; k <= GRID; ++k) {
        const double Jk = js + (double)k * h;
        const double cur = std::pow(std::max(opt_profile(pj, pc, Jk), min_chi), alpha);
        G[k] = G[k - 1] + 0.5 * (prev + cur) * h;
        prev = cur;
    }
    const double Gt = G[GRID];
    int k = 0;
    const double den = nt > 1 ? (double)(nt - 1) : 1.0;
    for (int t = 0; t < nt; ++t) {
        const double target = Gt > 0.0 ? ((double)t / den) * Gt : 0.0;
        while (k < GRID && G[k + 1] < target) ++k;
        const double g0 = G[k], g1 = G[k + 1];
        const double fr = g1 > g0 ? (target - g0) / (g1 - g0) : 0.0;
        jt[t] = js + ((double)k + fr) * h;
    }
    return jt;
}

}  // namespace

int qa_sqa_opt_run(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, const qa_sqaopt_params *prm,
                   qa_sqaopt_out *outs, qa_stats *stats) {
    QA_TRY(begin(ctx));
    if (!prm || !outs) return fail(QA_ERR_ARG, "null params");
    // sqa_annealer.cpp:513-521
    if (prm->num_steps <= 0) return fail(QA_ERR_ARG, "num_steps must be > 0.");
    if (prm->sweeps_per_step < 0 || prm->worldline_sweeps < 0 || prm->cluster_sweeps < 0)
        return fail(QA_ERR_ARG, "sweep counts must be >= 0.");
    if (prm->sweeps_per_step == 0 && prm->worldline_sweeps == 0 && prm->cluster_sweeps == 0)
        return fail(QA_ERR_ARG,
                    "At least one of sweeps_per_step, worldline_sweeps, or cluster_sweeps must be > 0.");
    if (!(prm->j_perp_end > prm->j_perp_start)) return fail(QA_ERR_ARG, "j_perp_end must be > j_perp_start.");
    if (prm->trotter_slices <= 0) return fail(QA_ERR_ARG, "trotter_slices must be > 0.");
    if (prm->replicas <= 0) return fail(QA_ERR_ARG, "replicas must be > 0.");
    if (prm->reads <= 0) return fail(QA_ERR_ARG, "reads must be > 0.");
    int kind, n_max;
    QA_TRY(check_batch(problems, n_problems, &kind, &n_max));
    const int P = prm->trotter_slices, K = prm->replicas, S = prm->num_steps;
    const int spb = prm->sweeps_per_step, wls = prm->worldline_sweeps, cls = prm->cluster_sweeps;
    if (cls > 0 && P > 64)
        return fail(QA_ERR_UNSUPPORTED, "cluster_sweeps > 0 runs with at most 64 Trotter slices on the GPU.");
    const bool calibrate = prm->eps_tilde <= 0.0;
    const int Mp = std::max(prm->calib_probes, 2), cs = std::max(prm->calib_sweeps, 1), pc = cls;
    const double beta = prm->beta, js = prm->j_perp_start, je = prm->j_perp_end, alpha = prm->alpha;
    int n1 = 0;
    if (prm->beta_ramp_fraction > 0.0) {
        n1 = (int)(prm->beta_ramp_fraction * (double)S);
        if (n1 >= S) n1 = S - 1;
    }
    const int n2 = S - n1, S_all = S + Mp, ns = spb + cls, nsc = cs + pc;
    const int reads_total = n_problems * prm->reads;

    Layout L;
    build_rings(L, problems, n_problems, prm->reads, K, P, prm->seed);
    for (auto &R : L.rings) R.sched = R.out * S_all;  // one schedule row per read
    const int nr = (int)L.rings.size();
    ProbDev *d_probs;
    RingDev *d_rings;
    uint32_t *d_spins;
    float *d_fields;
    QA_TRY(upload_common(ctx, problems, n_problems, L, &d_probs, &d_rings, &d_spins, &d_fields));
    std::vector<float> A((size_t)reads_total * S_all, 0.0f), T4(A.size(), 0.0f), JP(A.size(), 0.0f);
    auto set_col = [&](int rd, int col, double bscale, double J) {
        const size_t i = (size_t)rd * S_all + col;
        A[i] = (float)(2.0 * bscale);
        T4[i] = (float)(4.0 * J);
        JP[i] = (float)(1.0 - std::exp(-2.0 * J));
    };
    for (int rd = 0; rd < reads_total; ++rd)
        for (int s = 0; s < n1; ++s) {
            const double frac = n1 > 1 ? (double)s / (double)(n1 - 1) : 1.0;
            const double bt = prm->beta_ramp_start + (beta - prm->beta_ramp_start) * frac;
            set_col(rd, s, bt / (double)P, js);
        }
    float *d_A, *d_T4, *d_JP;
    double *d_sum, *d_best, *d_exact, *d_cbest;
    long long *d_bond, *d_bsamp, *d_cbond;
    int *d_bstep, *d_cbstep;
    uint32_t *d_bits, *d_cbits, *d_ssave;
    float *d_fsave;
    unsigned long long *d_cnt;
    const size_t samp_per_ring = (size_t)std::max({n1 * ns, Mp * nsc, ns, 1});
    QA_TRY(ws_array(ctx, W_A, A.size(), &d_A));
    QA_TRY(ws_array(ctx, W_T4, A.size(), &d_T4));
    QA_TRY(ws_array(ctx, W_JP, A.size(), &d_JP));
    QA_TRY(ws_array(ctx, W_SUM, (size_t)nr * S, &d_sum));
    QA_TRY(ws_array(ctx, W_BOND, (size_t)nr * S, &d_bond));
    QA_TRY(ws_array(ctx, W_BSAMP, (size_t)nr * samp_per_ring, &d_bsamp));
    QA_TRY(ws_array(ctx, W_CBOND, (size_t)nr * Mp, &d_cbond));
    QA_TRY(ws_array(ctx, W_BESTE, nr, &d_best));
    QA_TRY(ws_array(ctx, W_CBESTE, nr, &d_cbest));
    QA_TRY(ws_array(ctx, W_BESTSTEP, nr, &d_bstep));
    QA_TRY(ws_array(ctx, W_CBSTEP, nr, &d_cbstep));
    QA_TRY(ws_array(ctx, W_BITS, (size_t)nr * L.nw_max, &d_bits));
    QA_TRY(ws_array(ctx, W_CBITS, (size_t)nr * L.nw_max, &d_cbits));
    QA_TRY(ws_array(ctx, W_CNT, 5, &d_cnt));
    QA_TRY(ws_array(ctx, W_EXACT, nr, &d_exact));
    QA_CK(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long) * 5, ctx->stream));
    auto upload_tables = [&]() -> int {
        QA_CK(cudaMemcpyAsync(d_A, A.data(), sizeof(float) * A.size(), cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_T4, T4.data(), sizeof(float) * A.size(), cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_JP, JP.data(), sizeof(float) * A.size(), cudaMemcpyHostToDevice, ctx->stream));
        return QA_OK;
    };
    QA_TRY(upload_tables());
    {
        std::vector<double> inf(nr, INFINITY);
        std::vector<int> neg(nr, -1);
        QA_CK(cudaMemcpyAsync(d_best, inf.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_bstep, neg.data(), sizeof(int) * nr, cudaMemcpyHostToDevice, ctx->stream));
    }

    QA_CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    RingPlan pl;
    QA_TRY(plan_rings(ctx, problems, n_problems, kind, P, n_max, &pl, cls > 0, ctx->update_order == QA_ORDER_REFERENCE));
    QA_TRY(init_state(ctx, kind, d_probs, d_rings, nr, d_spins, d_fields, P, n_max, L.nw_max, DOM_INIT,
                      !pl.own_fields(), problems, n_problems, &L, d_cnt + 4));
    RingParams rp{};
    rp.probs = d_probs; rp.rings = d_rings; rp.spins = d_spins; rp.fields = d_fields;
    rp.P = P; rp.steps_total = S; rp.spb = spb; rp.wls = wls; rp.cls = cls;
    rp.slice_tag = DOM_SLICE; rp.slot = nullptr; rp.B = d_A; rp.T4 = d_T4; rp.JP = d_JP; rp.per_slot_sched = 0;
    rp.ring_sum = d_sum; rp.ring_min = nullptr; rp.ring_bond = d_bond; rp.rec_base = 0; rp.rec_stride = S;
    rp.best_E = d_best; rp.best_step = d_bstep; rp.best_bits = d_bits; rp.nw_max = L.nw_max; rp.mag = nullptr;
    rp.counters = d_cnt;
    QA_CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    bool fresh = true;  // the next launch builds its fields from the spins (own-field kernels)
    int n_launch = 0;
    const bool rotate = rotation_pays(ctx, kind, pl, nr);
    auto run_steps = [&](int s0, int s1, long long *bsamp, int bstride) -> int {
        // rotated launches of an eighth of the range where whole-grid ones
        // would leave slots idle and the range has at least 200 sweeps
        if (rotate && (long long)(s1 - s0) * (rp.spb + rp.wls + rp.cls) >= 200) {
            rp.step0 = s0;
            rp.init_fields = fresh;
            rp.bsamp = bsamp;
            rp.bstride = bstride;
            int nl = 0;
            QA_TRY(run_rings_rotated(ctx, kind, pl, rp, nr, s0, s1, rot_seg(ctx, std::max(1, (s1 - s0) / 8), s1 - s0),
                                         &nl));
            fresh = false;
            n_launch += nl;
            return QA_OK;
        }
        for (int a = s0; a < s1; a += 256) {
            rp.step0 = a;
            rp.step1 = std::min(s1, a + 256);
            rp.init_fields = fresh;
            rp.bsamp = bsamp ? bsamp + (size_t)(a - s0) * (rp.spb + rp.cls) : nullptr;
            rp.bstride = bstride;
            QA_TRY(launch_rings(ctx, kind, pl, rp, nr));
            fresh = false;
            ++n_launch;
        }
        return QA_OK;
    };
    std::vector<double> jtr((size_t)reads_total * S), chitr((size_t)reads_total * S);
    std::vector<double> eps(reads_total, prm->eps_tilde), minchi(reads_total, 1e-4 * (double)n_max * P);
    std::vector<double> Jcur(reads_total, js);
    std::vector<long long> hs, hb;
    // ---- phase 1: beta ramp at J_start (chi from the per-sweep bond sums)
    if (n1 > 0) {
        QA_TRY(run_steps(0, n1, ns > 0 ? d_bsamp : nullptr, (int)samp_per_ring));
        hs.resize((size_t)nr * samp_per_ring);
        hb.resize((size_t)nr * S);
        QA_CK(cudaMemcpyAsync(hs.data(), d_bsamp, sizeof(long long) * hs.size(), cudaMemcpyDeviceToHost, ctx->stream));
        QA_CK(cudaMemcpyAsync(hb.data(), d_bond, sizeof(long long) * hb.size(), cudaMemcpyDeviceToHost, ctx->stream));
        QA_CK(cudaStreamSynchronize(ctx->stream));
        for (int rd = 0; rd < reads_total; ++rd) {
            const int p = rd / prm->reads, base = rd * K;
            const double nM = (double)problems[p]->n * (double)P;
            for (int s = 0; s < n1; ++s) {
                const double chi = opt_chi_raw(hs.data() + (size_t)base * samp_per_ring + (size_t)s * ns, K, ns,
                                               samp_per_ring, hb[(size_t)base * S + s], nM);
                jtr[(size_t)rd * S + s] = js;
                chitr[(size_t)rd * S + s] = std::max(chi, 0.0);
            }
        }
    }
    // ---- calibration pilot: M probes from the post-ramp state, then restored
    std::vector<std::vector<double>> pj(reads_total), pcv(reads_total);
    std::vector<std::vector<double>> jtraj(reads_total);
    if (calibrate) {
        QA_TRY(ws_array(ctx, W_SSAVE, (size_t)std::max<long long>(L.spin_words, 1), &d_ssave));
        QA_TRY(ws_array(ctx, W_FSAVE, (size_t)std::max<long long>(L.field_floats, 1), &d_fsave));
        QA_CK(cudaMemcpyAsync(d_ssave, d_spins, sizeof(uint32_t) * L.spin_words, cudaMemcpyDeviceToDevice, ctx->stream));
        // field caches are valid unless an own-field kernel has not run yet (it then builds them from the spins)
        const bool fields_valid = !fresh || !pl.own_fields();
        if (fields_valid)
            QA_CK(cudaMemcpyAsync(d_fsave, d_fields, sizeof(float) * L.field_floats, cudaMemcpyDeviceToDevice,
                                  ctx->stream));
        const bool fresh_before = fresh;
        const double dJp = (je - js) / (double)Mp;
        const double bcold = beta / (double)P;
        for (int rd = 0; rd < reads_total; ++rd)
            for (int m = 0; m < Mp; ++m) set_col(rd, S + m, bcold, js + ((double)m + 0.5) * dJp);
        QA_TRY(upload_tables());
        {
            std::vector<double> inf(nr, INFINITY);
            QA_CK(cudaMemcpyAsync(d_cbest, inf.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, ctx->stream));
        }
        RingParams keep = rp;
        rp.spb = cs; rp.cls = pc; rp.wls = 0; rp.slice_tag = DOM_OPTCAL;
        rp.ring_sum = nullptr; rp.ring_bond = d_cbond; rp.rec_stride = 1; rp.rec_base = -S;
        rp.best_E = d_cbest; rp.best_step = d_cbstep; rp.best_bits = d_cbits;
        // ring_bond index = ring * rec_stride + rec_base + step: one slot per (ring, probe) via rec_base per launch
        std::vector<long long> cb((size_t)nr * Mp);
        hs.assign((size_t)nr * samp_per_ring, 0);
        for (int m = 0; m < Mp; ++m) {
            // the bond record of probe m lands at d_cbond[ring * Mp + m]
            rp.rec_stride = Mp;
            rp.rec_base = m - (S + m);
            QA_TRY(run_steps(S + m, S + m + 1, nsc > 0 ? d_bsamp + (size_t)m * nsc : nullptr, (int)samp_per_ring));
        }
        rp = keep;
        QA_CK(cudaMemcpyAsync(hs.data(), d_bsamp, sizeof(long long) * hs.size(), cudaMemcpyDeviceToHost, ctx->stream));
        QA_CK(cudaMemcpyAsync(cb.data(), d_cbond, sizeof(long long) * cb.size(), cudaMemcpyDeviceToHost, ctx->stream));
        // restore the post-ramp state (own-field kernels rebuild their exact fields from it)
        QA_CK(cudaMemcpyAsync(d_spins, d_ssave, sizeof(uint32_t) * L.spin_words, cudaMemcpyDeviceToDevice, ctx->stream));
        if (fields_valid)
            QA_CK(cudaMemcpyAsync(d_fields, d_fsave, sizeof(float) * L.field_floats, cudaMemcpyDeviceToDevice,
                                  ctx->stream));
        fresh = fresh_before || pl.own_fields();
        QA_CK(cudaStreamSynchronize(ctx->stream));
        for (int rd = 0; rd < reads_total; ++rd) {
            const int p = rd / prm->reads, base = rd * K;
            const double nM = (double)problems[p]->n * (double)P;
            pj[rd].resize(Mp);
            pcv[rd].resize(Mp);
            double integral = 0.0, maxc = 0.0;
            for (int m = 0; m < Mp; ++m) {
                double chi = opt_chi_raw(hs.data() + (size_t)base * samp_per_ring + (size_t)m * nsc, K, nsc,
                                         samp_per_ring, cb[(size_t)base * Mp + m], nM);
                if (!(chi > 0.0)) chi = 0.0;
                pj[rd][m] = js + ((double)m + 0.5) * dJp;
                pcv[rd][m] = chi;
                integral += std::pow(std::max(chi, 1e-12), alpha) * dJp;
                maxc = std::max(maxc, chi);
            }
            double e = integral / (double)n2;
            if (!(e > 0.0) || !std::isfinite(e)) {
                e = std::max(je - js, 0.0) / (double)S;
                if (!(e > 0.0)) e = 1e-9;
            }
            eps[rd] = e;
            minchi[rd] = std::max(1e-4 * maxc, 1e-12);
            jtraj[rd] = opt_trajectory(pj[rd], pcv[rd], js, je, minchi[rd], alpha, n2);
        }
    } else {
        for (int rd = 0; rd < reads_total; ++rd) minchi[rd] = 1e-4 * (double)problems[rd / prm->reads]->n * P;
    }
    // ---- phase 2 at the cold beta
    const double bcold = beta / (double)P;
    if (calibrate) {
        for (int rd = 0; rd < reads_total; ++rd)
            for (int t = 0; t < n2; ++t) {
                const double J = jtraj[rd][t];
                set_col(rd, n1 + t, bcold, J);
                const double cp = opt_profile(pj[rd], pcv[rd], J);
                jtr[(size_t)rd * S + n1 + t] = J;
                chitr[(size_t)rd * S + n1 + t] = std::max(cp, minchi[rd]);
            }
        for (int rd = 0; rd < reads_total; ++rd) Jcur[rd] = n2 > 0 ? jtraj[rd][n2 - 1] : js;
        QA_TRY(upload_tables());
        QA_TRY(run_steps(n1, S, nullptr, 0));
    } else {
        hs.assign((size_t)nr * samp_per_ring, 0);
        std::vector<long long> bnow((size_t)nr * S);
        for (int t = 0; t < n2; ++t) {
            const int s = n1 + t;
            for (int rd = 0; rd < reads_total; ++rd) set_col(rd, s, bcold, Jcur[rd]);
            QA_TRY(upload_tables());
            QA_TRY(run_steps(s, s + 1, ns > 0 ? d_bsamp : nullptr, (int)samp_per_ring));
            if (ns > 0)
                QA_CK(cudaMemcpyAsync(hs.data(), d_bsamp, sizeof(long long) * hs.size(), cudaMemcpyDeviceToHost,
                                      ctx->stream));
            QA_CK(cudaMemcpyAsync(bnow.data(), d_bond, sizeof(long long) * bnow.size(), cudaMemcpyDeviceToHost,
                                  ctx->stream));
            QA_CK(cudaStreamSynchronize(ctx->stream));
            for (int rd = 0; rd < reads_total; ++rd) {
                const int p = rd / prm->reads, base = rd * K;
                const double nM = (double)problems[p]->n * (double)P;
                const double on = opt_chi_raw(hs.data() + (size_t)base * samp_per_ring, K, ns, samp_per_ring,
                                              bnow[(size_t)base * S + s], nM);
                const double drive = std::max(on, minchi[rd]);
                jtr[(size_t)rd * S + s] = Jcur[rd];
                chitr[(size_t)rd * S + s] = drive;
                Jcur[rd] = std::min(Jcur[rd] + eps[rd] * std::pow(drive, -alpha), je);
            }
        }
    }
    QA_CK(cudaEventRecord(ctx->ev[2], ctx->stream));
    QA_TRY(exact_energies(ctx, kind, d_probs, L, d_bits, d_exact));
    QA_CK(cudaEventRecord(ctx->ev[3], ctx->stream));

    std::vector<double> sums((size_t)nr * S), bestE(nr), exact(nr);
    std::vector<int> bstep(nr);
    std::vector<uint32_t> bits((size_t)nr * L.nw_max);
    unsigned long long cnt[5];
    QA_CK(cudaMemcpyAsync(sums.data(), d_sum, sizeof(double) * sums.size(), cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(bestE.data(), d_best, sizeof(double) * nr, cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(bstep.data(), d_bstep, sizeof(int) * nr, cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(exact.data(), d_exact, sizeof(double) * nr, cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(bits.data(), d_bits, sizeof(uint32_t) * bits.size(), cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(cnt, d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaStreamSynchronize(ctx->stream));
    QA_TRY(check_device_error(cnt));
    for (int p = 0; p < n_problems; ++p) {
        const int n = problems[p]->n;
        qa_sqaopt_out &o = outs[p];
        for (int r = 0; r < prm->reads; ++r) {
            const int rd = p * prm->reads + r, base = rd * K;
            for (int s = 0; s < S; ++s) {
                double tot = 0.0;
                for (int k = 0; k < K; ++k) tot += sums[(size_t)(base + k) * S + s];
                if (o.energy_trace) o.energy_trace[(size_t)r * S + s] = tot / (double)(K * P);
                if (o.j_perp_trace) o.j_perp_trace[(size_t)r * S + s] = jtr[(size_t)rd * S + s];
                if (o.chi_B_trace) o.chi_B_trace[(size_t)r * S + s] = chitr[(size_t)rd * S + s];
            }
            int kb = 0;
            for (int k = 1; k < K; ++k) {
                const int a = base + k, b = base + kb;
                if (bestE[a] < bestE[b] || (bestE[a] == bestE[b] && bstep[a] < bstep[b])) kb = k;
            }
            const int ib = base + kb;
            if (o.best_spins) unpack_bits(bits.data() + (size_t)ib * L.nw_max, n, o.best_spins + (size_t)r * n);
            if (o.best_energy) o.best_energy[r] = exact[ib];
            if (o.scalars) {
                double *sc = o.scalars + (size_t)r * 4;
                sc[0] = eps[rd];
                sc[1] = js;
                sc[2] = je;
                sc[3] = Jcur[rd];
            }
        }
    }
    if (stats) {
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, ctx->ev[1], ctx->ev[2]);
        cudaEventElapsedTime(&b, ctx->ev[0], ctx->ev[3]);
        stats->slice_attempts = (int64_t)cnt[0];
        stats->slice_accepts = (int64_t)cnt[1];
        stats->worldline_attempts = (int64_t)cnt[2];
        stats->worldline_accepts = (int64_t)cnt[3];
        stats->sweep_ms = a;
        stats->total_ms = b;
        stats->max_field_drift = 0.0;
        stats->sweep_launches = n_launch;
        stats->launches = (pl.own_fields() ? 2 : 3) + n_launch;
        stats->h2d_bytes = 0;
        stats->d2h_bytes = (int64_t)(sizeof(double) * sums.size());
    }
    return QA_OK;
}

// ---------------------------------------------------------------------- SQA-PT
// Device records of a parallel-tempering run (rec_base 1, rec_stride steps + 1).
struct PTDev {
    double *best, *exact, *min, *avg, *swp;
    int *bstep, *bslot, *rin;
    uint32_t *bits, *fbits;
    unsigned long long *cnt;
};

// Downloads of a parallel-tempering run and the per-read outputs: the best
// state of a read is the lowest energy, then the earliest step (the starting
// state is step -1), then the lowest slot -- the (step, slot) scan order of
// sqa_parallel_tempering.cpp:177-185, 299-306; final states per slot; the
// average-energy and swap traces.  Fills the counters and times of stats.
static int pt_collect(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, int reads, int Rn, int steps,
                      const Layout &L, const PTDev &d, qa_sqapt_out *const *outs, qa_stats *stats, int64_t *d2h) {
    const int nr = (int)L.rings.size(), reads_total = n_problems * reads;
    std::vector<double> bestE(nr), exact(nr), lastmin(nr), avg((size_t)reads_total * steps),
        swp((size_t)reads_total * steps);
    std::vector<int> bstep(nr), bslot(nr), rin((size_t)reads_total * Rn);
    std::vector<uint32_t> bits((size_t)nr * L.nw_max), fbits((size_t)nr * L.nw_max);
    unsigned long long cnt[5];
    QA_CK(cudaMemcpyAsync(bestE.data(), d.best, sizeof(double) * nr, cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(exact.data(), d.exact, sizeof(double) * nr, cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpy2DAsync(lastmin.data(), sizeof(double), d.min + steps, sizeof(double) * (steps + 1),
                            sizeof(double), nr, cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(avg.data(), d.avg, sizeof(double) * avg.size(), cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(swp.data(), d.swp, sizeof(double) * swp.size(), cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(bstep.data(), d.bstep, sizeof(int) * nr, cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(bslot.data(), d.bslot, sizeof(int) * nr, cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(rin.data(), d.rin, sizeof(int) * rin.size(), cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(bits.data(), d.bits, sizeof(uint32_t) * bits.size(), cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(fbits.data(), d.fbits, sizeof(uint32_t) * fbits.size(), cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(cnt, d.cnt, sizeof(cnt), cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaStreamSynchronize(ctx->stream));
    QA_TRY(check_device_error(cnt));
    for (int p = 0; p < n_problems; ++p) {
        const int n = problems[p]->n;
        qa_sqapt_out &o = *outs[p];
        for (int r = 0; r < reads; ++r) {
            const int q = p * reads + r, base = q * Rn;
            int kb = 0;
            for (int k = 1; k < Rn; ++k) {
                const int a = base + k, b = base + kb;
                if (bestE[a] < bestE[b] || (bestE[a] == bestE[b] && (bstep[a] < bstep[b] ||
                                                                     (bstep[a] == bstep[b] && bslot[a] < bslot[b]))))
                    kb = k;
            }
            if (o.best_spins) unpack_bits(bits.data() + (size_t)(base + kb) * L.nw_max, n, o.best_spins + (size_t)r * n);
            if (o.best_energy) o.best_energy[r] = exact[base + kb];
            for (int s = 0; s < Rn; ++s) {
                const int k = rin[(size_t)q * Rn + s];
                if (o.final_energies) o.final_energies[(size_t)r * Rn + s] = lastmin[base + k];
                if (o.final_spins)
                    unpack_bits(fbits.data() + (size_t)(base + k) * L.nw_max, n,
                                o.final_spins + ((size_t)r * Rn + s) * n);
            }
            if (o.average_energy_trace)
                std::memcpy(o.average_energy_trace + (size_t)r * steps, avg.data() + (size_t)q * steps,
                            sizeof(double) * steps);
            if (o.swap_acceptance_trace)
                std::memcpy(o.swap_acceptance_trace + (size_t)r * steps, swp.data() + (size_t)q * steps,
                            sizeof(double) * steps);
        }
    }
    if (stats) {
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, ctx->ev[1], ctx->ev[2]);
        cudaEventElapsedTime(&b, ctx->ev[0], ctx->ev[3]);
        stats->slice_attempts = (int64_t)cnt[0];
        stats->slice_accepts = (int64_t)cnt[1];
        stats->worldline_attempts = (int64_t)cnt[2];
        stats->worldline_accepts = (int64_t)cnt[3];
        stats->sweep_ms = a;
        stats->total_ms = b;
        stats->max_field_drift = 0.0;
    }
    *d2h = (int64_t)(sizeof(double) * (3 * (size_t)nr + avg.size() + swp.size()) + 3 * sizeof(int) * (size_t)nr +
                     sizeof(int) * rin.size() + sizeof(uint32_t) * 2 * bits.size() + sizeof(cnt));
    return QA_OK;
}

// SQA-PT (qa_sqapt_run) and, with `classical`, the classical parallel
// tempering of qa_pt_run: one slice, B = 2 beta, no Trotter term (T4 = 0,
// J_perp = 0 in the swap action).
static int sqapt_impl(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, const qa_sqapt_params *prm,
                      qa_sqapt_out *outs, qa_stats *stats, bool classical) {
    QA_TRY(begin(ctx));
    if (!prm) return fail(QA_ERR_ARG, "null params");
    if (prm->rungs < 2 || !prm->betas || !prm->gammas)
        return fail(QA_ERR_ARG, "SQA parallel tempering requires >=2 beta/gamma pairs.");
    if (prm->trotter_slices <= 0) return fail(QA_ERR_ARG, "trotter_slices must be > 0.");
    if (prm->steps <= 0) return fail(QA_ERR_ARG, "steps must be > 0.");
    if (prm->swap_interval <= 0) return fail(QA_ERR_ARG, "swap_interval must be > 0.");
    if (prm->sweeps_per_step < 0 || prm->worldline_sweeps < 0 || prm->cluster_sweeps < 0)
        return fail(QA_ERR_ARG, "sweep counts must be >= 0.");
    if (prm->sweeps_per_step == 0 && prm->worldline_sweeps == 0 && prm->cluster_sweeps == 0)
        return fail(QA_ERR_ARG, "At least one of sweeps_per_step/worldline_sweeps/cluster_sweeps must be > 0.");
    if (prm->reads <= 0) return fail(QA_ERR_ARG, "reads must be > 0.");
    int kind, n_max;
    QA_TRY(check_batch(problems, n_problems, &kind, &n_max));
    const int P = (prm->continuous_time_slices > 0 && prm->continuous_time_slices > prm->trotter_slices)
                      ? prm->continuous_time_slices
                      : prm->trotter_slices;
    if (prm->cluster_sweeps > 0 && P > 64)
        return fail(QA_ERR_UNSUPPORTED, "cluster_sweeps > 0 runs with at most 64 Trotter slices on the GPU.");
    const int Rn = prm->rungs, steps = prm->steps, reads_total = n_problems * prm->reads;
    Layout L;
    build_rings(L, problems, n_problems, prm->reads, Rn, P, prm->seed);
    const int nr = (int)L.rings.size();
    ProbDev *d_probs;
    RingDev *d_rings;
    uint32_t *d_spins;
    float *d_fields;
    QA_TRY(upload_common(ctx, problems, n_problems, L, &d_probs, &d_rings, &d_spins, &d_fields));
    std::vector<float> B(Rn), T4(Rn), JP(Rn);
    std::vector<double> bpjp(2 * Rn);
    for (int r = 0; r < Rn; ++r) {
        B[r] = (float)(2.0 * (prm->betas[r] / (double)P));
        T4[r] = (float)(4.0 * trotter_coupling(prm->betas[r], prm->gammas[r], P));
        bpjp[r] = prm->betas[r] / (double)P;
        bpjp[Rn + r] = trotter_coupling(prm->betas[r], prm->gammas[r], P);
        JP[r] = (float)(1.0 - std::exp(-2.0 * bpjp[Rn + r]));  // sqa_parallel_tempering.cpp:201
        if (classical) {
            T4[r] = 0.0f;
            bpjp[Rn + r] = 0.0;
        }
    }
    float *d_B, *d_T4;
    double *d_bpjp, *d_sum, *d_min, *d_best, *d_exact, *d_avg, *d_swp;
    long long *d_bond;
    int *d_bstep, *d_bslot, *d_slot, *d_rin;
    uint32_t *d_bits, *d_fbits;
    unsigned long long *d_cnt;
    const size_t rec = (size_t)nr * (steps + 1);
    QA_TRY(ws_array(ctx, W_A, Rn, &d_B));
    QA_TRY(ws_array(ctx, W_T4, Rn, &d_T4));
    float *d_JP;
    QA_TRY(ws_array(ctx, W_JP, Rn, &d_JP));
    QA_TRY(ws_array(ctx, W_BPJP, 2 * Rn, &d_bpjp));
    QA_TRY(ws_array(ctx, W_SUM, rec, &d_sum));
    QA_TRY(ws_array(ctx, W_MIN, rec, &d_min));
    QA_TRY(ws_array(ctx, W_BOND, rec, &d_bond));
    QA_TRY(ws_array(ctx, W_BESTE, nr, &d_best));
    QA_TRY(ws_array(ctx, W_BESTSTEP, nr, &d_bstep));
    QA_TRY(ws_array(ctx, W_BSLOT, nr, &d_bslot));
    QA_TRY(ws_array(ctx, W_SLOT, nr, &d_slot));
    QA_TRY(ws_array(ctx, W_RIN, (size_t)reads_total * Rn, &d_rin));
    QA_TRY(ws_array(ctx, W_BITS, (size_t)nr * L.nw_max, &d_bits));
    QA_TRY(ws_array(ctx, W_FBITS, (size_t)nr * L.nw_max, &d_fbits));
    QA_TRY(ws_array(ctx, W_EXACT, nr, &d_exact));
    QA_TRY(ws_array(ctx, W_AVG, (size_t)reads_total * steps, &d_avg));
    QA_TRY(ws_array(ctx, W_SWP, (size_t)reads_total * steps, &d_swp));
    QA_TRY(ws_array(ctx, W_CNT, 5, &d_cnt));
    {
        std::vector<double> inf(nr, INFINITY);
        std::vector<int> neg(nr, -2), slot(nr), rin((size_t)reads_total * Rn);
        for (int i = 0; i < nr; ++i) slot[i] = L.rings[i].k;
        for (size_t i = 0; i < rin.size(); ++i) rin[i] = (int)(i % Rn);
        QA_CK(cudaMemcpyAsync(d_B, B.data(), sizeof(float) * Rn, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_T4, T4.data(), sizeof(float) * Rn, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_JP, JP.data(), sizeof(float) * Rn, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_bpjp, bpjp.data(), sizeof(double) * 2 * Rn, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_best, inf.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_bstep, neg.data(), sizeof(int) * nr, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_bslot, slot.data(), sizeof(int) * nr, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_slot, slot.data(), sizeof(int) * nr, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_rin, rin.data(), sizeof(int) * rin.size(), cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long) * 5, ctx->stream));
        QA_CK(cudaStreamSynchronize(ctx->stream));
    }
    RingPlan pl;
    // classical parallel tempering keeps its ascending order (parallel_tempering.cpp:36-122)
    QA_TRY(plan_rings(ctx, problems, n_problems, kind, P, n_max, &pl, prm->cluster_sweeps > 0,
                      !classical && ctx->update_order == QA_ORDER_REFERENCE));
    QA_CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    QA_TRY(init_state(ctx, kind, d_probs, d_rings, nr, d_spins, d_fields, P, n_max, L.nw_max, DOM_INIT, !pl.own_fields(),
                      problems, n_problems, &L, d_cnt + 4));
    RingParams rp{};
    rp.probs = d_probs; rp.rings = d_rings; rp.spins = d_spins; rp.fields = d_fields;
    rp.P = P; rp.steps_total = steps; rp.spb = prm->sweeps_per_step; rp.wls = prm->worldline_sweeps;
    rp.slice_tag = DOM_SLICE; rp.slot = d_slot; rp.B = d_B; rp.T4 = d_T4; rp.per_slot_sched = 1;
    rp.cls = prm->cluster_sweeps; rp.JP = d_JP;
    rp.ring_sum = d_sum; rp.ring_min = d_min; rp.ring_bond = d_bond; rp.rec_base = 1; rp.rec_stride = steps + 1;
    rp.best_E = d_best; rp.best_step = d_bstep; rp.best_slot = d_bslot; rp.best_bits = d_bits;
    rp.final_bits = d_fbits; rp.nw_max = L.nw_max; rp.counters = d_cnt;
    PTSegParams sp{};
    sp.rings = d_rings; sp.reads = reads_total; sp.R = Rn; sp.bp = d_bpjp; sp.jp = d_bpjp + Rn;
    sp.ring_sum = d_sum; sp.ring_min = d_min; sp.ring_bond = d_bond; sp.rec_base = 1; sp.rec_stride = steps + 1;
    sp.ring_in = d_rin; sp.slot_of = d_slot; sp.avg_trace = d_avg; sp.swap_trace = d_swp; sp.steps_total = steps;
    QA_CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    int n_seg = 0, n_launch = 0;
    const bool rotate = rotation_pays(ctx, kind, pl, nr);
    std::vector<ModelRun> mr;  // an instance set of uneven size: per-model launches
    if (!rotate)
        QA_TRY(plan_models(ctx, problems, n_problems, kind, P, pl, nr, prm->cluster_sweeps > 0,
                           !classical && ctx->update_order == QA_ORDER_REFERENCE, &mr));
    for (int s0 = 0; s0 < steps;) {
        const int s1 = std::min({steps, (s0 / prm->swap_interval + 1) * prm->swap_interval, s0 + 256});
        rp.step0 = s0;
        rp.step1 = s1;
        rp.init_scan = s0 == 0;
        rp.init_fields = s0 == 0;
        // at least 8 sweeps in the segment and rings worth rotating: launches
        // of an eighth of it (at least one step), joined before the swaps
        if ((long long)(s1 - s0) * (rp.spb + rp.wls + rp.cls) >= 8 && rotate) {
            int nl = 0;
            QA_TRY(run_rings_rotated(ctx, kind, pl, rp, nr, s0, s1, rot_seg(ctx, std::max(1, (s1 - s0) / 8), s1 - s0),
                                         &nl));
            n_launch += nl;
        } else if (!mr.empty()) {
            int nl = 0;
            QA_TRY(run_models(ctx, kind, mr, rp, s0, s1, &nl));
            n_launch += nl;
        } else {
            QA_TRY(launch_rings(ctx, kind, pl, rp, nr));
            ++n_launch;
        }
        sp.s0 = s0;
        sp.s1 = s1;
        sp.swap = s1 % prm->swap_interval == 0;
        sp.round = (uint32_t)(s1 / prm->swap_interval - 1);
        pt_segment_kernel<<<(reads_total + 127) / 128, 128, 0, ctx->stream>>>(sp);
        QA_CK(cudaGetLastError());
        ++n_seg;
        s0 = s1;
    }
    QA_CK(cudaEventRecord(ctx->ev[2], ctx->stream));
    QA_TRY(exact_energies(ctx, kind, d_probs, L, d_bits, d_exact));
    QA_CK(cudaEventRecord(ctx->ev[3], ctx->stream));
    std::vector<qa_sqapt_out *> po(n_problems);
    for (int p = 0; p < n_problems; ++p) po[p] = outs + p;
    const PTDev dv{d_best, d_exact, d_min, d_avg, d_swp, d_bstep, d_bslot, d_rin, d_bits, d_fbits, d_cnt};
    int64_t d2h = 0;
    QA_TRY(pt_collect(ctx, problems, n_problems, prm->reads, Rn, steps, L, dv, po.data(), stats, &d2h));
    if (stats) {
        stats->sweep_launches = n_launch;
        stats->launches = (pl.own_fields() ? 2 : 3) + n_launch + n_seg;
        stats->h2d_bytes = (int64_t)(sizeof(ProbDev) * n_problems + sizeof(RingDev) * nr + 2 * sizeof(float) * Rn +
                                     2 * sizeof(double) * Rn + (sizeof(double) + 3 * sizeof(int)) * nr +
                                     sizeof(int) * (size_t)reads_total * Rn);
        stats->d2h_bytes = d2h;
    }
    QA_TRY(check_drift(ctx, !pl.own_fields(), kind, d_probs, d_rings, nr, d_spins, d_fields, P, n_max, L.nw_max,
                       stats));
    return QA_OK;
}

// ---------------------------------------------------------------------- SQA-PT run_optimal
// SQAParallelTemperingAnnealer::run_optimal (sqa_parallel_tempering.cpp:348-882).
// Schedule tables are [read][step][slot]: rung slot r keeps B = 2 beta_r / P,
// every slot of a step shares T4 = 4 J and JP = 1 - e^{-2J}.  Calibration
// probes run as steps num_steps + m (slice tag OPTCAL) from the starting
// states, which are restored afterwards; the calibrated production runs in
// swap segments like qa_sqapt_run, the online one (eps_tilde > 0) a step per
// launch with chi_B reduced on the host.  Swaps use the rung action with
// J_perp = 0: the shared Trotter terms cancel (sqa_parallel_tempering.cpp:846-861).
int qa_sqapt_opt_run(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, const qa_sqaptopt_params *prm,
                     qa_sqaptopt_out *outs, qa_stats *stats) {
    QA_TRY(begin(ctx));
    if (!prm || !outs) return fail(QA_ERR_ARG, "null params");
    // sqa_parallel_tempering.cpp:361-366
    if (prm->num_steps <= 0) return fail(QA_ERR_ARG, "num_steps must be > 0.");
    if (prm->swap_interval <= 0) return fail(QA_ERR_ARG, "swap_interval must be > 0.");
    if (prm->sweeps_per_step < 0 || prm->worldline_sweeps < 0 || prm->cluster_sweeps < 0)
        return fail(QA_ERR_ARG, "sweep counts must be >= 0.");
    if (prm->sweeps_per_step == 0 && prm->worldline_sweeps == 0 && prm->cluster_sweeps == 0)
        return fail(QA_ERR_ARG, "At least one of sweeps_per_step/worldline_sweeps/cluster_sweeps must be > 0.");
    if (prm->rungs < 2 || !prm->betas || !prm->gammas)
        return fail(QA_ERR_ARG, "SQA parallel tempering requires >=2 beta/gamma pairs.");
    if (prm->trotter_slices <= 0) return fail(QA_ERR_ARG, "trotter_slices must be > 0.");
    if (prm->reads <= 0) return fail(QA_ERR_ARG, "reads must be > 0.");
    int kind, n_max;
    QA_TRY(check_batch(problems, n_problems, &kind, &n_max));
    const int P = (prm->continuous_time_slices > 0 && prm->continuous_time_slices > prm->trotter_slices)
                      ? prm->continuous_time_slices
                      : prm->trotter_slices;
    const int Rn = prm->rungs, S = prm->num_steps, spb = prm->sweeps_per_step, wls = prm->worldline_sweeps,
              cls = prm->cluster_sweeps;
    if (cls > 0 && P > 64)
        return fail(QA_ERR_UNSUPPORTED, "cluster_sweeps > 0 runs with at most 64 Trotter slices on the GPU.");
    const bool calibrate = prm->eps_tilde <= 0.0;
    const int Mp = std::max(prm->calib_probes, 2), cs = std::max(prm->calib_sweeps, 1), pc = cls;
    const int ns = spb + cls, nsc = cs + pc, S_all = S + Mp, reads_total = n_problems * prm->reads;
    const double alpha = prm->alpha;
    // J_start: the hottest rung's coupling; J_end <= 0: the coldest rung's (sqa_parallel_tempering.cpp:377-398)
    const double js = trotter_coupling(prm->betas[0], prm->gammas[0], P);
    double je = prm->j_perp_end;
    if (je <= 0.0) {
        je = trotter_coupling(prm->betas[Rn - 1], prm->gammas[Rn - 1], P);
        std::fprintf(stderr,
                     "[qanneal run_optimal] WARNING: j_perp_end not specified; defaulted to coldest-replica "
                     "trotter_coupling = %g (j_perp_start = %g). For benchmark runs pass an explicit j_perp_end "
                     "(e.g. 5*j_rms).\n", je, js);
    }
    if (je <= js) {
        std::fprintf(stderr,
                     "[qanneal run_optimal] WARNING: resolved j_perp_end (%g) <= j_perp_start (%g). The adaptive "
                     "schedule has no range to traverse and will not anneal. Installing finite ceiling "
                     "j_perp_start + 1e6 so the run terminates by num_steps.\n", je, js);
        je = js + 1e6;
    }

    Layout L;
    build_rings(L, problems, n_problems, prm->reads, Rn, P, prm->seed);
    for (auto &R : L.rings) R.sched = R.out * S_all * Rn;  // [read][step][slot]
    const int nr = (int)L.rings.size();
    ProbDev *d_probs;
    RingDev *d_rings;
    uint32_t *d_spins;
    float *d_fields;
    QA_TRY(upload_common(ctx, problems, n_problems, L, &d_probs, &d_rings, &d_spins, &d_fields));
    const size_t tab = (size_t)reads_total * S_all * Rn;
    std::vector<float> Bt(tab), T4t(tab), JPt(tab);
    auto set_step = [&](int rd, int step, double J) {
        const float t4 = (float)(4.0 * J), jp = (float)(1.0 - std::exp(-2.0 * J));
        for (int r = 0; r < Rn; ++r) {
            const size_t i = ((size_t)rd * S_all + step) * Rn + r;
            Bt[i] = (float)(2.0 * (prm->betas[r] / (double)P));
            T4t[i] = t4;
            JPt[i] = jp;
        }
    };
    std::vector<double> bpjp(2 * Rn, 0.0);
    for (int r = 0; r < Rn; ++r) bpjp[r] = prm->betas[r] / (double)P;
    float *d_B, *d_T4, *d_JP;
    double *d_bpjp, *d_sum, *d_min, *d_best, *d_cbest, *d_exact, *d_avg, *d_swp;
    long long *d_bond, *d_bsamp;
    int *d_bstep, *d_cbstep, *d_bslot, *d_slot, *d_rin;
    uint32_t *d_bits, *d_cbits, *d_fbits, *d_ssave;
    float *d_fsave;
    unsigned long long *d_cnt;
    const size_t rec = (size_t)nr * (S + 1);
    const size_t samp_per_ring = (size_t)std::max({calibrate ? Mp * nsc : 0, ns, 1});
    QA_TRY(ws_array(ctx, W_A, tab, &d_B));
    QA_TRY(ws_array(ctx, W_T4, tab, &d_T4));
    QA_TRY(ws_array(ctx, W_JP, tab, &d_JP));
    QA_TRY(ws_array(ctx, W_BPJP, 2 * Rn, &d_bpjp));
    QA_TRY(ws_array(ctx, W_SUM, rec, &d_sum));
    QA_TRY(ws_array(ctx, W_MIN, rec, &d_min));
    QA_TRY(ws_array(ctx, W_BOND, rec, &d_bond));
    QA_TRY(ws_array(ctx, W_BSAMP, (size_t)nr * samp_per_ring, &d_bsamp));
    QA_TRY(ws_array(ctx, W_BESTE, nr, &d_best));
    QA_TRY(ws_array(ctx, W_CBESTE, nr, &d_cbest));
    QA_TRY(ws_array(ctx, W_BESTSTEP, nr, &d_bstep));
    QA_TRY(ws_array(ctx, W_CBSTEP, nr, &d_cbstep));
    QA_TRY(ws_array(ctx, W_BSLOT, nr, &d_bslot));
    QA_TRY(ws_array(ctx, W_SLOT, nr, &d_slot));
    QA_TRY(ws_array(ctx, W_RIN, (size_t)reads_total * Rn, &d_rin));
    QA_TRY(ws_array(ctx, W_BITS, (size_t)nr * L.nw_max, &d_bits));
    QA_TRY(ws_array(ctx, W_CBITS, (size_t)nr * L.nw_max, &d_cbits));
    QA_TRY(ws_array(ctx, W_FBITS, (size_t)nr * L.nw_max, &d_fbits));
    QA_TRY(ws_array(ctx, W_EXACT, nr, &d_exact));
    QA_TRY(ws_array(ctx, W_AVG, (size_t)reads_total * S, &d_avg));
    QA_TRY(ws_array(ctx, W_SWP, (size_t)reads_total * S, &d_swp));
    QA_TRY(ws_array(ctx, W_CNT, 5, &d_cnt));
    auto upload_tables = [&]() -> int {
        QA_CK(cudaMemcpyAsync(d_B, Bt.data(), sizeof(float) * tab, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_T4, T4t.data(), sizeof(float) * tab, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_JP, JPt.data(), sizeof(float) * tab, cudaMemcpyHostToDevice, ctx->stream));
        return QA_OK;
    };
    // the rows of one step, [read] x [slot] at a pitch of S_all * Rn entries
    auto upload_step = [&](int step) -> int {
        const size_t pitch = sizeof(float) * S_all * Rn, off = (size_t)step * Rn, w = sizeof(float) * Rn;
        QA_CK(cudaMemcpy2DAsync(d_B + off, pitch, Bt.data() + off, pitch, w, reads_total, cudaMemcpyHostToDevice,
                                ctx->stream));
        QA_CK(cudaMemcpy2DAsync(d_T4 + off, pitch, T4t.data() + off, pitch, w, reads_total, cudaMemcpyHostToDevice,
                                ctx->stream));
        QA_CK(cudaMemcpy2DAsync(d_JP + off, pitch, JPt.data() + off, pitch, w, reads_total, cudaMemcpyHostToDevice,
                                ctx->stream));
        return QA_OK;
    };
    {
        std::vector<double> inf(nr, INFINITY);
        std::vector<int> neg(nr, -2), slot(nr), rin((size_t)reads_total * Rn);
        for (int i = 0; i < nr; ++i) slot[i] = L.rings[i].k;
        for (size_t i = 0; i < rin.size(); ++i) rin[i] = (int)(i % Rn);
        QA_CK(cudaMemcpyAsync(d_bpjp, bpjp.data(), sizeof(double) * 2 * Rn, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_best, inf.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_cbest, inf.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_bstep, neg.data(), sizeof(int) * nr, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_cbstep, neg.data(), sizeof(int) * nr, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_bslot, slot.data(), sizeof(int) * nr, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_slot, slot.data(), sizeof(int) * nr, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_rin, rin.data(), sizeof(int) * rin.size(), cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long) * 5, ctx->stream));
        QA_CK(cudaStreamSynchronize(ctx->stream));
    }
    RingPlan pl;
    QA_TRY(plan_rings(ctx, problems, n_problems, kind, P, n_max, &pl, cls > 0, ctx->update_order == QA_ORDER_REFERENCE));
    QA_CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    QA_TRY(init_state(ctx, kind, d_probs, d_rings, nr, d_spins, d_fields, P, n_max, L.nw_max, DOM_INIT,
                      !pl.own_fields(), problems, n_problems, &L, d_cnt + 4));
    RingParams rp{};
    rp.probs = d_probs; rp.rings = d_rings; rp.spins = d_spins; rp.fields = d_fields;
    rp.P = P; rp.steps_total = S; rp.spb = spb; rp.wls = wls; rp.cls = cls;
    rp.slice_tag = DOM_SLICE; rp.slot = d_slot; rp.B = d_B; rp.T4 = d_T4; rp.JP = d_JP;
    rp.per_slot_sched = 1; rp.slot_step = Rn;
    rp.ring_sum = d_sum; rp.ring_min = d_min; rp.ring_bond = d_bond; rp.rec_base = 1; rp.rec_stride = S + 1;
    rp.best_E = d_best; rp.best_step = d_bstep; rp.best_slot = d_bslot; rp.best_bits = d_bits;
    rp.final_bits = d_fbits; rp.nw_max = L.nw_max; rp.counters = d_cnt;
    PTSegParams sp{};
    sp.rings = d_rings; sp.reads = reads_total; sp.R = Rn; sp.bp = d_bpjp; sp.jp = d_bpjp + Rn;
    sp.ring_sum = d_sum; sp.ring_min = d_min; sp.ring_bond = d_bond; sp.rec_base = 1; sp.rec_stride = S + 1;
    sp.ring_in = d_rin; sp.slot_of = d_slot; sp.avg_trace = d_avg; sp.swap_trace = d_swp; sp.steps_total = S;
    QA_CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    bool fresh = true;  // the next launch builds its fields from the spins (own-field kernels)
    int n_launch = 0, n_seg = 0;
    std::vector<double> jtr((size_t)reads_total * S), chitr((size_t)reads_total * S), eps(reads_total, prm->eps_tilde),
        minchi(reads_total), Jcur(reads_total, js);
    std::vector<std::vector<double>> pj(reads_total), pcv(reads_total), jtraj(reads_total);
    for (int rd = 0; rd < reads_total; ++rd) minchi[rd] = 1e-4 * (double)problems[rd / prm->reads]->n * P;
    // ---- calibration probes from the starting states, which are then restored
    if (calibrate) {
        QA_TRY(ws_array(ctx, W_SSAVE, (size_t)std::max<long long>(L.spin_words, 1), &d_ssave));
        QA_TRY(ws_array(ctx, W_FSAVE, (size_t)std::max<long long>(L.field_floats, 1), &d_fsave));
        QA_CK(cudaMemcpyAsync(d_ssave, d_spins, sizeof(uint32_t) * L.spin_words, cudaMemcpyDeviceToDevice, ctx->stream));
        const bool fields_valid = !pl.own_fields();  // own-field kernels build theirs on their first launch
        if (fields_valid)
            QA_CK(cudaMemcpyAsync(d_fsave, d_fields, sizeof(float) * L.field_floats, cudaMemcpyDeviceToDevice,
                                  ctx->stream));
        const double dJp = (je - js) / (double)Mp;
        for (int rd = 0; rd < reads_total; ++rd)
            for (int m = 0; m < Mp; ++m) set_step(rd, S + m, js + ((double)m + 0.5) * dJp);
        QA_TRY(upload_tables());
        RingParams keep = rp;
        rp.spb = cs; rp.cls = pc; rp.wls = 0; rp.slice_tag = DOM_OPTCAL; rp.init_scan = 0;
        rp.ring_sum = nullptr; rp.ring_min = nullptr; rp.ring_bond = nullptr;
        rp.best_E = d_cbest; rp.best_step = d_cbstep; rp.best_slot = nullptr; rp.best_bits = d_cbits;
        rp.final_bits = nullptr; rp.bstride = (int)samp_per_ring;
        for (int m = 0; m < Mp; ++m) {
            rp.step0 = S + m;
            rp.step1 = S + m + 1;
            rp.init_fields = fresh;
            rp.bsamp = d_bsamp + (size_t)m * nsc;
            QA_TRY(launch_rings(ctx, kind, pl, rp, nr));
            fresh = false;
            ++n_launch;
        }
        rp = keep;
        std::vector<long long> hs((size_t)nr * samp_per_ring);
        QA_CK(cudaMemcpyAsync(hs.data(), d_bsamp, sizeof(long long) * hs.size(), cudaMemcpyDeviceToHost, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_spins, d_ssave, sizeof(uint32_t) * L.spin_words, cudaMemcpyDeviceToDevice, ctx->stream));
        if (fields_valid)
            QA_CK(cudaMemcpyAsync(d_fields, d_fsave, sizeof(float) * L.field_floats, cudaMemcpyDeviceToDevice,
                                  ctx->stream));
        fresh = true;
        QA_CK(cudaStreamSynchronize(ctx->stream));
        for (int rd = 0; rd < reads_total; ++rd) {
            const double nM = (double)problems[rd / prm->reads]->n * (double)P;
            pj[rd].resize(Mp);
            pcv[rd].resize(Mp);
            double integral = 0.0, maxc = 0.0;
            for (int m = 0; m < Mp; ++m) {
                // Rn >= 2 rings and nsc >= 1 samples each: the one-sample fallback never applies
                double chi = opt_chi_raw(hs.data() + (size_t)rd * Rn * samp_per_ring + (size_t)m * nsc, Rn, nsc,
                                         samp_per_ring, 0, nM);
                if (!(chi > 0.0)) chi = 0.0;
                pj[rd][m] = js + ((double)m + 0.5) * dJp;
                pcv[rd][m] = chi;
                integral += std::pow(std::max(chi, 1e-12), alpha) * dJp;
                maxc = std::max(maxc, chi);
            }
            double e = integral / (double)S;
            if (!(e > 0.0) || !std::isfinite(e)) {
                e = std::max(je - js, 0.0) / (double)S;
                if (!(e > 0.0)) e = 1e-9;
            }
            eps[rd] = e;
            minchi[rd] = std::max(1e-4 * maxc, 1e-12);
            jtraj[rd] = opt_trajectory(pj[rd], pcv[rd], js, je, minchi[rd], alpha, S);
        }
    }
    // ---- production
    if (calibrate) {
        for (int rd = 0; rd < reads_total; ++rd) {
            for (int s = 0; s < S; ++s) {
                const double J = jtraj[rd][s];
                set_step(rd, s, J);
                jtr[(size_t)rd * S + s] = J;
                chitr[(size_t)rd * S + s] = std::max(opt_profile(pj[rd], pcv[rd], J), minchi[rd]);
            }
            Jcur[rd] = jtraj[rd][S - 1];
        }
        QA_TRY(upload_tables());
        const bool rotate = rotation_pays(ctx, kind, pl, nr);
        for (int s0 = 0; s0 < S;) {
            const int s1 = std::min({S, (s0 / prm->swap_interval + 1) * prm->swap_interval, s0 + 256});
            rp.step0 = s0;
            rp.step1 = s1;
            rp.init_scan = s0 == 0;
            rp.init_fields = fresh;
            // as in SQA-PT runs: rotated launches of an eighth of a segment with
            // at least 8 sweeps, joined before the swaps
            if (rotate && (long long)(s1 - s0) * (rp.spb + rp.wls + rp.cls) >= 8) {
                int nl = 0;
                QA_TRY(run_rings_rotated(ctx, kind, pl, rp, nr, s0, s1, rot_seg(ctx, std::max(1, (s1 - s0) / 8), s1 - s0),
                                         &nl));
                n_launch += nl;
            } else {
                QA_TRY(launch_rings(ctx, kind, pl, rp, nr));
                ++n_launch;
            }
            fresh = false;
            sp.s0 = s0;
            sp.s1 = s1;
            sp.swap = s1 % prm->swap_interval == 0;
            sp.round = (uint32_t)(s1 / prm->swap_interval - 1);
            pt_segment_kernel<<<(reads_total + 127) / 128, 128, 0, ctx->stream>>>(sp);
            QA_CK(cudaGetLastError());
            ++n_seg;
            s0 = s1;
        }
    } else {
        std::vector<long long> hs((size_t)nr * std::max(ns, 1)), hb(nr);
        std::vector<int> rin_prev((size_t)reads_total * Rn);
        for (size_t i = 0; i < rin_prev.size(); ++i) rin_prev[i] = (int)(i % Rn);
        rp.bstride = (int)samp_per_ring;
        for (int s = 0; s < S; ++s) {
            for (int rd = 0; rd < reads_total; ++rd) set_step(rd, s, Jcur[rd]);
            QA_TRY(upload_step(s));
            rp.step0 = s;
            rp.step1 = s + 1;
            rp.init_scan = s == 0;
            rp.init_fields = fresh;
            rp.bsamp = ns > 0 ? d_bsamp : nullptr;
            QA_TRY(launch_rings(ctx, kind, pl, rp, nr));
            fresh = false;
            ++n_launch;
            if (ns > 0)
                QA_CK(cudaMemcpy2DAsync(hs.data(), sizeof(long long) * ns, d_bsamp, sizeof(long long) * samp_per_ring,
                                        sizeof(long long) * ns, nr, cudaMemcpyDeviceToHost, ctx->stream));
            else
                QA_CK(cudaMemcpy2DAsync(hb.data(), sizeof(long long), d_bond + 1 + s, sizeof(long long) * (S + 1),
                                        sizeof(long long), nr, cudaMemcpyDeviceToHost, ctx->stream));
            sp.s0 = s;
            sp.s1 = s + 1;
            sp.swap = (s + 1) % prm->swap_interval == 0;
            sp.round = (uint32_t)((s + 1) / prm->swap_interval - 1);
            pt_segment_kernel<<<(reads_total + 127) / 128, 128, 0, ctx->stream>>>(sp);
            QA_CK(cudaGetLastError());
            ++n_seg;
            QA_CK(cudaStreamSynchronize(ctx->stream));
            for (int rd = 0; rd < reads_total; ++rd) {
                const double nM = (double)problems[rd / prm->reads]->n * (double)P;
                // the fallback reads the bond sum of the ring in slot 0 before this step's swaps
                const long long b0 = ns > 0 ? 0 : hb[(size_t)rd * Rn + rin_prev[(size_t)rd * Rn]];
                const double on = opt_chi_raw(hs.data() + (size_t)rd * Rn * std::max(ns, 1), Rn, ns,
                                              (size_t)std::max(ns, 1), b0, nM);
                const double drive = std::max(on, minchi[rd]);
                jtr[(size_t)rd * S + s] = Jcur[rd];
                chitr[(size_t)rd * S + s] = drive;
                Jcur[rd] = std::min(Jcur[rd] + eps[rd] * std::pow(drive, -alpha), je);
            }
            if (ns == 0) {
                QA_CK(cudaMemcpyAsync(rin_prev.data(), d_rin, sizeof(int) * rin_prev.size(), cudaMemcpyDeviceToHost,
                                      ctx->stream));
                QA_CK(cudaStreamSynchronize(ctx->stream));
            }
        }
    }
    QA_CK(cudaEventRecord(ctx->ev[2], ctx->stream));
    QA_TRY(exact_energies(ctx, kind, d_probs, L, d_bits, d_exact));
    QA_CK(cudaEventRecord(ctx->ev[3], ctx->stream));
    std::vector<qa_sqapt_out *> po(n_problems);
    for (int p = 0; p < n_problems; ++p) po[p] = &outs[p].pt;
    const PTDev dv{d_best, d_exact, d_min, d_avg, d_swp, d_bstep, d_bslot, d_rin, d_bits, d_fbits, d_cnt};
    int64_t d2h = 0;
    QA_TRY(pt_collect(ctx, problems, n_problems, prm->reads, Rn, S, L, dv, po.data(), stats, &d2h));
    for (int p = 0; p < n_problems; ++p) {
        qa_sqaptopt_out &o = outs[p];
        for (int r = 0; r < prm->reads; ++r) {
            const int rd = p * prm->reads + r;
            if (o.j_perp_trace) std::memcpy(o.j_perp_trace + (size_t)r * S, jtr.data() + (size_t)rd * S, sizeof(double) * S);
            if (o.chi_B_trace) std::memcpy(o.chi_B_trace + (size_t)r * S, chitr.data() + (size_t)rd * S, sizeof(double) * S);
            if (o.scalars) {
                double *sc = o.scalars + (size_t)r * 4;
                sc[0] = eps[rd];
                sc[1] = js;
                sc[2] = je;
                sc[3] = Jcur[rd];
            }
        }
    }
    if (stats) {
        stats->sweep_launches = n_launch;
        stats->launches = (pl.own_fields() ? 2 : 3) + n_launch + n_seg;
        stats->h2d_bytes = 0;
        stats->d2h_bytes = d2h;
    }
    return QA_OK;
}

// ---------------------------------------------------------------------- MLP
int qa_mlp_create(qa_ctx *ctx, const int *dims, int n_dims, uint64_t seed, qa_mlp **out) {
    QA_TRY(begin(ctx));
    if (!out || !dims || n_dims < 2) return fail(QA_ERR_ARG, "an MLP needs at least an input and an output size.");
    for (int i = 0; i < n_dims; ++i)
        if (dims[i] <= 0 || dims[i] > 4096) return fail(QA_ERR_ARG, "MLP layer sizes must be in [1, 4096].");
    if (dims[n_dims - 1] % 2) return fail(QA_ERR_ARG, "the MLP output must hold M means and M log-variances.");
    qa_mlp *m = new qa_mlp();
    m->ctx = ctx;
    m->dims.assign(dims, dims + n_dims);
    const int L = n_dims - 1;
    std::vector<long long> wmap;
    for (int l = 0; l < L; ++l) {
        const long long kn = (long long)dims[l] * dims[l + 1];
        m->woff.push_back(m->nparams);
        m->w16off.push_back(m->nw16);
        for (long long i = 0; i < kn; ++i) wmap.push_back(m->nw16 + i);
        m->nparams += kn;
        m->nw16 += kn;
        m->boff.push_back(m->nparams);
        for (int i = 0; i < dims[l + 1]; ++i) wmap.push_back(-1);
        m->nparams += dims[l + 1];
    }
    // He-uniform initial weights from a splitmix64 stream, zero biases
    std::vector<float> W(m->nparams, 0.0f);
    uint64_t s = seed;
    auto next = [&s]() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    for (int l = 0; l < L; ++l) {
        const double a = std::sqrt(6.0 / dims[l]);
        for (long long i = 0; i < (long long)dims[l] * dims[l + 1]; ++i)
            W[m->woff[l] + i] = (float)(a * (2.0 * ((next() >> 11) * (1.0 / 9007199254740992.0)) - 1.0));
    }
    cudaError_t e = cudaMalloc(&m->W, sizeof(float) * m->nparams);
    if (e == cudaSuccess) e = cudaMalloc(&m->g, sizeof(float) * m->nparams);
    if (e == cudaSuccess) e = cudaMalloc(&m->mo, sizeof(float) * m->nparams);
    if (e == cudaSuccess) e = cudaMalloc(&m->vo, sizeof(float) * m->nparams);
    if (e == cudaSuccess) e = cudaMalloc(&m->W16, sizeof(__nv_bfloat16) * m->nw16);
    if (e == cudaSuccess) e = cudaMalloc(&m->wmap, sizeof(long long) * m->nparams);
    if (e != cudaSuccess) {
        qa_mlp_free(m);
        return fail(e == cudaErrorMemoryAllocation ? QA_ERR_OOM : QA_ERR_CUDA, cudaGetErrorString(e));
    }
    // all on the context's stream, ordered before the kernels that read them
    QA_CK(cudaMemcpyAsync(m->W, W.data(), sizeof(float) * m->nparams, cudaMemcpyHostToDevice, ctx->stream));
    QA_CK(cudaMemcpyAsync(m->wmap, wmap.data(), sizeof(long long) * m->nparams, cudaMemcpyHostToDevice, ctx->stream));
    QA_CK(cudaMemsetAsync(m->mo, 0, sizeof(float) * m->nparams, ctx->stream));
    QA_CK(cudaMemsetAsync(m->vo, 0, sizeof(float) * m->nparams, ctx->stream));
    mlp_to_bf16_kernel<<<(unsigned)((m->nparams + 255) / 256), 256, 0, ctx->stream>>>(m->W, m->nparams, m->wmap, m->W16);
    QA_CK(cudaGetLastError());
    QA_CK(cudaStreamSynchronize(ctx->stream));
    *out = m;
    return QA_OK;
}

int qa_mlp_free(qa_mlp *m) {
    if (!m) return QA_OK;
    cudaSetDevice(m->ctx->device);
    for (void *p : {(void *)m->W, (void *)m->g, (void *)m->mo, (void *)m->vo, (void *)m->W16, (void *)m->wmap,
                    (void *)m->acts, (void *)m->dacts, (void *)m->T, (void *)m->rowloss})
        if (p) cudaFree(p);
    delete m;
    return QA_OK;
}

int qa_mlp_num_params(const qa_mlp *m, int64_t *count) {
    if (!m || !count) return fail(QA_ERR_ARG, "null argument");
    *count = m->nparams;
    return QA_OK;
}

int qa_mlp_get_params(qa_mlp *m, float *host, int64_t count) {
    if (!m || !host || count != m->nparams) return fail(QA_ERR_ARG, "parameter buffer size mismatch");
    QA_TRY(begin(m->ctx));
    QA_CK(cudaMemcpyAsync(host, m->W, sizeof(float) * count, cudaMemcpyDeviceToHost, m->ctx->stream));
    QA_CK(cudaStreamSynchronize(m->ctx->stream));
    return QA_OK;
}

int qa_mlp_set_params(qa_mlp *m, const float *host, int64_t count) {
    if (!m || !host || count != m->nparams) return fail(QA_ERR_ARG, "parameter buffer size mismatch");
    QA_TRY(begin(m->ctx));
    QA_CK(cudaMemcpyAsync(m->W, host, sizeof(float) * count, cudaMemcpyHostToDevice, m->ctx->stream));
    QA_CK(cudaMemsetAsync(m->mo, 0, sizeof(float) * count, m->ctx->stream));
    QA_CK(cudaMemsetAsync(m->vo, 0, sizeof(float) * count, m->ctx->stream));
    m->step = 0;
    mlp_to_bf16_kernel<<<(unsigned)((m->nparams + 255) / 256), 256, 0, m->ctx->stream>>>(m->W, m->nparams, m->wmap,
                                                                                       m->W16);
    QA_CK(cudaGetLastError());
    QA_CK(cudaStreamSynchronize(m->ctx->stream));
    return QA_OK;
}

int qa_mlp_forward(qa_mlp *m, const float *X, int batch, float *Y) {
    if (!m || !X || !Y || batch <= 0) return fail(QA_ERR_ARG, "qa_mlp_forward: bad arguments");
    QA_TRY(begin(m->ctx));
    QA_TRY(mlp_prepare(m, batch, X, nullptr));
    QA_TRY(mlp_forward_dev(m, batch));
    const int L = (int)m->dims.size() - 1;
    QA_CK(cudaMemcpyAsync(Y, m->acts + m->aoff[L], sizeof(float) * (size_t)batch * m->dims[L], cudaMemcpyDeviceToHost,
                          m->ctx->stream));
    QA_CK(cudaStreamSynchronize(m->ctx->stream));
    return QA_OK;
}

int qa_mlp_loss_grad(qa_mlp *m, const float *X, const float *T, int batch, float *loss, float *grads) {
    if (!m || !X || !T || batch <= 0) return fail(QA_ERR_ARG, "qa_mlp_loss_grad: bad arguments");
    QA_TRY(begin(m->ctx));
    QA_TRY(mlp_prepare(m, batch, X, T));
    QA_TRY(mlp_forward_dev(m, batch));
    QA_TRY(mlp_backward_dev(m, batch, loss));
    if (grads) {
        QA_CK(cudaMemcpyAsync(grads, m->g, sizeof(float) * m->nparams, cudaMemcpyDeviceToHost, m->ctx->stream));
        QA_CK(cudaStreamSynchronize(m->ctx->stream));
    }
    return QA_OK;
}

int qa_mlp_train_step(qa_mlp *m, const float *X, const float *T, int batch, float lr, float *loss) {
    if (!m || !X || !T || batch <= 0 || !(lr > 0.0f)) return fail(QA_ERR_ARG, "qa_mlp_train_step: bad arguments");
    QA_TRY(begin(m->ctx));
    QA_TRY(mlp_prepare(m, batch, X, T));
    QA_TRY(mlp_forward_dev(m, batch));
    QA_TRY(mlp_backward_dev(m, batch, loss));
    m->step += 1;
    const float c1 = (float)(1.0 - std::pow(0.9, m->step)), c2 = (float)(1.0 - std::pow(0.999, m->step));
    mlp_adam_kernel<<<(unsigned)((m->nparams + 255) / 256), 256, 0, m->ctx->stream>>>(
        m->W, m->g, m->mo, m->vo, m->nparams, lr, 0.9f, 0.999f, 1e-8f, c1, c2, m->wmap, m->W16);
    QA_CK(cudaGetLastError());
    QA_CK(cudaStreamSynchronize(m->ctx->stream));
    return QA_OK;
}

// Stage 1 of run_chi: every (read, scan point) probe of the batch in one
// ring-kernel launch; chi[(problem*reads + read)*points + point].
static int chi_stage1(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, const qa_chi_params *prm,
                      int kind, int n_max, const std::vector<double> &scan_g, std::vector<double> &chi,
                      int64_t &launches, int64_t &h2d, int64_t &d2h, unsigned long long *cnt_total,
                      float &pilot_ms) {
    const int P = prm->trotter_slices, K = prm->replicas, Pts = prm->scan_points;
    const int reads_total = n_problems * prm->reads;
    Layout L;
    ProbDev *d_probs;
    RingDev *d_rings;
    uint32_t *d_spins;
    float *d_fields;
    double *d_sum, *d_best;
    int *d_bstep;
    uint32_t *d_bits;
    unsigned long long *d_cnt;
    float *d_B, *d_T4;
    QA_CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    // ---- Stage 1: all (read, point) probes in one launch
    build_rings(L, problems, n_problems, prm->reads, K, P, prm->seed, Pts);
    const int nr = (int)L.rings.size();
    const int sweeps_total = prm->scan_burn + prm->scan_sweeps;
    QA_TRY(upload_common(ctx, problems, n_problems, L, &d_probs, &d_rings, &d_spins, &d_fields));
    std::vector<float> B(Pts), T4(Pts);
    for (int m = 0; m < Pts; ++m) {
        B[m] = (float)(2.0 * (prm->beta / (double)P));
        T4[m] = (float)(4.0 * trotter_coupling(prm->beta, scan_g[m], P));
    }
    int *d_mag, *d_nof;
    double *d_chi;
    QA_TRY(ws_array(ctx, W_A, Pts, &d_B));
    QA_TRY(ws_array(ctx, W_T4, Pts, &d_T4));
    QA_TRY(ws_array(ctx, W_SUM, nr, &d_sum));
    QA_TRY(ws_array(ctx, W_BESTE, nr, &d_best));
    QA_TRY(ws_array(ctx, W_BESTSTEP, nr, &d_bstep));
    QA_TRY(ws_array(ctx, W_BITS, (size_t)nr * L.nw_max, &d_bits));
    QA_TRY(ws_array(ctx, W_CNT, 5, &d_cnt));
    QA_TRY(ws_array(ctx, W_MAG, (size_t)nr * sweeps_total, &d_mag));
    QA_TRY(ws_array(ctx, W_PROBOF, (size_t)reads_total * Pts, &d_nof));
    QA_TRY(ws_array(ctx, W_EXACT, (size_t)reads_total * Pts, &d_chi));
    std::vector<int> nof((size_t)reads_total * Pts);
    for (int p = 0; p < n_problems; ++p)
        for (int i = 0; i < prm->reads * Pts; ++i) nof[(size_t)p * prm->reads * Pts + i] = problems[p]->n;
    std::vector<double> inf(nr, INFINITY);
    QA_CK(cudaMemcpyAsync(d_B, B.data(), sizeof(float) * Pts, cudaMemcpyHostToDevice, ctx->stream));
    QA_CK(cudaMemcpyAsync(d_T4, T4.data(), sizeof(float) * Pts, cudaMemcpyHostToDevice, ctx->stream));
    QA_CK(cudaMemcpyAsync(d_nof, nof.data(), sizeof(int) * nof.size(), cudaMemcpyHostToDevice, ctx->stream));
    QA_CK(cudaMemcpyAsync(d_best, inf.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, ctx->stream));
    QA_CK(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long) * 5, ctx->stream));
    h2d += (int64_t)(sizeof(ProbDev) * n_problems + sizeof(RingDev) * nr + 2 * sizeof(float) * Pts +
                     sizeof(int) * nof.size() + sizeof(double) * nr);
    RingPlan pl;
    QA_TRY(plan_rings(ctx, problems, n_problems, kind, P, n_max, &pl));
    QA_TRY(init_state(ctx, kind, d_probs, d_rings, nr, d_spins, d_fields, P, n_max, L.nw_max, DOM_PILOT_INIT,
                      !pl.own_fields(), problems, n_problems, &L, d_cnt + 4));
    RingParams rp{};
    rp.probs = d_probs; rp.rings = d_rings; rp.spins = d_spins; rp.fields = d_fields;
    rp.P = P; rp.steps_total = 1; rp.spb = sweeps_total; rp.wls = 0; rp.slice_tag = DOM_PILOT;
    rp.B = d_B; rp.T4 = d_T4; rp.ring_sum = d_sum; rp.rec_base = 0; rp.rec_stride = 1;
    rp.best_E = d_best; rp.best_step = d_bstep; rp.best_bits = d_bits; rp.nw_max = L.nw_max;
    rp.mag = d_mag; rp.counters = d_cnt; rp.step0 = 0; rp.step1 = 1; rp.init_fields = 1;
    QA_TRY(launch_rings(ctx, kind, pl, rp, nr));
    const int probes = reads_total * Pts;
    chi_point_kernel<<<(probes + 127) / 128, 128, 0, ctx->stream>>>(d_mag, probes, K, sweeps_total,
                                                                     prm->scan_burn, d_nof, P, d_chi);
    QA_CK(cudaGetLastError());
    launches += (pl.own_fields() ? 1 : 2) + 2;
    unsigned long long c[5];
    QA_CK(cudaMemcpyAsync(chi.data(), d_chi, sizeof(double) * chi.size(), cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(c, d_cnt, sizeof(c), cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    QA_CK(cudaStreamSynchronize(ctx->stream));
    QA_TRY(check_device_error(c));
    QA_CK(cudaEventElapsedTime(&pilot_ms, ctx->ev[0], ctx->ev[1]));
    d2h += (int64_t)(sizeof(double) * chi.size() + sizeof(c));
    for (int i = 0; i < 4; ++i) cnt_total[i] += c[i];
    return QA_OK;
}

// Stage 1 alone: the chi_B curves of every (problem, read).
int qa_chi_pilot(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, const qa_chi_params *prm,
                 double *scan_chi, qa_stats *stats) {
    QA_TRY(begin(ctx));
    if (!prm || !scan_chi) return fail(QA_ERR_ARG, "null argument");
    if (!(prm->beta > 0.0)) return fail(QA_ERR_ARG, "beta must be > 0.");
    if (!(prm->gamma_end > 0.0) || !(prm->gamma_start > prm->gamma_end))
        return fail(QA_ERR_ARG, "Require gamma_start > gamma_end > 0.");
    if (prm->scan_points < 4) return fail(QA_ERR_ARG, "scan_points must be >= 4.");
    if (prm->scan_sweeps <= 0) return fail(QA_ERR_ARG, "scan_sweeps must be > 0.");
    if (prm->scan_burn < 0) return fail(QA_ERR_ARG, "scan_burn must be >= 0.");
    if (prm->trotter_slices <= 0) return fail(QA_ERR_ARG, "trotter_slices must be > 0.");
    if (prm->replicas <= 0) return fail(QA_ERR_ARG, "replicas must be > 0.");
    if (prm->reads <= 0) return fail(QA_ERR_ARG, "reads must be > 0.");
    int kind, n_max;
    QA_TRY(check_batch(problems, n_problems, &kind, &n_max));
    const int Pts = prm->scan_points;
    const double A0 = prm->driver_A0 > 0.0 ? prm->driver_A0 : prm->gamma_start;
    const double s_lo = A0 / (A0 + prm->gamma_start), s_hi = A0 / (A0 + prm->gamma_end);
    std::vector<double> scan_g(Pts), chi((size_t)n_problems * prm->reads * Pts);
    for (int m = 0; m < Pts; ++m)
        scan_g[m] = chi_s_to_gamma(A0, s_lo + (s_hi - s_lo) * (double)m / (double)(Pts - 1));
    int64_t launches = 0, h2d = 0, d2h = 0;
    unsigned long long cnt[4] = {0, 0, 0, 0};
    float ms = 0.0f;
    QA_TRY(chi_stage1(ctx, problems, n_problems, prm, kind, n_max, scan_g, chi, launches, h2d, d2h, cnt, ms));
    std::memcpy(scan_chi, chi.data(), sizeof(double) * chi.size());
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->slice_attempts = (int64_t)cnt[0];
        stats->slice_accepts = (int64_t)cnt[1];
        stats->sweep_ms = ms;
        stats->total_ms = ms;
        stats->max_field_drift = 0.0;
        stats->sweep_launches = 1;
        stats->launches = launches;
        stats->h2d_bytes = h2d;
        stats->d2h_bytes = d2h;
    }
    return QA_OK;
}

int qa_sqapt_run(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, const qa_sqapt_params *prm,
                 qa_sqapt_out *outs, qa_stats *stats) {
    return sqapt_impl(ctx, problems, n_problems, prm, outs, stats, false);
}

int qa_pt_run(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, const qa_pt_params *prm,
              qa_sqapt_out *outs, qa_stats *stats) {
    if (!prm) return fail(QA_ERR_ARG, "null params");
    // parallel_tempering.cpp:15-17, 39-47
    if (prm->rungs < 2 || !prm->betas) return fail(QA_ERR_ARG, "Parallel tempering requires at least two betas.");
    if (prm->sweeps_per_step <= 0) return fail(QA_ERR_ARG, "sweeps_per_step must be > 0.");
    if (prm->steps <= 0) return fail(QA_ERR_ARG, "steps must be > 0.");
    if (prm->swap_interval <= 0) return fail(QA_ERR_ARG, "swap_interval must be > 0.");
    qa_sqapt_params q{};
    q.betas = prm->betas;
    q.gammas = prm->betas;  // unused: no transverse field
    q.rungs = prm->rungs;
    q.trotter_slices = 1;
    q.sweeps_per_step = prm->sweeps_per_step;
    q.worldline_sweeps = 0;
    q.steps = prm->steps;
    q.swap_interval = prm->swap_interval;
    q.cluster_sweeps = 0;
    q.continuous_time_slices = 0;
    q.reads = prm->reads;
    q.seed = prm->seed;
    return sqapt_impl(ctx, problems, n_problems, &q, outs, stats, true);
}

// ---------------------------------------------------------------------- SQA-Chi
int qa_chi_run(qa_ctx *ctx, const qa_problem *const *problems, int n_problems, const qa_chi_params *prm,
               qa_chi_out *outs, qa_stats *stats) {
    QA_TRY(begin(ctx));
    if (!prm) return fail(QA_ERR_ARG, "null params");
    // sqa_chi_annealer.cpp:159-179
    if (prm->num_steps < 2) return fail(QA_ERR_ARG, "num_steps must be >= 2.");
    if (prm->sweeps_per_step <= 0) return fail(QA_ERR_ARG, "sweeps_per_step must be > 0.");
    if (!(prm->beta > 0.0)) return fail(QA_ERR_ARG, "beta must be > 0.");
    if (!(prm->gamma_end > 0.0) || !(prm->gamma_start > prm->gamma_end))
        return fail(QA_ERR_ARG, "Require gamma_start > gamma_end > 0.");
    if (prm->scan_points < 4) return fail(QA_ERR_ARG, "scan_points must be >= 4.");
    if (prm->scan_sweeps <= 0) return fail(QA_ERR_ARG, "scan_sweeps must be > 0.");
    if (prm->scan_burn < 0) return fail(QA_ERR_ARG, "scan_burn must be >= 0.");
    if (prm->chi_floor_fraction < 0.0) return fail(QA_ERR_ARG, "chi_floor_fraction must be >= 0.");
    if (prm->trotter_slices <= 0) return fail(QA_ERR_ARG, "trotter_slices must be > 0.");
    if (prm->replicas <= 0) return fail(QA_ERR_ARG, "replicas must be > 0.");
    if (prm->reads <= 0) return fail(QA_ERR_ARG, "reads must be > 0.");
    int kind, n_max;
    QA_TRY(check_batch(problems, n_problems, &kind, &n_max));
    const int P = prm->trotter_slices, K = prm->replicas, Pts = prm->scan_points, steps = prm->num_steps;
    const int reads_total = n_problems * prm->reads;
    const double A0 = prm->driver_A0 > 0.0 ? prm->driver_A0 : prm->gamma_start;
    const double s_lo = A0 / (A0 + prm->gamma_start), s_hi = A0 / (A0 + prm->gamma_end);
    std::vector<double> scan_s(Pts), scan_g(Pts), chi((size_t)reads_total * Pts);
    for (int m = 0; m < Pts; ++m) {
        scan_s[m] = s_lo + (s_hi - s_lo) * (double)m / (double)(Pts - 1);
        scan_g[m] = chi_s_to_gamma(A0, scan_s[m]);
    }
    int64_t launches = 0, h2d = 0, d2h = 0;
    unsigned long long cnt_total[4] = {0, 0, 0, 0};
    float pilot_ms = 0.0f;
    QA_CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    Layout L;
    ProbDev *d_probs;
    RingDev *d_rings;
    uint32_t *d_spins;
    float *d_fields;
    double *d_sum, *d_best, *d_exact;
    int *d_bstep;
    uint32_t *d_bits;
    unsigned long long *d_cnt;
    float *d_B, *d_T4;
    if (prm->scan_chi_in) {
        std::memcpy(chi.data(), prm->scan_chi_in, sizeof(double) * chi.size());
    } else {
        QA_TRY(chi_stage1(ctx, problems, n_problems, prm, kind, n_max, scan_g, chi, launches, h2d, d2h,
                          cnt_total, pilot_ms));
    }

    // ---- Stage 2 (host) per read
    std::vector<double> bs((size_t)reads_total * steps), gsch((size_t)reads_total * steps),
        ss((size_t)reads_total * steps), sc((size_t)reads_total * 5);
    for (int q = 0; q < reads_total; ++q) {
        chi_schedule(Pts, scan_s.data(), scan_g.data(), chi.data() + (size_t)q * Pts, prm->beta, prm->gamma_start,
                     prm->gamma_end, A0, P, steps, prm->chi_floor_fraction, prm->beta_ramp_fraction,
                     prm->beta_ramp_start, bs.data() + (size_t)q * steps, gsch.data() + (size_t)q * steps,
                     ss.data() + (size_t)q * steps, sc.data() + (size_t)q * 5);
        sc[(size_t)q * 5 + 4] = A0;
    }

    // ---- Stage 3: production on fresh worldlines, per-read schedules
    build_rings(L, problems, n_problems, prm->reads, K, P, prm->seed);
    for (auto &R : L.rings) R.sched = R.out * steps;
    const int nr = (int)L.rings.size();
    QA_TRY(upload_common(ctx, problems, n_problems, L, &d_probs, &d_rings, &d_spins, &d_fields));
    std::vector<float> B((size_t)reads_total * steps), T4((size_t)reads_total * steps);
    for (size_t i = 0; i < B.size(); ++i) {
        B[i] = (float)(2.0 * (bs[i] / (double)P));
        T4[i] = (float)(4.0 * trotter_coupling(bs[i], gsch[i], P));
    }
    QA_TRY(ws_array(ctx, W_A, B.size(), &d_B));
    QA_TRY(ws_array(ctx, W_T4, T4.size(), &d_T4));
    QA_TRY(ws_array(ctx, W_SUM, (size_t)nr * steps, &d_sum));
    QA_TRY(ws_array(ctx, W_BESTE, nr, &d_best));
    QA_TRY(ws_array(ctx, W_BESTSTEP, nr, &d_bstep));
    QA_TRY(ws_array(ctx, W_BITS, (size_t)nr * L.nw_max, &d_bits));
    QA_TRY(ws_array(ctx, W_CNT, 5, &d_cnt));
    QA_TRY(ws_array(ctx, W_EXACT, nr, &d_exact));
    {
        std::vector<double> inf(nr, INFINITY);
        std::vector<int> neg(nr, -1);
        QA_CK(cudaMemcpyAsync(d_B, B.data(), sizeof(float) * B.size(), cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_T4, T4.data(), sizeof(float) * T4.size(), cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_best, inf.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemcpyAsync(d_bstep, neg.data(), sizeof(int) * nr, cudaMemcpyHostToDevice, ctx->stream));
        QA_CK(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long) * 5, ctx->stream));
        QA_CK(cudaStreamSynchronize(ctx->stream));
        h2d += (int64_t)(sizeof(ProbDev) * n_problems + sizeof(RingDev) * nr + 2 * sizeof(float) * B.size() +
                         (sizeof(double) + sizeof(int)) * nr);
    }
    RingPlan pl;
    QA_TRY(plan_rings(ctx, problems, n_problems, kind, P, n_max, &pl));
    QA_CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    QA_TRY(init_state(ctx, kind, d_probs, d_rings, nr, d_spins, d_fields, P, n_max, L.nw_max, DOM_PROD_INIT, !pl.own_fields(),
                      problems, n_problems, &L, d_cnt + 4));
    RingParams rp{};
    rp.probs = d_probs; rp.rings = d_rings; rp.spins = d_spins; rp.fields = d_fields;
    rp.P = P; rp.steps_total = steps; rp.spb = prm->sweeps_per_step; rp.wls = 0; rp.slice_tag = DOM_PROD;
    rp.B = d_B; rp.T4 = d_T4; rp.ring_sum = d_sum; rp.rec_base = 0; rp.rec_stride = steps;
    rp.best_E = d_best; rp.best_step = d_bstep; rp.best_bits = d_bits; rp.nw_max = L.nw_max; rp.counters = d_cnt;
    int n_seg = 0;
    // rotated launches of an eighth of the anneal where whole-grid ones would
    // leave slots idle and the anneal has at least 200 sweeps
    if ((long long)steps * rp.spb >= 200 && rotation_pays(ctx, kind, pl, nr)) {
        rp.init_fields = 1;
        QA_TRY(run_rings_rotated(ctx, kind, pl, rp, nr, 0, steps, rot_seg(ctx, std::max(1, steps / 8), steps),
                                 &n_seg));
    } else {
        for (int s0 = 0; s0 < steps; s0 += 256) {
            rp.step0 = s0;
            rp.step1 = std::min(steps, s0 + 256);
            rp.init_fields = s0 == 0;
            QA_TRY(launch_rings(ctx, kind, pl, rp, nr));
            ++n_seg;
        }
    }
    QA_CK(cudaEventRecord(ctx->ev[2], ctx->stream));
    QA_TRY(exact_energies(ctx, kind, d_probs, L, d_bits, d_exact));
    QA_CK(cudaEventRecord(ctx->ev[3], ctx->stream));
    launches += (pl.own_fields() ? 2 : 3) + n_seg;
    std::vector<double> sums((size_t)nr * steps), bestE(nr), exact(nr);
    std::vector<int> bstep(nr);
    std::vector<uint32_t> bits((size_t)nr * L.nw_max);
    unsigned long long cnt[5];
    QA_CK(cudaMemcpyAsync(sums.data(), d_sum, sizeof(double) * sums.size(), cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(bestE.data(), d_best, sizeof(double) * nr, cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(bstep.data(), d_bstep, sizeof(int) * nr, cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(exact.data(), d_exact, sizeof(double) * nr, cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(bits.data(), d_bits, sizeof(uint32_t) * bits.size(), cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaMemcpyAsync(cnt, d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, ctx->stream));
    QA_CK(cudaStreamSynchronize(ctx->stream));
    QA_TRY(check_device_error(cnt));
    d2h += (int64_t)(sizeof(double) * (sums.size() + 2 * nr) + sizeof(int) * nr + sizeof(uint32_t) * bits.size() +
                     sizeof(cnt));
    for (int i = 0; i < 4; ++i) cnt_total[i] += cnt[i];

    for (int p = 0; p < n_problems; ++p) {
        const int n = problems[p]->n;
        qa_chi_out &o = outs[p];
        for (int r = 0; r < prm->reads; ++r) {
            const int q = p * prm->reads + r, base = q * K;
            if (o.energy_trace)
                for (int s = 0; s < steps; ++s) {
                    double tot = 0.0;
                    for (int k = 0; k < K; ++k) tot += sums[(size_t)(base + k) * steps + s];
                    o.energy_trace[(size_t)r * steps + s] = tot / (double)(K * P);
                }
            int kb = 0;
            for (int k = 1; k < K; ++k) {
                const int a = base + k, b = base + kb;
                if (bestE[a] < bestE[b] || (bestE[a] == bestE[b] && bstep[a] < bstep[b])) kb = k;
            }
            if (o.best_spins) unpack_bits(bits.data() + (size_t)(base + kb) * L.nw_max, n, o.best_spins + (size_t)r * n);
            if (o.best_energy) o.best_energy[r] = exact[base + kb];
            auto cp = [&](double *dst, const double *src, size_t len) {
                if (dst) std::memcpy(dst + (size_t)r * len, src, sizeof(double) * len);
            };
            cp(o.beta_schedule, bs.data() + (size_t)q * steps, steps);
            cp(o.gamma_schedule, gsch.data() + (size_t)q * steps, steps);
            cp(o.s_schedule, ss.data() + (size_t)q * steps, steps);
            cp(o.scan_s, scan_s.data(), Pts);
            cp(o.scan_gamma, scan_g.data(), Pts);
            cp(o.scan_chi_B, chi.data() + (size_t)q * Pts, Pts);
            cp(o.scalars, sc.data() + (size_t)q * 5, 5);
        }
    }
    if (stats) {
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, ctx->ev[1], ctx->ev[2]);
        cudaEventElapsedTime(&b, ctx->ev[1], ctx->ev[3]);
        stats->slice_attempts = (int64_t)cnt_total[0];
        stats->slice_accepts = (int64_t)cnt_total[1];
        stats->worldline_attempts = (int64_t)cnt_total[2];
        stats->worldline_accepts = (int64_t)cnt_total[3];
        stats->sweep_ms = a + pilot_ms;
        stats->total_ms = b + pilot_ms;
        stats->max_field_drift = 0.0;
        stats->sweep_launches = n_seg + (prm->scan_chi_in ? 0 : 1);
        stats->launches = launches;
        stats->h2d_bytes = h2d;
        stats->d2h_bytes = d2h;
    }
    return QA_OK;
}

}  // extern "C"
