// qa_noalloc.cu -- qa_sa_dense_run_noalloc: dense SA runs without any device
// allocation by this library.
//
// Who needs it: callers whose GPU memory is owned by someone else's allocator
// (PyTorch's caching allocator, JAX/XLA, which reserves most of HBM up front,
// or a serving process with a fixed memory budget) cannot let a library call
// cudaMalloc/cudaFree in the middle of their work: the allocation may fail
// because their pool already holds the memory, and it also synchronises the
// device.  They allocate inputs and outputs themselves and hand over device
// pointers; everything else this run needs lives in g_scratch below.
//
// g_scratch is a file-scope __device__ array of QA_NOALLOC_SCRATCH_BYTES
// (16 MiB).  Every GPU that loads the library's device code holds it until
// the process exits.  Under CUDA's default lazy module loading that happens
// inside the first call on a device, which is when the 16 MiB are reserved:
// make that first call (a small warm-up run will do) before the framework
// reserves most of the device memory, or set CUDA_MODULE_LOADING=EAGER so the
// array is reserved when the context is created.  Host code never
// dereferences the symbol: its device address is looked up once per device
// with cudaGetSymbolAddress, on the first call made with that device (make
// that first call before any stream capture).  The call switches to `device`
// for its work and puts the caller's current device back before it returns.
// Every call reuses the same array and leaves its contents behind; what must
// start at zero (the counters) is cleared on each call.  Two calls whose work
// overlaps on the GPU (different streams, or different host threads) race on
// the array: serialise them.
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "qa_gpu.h"
#include "qa_kernels.cuh"

using namespace qa;

namespace qa {
int set_last_error(int code, const char *msg);  // qa_capi.cu
}

#define QA_NOALLOC_SCRATCH_BYTES (size_t(16) << 20)

static __device__ __align__(256) unsigned char g_scratch[QA_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int QA_NOALLOC_MAX_DEVICES = 64;

std::mutex g_scratch_mu;
unsigned char *g_scratch_addr[QA_NOALLOC_MAX_DEVICES] = {};

int noalloc_fail(int code, const std::string &msg) { return qa::set_last_error(code, msg.c_str()); }

// Puts the calling thread's current device back when the call returns, on
// every path: a framework caller working on another device must not find
// itself switched to this call's device.
struct DeviceRestore {
    int prev = -1;
    DeviceRestore() {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    }
    ~DeviceRestore() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

size_t carve(size_t &off, size_t bytes) {
    const size_t at = (off + 255) / 256 * 256;
    off = at + bytes;
    return at;
}

// float32 copies of h and of the upper triangle of J (mirrored, zero
// diagonal), as qa_problem_dense prepares them on the host.
__global__ void noalloc_prepare_dense(const double *h, const double *J, int n, float *h32, float *J32) {
    const long long nn = (long long)n * n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < nn;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx / n), j = (int)(idx - (long long)i * n);
        const int a = i < j ? i : j, b = i < j ? j : i;
        J32[idx] = i == j ? 0.0f : (float)J[(long long)a * n + b];
        if (j == 0) h32[i] = (float)h[i];
    }
}

__global__ void noalloc_unpack(const uint32_t *bits, int nw_max, int n, int reads, int8_t *out) {
    const long long total = (long long)reads * n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(idx / n), i = (int)(idx - (long long)r * n);
        out[idx] = ((bits[(long long)r * nw_max + (i >> 5)] >> (i & 31)) & 1u) ? 1 : -1;
    }
}

}  // namespace

#define NA_CK(call)                                                                       \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return noalloc_fail(QA_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

extern "C" int qa_sa_dense_run_noalloc(int device, void *stream, int n, const double *d_h, const double *d_J,
                                       double c, const qa_sa_params *prm, int8_t *d_best_spins,
                                       double *d_best_energy, double *d_energy_trace, qa_stats *stats) {
    if (!prm || !prm->betas || prm->steps <= 0) return noalloc_fail(QA_ERR_ARG, "Schedule must contain at least one beta.");
    if (prm->sweeps_per_beta <= 0) return noalloc_fail(QA_ERR_ARG, "sweeps_per_beta must be > 0.");
    if (prm->reads <= 0) return noalloc_fail(QA_ERR_ARG, "reads must be > 0.");
    if (n <= 0) return noalloc_fail(QA_ERR_ARG, "DenseIsing size must be > 0.");
    if (!d_h || !d_J || !d_best_spins || !d_best_energy || !d_energy_trace)
        return noalloc_fail(QA_ERR_ARG, "qa_sa_dense_run_noalloc: every device pointer must be non-null.");
    if (device < 0 || device >= QA_NOALLOC_MAX_DEVICES) return noalloc_fail(QA_ERR_ARG, "device index out of range");
    for (int s = 0; s < prm->steps; ++s)
        if (!(prm->betas[s] >= 0.0)) return noalloc_fail(QA_ERR_ARG, "betas must be >= 0.");

    // scratch layout for this call
    const int reads = prm->reads, steps = prm->steps, nw = (n + 31) / 32;
    size_t off = 0;
    const size_t o_prob = carve(off, sizeof(ProbDev));
    const size_t o_rings = carve(off, sizeof(RingDev) * (size_t)reads);
    const size_t o_h32 = carve(off, sizeof(float) * (size_t)n);
    const size_t o_J32 = carve(off, sizeof(float) * (size_t)n * n);
    const size_t o_B = carve(off, sizeof(float) * (size_t)steps);
    const size_t o_spins = carve(off, sizeof(uint32_t) * (size_t)reads * nw);
    const size_t o_fields = carve(off, sizeof(float) * (size_t)reads * n);
    const size_t o_best = carve(off, sizeof(double) * (size_t)reads);
    const size_t o_bits = carve(off, sizeof(uint32_t) * (size_t)reads * nw);
    const size_t o_cnt = carve(off, sizeof(unsigned long long) * 4);
    const size_t o_pof = carve(off, sizeof(int) * (size_t)reads);
    if (off > QA_NOALLOC_SCRATCH_BYTES)
        return noalloc_fail(QA_ERR_ARG, "qa_sa_dense_run_noalloc: this run needs " + std::to_string(off) +
                                            " bytes of scratch (about 4*n*n + 8*reads*n + 4*steps); the static "
                                            "scratch holds " + std::to_string(QA_NOALLOC_SCRATCH_BYTES) + " bytes.");

    DeviceRestore restore_device;
    NA_CK(cudaSetDevice(device));
    unsigned char *base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_scratch_mu);
        if (!g_scratch_addr[device]) {
            void *p = nullptr;
            NA_CK(cudaGetSymbolAddress(&p, g_scratch));
            g_scratch_addr[device] = static_cast<unsigned char *>(p);
        }
        base = g_scratch_addr[device];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    ProbDev pd{};
    pd.kind = K_DENSE;
    pd.n = n;
    pd.nw = nw;
    pd.c = c;
    pd.h32 = reinterpret_cast<const float *>(base + o_h32);
    pd.h64 = d_h;
    pd.J32 = reinterpret_cast<const float *>(base + o_J32);
    pd.J64 = d_J;
    std::vector<RingDev> rings(reads);
    for (int r = 0; r < reads; ++r) {
        rings[r] = RingDev{};
        rings[r].prob = 0;
        rings[r].out = r;
        rings[r].key = prm->seed + (uint64_t)r;
        rings[r].spin_off = (long long)r * nw;
        rings[r].field_off = (long long)r * n;
    }
    std::vector<float> B(steps);
    for (int s = 0; s < steps; ++s) B[s] = (float)(2.0 * prm->betas[s]);
    std::vector<int> pof(reads, 0);
    NA_CK(cudaMemcpyAsync(base + o_prob, &pd, sizeof(pd), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(base + o_rings, rings.data(), sizeof(RingDev) * reads, cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(base + o_B, B.data(), sizeof(float) * steps, cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(base + o_pof, pof.data(), sizeof(int) * reads, cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemsetAsync(base + o_cnt, 0, sizeof(unsigned long long) * 4, st));

    const ProbDev *d_prob = reinterpret_cast<const ProbDev *>(base + o_prob);
    const RingDev *d_rings = reinterpret_cast<const RingDev *>(base + o_rings);
    uint32_t *d_spins = reinterpret_cast<uint32_t *>(base + o_spins);
    float *d_fields = reinterpret_cast<float *>(base + o_fields);
    uint32_t *d_bits = reinterpret_cast<uint32_t *>(base + o_bits);
    unsigned long long *d_cnt = reinterpret_cast<unsigned long long *>(base + o_cnt);

    noalloc_prepare_dense<<<256, 256, 0, st>>>(d_h, d_J, n, reinterpret_cast<float *>(base + o_h32),
                                               reinterpret_cast<float *>(base + o_J32));
    NA_CK(cudaGetLastError());
    init_spins_kernel<<<dim3(reads, 1), 128, 0, st>>>(d_prob, d_rings, d_spins, 1, DOM_INIT, nw);
    NA_CK(cudaGetLastError());
    const int zb = std::max(1, std::min(64, (n + 127) / 128));
    init_fields_kernel<K_DENSE><<<dim3(reads, 1, zb), 128, nw * 4, st>>>(d_prob, d_rings, d_spins, d_fields, 1);
    NA_CK(cudaGetLastError());
    SAParams sp{};
    sp.probs = d_prob;
    sp.rings = d_rings;
    sp.spins = d_spins;
    sp.fields = d_fields;
    sp.B = reinterpret_cast<const float *>(base + o_B);
    sp.steps = steps;
    sp.spb = prm->sweeps_per_beta;
    const size_t smem_base = (size_t)((nw + 3) & ~3) * 4 + (size_t)((n + 3) & ~3) * 4;
    sp.smem_fields = smem_base + (size_t)n * 4 <= 48 * 1024 ? 1 : 0;
    const size_t smem = smem_base + (sp.smem_fields ? (size_t)n * 4 : 0);
    if (smem > 48 * 1024)
        NA_CK(cudaFuncSetAttribute(sa_kernel<K_DENSE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    sp.trace = d_energy_trace;
    sp.best_E = reinterpret_cast<double *>(base + o_best);
    sp.best_bits = d_bits;
    sp.nw_max = nw;
    sp.counters = d_cnt;
    sa_kernel<K_DENSE><<<reads, 32, smem, st>>>(sp);
    NA_CK(cudaGetLastError());
    exact_energy_kernel<K_DENSE><<<reads, 32, nw * 4, st>>>(d_prob, reinterpret_cast<const int *>(base + o_pof),
                                                             d_bits, nw, d_best_energy, reads);
    NA_CK(cudaGetLastError());
    noalloc_unpack<<<256, 256, 0, st>>>(d_bits, nw, n, reads, d_best_spins);
    NA_CK(cudaGetLastError());
    if (stats) {
        unsigned long long cnt[4];
        NA_CK(cudaMemcpyAsync(cnt, d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, st));
        NA_CK(cudaStreamSynchronize(st));
        std::memset(stats, 0, sizeof(*stats));
        stats->slice_attempts = (int64_t)cnt[0];
        stats->slice_accepts = (int64_t)cnt[1];
        stats->launches = 6;
        stats->max_field_drift = 0.0;
        stats->sweep_launches = 1;
    }
    NA_CK(cudaStreamSynchronize(st));
    return QA_OK;
}
