// qa_order.cuh -- qanneal's update order for the Trotter-ring sweeps.
//
// qanneal's SQAAnnealer and SQAParallelTemperingAnnealer shuffle the spin
// order of a replica before every slice, cluster and worldline sweep
// (std::shuffle at sqa_annealer.cpp:181,216,295,599,631,703 and
// sqa_parallel_tempering.cpp:209,224,281,489) and sweep the Trotter slices one
// after another, t = 0 .. P-1, each in that order.  The engine samples the
// same Markov chain:
//  * the order of a sweep is a uniformly random permutation drawn from Philox:
//    spin i gets the key K_i = (r_i with its low 20 bits cleared) | i, where
//    r_i = (x_a << 32) | x_b comes from philox(i >> 1, ring, sweep,
//    (tag << 8) | DOM_PERM) (words 0, 1 for even i, 2, 3 for odd i), and the
//    spins are visited in increasing key order.  44 random bits a key make a
//    tie (broken by the spin index) a one-in-10^9 event for n = 512;
//  * the keys are bucketed by their top bits (a counting sort in shared
//    memory, about four spins a bucket) and each bucket is put in key order,
//    which is the full sort by K_i in O(n) work and five barriers;
//  * the slices of a ring run concurrently in a pipeline: slice t takes a
//    block of 32 visiting positions once slice t - 1 has finished that block
//    (bounded waits on per-slice progress counters in shared memory).  A move of spin i in slice t then sees slice t - 1 after this sweep and
//    slice t + 1 before it, exactly as the sequential loop does: the block's
//    spins are touched by no other slice while slice t holds them.
#pragma once
#include "qa_device.cuh"

namespace qa {

__host__ __device__ inline size_t ord_align16(size_t x) { return (x + 15) / 16 * 16; }

// log2 of the bucket count of an order build: about four spins a bucket.
__host__ __device__ inline int order_nb_log2(int n) {
    int c = 0;
    while ((1 << c) < n) ++c;
    c -= 2;
    return c < 0 ? 0 : (c > 11 ? 11 : c);
}

// Shared memory of the order build: the keys (scratch), the bucket counters
// (scratch) and the order itself (read through the sweep).
__host__ __device__ inline size_t order_keys_bytes(int n) { return ord_align16((size_t)((n + 1) & ~1) * 8); }
__host__ __device__ inline size_t order_cnt_bytes(int n) { return ord_align16((size_t)4 << order_nb_log2(n)); }
__host__ __device__ inline size_t order_idx_bytes(int n) { return ord_align16((size_t)n * 4); }

// A visiting order's entries: spins < 2^16.
typedef uint16_t OrdT;
constexpr int QA_ORDER_MAX_N = 1 << 16;

// A bounded wait gives up after a second (device global timer), records
// QA_DEV_ERR_TIMEOUT and stops every later wait of the CTA.
constexpr unsigned long long QA_WAIT_NS = 1000000000ull;
constexpr unsigned long long QA_DEV_ERR_TIMEOUT = 1ull;

// The visiting order of one sweep: order[p] = the spin visited p-th.  Whole
// CTA; ends with a barrier.  keys: [n] scratch, cnt: [2^order_nb_log2(n)]
// scratch, order: [n] (shared or global memory).
//  1. every key is drawn and counted in its bucket (top bits of the key);
//  2. one warp turns the counts into bucket starts;
//  3. the keys are drawn again and scattered into their buckets;
//  4. each key's position is its bucket's start plus the number of smaller
//     keys in its bucket (about four), written as the spin (the key's low
//     bits).
__device__ __forceinline__ void build_sweep_order(uint64_t key, uint32_t ring, uint32_t sigma, uint32_t tag, int n,
                                                  unsigned long long *keys, int *cnt, OrdT *order) {
    const int nbl = order_nb_log2(n), NB = 1 << nbl;
    const int tid = threadIdx.x, T = blockDim.x;
    const uint32_t c3 = (tag << 8) | (uint32_t)DOM_PERM;
    const int npairs = (n + 1) >> 1;
    auto bucket = [&](unsigned long long k) { return nbl ? (int)(k >> (64 - nbl)) : 0; };
    for (int b = tid; b < NB; b += T) cnt[b] = 0;
    __syncthreads();
    for (int j = tid; j < npairs; j += T) {
        const U4 r = philox((uint32_t)j, ring, sigma, c3, key);
        atomicAdd(cnt + bucket(((unsigned long long)r.x << 32) | r.y), 1);
        if (2 * j + 1 < n) atomicAdd(cnt + bucket(((unsigned long long)r.z << 32) | r.w), 1);
    }
    __syncthreads();
    // exclusive prefix sum of the bucket counts, one warp: lane l owns a run of buckets
    if (tid < 32) {
        const int per = (NB + 31) >> 5;
        const int b0 = min(NB, tid * per), b1 = min(NB, b0 + per);
        int s = 0;
        for (int b = b0; b < b1; ++b) s += cnt[b];
        int incl = s;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int v = __shfl_up_sync(FULL, incl, off);
            if (tid >= off) incl += v;
        }
        int run = incl - s;
        for (int b = b0; b < b1; ++b) {
            const int c = cnt[b];
            cnt[b] = run;
            run += c;
        }
    }
    __syncthreads();
    // scatter (cnt[b] ends as the end of bucket b)
    for (int j = tid; j < npairs; j += T) {
        const U4 r = philox((uint32_t)j, ring, sigma, c3, key);
        const int i0 = 2 * j, i1 = i0 + 1;
        const unsigned long long k0 =
            ((((unsigned long long)r.x << 32) | r.y) & ~0xFFFFFull) | (unsigned long long)i0;
        keys[atomicAdd(cnt + bucket(k0), 1)] = k0;
        if (i1 < n) {
            const unsigned long long k1 =
                ((((unsigned long long)r.z << 32) | r.w) & ~0xFFFFFull) | (unsigned long long)i1;
            keys[atomicAdd(cnt + bucket(k1), 1)] = k1;
        }
    }
    __syncthreads();
    for (int x = tid; x < n; x += T) {
        const unsigned long long kx = keys[x];
        const int b = bucket(kx);
        const int s0 = b == 0 ? 0 : cnt[b - 1], s1 = cnt[b];
        int rank = 0;
        for (int y = s0; y < s1; ++y) rank += keys[y] < kx;
        order[s0 + rank] = (OrdT)(kx & 0xFFFFFull);
    }
    __syncthreads();
}

// The ring kernels take the orders of their sweeps from a buffer that
// order_fill_kernel writes before each launch (the orders of every sweep of
// the launch, one row of ord_row_entries(n) entries each): a sweep copies its
// row into shared memory with 16-byte cp.async chunks while the previous sweep
// runs.  Whole CTA; order_wait() and a barrier make the copy visible.
__host__ __device__ inline int ord_row_entries(int n) { return (n + 7) & ~7; }
__host__ __device__ inline size_t ord_row_bytes(int n) { return (size_t)ord_row_entries(n) * sizeof(OrdT); }

__device__ __forceinline__ void order_fetch(OrdT *dst, const OrdT *src, int n) {
    const int chunks = ord_row_entries(n) >> 3;
    for (int c = threadIdx.x; c < chunks; c += blockDim.x)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst + 8 * c)),
                     "l"(src + 8 * c)
                     : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void order_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// The order rows of one ring's sweeps, taken in the order the kernel sweeps.
// With shared-memory buffers, row r is copied while row r - 1 is swept.
struct OrderFeed {
    OrdT *buf0, *buf1;  // shared memory (null: the rows are read in global memory)
    const OrdT *g;      // the ring's first row
    long long stride;   // entries per row
    int n, rows, row;   // spins, rows of the launch, the next row
};

__device__ __forceinline__ OrderFeed feed_open(OrdT *buf0, OrdT *buf1, const OrdT *g, long long stride, int n,
                                               int rows) {
    OrderFeed f{buf0, buf1, g, stride, n, rows, 0};
    if (buf0 && rows > 0) order_fetch(buf0, g, n);
    return f;
}

// The next sweep's order.  Whole CTA; ends with a barrier after which every
// thread sees the row (and whatever the CTA wrote before it); starts the copy
// of the row after it into the buffer the previous sweep used.
__device__ __forceinline__ const OrdT *feed_take(OrderFeed &f) {
    const int r = min(f.row, max(f.rows - 1, 0));  // never past the launch's rows
    ++f.row;
    if (!f.buf0) {
        __syncthreads();
        return f.g + r * f.stride;
    }
    order_wait();
    __syncthreads();
    if (r + 1 < f.rows) order_fetch((r & 1) ? f.buf0 : f.buf1, f.g + (r + 1) * f.stride, f.n);
    return (r & 1) ? f.buf1 : f.buf0;
}

// Pipeline counters: acquire / release accesses of a shared-memory word.
__device__ __forceinline__ int ld_acquire_cta(const int *p) {
    int v;
    asm volatile("ld.acquire.cta.shared.b32 %0, [%1];"
                 : "=r"(v)
                 : "r"((unsigned)__cvta_generic_to_shared(p))
                 : "memory");
    return v;
}
__device__ __forceinline__ void st_release_cta(int *p, int v) {
    asm volatile("st.release.cta.shared.b32 [%0], %1;" ::"r"((unsigned)__cvta_generic_to_shared(p)), "r"(v)
                 : "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// The slice pipeline of one ring: prog[t] counts the blocks slice t has
// finished in the current sweep.
__host__ __device__ inline size_t pipe_bytes(int P) { return ord_align16((size_t)P * 4) + 16; }

struct SlicePipe {
    int *prog;                 // [P]
    int *abortf;               // set when a wait ran out: later waits return at once
    unsigned long long *err;   // the run's device error word
};

// Carve the pipeline out of pipe_bytes(P) bytes of shared memory at ptr and
// initialise it (whole CTA; a barrier must follow before the first sweep).
__device__ __forceinline__ SlicePipe pipe_open(unsigned char *ptr, int P, unsigned long long *err) {
    SlicePipe pp;
    pp.prog = reinterpret_cast<int *>(ptr);
    pp.abortf = reinterpret_cast<int *>(ptr + ord_align16((size_t)P * 4));
    pp.err = err;
    if (threadIdx.x == 0) *pp.abortf = 0;
    return pp;
}

// Before a sweep (whole CTA, ahead of the barrier that starts it).
__device__ __forceinline__ void pipe_reset(const SlicePipe &pp, int P) {
    for (int t = threadIdx.x; t < P; t += blockDim.x) pp.prog[t] = 0;
}

// Whole warp: wait until slice tp has finished block q.  Every lane polls
// (one broadcast load a poll, so the warp stays converged and each lane's
// later reads are ordered after its own acquire), with a short back-off.
// Past QA_WAIT_NS lane 0 sets the abort flag (no later wait of the CTA spins)
// and the error word, and the warp carries on: the run's outputs are then
// void and the host reports QA_ERR_TIMEOUT.
__device__ __forceinline__ void pipe_wait(const SlicePipe &pp, int tp, int q, int lane) {
    const int need = q + 1;
    if (ld_acquire_cta(pp.prog + tp) >= need) return;
    const unsigned long long t0 = global_ns();
    while (ld_acquire_cta(pp.prog + tp) < need) {
        if (*(volatile int *)pp.abortf) break;
        if (global_ns() - t0 > QA_WAIT_NS) {
            if (lane == 0) {
                *(volatile int *)pp.abortf = 1;
                atomicExch(pp.err, QA_DEV_ERR_TIMEOUT);
            }
            break;
        }
        __nanosleep(40);
    }
}

// Whole warp, block q of slice t finished.  fenced: the warp wrote state a
// later slice reads (every lane fences its writes and the warp synchronises
// first).  Every lane stores the count (release; the same value, one store
// instruction).
__device__ __forceinline__ void pipe_publish(const SlicePipe &pp, int t, int q, int lane, bool fenced = true) {
    (void)lane;
    if (fenced) {
        __threadfence_block();
        __syncwarp();
    }
    st_release_cta(pp.prog + t, q + 1);
}

}  // namespace qa
