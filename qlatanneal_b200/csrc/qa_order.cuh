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
//    (bounded waits on per-slice progress counters in shared memory).  A
//    move of spin i in slice t then sees slice t - 1 after this sweep and
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

// A bounded wait gives up after this many polls (about a second with the
// back-off), records QA_DEV_ERR_TIMEOUT and stops every later wait of the CTA.
constexpr int QA_WAIT_LIMIT = 1 << 23;
constexpr unsigned long long QA_DEV_ERR_TIMEOUT = 1ull;

// The visiting order of one sweep: order[p] = the spin visited p-th.  Whole
// CTA; ends with a barrier.  keys: [even(n)] scratch, cnt: [2^order_nb_log2(n)]
// scratch, order: [n].
__device__ __forceinline__ void build_sweep_order(uint64_t key, uint32_t ring, uint32_t sigma, uint32_t tag, int n,
                                                  unsigned long long *keys, int *cnt, int *order) {
    const int nbl = order_nb_log2(n), NB = 1 << nbl;
    const int tid = threadIdx.x, T = blockDim.x;
    for (int b = tid; b < NB; b += T) cnt[b] = 0;
    __syncthreads();
    const uint32_t c3 = (tag << 8) | (uint32_t)DOM_PERM;
    const int npairs = (n + 1) >> 1;
    for (int j = tid; j < npairs; j += T) {
        const U4 r = philox((uint32_t)j, ring, sigma, c3, key);
        const int i0 = 2 * j, i1 = i0 + 1;
        const unsigned long long k0 =
            ((((unsigned long long)r.x << 32) | r.y) & ~0xFFFFFull) | (unsigned long long)i0;
        keys[i0] = k0;
        atomicAdd(cnt + (nbl ? (int)(k0 >> (64 - nbl)) : 0), 1);
        if (i1 < n) {
            const unsigned long long k1 =
                ((((unsigned long long)r.z << 32) | r.w) & ~0xFFFFFull) | (unsigned long long)i1;
            keys[i1] = k1;
            atomicAdd(cnt + (nbl ? (int)(k1 >> (64 - nbl)) : 0), 1);
        }
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
    // scatter by bucket (within a bucket in arrival order: sorted next)
    for (int i = tid; i < n; i += T) {
        const unsigned long long k = keys[i];
        const int pos = atomicAdd(cnt + (nbl ? (int)(k >> (64 - nbl)) : 0), 1);
        order[pos] = i;
    }
    __syncthreads();
    // cnt[b] now ends bucket b; put each bucket in key order
    for (int b = tid; b < NB; b += T) {
        const int s0 = b == 0 ? 0 : cnt[b - 1], s1 = cnt[b];
        for (int x = s0 + 1; x < s1; ++x) {
            const int v = order[x];
            const unsigned long long kv = keys[v];
            int y = x - 1;
            while (y >= s0 && keys[order[y]] > kv) {
                order[y + 1] = order[y];
                --y;
            }
            order[y + 1] = v;
        }
    }
    __syncthreads();
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

// Whole warp: wait until *flag >= need.  Lane 0 polls (acquire) with a short
// back-off and at most QA_WAIT_LIMIT polls; past that it sets *abort (shared,
// so no later wait of the CTA spins) and the error word *err (global), and
// the warp carries on: the run's outputs are then void and the host reports
// QA_ERR_TIMEOUT.  The __syncwarp orders the other lanes' reads after the
// acquire.
__device__ __forceinline__ void wait_at_least(const int *flag, int need, int *abort, unsigned long long *err,
                                              int lane) {
    if (lane == 0 && ld_acquire_cta(flag) < need) {
        int it = 0;
        while (ld_acquire_cta(flag) < need) {
            if (*(volatile int *)abort) break;
            if (++it > QA_WAIT_LIMIT) {
                *(volatile int *)abort = 1;
                atomicExch(err, QA_DEV_ERR_TIMEOUT);
                break;
            }
            __nanosleep(40);
        }
    }
    __syncwarp();
}

// Whole warp, after the warp's writes of a finished block: every lane fences
// its writes, lane 0 publishes the count (release).
__device__ __forceinline__ void publish_count(int *flag, int value, int lane) {
    __threadfence_block();
    __syncwarp();
    if (lane == 0) st_release_cta(flag, value);
}

}  // namespace qa
