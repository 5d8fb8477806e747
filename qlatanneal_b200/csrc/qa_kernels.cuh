// qa_kernels.cuh -- the field-cache sweep kernels (every model kind).
//
//  * init_spins_kernel / init_fields_kernel: fresh random worldlines and their
//    local-field caches (the reference's SQAState::random + compute_local_fields,
//    sqa_annealer.cpp:100,130-137).
//  * sa_kernel: SA Metropolis, one warp per read (annealer.cpp:33-75), with the
//    running energy and per-flip best tracking of the reference.
//  * ring_kernel: one CTA per Trotter ring (a replica of a read, a PT rung or a
//    chi pilot probe): parity-phase slice sweeps (warp per slice), CTA-wide
//    worldline sweeps, step-end energy scan and best tracking
//    (sqa_annealer.cpp:153-469, sqa_parallel_tempering.cpp:187-306,
//    sqa_chi_annealer.cpp:81-140).
//
// Inside a slice, 32 consecutive spins form a block owned lane-by-lane.  Each
// lane draws its uniform (one Philox call serves four blocks) and tests its own
// spin; the warp then resolves the block in spin order by balloting the
// decisions and taking the first accepting lane.  Spins before it were
// rejected on current fields; after its flip the fields are updated and the
// remaining lanes re-test.  This is the sequential Metropolis sweep exactly,
// at a cost of (accepted flips + 1) ballots per block.
#pragma once
#include "qa_device.cuh"
#include "qa_order.cuh"

namespace qa {

// One Trotter ring (or one SA chain when P == 1).
struct RingDev {
    int prob;            // problem index
    int out;             // result slot (problem, read)
    int k;               // replica index inside the read (slice-RNG cell base k*P)
    int sched;           // offset into the per-step B/T4 tables
    uint32_t tag_extra;  // OR-ed into the domain tags of this ring (chi pilot: point << 8)
    uint64_t key;        // Philox key = seed + read
    long long spin_off;  // uint32 words, P * nw
    long long field_off; // floats, P * n
};

struct RingParams {
    const ProbDev *probs;
    const RingDev *rings;
    uint32_t *spins;
    float *fields;
    int P, W;             // slices per ring, warps per CTA
    int step0, step1;     // steps run by this launch
    int steps_total;
    int spb, wls;         // slice / worldline sweeps per step
    uint32_t slice_tag;   // DOM_SLICE, DOM_PROD or DOM_PILOT|(point<<8)
    const int *slot;      // PT: rung slot of each ring (null: slot = k)
    const float *B, *T4;  // [sched + step] (PT: [sched + slot + step * slot_step]): B = 2 beta/P, T4 = 4 J_perp
    int cls;              // cluster sweeps per step (ring_kernel only; P <= 64)
    const float *JP;      // like B: bond probability 1 - exp(-2 J_perp) of the cluster moves
    long long *bsamp;     // bond sum after every slice and cluster sweep, or null:
    int bstride;          //   [ring * bstride + (step - step0) * (spb + cls) + sweep]
    int per_slot_sched;   // 1: index B/T4/JP by slot (+ step * slot_step) instead of step
    int slot_step;        //   0: one entry per slot; R: a row of R slots per step (one J_perp per step)
    int smem_fields;
    int ref_order;        // 1: qanneal's order (a random spin order per sweep, slices in turn); 0: parity
                          //    checkerboard, spins ascending (the SQA-Chi kernel's order)
    OrdT *ordg;           // qanneal's order: the visiting orders of this launch's sweeps, written by
    long long ord_ring;   //   order_fill_kernel before it.  Ring b's rows start at ordg + b * ord_ring;
    int ord_stride;       //   row (s - step0) * ord_per_step + k holds the k-th ordered sweep of step s
    int ord_per_step;     //   (slice sweeps, cluster sweeps where the kernel has them, worldline sweeps)
    int ord_in_smem;      // ring_kernel: rows copied into shared memory (else read from ordg)
    int init_fields;      // ring_pm1_kernel: build the int32 fields from the spins first
    int init_scan;        // score the starting state as "step -1" before step0 (PT)
    int rec_base;         // per-step records live at [ring][rec_base + step]
    int rec_stride;       //   with this row stride
    // outputs
    double *ring_sum;     // sum of slice energies per (ring, step)
    double *ring_min;     // min slice energy (PT projected energy) per (ring, step), may be null
    long long *ring_bond; // imaginary-time bond sum B per (ring, step), may be null
    double *best_E;       // [ring]
    int *best_step;       // [ring]
    int *best_slot;       // [ring] slot the ring held at its best step, may be null
    uint32_t *best_bits;  // [ring][nw_max]
    uint32_t *final_bits; // [ring][nw_max] min-energy slice after the last step, may be null
    int nw_max;
    int *mag;             // [ring][sweeps] spin sums after each sweep (chi pilot), may be null
    unsigned long long *counters;  // [5]: slice attempts, accepts, worldline attempts, accepts, error word
    // sweep traces (observers; ring_kernel only), or null.  After every sweep
    // whose index in its phase is a multiple of tr_stride: the ring's bits and
    // slice energies at record [ring][step][tr_rps] (records of a step: slice,
    // cluster, worldline sweeps in that order).  At the start and at each step
    // end the same at [ring][step + 1] (0: the starting state).
    uint32_t *tr_bits;     // [ring][steps][tr_rps][P][nw_max]
    double *tr_E;          // [ring][steps][tr_rps][P]
    uint32_t *tr_end_bits; // [ring][steps + 1][P][nw_max]
    double *tr_end_E;      // [ring][steps + 1][P]
    long long *ring_spin;  // [ring][steps] sum of the ring's spins at each step end
    int tr_stride, tr_rps;
};

__device__ __forceinline__ int phase_count(int P, int ph) {
    if (ph == 0) return (P & 1) ? (P - 1) / 2 : P / 2;
    if (ph == 1) return P / 2;
    return (P & 1) ? 1 : 0;
}
__device__ __forceinline__ int phase_slice(int P, int ph, int c) {
    if (ph == 0) return 2 * c;
    if (ph == 1) return 2 * c + 1;
    return P - 1;
}

// ------------------------------------------------------------------ init
static __global__ void init_spins_kernel(const ProbDev *probs, const RingDev *rings, uint32_t *spins, int P,
                                  uint32_t tag, int nw_max) {
    const RingDev R = rings[blockIdx.x];
    const ProbDev Pd = probs[R.prob];
    const int t = blockIdx.y;
    const int ring_cell_base = R.k * P;
    for (int q = threadIdx.x; q < Pd.nw; q += blockDim.x) {
        const U4 r = philox((uint32_t)(q >> 2), (uint32_t)(ring_cell_base + t), 0u, tag | R.tag_extra, R.key);
        uint32_t w = pick(r, q & 3);
        const int rem = Pd.n - 32 * q;
        if (rem < 32) w &= (1u << rem) - 1u;
        spins[R.spin_off + (long long)t * Pd.nw + q] = w;
    }
}

template <int KIND>
__global__ void init_fields_kernel(const ProbDev *probs, const RingDev *rings, const uint32_t *spins,
                                   float *fields, int P) {
    extern __shared__ uint32_t sS[];
    const RingDev R = rings[blockIdx.x];
    const ProbDev Pd = probs[R.prob];
    const int t = blockIdx.y;
    for (int q = threadIdx.x; q < Pd.nw; q += blockDim.x) sS[q] = spins[R.spin_off + (long long)t * Pd.nw + q];
    __syncthreads();
    float *g = fields + R.field_off + (long long)t * Pd.n;
    for (int i = blockIdx.z * blockDim.x + threadIdx.x; i < Pd.n; i += gridDim.z * blockDim.x)
        g[i] = field_init_one<KIND>(Pd, sS, i);
}

// Drift of the float32 field caches: the largest |g - float64 recompute from
// the same float32 couplings| over every (ring, slice, spin) of the grid
// (blockIdx.x ring, blockIdx.y slice).  Non-negative doubles order as their
// bit patterns, so the maximum is an integer atomicMax.
template <int KIND>
__global__ void field_drift_kernel(const ProbDev *probs, const RingDev *rings, const uint32_t *spins,
                                   const float *fields, int P, unsigned long long *max_bits) {
    extern __shared__ uint32_t sS[];
    const RingDev R = rings[blockIdx.x];
    const ProbDev Pd = probs[R.prob];
    const int t = blockIdx.y;
    for (int q = threadIdx.x; q < Pd.nw; q += blockDim.x) sS[q] = spins[R.spin_off + (long long)t * Pd.nw + q];
    __syncthreads();
    const float *g = fields + R.field_off + (long long)t * Pd.n;
    double mx = 0.0;
    for (int i = blockIdx.z * blockDim.x + threadIdx.x; i < Pd.n; i += gridDim.z * blockDim.x)
        mx = fmax(mx, fabs((double)g[i] - field_exact64<KIND>(Pd, sS, i)));
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) mx = fmax(mx, __shfl_xor_sync(FULL, mx, off));
    if ((threadIdx.x & 31) == 0) atomicMax(max_bits, (unsigned long long)__double_as_longlong(mx));
    (void)P;
}

// ------------------------------------------------------------------ slice sweep
// One warp sweeps slice t of a ring (sqa_annealer.cpp:180-209 with the parity
// schedule of sqa_chi_annealer.cpp:90-122).
template <int KIND>
__device__ __forceinline__ void sweep_slice(const ProbDev &Pd, uint32_t *S, int NP, int t, float *gt, const float *h,
                                            float B, float T4, uint64_t key, uint32_t rng_cell, uint32_t sigma,
                                            uint32_t tag, int lane, unsigned long long &att,
                                            unsigned long long &acc) {
    const int n = Pd.n, nw = Pd.nw;
    uint32_t *St = S + t * nw;
    const int prev = t == 0 ? NP - 1 : t - 1;
    const int next = t + 1 == NP ? 0 : t + 1;
    const uint32_t *Sp = S + prev * nw;
    const uint32_t *Sn = S + next * nw;
    U4 rnd = {0, 0, 0, 0};
    for (int q = 0; q < nw; ++q) {
        if ((q & 3) == 0) rnd = philox((uint32_t)(((q >> 2) << 5) | lane), rng_cell, sigma, tag, key);
        const int i = (q << 5) | lane;
        const bool valid = i < n;
        const uint32_t sw = St[q], pw = Sp[q], nx = Sn[q];
        const int si = ((sw >> lane) & 1u) ? 1 : -1;
        const int nsum = (((pw >> lane) & 1u) ? 1 : -1) + (((nx >> lane) & 1u) ? 1 : -1);
        const int qv = si * nsum;
        const float tro = qv == 0 ? 0.0f : (qv > 0 ? T4 : -T4);
        const float u = u24(pick(rnd, q & 3));
        const float hi = valid ? h[i] : 0.0f;
        att += (unsigned long long)min(32, n - (q << 5));
        uint32_t pending = FULL;
        for (;;) {
            const float gi = valid ? gt[i] : 0.0f;
            const float loc = __fadd_rn(hi, gi);
            const float x = si > 0 ? loc : -loc;
            const bool ok = valid & metropolis_nb24(__fsub_rn(__fmul_rn(x, B), tro), u);
            const uint32_t m = __ballot_sync(FULL, ok) & pending;
            if (!m) break;
            const int j = __ffs(m) - 1;
            const int so = ((sw >> j) & 1u) ? 1 : -1;
            if (lane == 0) St[q] = St[q] ^ (1u << j);
            __syncwarp();
            apply_flip<KIND>(Pd, gt, St, (q << 5) | j, so, lane);
            ++acc;
            pending = j == 31 ? 0u : (FULL << (j + 1));
        }
    }
}

// Slice t of a ring in qanneal's order: visiting position p holds spin
// ord[p]; the uniform belongs to the position.  Block q (positions
// 32q .. 32q+31) waits until slice t - 1 has finished it (the slice
// pipeline, pipe_wait) and publishes its own progress after.  The Trotter neighbours' bits
// of the block's spins are final for this sweep in slice t - 1 and untouched
// in slice t + 1 while slice t holds the block.
template <int KIND>
__device__ __forceinline__ void sweep_slice_ord(const ProbDev &Pd, uint32_t *S, int NP, int t, float *gt,
                                                const float *h, const OrdT *ord, const SlicePipe &pp,
                                                float B, float T4, uint64_t key,
                                                uint32_t rng_cell, uint32_t sigma, uint32_t tag, int lane,
                                                unsigned long long &att, unsigned long long &acc) {
    const int n = Pd.n, nw = Pd.nw;
    uint32_t *St = S + t * nw;
    const int prev = t == 0 ? NP - 1 : t - 1;
    const int next = t + 1 == NP ? 0 : t + 1;
    const uint32_t *Sp = S + prev * nw;
    const uint32_t *Sn = S + next * nw;
    U4 rnd = {0, 0, 0, 0};
    att += (unsigned long long)n;
    for (int q = 0; q < nw; ++q) {
        if ((q & 3) == 0) rnd = philox((uint32_t)(((q >> 2) << 5) | lane), rng_cell, sigma, tag, key);
        if (t > 0) pipe_wait(pp, t - 1, q, lane);
        const int pos = (q << 5) | lane;
        const bool valid = pos < n;
        const int i = valid ? ord[pos] : 0;
        const int si = spin_of(St, i);
        const int qv = si * (spin_of(Sp, i) + spin_of(Sn, i));
        const float tro = qv == 0 ? 0.0f : (qv > 0 ? T4 : -T4);
        const float u = u24(pick(rnd, q & 3));
        const float hi = valid ? h[i] : 0.0f;
        uint32_t pending = FULL;
        for (;;) {
            const float gi = valid ? gt[i] : 0.0f;
            const float loc = __fadd_rn(hi, gi);
            const float x = si > 0 ? loc : -loc;
            const bool ok = valid & metropolis_nb24(__fsub_rn(__fmul_rn(x, B), tro), u);
            const uint32_t m = __ballot_sync(FULL, ok) & pending;
            if (!m) break;
            const int j = __ffs(m) - 1;
            const int jj = __shfl_sync(FULL, i, j);
            const int so = __shfl_sync(FULL, si, j);
            if (lane == 0) St[jj >> 5] ^= 1u << (jj & 31);
            __syncwarp();
            apply_flip<KIND>(Pd, gt, St, jj, so, lane);
            __syncwarp();
            ++acc;
            pending = j == 31 ? 0u : (FULL << (j + 1));
        }
        pipe_publish(pp, t, q, lane);
    }
}

// ------------------------------------------------------------------ SA
struct SAParams {
    const ProbDev *probs;
    const RingDev *rings;   // P == 1 chains
    uint32_t *spins;
    float *fields;
    const float *B;         // [step]: 2 beta
    int steps, spb;
    int smem_fields;
    double *trace;          // [ring][steps]
    double *best_E;         // [ring]
    uint32_t *best_bits;    // [ring][nw_max]
    int nw_max;
    unsigned long long *counters;
    double *mag_trace;      // [ring][steps] magnetisation after each step, or null
    int *best_step;         // [ring] step of the last best improvement (-1: start), or null
    // sweep trace (observers), or null: after every sweep whose index in its
    // step is a multiple of tr_stride, the state and the running energy at
    // record [ring][step][tr_rps]
    uint32_t *tr_bits;      // [ring][steps][tr_rps][nw_max]
    double *tr_E;           // [ring][steps][tr_rps]
    uint32_t *tr_end_bits;  // [ring][steps][nw_max] the state at each step end, or null
    int tr_stride, tr_rps;
};

// Magnetisation sum(s) / n of the current state (metrics.hpp:11-20), exact.
__device__ __forceinline__ void sa_record_mag(const SAParams &p, const uint32_t *S, int n, int nw, int step,
                                              int lane) {
    int up = 0;
    for (int q = lane; q < nw; q += 32) up += __popc(S[q]);
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) up += __shfl_xor_sync(FULL, up, off);
    if (lane == 0) p.mag_trace[(long long)blockIdx.x * p.steps + step] = (double)(2 * up - n) / (double)n;
}

// annealer.cpp:50-67: spins in fixed order, running energy, best copied on
// every new minimum.  One warp per read.
template <int KIND>
__global__ void __launch_bounds__(32) sa_kernel(SAParams p) {
    extern __shared__ __align__(16) unsigned char smem[];
    const RingDev R = p.rings[blockIdx.x];
    const ProbDev Pd = p.probs[R.prob];
    const int lane = threadIdx.x, n = Pd.n, nw = Pd.nw;
    uint32_t *S = reinterpret_cast<uint32_t *>(smem);
    float *h = reinterpret_cast<float *>(S + ((nw + 3) & ~3));
    float *g = p.smem_fields ? h + ((n + 3) & ~3) : p.fields + R.field_off;
    for (int q = lane; q < nw; q += 32) S[q] = p.spins[R.spin_off + q];
    for (int i = lane; i < n; i += 32) {
        h[i] = Pd.h32[i];
        if (p.smem_fields) g[i] = p.fields[R.field_off + i];
    }
    __syncwarp();
    uint32_t *bb = p.best_bits + (long long)blockIdx.x * p.nw_max;
    double E = cell_energy<KIND>(Pd, S, g, h, lane);
    double best = E;
    int bstep = -1;
    for (int q = lane; q < nw; q += 32) bb[q] = S[q];
    unsigned long long att = 0, acc = 0;
    for (int step = 0; step < p.steps; ++step) {
        const float B = p.B[step];
        for (int sw = 0; sw < p.spb; ++sw) {
            const uint32_t sigma = (uint32_t)(step * p.spb + sw);
            U4 rnd = {0, 0, 0, 0};
            for (int q = 0; q < nw; ++q) {
                if ((q & 3) == 0) rnd = philox((uint32_t)(((q >> 2) << 5) | lane), 0u, sigma, DOM_SA, R.key);
                const int i = (q << 5) | lane;
                const bool valid = i < n;
                const uint32_t sword = S[q];
                const int si = ((sword >> lane) & 1u) ? 1 : -1;
                const float u = u24(pick(rnd, q & 3));
                const float hi = valid ? h[i] : 0.0f;
                att += (unsigned long long)min(32, n - (q << 5));
                uint32_t pending = FULL;
                for (;;) {
                    const float gi = valid ? g[i] : 0.0f;
                    const float loc = __fadd_rn(hi, gi);
                    const float x = si > 0 ? loc : -loc;
                    const bool ok = valid & metropolis_nb24(__fmul_rn(x, B), u);
                    const uint32_t m = __ballot_sync(FULL, ok) & pending;
                    if (!m) break;
                    const int j = __ffs(m) - 1;
                    const double xd = si > 0 ? __dadd_rn((double)hi, (double)gi) : -__dadd_rn((double)hi, (double)gi);
                    const double xj = __shfl_sync(FULL, xd, j);
                    const int so = ((sword >> j) & 1u) ? 1 : -1;
                    if (lane == 0) S[q] = S[q] ^ (1u << j);
                    __syncwarp();
                    apply_flip<KIND>(Pd, g, S, (q << 5) | j, so, lane);
                    ++acc;
                    E = __dadd_rn(E, __dmul_rn(-2.0, xj));
                    if (E < best) {
                        best = E;
                        bstep = step;
                        for (int w = lane; w < nw; w += 32) bb[w] = S[w];
                    }
                    pending = j == 31 ? 0u : (FULL << (j + 1));
                }
            }
            if (p.tr_bits && sw % p.tr_stride == 0) {
                const long long rec = ((long long)blockIdx.x * p.steps + step) * p.tr_rps + sw / p.tr_stride;
                for (int q = lane; q < nw; q += 32) p.tr_bits[rec * p.nw_max + q] = S[q];
                if (lane == 0) p.tr_E[rec] = E;
                __syncwarp();
            }
        }
        if (lane == 0) p.trace[(long long)blockIdx.x * p.steps + step] = E;
        if (p.tr_end_bits)
            for (int q = lane; q < nw; q += 32) p.tr_end_bits[((long long)blockIdx.x * p.steps + step) * p.nw_max + q] = S[q];
        if (p.mag_trace) sa_record_mag(p, S, n, nw, step, lane);
    }
    for (int q = lane; q < nw; q += 32) p.spins[R.spin_off + q] = S[q];
    if (p.smem_fields)
        for (int i = lane; i < n; i += 32) p.fields[R.field_off + i] = g[i];
    if (lane == 0) {
        p.best_E[blockIdx.x] = best;
        if (p.best_step) p.best_step[blockIdx.x] = bstep;
        atomicAdd(p.counters + 0, att);
        atomicAdd(p.counters + 1, acc);
    }
}

// ------------------------------------------------------------------ rings
// smem layout: S[P*nw] | h[n] | cellE[P] (double) | wl_sh[W*32] | wl_G[W*32] (double) | flags | fields?
struct RingSmem {
    uint32_t *S;
    float *h;
    double *cellE;
    int *wl_sh;
    double *wl_G;
    int *flag;
    float *g;
    // qanneal's order: the two order rows in shared memory (null: read
    // from global memory), the slice pipeline
    OrdT *obuf[2];
    SlicePipe pipe;
};

__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Imaginary-time bond sum of the ring, sum_{t,i} s_t,i s_t+1,i (whole CTA;
// the total is valid on thread 0).  part: one int per warp.
__device__ __forceinline__ long long ring_bond_total(const uint32_t *S, int NP, int nw, int n, int *part, int W) {
    int b = 0;
    for (int idx = threadIdx.x; idx < NP * nw; idx += blockDim.x) {
        const int t = idx / nw, q = idx - t * nw;
        const int tn = t + 1 == NP ? 0 : t + 1;
        const int rem = n - 32 * q;
        const uint32_t vm = rem >= 32 ? FULL : ((1u << rem) - 1u);
        b += 2 * __popc(~(S[idx] ^ S[tn * nw + q]) & vm) - __popc(vm);
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) b += __shfl_xor_sync(FULL, b, off);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = b;
    __syncthreads();
    long long tb = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < W; ++w) tb += part[w];
    __syncthreads();
    return tb;
}

__device__ __forceinline__ void record_bond_sample(const RingParams &p, const uint32_t *S, int NP, int nw, int n,
                                                   int *part, int W, int step, int j) {
    const long long tb = ring_bond_total(S, NP, nw, n, part, W);
    if (threadIdx.x == 0)
        p.bsamp[(long long)blockIdx.x * p.bstride + (long long)(step - p.step0) * (p.spb + p.cls) + j] = tb;
}

// qanneal's order in shared memory: two order rows unless they are read from
// global memory, plus the slices' progress counters and the abort flag.
__host__ __device__ inline size_t ring_order_bytes(int P, int n, bool rows_in_smem = true) {
    return (rows_in_smem ? 2 * ord_row_bytes(n) : 0) + pipe_bytes(P);
}

// qanneal's order for a launch, run before it on its stream: row k of step s
// of ring b is the visiting order of the k-th ordered sweep of that step (its
// slice sweeps, cluster sweeps when with_cls, worldline sweeps), keyed like
// the sweep (ring key, slot, sweep index, domain tag).  One CTA per row
// (grid-stride loop); the keys and bucket counters in shared memory, or in
// `scratch` (scratch_bytes per CTA) when they do not fit.
static __global__ void __launch_bounds__(256) order_fill_kernel(RingParams p, int n_rings, int with_cls,
                                                         unsigned char *scratch, long long scratch_bytes) {
    extern __shared__ __align__(16) unsigned char osm[];
    const int per = p.ord_per_step, cl = with_cls ? p.cls : 0;
    const long long per_ring = (long long)(p.step1 - p.step0) * per, total = per_ring * n_rings;
    unsigned char *base = scratch ? scratch + (long long)blockIdx.x * scratch_bytes : osm;
    for (long long o = blockIdx.x; o < total; o += gridDim.x) {
        const int b = (int)(o / per_ring);
        const long long rem = o - (long long)b * per_ring;
        const int step = p.step0 + (int)(rem / per), k = (int)(rem % per);
        const RingDev R = p.rings[b];
        const int n = p.probs[R.prob].n;
        const int slot = p.slot ? p.slot[b] : R.k;
        uint32_t tag, sigma;
        if (k < p.spb) {
            tag = p.slice_tag | R.tag_extra;
            sigma = (uint32_t)(step * p.spb + k);
        } else if (k < p.spb + cl) {
            tag = DOM_CSPIN;
            sigma = (uint32_t)(step * p.cls + (k - p.spb));
        } else {
            tag = DOM_WORLD;
            sigma = (uint32_t)(step * p.wls + (k - p.spb - cl));
        }
        build_sweep_order(R.key, (uint32_t)slot, sigma, tag, n, reinterpret_cast<unsigned long long *>(base),
                          reinterpret_cast<int *>(base + order_keys_bytes(n)),
                          p.ordg + (long long)b * p.ord_ring + rem * p.ord_stride);
    }
}

// Shared or scratch bytes of one order_fill_kernel CTA.
__host__ __device__ inline size_t order_fill_bytes(int n) { return order_keys_bytes(n) + order_cnt_bytes(n); }

__host__ __device__ inline size_t ring_smem_bytes(int P, int n, int W, bool fields, bool ref_order = false,
                                                 bool order_in_smem = true) {
    const int nw = (n + 31) / 32;
    size_t b = align_up((size_t)P * nw * 4, 16);
    b += align_up((size_t)n * 4, 16);
    b += align_up((size_t)P * 8, 16);
    b += align_up((size_t)W * 32 * 4, 16);
    b += align_up((size_t)W * 32 * 8, 16);
    b += 16;
    if (ref_order) b += ring_order_bytes(P, n, order_in_smem);
    if (fields) b += (size_t)P * n * 4;
    return b;
}

// Cluster move of spin i along imaginary time (sqa_annealer.cpp:215-288,
// sqa_parallel_tempering.cpp:224-278), one warp.  Seed slice and acceptance
// uniform from philox(0, ring, sweep, CSPIN | i << 8); bond b (slices b and
// b+1) joins when both carry the seed's spin and its uniform, word b & 3 of
// philox(b >> 2, ring, sweep, CBOND | i << 8), is below JP.  The cluster is
// the run of joined bonds through the seed (every slice when the run closes
// the ring); y = x B - k T4/2 with x = h s0 |C| + sum_{t in C} s0 g_t (warp
// order over t = lane, lane + 32) and k the seed spin times the two spins just
// outside the cluster.  Lane t holds slices t and t + 32 (P <= 64).
template <int KIND>
__device__ __forceinline__ void cluster_move(const ProbDev &Pd, uint32_t *S, float *gbase, const float *h, int NP,
                                             int i, uint32_t ring, uint32_t sigma, float B, float T4, float JP,
                                             uint64_t key, int lane) {
    const int n = Pd.n, nw = Pd.nw;
    const uint32_t c3s = DOM_CSPIN | ((uint32_t)i << 8), c3b = DOM_CBOND | ((uint32_t)i << 8);
    const U4 w = philox(0u, ring, sigma, c3s, key);
    const int t0 = (int)(((unsigned long long)(w.x >> 8) * (unsigned long long)NP) >> 24);
    const float u = u24(w.y);
    const int q = i >> 5;
    const uint32_t bit = 1u << (i & 31);
    const int ta = lane, tb = lane + 32;
    const bool upa = ta < NP && (S[ta * nw + q] & bit), upb = tb < NP && (S[tb * nw + q] & bit);
    const unsigned long long Wi =
        (unsigned long long)__ballot_sync(FULL, upa) | ((unsigned long long)__ballot_sync(FULL, upb) << 32);
    const unsigned long long pmask = NP == 64 ? ~0ull : ((1ull << NP) - 1ull);
    const bool s0up = (Wi >> t0) & 1ull;
    const int s0 = s0up ? 1 : -1;
    const unsigned long long same = (s0up ? Wi : ~Wi) & pmask;
    // bond uniforms: lane l draws bonds 4l .. 4l+3; bond b takes its word from lane b >> 2
    U4 bw = {0u, 0u, 0u, 0u};
    if (4 * lane < NP) bw = philox((uint32_t)lane, ring, sigma, c3b, key);
    bool act[2];
#pragma unroll
    for (int h2 = 0; h2 < 2; ++h2) {
        const int b = lane + 32 * h2;
        const int src = b >> 2;
        const uint32_t x0 = __shfl_sync(FULL, bw.x, src), x1 = __shfl_sync(FULL, bw.y, src);
        const uint32_t x2 = __shfl_sync(FULL, bw.z, src), x3 = __shfl_sync(FULL, bw.w, src);
        const uint32_t wb = (b & 3) == 0 ? x0 : ((b & 3) == 1 ? x1 : ((b & 3) == 2 ? x2 : x3));
        const int b1 = b + 1 == NP ? 0 : b + 1;
        act[h2] = b < NP && ((same >> b) & 1ull) && ((same >> b1) & 1ull) && u01(wb) < JP;
    }
    const unsigned long long A0 =
        (unsigned long long)__ballot_sync(FULL, act[0]) | ((unsigned long long)__ballot_sync(FULL, act[1]) << 32);
    bool all = (A0 & pmask) == pmask;
    int r = 0, l = 0;
    if (!all) {
        const unsigned long long A = t0 == 0 ? A0 : (((A0 >> t0) | (A0 << (NP - t0))) & pmask);
        r = __ffsll((long long)~A) - 1;                         // joined bonds right of the seed
        l = NP - 1 - (63 - __clzll((long long)(~A & pmask)));  // joined bonds left of it
        all = l + r + 1 >= NP;
    }
    unsigned long long Cm = pmask;
    int kb = 0, size = NP;
    if (!all) {
        unsigned long long Cr = (r >= 63 ? ~0ull : ((2ull << r) - 1ull));
        if (l > 0) Cr |= pmask & ~((1ull << (NP - l)) - 1ull);
        Cr &= pmask;
        Cm = t0 == 0 ? Cr : (((Cr << t0) | (Cr >> (NP - t0))) & pmask);
        const int tl = (t0 - l - 1 + NP) % NP, tr = (t0 + r + 1) % NP;
        kb = s0 * ((((Wi >> tl) & 1ull) ? 1 : -1) + (((Wi >> tr) & 1ull) ? 1 : -1));
        size = l + r + 1;
    }
    double acc = 0.0;
    if (ta < NP && ((Cm >> ta) & 1ull)) acc = __dadd_rn(acc, (double)s0 * (double)gbase[(long long)ta * n + i]);
    if (tb < NP && ((Cm >> tb) & 1ull)) acc = __dadd_rn(acc, (double)s0 * (double)gbase[(long long)tb * n + i]);
    const double G = warp_sum_d(acc);
    const float x = __double2float_rn(__dadd_rn(__dmul_rn((double)h[i], (double)(s0 * size)), G));
    const float y = __fsub_rn(__fmul_rn(x, B), __fmul_rn(__int2float_rn(kb), __fmul_rn(0.5f, T4)));
    if (!metropolis_nb24(y, u)) return;
    if (ta < NP && ((Cm >> ta) & 1ull)) S[ta * nw + q] ^= bit;
    if (tb < NP && ((Cm >> tb) & 1ull)) S[tb * nw + q] ^= bit;
    __syncwarp();
    for (unsigned long long c = Cm; c; c &= c - 1ull) {
        const int t = __ffsll((long long)c) - 1;
        apply_flip<KIND>(Pd, gbase + (long long)t * n, S + t * nw, i, s0, lane);
    }
    __syncwarp();
}

// One trace record of a ring: the slice energies (as the step-end scan
// computes them) and the bits of every slice.  Whole CTA; ends with a barrier.
template <int KIND>
__device__ __forceinline__ void ring_trace(const RingParams &p, const ProbDev &Pd, const RingSmem &sm,
                                           const float *gbase, int NP, int nw, int n, int W, int warp, int lane,
                                           uint32_t *bits, double *E) {
    for (int t = warp; t < NP; t += W) {
        const double e = cell_energy<KIND>(Pd, sm.S + t * nw, gbase + (long long)t * n, sm.h, lane);
        if (lane == 0) E[t] = e;
    }
    for (int idx = threadIdx.x; idx < NP * nw; idx += blockDim.x) {
        const int t = idx / nw, q = idx - t * nw;
        bits[(long long)t * p.nw_max + q] = sm.S[idx];
    }
    __syncthreads();
}

template <int KIND>
__global__ void __launch_bounds__(1024, 1) ring_kernel(RingParams p) {
    extern __shared__ __align__(16) unsigned char smem[];
    const RingDev R = p.rings[blockIdx.x];
    const ProbDev Pd = p.probs[R.prob];
    const int NP = p.P, W = p.W;
    const int n = Pd.n, nw = Pd.nw;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    RingSmem sm;
    unsigned char *ptr = smem;
    sm.S = reinterpret_cast<uint32_t *>(ptr); ptr += align_up((size_t)NP * nw * 4, 16);
    sm.h = reinterpret_cast<float *>(ptr); ptr += align_up((size_t)n * 4, 16);
    sm.cellE = reinterpret_cast<double *>(ptr); ptr += align_up((size_t)NP * 8, 16);
    sm.wl_sh = reinterpret_cast<int *>(ptr); ptr += align_up((size_t)W * 32 * 4, 16);
    sm.wl_G = reinterpret_cast<double *>(ptr); ptr += align_up((size_t)W * 32 * 8, 16);
    sm.flag = reinterpret_cast<int *>(ptr); ptr += 16;
    sm.obuf[0] = sm.obuf[1] = nullptr;
    if (p.ref_order) {
        if (p.ord_in_smem) {
            sm.obuf[0] = reinterpret_cast<OrdT *>(ptr); ptr += ord_row_bytes(n);
            sm.obuf[1] = reinterpret_cast<OrdT *>(ptr); ptr += ord_row_bytes(n);
        }
        sm.pipe = pipe_open(ptr, NP, p.counters + 4); ptr += pipe_bytes(NP);
    }
    float *gbase = p.smem_fields ? reinterpret_cast<float *>(ptr) : p.fields + R.field_off;

    for (int idx = threadIdx.x; idx < NP * nw; idx += blockDim.x) sm.S[idx] = p.spins[R.spin_off + idx];
    for (int i = threadIdx.x; i < n; i += blockDim.x) sm.h[i] = Pd.h32[i];
    if (p.smem_fields)
        for (long long idx = threadIdx.x; idx < (long long)NP * n; idx += blockDim.x) gbase[idx] = p.fields[R.field_off + idx];
    __syncthreads();

    const int slot = p.slot ? p.slot[blockIdx.x] : R.k;
    OrderFeed feed = feed_open(sm.obuf[0], sm.obuf[1], p.ref_order ? p.ordg + blockIdx.x * p.ord_ring : nullptr,
                               p.ord_stride, n, p.ref_order ? (p.step1 - p.step0) * p.ord_per_step : 0);
    unsigned long long att_s = 0, acc_s = 0, att_w = 0, acc_w = 0;
    double bestE = p.best_E[blockIdx.x];
    int bestStep = p.best_step[blockIdx.x];
    // trace records: slice sweeps first, then cluster, then worldline sweeps
    const int tr_s = p.tr_bits ? (p.spb + p.tr_stride - 1) / p.tr_stride : 0;
    const int tr_c = p.tr_bits ? (p.cls + p.tr_stride - 1) / p.tr_stride : 0;
    auto trace_rec = [&](int step, int idx) {
        const long long rec = ((long long)blockIdx.x * p.steps_total + step) * p.tr_rps + idx;
        ring_trace<KIND>(p, Pd, sm, gbase, NP, nw, n, W, warp, lane, p.tr_bits + rec * NP * p.nw_max,
                         p.tr_E + rec * NP);
    };
    auto trace_end = [&](int step) {  // the state after `step` (step -1: the start)
        const long long rec = (long long)blockIdx.x * (p.steps_total + 1) + step + 1;
        ring_trace<KIND>(p, Pd, sm, gbase, NP, nw, n, W, warp, lane, p.tr_end_bits + rec * NP * p.nw_max,
                         p.tr_end_E + rec * NP);
    };
    if (p.tr_end_bits && p.step0 == 0) trace_end(-1);

    for (int step = p.step0 - (p.init_scan ? 1 : 0); step < p.step1; ++step) {
        // step -1 (init_scan) only scores the starting state
        const int spb = step >= 0 ? p.spb : 0, wls = step >= 0 ? p.wls : 0;
        const int si_tab = R.sched + (p.per_slot_sched ? slot + max(step, 0) * p.slot_step : max(step, 0));
        const float B = p.B[si_tab], T4 = p.T4[si_tab];
        for (int sw = 0; sw < spb; ++sw) {
            const uint32_t sigma = (uint32_t)(step * p.spb + sw);
            if (p.ref_order) {
                const uint32_t tag = p.slice_tag | R.tag_extra;
                pipe_reset(sm.pipe, NP);
                const OrdT *ord = feed_take(feed);
                for (int t = warp; t < NP; t += W)
                    sweep_slice_ord<KIND>(Pd, sm.S, NP, t, gbase + (long long)t * n, sm.h, ord, sm.pipe, B, T4,
                                          R.key, (uint32_t)(slot * NP + t), sigma, tag, lane, att_s, acc_s);
                __syncthreads();
            } else {
                for (int ph = 0; ph < 3; ++ph) {
                    const int cnt = phase_count(NP, ph);
                    for (int c = warp; c < cnt; c += W) {
                        const int t = phase_slice(NP, ph, c);
                        sweep_slice<KIND>(Pd, sm.S, NP, t, gbase + (long long)t * n, sm.h, B, T4, R.key,
                                          (uint32_t)(slot * NP + t), sigma, p.slice_tag | R.tag_extra, lane, att_s,
                                          acc_s);
                    }
                    if (cnt) __syncthreads();
                }
            }
            if (p.mag) {
                long long ps = 0;
                for (int idx = threadIdx.x; idx < NP * nw; idx += blockDim.x) ps += __popc(sm.S[idx]);
                ps = warp_sum_ll(ps);
                if (lane == 0) sm.wl_sh[warp] = (int)ps;
                __syncthreads();
                if (threadIdx.x == 0) {
                    long long tot = 0;
                    for (int w = 0; w < W; ++w) tot += sm.wl_sh[w];
                    p.mag[(long long)blockIdx.x * (p.steps_total * p.spb) + sigma] = (int)(2 * tot - (long long)NP * n);
                }
                __syncthreads();
            }
            if (p.bsamp) record_bond_sample(p, sm.S, NP, nw, n, sm.wl_sh, W, step, sw);
            if (p.tr_bits && sw % p.tr_stride == 0) trace_rec(step, sw / p.tr_stride);
        }
        // cluster sweeps: one warp, spins in the sweep's visiting order
        // (qanneal's order) or ascending
        const int cls = step >= 0 ? p.cls : 0;
        for (int sw = 0; sw < cls; ++sw) {
            const uint32_t sigma = (uint32_t)(step * p.cls + sw);
            const OrdT *cord = p.ref_order ? feed_take(feed) : nullptr;
            if (warp == 0) {
                const float JPv = p.JP[si_tab];
                for (int pos = 0; pos < n; ++pos)
                    cluster_move<KIND>(Pd, sm.S, gbase, sm.h, NP, p.ref_order ? (int)cord[pos] : pos, (uint32_t)slot,
                                       sigma, B, T4, JPv, R.key, lane);
            }
            __syncthreads();
            if (p.bsamp) record_bond_sample(p, sm.S, NP, nw, n, sm.wl_sh, W, step, p.spb + sw);
            if (p.tr_bits && sw % p.tr_stride == 0) trace_rec(step, tr_s + sw / p.tr_stride);
        }
        for (int sw = 0; sw < wls; ++sw) {
            const uint32_t sigma = (uint32_t)(step * p.wls + sw);
            // visiting position (q << 5) | lane holds spin ord[position]
            // (qanneal's order) or spin position (ascending)
            const OrdT *word = p.ref_order ? feed_take(feed) : nullptr;
            U4 rnd = {0, 0, 0, 0};
            for (int q = 0; q < nw; ++q) {
                if ((q & 3) == 0)
                    rnd = philox((uint32_t)(((q >> 2) << 5) | lane), (uint32_t)slot, sigma, DOM_WORLD, R.key);
                const int pos = (q << 5) | lane;
                const bool valid = pos < n;
                const int i = !valid ? 0 : (p.ref_order ? (int)word[pos] : pos);
                const float u = u24(pick(rnd, q & 3));
                const float hi = valid ? sm.h[i] : 0.0f;
                if (threadIdx.x == 0) att_w += (unsigned long long)min(32, n - (q << 5));
                uint32_t pending = FULL;
                for (;;) {
                    int sh = 0;
                    double G = 0.0;
                    if (valid)
                        for (int t = warp; t < NP; t += W) {
                            const int st = spin_of(sm.S + t * nw, i);
                            const double gv = (double)gbase[(long long)t * n + i];
                            sh += st;
                            G = __dadd_rn(G, st > 0 ? gv : -gv);
                        }
                    sm.wl_sh[warp * 32 + lane] = sh;
                    sm.wl_G[warp * 32 + lane] = G;
                    __syncthreads();
                    int Sh = 0;
                    double Gt = 0.0;
                    for (int w = 0; w < W; ++w) {
                        Sh += sm.wl_sh[w * 32 + lane];
                        Gt = __dadd_rn(Gt, sm.wl_G[w * 32 + lane]);
                    }
                    __syncthreads();
                    const float x = valid ? __double2float_rn(__dadd_rn(__dmul_rn((double)hi, (double)Sh), Gt)) : 0.0f;
                    const bool ok = valid & metropolis_nb24(__fmul_rn(x, B), u);
                    const uint32_t m = __ballot_sync(FULL, ok) & pending;
                    if (!m) break;
                    const int j = __ffs(m) - 1;
                    const int jj = __shfl_sync(FULL, i, j);
                    for (int t = warp; t < NP; t += W) {
                        uint32_t *St = sm.S + t * nw;
                        const int so = spin_of(St, jj);
                        __syncwarp();
                        if (lane == 0) St[jj >> 5] = St[jj >> 5] ^ (1u << (jj & 31));
                        __syncwarp();
                        apply_flip<KIND>(Pd, gbase + (long long)t * n, St, jj, so, lane);
                    }
                    __syncthreads();
                    if (threadIdx.x == 0) ++acc_w;
                    pending = j == 31 ? 0u : (FULL << (j + 1));
                }
            }
            if (p.tr_bits && sw % p.tr_stride == 0) trace_rec(step, tr_s + tr_c + sw / p.tr_stride);
        }
        // ---- step end: energy of every slice, ring sum, best (sqa_annealer.cpp:455-469)
        if (KIND == K_HUBO && Pd.trec) {
            // slices t and t + W of this warp in one pass over the term records
            for (int t = warp; t < NP; t += 2 * W) {
                const int t2 = t + W < NP ? t + W : t;
                double Ea, Eb;
                hubo_energy2(Pd, sm.S + t * nw, sm.S + t2 * nw, sm.h, lane, &Ea, &Eb);
                if (lane == 0) {
                    sm.cellE[t] = Ea;
                    if (t2 != t) sm.cellE[t2] = Eb;
                }
            }
        } else {
            for (int t = warp; t < NP; t += W) {
                const double E = cell_energy<KIND>(Pd, sm.S + t * nw, gbase + (long long)t * n, sm.h, lane);
                if (lane == 0) sm.cellE[t] = E;
            }
        }
        if (p.ring_bond) {
            long long b = 0;
            for (int idx = threadIdx.x; idx < NP * nw; idx += blockDim.x) {
                const int t = idx / nw, q = idx - t * nw;
                const int tn = t + 1 == NP ? 0 : t + 1;
                uint32_t x = ~(sm.S[idx] ^ sm.S[tn * nw + q]);
                const int rem = n - 32 * q;
                if (rem < 32) x &= (1u << rem) - 1u;
                const int valid_bits = min(32, rem);
                b += 2 * __popc(x) - valid_bits;
            }
            b = warp_sum_ll(b);
            if (lane == 0) sm.wl_sh[warp] = (int)b;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double sum = 0.0, emin = __longlong_as_double(0x7ff0000000000000LL);
            int tmin = 0;
            for (int t = 0; t < NP; ++t) {
                const double E = sm.cellE[t];
                sum = __dadd_rn(sum, E);
                if (E < emin) { emin = E; tmin = t; }
            }
            const long long ro = (long long)blockIdx.x * p.rec_stride + p.rec_base + step;
            if (p.ring_sum) p.ring_sum[ro] = sum;
            if (p.ring_min) p.ring_min[ro] = emin;
            if (p.ring_bond) {
                long long tb = 0;
                for (int w = 0; w < W; ++w) tb += sm.wl_sh[w];
                p.ring_bond[ro] = tb;
            }
            sm.flag[0] = -1;
            sm.flag[1] = tmin;
            if (emin < bestE) {
                bestE = emin;
                bestStep = step;
                sm.flag[0] = tmin;
            }
        }
        __syncthreads();
        const int tb = sm.flag[0];
        if (tb >= 0) {
            bestE = sm.cellE[tb];
            bestStep = step;
            if (threadIdx.x == 0 && p.best_slot) p.best_slot[blockIdx.x] = slot;
            for (int q = threadIdx.x; q < nw; q += blockDim.x)
                p.best_bits[(long long)blockIdx.x * p.nw_max + q] = sm.S[tb * nw + q];
        }
        if (p.final_bits && step == p.steps_total - 1)
            for (int q = threadIdx.x; q < nw; q += blockDim.x)
                p.final_bits[(long long)blockIdx.x * p.nw_max + q] = sm.S[sm.flag[1] * nw + q];
        __syncthreads();
        if (p.tr_end_bits && step >= 0) trace_end(step);
        if (p.ring_spin && step >= 0) {
            long long c = 0;
            for (int idx = threadIdx.x; idx < NP * nw; idx += blockDim.x) {
                const int q = idx % nw, rem = n - 32 * q;
                uint32_t x = sm.S[idx];
                if (rem < 32) x &= (1u << rem) - 1u;
                c += 2 * __popc(x) - min(32, rem);
            }
            c = warp_sum_ll(c);
            if (lane == 0) sm.wl_sh[warp] = (int)c;
            __syncthreads();
            if (threadIdx.x == 0) {
                long long tot = 0;
                for (int w = 0; w < W; ++w) tot += sm.wl_sh[w];
                p.ring_spin[(long long)blockIdx.x * p.steps_total + step] = tot;
            }
            __syncthreads();
        }
    }
    for (int idx = threadIdx.x; idx < NP * nw; idx += blockDim.x) p.spins[R.spin_off + idx] = sm.S[idx];
    if (p.smem_fields)
        for (long long idx = threadIdx.x; idx < (long long)NP * n; idx += blockDim.x) p.fields[R.field_off + idx] = gbase[idx];
    if (lane == 0) {
        atomicAdd(p.counters + 0, att_s);
        atomicAdd(p.counters + 1, acc_s);
    }
    if (threadIdx.x == 0) {
        atomicAdd(p.counters + 2, att_w);
        atomicAdd(p.counters + 3, acc_w);
        p.best_E[blockIdx.x] = bestE;
        p.best_step[blockIdx.x] = bestStep;
    }
}

// ------------------------------------------------------------------ exact energies
// Float64 energies of bit-packed states from the original coefficients.
template <int KIND>
__global__ void exact_energy_kernel(const ProbDev *probs, const int *prob_of, const uint32_t *bits, int nw_max,
                                    double *out, int count) {
    extern __shared__ uint32_t sS[];
    const int idx = blockIdx.x;
    if (idx >= count) return;
    const ProbDev Pd = probs[prob_of[idx]];
    for (int q = threadIdx.x; q < Pd.nw; q += 32) sS[q] = bits[(long long)idx * nw_max + q];
    __syncwarp();
    const double E = exact_energy<KIND>(Pd, sS, threadIdx.x);
    if (threadIdx.x == 0) out[idx] = E;
}

}  // namespace qa
