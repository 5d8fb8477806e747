// qa_pm1.cuh -- Trotter-ring sweep kernel specialised for dense couplings in
// {-1, +1} (the Sherrington-Kirkpatrick instances of the benchmark set).
//
// Same replay semantics as ring_kernel (qa_kernels.cuh), different data path:
//  * J is bit-packed (1 bit per coupling) and staged once per CTA in shared
//    memory: Jw[q*n + m] holds bits J[m][32q .. 32q+31] (J is symmetric, so it
//    is also column m).  n = 512 takes 32 KB.
//  * Local fields are exact int32 (g = J.s is an integer) in shared memory.
//  * A block of 32 spins is resolved as in ring_kernel, but the fields of the
//    whole slice are updated once per block, for all flips F of the block
//    together: g[m] += 2|F| - 4 popc(~(Jw[q*n+m] ^ s_old) & F), i.e. a few
//    integer ops per field instead of one update per flip.
//  * Worldline moves (sqa_annealer.cpp:294-315) are evaluated speculatively for
//    all remaining spins at once (thread per spin, sum over the P slices),
//    then the first accepted spin in sweep order is applied and the pass
//    repeats from the next spin: the sequential sweep, with one CTA barrier
//    pair per accepted move instead of per spin.
#pragma once
#include "qa_kernels.cuh"

namespace qa {

__host__ __device__ inline size_t pm1_smem_bytes(int P, int n) {
    const int nw = (n + 31) / 32;
    size_t b = align_up((size_t)nw * n * 4, 16);  // Jw
    b += align_up((size_t)P * nw * 4, 16);         // S
    b += align_up((size_t)n * 4, 16);              // h
    b += align_up((size_t)P * n * 4, 16);          // G
    b += align_up((size_t)P * 8, 16);              // cellE
    b += align_up((size_t)32 * 4, 16);             // per-block accept masks (nw <= 32)
    b += 32;                                       // flags + per-warp partials
    return b + 128;
}

__device__ __forceinline__ int warp_sum_i(int v) {
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) v += __shfl_xor_sync(FULL, v, off);
    return v;
}

// One warp sweeps slice t.
__device__ __forceinline__ void pm1_sweep_slice(const uint32_t *Jw, uint32_t *S, int *G, const float *h, int n, int nw,
                                                int NP, int t, float B, float T4, uint64_t key, uint32_t rng_cell,
                                                uint32_t sigma, uint32_t tag, int lane, unsigned long long &att,
                                                unsigned long long &acc) {
    uint32_t *St = S + t * nw;
    const uint32_t *Sp = S + (t == 0 ? NP - 1 : t - 1) * nw;
    const uint32_t *Sn = S + (t + 1 == NP ? 0 : t + 1) * nw;
    int *Gt = G + t * n;
    U4 rnd = {0, 0, 0, 0};
    for (int q = 0; q < nw; ++q) {
        if ((q & 3) == 0) rnd = philox((uint32_t)(((q >> 2) << 5) | lane), rng_cell, sigma, tag, key);
        const int i = (q << 5) | lane;
        const bool valid = i < n;
        const uint32_t sw = St[q], pw = Sp[q], nx = Sn[q];
        const int si = ((sw >> lane) & 1u) ? 1 : -1;
        const int qv = si * ((((pw >> lane) & 1u) ? 1 : -1) + (((nx >> lane) & 1u) ? 1 : -1));
        const float tro = qv == 0 ? 0.0f : (qv > 0 ? T4 : -T4);
        const float u = u01(pick(rnd, q & 3));
        const float hi = valid ? h[i] : 0.0f;
        const int gi = valid ? Gt[i] : 0;
        att += (unsigned long long)min(32, n - (q << 5));
        float loc = __fadd_rn(hi, __int2float_rn(gi));
        bool ok = valid && metropolis(__fsub_rn(__fmul_rn(si > 0 ? loc : -loc, B), tro), u);
        uint32_t m = __ballot_sync(FULL, ok);
        if (m == 0) continue;
        // resolve the block in spin order; gk is this lane's field with the
        // block's earlier flips applied
        const uint32_t jd = valid ? Jw[q * n + i] : 0u;
        uint32_t F = 0;
        int gk = gi;
        do {
            const int j = __ffs(m) - 1;
            F |= 1u << j;
            if (lane != j) gk += (((sw ^ jd) >> j) & 1u) ? 2 : -2;
            const uint32_t pending = j == 31 ? 0u : (FULL << (j + 1));
            loc = __fadd_rn(hi, __int2float_rn(gk));
            ok = valid && metropolis(__fsub_rn(__fmul_rn(si > 0 ? loc : -loc, B), tro), u);
            m = __ballot_sync(FULL, ok) & pending;
            ++acc;
        } while (m);
        if (lane == 0) St[q] = sw ^ F;
        for (int qq = 0; qq < nw; ++qq) {
            const int mm = (qq << 5) | lane;
            if (mm < n) {
                const uint32_t Fm = qq == q ? (F & ~(1u << lane)) : F;
                const int agree = __popc(~(Jw[q * n + mm] ^ sw) & Fm);
                Gt[mm] += 2 * __popc(Fm) - 4 * agree;
            }
        }
        __syncwarp();
    }
}

__global__ void __launch_bounds__(1024, 1) ring_pm1_kernel(RingParams p) {
    extern __shared__ __align__(16) unsigned char smem[];
    const RingDev R = p.rings[blockIdx.x];
    const ProbDev Pd = p.probs[R.prob];
    const int NP = p.P, W = p.W, n = Pd.n, nw = Pd.nw;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char *ptr = smem;
    uint32_t *Jw = reinterpret_cast<uint32_t *>(ptr); ptr += align_up((size_t)nw * n * 4, 16);
    uint32_t *S = reinterpret_cast<uint32_t *>(ptr); ptr += align_up((size_t)NP * nw * 4, 16);
    float *h = reinterpret_cast<float *>(ptr); ptr += align_up((size_t)n * 4, 16);
    int *G = reinterpret_cast<int *>(ptr); ptr += align_up((size_t)NP * n * 4, 16);
    double *cellE = reinterpret_cast<double *>(ptr); ptr += align_up((size_t)NP * 8, 16);
    uint32_t *mask = reinterpret_cast<uint32_t *>(ptr); ptr += align_up((size_t)32 * 4, 16);
    int *flag = reinterpret_cast<int *>(ptr); ptr += 32;
    int *wpart = reinterpret_cast<int *>(ptr);  // [32]

    for (int idx = threadIdx.x; idx < nw * n; idx += blockDim.x) Jw[idx] = Pd.Jw[idx];
    for (int idx = threadIdx.x; idx < NP * nw; idx += blockDim.x) S[idx] = p.spins[R.spin_off + idx];
    for (int i = threadIdx.x; i < n; i += blockDim.x) h[i] = Pd.h32[i];
    int *Gg = reinterpret_cast<int *>(p.fields) + R.field_off;
    __syncthreads();
    if (p.init_fields) {
        // g_m = sum_{j != m} J_mj s_j by popcount over the packed rows
        for (int idx = threadIdx.x; idx < NP * n; idx += blockDim.x) {
            const int t = idx / n, mm = idx - t * n;
            int g = 0;
            for (int q = 0; q < nw; ++q) {
                const int rem = n - 32 * q;
                uint32_t vm = rem >= 32 ? FULL : ((1u << rem) - 1u);
                if (q == (mm >> 5)) vm &= ~(1u << (mm & 31));
                g += 2 * __popc(~(Jw[q * n + mm] ^ S[t * nw + q]) & vm) - __popc(vm);
            }
            G[idx] = g;
        }
    } else {
        for (int idx = threadIdx.x; idx < NP * n; idx += blockDim.x) G[idx] = Gg[idx];
    }
    __syncthreads();

    const int slot = p.slot ? p.slot[blockIdx.x] : R.k;
    unsigned long long att_s = 0, acc_s = 0, att_w = 0, acc_w = 0;
    double bestE = p.best_E[blockIdx.x];
    int bestStep = p.best_step[blockIdx.x];

    for (int step = p.step0; step < p.step1; ++step) {
        const int si_tab = R.sched + (p.per_slot_sched ? slot : step);
        const float B = p.B[si_tab], T4 = p.T4[si_tab];
        for (int sw = 0; sw < p.spb; ++sw) {
            const uint32_t sigma = (uint32_t)(step * p.spb + sw);
            for (int ph = 0; ph < 3; ++ph) {
                const int cnt = phase_count(NP, ph);
                for (int c = warp; c < cnt; c += W) {
                    const int t = phase_slice(NP, ph, c);
                    pm1_sweep_slice(Jw, S, G, h, n, nw, NP, t, B, T4, R.key, (uint32_t)(slot * NP + t), sigma,
                                    p.slice_tag, lane, att_s, acc_s);
                }
                if (cnt) __syncthreads();
            }
            if (p.mag) {
                int ps = 0;
                for (int idx = threadIdx.x; idx < NP * nw; idx += blockDim.x) ps += __popc(S[idx]);
                ps = warp_sum_i(ps);
                if (lane == 0) wpart[warp] = ps;
                __syncthreads();
                if (threadIdx.x == 0) {
                    long long tot = 0;
                    for (int w = 0; w < W; ++w) tot += wpart[w];
                    p.mag[(long long)blockIdx.x * (p.steps_total * p.spb) + sigma] = (int)(2 * tot - (long long)NP * n);
                }
                __syncthreads();
            }
        }
        for (int sw = 0; sw < p.wls; ++sw) {
            const uint32_t sigma = (uint32_t)(step * p.wls + sw);
            int start = 0;
            for (;;) {
                const int q0 = start >> 5;
                for (int q = q0 + warp; q < nw; q += W) {
                    const int i = (q << 5) | lane;
                    int sh = 0, gs = 0;
                    if (i < n)
                        for (int t = 0; t < NP; ++t) {
                            const int st = ((S[t * nw + q] >> lane) & 1u) ? 1 : -1;
                            sh += st;
                            gs += st * G[t * n + i];
                        }
                    const float hi = i < n ? h[i] : 0.0f;
                    const float x = __double2float_rn(__dadd_rn(__dmul_rn((double)hi, (double)sh), (double)gs));
                    const U4 r = philox((uint32_t)(((q >> 2) << 5) | lane), (uint32_t)slot, sigma, DOM_WORLD, R.key);
                    const bool ok = i < n && i >= start && metropolis(__fmul_rn(x, B), u01(pick(r, q & 3)));
                    const uint32_t m = __ballot_sync(FULL, ok);
                    if (lane == 0) mask[q] = m;
                }
                __syncthreads();
                int first = -1;
                for (int q = q0; q < nw; ++q) {
                    const uint32_t m = mask[q];
                    if (m) {
                        first = (q << 5) | (__ffs(m) - 1);
                        break;
                    }
                }
                if (threadIdx.x == 0) att_w += (unsigned long long)((first < 0 ? n : first + 1) - start);
                __syncthreads();  // every thread has read mask[] before the next pass rewrites it
                if (first < 0) break;
                const int fq = first >> 5, fj = first & 31;
                for (int t = warp; t < NP; t += W) {
                    const uint32_t sw0 = S[t * nw + fq];
                    __syncwarp();
                    if (lane == 0) S[t * nw + fq] = sw0 ^ (1u << fj);
                    const uint32_t sj = (sw0 >> fj) & 1u;
                    int *Gt = G + t * n;
                    for (int mm = lane; mm < n; mm += 32)
                        if (mm != first) Gt[mm] += (((Jw[fq * n + mm] >> fj) & 1u) == sj) ? -2 : 2;
                }
                if (threadIdx.x == 0) ++acc_w;
                __syncthreads();
                start = first + 1;
                if (start >= n) break;
            }
        }
        // ---- step end: slice energies E = c + (sum s h + (sum s g)/2), ring sum, best
        for (int t = warp; t < NP; t += W) {
            double ph = 0.0;
            int pg = 0;
            for (int i = lane; i < n; i += 32) {
                const bool up = (S[t * nw + (i >> 5)] >> (i & 31)) & 1u;
                ph = __dadd_rn(ph, up ? (double)h[i] : -(double)h[i]);
                pg += up ? G[t * n + i] : -G[t * n + i];
            }
            ph = warp_sum_d(ph);
            pg = warp_sum_i(pg);
            if (lane == 0) cellE[t] = __dadd_rn(Pd.c, __dadd_rn(ph, __dmul_rn(0.5, (double)pg)));
        }
        if (p.ring_bond) {
            int b = 0;
            for (int idx = threadIdx.x; idx < NP * nw; idx += blockDim.x) {
                const int t = idx / nw, q = idx - t * nw;
                const int tn = t + 1 == NP ? 0 : t + 1;
                const int rem = n - 32 * q;
                const uint32_t vm = rem >= 32 ? FULL : ((1u << rem) - 1u);
                b += 2 * __popc(~(S[idx] ^ S[tn * nw + q]) & vm) - __popc(vm);
            }
            b = warp_sum_i(b);
            if (lane == 0) wpart[warp] = b;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double sum = 0.0, emin = __longlong_as_double(0x7ff0000000000000LL);
            int tmin = 0;
            for (int t = 0; t < NP; ++t) {
                const double E = cellE[t];
                sum = __dadd_rn(sum, E);
                if (E < emin) { emin = E; tmin = t; }
            }
            const long long ro = (long long)blockIdx.x * p.steps_total + step;
            if (p.ring_sum) p.ring_sum[ro] = sum;
            if (p.ring_min) p.ring_min[ro] = emin;
            if (p.ring_bond) {
                long long tb = 0;
                for (int w = 0; w < W; ++w) tb += wpart[w];
                p.ring_bond[ro] = tb;
            }
            flag[0] = emin < bestE ? tmin : -1;
        }
        __syncthreads();
        const int tb = flag[0];
        if (tb >= 0) {
            bestE = cellE[tb];
            bestStep = step;
            for (int q = threadIdx.x; q < nw; q += blockDim.x)
                p.best_bits[(long long)blockIdx.x * p.nw_max + q] = S[tb * nw + q];
        }
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < NP * nw; idx += blockDim.x) p.spins[R.spin_off + idx] = S[idx];
    for (int idx = threadIdx.x; idx < NP * n; idx += blockDim.x) Gg[idx] = G[idx];
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

}  // namespace qa
