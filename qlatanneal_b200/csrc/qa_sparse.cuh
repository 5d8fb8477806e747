// qa_sparse.cuh -- Trotter-ring sweep kernel for sparse models with integer
// couplings (the random 3-regular +-1 instances of the benchmark set).
//
// Same replay semantics as ring_kernel<K_SPARSE> (qa_kernels.cuh); different
// data path.  With integer couplings every local field g = J.s is an exact
// integer, so the kernel keeps no field cache at all:
//  * slice moves read the field on demand from the CSR row and the
//    neighbours' spin bits (deg loads; a flip only toggles a bit);
//  * worldline moves (sqa_annealer.cpp:294-315) need the slice sum
//    G_i = sum_t s_t,i g_t,i = sum_j J_ij (P - 2 popc(W_i ^ W_j)), where W_i
//    is spin i's worldline (its bits over the P <= 64 slices): deg popcounts.
// Both equal the maintained float fields of the generic kernel bit for bit
// (integer sums below 2^24 are exact in float32), so results are identical.
#pragma once
#include "qa_pm1.cuh"

namespace qa {

__host__ __device__ inline size_t sparse_smem_bytes(int P, int n, bool ref_order = false) {
    const int nw = (n + 31) / 32, n32 = nw * 32;
    size_t b = align_up((size_t)P * nw * 4, 16);  // S
    b += (size_t)n32 * 8;                          // W (worldline bits)
    b += (size_t)n32 * 4;                          // h
    b += align_up((size_t)P * 8, 16);              // cellE
    b += (size_t)n32 * 4;                          // worldline uniforms
    b += align_up((size_t)nw * 8, 16);             // worldline decisions per block, marks per spin
    b += 32 * 4 + 64;                              // partials, flags
    if (ref_order)                                 // two order rows, the slice pipeline
        b += 2 * ord_row_bytes(n32) + pipe_bytes(P);
    return b + 64;
}

// Neighbour k (0..3) of a slab record: column and value.
__device__ __forceinline__ int slab_col(const uint4 &r, int k) {
    return (int)(((k < 2 ? r.x : r.y) >> (16 * (k & 1))) & 0xFFFFu);
}
__device__ __forceinline__ int slab_val(const uint4 &r, int k) { return (int)(signed char)(r.z >> (8 * k)); }

// Local field of spin i in slice St (its spin bits): from the spin's slab
// record where the model has one (one 16-byte load), else its CSR row.  The
// sum of the same integers either way.
__device__ __forceinline__ int sp_field(const ProbDev &Pd, const uint32_t *St, int i) {
    int g = 0;
    if (Pd.spslab) {
        const uint4 r = __ldg(Pd.spslab + i);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int c = slab_col(r, k), v = slab_val(r, k);
            g += ((St[c >> 5] >> (c & 31)) & 1u) ? v : -v;
        }
        return g;
    }
    const int e0 = __ldg(Pd.rowptr + i), e1 = __ldg(Pd.rowptr + i + 1);
    for (int e = e0; e < e1; ++e) {
        const int2 c = __ldg(Pd.spcv + e);
        g += ((St[c.x >> 5] >> (c.x & 31)) & 1u) ? c.y : -c.y;
    }
    return g;
}

// Slice sum over the worldlines: sum_t s_t,i g_t,i.
__device__ __forceinline__ int sp_world_sum(const ProbDev &Pd, const unsigned long long *Wc,
                                            unsigned long long pmask, int NP, int i) {
    const unsigned long long wi = Wc[i];
    int g = 0;
    if (Pd.spslab) {
        const uint4 r = __ldg(Pd.spslab + i);
#pragma unroll
        for (int k = 0; k < 4; ++k)
            g += slab_val(r, k) * (NP - 2 * __popcll((wi ^ Wc[slab_col(r, k)]) & pmask));
        return g;
    }
    const int e0 = __ldg(Pd.rowptr + i), e1 = __ldg(Pd.rowptr + i + 1);
    for (int e = e0; e < e1; ++e) {
        const int2 c = __ldg(Pd.spcv + e);
        g += c.y * (NP - 2 * __popcll((wi ^ Wc[c.x]) & pmask));
    }
    return g;
}

// The worldline move of spin i (sqa_annealer.cpp:294-315) on the current
// worldlines: a function of W_i and its neighbours' worldlines only.
__device__ __forceinline__ bool sp_world_ok(const ProbDev &Pd, const unsigned long long *Wc, const float *h,
                                            unsigned long long pmask, int NP, int i, float B, float u) {
    const int sh = 2 * __popcll(Wc[i] & pmask) - NP;
    const int gs = sp_world_sum(Pd, Wc, pmask, NP, i);
    const float x = __double2float_rn(__dadd_rn(__dmul_rn((double)h[i], (double)sh), (double)gs));
    return metropolis_nb24(__fmul_rn(x, B), u);
}

__device__ __forceinline__ void sp_sweep_slice(const ProbDev &Pd, uint32_t *S, unsigned long long *Wc,
                                               const float *h, int NP, int t, float B, float T4, uint64_t key,
                                               uint32_t rng_cell, uint32_t sigma, uint32_t tag, int lane,
                                               unsigned long long &att, unsigned long long &acc) {
    const int n = Pd.n, nw = Pd.nw;
    uint32_t *St = S + t * nw;
    const uint32_t *Sp = S + (t == 0 ? NP - 1 : t - 1) * nw;
    const uint32_t *Sn = S + (t + 1 == NP ? 0 : t + 1) * nw;
    U4 rnd = {0, 0, 0, 0};
    att += (unsigned long long)n;
    for (int q = 0; q < nw; ++q) {
        if ((q & 3) == 0) rnd = philox((uint32_t)(((q >> 2) << 5) | lane), rng_cell, sigma, tag, key);
        const int i = (q << 5) | lane;
        const bool valid = i < n;
        const uint32_t sw = St[q];
        const uint32_t sbit = (sw >> lane) & 1u;
        const int d = (int)(((sw ^ Sp[q]) >> lane) & 1u) + (int)(((sw ^ Sn[q]) >> lane) & 1u);
        const float tro = __fmul_rn(__int2float_rn(1 - d), T4);
        const float u = u24(pick(rnd, q & 3));
        const float hi = h[i];
        // a lane's move depends on its own and its neighbours' bits: after a
        // flip only the flipped spin's neighbours later in this block are
        // evaluated again (later blocks read their fields from the current
        // bits anyway), so every decision is the spin-at-a-time sweep's
        auto decide = [&]() {
            const int g = valid ? sp_field(Pd, St, i) : 0;
            const float loc = __fadd_rn(hi, __int2float_rn(g));
            return valid & metropolis_nb24(__fsub_rn(__fmul_rn(signed_by_bit(loc, sbit), B), tro), u);
        };
        uint32_t m = __ballot_sync(FULL, decide());
        uint32_t pending = FULL;
        while (m & pending) {
            const int j = __ffs(m & pending) - 1;
            const int jj = (q << 5) | j;
            if (lane == 0) St[q] = St[q] ^ (1u << j);
            // bit t of the worldline, as a 32-bit atomic on the half that holds it (little-endian)
            if (lane == j) atomicXor(reinterpret_cast<uint32_t *>(Wc + i) + (t >> 5), 1u << (t & 31));
            ++acc;
            pending = j == 31 ? 0u : (FULL << (j + 1));
            uint32_t here = 0;
            const int e0 = __ldg(Pd.rowptr + jj), e1 = __ldg(Pd.rowptr + jj + 1);
            for (int e = e0 + lane; e < e1; e += 32) {
                const int v = __ldg(Pd.spcv + e).x;
                if ((v >> 5) == q) here |= 1u << (v & 31);
            }
            here = __reduce_or_sync(FULL, here) & pending;
            __syncwarp();
            if (here) {
                const bool ok = ((here >> lane) & 1u) && decide();
                m = (m & ~here) | (__ballot_sync(FULL, ok) & here);
            }
            __syncwarp();
        }
    }
}

// Slice t in qanneal's order (the pipelined form of sp_sweep_slice; see
// sweep_slice_ord): visiting position p holds spin ord[p], the Trotter
// neighbours' bits come from the worldline words.  After a flip every later
// lane of the block decides again on the current bits.
__device__ __forceinline__ void sp_sweep_slice_ord(const ProbDev &Pd, uint32_t *S, unsigned long long *Wc,
                                                   const float *h, const OrdT *ord, const SlicePipe &pp,
                                                   int NP, int t, float B, float T4,
                                                   uint64_t key, uint32_t rng_cell, uint32_t sigma, uint32_t tag,
                                                   int lane, unsigned long long &att, unsigned long long &acc) {
    const int n = Pd.n, nw = Pd.nw;
    uint32_t *St = S + t * nw;
    const int tp = t == 0 ? NP - 1 : t - 1, tn = t + 1 == NP ? 0 : t + 1;
    U4 rnd = {0, 0, 0, 0};
    att += (unsigned long long)n;
    for (int q = 0; q < nw; ++q) {
        if ((q & 3) == 0) rnd = philox((uint32_t)(((q >> 2) << 5) | lane), rng_cell, sigma, tag, key);
        if (t > 0) pipe_wait(pp, t - 1, q, lane);
        const int pos = (q << 5) | lane;
        const bool valid = pos < n;
        const int i = valid ? ord[pos] : 0;
        const unsigned long long wc = Wc[i];
        const uint32_t sbit = (uint32_t)(wc >> t) & 1u;
        const int d = (int)(((uint32_t)(wc >> tp) & 1u) ^ sbit) + (int)(((uint32_t)(wc >> tn) & 1u) ^ sbit);
        const float tro = __fmul_rn(__int2float_rn(1 - d), T4);
        const float u = u24(pick(rnd, q & 3));
        const float hi = h[i];
        auto decide = [&]() {
            const int g = valid ? sp_field(Pd, St, i) : 0;
            const float loc = __fadd_rn(hi, __int2float_rn(g));
            return valid & metropolis_nb24(__fsub_rn(__fmul_rn(signed_by_bit(loc, sbit), B), tro), u);
        };
        uint32_t m = __ballot_sync(FULL, decide());
        uint32_t pending = FULL;
        while (m & pending) {
            const int j = __ffs(m & pending) - 1;
            const int jj = __shfl_sync(FULL, i, j);
            if (lane == 0) St[jj >> 5] ^= 1u << (jj & 31);
            // bit t of the worldline, as a 32-bit atomic on the half that holds it (little-endian)
            if (lane == j) atomicXor(reinterpret_cast<uint32_t *>(Wc + i) + (t >> 5), 1u << (t & 31));
            ++acc;
            pending = j == 31 ? 0u : (FULL << (j + 1));
            __syncwarp();
            const bool again = ((pending >> lane) & 1u) && decide();
            m = (m & ~pending) | (__ballot_sync(FULL, again) & pending);
            __syncwarp();
        }
        pipe_publish(pp, t, q, lane);
    }
}

__global__ void __launch_bounds__(1024, 1) ring_sparse_kernel(RingParams p) {
    extern __shared__ __align__(16) unsigned char smem[];
    const RingDev R = p.rings[blockIdx.x];
    const ProbDev Pd = p.probs[R.prob];
    const int NP = p.P, W = p.W, n = Pd.n, nw = Pd.nw, n32 = nw * 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char *ptr = smem;
    uint32_t *S = reinterpret_cast<uint32_t *>(ptr); ptr += align_up((size_t)NP * nw * 4, 16);
    unsigned long long *Wc = reinterpret_cast<unsigned long long *>(ptr); ptr += (size_t)n32 * 8;
    float *h = reinterpret_cast<float *>(ptr); ptr += (size_t)n32 * 4;
    double *cellE = reinterpret_cast<double *>(ptr); ptr += align_up((size_t)NP * 8, 16);
    float *uw = reinterpret_cast<float *>(ptr); ptr += (size_t)n32 * 4;
    uint32_t *wmask = reinterpret_cast<uint32_t *>(ptr);  // [nw] decisions on the sweep's starting state
    uint32_t *wdirty = wmask + nw;                        // [nw] spins whose neighbours have flipped since
    ptr += align_up((size_t)nw * 8, 16);
    int *wpart = reinterpret_cast<int *>(ptr); ptr += 32 * 4;
    int *flag = reinterpret_cast<int *>(ptr); ptr += 64;  // [0]: best slice, [3]: lowest slice (final state)
    // qanneal's order: two rows of visiting orders (the current sweep's and
    // the next one's, copied in the background), the slice pipeline
    OrdT *ob0 = nullptr, *ob1 = nullptr;
    SlicePipe pp{};
    if (p.ref_order) {
        ob0 = reinterpret_cast<OrdT *>(ptr); ptr += ord_row_bytes(n32);
        ob1 = reinterpret_cast<OrdT *>(ptr); ptr += ord_row_bytes(n32);
        pp = pipe_open(ptr, NP, p.counters + 4);
    }

    for (int idx = threadIdx.x; idx < NP * nw; idx += blockDim.x) S[idx] = p.spins[R.spin_off + idx];
    for (int i = threadIdx.x; i < n32; i += blockDim.x) h[i] = i < n ? Pd.h32[i] : 0.0f;
    __syncthreads();
    for (int i = threadIdx.x; i < n32; i += blockDim.x) {
        unsigned long long wc = 0;
        if (i < n)
            for (int t = 0; t < NP; ++t) wc |= (unsigned long long)((S[t * nw + (i >> 5)] >> (i & 31)) & 1u) << t;
        Wc[i] = wc;
    }
    __syncthreads();

    const unsigned long long pmask = NP == 64 ? ~0ull : ((1ull << NP) - 1ull);
    const int slot = p.slot ? p.slot[blockIdx.x] : R.k;
    OrderFeed feed = feed_open(ob0, ob1, p.ref_order ? p.ordg + blockIdx.x * p.ord_ring : nullptr, p.ord_stride, n,
                               p.ref_order ? (p.step1 - p.step0) * p.ord_per_step : 0);
    unsigned long long att_s = 0, acc_s = 0, att_w = 0, acc_w = 0;
    double bestE = p.best_E[blockIdx.x];
    int bestStep = p.best_step[blockIdx.x];

    for (int step = p.step0 - (p.init_scan ? 1 : 0); step < p.step1; ++step) {
        // step -1 (init_scan) only scores the starting state
        const int spb = step >= 0 ? p.spb : 0, wls = step >= 0 ? p.wls : 0;
        const int si_tab = R.sched + (p.per_slot_sched ? slot + max(step, 0) * p.slot_step : max(step, 0));
        const float B = p.B[si_tab], T4 = p.T4[si_tab];
        for (int sw = 0; sw < spb; ++sw) {
            const uint32_t sigma = (uint32_t)(step * p.spb + sw);
            if (p.ref_order) {
                const uint32_t tag = p.slice_tag | R.tag_extra;
                pipe_reset(pp, NP);
                const OrdT *ord = feed_take(feed);
                for (int t = warp; t < NP; t += W)
                    sp_sweep_slice_ord(Pd, S, Wc, h, ord, pp, NP, t, B, T4, R.key, (uint32_t)(slot * NP + t), sigma,
                                       tag, lane, att_s, acc_s);
                __syncthreads();
            } else {
                for (int ph = 0; ph < 3; ++ph) {
                    const int cnt = phase_count(NP, ph);
                    for (int c = warp; c < cnt; c += W) {
                        const int t = phase_slice(NP, ph, c);
                        sp_sweep_slice(Pd, S, Wc, h, NP, t, B, T4, R.key, (uint32_t)(slot * NP + t), sigma,
                                       p.slice_tag | R.tag_extra, lane, att_s, acc_s);
                    }
                    if (cnt) __syncthreads();
                }
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
            if (p.bsamp) record_bond_sample(p, S, NP, nw, n, wpart, W, step, sw);
        }
        // worldline sweeps, spins in order, sums from the worldline bits.  Every
        // warp first evaluates all spins' moves on the sweep's starting
        // worldlines; warp 0 then takes the spins in order.  A move depends only
        // on the spin's own worldline and its neighbours', so a decision stands
        // unless a neighbour flipped earlier in the sweep: such spins are marked
        // and evaluated again when their turn comes.  Every decision is thus
        // taken on the state the one-spin-at-a-time sweep sees.
        for (int sw = 0; sw < wls && p.ref_order; ++sw) {
            // qanneal's order: the same scheme over visiting positions; the
            // marks of flipped neighbours are kept per spin
            const uint32_t sigma = (uint32_t)(step * p.wls + sw);
            const OrdT *ord = feed_take(feed);
            for (int pp = threadIdx.x; pp < n32; pp += blockDim.x) {  // a warp covers one block of positions
                const int q = pp >> 5, l = pp & 31;
                const U4 r = philox((uint32_t)(((q >> 2) << 5) | l), (uint32_t)slot, sigma, DOM_WORLD, R.key);
                const float u = u24(pick(r, q & 3));
                uw[pp] = u;
                const bool valid = pp < n;
                const int i = valid ? ord[pp] : 0;
                const bool ok = valid && sp_world_ok(Pd, Wc, h, pmask, NP, i, B, u);
                const uint32_t m = __ballot_sync(FULL, ok);
                if (l == 0) {
                    wmask[q] = m;
                    wdirty[q] = 0u;
                }
            }
            if (threadIdx.x == 0) att_w += (unsigned long long)n;
            __syncthreads();
            if (warp == 0) {
                for (int q = 0; q < nw; ++q) {
                    const int pos = (q << 5) | lane;
                    const bool valid = pos < n;
                    const int i = valid ? ord[pos] : 0;
                    const float u = uw[pos];
                    uint32_t m = wmask[q];
                    const bool dirty0 = valid && ((wdirty[i >> 5] >> (i & 31)) & 1u);  // a neighbour flipped earlier
                    const uint32_t dq = __ballot_sync(FULL, dirty0);
                    if (dq) {
                        const bool ok = dirty0 && sp_world_ok(Pd, Wc, h, pmask, NP, i, B, u);
                        m = (m & ~dq) | (__ballot_sync(FULL, ok) & dq);
                    }
                    uint32_t pending = FULL;
                    if (Pd.spslab && m) {
                        // a decision of m stands unless an earlier lane of the
                        // block that flips is a neighbour: every lane before the
                        // first lane with an accepted earlier neighbour is final,
                        // so those moves are applied together
                        const uint4 rec = __ldg(Pd.spslab + i);
                        uint32_t nbl = 0;  // earlier lanes holding a neighbour of this lane's spin
                        for (int l = 0; l < 31; ++l) {
                            const int il = __shfl_sync(FULL, i, l);
                            bool nb = false;
#pragma unroll
                            for (int k = 0; k < 4; ++k) nb |= slab_val(rec, k) != 0 && slab_col(rec, k) == il;
                            if (l < lane && nb) nbl |= 1u << l;
                        }
                        const uint32_t conf = __ballot_sync(FULL, valid && (nbl & m) != 0u);
                        const uint32_t pre = conf ? (1u << (__ffs(conf) - 1)) - 1u : FULL;
                        const uint32_t F = m & pre;
                        if (F) {
                            if ((F >> lane) & 1u) {
                                for (int t = 0; t < NP; ++t) atomicXor(S + t * nw + (i >> 5), 1u << (i & 31));
                                Wc[i] ^= pmask;
#pragma unroll
                                for (int k = 0; k < 4; ++k)
                                    if (slab_val(rec, k) != 0) {
                                        const int v = slab_col(rec, k);
                                        atomicOr(wdirty + (v >> 5), 1u << (v & 31));
                                    }
                            }
                            acc_w += (unsigned long long)__popc(F);
                            pending = ~pre;  // the first conflicted lane and after (none when pre == FULL)
                            __syncwarp();
                            const bool mark = ((pending >> lane) & 1u) && valid && ((wdirty[i >> 5] >> (i & 31)) & 1u);
                            const uint32_t here = __ballot_sync(FULL, mark);
                            if (here) {
                                const bool ok = mark && sp_world_ok(Pd, Wc, h, pmask, NP, i, B, u);
                                m = (m & ~here) | (__ballot_sync(FULL, ok) & here);
                            }
                            __syncwarp();
                        }
                    }
                    while (m & pending) {
                        const int j = __ffs(m & pending) - 1;
                        const int jj = __shfl_sync(FULL, i, j);
                        for (int t = lane; t < NP; t += 32) S[t * nw + (jj >> 5)] ^= 1u << (jj & 31);
                        if (lane == j) Wc[jj] ^= pmask;
                        ++acc_w;
                        pending = j == 31 ? 0u : (FULL << (j + 1));
                        const int e0 = __ldg(Pd.rowptr + jj), e1 = __ldg(Pd.rowptr + jj + 1);
                        for (int e = e0 + lane; e < e1; e += 32) {
                            const int v = __ldg(Pd.spcv + e).x;
                            atomicOr(wdirty + (v >> 5), 1u << (v & 31));
                        }
                        __syncwarp();
                        const bool mark = ((pending >> lane) & 1u) && valid && ((wdirty[i >> 5] >> (i & 31)) & 1u);
                        const uint32_t here = __ballot_sync(FULL, mark);
                        if (here) {
                            const bool ok = mark && sp_world_ok(Pd, Wc, h, pmask, NP, i, B, u);
                            m = (m & ~here) | (__ballot_sync(FULL, ok) & here);
                        }
                        __syncwarp();
                    }
                }
            }
            __syncthreads();
        }
        for (int sw = 0; sw < wls && !p.ref_order; ++sw) {
            const uint32_t sigma = (uint32_t)(step * p.wls + sw);
            for (int i = threadIdx.x; i < n32; i += blockDim.x) {  // a warp covers one 32-spin block
                const int q = i >> 5, l = i & 31;
                const U4 r = philox((uint32_t)(((q >> 2) << 5) | l), (uint32_t)slot, sigma, DOM_WORLD, R.key);
                const float u = u24(pick(r, q & 3));
                uw[i] = u;
                const bool ok = i < n && sp_world_ok(Pd, Wc, h, pmask, NP, i, B, u);
                const uint32_t m = __ballot_sync(FULL, ok);
                if (l == 0) {
                    wmask[q] = m;
                    wdirty[q] = 0u;
                }
            }
            if (threadIdx.x == 0) att_w += (unsigned long long)n;
            __syncthreads();
            if (warp == 0) {
                for (int q = 0; q < nw; ++q) {
                    const int i = (q << 5) | lane;
                    const bool valid = i < n;
                    const float u = uw[i];
                    uint32_t m = wmask[q];
                    const uint32_t dq = wdirty[q];  // neighbours flipped in earlier blocks
                    if (dq) {
                        const bool ok = valid && ((dq >> lane) & 1u) && sp_world_ok(Pd, Wc, h, pmask, NP, i, B, u);
                        m = (m & ~dq) | (__ballot_sync(FULL, ok) & dq);
                    }
                    uint32_t pending = FULL;
                    if (Pd.spslab && m) {
                        // as in qanneal's order: the moves before the first lane
                        // with an accepted earlier neighbour in the block are final
                        const uint4 rec = __ldg(Pd.spslab + (valid ? i : 0));
                        uint32_t nbl = 0, nbi = 0;  // in-block neighbours: earlier lanes, all lanes
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const int c = slab_col(rec, k);
                            if (slab_val(rec, k) != 0 && (c >> 5) == q) {
                                nbi |= 1u << (c & 31);
                                if ((c & 31) < lane) nbl |= 1u << (c & 31);
                            }
                        }
                        const uint32_t conf = __ballot_sync(FULL, valid && (nbl & m) != 0u);
                        const uint32_t pre = conf ? (1u << (__ffs(conf) - 1)) - 1u : FULL;
                        const uint32_t F = m & pre;
                        if (F) {
                            const bool fl = (F >> lane) & 1u;
                            for (int t = lane; t < NP; t += 32) S[t * nw + q] ^= F;
                            if (fl) {
                                Wc[i] ^= pmask;
#pragma unroll
                                for (int k = 0; k < 4; ++k) {
                                    const int v = slab_col(rec, k);
                                    if (slab_val(rec, k) != 0 && (v >> 5) > q) atomicOr(wdirty + (v >> 5), 1u << (v & 31));
                                }
                            }
                            acc_w += (unsigned long long)__popc(F);
                            pending = ~pre;
                            const uint32_t here = __reduce_or_sync(FULL, fl ? nbi : 0u) & pending;
                            __syncwarp();
                            if (here) {
                                const bool ok =
                                    valid && ((here >> lane) & 1u) && sp_world_ok(Pd, Wc, h, pmask, NP, i, B, u);
                                m = (m & ~here) | (__ballot_sync(FULL, ok) & here);
                            }
                            __syncwarp();
                        }
                    }
                    while (m & pending) {
                        const int j = __ffs(m & pending) - 1;
                        const int jj = (q << 5) | j;
                        for (int t = lane; t < NP; t += 32) S[t * nw + q] ^= 1u << j;
                        if (lane == j) Wc[jj] ^= pmask;
                        ++acc_w;
                        pending = j == 31 ? 0u : (FULL << (j + 1));
                        // jj's neighbours: later spins of this block now, later blocks marked
                        uint32_t here = 0;
                        const int e0 = __ldg(Pd.rowptr + jj), e1 = __ldg(Pd.rowptr + jj + 1);
                        for (int e = e0 + lane; e < e1; e += 32) {
                            const int v = __ldg(Pd.spcv + e).x;
                            if ((v >> 5) == q) here |= 1u << (v & 31);
                            else if ((v >> 5) > q) atomicOr(wdirty + (v >> 5), 1u << (v & 31));
                        }
                        here = __reduce_or_sync(FULL, here) & pending;
                        __syncwarp();
                        if (here) {
                            const bool ok =
                                valid && ((here >> lane) & 1u) && sp_world_ok(Pd, Wc, h, pmask, NP, i, B, u);
                            m = (m & ~here) | (__ballot_sync(FULL, ok) & here);
                        }
                        __syncwarp();
                    }
                }
            }
            __syncthreads();
        }
        // ---- step end: slice energies E = c + (sum s h + (sum s g)/2), ring sum, best
        for (int t = warp; t < NP; t += W) {
            const uint32_t *St = S + t * nw;
            double ph = 0.0;
            int pg = 0;
            for (int i = lane; i < n; i += 32) {
                const bool up = (St[i >> 5] >> (i & 31)) & 1u;
                ph = __dadd_rn(ph, up ? (double)h[i] : -(double)h[i]);
                const int g = sp_field(Pd, St, i);
                pg += up ? g : -g;
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
            const long long ro = (long long)blockIdx.x * p.rec_stride + p.rec_base + step;
            if (p.ring_sum) p.ring_sum[ro] = sum;
            if (p.ring_min) p.ring_min[ro] = emin;
            if (p.ring_bond) {
                long long tb = 0;
                for (int w = 0; w < W; ++w) tb += wpart[w];
                p.ring_bond[ro] = tb;
            }
            flag[0] = emin < bestE ? tmin : -1;
            flag[3] = tmin;
        }
        __syncthreads();
        const int tb = flag[0];
        if (tb >= 0) {
            bestE = cellE[tb];
            bestStep = step;
            if (threadIdx.x == 0 && p.best_slot) p.best_slot[blockIdx.x] = slot;
            for (int q = threadIdx.x; q < nw; q += blockDim.x)
                p.best_bits[(long long)blockIdx.x * p.nw_max + q] = S[tb * nw + q];
        }
        if (p.final_bits && step == p.steps_total - 1)
            for (int q = threadIdx.x; q < nw; q += blockDim.x)
                p.final_bits[(long long)blockIdx.x * p.nw_max + q] = S[flag[3] * nw + q];
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < NP * nw; idx += blockDim.x) p.spins[R.spin_off + idx] = S[idx];
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
