// qa_pm1.cuh -- Trotter-ring sweep kernel specialised for dense couplings in
// {-1, +1} (the Sherrington-Kirkpatrick instances of the benchmark set).
//
// Same replay semantics as ring_kernel (qa_kernels.cuh), different data path:
//  * J is bit-packed (1 bit per coupling) and staged once per CTA in shared
//    memory: Jw[q*npad + m] holds bits J[m][32q .. 32q+31] (J is symmetric, so
//    it is also column m); rows are padded to npad, a multiple of 128.
//  * Local fields are exact int32 (g = J.s is an integer) in shared memory.
//  * A block of 32 spins is resolved in spin order by ballots; the fields of
//    the whole slice are then updated once for all flips F of the block:
//        g[m] += 2|F| - 4 popc(~(Jw[q*npad+m] ^ s_old) & F)
//    four fields per lane per 128-bit shared-memory access; a flipped spin's
//    own field then takes -2 s_m(old) (its zero diagonal bit reads as -1).
//  * Worldline moves (sqa_annealer.cpp:294-315): the slice sums
//    G_i = sum_t s_t,i g_t,i are built once per sweep; decisions for all
//    remaining spins are taken in parallel; the first block holding an
//    accepted move is resolved in spin order by one warp, its flips applied to
//    every slice by the block update above, and the sums of later spins
//    corrected exactly by  dG_i = -2 J_ij (P - 2 popc(W_i ^ W_j))  where W_i
//    is spin i's worldline (its bits over the P slices).  The result is the
//    sequential sweep; the cost is one parallel pass per block with moves.
#pragma once
#include "qa_kernels.cuh"

namespace qa {

__host__ __device__ inline int pm1_npad(int n) { return (n + 127) / 128 * 128; }

// Shared memory of one ring: gbytes = bytes per field (4: int32, 2: int16);
// jw_smem = J bits staged in shared memory (else read through L1/L2);
// ref_order = qanneal's update order (two rows of visiting orders, the
// slices' progress counters and the flipped spins of a worldline block).
__host__ __device__ inline size_t pm1_smem_bytes(int P, int n, int gbytes = 4, bool jw_smem = true,
                                                 bool ref_order = false) {
    const int nw = (n + 31) / 32, np = pm1_npad(n);
    size_t b = jw_smem ? (size_t)nw * np * 4 : 0;  // Jw
    b += align_up((size_t)P * nw * 4, 16);         // S
    b += (size_t)np * 4;                           // h
    b += align_up((size_t)P * np * gbytes, 16);    // G
    b += (size_t)np * 8;                           // W (worldline bits)
    b += (size_t)np * 4;                           // Gsum (worldline slice sums)
    b += (size_t)np * 4;                           // uw (worldline uniforms)
    b += align_up((size_t)P * 8, 16);              // cellE
    b += (size_t)(np / 32) * 4;                    // worldline move masks, one per block (np/32 >= nw)
    b += 32 * 8 + 32 * 4 + 64;                     // old worldlines, partials, flags
    if (ref_order)
        b += 2 * ord_row_bytes(np) + pipe_bytes(P) + 32 * 4;
    return b + 64;
}

__device__ __forceinline__ int warp_sum_i(int v) {
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) v += __shfl_xor_sync(FULL, v, off);
    return v;
}

// x = s*(h+g) with the sign taken from the spin bit (bit 1 = +1).
__device__ __forceinline__ float signed_by_bit(float v, uint32_t bit) {
    return __int_as_float(__float_as_int(v) ^ (int)((bit ^ 1u) << 31));
}

__device__ __forceinline__ int flip_delta(uint32_t jw, uint32_t sold, uint32_t Fm) {
    return 2 * __popc(Fm) - 4 * __popc(~(jw ^ sold) & Fm);
}

// Fields of one slice after the spins F of block q (old word sold) flipped.
// Whole warp.  Every field takes the flips of all of F: the diagonal bit of
// a row is 0, which the sum reads as J_mm = -1, so a flipped spin m's own
// field comes out 2 s_m too high and is corrected by its lane afterwards.
__device__ __forceinline__ void pm1_self_fix(int *Gt, int q, uint32_t F, uint32_t sold, int lane) {
    __syncwarp();
    if ((F >> lane) & 1u) Gt[(q << 5) | lane] += ((sold >> lane) & 1u) ? -2 : 2;
}
__device__ __forceinline__ void pm1_self_fix(short *Gt, int q, uint32_t F, uint32_t sold, int lane) {
    __syncwarp();
    if ((F >> lane) & 1u) Gt[(q << 5) | lane] = (short)(Gt[(q << 5) | lane] + (((sold >> lane) & 1u) ? -2 : 2));
}
__device__ __forceinline__ void pm1_block_update(int *Gt, const uint32_t *Jw, int npad, int n, int q, uint32_t F,
                                                 uint32_t sold, int lane) {
    const uint32_t *Jq = Jw + q * npad;
    const int f2 = 2 * __popc(F);
    for (int base = lane * 4; base < n; base += 128) {
        const uint4 jw = *reinterpret_cast<const uint4 *>(Jq + base);
        int4 g = *reinterpret_cast<int4 *>(Gt + base);
        g.x += f2 - 4 * __popc(~(jw.x ^ sold) & F);
        g.y += f2 - 4 * __popc(~(jw.y ^ sold) & F);
        g.z += f2 - 4 * __popc(~(jw.z ^ sold) & F);
        g.w += f2 - 4 * __popc(~(jw.w ^ sold) & F);
        *reinterpret_cast<int4 *>(Gt + base) = g;
    }
    pm1_self_fix(Gt, q, F, sold, lane);
}

// int16 fields (|g| <= n - 1 < 2^15): eight per lane per 128-bit access,
// two per 32-bit word updated by a halfword-wise add (no carry between them).
__device__ __forceinline__ uint32_t pack_delta2(int lo, int hi) {
    return ((uint32_t)lo & 0xffffu) | ((uint32_t)hi << 16);
}

__device__ __forceinline__ void pm1_block_update(short *Gt, const uint32_t *Jw, int npad, int n, int q, uint32_t F,
                                                 uint32_t sold, int lane) {
    const uint32_t *Jq = Jw + q * npad;
    for (int base = lane * 8; base < n; base += 256) {
        const uint4 ja = *reinterpret_cast<const uint4 *>(Jq + base);
        const uint4 jb = *reinterpret_cast<const uint4 *>(Jq + base + 4);
        uint4 g = *reinterpret_cast<uint4 *>(Gt + base);
        g.x = __vadd2(g.x, pack_delta2(flip_delta(ja.x, sold, F), flip_delta(ja.y, sold, F)));
        g.y = __vadd2(g.y, pack_delta2(flip_delta(ja.z, sold, F), flip_delta(ja.w, sold, F)));
        g.z = __vadd2(g.z, pack_delta2(flip_delta(jb.x, sold, F), flip_delta(jb.y, sold, F)));
        g.w = __vadd2(g.w, pack_delta2(flip_delta(jb.z, sold, F), flip_delta(jb.w, sold, F)));
        *reinterpret_cast<uint4 *>(Gt + base) = g;
    }
    pm1_self_fix(Gt, q, F, sold, lane);
}

// One block of 32 spins (lane = spin) of slice t; rw is this lane's Philox word.
template <typename GT>
__device__ __forceinline__ void pm1_block(const uint32_t *Jw, uint32_t *St, const uint32_t *Sp, const uint32_t *Sn,
                                          GT *Gt, unsigned long long *Wc, const float *h, int n, int npad, int q,
                                          int t, uint32_t rw, float B, float T4, int lane, unsigned long long &acc) {
    const int i = (q << 5) | lane;
    const bool valid = i < n;
    const uint32_t sw = St[q];
    const uint32_t sbit = (sw >> lane) & 1u;
    // s*(s_prev + s_next)/2 = 1 - (number of Trotter neighbours that differ)
    const int d = (int)(((sw ^ Sp[q]) >> lane) & 1u) + (int)(((sw ^ Sn[q]) >> lane) & 1u);
    const float tro = __fmul_rn(__int2float_rn(1 - d), T4);
    const float u = u24(rw);
    const float hi = h[i];
    const int gi = (int)Gt[i];
    const float y = __fsub_rn(__fmul_rn(signed_by_bit(__fadd_rn(hi, __int2float_rn(gi)), sbit), B), tro);
    // most blocks reject every proposal: a sufficient test first, the exact one if any lane may accept
    if (!__any_sync(FULL, valid & metropolis_maybe24(y, u))) return;
    bool ok = valid & metropolis_nb24(y, u);
    uint32_t m = __ballot_sync(FULL, ok);
    if (m == 0) return;
    // resolve the block in spin order; gk is this lane's field with the
    // block's earlier flips applied
    const uint32_t jd = Jw[q * npad + i];
    uint32_t F = 0;
    int gk = gi;
    do {
        const int j = __ffs(m) - 1;
        F |= 1u << j;
        if (lane != j) gk += (((sw ^ jd) >> j) & 1u) ? 2 : -2;
        const uint32_t pending = j == 31 ? 0u : (FULL << (j + 1));
        ok = valid & metropolis_nb24(
            __fsub_rn(__fmul_rn(signed_by_bit(__fadd_rn(hi, __int2float_rn(gk)), sbit), B), tro), u);
        m = __ballot_sync(FULL, ok) & pending;
        ++acc;
    } while (m);
    if (lane == 0) St[q] = sw ^ F;
    // bit t of the worldline, as a 32-bit atomic on the half that holds it (little-endian)
    if ((F >> lane) & 1u) atomicXor(reinterpret_cast<uint32_t *>(Wc + i) + (t >> 5), 1u << (t & 31));
    pm1_block_update(Gt, Jw, npad, n, q, F, sw, lane);
    __syncwarp();
}

// Flip the spins of mask F (lanes; spin sp of each lane) in slice t's spin
// words St and update its fields: one block update per 32-spin word holding
// flipped spins (spins in one word share a popcount pass).  Whole warp.
template <typename GT>
__device__ __forceinline__ void pm1_flip_spins(uint32_t *St, GT *Gt, const uint32_t *Jw, int npad, int n, uint32_t F,
                                               int sp, int lane) {
    uint32_t rest = F;
    while (rest) {
        const int wq = __shfl_sync(FULL, sp, __ffs(rest) - 1) >> 5;
        const bool in = ((rest >> lane) & 1u) && (sp >> 5) == wq;
        const uint32_t lanes = __ballot_sync(FULL, in);
        const uint32_t Fq = __reduce_or_sync(FULL, in ? (1u << (sp & 31)) : 0u);
        const uint32_t sold = St[wq];
        __syncwarp();
        if (lane == 0) St[wq] = sold ^ Fq;
        pm1_block_update(Gt, Jw, npad, n, wq, Fq, sold, lane);
        rest &= ~lanes;
    }
    __syncwarp();
}

// One block of 32 visiting positions of slice t in qanneal's order: lane =
// position (q << 5) | lane, spin ord[position]; rw is the position's Philox
// word.  What does not depend on slice t - 1 -- the spin, its h, its own
// field, the uniform -- is loaded before the wait for slice t - 1 to finish
// the block; the spin's own and Trotter neighbours' bits (slices tp, tn) come
// from its worldline word.  While slice t holds the block no other slice
// touches these spins (the pipeline), so slice tp shows this sweep's state
// and slice tn the last sweep's (slice 0's of this sweep for the last slice,
// which therefore also waits for slice 0 to finish the block).
// Before waiting for slice tp, the block is tried with both values of the one
// bit slice tp may still change: if every lane rejects under either value
// (the pre-test), the block has no flips whatever slice tp does, and it is
// published at once.  Most blocks end there, so the slices stop waiting on one
// another except where a Trotter neighbour can change a decision.  Flips are
// resolved in position order; the block is published to slice t + 1 as soon
// as its bits are final (the worldline atomics), before the slice's own field
// update, which slice t + 1 never reads.
template <typename GT>
__device__ __forceinline__ void pm1_block_ord(const uint32_t *Jw, uint32_t *St, GT *Gt, unsigned long long *Wc,
                                              const float *h, const OrdT *ord, int n, int npad, int q, int t, int tp,
                                              int tn, uint32_t rw, float B, float T4, int lane,
                                              unsigned long long &acc, const SlicePipe &pp) {
    const int pos = (q << 5) | lane;
    const bool valid = pos < n;
    const int i = valid ? ord[pos] : 0;
    const float u = u24(rw);
    const float hi = h[i];
    const int gi = (int)Gt[i];
    const float hg = __fadd_rn(hi, __int2float_rn(gi));
    if (t > 0) {
        if (tn == 0) pipe_wait(pp, 0, q, lane);  // the last slice: slice 0 after this sweep
        // bits t and tn are final; y with slice tp's bit equal to and
        // differing from s, computed as the exact test below computes it
        const unsigned long long w0 = Wc[i];
        const uint32_t sb = (uint32_t)(w0 >> t) & 1u;
        const int dn = (int)(((uint32_t)(w0 >> tn) & 1u) ^ sb);
        const float xs = __fmul_rn(signed_by_bit(hg, sb), B);
        const float ya = __fsub_rn(xs, __fmul_rn(__int2float_rn(1 - dn), T4));
        const float yb = __fsub_rn(xs, __fmul_rn(__int2float_rn(-dn), T4));
        if (!__any_sync(FULL, valid & (metropolis_maybe24(ya, u) | metropolis_maybe24(yb, u)))) {
            pipe_publish(pp, t, q, lane, false);  // no flips in the block, nothing written
            return;
        }
        pipe_wait(pp, t - 1, q, lane);
    }
    const unsigned long long wc = Wc[i];
    const uint32_t sbit = (uint32_t)(wc >> t) & 1u;
    const int d = (int)(((uint32_t)(wc >> tp) & 1u) ^ sbit) + (int)(((uint32_t)(wc >> tn) & 1u) ^ sbit);
    const float tro = __fmul_rn(__int2float_rn(1 - d), T4);
    const float y = __fsub_rn(__fmul_rn(signed_by_bit(hg, sbit), B), tro);
    if (!__any_sync(FULL, valid & metropolis_maybe24(y, u))) {
        pipe_publish(pp, t, q, lane, false);  // nothing written
        return;
    }
    bool ok = valid & metropolis_nb24(y, u);
    uint32_t m = __ballot_sync(FULL, ok);
    if (m == 0) {
        pipe_publish(pp, t, q, lane, false);  // nothing written
        return;
    }
    // gk: this lane's field with the block's earlier flips applied,
    // g_i += -2 J_i,j s_j(old) for each flipped spin j
    uint32_t F = 0;
    int gk = gi;
    do {
        const int j = __ffs(m) - 1;
        F |= 1u << j;
        const int ij = __shfl_sync(FULL, i, j);
        const uint32_t sj = __shfl_sync(FULL, sbit, j);
        if (lane != j) gk += ((((Jw[(ij >> 5) * npad + i] >> (ij & 31)) & 1u) ^ sj) != 0u) ? 2 : -2;
        const uint32_t pending = j == 31 ? 0u : (FULL << (j + 1));
        ok = valid & metropolis_nb24(
            __fsub_rn(__fmul_rn(signed_by_bit(__fadd_rn(hi, __int2float_rn(gk)), sbit), B), tro), u);
        m = __ballot_sync(FULL, ok) & pending;
        ++acc;
    } while (m);
    // bit t of each flipped spin's worldline (32-bit atomic on the half that
    // holds it), then the block is final for slice t + 1
    if ((F >> lane) & 1u) atomicXor(reinterpret_cast<uint32_t *>(Wc + i) + (t >> 5), 1u << (t & 31));
    pipe_publish(pp, t, q, lane);
    pm1_flip_spins(St, Gt, Jw, npad, n, F, i, lane);
}

// y = -dE of a worldline move of spin i with slice sum gs (B = 2 beta/P).
__device__ __forceinline__ float pm1_world_y(float hi, unsigned long long wi, int gs, int NP, float B) {
    const int sh = 2 * __popcll(wi) - NP;
    return __fmul_rn(__double2float_rn(__dadd_rn(__dmul_rn((double)hi, (double)sh), (double)gs)), B);
}

// One warp sweeps slice t; one Philox call per lane serves four blocks.
template <typename GT>
__device__ __forceinline__ void pm1_sweep_slice(const uint32_t *Jw, uint32_t *S, GT *G, unsigned long long *Wc,
                                                const float *h, int n, int nw, int npad, int NP, int t, float B,
                                                float T4, uint64_t key, uint32_t rng_cell, uint32_t sigma,
                                                uint32_t tag, int lane, unsigned long long &att,
                                                unsigned long long &acc) {
    uint32_t *St = S + t * nw;
    const uint32_t *Sp = S + (t == 0 ? NP - 1 : t - 1) * nw;
    const uint32_t *Sn = S + (t + 1 == NP ? 0 : t + 1) * nw;
    GT *Gt = G + t * npad;
    att += (unsigned long long)n;
    for (int q4 = 0; q4 < nw; q4 += 4) {
        const U4 r = philox((uint32_t)(((q4 >> 2) << 5) | lane), rng_cell, sigma, tag, key);
        pm1_block(Jw, St, Sp, Sn, Gt, Wc, h, n, npad, q4, t, r.x, B, T4, lane, acc);
        if (q4 + 1 < nw) pm1_block(Jw, St, Sp, Sn, Gt, Wc, h, n, npad, q4 + 1, t, r.y, B, T4, lane, acc);
        if (q4 + 2 < nw) pm1_block(Jw, St, Sp, Sn, Gt, Wc, h, n, npad, q4 + 2, t, r.z, B, T4, lane, acc);
        if (q4 + 3 < nw) pm1_block(Jw, St, Sp, Sn, Gt, Wc, h, n, npad, q4 + 3, t, r.w, B, T4, lane, acc);
    }
}

__device__ __forceinline__ bool pm1_world_ok(const float *h, const int *Gs, const unsigned long long *Wc,
                                             const float *uw, int i, int n, int NP, float B) {
    const int sh = 2 * __popcll(Wc[i]) - NP;
    const float x = __double2float_rn(__dadd_rn(__dmul_rn((double)h[i], (double)sh), (double)Gs[i]));
    return (i < n) & metropolis_nb24(__fmul_rn(x, B), uw[i]);
}

// The warp's ballot of pm1_world_ok over spins i (one per lane, i < npad),
// the exponential skipped when the pre-test rejects every lane.
__device__ __forceinline__ uint32_t pm1_world_ballot(const float *h, const int *Gs, const unsigned long long *Wc,
                                                     const float *uw, int i, int n, int NP, float B) {
    const int sh = 2 * __popcll(Wc[i]) - NP;
    const float y =
        __fmul_rn(__double2float_rn(__dadd_rn(__dmul_rn((double)h[i], (double)sh), (double)Gs[i])), B);
    if (!__any_sync(FULL, (i < n) & metropolis_maybe24(y, uw[i]))) return 0u;
    return __ballot_sync(FULL, (i < n) & metropolis_nb24(y, uw[i]));
}

// GT: field type (int: fields as int32; short: int16, for rings whose int32
// fields would not fit).  JW_SMEM: J bits staged in shared memory, else read
// from global memory (L2-resident: every ring of an instance reads the same
// n^2/8 bytes).
template <typename GT, bool JW_SMEM>
__global__ void __launch_bounds__(1024, 1) ring_pm1_kernel(RingParams p) {
    extern __shared__ __align__(16) unsigned char smem[];
    const RingDev R = p.rings[blockIdx.x];
    const ProbDev Pd = p.probs[R.prob];
    const int NP = p.P, W = p.W, n = Pd.n, nw = Pd.nw, npad = pm1_npad(n);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char *ptr = smem;
    uint32_t *Jw_s = reinterpret_cast<uint32_t *>(ptr);
    if (JW_SMEM) ptr += (size_t)nw * npad * 4;
    const uint32_t *Jw = JW_SMEM ? Jw_s : Pd.Jw;
    uint32_t *S = reinterpret_cast<uint32_t *>(ptr); ptr += align_up((size_t)NP * nw * 4, 16);
    float *h = reinterpret_cast<float *>(ptr); ptr += (size_t)npad * 4;
    GT *G = reinterpret_cast<GT *>(ptr); ptr += align_up((size_t)NP * npad * sizeof(GT), 16);
    unsigned long long *Wc = reinterpret_cast<unsigned long long *>(ptr); ptr += (size_t)npad * 8;
    int *Gs = reinterpret_cast<int *>(ptr); ptr += (size_t)npad * 4;
    float *uw = reinterpret_cast<float *>(ptr); ptr += (size_t)npad * 4;
    double *cellE = reinterpret_cast<double *>(ptr); ptr += align_up((size_t)NP * 8, 16);
    uint32_t *mask = reinterpret_cast<uint32_t *>(ptr); ptr += (size_t)(npad / 32) * 4;
    unsigned long long *Wold = reinterpret_cast<unsigned long long *>(ptr); ptr += 32 * 8;
    int *wpart = reinterpret_cast<int *>(ptr); ptr += 32 * 4;
    int *flag = reinterpret_cast<int *>(ptr); ptr += 64;  // [1]: worldline block flips F, [2]: their block index
    // qanneal's order: two rows of visiting orders (the current sweep's and
    // the next one's, copied in the background), the slices' progress
    // counters, the wait-abort flag and the spins of a resolved worldline block
    OrdT *ob0 = nullptr, *ob1 = nullptr;
    int *Wsp = nullptr;
    SlicePipe pp{};
    if (p.ref_order) {
        ob0 = reinterpret_cast<OrdT *>(ptr); ptr += ord_row_bytes(npad);
        ob1 = reinterpret_cast<OrdT *>(ptr); ptr += ord_row_bytes(npad);
        pp = pipe_open(ptr, NP, p.counters + 4); ptr += pipe_bytes(NP);
        Wsp = reinterpret_cast<int *>(ptr);
    }

    if (JW_SMEM)
        for (int idx = threadIdx.x; idx < nw * npad; idx += blockDim.x) Jw_s[idx] = Pd.Jw[idx];
    for (int idx = threadIdx.x; idx < NP * nw; idx += blockDim.x) S[idx] = p.spins[R.spin_off + idx];
    for (int i = threadIdx.x; i < npad; i += blockDim.x) h[i] = i < n ? Pd.h32[i] : 0.0f;
    GT *Gg = reinterpret_cast<GT *>(p.fields) + R.field_off;
    __syncthreads();
    if (p.init_fields) {
        // g_m = sum_{j != m} J_mj s_j by popcount over the packed rows
        for (int idx = threadIdx.x; idx < NP * npad; idx += blockDim.x) {
            const int t = idx / npad, mm = idx - t * npad;
            int g = 0;
            if (mm < n)
                for (int q = 0; q < nw; ++q) {
                    const int rem = n - 32 * q;
                    uint32_t vm = rem >= 32 ? FULL : ((1u << rem) - 1u);
                    if (q == (mm >> 5)) vm &= ~(1u << (mm & 31));
                    g += 2 * __popc(~(Jw[q * npad + mm] ^ S[t * nw + q]) & vm) - __popc(vm);
                }
            G[idx] = (GT)g;
        }
    } else {
        for (int idx = threadIdx.x; idx < NP * npad; idx += blockDim.x) G[idx] = Gg[idx];
    }
    for (int i = threadIdx.x; i < npad; i += blockDim.x) {
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
                // one visiting order for the sweep; slices in turn, pipelined:
                // slice t takes block q once slice t - 1 has finished it
                const uint32_t tag = p.slice_tag | R.tag_extra;
                pipe_reset(pp, NP);
                const OrdT *ord = feed_take(feed);
                for (int t = warp; t < NP; t += W) {
                    const int tp = t == 0 ? NP - 1 : t - 1, tn = t + 1 == NP ? 0 : t + 1;
                    uint32_t *St = S + t * nw;
                    GT *Gt = G + t * npad;
                    const uint32_t rng_cell = (uint32_t)(slot * NP + t);
                    att_s += (unsigned long long)n;
                    for (int q4 = 0; q4 < nw; q4 += 4) {
                        const U4 r = philox((uint32_t)(((q4 >> 2) << 5) | lane), rng_cell, sigma, tag, R.key);
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const int q = q4 + k;
                            if (q < nw)
                                pm1_block_ord(Jw, St, Gt, Wc, h, ord, n, npad, q, t, tp, tn, pick(r, k), B, T4, lane,
                                              acc_s, pp);
                        }
                    }
                }
                __syncthreads();
            } else {
                for (int ph = 0; ph < 3; ++ph) {
                    const int cnt = phase_count(NP, ph);
                    for (int c = warp; c < cnt; c += W) {
                        const int t = phase_slice(NP, ph, c);
                        pm1_sweep_slice(Jw, S, G, Wc, h, n, nw, npad, NP, t, B, T4, R.key,
                                        (uint32_t)(slot * NP + t), sigma, p.slice_tag | R.tag_extra, lane, att_s,
                                        acc_s);
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
        for (int sw = 0; sw < wls && p.ref_order; ++sw) {
            // qanneal's order: a fresh visiting order; slice sums by spin,
            // uniforms by visiting position
            const uint32_t sigma = (uint32_t)(step * p.wls + sw);
            const OrdT *ord = feed_take(feed);
            for (int i = threadIdx.x; i < npad; i += blockDim.x) {
                const int q = i >> 5;
                int gs = 0;
                if (i < n)
                    for (int t = 0; t < NP; ++t) {
                        const int g = (int)G[t * npad + i];
                        gs += ((S[t * nw + q] >> lane) & 1u) ? g : -g;
                    }
                Gs[i] = gs;
                if ((q & 3) == 0) {  // positions q*32 + lane .. + 96: one Philox call
                    const U4 r = philox((uint32_t)(((q >> 2) << 5) | lane), (uint32_t)slot, sigma, DOM_WORLD, R.key);
                    uw[i] = u24(r.x);
                    uw[i + 32] = u24(r.y);
                    uw[i + 64] = u24(r.z);
                    uw[i + 96] = u24(r.w);
                }
            }
            if (threadIdx.x == 0) att_w += (unsigned long long)n;
            __syncthreads();
            int q0 = 0;
            for (;;) {
                // decisions of every later position on the current worldlines
                for (int pp = threadIdx.x + q0 * 32; pp < npad; pp += blockDim.x) {
                    const bool valid = pp < n;
                    const int i = valid ? ord[pp] : 0;
                    const float y = pm1_world_y(h[i], Wc[i], Gs[i], NP, B);
                    const float u = uw[pp];
                    uint32_t m = 0u;
                    if (__any_sync(FULL, valid & metropolis_maybe24(y, u)))
                        m = __ballot_sync(FULL, valid & metropolis_nb24(y, u));
                    if (lane == 0) mask[pp >> 5] = m;
                }
                __syncthreads();
                int qs = -1;
                for (int q = q0; q < nw; ++q)
                    if (mask[q]) { qs = q; break; }
                if (qs < 0) break;
                if (warp == 0) {
                    // resolve block qs in position order; sums of the block's
                    // later spins corrected by -2 J_ij (P - 2 popc(W_i ^ W_j))
                    const int pos = (qs << 5) | lane;
                    const bool valid = pos < n;
                    const int i = valid ? ord[pos] : 0;
                    const unsigned long long wi = Wc[i];
                    const float hi = h[i], u = uw[pos];
                    int gk = Gs[i];
                    uint32_t m = mask[qs], F = 0;
                    do {
                        const int j = __ffs(m) - 1;
                        F |= 1u << j;
                        const int ij = __shfl_sync(FULL, i, j);
                        const unsigned long long wj = __shfl_sync(FULL, wi, j);
                        const int overlap = NP - 2 * __popcll(wi ^ wj);  // sum_t s_t,i s_t,j
                        if (lane != j)
                            gk += ((Jw[(ij >> 5) * npad + i] >> (ij & 31)) & 1u) ? -2 * overlap : 2 * overlap;
                        const uint32_t pending = j == 31 ? 0u : (FULL << (j + 1));
                        m = __ballot_sync(FULL, valid & metropolis_nb24(pm1_world_y(hi, wi, gk, NP, B), u)) & pending;
                    } while (m);
                    Wold[lane] = wi;
                    Wsp[lane] = i;
                    if (lane == 0) { flag[1] = (int)F; flag[2] = qs; }
                }
                __syncthreads();
                const uint32_t F = (uint32_t)flag[1];
                // later positions: exact correction of their spins' slice sums
                for (int pp = threadIdx.x + (qs + 1) * 32; pp < n; pp += blockDim.x) {
                    const int i = ord[pp];
                    const unsigned long long wi = Wc[i];
                    int dg = 0;
                    for (uint32_t f = F; f; f &= f - 1) {
                        const int j = __ffs(f) - 1, sj = Wsp[j];
                        const int overlap = NP - 2 * __popcll(wi ^ Wold[j]);
                        dg += ((Jw[(sj >> 5) * npad + i] >> (sj & 31)) & 1u) ? -2 * overlap : 2 * overlap;
                    }
                    Gs[i] += dg;
                }
                // every slice: flip the block's flipped spins and update its fields
                const int spl = Wsp[lane];
                for (int t = warp; t < NP; t += W) pm1_flip_spins(S + t * nw, G + t * npad, Jw, npad, n, F, spl, lane);
                if (warp == 0 && ((F >> lane) & 1u)) Wc[spl] = Wold[lane] ^ pmask;
                if (threadIdx.x == 0) acc_w += (unsigned long long)__popc(F);
                __syncthreads();
                q0 = qs + 1;
                if (q0 >= nw) break;
            }
        }
        for (int sw = 0; sw < wls && !p.ref_order; ++sw) {
            const uint32_t sigma = (uint32_t)(step * p.wls + sw);
            // slice sums and uniforms of every spin (thread per spin; a warp
            // holds one 32-spin block, so lane == spin & 31)
            for (int i = threadIdx.x; i < npad; i += blockDim.x) {
                const int q = i >> 5;
                int gs = 0;
                if (i < n)
                    for (int t = 0; t < NP; ++t) {
                        const int g = (int)G[t * npad + i];
                        gs += ((S[t * nw + q] >> lane) & 1u) ? g : -g;
                    }
                Gs[i] = gs;
                if ((q & 3) == 0) {  // one Philox call per lane serves blocks q .. q+3 (npad: a multiple of 128)
                    const U4 r = philox((uint32_t)(((q >> 2) << 5) | lane), (uint32_t)slot, sigma, DOM_WORLD, R.key);
                    uw[i] = u24(r.x);
                    uw[i + 32] = u24(r.y);
                    uw[i + 64] = u24(r.z);
                    uw[i + 96] = u24(r.w);
                }
            }
            if (threadIdx.x == 0) att_w += (unsigned long long)n;
            __syncthreads();
            int q0 = 0;
            for (;;) {
                for (int i = threadIdx.x + q0 * 32; i < npad; i += blockDim.x) {
                    const uint32_t m = pm1_world_ballot(h, Gs, Wc, uw, i, n, NP, B);
                    if (lane == 0) mask[i >> 5] = m;
                }
                __syncthreads();
                int qs = -1;
                for (int q = q0; q < nw; ++q)
                    if (mask[q]) { qs = q; break; }
                // no block with a move: done.  mask[] is written next by the next
                // sweep's decision pass, behind that sweep's barrier after its sums
                if (qs < 0) break;
                if (warp == 0) {
                    // resolve block qs in spin order
                    const int i = (qs << 5) | lane;
                    const unsigned long long wi = Wc[i];
                    const uint32_t jd = Jw[qs * npad + i];
                    int gk = Gs[i];
                    uint32_t m = mask[qs], F = 0;
                    do {
                        const int j = __ffs(m) - 1;
                        F |= 1u << j;
                        const unsigned long long wj = __shfl_sync(FULL, wi, j);
                        const int overlap = NP - 2 * __popcll(wi ^ wj);  // sum_t s_t,i s_t,j
                        if (lane != j) gk += ((jd >> j) & 1u) ? -2 * overlap : 2 * overlap;
                        const uint32_t pending = j == 31 ? 0u : (FULL << (j + 1));
                        Gs[i] = gk;
                        __syncwarp();
                        m = __ballot_sync(FULL, pm1_world_ok(h, Gs, Wc, uw, i, n, NP, B)) & pending;
                        __syncwarp();
                    } while (m);
                    Wold[lane] = wi;
                    if (lane == 0) { flag[1] = (int)F; flag[2] = qs; }
                }
                __syncthreads();
                const uint32_t F = (uint32_t)flag[1];
                // later spins: exact correction of their slice sums
                for (int i = threadIdx.x + (qs + 1) * 32; i < n; i += blockDim.x) {
                    const unsigned long long wi = Wc[i];
                    const uint32_t jd = Jw[qs * npad + i];
                    int dg = 0;
                    for (uint32_t f = F; f; f &= f - 1) {
                        const int j = __ffs(f) - 1;
                        const int overlap = NP - 2 * __popcll(wi ^ Wold[j]);
                        dg += ((jd >> j) & 1u) ? -2 * overlap : 2 * overlap;
                    }
                    Gs[i] += dg;
                }
                // every slice: flip the spins F of block qs and update its fields
                for (int t = warp; t < NP; t += W) {
                    const uint32_t sold = S[t * nw + qs];
                    __syncwarp();
                    if (lane == 0) S[t * nw + qs] = sold ^ F;
                    pm1_block_update(G + t * npad, Jw, npad, n, qs, F, sold, lane);
                }
                if (warp == 0 && ((F >> lane) & 1u)) Wc[(qs << 5) | lane] = Wold[lane] ^ pmask;
                if (threadIdx.x == 0) acc_w += (unsigned long long)__popc(F);
                __syncthreads();
                q0 = qs + 1;
                if (q0 >= nw) break;
            }
        }
        // ---- step end: slice energies E = c + (sum s h + (sum s g)/2), ring sum, best
        for (int t = warp; t < NP; t += W) {
            double ph = 0.0;
            int pg = 0;
            for (int i = lane; i < n; i += 32) {
                const bool up = (S[t * nw + (i >> 5)] >> (i & 31)) & 1u;
                ph = __dadd_rn(ph, up ? (double)h[i] : -(double)h[i]);
                const int g = (int)G[t * npad + i];
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
        // warp 0 alone: ring sum, minimum, records, best and final states (only
        // its lanes keep bestE / bestStep; thread 0 writes them at the end)
        if (warp == 0) {
            int tb = -1, tmin = 0;
            if (lane == 0) {
                double sum = 0.0, emin = __longlong_as_double(0x7ff0000000000000LL);
                for (int t = 0; t < NP; ++t) {
                    const double E = cellE[t];
                    sum = __dadd_rn(sum, E);
                    if (E < emin) { emin = E; tmin = t; }
                }
                const long long ro = (long long)blockIdx.x * p.rec_stride + p.rec_base + step;
                if (p.ring_sum) p.ring_sum[ro] = sum;
                if (p.ring_min) p.ring_min[ro] = emin;
                if (p.ring_bond) {
                    long long bsum = 0;
                    for (int w = 0; w < W; ++w) bsum += wpart[w];
                    p.ring_bond[ro] = bsum;
                }
                tb = emin < bestE ? tmin : -1;
            }
            tb = __shfl_sync(FULL, tb, 0);
            tmin = __shfl_sync(FULL, tmin, 0);
            if (tb >= 0) {
                bestE = cellE[tb];
                bestStep = step;
                if (lane == 0 && p.best_slot) p.best_slot[blockIdx.x] = slot;
                for (int q = lane; q < nw; q += 32) p.best_bits[(long long)blockIdx.x * p.nw_max + q] = S[tb * nw + q];
            }
            if (p.final_bits && step == p.steps_total - 1)
                for (int q = lane; q < nw; q += 32) p.final_bits[(long long)blockIdx.x * p.nw_max + q] = S[tmin * nw + q];
        }
        __syncthreads();  // S is swept again next step
    }
    for (int idx = threadIdx.x; idx < NP * nw; idx += blockDim.x) p.spins[R.spin_off + idx] = S[idx];
    for (int idx = threadIdx.x; idx < NP * npad; idx += blockDim.x) Gg[idx] = G[idx];
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

// ------------------------------------------------------------------ SA, dense +-1
// sa_kernel's run (annealer.cpp:50-67: fixed spin order, running energy, best
// copied on every new minimum; one warp per read) with the couplings as bits
// and exact int32 fields in shared memory: a flip of spin j updates the
// fields from the bits of column j, g_m += -2 J_mj s_j(old), no global loads.
__host__ __device__ inline size_t sa_pm1_smem_bytes(int n) {
    const int nw = (n + 31) / 32, np = pm1_npad(n);
    return (size_t)nw * np * 4 + (size_t)((nw + 3) & ~3) * 4 + (size_t)np * 4 + (size_t)np * 4;
}

__global__ void __launch_bounds__(32) sa_pm1_kernel(SAParams p) {
    extern __shared__ __align__(16) unsigned char smem[];
    const RingDev R = p.rings[blockIdx.x];
    const ProbDev Pd = p.probs[R.prob];
    const int lane = threadIdx.x, n = Pd.n, nw = Pd.nw, npad = pm1_npad(n);
    uint32_t *Jw = reinterpret_cast<uint32_t *>(smem);
    uint32_t *S = Jw + (size_t)nw * npad;
    float *h = reinterpret_cast<float *>(S + ((nw + 3) & ~3));
    int *G = reinterpret_cast<int *>(h + npad);
    for (int idx = lane * 4; idx < nw * npad; idx += 128)
        *reinterpret_cast<uint4 *>(Jw + idx) = __ldg(reinterpret_cast<const uint4 *>(Pd.Jw + idx));
    for (int q = lane; q < nw; q += 32) S[q] = p.spins[R.spin_off + q];
    for (int i = lane; i < npad; i += 32) h[i] = i < n ? Pd.h32[i] : 0.0f;
    __syncwarp();
    for (int m = lane; m < npad; m += 32) {
        int g = 0;
        if (m < n)
            for (int q = 0; q < nw; ++q) {
                const int rem = n - 32 * q;
                uint32_t vm = rem >= 32 ? FULL : ((1u << rem) - 1u);
                if (q == (m >> 5)) vm &= ~(1u << (m & 31));
                g += 2 * __popc(~(Jw[q * npad + m] ^ S[q]) & vm) - __popc(vm);
            }
        G[m] = g;
    }
    __syncwarp();
    // E = c + (sum s h + (sum s g) / 2), sums in warp order (cell_energy)
    double ph = 0.0;
    int pg = 0;
    for (int i = lane; i < n; i += 32) {
        const bool up = (S[i >> 5] >> (i & 31)) & 1u;
        ph = __dadd_rn(ph, up ? (double)h[i] : -(double)h[i]);
        pg += up ? G[i] : -G[i];
    }
    double E = __dadd_rn(Pd.c, __dadd_rn(warp_sum_d(ph), __dmul_rn(0.5, (double)warp_sum_i(pg))));
    uint32_t *bb = p.best_bits + (long long)blockIdx.x * p.nw_max;
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
                const uint32_t sbit = (sword >> lane) & 1u;
                const float u = u24(pick(rnd, q & 3));
                const float hi = h[i];
                att += (unsigned long long)min(32, n - (q << 5));
                uint32_t pending = FULL;
                for (;;) {
                    const float gi = __int2float_rn(G[i]);
                    const float loc = __fadd_rn(hi, gi);
                    const bool ok = valid & metropolis_nb24(__fmul_rn(signed_by_bit(loc, sbit), B), u);
                    const uint32_t m = __ballot_sync(FULL, ok) & pending;
                    if (!m) break;
                    const int j = __ffs(m) - 1;
                    const double xd = sbit ? __dadd_rn((double)hi, (double)gi) : -__dadd_rn((double)hi, (double)gi);
                    const double xj = __shfl_sync(FULL, xd, j);
                    const uint32_t sj = (sword >> j) & 1u;  // old spin bit of j
                    if (lane == 0) S[q] = S[q] ^ (1u << j);
                    const int jj = (q << 5) | j;
                    // g_m += -2 J_mj s_j = 4 (bit_j(row m) ^ s_j) - 2 for every m; the zero
                    // diagonal bit gives spin j's own field 4 s_j - 2, taken back after
                    const uint32_t *Jq = Jw + q * npad;
                    for (int base = lane * 4; base < n; base += 128) {
                        const uint4 jw = *reinterpret_cast<const uint4 *>(Jq + base);
                        int4 g = *reinterpret_cast<int4 *>(G + base);
                        g.x += 4 * (int)(((jw.x >> j) ^ sj) & 1u) - 2;
                        g.y += 4 * (int)(((jw.y >> j) ^ sj) & 1u) - 2;
                        g.z += 4 * (int)(((jw.z >> j) ^ sj) & 1u) - 2;
                        g.w += 4 * (int)(((jw.w >> j) ^ sj) & 1u) - 2;
                        *reinterpret_cast<int4 *>(G + base) = g;
                    }
                    __syncwarp();
                    if (lane == 0) G[jj] -= 4 * (int)sj - 2;
                    __syncwarp();
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
        }
        if (lane == 0) p.trace[(long long)blockIdx.x * p.steps + step] = E;
        if (p.mag_trace) sa_record_mag(p, S, n, nw, step, lane);
    }
    for (int q = lane; q < nw; q += 32) p.spins[R.spin_off + q] = S[q];
    if (lane == 0) {
        p.best_E[blockIdx.x] = best;
        if (p.best_step) p.best_step[blockIdx.x] = bstep;
        atomicAdd(p.counters + 0, att);
        atomicAdd(p.counters + 1, acc);
    }
}

}  // namespace qa
