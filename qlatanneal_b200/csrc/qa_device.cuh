// qa_device.cuh -- device primitives of the sweep engine: the counter RNG, the
// deterministic float32 logarithm of the Metropolis threshold, warp helpers
// and the three local-field models (dense, sparse CSR, higher-order).
//
// Numerical contract (shared with the CPU restatement used by the tests):
//   * Philox4x32-10 (Salmon et al., SC'11), key = seed + read,
//     counter = (spin slot, cell, sweep, domain tag).
//   * Local fields g = J.s in float32 with h kept apart; couplings rounded to
//     float32; initial fields accumulated in float64 then rounded.
//   * Metropolis on y = -dE = x*B - trotter, x = s*(h+g), B = 2*beta/P
//     (2*beta for SA): accept iff y >= 0 or (y > -17 and u < e^y), the rule
//     "dE <= 0 || u < exp(-dE)" of sqa_annealer.cpp:196-205 with a
//     deterministic float32 e^y.
//   * Every float op that feeds a decision is an explicit round-to-nearest
//     intrinsic, so no FMA contraction changes a bit.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace qa {

constexpr unsigned FULL = 0xffffffffu;

enum Dom : uint32_t {
    DOM_INIT = 1, DOM_SA = 2, DOM_SLICE = 3, DOM_WORLD = 4, DOM_SWAP = 5,
    DOM_PILOT_INIT = 6, DOM_PILOT = 7, DOM_PROD_INIT = 8, DOM_PROD = 9, DOM_CSPIN = 10, DOM_CBOND = 11,
    DOM_OPTCAL = 12, DOM_PERM = 13
};

enum Kind : int { K_DENSE = 0, K_SPARSE = 1, K_HUBO = 2 };

// ---------------------------------------------------------------- Philox
struct U4 { uint32_t x, y, z, w; };

__device__ __forceinline__ U4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint64_t key) {
    uint32_t k0 = (uint32_t)key, k1 = (uint32_t)(key >> 32);
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    return U4{c0, c1, c2, c3};
}

__device__ __forceinline__ uint32_t pick(const U4 &r, int w) {
    return w == 0 ? r.x : (w == 1 ? r.y : (w == 2 ? r.z : r.w));
}

// Counter slot of a spin: 4 consecutive 32-spin blocks share one Philox call,
// lane-strided, so one call per lane serves four blocks.
__device__ __forceinline__ uint32_t spin_slot(int i) { return (uint32_t)(((i >> 7) << 5) | (i & 31)); }

__device__ __forceinline__ float u01(uint32_t x) { return __uint2float_rn(x >> 8) * (1.0f / 16777216.0f); }

// The same uniform scaled by 2^24: the integer x >> 8 as a float (exact), so
// that u24(x) = u01(x) * 2^24 without the multiply.
__device__ __forceinline__ float u24(uint32_t x) { return __uint2float_rn(x >> 8); }

// Deterministic float32 e^y for y in (-17, 0]: y*log2(e) split into its
// nearest integer k and a remainder f in [-1/2, 1/2]; 2^f by its Taylor series
// (coefficients ln2^n/n!, n <= 6, Horner); 2^k added to the exponent field.
// Each step is one IEEE round-to-nearest op, reproduced bit for bit by the
// CPU restatement.
// det_expf(y) * 2^scale_log2: the scaling is folded into the exponent add,
// exact while the result stays a normal float.
template <int SCALE_LOG2 = 0>
__device__ __forceinline__ float det_expf_scaled(float y) {
    const float t = __fmul_rn(y, 1.44269504f);
    const int k = __float2int_rn(t);
    const float f = __fsub_rn(t, __int2float_rn(k));
    float p = __fmaf_rn(1.5403530e-4f, f, 1.3333558e-3f);
    p = __fmaf_rn(p, f, 9.6181291e-3f);
    p = __fmaf_rn(p, f, 5.5504109e-2f);
    p = __fmaf_rn(p, f, 2.4022651e-1f);
    p = __fmaf_rn(p, f, 6.9314718e-1f);
    p = __fmaf_rn(p, f, 1.0f);
    return __int_as_float(__float_as_int(p) + ((k + SCALE_LOG2) << 23));
}
__device__ __forceinline__ float det_expf(float y) { return det_expf_scaled<0>(y); }

// Metropolis decision on y = -dE: qanneal accepts iff dE <= 0 || u < exp(-dE)
// (annealer.cpp:55, sqa_annealer.cpp:198).  Moves with y <= -17 are rejected
// outright: e^-17 = 4.1e-8 is below the finest step of u (2^-24).
__device__ __forceinline__ bool metropolis(float y, float u) {
    return y >= 0.0f || (y > -17.0f && u < det_expf(y));
}

// The same decision without divergent branches, on the scaled uniform
// u24 = u * 2^24: e^y * 2^24 is evaluated on y clamped to [-17, 0]; at y >= 0
// it is exactly 2^24, above every u24 (at most 2^24 - 1), and the power-of-two
// scaling is exact on both sides, so the result is identical to
// metropolis(y, u).
__device__ __forceinline__ bool metropolis_nb24(float y, float u24v) {
    return (y > -17.0f) & (u24v < det_expf_scaled<24>(fminf(fmaxf(y, -17.0f), 0.0f)));
}

// False only when metropolis_nb24(y, u24v) is false, without the exponential.
// With t = y log2(e): det_expf_scaled<24>(y) = p 2^(k + 24), p within 1e-6 of
// 2^(t - k) (degree-6 Taylor remainder on [-1/2, 1/2] plus the roundings), so
// log2 of it is below t + 24 + 1e-5; at y >= 0 it is 2^24.  The float bits of
// u24v give bits / 2^23 - 127 = e + m <= e + log2(1 + m) = log2(u24v).  Hence
// bits(u24v) >= (t + 151.001) 2^23 implies u24v > e^y 2^24: rejected.  The
// 0.001 margin covers this test's own roundings (the fused multiply-add of a
// value near 2^30: below 1e-5 in log2 units) a hundred times over.  y <= -17
// and non-finite y land on either side; metropolis_nb24 rejects them anyway.
__device__ __forceinline__ bool metropolis_maybe24(float y, float u24v) {
    const int K = __float2int_ru(__fmaf_rn(y, 1.44269504f * 8388608.0f, 151.001f * 8388608.0f));
    return __float_as_int(u24v) < K;
}

__device__ __forceinline__ float f_inf() { return __int_as_float(0x7f800000); }

// float64 warp sum in the canonical order: lane-strided partials (already in
// v), then an xor butterfly; every lane ends with the same value.
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) v = __dadd_rn(v, __shfl_xor_sync(FULL, v, off));
    return v;
}
__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) v += __shfl_xor_sync(FULL, v, off);
    return v;
}

// ---------------------------------------------------------------- models
// Device view of one problem instance (all arrays in global memory, L2-resident).
struct ProbDev {
    int kind, n, nw, T, m;
    double c;
    const float *h32;
    const double *h64;
    // dense: J32 row-major n x n (symmetric, zero diagonal), J64 as given
    const float *J32;
    const double *J64;
    // sparse: merged adjacency CSR + original edge list (float64 energy)
    const int *rowptr, *col;
    const float *val32;
    const int *ei, *ej;
    const double *ew;
    // hubo: consolidated terms + incidence lists
    const int *incptr, *incterm, *tptr, *tvars;
    const float *coef32;
    const double *coef64;
    // dense with every coupling in {-1,+1}: bit-packed rows, Jw[q*np + m] =
    // bits J[m][32q .. 32q+31] (1 = +1; diagonal and padding bits 0); else null
    const uint32_t *Jw;
    // hubo with every term of degree <= 4: the field updates of a flip of
    // spin j grouped by target.  Runs upd_run[upd_ptr[j] .. upd_ptr[j+1]) of
    // j; run r = records upd_rec[upd_run[r] .. upd_run[r+1]), one target v,
    // its terms in increasing term order; record = {v, w1, w2, bits(2 J_t)}
    // with w1, w2 the term's other spins (-1: none).  Else null.
    const int *upd_ptr, *upd_run;
    const int4 *upd_rec;
    // hubo with every term of degree <= 4: term t's spins {v0, v1, v2, v3}
    // (-1: none) in one 16-byte record, for the per-step energy scan; else null
    const int4 *trec;
    // sparse with integer couplings: CSR (column, value) pairs; else null
    const int2 *spcv;
    // sparse with integer couplings in [-127, 127], at most 4 neighbours a
    // spin and n < 65536: spin i's row in one 16-byte record {c0 | c1 << 16,
    // c2 | c3 << 16, int8 values v0 .. v3, 0} (unused entries: column 0,
    // value 0), the same neighbours and values as its CSR row; else null
    const uint4 *spslab;
};

__device__ __forceinline__ int spin_of(const uint32_t *S, int i) { return ((S[i >> 5] >> (i & 31)) & 1u) ? 1 : -1; }

// Field update after spin j (old value so) flipped in one slice whose spin bits
// (already holding the new value) are S and whose fields are g.  Whole warp
// calls it; ends with __syncwarp.  Update order per field is the flip order,
// identical to the sequential restatement (dense_ising.cpp:88-106,
// sparse_ising.cpp:90-102, higher_order_ising.cpp:167-189).
template <int KIND>
__device__ __forceinline__ void apply_flip(const ProbDev &P, float *g, const uint32_t *S, int j, int so, int lane) {
    const float cf = so > 0 ? -2.0f : 2.0f;
    if (KIND == K_DENSE) {
        const float *row = P.J32 + (size_t)j * P.n;
        for (int m = lane; m < P.n; m += 32)
            if (m != j) g[m] = __fadd_rn(g[m], __fmul_rn(cf, __ldg(row + m)));
    } else if (KIND == K_SPARSE) {
        const int e0 = __ldg(P.rowptr + j), e1 = __ldg(P.rowptr + j + 1);
        for (int e = e0 + lane; e < e1; e += 32) {
            const int m = __ldg(P.col + e);
            g[m] = __fadd_rn(g[m], __fmul_rn(cf, __ldg(P.val32 + e)));
        }
    } else if (P.upd_rec) {
        // one lane per target spin v, its terms in order: the same float
        // additions, in the same order per field, as the term-by-term loop
        const int sj = spin_of(S, j);  // S holds the new spin
        const int r0 = __ldg(P.upd_ptr + j), r1 = __ldg(P.upd_ptr + j + 1);
        for (int r = r0 + lane; r < r1; r += 32) {
            const int a = __ldg(P.upd_run + r), b = __ldg(P.upd_run + r + 1);
            for (int k = a; k < b; ++k) {
                const int4 rc = __ldg(P.upd_rec + k);
                int pr = sj;
                if (rc.y >= 0) pr *= spin_of(S, rc.y);
                if (rc.z >= 0) pr *= spin_of(S, rc.z);
                const float two = __int_as_float(rc.w);
                g[rc.x] = __fadd_rn(g[rc.x], pr > 0 ? two : -two);
            }
        }
    } else {
        const int q0 = __ldg(P.incptr + j), q1 = __ldg(P.incptr + j + 1);
        for (int q = q0; q < q1; ++q) {
            const int t = __ldg(P.incterm + q);
            const int a = __ldg(P.tptr + t), d = __ldg(P.tptr + t + 1) - a;
            // sign of the product of the term's (new) spins
            int neg = 0;
            for (int base = 0; base < d; base += 32) {
                const int k = base + lane;
                const bool in = k < d;
                const int v = in ? __ldg(P.tvars + a + k) : 0;
                neg ^= __popc(__ballot_sync(FULL, in && spin_of(S, v) < 0)) & 1;
            }
            const float two = __fmul_rn(2.0f, __ldg(P.coef32 + t));
            for (int base = 0; base < d; base += 32) {
                const int k = base + lane;
                if (k < d) {
                    const int v = __ldg(P.tvars + a + k);
                    if (v != j) {
                        const int sv = spin_of(S, v);
                        const bool pos = (neg == 0) == (sv > 0);
                        g[v] = __fadd_rn(g[v], pos ? two : -two);
                    }
                }
            }
            __syncwarp();
        }
    }
    __syncwarp();
}

// Local field of spin i (J.s part, no h), accumulated in float64 in the
// model's natural order, then rounded: the field-cache initialisation.
template <int KIND>
__device__ __forceinline__ double field_exact64(const ProbDev &P, const uint32_t *S, int i) {
    double acc = 0.0;
    if (KIND == K_DENSE) {
        // J32 is symmetric: read column i (coalesced across the lanes' rows)
        for (int j = 0; j < P.n; ++j) {
            const double w = (double)__ldg(P.J32 + (size_t)j * P.n + i);
            acc = __dadd_rn(acc, spin_of(S, j) > 0 ? w : -w);
        }
    } else if (KIND == K_SPARSE) {
        for (int e = __ldg(P.rowptr + i); e < __ldg(P.rowptr + i + 1); ++e) {
            const double w = (double)__ldg(P.val32 + e);
            acc = __dadd_rn(acc, spin_of(S, __ldg(P.col + e)) > 0 ? w : -w);
        }
    } else {
        for (int q = __ldg(P.incptr + i); q < __ldg(P.incptr + i + 1); ++q) {
            const int t = __ldg(P.incterm + q);
            int sg = 1;
            for (int k = __ldg(P.tptr + t); k < __ldg(P.tptr + t + 1); ++k) {
                const int v = __ldg(P.tvars + k);
                if (v != i) sg *= spin_of(S, v);
            }
            const double w = (double)__ldg(P.coef32 + t);
            acc = __dadd_rn(acc, sg > 0 ? w : -w);
        }
    }
    return acc;
}

template <int KIND>
__device__ __forceinline__ float field_init_one(const ProbDev &P, const uint32_t *S, int i) {
    return __double2float_rn(field_exact64<KIND>(P, S, i));
}

// Tracking energy of one slice from its field cache (whole warp, all lanes
// return the same value):
//   quadratic: E = c + (sum_i s_i h_i + (sum_i s_i g_i) / 2)
//   HUBO:      E = c + (sum_i s_i h_i + sum_t J_t prod_t s)
// in float64, each sum in canonical warp order.
template <int KIND>
__device__ __forceinline__ double cell_energy(const ProbDev &P, const uint32_t *S, const float *g, const float *h32,
                                              int lane) {
    double ph = 0.0;
    for (int i = lane; i < P.n; i += 32) ph = __dadd_rn(ph, spin_of(S, i) > 0 ? (double)h32[i] : -(double)h32[i]);
    ph = warp_sum_d(ph);
    if (KIND != K_HUBO) {
        double pg = 0.0;
        for (int i = lane; i < P.n; i += 32) pg = __dadd_rn(pg, spin_of(S, i) > 0 ? (double)g[i] : -(double)g[i]);
        return __dadd_rn(P.c, __dadd_rn(ph, __dmul_rn(0.5, warp_sum_d(pg))));
    }
    double pj = 0.0;
    for (int t = lane; t < P.T; t += 32) {
        int sg = 1;
        for (int k = __ldg(P.tptr + t); k < __ldg(P.tptr + t + 1); ++k) sg *= spin_of(S, __ldg(P.tvars + k));
        const double w = (double)__ldg(P.coef32 + t);
        pj = __dadd_rn(pj, sg > 0 ? w : -w);
    }
    pj = warp_sum_d(pj);
    return __dadd_rn(P.c, __dadd_rn(ph, pj));
}

// 1 when spin v of the bits S is down (-1).
__device__ __forceinline__ uint32_t down_bit(const uint32_t *S, int v) { return ~(S[v >> 5] >> (v & 31)) & 1u; }

// cell_energy<K_HUBO> of two slices Sa, Sb in one pass over the term records:
// every term's sign is the parity of its down spins.  Each slice's sums take
// the spins and terms in cell_energy's order, so both results equal it bit
// for bit; the records are read once for the two slices.
__device__ __forceinline__ void hubo_energy2(const ProbDev &P, const uint32_t *Sa, const uint32_t *Sb,
                                             const float *h32, int lane, double *Ea, double *Eb) {
    double ha = 0.0, hb = 0.0;
    for (int i = lane; i < P.n; i += 32) {
        const double hv = (double)h32[i];
        ha = __dadd_rn(ha, spin_of(Sa, i) > 0 ? hv : -hv);
        hb = __dadd_rn(hb, spin_of(Sb, i) > 0 ? hv : -hv);
    }
    double ja = 0.0, jb = 0.0;
    for (int t = lane; t < P.T; t += 32) {
        const int4 r = __ldg(P.trec + t);
        const double w = (double)__ldg(P.coef32 + t);
        uint32_t da = down_bit(Sa, r.x) ^ down_bit(Sa, r.y), db = down_bit(Sb, r.x) ^ down_bit(Sb, r.y);
        if (r.z >= 0) {
            da ^= down_bit(Sa, r.z);
            db ^= down_bit(Sb, r.z);
        }
        if (r.w >= 0) {
            da ^= down_bit(Sa, r.w);
            db ^= down_bit(Sb, r.w);
        }
        ja = __dadd_rn(ja, da ? -w : w);
        jb = __dadd_rn(jb, db ? -w : w);
    }
    *Ea = __dadd_rn(P.c, __dadd_rn(warp_sum_d(ha), warp_sum_d(ja)));
    *Eb = __dadd_rn(P.c, __dadd_rn(warp_sum_d(hb), warp_sum_d(jb)));
}

// Float64 energy from the ORIGINAL float64 coefficients (reported energies).
template <int KIND>
__device__ __forceinline__ double exact_energy(const ProbDev &P, const uint32_t *S, int lane) {
    double p = 0.0;
    for (int i = lane; i < P.n; i += 32) p = __dadd_rn(p, spin_of(S, i) > 0 ? P.h64[i] : -P.h64[i]);
    if (KIND == K_DENSE) {
        for (int i = lane; i < P.n; i += 32) {
            const double *row = P.J64 + (size_t)i * P.n;
            double r = 0.0;
            for (int j = i + 1; j < P.n; ++j) r = __dadd_rn(r, spin_of(S, j) > 0 ? row[j] : -row[j]);
            p = __dadd_rn(p, spin_of(S, i) > 0 ? r : -r);
        }
    } else if (KIND == K_SPARSE) {
        for (int e = lane; e < P.m; e += 32) {
            const double w = P.ew[e];
            p = __dadd_rn(p, spin_of(S, P.ei[e]) * spin_of(S, P.ej[e]) > 0 ? w : -w);
        }
    } else {
        for (int t = lane; t < P.T; t += 32) {
            int sg = 1;
            for (int k = P.tptr[t]; k < P.tptr[t + 1]; ++k) sg *= spin_of(S, P.tvars[k]);
            p = __dadd_rn(p, sg > 0 ? P.coef64[t] : -P.coef64[t]);
        }
    }
    return __dadd_rn(P.c, warp_sum_d(p));
}

}  // namespace qa
