// qa_pt.cuh -- per-read bookkeeping of SQA parallel tempering
// (sqa_parallel_tempering.cpp:299-335): replica swaps between neighbouring
// (beta, Gamma) rungs and the per-step traces.
//
// Rung r ("slot") keeps its (beta_r, Gamma_r) and its random streams; a swap
// exchanges which ring sits in which slot, so no spin state is copied.  Pairs
// r = 0..R-2 are visited in order and a swap changes the pair that follows
// (the reference's cascading loop).  The action of a ring x at rung r is
//   S_r(x) = (beta_r/P) sum_t E(x_t) - J_perp(beta_r, Gamma_r) B(x),
// B(x) = sum_t sum_i s_t,i s_t+1,i, from the ring kernel's step-end records.
#pragma once
#include "qa_kernels.cuh"

namespace qa {

struct PTSegParams {
    const RingDev *rings;      // rings of read q are q*R .. q*R+R-1 (ring k started in slot k)
    int reads, R;              // reads of the call (all problems), rungs per read
    int s0, s1;                // steps of this segment
    int swap;                  // swap after step s1-1
    uint32_t round;            // swap round index (counter word of the swap draws)
    const double *bp, *jp;     // [R]: beta_r / P and J_perp(beta_r, Gamma_r, P)
    const double *ring_sum, *ring_min;
    const long long *ring_bond;
    int rec_base, rec_stride;  // record (ring, step) at ring*rec_stride + rec_base + step
    int *ring_in;              // [read][R]: ring (0..R-1) in each slot
    int *slot_of;              // [ring]: slot of each ring
    double *avg_trace, *swap_trace;  // [read][steps_total]
    int steps_total;
};

__global__ void pt_segment_kernel(PTSegParams p) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= p.reads) return;
    const int R = p.R;
    int *rin = p.ring_in + (long long)q * R;
    const long long rb = (long long)q * R;
    const uint64_t key = p.rings[rb].key;
    for (int s = p.s0; s < p.s1; ++s) {
        double acc = 0.0, att = 0.0;
        if (p.swap && s == p.s1 - 1) {
            for (int r = 0; r + 1 < R; ++r) {
                const int a = rin[r], b = rin[r + 1];
                const long long ia = (rb + a) * p.rec_stride + p.rec_base + s;
                const long long ib = (rb + b) * p.rec_stride + p.rec_base + s;
                const double e_aa = __dsub_rn(__dmul_rn(p.bp[r], p.ring_sum[ia]), __dmul_rn(p.jp[r], (double)p.ring_bond[ia]));
                const double e_bb =
                    __dsub_rn(__dmul_rn(p.bp[r + 1], p.ring_sum[ib]), __dmul_rn(p.jp[r + 1], (double)p.ring_bond[ib]));
                const double e_ab = __dsub_rn(__dmul_rn(p.bp[r], p.ring_sum[ib]), __dmul_rn(p.jp[r], (double)p.ring_bond[ib]));
                const double e_ba =
                    __dsub_rn(__dmul_rn(p.bp[r + 1], p.ring_sum[ia]), __dmul_rn(p.jp[r + 1], (double)p.ring_bond[ia]));
                const double delta = __dsub_rn(__dadd_rn(e_ab, e_ba), __dadd_rn(e_aa, e_bb));
                att += 1.0;
                const float u = u01(philox((uint32_t)r, 0u, p.round, DOM_SWAP, key).x);
                if (metropolis(__double2float_rn(-delta), u)) {
                    rin[r] = b;
                    rin[r + 1] = a;
                    p.slot_of[rb + b] = r;
                    p.slot_of[rb + a] = r + 1;
                    acc += 1.0;
                }
            }
        }
        double avg = 0.0;
        for (int r = 0; r < R; ++r) avg = __dadd_rn(avg, p.ring_min[(rb + rin[r]) * p.rec_stride + p.rec_base + s]);
        p.avg_trace[(long long)q * p.steps_total + s] = __ddiv_rn(avg, (double)R);
        p.swap_trace[(long long)q * p.steps_total + s] = att > 0.0 ? __ddiv_rn(acc, att) : 0.0;
    }
}

}  // namespace qa
