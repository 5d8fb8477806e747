// qa_chi.cuh -- the chi_B susceptibility of SQA-Chi's pilot scan
// (sqa_chi_annealer.cpp:245-265) from the per-sweep magnetisation sums the
// ring kernels record.
//
// One thread per (read, scan point): the K replica rings of that probe are
// pooled in the reference's order (sweep-major, replica-minor), so the float64
// sums round exactly as the sequential loop's:
//   m = sum / (n P),  chi_B = n P (<m^2> - <|m|>^2), clipped at 0.
#pragma once
#include "qa_device.cuh"

namespace qa {

__global__ void chi_point_kernel(const int *mag, int probes, int K, int sweeps_total, int burn, const int *n_of,
                                 int P, double *chi_out) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= probes) return;
    const int n = n_of[idx];
    const double inv_nM = __ddiv_rn(1.0, (double)(n * P));
    double m2 = 0.0, ma = 0.0;
    long long count = 0;
    for (int sw = burn; sw < sweeps_total; ++sw)
        for (int k = 0; k < K; ++k) {
            const double m = __dmul_rn((double)mag[((long long)idx * K + k) * sweeps_total + sw], inv_nM);
            m2 = __dadd_rn(m2, __dmul_rn(m, m));
            ma = __dadd_rn(ma, fabs(m));
            ++count;
        }
    double chi = 0.0;
    if (count >= 2) {
        const double m2_mean = __ddiv_rn(m2, (double)count), ma_mean = __ddiv_rn(ma, (double)count);
        chi = __dmul_rn((double)(n * P), __dsub_rn(m2_mean, __dmul_rn(ma_mean, ma_mean)));
        if (!(chi > 0.0)) chi = 0.0;
    }
    chi_out[idx] = chi;
}

}  // namespace qa
