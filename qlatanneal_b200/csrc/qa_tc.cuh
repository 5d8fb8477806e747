// qa_tc.cuh -- the initial local fields H = J.S of every Trotter cell on the
// tensor cores (tcgen05, int8 x int8 -> int32, accumulators in TMEM).
//
// DenseIsing::compute_local_fields (dense_ising.cpp:64-83) for all cells of a
// run at once: G[c][m] = sum_j S[c][j] J[m][j], S the +-1 spins of cell c
// (ring, slice), J the couplings with a zero diagonal.  For couplings that
// are integers in [-127, 127] the int8 products and int32 sums are exact, so
// the result equals the float64-accumulated field init bit for bit and the
// fields (float32 for the generic ring kernels) are unchanged.
//
// One CTA of four warps computes a tile of 128 cells (TMEM lanes) x 256 fields
// (TMEM columns), K in steps of 64 couplings:
//  * the warps stage the step's S tile (cells x 64, from the packed spin
//    bits) and J tile (fields x 64, int8 rows) in shared memory in the
//    canonical K-major layout without swizzle: 16-byte core-matrix rows, eight
//    rows of a core matrix 16 bytes apart, 8-row groups 128 bytes apart (SBO),
//    16-byte K chunks one tile column apart (LBO);
//  * after fence.proxy.async (the writes become visible to the tensor core),
//    one thread issues two tcgen05.mma of K = 32 and commits them to an
//    mbarrier; the CTA waits on it (bounded) before restaging;
//  * the epilogue: each warp reads its 32 TMEM lanes with tcgen05.ld and
//    writes its cells' fields.
// No TMA: the spin tile is built from bits anyway, and J rows are read once
// per tile with 16-byte loads.
#pragma once
#include "qa_kernels.cuh"

namespace qa {

constexpr int TC_M = 128, TC_N = 256, TC_K = 64;

struct TcFieldParams {
    const RingDev *rings;    // rings of one problem, ring0 .. ring0 + n_rings - 1
    const uint32_t *spins;
    float *fields;
    const int8_t *J8;        // [round_up(n, TC_N)][ldj] int8, zero padded, zero diagonal
    int ldj;                 // round_up(n, TC_K)
    int n, nw, P, n_cells;   // cells = rings x P
    unsigned long long *err; // error word: QA_DEV_ERR_TIMEOUT when the MMA wait runs out
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, K-major, no swizzle (version 1 for tcgen05).
__device__ __forceinline__ uint64_t tc_smem_desc(const void *tile, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((smem_u32(tile) >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version
    return d;                // base offset 0, layout type 0 (no swizzle)
}

// Instruction descriptor: D s32, A and B s8, both K-major, N = 256, M = 128.
constexpr uint32_t TC_IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                              ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(TC_IDESC), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// Bounded wait for the mbarrier phase `parity`; false when it ran out.
__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t parity) {
    for (int it = 0; it < (1 << 24); ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
        if (it > 64) __nanosleep(64);
    }
    return false;
}

__global__ void __launch_bounds__(128, 1) tc_fields_kernel(TcFieldParams p) {
    __shared__ __align__(1024) uint8_t sA[TC_M * TC_K];  // cells x 64 couplings
    __shared__ __align__(1024) uint8_t sB[TC_N * TC_K];  // fields x 64 couplings
    __shared__ __align__(8) unsigned long long mbar;
    __shared__ uint32_t tmem_base;
    __shared__ int failed;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int c0 = blockIdx.x * TC_M, f0 = blockIdx.y * TC_N;
    const int n = p.n, nw = p.nw, P = p.P;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"((uint32_t)TC_N));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        failed = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;
    const uint32_t mb = smem_u32(&mbar);

    // the packed spin words of this thread's staging rows: cell c0 + r
    uint32_t phase = 0;
    for (int k0 = 0; k0 < p.ldj; k0 += TC_K) {
        // S tile: 128 cells x 4 chunks of 16 spins, one 16-byte row per item
        for (int it = tid; it < TC_M * 4; it += 128) {
            const int r = it & (TC_M - 1), ch = it >> 7;
            const int c = c0 + r, k = k0 + 16 * ch;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (c < p.n_cells && k < n) {
                const RingDev R = p.rings[c / P];
                const uint32_t *Sw = p.spins + R.spin_off + (long long)(c % P) * nw;
                uint32_t bits = (Sw[k >> 5] >> (k & 16)) & 0xFFFFu;  // spins k .. k+15 (k is a multiple of 16)
                const int valid = min(16, n - k);
                uint32_t b[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    uint32_t w = 0;
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const int jj = 4 * q + e;
                        const uint32_t v8 = jj < valid ? (((bits >> jj) & 1u) ? 0x01u : 0xFFu) : 0u;  // +1 / -1 / 0
                        w |= v8 << (8 * e);
                    }
                    b[q] = w;
                }
                v = make_uint4(b[0], b[1], b[2], b[3]);
            }
            *reinterpret_cast<uint4 *>(sA + ch * (TC_M * 16) + (r >> 3) * 128 + (r & 7) * 16) = v;
        }
        // J tile: 256 fields x 4 chunks of 16 couplings
        for (int it = tid; it < TC_N * 4; it += 128) {
            const int r = it & (TC_N - 1), ch = it >> 8;
            const uint4 v = *reinterpret_cast<const uint4 *>(p.J8 + (long long)(f0 + r) * p.ldj + k0 + 16 * ch);
            *reinterpret_cast<uint4 *>(sB + ch * (TC_N * 16) + (r >> 3) * 128 + (r & 7) * 16) = v;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            // two MMAs of K = 32: chunks 0-1, then chunks 2-3 (LBO = one chunk column)
            tc_mma(tmem, tc_smem_desc(sA, TC_M * 16, 128), tc_smem_desc(sB, TC_N * 16, 128), k0 > 0 ? 1u : 0u);
            tc_mma(tmem, tc_smem_desc(sA + 2 * TC_M * 16, TC_M * 16, 128),
                   tc_smem_desc(sB + 2 * TC_N * 16, TC_N * 16, 128), 1u);
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mb)
                         : "memory");
        }
        if (!tc_wait(mb, phase) && lane == 0) failed = 1;
        phase ^= 1u;
        __syncthreads();
        if (failed) break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (!failed) {
        // epilogue: warp w holds cells c0 + 32w .. c0 + 32w + 31 (its TMEM lanes)
        const int c = c0 + 32 * warp + lane;
        float *g = nullptr;
        if (c < p.n_cells) {
            const RingDev R = p.rings[c / P];
            g = p.fields + R.field_off + (long long)(c % P) * n;
        }
        for (int col = 0; col < TC_N; col += 8) {
            uint32_t v[8];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                : "r"(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)col));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (g) {
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    const int m = f0 + col + e;
                    if (m < n) g[m] = (float)(int)v[e];
                }
            }
        }
    } else if (tid == 0) {
        atomicExch(p.err, QA_DEV_ERR_TIMEOUT);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)TC_N));
}

// The int8 coupling rows of a dense problem with integer couplings in
// [-127, 127]: [rows][ldj], zero padded, zero diagonal (J32 has one).
__global__ void tc_pack_couplings_kernel(const float *J32, int n, int ldj, int rows, int8_t *J8) {
    const long long total = (long long)rows * ldj;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int m = (int)(idx / ldj), j = (int)(idx - (long long)m * ldj);
        J8[idx] = (m < n && j < n) ? (int8_t)(int)J32[(long long)m * n + j] : (int8_t)0;
    }
}

// 1 when every coupling is an integer in [-127, 127].
__global__ void tc_int8_check_kernel(const float *J32, long long count, int *ok) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        const float v = J32[i];
        if (!(v == rintf(v) && fabsf(v) <= 127.0f)) atomicExch(ok, 0);
    }
}

}  // namespace qa
