// Problem ingestion on the device: QUBO::to_ising (qubo.cpp:33-69) and the
// arrays the sweep kernels derive from a dense model (the float32 mirror of the
// upper triangle and the bit-packed rows of a +-1 model).
#pragma once

#include <cstdint>

namespace qa {

constexpr int kIngestTile = 32;

// Rows of QUBO::to_ising, one CTA (32 x 8 threads) per 32 rows, column tiles
// staged through shared memory so every global access is coalesced:
//   W[i][j] = 0.5 (Q[i][j] + Q[j][i])     (qubo.cpp:35-41)
//   J64[i][j] = 0.5 W[i][j], full matrix   (qubo.cpp:63)
//   h64[i] = 0.5 sum_j W[i][j]             (qubo.cpp:48-54), summed in column
//                                          order by one thread per row
//   h32[i] = (float) h64[i]
// The constant c is one running sum over every (i, j) and is left to the host.
__global__ void qubo_rows_kernel(const double *__restrict__ Q, int n, double *__restrict__ J64,
                                 double *__restrict__ h64, float *__restrict__ h32) {
    __shared__ double A[kIngestTile][kIngestTile + 1];   // Q[r0 + y][c0 + x]
    __shared__ double Bt[kIngestTile][kIngestTile + 1];  // Q[c0 + y][r0 + x]
    __shared__ double W[kIngestTile][kIngestTile + 1];   // W[r0 + y][c0 + x]
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int r0 = blockIdx.x * kIngestTile;
    double acc = 0.0;  // row r0 + tx, kept by the threads with ty == 0
    for (int c0 = 0; c0 < n; c0 += kIngestTile) {
        for (int y = ty; y < kIngestTile; y += blockDim.y) {
            const int i = r0 + y, j = c0 + tx;
            A[y][tx] = (i < n && j < n) ? Q[(size_t)i * n + j] : 0.0;
            const int i2 = c0 + y, j2 = r0 + tx;
            Bt[y][tx] = (i2 < n && j2 < n) ? Q[(size_t)i2 * n + j2] : 0.0;
        }
        __syncthreads();
        for (int y = ty; y < kIngestTile; y += blockDim.y) {
            const int i = r0 + y, j = c0 + tx;
            const double w = 0.5 * (A[y][tx] + Bt[tx][y]);
            W[y][tx] = w;
            if (i < n && j < n) J64[(size_t)i * n + j] = 0.5 * w;
        }
        __syncthreads();
        if (ty == 0 && r0 + tx < n) {
            const int cols = min(kIngestTile, n - c0);
            for (int k = 0; k < cols; ++k) acc = __dadd_rn(acc, W[tx][k]);
        }
        __syncthreads();
    }
    if (ty == 0 && r0 + tx < n) {
        const double hv = 0.5 * acc;
        h64[r0 + tx] = hv;
        h32[r0 + tx] = __double2float_rn(hv);
    }
}

// Derived dense arrays, one CTA (32 x 8 threads) per 32 x 32 tile (row tile
// blockIdx.y, column tile blockIdx.x).  The upper triangle of J64 defines the
// model (DenseIsing::energy reads i < j):
//   J32[i][j] = (float) J64[min(i,j)][max(i,j)] for i != j, 0 on the diagonal
//   Jw[q * np + m]: bit (j & 31) of row m, column word q = (J32[m][j] > 0), j != m
//   *not_pm1 = 1 when an upper off-diagonal entry is neither +1 nor -1.
// Jw must be zeroed beforehand (rows n .. np-1 stay 0).
__global__ void dense_derive_kernel(const double *__restrict__ J64, int n, float *__restrict__ J32,
                                    uint32_t *__restrict__ Jw, int np, int *__restrict__ not_pm1) {
    __shared__ double S[kIngestTile][kIngestTile + 1];  // J64[a0 + y][b0 + x]
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int bx = blockIdx.x, by = blockIdx.y;
    const int a0 = kIngestTile * min(bx, by), b0 = kIngestTile * max(bx, by);
    for (int y = ty; y < kIngestTile; y += blockDim.y) {
        const int i = a0 + y, j = b0 + tx;
        S[y][tx] = (i < n && j < n) ? J64[(size_t)i * n + j] : 0.0;
    }
    __syncthreads();
    const int r0 = kIngestTile * by, c0 = kIngestTile * bx;
    bool bad = false;
    for (int y = ty; y < kIngestTile; y += blockDim.y) {
        const int i = r0 + y, j = c0 + tx;
        const bool in = i < n && j < n;
        const int lo = min(i, j), hi = max(i, j);
        const double v = (in && i != j) ? S[lo - a0][hi - b0] : 0.0;
        if (in && i < j && v != 1.0 && v != -1.0) bad = true;
        if (in) J32[(size_t)i * n + j] = i == j ? 0.0f : __double2float_rn(v);
        const float f = __double2float_rn(v);
        const uint32_t word = __ballot_sync(0xffffffffu, in && i != j && f > 0.0f);
        if (tx == 0 && i < n) Jw[(size_t)bx * np + i] = word;
    }
    if (__any_sync(0xffffffffu, bad) && tx == 0) *not_pm1 = 1;
}

}  // namespace qa
