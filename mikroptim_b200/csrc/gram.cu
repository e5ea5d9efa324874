// Normal equations G = [J r]^T [J r] per run (A = J^T J in the top-left P x P block,
// g = J^T r in column P, r^T r in the corner).
//
// Two kernels:
//   gram_exact_kernel -- every entry is one fused multiply-add chain over the rows in ascending
//     order, acc = fma(u_r, v_r, acc) from acc = 0: bit-identical to the reference's
//     normal_equations_host / gram_dot (include/mikroptim/optim/normal_equations.hpp:19,33).
//     One CTA per run streams row tiles through shared memory; each thread advances the chains
//     of its entries tile by tile.
//   gram_dmma_kernel -- FP64 tensor cores: mma.sync.m8n8k4 (f64) on 8 x 8 output tiles of the
//     upper triangle, row tiles of J staged in shared memory; fixed k order (deterministic, not
//     bit-identical to the chain).
#include "launch.cuh"

namespace mkb {

namespace {

constexpr int kGramThreads = 256;
constexpr int kExactRows = 64;   // rows per shared tile (exact kernel)
constexpr int kMaxCols = MKB_MAX_VARIABLES + 1;
constexpr int kExactStride = kExactRows + 1;  // padded column stride (bank spread)
constexpr int kMaxPairsPerThread = (kMaxCols * (kMaxCols + 1) / 2 + kGramThreads - 1) / kGramThreads;

// Column c of run `run`: J columns are strided by `stride` per run (the largest P of an uneven
// batch, else P); column P is the residual.
__device__ inline const double* column(const double* J, const double* r, int64_t run, int c,
                                       int P, int stride, int64_t R) {
    return c < P ? J + (run * stride + c) * R : r + run * R;
}

__global__ void __launch_bounds__(kGramThreads)
gram_exact_kernel(const double* __restrict__ J, const double* __restrict__ r, int P_all,
                  int64_t R, double* __restrict__ gram, const int* __restrict__ run_mask,
                  const VarParams* __restrict__ vt, int stride) {
    __shared__ double tile[kMaxCols * kExactStride];
    const int64_t run = blockIdx.x;
    if (run_mask != nullptr && run_mask[run] == 0) return;
    const int P = vt != nullptr ? vt[run].P : P_all;
    const int n = P + 1;
    const int pairs = n * (n + 1) / 2;
    // pair index -> (p, q), p <= q, row-major over the upper triangle
    int pp[kMaxPairsPerThread], qq[kMaxPairsPerThread];
    double acc[kMaxPairsPerThread];
    int mine = 0;
    for (int e = threadIdx.x; e < pairs; e += kGramThreads) {
        int q = 0, rem = e;
        while (rem >= q + 1) {
            rem -= q + 1;
            ++q;
        }
        pp[mine] = rem;
        qq[mine] = q;
        acc[mine] = 0.0;
        ++mine;
    }
    for (int64_t r0 = 0; r0 < R; r0 += kExactRows) {
        const int rows = static_cast<int>(R - r0 < kExactRows ? R - r0 : kExactRows);
        __syncthreads();
        for (int i = threadIdx.x; i < n * kExactRows; i += kGramThreads) {
            const int c = i / kExactRows;
            const int k = i - c * kExactRows;
            tile[c * kExactStride + k] = k < rows ? column(J, r, run, c, P, stride, R)[r0 + k] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int m = 0; m < kMaxPairsPerThread; ++m) {
            if (m < mine) {
                const double* u = tile + pp[m] * kExactStride;
                const double* v = tile + qq[m] * kExactStride;
                double a = acc[m];
                for (int k = 0; k < rows; ++k) a = fma(u[k], v[k], a);
                acc[m] = a;
            }
        }
    }
    double* g = gram + run * (stride + 1) * (stride + 1);
    for (int m = 0; m < mine; ++m) {
        g[static_cast<int64_t>(qq[m]) * n + pp[m]] = acc[m];
        g[static_cast<int64_t>(pp[m]) * n + qq[m]] = acc[m];
    }
}

// ---- DMMA ------------------------------------------------------------------------------------
constexpr int kDmmaRows = 64;                  // rows per shared tile (16 k-steps of 4)
constexpr int kDmmaMaxTiles = (kMaxCols + 7) / 8;  // 9 column tiles of 8 for P <= 64
constexpr int kDmmaMaxPairs = kDmmaMaxTiles * (kDmmaMaxTiles + 1) / 2;  // 45
constexpr int kDmmaWarps = kGramThreads / 32;
constexpr int kDmmaTilesPerWarp = (kDmmaMaxPairs + kDmmaWarps - 1) / kDmmaWarps;  // 6

// D = A * B + C for one 8x8x4 FP64 tile. Fragments (PTX ISA, mma.m8n8k4 .f64): lane l holds
// A[l/4][l%4], B[l%4][l/4] and D[l/4][2(l%4) + {0, 1}].
__device__ inline void dmma_8x8x4(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(kGramThreads)
gram_dmma_kernel(const double* __restrict__ J, const double* __restrict__ r, int P_all,
                 int64_t R, double* __restrict__ gram, const int* __restrict__ run_mask,
                 const VarParams* __restrict__ vt, int stride) {
    // tile[k][c] row-major with a padded row stride (columns of the 8-wide tiles are read
    // across lanes)
    constexpr int kStride = kDmmaMaxTiles * 8 + 1;
    __shared__ double tile[kDmmaRows * kStride];
    const int64_t run = blockIdx.x;
    if (run_mask != nullptr && run_mask[run] == 0) return;
    const int P = vt != nullptr ? vt[run].P : P_all;
    const int n = P + 1;
    const int T = (n + 7) / 8;
    const int pairs = T * (T + 1) / 2;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int gid = lane >> 2, tig = lane & 3;
    int ti[kDmmaTilesPerWarp], tj[kDmmaTilesPerWarp];
    double c0[kDmmaTilesPerWarp], c1[kDmmaTilesPerWarp];
    int mine = 0;
    for (int e = warp; e < pairs; e += kDmmaWarps) {
        int j = 0, rem = e;
        while (rem >= j + 1) {
            rem -= j + 1;
            ++j;
        }
        ti[mine] = rem;
        tj[mine] = j;
        c0[mine] = c1[mine] = 0.0;
        ++mine;
    }
    for (int64_t r0 = 0; r0 < R; r0 += kDmmaRows) {
        const int rows = static_cast<int>(R - r0 < kDmmaRows ? R - r0 : kDmmaRows);
        __syncthreads();
        for (int i = threadIdx.x; i < T * 8 * kDmmaRows; i += kGramThreads) {
            const int c = i / kDmmaRows;
            const int k = i - c * kDmmaRows;
            double v = 0.0;
            if (c < n && k < rows) v = column(J, r, run, c, P, stride, R)[r0 + k];
            tile[k * kStride + c] = v;
        }
        __syncthreads();
        const int ksteps = (rows + 3) / 4;
#pragma unroll
        for (int m = 0; m < kDmmaTilesPerWarp; ++m) {
            if (m < mine) {
                const int ca = ti[m] * 8 + gid;
                const int cb = tj[m] * 8 + gid;
                double d0 = c0[m], d1 = c1[m];
                for (int ks = 0; ks < ksteps; ++ks) {
                    const int k = ks * 4 + tig;
                    dmma_8x8x4(d0, d1, tile[k * kStride + ca], tile[k * kStride + cb]);
                }
                c0[m] = d0;
                c1[m] = d1;
            }
        }
    }
    double* g = gram + run * (stride + 1) * (stride + 1);
    for (int m = 0; m < mine; ++m) {
        const int row = ti[m] * 8 + gid;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int col = tj[m] * 8 + 2 * tig + h;
            const double v = h == 0 ? c0[m] : c1[m];
            if (row < n && col < n) {
                g[static_cast<int64_t>(col) * n + row] = v;
                g[static_cast<int64_t>(row) * n + col] = v;
            }
        }
    }
}

}  // namespace

int launch_gram(const double* J, const double* r, int runs, int P, int64_t R, double* gram,
                bool exact, cudaStream_t stream, const int* run_mask, RunVars rv) {
    if (runs <= 0) return MKB_OK;
    const int stride = rv.table != nullptr ? rv.stride : P;
    if (exact)
        gram_exact_kernel<<<runs, kGramThreads, 0, stream>>>(J, r, P, R, gram, run_mask, rv.table,
                                                             stride);
    else
        gram_dmma_kernel<<<runs, kGramThreads, 0, stream>>>(J, r, P, R, gram, run_mask, rv.table,
                                                            stride);
    count_launch();
    return cuda_status(cudaGetLastError(), "normal equations launch");
}

MKB_DEFINE_ERROR_READER(gram_device_error)

}  // namespace mkb

extern "C" int mkb_normal_equations_device(const double* J, const double* r, int32_t runs,
                                           int32_t P, int64_t R, double* gram, int32_t exact,
                                           void* stream) {
    using namespace mkb;
    if (runs < 0 || P < 1 || P > MKB_MAX_VARIABLES || R < 0) {
        set_error("normal equations: runs %d, P %d (1..%d) or R %lld out of range", runs, P,
                  MKB_MAX_VARIABLES, static_cast<long long>(R));
        return MKB_ERR_ARGUMENT;
    }
    if (runs > 0 && (J == nullptr || r == nullptr || gram == nullptr)) {
        set_error("normal equations: null pointer");
        return MKB_ERR_ARGUMENT;
    }
    return launch_gram(J, r, runs, P, R, gram, exact != 0, static_cast<cudaStream_t>(stream));
}
