// Scalar PSF and MTF from EVAL OPD maps, for sm_100a.
//
// The pupil function P = exp(2 pi i OPD / lambda) of every tuple lies in the corner of an M x M
// field (M a power of two >= 2N, the rest zero); the PSF is |FFT2(P)|^2 / n_full^2, centred (and
// mirrored for a divergent wave), and the MTF cuts are |OTF| / OTF(0) with OTF = FFT2^-1(I)
// (PsfEngine::compute, src/cuda/psf.cu; CPU reference psf_cpu, src/eval/psf.cpp:330). Here the
// transform is this file's own shared-memory FFT, built around the zero padding:
//   psf_rows_kernel     the N non-zero rows of every pupil field: exp(i phase) of the row's N
//                       points, a length-M FFT in shared memory, the row spectra to HBM
//                       column-major ([T][M][N] complex; the M - N zero rows are never
//                       formed)
//   psf_cols_kernel     C adjacent columns per CTA: the N non-zero entries of each column, a
//                       length-M FFT, then in the same pass the intensity I = |U|^2 s, the
//                       centred PSF written once, and the two projections of I the MTF cuts
//                       need: per column the sum over the rows (in a fixed order), per row the
//                       sum over this CTA's columns (a partial per tile)
//   psf_mtf_kernel      per tuple: OTF(k, 0) and OTF(0, k), k = 0 .. N, as direct DFTs of the
//                       two projections (OTF(kx, 0) = sum_q colsum[q] exp(+2 pi i kx q / M)),
//                       OTF(0) = sum of the column sums; a warp per frequency, fixed-order
//                       shuffle sums -- no inverse 2-D transform
// Everything is FP64; every sum has a fixed order, so results repeat bit for bit. Against the
// reference's radix-2 CPU FFT the PSF and MTF agree to rounding (the reference's own CPU/GPU bar
// is 1e-13 in units of the unaberrated peak, tests/tolerances.hpp:286).
#include "launch.cuh"

#include <cmath>
#include <cstdint>

namespace mkb {

namespace {

constexpr int kPsfThreads = 256;
constexpr int kPsfSmemElems = 4096;  // complex values per CTA below M = 8192 (64 KB)

struct PsfArgs {
    int T, N, M, log_m;
    int rows_per_cta;        // R: rows per CTA in the row pass
    int cols_per_cta;        // C: columns per CTA in the column pass (a power of two)
    int tiles;               // M / C
    const double* maps;      // [T][N][N] OPD [mm], NaN: no transmission
    const mkb_psf_pupil_params* params;  // [T]
    const double2* tw;       // [M / 2] exp(-2 pi i k / M)
    double2* spec;           // [T][M][N] row spectra, column-major per tuple
    double* psf;             // [T][M][M]
    double* colsum;          // [T][M]      sum over the rows of I[.][q]
    double* rowpart;         // [T][tiles][M] sum over a tile's columns of I[q][.]
    double* mtf;             // [T][2][N + 1]
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// exp(-2 pi i m / M) for any m >= 0 from the half table
__device__ __forceinline__ double2 twiddle(const double2* tw, int m, int M) {
    m &= M - 1;
    const int h = M >> 1;
    if (m < h) return tw[m];
    const double2 w = tw[m - h];
    return make_double2(-w.x, -w.y);
}

__device__ __forceinline__ int bit_reverse(int i, int log_m) {
    return log_m == 0 ? 0 : static_cast<int>(__brev(static_cast<unsigned>(i)) >> (32 - log_m));
}

// In-place decimation-in-time FFT (forward, exp(-2 pi i jk/M)) of `count` sequences of length
// M held in bit-reversed order in shared memory, element i of sequence c at a[i * count + c]
// (sequence index fastest, so the lanes of a warp touch adjacent 16-byte words). The log2 M
// radix-2 stages run in passes of up to four: a thread loads the 2^NS elements one butterfly
// group of the pass touches into registers, runs the NS stages there and stores them back, so
// shared memory is read and written once per pass instead of once per stage.
// kFirst: the pass reads its inputs through load(c, i) (the value at bit-reversed position i
// of sequence c) instead of from shared memory.
template <int NS, bool kFirst, class Load>
__device__ __forceinline__ void fft_pass(double2* a, int M, int count, int s, const double2* tw,
                                         const Load& load) {
    constexpr int R = 1 << NS;
    const int total = (M >> NS) * count;
    const int h0 = 1 << s;
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
        const int c = b % count, g = b / count;
        const int pos = g & (h0 - 1);
        const int base = ((g >> s) << (s + NS)) + pos;
        double2 x[R];
#pragma unroll
        for (int k = 0; k < R; ++k)
            x[k] = kFirst ? load(c, base + k * h0) : a[(base + k * h0) * count + c];
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            const int hj = 1 << j;
            const int step = M >> (s + j + 1);
#pragma unroll
            for (int k = 0; k < R; ++k) {
                if (k & hj) continue;
                // stage s + j pairs k and k + 2^j; the element's offset in its 2^(s+j) block
                // is pos + (k mod 2^j) 2^s
                const double2 w = tw[(pos + ((k & (hj - 1)) << s)) * step];
                const double2 t = cmul(x[k + hj], w);
                x[k + hj] = make_double2(x[k].x - t.x, x[k].y - t.y);
                x[k] = make_double2(x[k].x + t.x, x[k].y + t.y);
            }
        }
#pragma unroll
        for (int k = 0; k < R; ++k) a[(base + k * h0) * count + c] = x[k];
    }
    __syncthreads();
}

struct FromShared {
    __device__ double2 operator()(int, int) const { return make_double2(0.0, 0.0); }
};

// The whole transform in passes of at most kPassStages radix-2 stages (2^kPassStages values
// per thread in registers); the first pass takes its inputs from load (kFirst) or shared memory.
constexpr int kPassStages = 3;

template <bool kFirst, class Load>
__device__ __forceinline__ void fft_pass_n(int n, double2* a, int M, int count, int s,
                                           const double2* tw, const Load& load) {
    switch (n) {
    case 1: fft_pass<1, kFirst>(a, M, count, s, tw, load); break;
    case 2: fft_pass<2, kFirst>(a, M, count, s, tw, load); break;
    default:
        if constexpr (kPassStages >= 4) {
            if (n == 4) {
                fft_pass<(kPassStages >= 4 ? 4 : 3), kFirst>(a, M, count, s, tw, load);
                break;
            }
        }
        fft_pass<3, kFirst>(a, M, count, s, tw, load);
        break;
    }
}

template <bool kFirst, class Load>
__device__ void fft_shared(double2* a, int M, int log_m, int count, const double2* tw,
                           const Load& load) {
    const int n0 = log_m < kPassStages ? log_m : kPassStages;
    if (n0 > 0) fft_pass_n<kFirst>(n0, a, M, count, 0, tw, load);
    const FromShared none;
    for (int s = n0; s < log_m; s += kPassStages)
        fft_pass_n<false>(log_m - s < kPassStages ? log_m - s : kPassStages, a, M, count, s, tw,
                          none);
}

// the twiddle table into shared memory (read by every butterfly)
__device__ __forceinline__ void stage_twiddles(double2* tws, const double2* tw, int M) {
    for (int k = threadIdx.x; k < (M >> 1); k += blockDim.x) tws[k] = tw[k];
}

__global__ void psf_twiddle_kernel(double2* tw, int M) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M / 2) return;
    double s, c;
    sincospi(2.0 * static_cast<double>(k) / static_cast<double>(M), &s, &c);
    tw[k] = make_double2(c, -s);
}

// The pupil function of rows [r0, r0 + R) of tuple t, transformed along x (R = kRows, rows past
// N are zero and not written). Row r's element i sits at sm[i * R + r]; the spectra go out
// column-major per tuple, spec[t][q][j], so that the column pass reads each column's N values
// contiguously.
template <int kRows>
__global__ void __launch_bounds__(kPsfThreads, 3) psf_rows_kernel(const PsfArgs a) {
    extern __shared__ double2 sm[];
    const int per_t = (a.N + kRows - 1) / kRows;
    const int t = blockIdx.x / per_t;
    const int r0 = (blockIdx.x - t * per_t) * kRows;
    const int M = a.M, N = a.N, lm = a.log_m;
    const double lambda = a.params[t].lambda_mm;
    const double* map = a.maps + (static_cast<int64_t>(t) * N + r0) * N;
    double2* tws = sm + kRows * M;
    stage_twiddles(tws, a.tw, M);
    for (int e = threadIdx.x; e < kRows * M; e += blockDim.x) {
        const int r = e >> lm, i = e & (M - 1);
        double2 v = make_double2(0.0, 0.0);
        if (i < N && r0 + r < N) {
            const double opd = map[static_cast<int64_t>(r) * N + i];
            if (opd == opd) {  // NaN: outside the pupil or a failed ray
                const double phase = 6.283185307179586 * (opd / lambda);
                double s, c;
                sincos(phase, &s, &c);
                v = make_double2(c, s);
            }
        }
        sm[bit_reverse(i, lm) * kRows + r] = v;
    }
    __syncthreads();
    fft_shared<false>(sm, M, lm, kRows, tws, FromShared{});
    const int R = min(kRows, N - r0);
    double2* out = a.spec + static_cast<int64_t>(t) * M * N + r0;
    for (int e = threadIdx.x; e < kRows * M; e += blockDim.x) {
        const int q = e / kRows, r = e - q * kRows;
        if (r < R) out[static_cast<int64_t>(q) * N + r] = sm[e];
    }
}

// Columns [q0, q0 + C) of tuple t (C = kCols): transform along y, then one pass over the
// result for the intensity, the centred PSF and the two projections.
template <int kCols>
__global__ void __launch_bounds__(kPsfThreads, 3) psf_cols_kernel(const PsfArgs a) {
    constexpr int C = kCols;
    extern __shared__ double2 sm[];
    __shared__ double wsum[kPsfThreads / 32][C];
    const int M = a.M, N = a.N, lm = a.log_m;
    const int t = blockIdx.x / a.tiles;
    const int tile = blockIdx.x - t * a.tiles;
    const int q0 = tile * C;
    const double2* in = a.spec + (static_cast<int64_t>(t) * M + q0) * N;
    double2* tws = sm + C * M;
    stage_twiddles(tws, a.tw, M);
    __syncthreads();
    // the first pass reads the column's entries straight from the spectra (contiguous per
    // column, cached in L1 across the pass): position i holds row brev(i), zero past N
    auto load = [&](int c, int i) {
        const int j = bit_reverse(i, lm);
        return j < N ? in[c * N + j] : make_double2(0.0, 0.0);
    };
    fft_shared<true>(sm, M, lm, C, tws, load);
    const mkb_psf_pupil_params p = a.params[t];
    double* psf = a.psf + static_cast<int64_t>(t) * M * M;
    double* part = a.rowpart + (static_cast<int64_t>(t) * a.tiles + tile) * M;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // e = (qj, c), c fastest: a thread keeps one column (256 is a multiple of C) and adds its
    // rows in ascending order; the C lanes of a row add the row in a fixed xor tree. The PSF
    // element goes to its centred, possibly mirrored position: output index
    // o = (M / 2 + sign q) mod M of FFT index q (psf_output_index, psf_ops.hpp).
    const int total = M * C;
    double col_acc = 0.0;
    for (int e0 = threadIdx.x - lane; e0 < total; e0 += blockDim.x) {  // warp-uniform bound
        const int e = e0 + lane;
        double I = 0.0;
        if (e < total) {
            const int qj = e / C, qi = q0 + (e - qj * C);
            const double2 u = sm[e];
            I = (u.x * u.x + u.y * u.y) * p.scale;
            col_acc += I;
            const int oi = ((M >> 1) + p.sign_x * qi) & (M - 1);
            const int oj = ((M >> 1) + p.sign_y * qj) & (M - 1);
            psf[static_cast<int64_t>(oj) * M + oi] = I;
        }
        double r = I;
#pragma unroll
        for (int o = C >> 1; o >= 1; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
        if (e < total && e % C == 0) part[e / C] = r;
    }
    // column sums: the lanes of a warp with the same column, then the warps in ascending order
#pragma unroll
    for (int o = 16; o >= C; o >>= 1) col_acc += __shfl_xor_sync(0xffffffffu, col_acc, o);
    if (lane < C) wsum[warp][lane] = col_acc;
    __syncthreads();
    if (threadIdx.x < C) {
        double tot = 0.0;
        for (int w = 0; w < kPsfThreads / 32; ++w) tot += wsum[w][threadIdx.x];
        a.colsum[static_cast<int64_t>(t) * M + q0 + threadIdx.x] = tot;
    }
}

// MTF cuts of tuple t (one CTA): sagittal |OTF(k, 0)| and tangential |OTF(0, k)| over OTF(0).
__global__ void __launch_bounds__(kPsfThreads) psf_mtf_kernel(const PsfArgs a) {
    extern __shared__ double proj[];  // [2][M]: column sums, row sums
    const int t = blockIdx.x, M = a.M, N = a.N;
    double* cs = proj;
    double* rs = proj + M;
    for (int q = threadIdx.x; q < M; q += blockDim.x) {
        cs[q] = a.colsum[static_cast<int64_t>(t) * M + q];
        const double* part = a.rowpart + static_cast<int64_t>(t) * a.tiles * M + q;
        double s = 0.0;
        for (int k = 0; k < a.tiles; ++k) s += part[static_cast<int64_t>(k) * M];
        rs[q] = s;
    }
    __syncthreads();
    __shared__ double otf0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        double s = 0.0;
        for (int q = lane; q < M; q += 32) s += cs[q];
        for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) otf0 = s;
    }
    __syncthreads();
    const double z = otf0;
    const int per = N + 1;
    double* out = a.mtf + static_cast<int64_t>(t) * 2 * per;
    for (int job = warp; job < 2 * per; job += kPsfThreads / 32) {
        const int cut = job / per, k = job - cut * per;
        const double* v = cut == 0 ? cs : rs;
        double re = 0.0, im = 0.0;
        for (int q = lane; q < M; q += 32) {
            const double2 w = twiddle(a.tw, k * q, M);  // exp(-i ...); the OTF uses exp(+i ...)
            re += v[q] * w.x;
            im -= v[q] * w.y;
        }
        for (int o = 16; o >= 1; o >>= 1) {
            re += __shfl_xor_sync(0xffffffffu, re, o);
            im += __shfl_xor_sync(0xffffffffu, im, o);
        }
        if (lane == 0) out[cut * per + k] = z > 0.0 ? sqrt(re * re + im * im) / z : nan("");
    }
}

// EVAL output -> OPD maps (eval_opd_map with piston removal, src/eval/eval.cpp:512): NaN, then
// the OPD of every ray with status Ok at (row, column) of its grid point, mirrored to column
// N - 1 - i for a half pupil.
__global__ void psf_maps_fill_kernel(double* maps, int64_t count) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count) maps[i] = nan("");
}

__global__ void psf_maps_scatter_kernel(int T, int N, int64_t n, int half, const double* opd,
                                        const uint8_t* status, const int32_t* column,
                                        const int32_t* row, double* maps) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= static_cast<int64_t>(T) * n) return;
    if (status[e] != MKB_STATUS_OK) return;
    const int64_t t = e / n, k = e - t * n;
    double* m = maps + t * N * N + static_cast<int64_t>(row[k]) * N;
    m[column[k]] = opd[e];
    if (half) m[N - 1 - column[k]] = opd[e];
}

int psf_shape(int32_t grid, int32_t fft_size, int& log_m, int& R, int& C) {
    if (grid < 1 || grid > MKB_MAX_EVAL_GRID) {
        set_error("psf: grid edge %d outside [1, %d]", grid, MKB_MAX_EVAL_GRID);
        return MKB_ERR_ARGUMENT;
    }
    if (fft_size < 2 * grid || fft_size > MKB_MAX_PSF_FFT || (fft_size & (fft_size - 1)) != 0) {
        set_error("psf: FFT size %d must be a power of two in [2N, %d] (N = %d)", fft_size,
                  MKB_MAX_PSF_FFT, grid);
        return MKB_ERR_ARGUMENT;
    }
    log_m = 0;
    while ((1 << log_m) < fft_size) ++log_m;
    const int fit = kPsfSmemElems / fft_size;
    C = fit >= 16 ? 16 : fit >= 1 ? fit : 1;
    if (C > fft_size) C = fft_size;
    R = C < grid ? C : grid;
    return MKB_OK;
}

size_t psf_regions(int T, int N, int M, int C, size_t* off) {
    // tw | spec | colsum | rowpart, each 256-byte aligned
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t tiles = static_cast<size_t>(M / C);
    size_t o = 0;
    off[0] = o;
    o += al(sizeof(double2) * static_cast<size_t>(M / 2 > 0 ? M / 2 : 1));
    off[1] = o;
    o += al(sizeof(double2) * static_cast<size_t>(T) * N * M);
    off[2] = o;
    o += al(sizeof(double) * static_cast<size_t>(T) * M);
    off[3] = o;
    o += al(sizeof(double) * static_cast<size_t>(T) * tiles * M);
    return o;
}

}  // namespace

// ---- host side: aperture of a tuple and the PSF's figures (the reference's make_psf_pupil
// and finish_psf, src/eval/psf.cpp:196,290), compiled without FP contraction so that the sums
// and the tilt fit repeat the reference's bits on the same PSF
namespace psf_host {

double cell_center(int i, int n) {
    return static_cast<double>(2 * i + 1 - n) / static_cast<double>(n);
}

// |sum exp(2 pi i (OPD - t_x x - t_y y) / lambda)|^2 / n_full^2 over the transmitting points,
// rows ascending (direct_strehl, src/eval/psf.cpp:33)
double direct_strehl(const double* opd, int n, double lambda, int full, double tx, double ty) {
    double sr = 0.0, si = 0.0;
    for (int j = 0; j < n; ++j) {
        const double y = cell_center(j, n);
        for (int i = 0; i < n; ++i) {
            const double o = opd[static_cast<size_t>(j) * n + i];
            if (!std::isfinite(o)) continue;
            const double x = cell_center(i, n);
            const double v = o - tx * x - ty * y;
            double re = 0.0, im = 0.0;
            if (v == v) {
                const double phase = 6.283185307179586 * (v / lambda);
                re = std::cos(phase);
                im = std::sin(phase);
            }
            sr += re;
            si += im;
        }
    }
    const double f = static_cast<double>(full);
    return (sr * sr + si * si) / (f * f);
}

// least-squares OPD ~ c0 + t_x x + t_y y over the transmitting points, Gaussian elimination
// with column pivoting (fit_tilt, src/eval/psf.cpp:60)
bool fit_tilt(const double* opd, int n, double& tx, double& ty) {
    double g[3][3] = {};
    double h[3] = {};
    for (int j = 0; j < n; ++j) {
        const double y = cell_center(j, n);
        for (int i = 0; i < n; ++i) {
            const double o = opd[static_cast<size_t>(j) * n + i];
            if (!std::isfinite(o)) continue;
            const double phi[3] = {1.0, cell_center(i, n), y};
            for (int a = 0; a < 3; ++a) {
                for (int b = 0; b < 3; ++b) g[a][b] += phi[a] * phi[b];
                h[a] += phi[a] * o;
            }
        }
    }
    for (int c = 0; c < 3; ++c) {
        int piv = c;
        for (int a = c + 1; a < 3; ++a)
            if (std::abs(g[a][c]) > std::abs(g[piv][c])) piv = a;
        if (!(std::abs(g[piv][c]) > 0.0)) return false;
        for (int b = 0; b < 3; ++b) {
            const double t = g[c][b];
            g[c][b] = g[piv][b];
            g[piv][b] = t;
        }
        const double t = h[c];
        h[c] = h[piv];
        h[piv] = t;
        for (int a = c + 1; a < 3; ++a) {
            const double q = g[a][c] / g[c][c];
            for (int b = c; b < 3; ++b) g[a][b] -= q * g[c][b];
            h[a] -= q * h[c];
        }
    }
    double x[3] = {};
    for (int a = 2; a >= 0; --a) {
        double s = h[a];
        for (int b = a + 1; b < 3; ++b) s -= g[a][b] * x[b];
        x[a] = s / g[a][a];
    }
    tx = x[1];
    ty = x[2];
    return std::isfinite(tx) && std::isfinite(ty);
}

}  // namespace psf_host

extern "C" {

int mkb_psf_fft_size_host(int32_t grid, double padding, int32_t* fft_size) {
    if (fft_size == nullptr) {
        set_error("psf: null output");
        return MKB_ERR_ARGUMENT;
    }
    if (grid < 1 || grid > MKB_MAX_EVAL_GRID) {
        set_error("psf: grid edge %d outside [1, %d]", grid, MKB_MAX_EVAL_GRID);
        return MKB_ERR_ARGUMENT;
    }
    if (!(padding >= 2.0) || !std::isfinite(padding)) {
        set_error("psf: zero-padding factor must be >= 2");
        return MKB_ERR_ARGUMENT;
    }
    const double target = std::ceil(padding * static_cast<double>(grid));
    const double minimum = target > 2.0 * grid ? target : 2.0 * grid;
    if (minimum > static_cast<double>(MKB_MAX_PSF_FFT)) {
        set_error("psf: FFT size %.0f exceeds %d; reduce the grid or the zero padding", minimum,
                  MKB_MAX_PSF_FFT);
        return MKB_ERR_ARGUMENT;
    }
    int m = 1;
    while (static_cast<double>(m) < minimum) m *= 2;
    *fft_size = m;
    return MKB_OK;
}

size_t mkb_psf_workspace_bytes(int32_t tuples, int32_t grid, int32_t fft_size) {
    int log_m = 0, R = 0, C = 0;
    if (tuples < 0 || psf_shape(grid, fft_size, log_m, R, C) != MKB_OK) return 0;
    size_t off[4];
    return psf_regions(tuples, grid, fft_size, C, off);
}

int mkb_psf_device(int32_t tuples, int32_t grid, int32_t fft_size, const double* maps,
                   const mkb_psf_pupil_params* params, double* psf, double* mtf, void* workspace,
                   size_t workspace_bytes, void* stream_ptr) {
    const cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    int log_m = 0, R = 0, C = 0;
    int rc = psf_shape(grid, fft_size, log_m, R, C);
    if (rc != MKB_OK) return rc;
    if (tuples < 0) {
        set_error("psf: tuples must be >= 0");
        return MKB_ERR_ARGUMENT;
    }
    if (tuples == 0) return MKB_OK;
    if (maps == nullptr || params == nullptr || psf == nullptr || mtf == nullptr) {
        set_error("psf: null maps, params or outputs");
        return MKB_ERR_ARGUMENT;
    }
    size_t off[4];
    const size_t need = psf_regions(tuples, grid, fft_size, C, off);
    if (workspace == nullptr || workspace_bytes < need) {
        set_error("psf: workspace of %zu bytes needed", need);
        return MKB_ERR_WORKSPACE;
    }
    char* ws = static_cast<char*>(workspace);
    PsfArgs a;
    a.T = tuples;
    a.N = grid;
    a.M = fft_size;
    a.log_m = log_m;
    a.rows_per_cta = C;
    a.cols_per_cta = C;
    a.tiles = fft_size / C;
    a.maps = maps;
    a.params = params;
    a.tw = reinterpret_cast<const double2*>(ws + off[0]);
    a.spec = reinterpret_cast<double2*>(ws + off[1]);
    a.colsum = reinterpret_cast<double*>(ws + off[2]);
    a.rowpart = reinterpret_cast<double*>(ws + off[3]);
    a.psf = psf;
    a.mtf = mtf;
    const int half = fft_size / 2;
    psf_twiddle_kernel<<<(half + 255) / 256, 256, 0, stream>>>(
        reinterpret_cast<double2*>(ws + off[0]), fft_size);
    count_launch();
    // data [C][M] and the twiddles [M / 2]
    const size_t smem_rows = sizeof(double2) * (static_cast<size_t>(C) * fft_size + fft_size / 2);
    const size_t smem_cols = smem_rows;
    const size_t smem_mtf = sizeof(double) * 2 * static_cast<size_t>(fft_size);
    using Fn = void (*)(PsfArgs);
    Fn rows = C == 16 ? psf_rows_kernel<16> : C == 8 ? psf_rows_kernel<8>
            : C == 4 ? psf_rows_kernel<4> : C == 2 ? psf_rows_kernel<2> : psf_rows_kernel<1>;
    Fn cols = C == 16 ? psf_cols_kernel<16> : C == 8 ? psf_cols_kernel<8>
            : C == 4 ? psf_cols_kernel<4> : C == 2 ? psf_cols_kernel<2> : psf_cols_kernel<1>;
    cudaError_t err = cudaFuncSetAttribute(rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(smem_rows));
    if (err == cudaSuccess)
        err = cudaFuncSetAttribute(cols, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem_cols));
    if (err == cudaSuccess)
        err = cudaFuncSetAttribute(psf_mtf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem_mtf));
    if (err != cudaSuccess) return cuda_status(err, "psf: shared memory attribute");
    const int per_t = (grid + C - 1) / C;
    rows<<<static_cast<unsigned>(tuples) * per_t, kPsfThreads, smem_rows, stream>>>(a);
    count_launch();
    cols<<<static_cast<unsigned>(tuples) * a.tiles, kPsfThreads, smem_cols, stream>>>(a);
    count_launch();
    psf_mtf_kernel<<<static_cast<unsigned>(tuples), kPsfThreads, smem_mtf, stream>>>(a);
    count_launch();
    return cuda_status(cudaGetLastError(), "psf launch");
}

int mkb_psf_aperture_host(const double* field_rays, const uint8_t* field_status, double n_image,
                          double field_ray_offset, double numerical_aperture, double* na_x,
                          double* na_y, int32_t* flip_x, int32_t* flip_y) {
    if (field_rays == nullptr || field_status == nullptr || na_x == nullptr || na_y == nullptr ||
        flip_x == nullptr || flip_y == nullptr) {
        set_error("psf aperture: null argument");
        return MKB_ERR_ARGUMENT;
    }
    if (!(numerical_aperture >= 0.0) || !std::isfinite(numerical_aperture)) {
        set_error("psf aperture: the given NA must be >= 0 (0: from the field rays)");
        return MKB_ERR_ARGUMENT;
    }
    // field rays: chief (0, 0), tangential (0, +d), (0, -d), sagittal (+d, 0); values x, y,
    // d_x, d_y, d_z
    const double nan_v = std::nan("");
    auto ok = [&](int j) { return field_status[j] == MKB_STATUS_OK; };
    double ax = nan_v, ay = nan_v;
    if (ok(0) && ok(3)) ax = n_image * (field_rays[3 * 5 + 2] - field_rays[0 * 5 + 2]) /
                             field_ray_offset;
    if (ok(1) && ok(2)) ay = n_image * (field_rays[1 * 5 + 3] - field_rays[2 * 5 + 3]) /
                             (2.0 * field_ray_offset);
    *flip_x = std::isfinite(ax) && ax > 0.0 ? 1 : 0;
    *flip_y = std::isfinite(ay) && ay > 0.0 ? 1 : 0;
    if (numerical_aperture > 0.0) {
        *na_x = numerical_aperture;
        *na_y = numerical_aperture;
        return MKB_OK;
    }
    if (!std::isfinite(ax) || !std::isfinite(ay) || ax == 0.0 || ay == 0.0) {
        set_error("psf aperture: the NA of the pupil imaging is undetermined (a field ray "
                  "failed, or the system is afocal); give the NA");
        return MKB_ERR_ARGUMENT;
    }
    *na_x = std::abs(ax);
    *na_y = std::abs(ay);
    return MKB_OK;
}

int mkb_psf_finish_host(int32_t grid, int32_t fft_size, const double* opd_map, int32_t full_count,
                        double wavelength_nm, double na_x, double na_y, int32_t flip_x,
                        int32_t flip_y, const double* psf, mkb_psf_metrics* out) {
    int log_m = 0, R = 0, C = 0;
    const int rc = psf_shape(grid, fft_size, log_m, R, C);
    if (rc != MKB_OK) return rc;
    if (opd_map == nullptr || psf == nullptr || out == nullptr) {
        set_error("psf finish: null argument");
        return MKB_ERR_ARGUMENT;
    }
    if (full_count < 1 || !(wavelength_nm > 0.0) || !std::isfinite(wavelength_nm) ||
        !(na_x > 0.0) || !(na_y > 0.0) || !std::isfinite(na_x) || !std::isfinite(na_y)) {
        set_error("psf finish: full count, wavelength and NA must be positive");
        return MKB_ERR_ARGUMENT;
    }
    const double nan_v = std::nan("");
    const int n = grid;
    const size_t m = static_cast<size_t>(fft_size);
    const double lambda = wavelength_nm * 1e-6;
    // geometry (prepare_psf_result, src/eval/psf.cpp:262)
    const double scale = lambda * static_cast<double>(n) / (2.0 * fft_size);
    out->dx = scale / na_x;
    out->dy = scale / na_y;
    out->airy_radius = 3.8317059702075123 / (2.0 * 3.141592653589793) * lambda /
                       std::sqrt(na_x * na_y);
    int64_t transmitted = 0;
    for (size_t k = 0; k < static_cast<size_t>(n) * n; ++k)
        transmitted += std::isfinite(opd_map[k]) ? 1 : 0;
    out->transmitted = transmitted;
    double sum = 0.0;
    size_t peak_index = 0;
    for (size_t k = 0; k < m * m; ++k) {
        sum += psf[k];
        if (psf[k] > psf[peak_index]) peak_index = k;
    }
    const double md = static_cast<double>(m);
    out->energy = sum * static_cast<double>(full_count) / (md * md);
    out->strehl_fft = psf[(m / 2) * m + m / 2];
    out->strehl_origin = psf_host::direct_strehl(opd_map, n, lambda, full_count, 0.0, 0.0);
    double tx = 0.0, ty = 0.0;
    if (psf_host::fit_tilt(opd_map, n, tx, ty)) {
        out->strehl = psf_host::direct_strehl(opd_map, n, lambda, full_count, tx, ty);
        out->reference_x = (flip_x ? -tx : tx) / na_x;
        out->reference_y = (flip_y ? -ty : ty) / na_y;
    } else {
        out->strehl = nan_v;
        out->reference_x = nan_v;
        out->reference_y = nan_v;
    }
    out->peak = psf[peak_index];
    out->peak_x = (static_cast<double>(peak_index % m) - md / 2.0) * out->dx;
    out->peak_y = (static_cast<double>(peak_index / m) - md / 2.0) * out->dy;
    return MKB_OK;
}

int mkb_psf_maps_device(int32_t tuples, int32_t grid, int64_t samples, int32_t half_pupil,
                        const double* opd, const uint8_t* status, const int32_t* column,
                        const int32_t* row, double* maps, void* stream_ptr) {
    const cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    if (grid < 1 || grid > MKB_MAX_EVAL_GRID || tuples < 0 || samples < 0) {
        set_error("psf maps: grid, tuples or samples out of range");
        return MKB_ERR_ARGUMENT;
    }
    if (tuples == 0) return MKB_OK;
    if (maps == nullptr || (samples > 0 && (opd == nullptr || status == nullptr ||
                                            column == nullptr || row == nullptr))) {
        set_error("psf maps: null input or output");
        return MKB_ERR_ARGUMENT;
    }
    const int64_t count = static_cast<int64_t>(tuples) * grid * grid;
    psf_maps_fill_kernel<<<static_cast<unsigned>((count + 255) / 256), 256, 0, stream>>>(maps,
                                                                                          count);
    count_launch();
    const int64_t rays = static_cast<int64_t>(tuples) * samples;
    if (rays > 0) {
        psf_maps_scatter_kernel<<<static_cast<unsigned>((rays + 255) / 256), 256, 0, stream>>>(
            tuples, grid, samples, half_pupil != 0, opd, status, column, row, maps);
        count_launch();
    }
    return cuda_status(cudaGetLastError(), "psf maps launch");
}

}  // extern "C"

}  // namespace mkb
