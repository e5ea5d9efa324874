// Shared device code of the B200 trace kernels: kernel parameter block, record layout, the
// per-surface ray step in FP64, bulk-copy staging with bounded mbarrier waits, and the
// host-side helpers shared by the entry points.
#pragma once

#include "mikroptim_b200.h"

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace mkb {

// ---- limits ------------------------------------------------------------------------------
constexpr int kMaxSurfaces = MKB_MAX_SURFACES;
constexpr int kMaxRings = MKB_MAX_RINGS;
constexpr int kMaxSpokes = MKB_MAX_SPOKES;
constexpr int kMaxFields = MKB_MAX_FIELDS;
constexpr int kMaxTuples = MKB_MAX_TUPLES;
constexpr int kMaxPacks = 256;
constexpr int kMaxPackTuples = 16;
constexpr int kMaxGhostTerms = MKB_MAX_GHOST_TERMS;  // the reference's kMaxGhostTerms
constexpr int kMaxGhostPlates = MKB_MAX_GHOST_PLATES;

// Trace status and soft-failure branch codes (reference: trace/surface_ops.hpp:24,113).
enum : int { kOk = 0, kMissed = 1, kTir = 2, kBackward = 3, kUnsupported = 4,
             kSoftMissed = 5, kSoftTir = 6 };
enum : int { kBranchRegular = 0, kBranchSoftMissed = 1, kBranchSoftTir = 2 };

__host__ __device__ inline bool is_soft(int s) { return s == kSoftMissed || s == kSoftTir; }
__host__ __device__ inline bool in_piston(int s) { return s == kOk || is_soft(s); }

// ---- record layout (doubles): curvature[S] | thickness[S] | index[S*L] | pupil_radius |
//      sin theta[F] | cos theta[F] | field_target[F] | [non-coaxial batches: per surface
//      kXfValues transform values] | [ghost plates: coefficients [G][K] | normalisation
//      radius [G] | plate index [G][L]] | pad to even --------------------------------------
// Transform values of surface s (SurfaceTransform, trace/surface_transform.hpp:27, with the
// sines and cosines taken on the host): dx, dy, cos a, sin a, cos b, sin b, moved (1 when
// any of dx, dy, a, b is nonzero, else 0 and the surface is traced coaxially), 0.
constexpr int kXfValues = 8;

struct RecordLayout {
    int curvature, thickness, index, pupil, sin_theta, cos_theta, target, stride, surfaces;
    int xf;                                      // transforms, or -1 (coaxial)
    int ghost_coeff, ghost_radius, ghost_index;  // ghost plate data, or -1 (no plates)
    int ghost_terms;                             // K
    int glass;                                   // Buchdahl coefficients [S][4], or -1
    int stop;                                    // interior aperture stop s_a, or 0 (none)
    int L;                                       // wavelengths (index columns)
    uint64_t spheres;                            // bit s: surface s is a sphere (s < 64)
};

__host__ __device__ inline RecordLayout record_layout(int S, int L, int F, int non_coaxial = 0,
                                                      int G = 0, int K = 0, int glass = 0) {
    RecordLayout r;
    r.surfaces = S;
    r.curvature = 0;
    r.thickness = S;
    r.index = 2 * S;
    r.pupil = 2 * S + S * L;
    r.sin_theta = r.pupil + 1;
    r.cos_theta = r.sin_theta + F;
    r.target = r.cos_theta + F;
    int n = r.target + F;
    r.xf = non_coaxial ? n : -1;
    if (non_coaxial) n += S * kXfValues;
    r.ghost_coeff = r.ghost_radius = r.ghost_index = -1;
    r.ghost_terms = K;
    if (G > 0) {
        r.ghost_coeff = n;
        n += G * K;
        r.ghost_radius = n;
        n += G;
        r.ghost_index = n;
        n += G * L;
    }
    r.glass = glass ? n : -1;
    if (glass) n += S * 4;
    r.stride = (n + 1) & ~1;
    r.stop = 0;
    r.L = L;
    r.spheres = 0;
    return r;
}

// ---- kernel parameter block (passed by value; < 16 KB) -----------------------------------
struct Pack {
    int16_t first_tuple;  // first tuple (f * L + l) of the pack
    int16_t tuples;       // tuples in the pack (<= kMaxPackTuples)
    int32_t first_ray;    // offset of the pack's first ray in the variant's ray rows
    int32_t rays;         // rays of the pack (<= rays per CTA)
};

struct TraceParams {
    int V, S, L, F;
    int non_coaxial;        // records carry per-surface transforms
    int G, K;               // ghost plates and their profile terms
    int glass;              // records carry Buchdahl coefficients
    int stride;             // doubles per variant record
    int failure;            // MKB_FAILURE_*
    int rays;               // rays per variant
    int rings, spokes;
    int n_tuples, n_packs;
    int pack_max;           // rays of the largest pack
    int vpc;                // variants one CTA traces (its packs side by side), >= 1
    int sample_count[kMaxFields];   // n_f
    int field_offset[kMaxFields];   // ray offset of tuple (f, 0)
    uint8_t pupil_mode[kMaxFields];
    uint8_t type[kMaxSurfaces];
    // pupil tables: radial rho_i, weights W_i/M and sqrt, azimuth sin/cos per mode
    double rho[kMaxRings];
    double w_axis[kMaxRings], rw_axis[kMaxRings];
    double w_spoke[kMaxRings], rw_spoke[kMaxRings];
    double sin_half[kMaxSpokes], cos_half[kMaxSpokes];
    double sin_full[kMaxSpokes], cos_full[kMaxSpokes];
    double scale[kMaxTuples];       // residual_scale per tuple
    double pscale[kMaxTuples];      // penalty_scale per tuple
    double tscale[kMaxTuples];      // sqrt(transverse_weight * tuple weight) per tuple
    int transverse;                 // transverse ray-error rows (plan transverse_weight > 0)
    Pack packs[kMaxPacks];
    int8_t ghost_of[kMaxSurfaces];  // plate number of a ghost-plate surface (table order), or -1
    const uint8_t* vsurf;           // device [V] table surfaces of each variant, or null (S)
    const int* order;               // device [V] processing order of the variants, or null
    int stop;                       // interior aperture stop s_a (MKB_SURFACE_APERTURE_STOP), or 0
    uint64_t spheres;               // bit s: surface s is a sphere
};

__host__ __device__ inline RecordLayout layout_of(const TraceParams& p) {
    RecordLayout r = record_layout(p.S, p.L, p.F, p.non_coaxial, p.G, p.K, p.glass);
    r.stop = p.stop;
    r.spheres = p.spheres;
    return r;
}

// ---- paraxial ray aiming for an interior aperture stop ----------------------------------------
// Separately rounded operations on host and device (the host side is compiled without
// contraction), so the packed and the device-applied records agree bit for bit.
__host__ __device__ __forceinline__ double aim_mul(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
__host__ __device__ __forceinline__ double aim_add(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
__host__ __device__ __forceinline__ double aim_sub(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
__host__ __device__ __forceinline__ double aim_div(double a, double b) {
#ifdef __CUDA_ARCH__
    return __ddiv_rn(a, b);
#else
    return a / b;
#endif
}

// The stop heights y_A (ray y = 1, u = 0 at surface 1) and y_B (ray y = 0, u = 1) of the y-u
// trace from surface 1 to the stop s_a at the index of wavelength column 0: at surface s,
// u' = (n u - y c (n' - n)) / n' (c = 0 off spheres), then y += thickness[s] u'.
__host__ __device__ inline void aim_heights(const double* rec, const RecordLayout& lay,
                                            double& ya, double& yb) {
    double y1 = 1.0, u1 = 0.0, y2 = 0.0, u2 = 1.0;
    double n = rec[lay.index];
    for (int s = 1; s < lay.stop; ++s) {
        const double n2 = rec[lay.index + s * lay.L];
        const double c = (lay.spheres >> s) & 1u ? rec[lay.curvature + s] : 0.0;
        const double phi = aim_mul(c, aim_sub(n2, n));
        u1 = aim_div(aim_sub(aim_mul(n, u1), aim_mul(y1, phi)), n2);
        u2 = aim_div(aim_sub(aim_mul(n, u2), aim_mul(y2, phi)), n2);
        const double t = rec[lay.thickness + s];
        y1 = aim_add(y1, aim_mul(t, u1));
        y2 = aim_add(y2, aim_mul(t, u2));
        n = n2;
    }
    ya = y1;
    yb = y2;
}

// The layout with the table's interior stop and sphere mask filled in from its surface kinds.
inline RecordLayout with_stop(RecordLayout lay, const uint8_t* type, int S) {
    lay.stop = 0;
    lay.spheres = 0;
    for (int s = 0; s < S && s < 64; ++s) {
        if (type[s] == MKB_SURFACE_SPHERE) lay.spheres |= uint64_t(1) << s;
        if (s > 0 && type[s] == MKB_SURFACE_APERTURE_STOP) lay.stop = s;
    }
    return lay;
}

// Writes the entrance pupil (radius R / |y_A|, thickness[0] = -y_B / y_A) into a record whose
// table has an interior stop; R is the stop surface's curvature slot. Returns false when the
// stop's image is at infinity (y_A = 0) or a value is not finite (the record is then left with
// those non-finite values, which fail every ray).
__host__ __device__ inline bool aim_record(const RecordLayout& lay, double* rec) {
    double ya, yb;
    aim_heights(rec, lay, ya, yb);
    const double R = rec[lay.curvature + lay.stop];
    const double a = aim_div(R, ya < 0.0 ? -ya : ya);
    const double t0 = -aim_div(yb, ya);
    rec[lay.pupil] = a;
    rec[lay.thickness] = t0;
    return ya != 0.0 && a == a && t0 == t0 && a - a == 0.0 && t0 - t0 == 0.0;
}

// Table surfaces variant v traces (uneven batches share the table of the largest; the value
// is clamped to [2, S] so that no index leaves the record).
__device__ __forceinline__ int surfaces_of(const TraceParams& p, int v) {
    if (p.vsurf == nullptr) return p.S;
    const int n = p.vsurf[v];
    return n < 2 ? 2 : (n > p.S ? p.S : n);
}

// ---- error word written by bounded waits that gave up -------------------------------------
// One word per translation unit (no relocatable device code); each .cu file that launches
// kernels defines a reader with MKB_DEFINE_ERROR_READER and lists it in capi.cu, and
// mkb_device_status() polls them all.
static __device__ int g_device_error = 0;
// Polls the first wait of a bulk copy makes before it gives up (per translation unit, like the
// error word). mkb_set_wait_limit changes it so that a test can make the wait run out; the wait
// that drains the copy after a give-up always keeps the full limit.
static __device__ uint32_t g_wait_polls = MKB_WAIT_POLLS_DEFAULT;

#define MKB_DEFINE_ERROR_READER(name)                                                     \
    int name() {                                                                           \
        int value = 0;                                                                     \
        if (cudaMemcpyFromSymbol(&value, g_device_error, sizeof(int)) != cudaSuccess)      \
            return MKB_ERR_CUDA;                                                           \
        if (value != 0) {                                                                  \
            const int zero = 0;                                                            \
            cudaMemcpyToSymbol(g_device_error, &zero, sizeof(int));                        \
        }                                                                                  \
        return value;                                                                      \
    }                                                                                      \
    int name##_wait_limit(uint32_t polls) {                                                \
        return cudaMemcpyToSymbol(g_wait_polls, &polls, sizeof(polls)) == cudaSuccess      \
                   ? MKB_OK                                                                \
                   : MKB_ERR_CUDA;                                                         \
    }

// ---- bulk copy into shared memory with an mbarrier (each CTA its own copy) --------------
__device__ inline uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ inline void mbar_init(uint64_t* bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

__device__ inline void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ inline void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Waits for phase `parity` of the barrier; gives up after `limit` polls. Returns true when
// the phase completed.
__device__ inline bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Stages `bytes` (multiple of 16, both addresses 16-byte aligned) from global into shared
// memory with one bulk copy issued by thread 0. Every thread of the block calls it. On a
// timed-out wait the block records MKB_ERR_TIMEOUT, waits once more (bounded) for the copy
// still in flight, and the function returns false: the caller must return without touching
// the staged data. A block that stages repeatedly through the same barrier passes the number of
// earlier uses (`use`): the barrier is initialised on the first and waited on by phase parity.
__device__ inline bool stage_to_shared(void* dst, const void* src, uint32_t bytes,
                                       uint64_t* bar, uint32_t use = 0) {
    // alignment guard: a misaligned bulk copy faults, so record the error and skip it
    if (((smem_addr(dst) | reinterpret_cast<uintptr_t>(src) | bytes) & 15u) != 0 ||
        (smem_addr(bar) & 7u) != 0) {
        if (threadIdx.x == 0) atomicExch(&g_device_error, MKB_ERR_ARGUMENT);
        return false;
    }
    if (threadIdx.x == 0 && use == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_expect_tx(bar, bytes);
        bulk_copy_g2s(dst, src, bytes, bar);
    }
    bool ok = mbar_wait(bar, use & 1u, g_wait_polls);
    ok = __syncthreads_and(ok);
    if (!ok) {
        if (threadIdx.x == 0) atomicExch(&g_device_error, MKB_ERR_TIMEOUT);
        // the copy may still be in flight: drain it (bounded, full limit) before the block
        // leaves, so that no bulk copy writes into shared memory a later block owns
        mbar_wait(bar, use & 1u, MKB_WAIT_POLLS_DEFAULT);
        __syncthreads();
    }
    return ok;
}

// Stages `count` records of `bytes` each (multiple of 16, 16-byte aligned) from src[j] into
// dst + j * dst_stride doubles with one barrier: thread 0 expects the total and issues one bulk
// copy per record whose src[j] is not null. Waits and error handling as stage_to_shared.
__device__ inline bool stage_records(double* dst, int dst_stride, const double* const* src,
                                     int count, uint32_t bytes, uint64_t* bar) {
    bool bad = (smem_addr(dst) & 15u) != 0 || (bytes & 15u) != 0 ||
               ((dst_stride * 8) & 15) != 0 || (smem_addr(bar) & 7u) != 0;
    uint32_t total = 0;
    for (int j = 0; j < count; ++j)
        if (src[j] != nullptr) {
            bad |= (reinterpret_cast<uintptr_t>(src[j]) & 15u) != 0;
            total += bytes;
        }
    if (bad) {
        if (threadIdx.x == 0) atomicExch(&g_device_error, MKB_ERR_ARGUMENT);
        return false;
    }
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_expect_tx(bar, total);
        for (int j = 0; j < count; ++j)
            if (src[j] != nullptr) bulk_copy_g2s(dst + j * dst_stride, src[j], bytes, bar);
    }
    bool ok = mbar_wait(bar, 0, g_wait_polls);
    ok = __syncthreads_and(ok);
    if (!ok) {
        if (threadIdx.x == 0) atomicExch(&g_device_error, MKB_ERR_TIMEOUT);
        mbar_wait(bar, 0, MKB_WAIT_POLLS_DEFAULT);
        __syncthreads();
    }
    return ok;
}

// ---- number types of the FP64 trace ------------------------------------------------------
// `double`: operators as written, the compiler may contract a*b+c into one FMA (faster, not
// bit-identical to the CPU). `Exact64`: every operation is a separately rounded IEEE operation
// (__dadd_rn, __dmul_rn, ... are never fused), division and square root are correctly
// rounded -- the same arithmetic as the reference CPU build (-ffp-contract=off), so a trace
// written in the reference's order of operations reproduces it bit for bit.
struct Exact64 {
    double v;
    Exact64() = default;
    __host__ __device__ constexpr Exact64(double x) : v(x) {}
};
__device__ __forceinline__ Exact64 operator+(Exact64 a, Exact64 b) { return __dadd_rn(a.v, b.v); }
__device__ __forceinline__ Exact64 operator-(Exact64 a, Exact64 b) { return __dsub_rn(a.v, b.v); }
__device__ __forceinline__ Exact64 operator*(Exact64 a, Exact64 b) { return __dmul_rn(a.v, b.v); }
__device__ __forceinline__ Exact64 operator/(Exact64 a, Exact64 b) { return __ddiv_rn(a.v, b.v); }
__device__ __forceinline__ Exact64 operator-(Exact64 a) { return -a.v; }
__device__ __forceinline__ Exact64& operator+=(Exact64& a, Exact64 b) { return a = a + b; }
__device__ __forceinline__ Exact64& operator-=(Exact64& a, Exact64 b) { return a = a - b; }
__device__ __forceinline__ bool operator<(Exact64 a, Exact64 b) { return a.v < b.v; }
__device__ __forceinline__ bool operator>(Exact64 a, Exact64 b) { return a.v > b.v; }
__device__ __forceinline__ bool operator>=(Exact64 a, Exact64 b) { return a.v >= b.v; }
__device__ __forceinline__ Exact64 nsqrt(Exact64 a) { return __dsqrt_rn(a.v); }

// `Exact32`: the same for float (the FP32 prefilter): every operation separately rounded,
// division and square root correctly rounded -- the reference's CPU float arithmetic.
struct Exact32 {
    float v;
    Exact32() = default;
    __host__ __device__ constexpr Exact32(float x) : v(x) {}
    __host__ __device__ constexpr Exact32(double x) : v(static_cast<float>(x)) {}
};
__device__ __forceinline__ Exact32 operator+(Exact32 a, Exact32 b) { return __fadd_rn(a.v, b.v); }
__device__ __forceinline__ Exact32 operator-(Exact32 a, Exact32 b) { return __fsub_rn(a.v, b.v); }
__device__ __forceinline__ Exact32 operator*(Exact32 a, Exact32 b) { return __fmul_rn(a.v, b.v); }
__device__ __forceinline__ Exact32 operator/(Exact32 a, Exact32 b) { return __fdiv_rn(a.v, b.v); }
__device__ __forceinline__ Exact32 operator-(Exact32 a) { return -a.v; }
__device__ __forceinline__ Exact32& operator+=(Exact32& a, Exact32 b) { return a = a + b; }
__device__ __forceinline__ Exact32& operator-=(Exact32& a, Exact32 b) { return a = a - b; }
__device__ __forceinline__ bool operator<(Exact32 a, Exact32 b) { return a.v < b.v; }
__device__ __forceinline__ bool operator>(Exact32 a, Exact32 b) { return a.v > b.v; }
__device__ __forceinline__ bool operator>=(Exact32 a, Exact32 b) { return a.v >= b.v; }
__device__ __forceinline__ Exact32 nsqrt(Exact32 a) { return __fsqrt_rn(a.v); }
__device__ __forceinline__ float value_of(Exact32 a) { return a.v; }
__device__ __forceinline__ double nsqrt(double a) { return sqrt(a); }
__device__ __forceinline__ float nsqrt(float a) { return sqrtf(a); }
__device__ __forceinline__ double value_of(double a) { return a; }
__device__ __forceinline__ double value_of(Exact64 a) { return a.v; }
__device__ __forceinline__ float value_of(float a) { return a; }

// ---- ray state and surface step -------------------------------------------------------------
// Formulas and order of operations: transfer_to_tangent_plane, intersect_sphere and
// refract_sphere (reference trace/surface_ops.hpp:122,144,181), propagate_surface_local
// (trace/trace.hpp:174), reference_sphere_step (trace/reference_sphere.hpp:55).
template <class N>
struct RayT {
    N px, py, pz, dx, dy, dz, opl;
};

template <class N>
struct SoftT {
    N penalty;
    int first;
    __device__ void add(N amount, int kind) {
        penalty += amount;
        if (first == kOk) first = kind;
    }
};

// The quantities of one surface step that its reverse sweep needs and that cost a division
// or a square root: the transfer length s0, the intersection length s, sqrt(D), mu = n / n'
// and sqrt(k) of the refraction.
template <class N>
struct StepLocal {
    N s0, s, root_d, mu, root_k;
};

// One surface step (stop/plane: c = 0) with mu = n / n' given (the rounded quotient of the
// two indices, taken once per surface and wavelength by callers that trace many rays).
// Returns the status; `branch` gets the taken soft-failure continuation. With soft == nullptr
// the hard-failure rules apply. kKeep also returns the step's StepLocal quantities (the
// arithmetic is the same either way).
template <class N, bool kKeep = false>
__device__ __forceinline__ int step_surface_mu(RayT<N>& r, N t, N c, N n_before, N mu,
                                               SoftT<N>* soft, int& branch,
                                               StepLocal<N>* keep = nullptr) {
    const N zero(0.0), one(1.0);
    if (!(r.dz > zero)) return kBackward;
    // transfer to the tangent plane
    r.pz -= t;
    const N s0 = -r.pz / r.dz;
    if constexpr (kKeep) keep->s0 = s0;
    r.px = r.px + s0 * r.dx;
    r.py = r.py + s0 * r.dy;
    r.pz = zero;
    // intersection with the sphere (Spencer-Murty form)
    const N H = c * (r.px * r.px + r.py * r.py);
    const N B = r.dz - c * (r.px * r.dx + r.py * r.dy);
    const N D = B * B - c * H;
    N s;
    bool missed = false;
    if (D < zero) {
        if (soft == nullptr || (!(c > zero) && !(c < zero))) return kMissed;
        soft->add(-D, kSoftMissed);
        s = B / c;
        missed = true;
        if constexpr (kKeep) keep->root_d = zero;
    } else {
        const N root_d = nsqrt(D);
        const N denom = B + root_d;
        if (!(denom > zero)) return kMissed;
        s = H / denom;
        if constexpr (kKeep) keep->root_d = root_d;
    }
    if constexpr (kKeep) keep->s = s;
    r.px = r.px + s * r.dx;
    r.py = r.py + s * r.dy;
    r.pz = r.pz + s * r.dz;
    r.opl += n_before * (s0 + s);
    // refraction, mu = n / n'
    if constexpr (kKeep) keep->mu = mu;
    N nx = -c * r.px, ny = -c * r.py, nz = one - c * r.pz;
    if (missed) {
        const N inv = one / nsqrt(nx * nx + ny * ny + nz * nz);
        nx = inv * nx;
        ny = inv * ny;
        nz = inv * nz;
    }
    const N cos_i = r.dx * nx + r.dy * ny + r.dz * nz;
    const N k = one - mu * mu * (one - cos_i * cos_i);
    branch = missed ? kBranchSoftMissed : kBranchRegular;
    if (k < zero) {
        if (soft == nullptr) return kTir;
        soft->add(-k, kSoftTir);
        if constexpr (kKeep) keep->root_k = zero;
        const N tx = r.dx - cos_i * nx, ty = r.dy - cos_i * ny, tz = r.dz - cos_i * nz;
        const N inv = one / nsqrt(tx * tx + ty * ty + tz * tz);
        r.dx = inv * tx;
        r.dy = inv * ty;
        r.dz = inv * tz;
        branch |= kBranchSoftTir;
        return kOk;
    }
    const N root_k = nsqrt(k);
    if constexpr (kKeep) keep->root_k = root_k;
    const N a = root_k - mu * cos_i;
    r.dx = mu * r.dx + a * nx;
    r.dy = mu * r.dy + a * ny;
    r.dz = mu * r.dz + a * nz;
    return kOk;
}

// One surface step with mu = n_before / n_after divided here.
template <class N, bool kKeep = false>
__device__ __forceinline__ int step_surface(RayT<N>& r, N t, N c, N n_before, N n_after,
                                            SoftT<N>* soft, int& branch,
                                            StepLocal<N>* keep = nullptr) {
    return step_surface_mu<N, kKeep>(r, t, c, n_before, n_before / n_after, soft, branch, keep);
}

// ---- ghost plates (trace/ghost_plate.hpp) ---------------------------------------------------
// One plate at one wavelength: profile coefficients a_1..a_K, normalisation radius r_g, glass
// index n_G (GhostPlateParams, ghost_plate.hpp:24).
struct GhostData {
    const double* coeff;
    int K;
    double radius;
    double n_glass;
};

// The plate data of surface s at wavelength l when the kernel was built for ghost plates
// (kGhost) and s is one; false otherwise (at compile time for kernels without plates).
template <bool kGhost>
__device__ __forceinline__ bool ghost_at(const TraceParams& p, const double* rec,
                                         const RecordLayout& lay, int s, int l, GhostData& g) {
    if constexpr (!kGhost) {
        return false;
    } else {
        const int gi = p.ghost_of[s];
        if (gi < 0) return false;
        g = {rec + lay.ghost_coeff + gi * p.K, p.K, rec[lay.ghost_radius + gi],
             rec[lay.ghost_index + gi * p.L + l]};
        return true;
    }
}

// The plain double and float steps divide by a quantity that does not depend on the ray (a
// small integer, a refractive index) by multiplying with its rounded reciprocal: within an ulp
// of the division and off the ray's dependent chain. Exact64 (the reference's order of
// operations) and Df64 keep the division.
template <class N>
constexpr bool kMulByReciprocal = std::is_same<N, double>::value || std::is_same<N, float>::value;

// 1 / k for k = 1 .. 36, rounded at compile time (the Legendre recurrences' 1 / (k + 1))
#define MKB_RECIP4(k) 1.0 / (k), 1.0 / ((k) + 1), 1.0 / ((k) + 2), 1.0 / ((k) + 3)
static __constant__ double kRecipInt[37] = {0.0,            MKB_RECIP4(1),  MKB_RECIP4(5),
                                            MKB_RECIP4(9),  MKB_RECIP4(13), MKB_RECIP4(17),
                                            MKB_RECIP4(21), MKB_RECIP4(25), MKB_RECIP4(29),
                                            MKB_RECIP4(33)};
#undef MKB_RECIP4
static_assert(kMaxGhostTerms + 1 <= 36, "kRecipInt covers 1 / (k + 1) for k <= kMaxGhostTerms");

// x / (k + 1) in the Legendre recurrence
template <class N>
__device__ __forceinline__ N legendre_div(N x, int k) {
    if constexpr (kMulByReciprocal<N>) return x * N(kRecipInt[k + 1]);
    else return x / N(double(k + 1));
}

// Thickness profile t(u) = sum_k a_k P_k(2u - 1) and dt/du = 2 sum_k a_k P'_k(2u - 1) by the
// Legendre recurrences in ascending k (ghost_profile, ghost_plate.hpp:67).
template <class N>
__device__ __forceinline__ void ghost_profile(const GhostData& g, N u, N& t, N& dt_du) {
    const N one(1.0), two(2.0);
    const N xi = two * u - one;
    N p_prev = one, p_cur = xi, dp_prev(0.0), dp_cur = one;
    N tt(0.0), dt(0.0);
    for (int k = 1; k <= g.K; ++k) {
        const N a = g.coeff[k - 1];
        tt += a * p_cur;
        dt += a * dp_cur;
        const N p_next = legendre_div<N>(N(double(2 * k + 1)) * xi * p_cur - N(double(k)) * p_prev,
                                         k);
        const N dp_next = dp_prev + N(double(2 * k + 1)) * p_cur;
        p_prev = p_cur;
        p_cur = p_next;
        dp_prev = dp_cur;
        dp_cur = dp_next;
    }
    t = tt;
    dt_du = two * dt;
}

// The step onto a ghost plate (propagate_surface_local with kind GhostPlate, trace.hpp:191, and
// ghost_plate_step / phase_surface_step, ghost_plate.hpp:130,159): transfer to the plane z = 0,
// OPL += n s0, OPL += Phi = (n_G - n) t(u), n' d'_perp = n d_perp + grad Phi, d'_z =
// sqrt(1 - |d'_perp|^2); a negative radicand is TIR (soft: penalty -radicand, d' in the plane).
template <class N, bool kKeep = false>
__device__ __forceinline__ int ghost_step(RayT<N>& r, N t, N n_before, N n_after,
                                          const GhostData& g, SoftT<N>* soft, int& branch,
                                          StepLocal<N>* keep = nullptr) {
    const N zero(0.0), one(1.0), two(2.0);
    if (!(r.dz > zero)) return kBackward;
    r.pz -= t;
    const N s0 = -r.pz / r.dz;
    r.px = r.px + s0 * r.dx;
    r.py = r.py + s0 * r.dy;
    r.pz = zero;
    r.opl += n_before * s0;
    const N radius = g.radius;
    const N inv_r2 = one / (radius * radius);
    const N u = (r.px * r.px + r.py * r.py) * inv_r2;
    N prof_t, dt_du;
    ghost_profile<N>(g, u, prof_t, dt_du);
    const N dn = N(g.n_glass) - n_before;
    const N radial = dn * dt_du * two * inv_r2;
    const N gx = radial * r.px, gy = radial * r.py;
    r.opl += dn * prof_t;
    N dx, dy;
    if constexpr (kMulByReciprocal<N>) {
        const N inv_after = one / n_after;
        dx = (n_before * r.dx + gx) * inv_after;
        dy = (n_before * r.dy + gy) * inv_after;
    } else {
        dx = (n_before * r.dx + gx) / n_after;
        dy = (n_before * r.dy + gy) / n_after;
    }
    const N radicand = one - dx * dx - dy * dy;
    if constexpr (kKeep) *keep = {s0, zero, zero, zero, zero};
    branch = kBranchRegular;
    if (radicand < zero) {
        if (soft == nullptr) return kTir;
        soft->add(-radicand, kSoftTir);
        const N inv = one / nsqrt(dx * dx + dy * dy);
        r.dx = dx * inv;
        r.dy = dy * inv;
        r.dz = zero;
        branch = kBranchSoftTir;
        return kOk;
    }
    r.dx = dx;
    r.dy = dy;
    r.dz = nsqrt(radicand);
    return kOk;
}

// ---- decenter and tilt of a surface (trace/surface_transform.hpp:27-85) -----------------
// R = R_y(b) R_x(a); a point q of the tilted surface frame lies at R q + (dx, dy, 0) in the
// nominal frame. xf points at the surface's kXfValues record values.
template <class N>
struct Transform {
    N dx, dy, ca, sa, cb, sb;
};

template <class N>
__device__ __forceinline__ Transform<N> transform_at(const double* xf) {
    return {N(xf[0]), N(xf[1]), N(xf[2]), N(xf[3]), N(xf[4]), N(xf[5])};
}

// R^T v (rotate_to_surface)
template <class N>
__device__ __forceinline__ void rotate_to(const Transform<N>& t, N& vx, N& vy, N& vz) {
    const N x = t.cb * vx - t.sb * vz;
    const N z = t.sb * vx + t.cb * vz;
    const N y = t.ca * vy + t.sa * z;
    vz = t.ca * z - t.sa * vy;
    vx = x;
    vy = y;
}

// R v (rotate_from_surface)
template <class N>
__device__ __forceinline__ void rotate_from(const Transform<N>& t, N& vx, N& vy, N& vz) {
    const N y = t.ca * vy - t.sa * vz;
    const N z = t.sa * vy + t.ca * vz;
    const N x = t.cb * vx + t.sb * z;
    vz = t.cb * z - t.sb * vx;
    vx = x;
    vy = y;
}

// ray_to_surface: p <- R^T (p - D), d <- R^T d
template <class N>
__device__ __forceinline__ void ray_to_surface(RayT<N>& r, const Transform<N>& t) {
    N x = r.px - t.dx, y = r.py - t.dy, z = r.pz;
    rotate_to(t, x, y, z);
    r.px = x;
    r.py = y;
    r.pz = z;
    rotate_to(t, r.dx, r.dy, r.dz);
}

// ray_from_surface: p <- R p + D, d <- R d
template <class N>
__device__ __forceinline__ void ray_from_surface(RayT<N>& r, const Transform<N>& t) {
    N x = r.px, y = r.py, z = r.pz;
    rotate_from(t, x, y, z);
    r.px = x + t.dx;
    r.py = y + t.dy;
    r.pz = z;
    rotate_from(t, r.dx, r.dy, r.dz);
}

// propagate_surface (trace/trace.hpp:233): the step onto surface s with its transform when
// the batch is non-coaxial and the surface moved (xf = its record values, or null): d_z > 0,
// z -= t in the nominal frame, into the tilted frame, the local step with t = 0 (its own
// d_z > 0 check), and back into the nominal frame when it succeeded. The StepLocal values
// are those of the local step.
// `ghost` (or null): the surface is a ghost plate with these data; the step then divides by
// n_after itself (mu is not used).
template <class N, bool kKeep = false>
__device__ __forceinline__ int step_surface_xf(RayT<N>& r, N t, N c, N n_before, N mu,
                                               const double* xf, SoftT<N>* soft, int& branch,
                                               StepLocal<N>* keep = nullptr,
                                               const GhostData* ghost = nullptr,
                                               N n_after = N(1.0)) {
    auto local = [&](N tl) {
        return ghost != nullptr
                   ? ghost_step<N, kKeep>(r, tl, n_before, n_after, *ghost, soft, branch, keep)
                   : step_surface_mu<N, kKeep>(r, tl, c, n_before, mu, soft, branch, keep);
    };
    if (xf == nullptr || !(xf[6] > 0.0)) return local(t);
    if (!(r.dz > N(0.0))) return kBackward;
    r.pz -= t;
    const Transform<N> tr = transform_at<N>(xf);
    ray_to_surface(r, tr);
    const int st = local(N(0.0));
    if (st == kOk) ray_from_surface(r, tr);
    return st;
}

// Record values of surface s's transform when the kernel was built for non-coaxial records
// (kXf), else null at compile time: a coaxial launch carries no transform code.
template <bool kXf>
__device__ __forceinline__ const double* xf_at(const double* rec, const RecordLayout& lay, int s) {
    if constexpr (kXf) return rec + lay.xf + s * kXfValues;
    else return nullptr;
}

// Record values of surface s's transform, or null (coaxial batch).
__device__ __forceinline__ const double* xf_of(const double* rec, const RecordLayout& lay, int s) {
    return lay.xf >= 0 ? rec + lay.xf + s * kXfValues : nullptr;
}

// Step onto the reference sphere about M = (0, h, w) through the vertex of the last surface.
template <class N>
__device__ __forceinline__ int reference_step(RayT<N>& r, N h, N w, N n_image, SoftT<N>* soft,
                                              int& branch) {
    const N zero(0.0), two(2.0);
    const N qx = r.px, qy = r.py - h, qz = r.pz - w;
    const N b = -(qx * r.dx + qy * r.dy + qz * r.dz);
    const N g = r.px * r.px + r.py * (r.py - two * h) + r.pz * (r.pz - two * w);
    const N disc = b * b - g;
    branch = kBranchRegular;
    if (disc < zero) {
        const N radius_sq = h * h + w * w;
        if (soft == nullptr || !(radius_sq > zero)) return kMissed;
        soft->add(-disc / radius_sq, kSoftMissed);
        r.px = r.px + b * r.dx;
        r.py = r.py + b * r.dy;
        r.pz = r.pz + b * r.dz;
        r.opl += n_image * b;
        branch = kBranchSoftMissed;
        return kSoftMissed;
    }
    const N root = nsqrt(disc);
    const bool real_image = w >= zero;
    const N denom = real_image ? b + root : b - root;
    if (!(real_image ? denom > zero : denom < zero)) return kMissed;
    const N s = g / denom;
    r.px = r.px + s * r.dx;
    r.py = r.py + s * r.dy;
    r.pz = r.pz + s * r.dz;
    r.opl += n_image * s;
    return kOk;
}

// ---- FP32-bulk trace (MKB_PRECISION_FP32_BULK) -------------------------------------------------
// The ray's position, its optical path and the steps that need FP64 for stability in double;
// its direction and the refraction in float. Same formulas and branches as step_surface_mu.
struct RayBulk {
    double px, py, pz;
    float dx, dy, dz;
    double opl;
};

// kKeep: the step's quantities for the reverse sweep (s0, s, sqrt D, sqrt k; mu is the
// caller's), rounded to float as the MIXED sweep keeps them.
template <bool kKeep = false>
__device__ __forceinline__ int step_surface_bulk(RayBulk& r, double t, double c, double n_before,
                                                 float mu, SoftT<double>* soft, int& branch,
                                                 StepLocal<float>* keep = nullptr) {
    if (!(r.dz > 0.0f)) return kBackward;
    // transfer to the tangent plane (FP64: the point must land on z = 0)
    r.pz -= t;
    const double dxd = r.dx, dyd = r.dy, dzd = r.dz;
    const double s0 = -r.pz / dzd;
    if constexpr (kKeep) keep->s0 = static_cast<float>(s0);
    r.px = r.px + s0 * dxd;
    r.py = r.py + s0 * dyd;
    r.pz = 0.0;
    // the cancellation-safe intersection with the sphere (FP64)
    const double H = c * (r.px * r.px + r.py * r.py);
    const double B = dzd - c * (r.px * dxd + r.py * dyd);
    const double D = B * B - c * H;
    double s;
    bool missed = false;
    if (D < 0.0) {
        if (soft == nullptr || (!(c > 0.0) && !(c < 0.0))) return kMissed;
        soft->add(-D, kSoftMissed);
        s = B / c;
        missed = true;
        if constexpr (kKeep) keep->root_d = 0.0f;
    } else {
        const double root_d = sqrt(D);
        const double denom = B + root_d;
        if (!(denom > 0.0)) return kMissed;
        s = H / denom;
        if constexpr (kKeep) keep->root_d = static_cast<float>(root_d);
    }
    if constexpr (kKeep) keep->s = static_cast<float>(s);
    r.px = r.px + s * dxd;
    r.py = r.py + s * dyd;
    r.pz = r.pz + s * dzd;
    r.opl += n_before * (s0 + s);
    // refraction in FP32, mu = n / n'
    const float cf = static_cast<float>(c);
    float nx = -cf * static_cast<float>(r.px), ny = -cf * static_cast<float>(r.py);
    float nz = 1.0f - cf * static_cast<float>(r.pz);
    if (missed) {
        const float inv = rsqrtf(nx * nx + ny * ny + nz * nz);
        nx *= inv;
        ny *= inv;
        nz *= inv;
    }
    const float cos_i = r.dx * nx + r.dy * ny + r.dz * nz;
    const float k = 1.0f - mu * mu * (1.0f - cos_i * cos_i);
    branch = missed ? kBranchSoftMissed : kBranchRegular;
    float ex, ey, ez;
    if (k < 0.0f) {
        if (soft == nullptr) return kTir;
        soft->add(-static_cast<double>(k), kSoftTir);
        if constexpr (kKeep) keep->root_k = 0.0f;
        ex = r.dx - cos_i * nx;
        ey = r.dy - cos_i * ny;
        ez = r.dz - cos_i * nz;
        branch |= kBranchSoftTir;
    } else {
        const float root_k = sqrtf(k);
        if constexpr (kKeep) keep->root_k = root_k;
        const float a = root_k - mu * cos_i;
        ex = mu * r.dx + a * nx;
        ey = mu * r.dy + a * ny;
        ez = mu * r.dz + a * nz;
    }
    // unit length: one Newton step of 1 / |e| from 1 (|e| = 1 up to float rounding after a
    // refraction; the TIR tangent needs the full normalisation)
    const float e2 = ex * ex + ey * ey + ez * ez;
    const float inv = k < 0.0f ? rsqrtf(e2) : 1.5f - 0.5f * e2;
    r.dx = inv * ex;
    r.dy = inv * ey;
    r.dz = inv * ez;
    return kOk;
}

// reference_step with the float direction (FP64 arithmetic).
__device__ __forceinline__ int reference_step_bulk(RayBulk& r, double h, double w,
                                                   double n_image, SoftT<double>* soft,
                                                   int& branch) {
    RayT<double> q{r.px, r.py, r.pz, r.dx, r.dy, r.dz, r.opl};
    const int st = reference_step<double>(q, h, w, n_image, soft, branch);
    r.px = q.px;
    r.py = q.py;
    r.pz = q.pz;
    r.opl = q.opl;
    return st;
}

// ---- optimiser variables (VariableSet, reference include/mikroptim/optim/variable_set.hpp:63)
struct VarParams {
    int P;
    int8_t type[MKB_MAX_VARIABLES];       // MKB_VAR_*
    int8_t surface[MKB_MAX_VARIABLES];    // table surface of the parameter
    int8_t col_curvature[kMaxSurfaces];   // column of curvature[s], -1 if none
    int8_t col_thickness[kMaxSurfaces];   // column of thickness[s], -1 if none
    int8_t ghost_plate[MKB_MAX_VARIABLES];  // GhostCoefficient variables: plate g
    int8_t ghost_order[MKB_MAX_VARIABLES];  // and order k (1 .. K)
    int8_t col_ghost[kMaxGhostPlates][kMaxGhostTerms];  // column of a_{k+1} of plate g, or -1
    int8_t glass_component[MKB_MAX_VARIABLES];  // Glass variables: 0 n0, 1 nu1, 2 nu2
    int8_t col_glass[kMaxSurfaces][3];          // column of (n0, nu1, nu2) of medium s, or -1
    int has_glass;                              // any Glass variable
    // the lowest slot c (the step onto surface c + 1) whose reverse step writes a column:
    // the reverse sweep of the fused kernel ends there, the steps below it feed no variable
    int sweep_floor;
    int L;                                      // wavelengths (glass index refresh)
    double omega[MKB_MAX_WAVELENGTHS];          // Buchdahl coordinate of every wavelength
    double lower[MKB_MAX_VARIABLES], upper[MKB_MAX_VARIABLES], typical[MKB_MAX_VARIABLES];
};

// Builds the variable block for a batch with S surfaces; MKB_OK or MKB_ERR_ARGUMENT.
// ghost_terms: K of the batch (GhostCoefficient variables need k <= K).
int make_var_params(const mkb_variables* vars, int S, const uint8_t* type, VarParams* out,
                    int ghost_terms = 0, int L = 0, const double* wavelength_nm = nullptr,
                    int glass = 0);

// The sweep floor (VarParams::sweep_floor) of a variable set, from its raw arrays (the same
// rule make_var_params applies; the set must be valid).
int sweep_floor_of(const mkb_variables* vars, int S, const uint8_t* type);

// Writes x into a packed record (VariableSet::apply, src/optim/variable_set.cpp:237).
// Writes variable k's value into a record (curvature, thickness / working distance, or a ghost
// plate's profile coefficient).
__device__ __forceinline__ void write_variable(const VarParams& v, const RecordLayout& lay, int k,
                                               double x, double* rec) {
    const int s = v.surface[k];
    if (v.type[k] == MKB_VAR_CURVATURE) rec[lay.curvature + s] = x;
    else if (v.type[k] == MKB_VAR_GHOST_COEFFICIENT)
        rec[lay.ghost_coeff + v.ghost_plate[k] * lay.ghost_terms + v.ghost_order[k] - 1] = x;
    else if (v.type[k] == MKB_VAR_GLASS) rec[lay.glass + s * 4 + v.glass_component[k]] = x;
    else rec[lay.thickness + s] = x;
}

// Recomputes the index of every medium with a glass variable from its Buchdahl coefficients,
// n = n0 + w (nu1 + w (nu2 + w nu3)) with separately rounded operations (buchdahl_index,
// glass/dispersion.hpp:93, as VariableSet::apply does on the host).
__device__ __forceinline__ void refresh_glass(const VarParams& v, const RecordLayout& lay,
                                              double* rec) {
    if (!v.has_glass) return;
    for (int s = 0; s < lay.surfaces; ++s) {
        if (v.col_glass[s][0] < 0 && v.col_glass[s][1] < 0 && v.col_glass[s][2] < 0) continue;
        const double* b = rec + lay.glass + s * 4;
        for (int l = 0; l < v.L; ++l) {
            const double w = v.omega[l];
            const double inner = __dadd_rn(b[2], __dmul_rn(w, b[3]));
            const double mid = __dadd_rn(b[1], __dmul_rn(w, inner));
            rec[lay.index + s * v.L + l] = __dadd_rn(b[0], __dmul_rn(w, mid));
        }
    }
}

__device__ __forceinline__ void apply_variables(const VarParams& v, const RecordLayout& lay,
                                                const double* x, double* rec) {
    for (int k = 0; k < v.P; ++k) write_variable(v, lay, k, x[k], rec);
    refresh_glass(v, lay, rec);
    if (lay.stop > 0) aim_record(lay, rec);  // the entrance pupil follows the variables
}

// d(a, t0)/dx_k of the aimed entrance pupil (aim_record) for variable k: the y-u trace of
// aim_heights carrying every quantity's derivative with respect to x_k (a curvature or a
// thickness of a surface before the stop, or a Buchdahl component of a medium before it, whose
// index at wavelength column 0 moves with slope w^c); 0 for every other variable. Forward-mode
// derivatives of the same arithmetic (contraction allowed: the adjoint rows are not bit-exact).
__device__ inline void aim_sensitivity(const double* rec, const RecordLayout& lay,
                                       const VarParams& v, int k, double& da, double& dt0) {
    const int type = v.type[k], sk = v.surface[k];
    double slope = 0.0;
    if (type == MKB_VAR_GLASS) {
        const double w = v.omega[0];
        slope = v.glass_component[k] == 0 ? 1.0 : v.glass_component[k] == 1 ? w : w * w;
    }
    double y1 = 1.0, u1 = 0.0, y2 = 0.0, u2 = 1.0;
    double dy1 = 0.0, du1 = 0.0, dy2 = 0.0, du2 = 0.0;
    double n = rec[lay.index];
    double dn = type == MKB_VAR_GLASS && sk == 0 ? slope : 0.0;
    for (int s = 1; s < lay.stop; ++s) {
        const double n2 = rec[lay.index + s * lay.L];
        const double dn2 = type == MKB_VAR_GLASS && sk == s ? slope : 0.0;
        const bool sphere = (lay.spheres >> s) & 1u;
        const double c = sphere ? rec[lay.curvature + s] : 0.0;
        const double dc = sphere && type == MKB_VAR_CURVATURE && sk == s ? 1.0 : 0.0;
        const double phi = c * (n2 - n);
        const double dphi = dc * (n2 - n) + c * (dn2 - dn);
        const double a1 = n * u1 - y1 * phi, a2 = n * u2 - y2 * phi;
        const double da1 = dn * u1 + n * du1 - dy1 * phi - y1 * dphi;
        const double da2 = dn * u2 + n * du2 - dy2 * phi - y2 * dphi;
        u1 = a1 / n2;
        u2 = a2 / n2;
        du1 = (da1 - u1 * dn2) / n2;
        du2 = (da2 - u2 * dn2) / n2;
        const double t = rec[lay.thickness + s];
        const double dt = type == MKB_VAR_THICKNESS && sk == s ? 1.0 : 0.0;
        dy1 += dt * u1 + t * du1;
        dy2 += dt * u2 + t * du2;
        y1 += t * u1;
        y2 += t * u2;
        n = n2;
        dn = dn2;
    }
    const double R = rec[lay.curvature + lay.stop];
    const double sgn = y1 < 0.0 ? -1.0 : 1.0;
    da = -R * sgn * dy1 / (y1 * y1);
    dt0 = -(dy2 * y1 - y2 * dy1) / (y1 * y1);
}

// ---- launch bookkeeping (host) -------------------------------------------------------------
void count_launch(int n = 1);
void set_error(const char* fmt, ...);
int cuda_status(cudaError_t err, const char* what);

// Rows of one variant's residual vector: rays, penalty rows (soft failure), transverse rows.
int64_t trace_rows_of(const mkb_residual_plan* plan, int64_t rays);

// residual_scale of every tuple (f-major, then l) into scale[F * L], as make_trace_params
// computes them; checks the plan first (MKB_OK or MKB_ERR_ARGUMENT).
int residual_scales(const mkb_residual_plan* plan, double* scale);

// Builds the parameter block from the batch and plan; returns MKB_OK or MKB_ERR_ARGUMENT.
// `pack_rays` = rays one CTA traces (tuples are packed until this many rays).
int make_trace_params(const mkb_device_batch* batch, const mkb_residual_plan* plan,
                      int pack_rays, TraceParams* out);

}  // namespace mkb
