// C++ host API of the B200 batched trace-and-optimise path.
//
// Mirrors the reference's host classes so that its callers (`mikroptim trace --gpu`,
// `mikroptim optimize --gpu`) can switch by changing the namespace:
//   BatchTopology, SystemBatchHost   include/mikroptim/batch/system_batch.hpp:229,268
//   ResidualSettings, ResidualLayout include/mikroptim/batch/batch_residuals.hpp:24,62
//   Variable, VariableSet            include/mikroptim/optim/variable_set.hpp:20,63
//   LmOptions, LmStatus              include/mikroptim/optim/levenberg_marquardt.hpp:26,85
//   cuda::TraceEngine                include/mikroptim/cuda/trace_engine.hpp
//   cuda::DeviceFdJacobian, cuda::DeviceAdjointJacobian, cuda::DeviceNormalEquations,
//   cuda::optimize_lm_gpu            include/mikroptim/cuda/*.hpp
// Everything runs through the C ABI of libmikroptim_b200.so (include/mikroptim_b200.h).
// Errors are thrown before any device work: std::invalid_argument for bad arguments,
// std::out_of_range for indices, std::logic_error for features this build does not trace,
// cuda::CudaError for device failures -- the reference's exception classes.
#pragma once

#include <cstddef>
#include <cstdint>
#include <functional>
#include <limits>
#include <memory>
#include <optional>
#include <span>
#include <stdexcept>
#include <string>
#include <vector>

#include "mikroptim_b200.h"

namespace mkb {

// ApertureStop: an aperture stop inside the system (no reference counterpart; its curvature
// slot holds the semi-aperture, surface 0 becomes the aimed entrance pupil,
// MKB_SURFACE_APERTURE_STOP)
enum class SurfaceKind : uint8_t { Stop = 0, Plane = 1, Sphere = 2, GhostPlate = 3,
                                   ApertureStop = 4 };
enum class PupilMode : uint8_t { Half = 0, Full = 1, Axis = 2 };
enum class FailureMode : int32_t { Soft = 0, Hard = 1 };
enum class Precision : int32_t { FP64 = 0, Mixed = 1, FP64_FMA = 2, DF64 = 3, FP32_Bulk = 4 };
enum class VariableType : int32_t { Curvature = 0, Thickness = 1, WorkingDistance = 2,
                                    GhostCoefficient = 3, Glass = 4 };
enum class JacobianMethod : int32_t { FiniteDifference = 0, Adjoint = 1 };
enum class LmStatus : int32_t {
    Running = 0, ConvergedMerit = 1, ConvergedStep = 2, ConvergedGradient = 3,
    ConvergedStall = 4, MaxIterations = 5, DampingLimit = 6, NumericalError = 7
};

// What every variant of a batch shares (one topology per batch).
struct BatchTopology {
    int surfaces = 0, wavelengths = 0, fields = 0;
    std::vector<SurfaceKind> type;      // [S], type[0] = Stop
    std::vector<PupilMode> pupil_mode;  // [F]
    // per-surface decenter and tilt (system_batch.hpp:45); every field then uses the Full pupil
    bool non_coaxial = false;
    // ghost plates: one per GhostPlate surface (table order), each with ghost_terms profile
    // coefficients (BatchTopology::ghost_plates / ghost_terms, system_batch.hpp:30)
    int ghost_plates = 0, ghost_terms = 0;
    void validate() const;
};

// V variants as FP64 structure of arrays, variant outermost.
class SystemBatchHost {
public:
    SystemBatchHost(BatchTopology topology, int variants);

    int variants() const { return variants_; }
    int surfaces() const { return topology_.surfaces; }
    int wavelengths() const { return topology_.wavelengths; }
    int fields() const { return topology_.fields; }
    const BatchTopology& topology() const { return topology_; }

    double& curvature(int v, int s) { return curvature_.at(index2(v, s, surfaces())); }
    double& thickness(int v, int s) { return thickness_.at(index2(v, s, surfaces())); }
    double& index(int v, int s, int l);
    double& pupil_radius(int v) { return pupil_radius_.at(check_v(v)); }
    double& field_angle(int v, int f) { return field_angle_.at(index2(v, f, fields())); }
    double& field_target(int v, int f) { return field_target_.at(index2(v, f, fields())); }
    double curvature(int v, int s) const { return curvature_.at(index2(v, s, surfaces())); }
    double thickness(int v, int s) const { return thickness_.at(index2(v, s, surfaces())); }
    // decenter dx, dy [mm] and tilts alpha, beta [rad] of surface s (k = 0..3); writing needs
    // a non-coaxial topology (std::invalid_argument otherwise), reading a coaxial batch gives 0
    // (SystemBatchHost::decenter_tilt, system_batch.hpp:156)
    double& decenter_tilt(int v, int s, int k);
    double decenter_tilt(int v, int s, int k) const;
    void set_decenter_tilt(int v, int s, double dx, double dy, double alpha, double beta);
    bool coaxial() const { return !topology_.non_coaxial; }
    // ghost plate g: profile coefficient a_{k+1}, glass index at wavelength l (per variant),
    // normalisation radius (shared), table surface (system_batch.hpp:102-131)
    double& ghost_coeff(int v, int g, int k);
    double& ghost_index(int v, int g, int l);
    double& ghost_norm_radius(int g);
    int ghost_surface(int g) const;
    // Buchdahl coefficients (n0, nu1, nu2, nu3) of the medium after surface s (j = 0..3); set
    // `glass` to pass them (and wavelength_nm) to the device for glass variables
    double& buchdahl_coeff(int v, int s, int j);
    double buchdahl_coeff(int v, int s, int j) const;
    // index[v][s][:] from the Buchdahl coefficients (buchdahl_index, glass/dispersion.hpp:93)
    void refresh_glass_index(int v, int s);

    double reference_wavelength_nm = 0.0;
    std::vector<double> wavelength_nm;      // [L] (glass variables)
    bool glass = false;                     // the batch carries Buchdahl coefficients
    std::vector<double> wavelength_weight;  // [L]
    std::vector<double> field_weight;       // [F]

    // validate_values (src/batch/system_batch.cpp:558) for the traced fields
    void validate_values() const;
    // C view over the arrays (valid while the batch is alive and unresized)
    mkb_batch_view view() const;

private:
    size_t check_v(int v) const;
    size_t index2(int v, int i, int n) const;
    BatchTopology topology_;
    int variants_;
    std::vector<uint8_t> type_;
    std::vector<double> curvature_, thickness_, index_, pupil_radius_, field_angle_,
        field_target_, decenter_tilt_, ghost_coeff_, ghost_index_, ghost_norm_radius_,
        buchdahl_coeff_;
    friend SystemBatchHost make_non_coaxial(const SystemBatchHost& batch);
    friend SystemBatchHost take_variants(const SystemBatchHost& batch,
                                         const std::vector<int>& variants);
};

// Batch of the listed variants of `batch`, in that order (lm_template_batch).
SystemBatchHost take_variants(const SystemBatchHost& batch, const std::vector<int>& variants);

// Copy of `batch` with a non-coaxial topology (decenter and tilt zero, Full pupils).
SystemBatchHost make_non_coaxial(const SystemBatchHost& batch);

struct ResidualSettings {
    int rings = 10;
    int spokes = 8;
    FailureMode failure = FailureMode::Soft;
    double fail_weight = 1e6;  // kDefaultFailWeight (merit/ray_residual.hpp:175)
    Precision precision = Precision::FP64;
    // transverse ray-error rows after the ray and penalty rows (no reference counterpart:
    // mkb_residual_plan.transverse_weight); 0 = none
    double transverse_weight = 0.0;
};

// The C plan for one batch; owns the arrays its pointers reference (not copyable).
class ResidualPlan {
public:
    const mkb_residual_plan* get() const { return &plan_; }
    ResidualPlan(const ResidualPlan&) = delete;
    ResidualPlan& operator=(const ResidualPlan&) = delete;

private:
    friend class ResidualLayout;
    ResidualPlan() = default;
    mkb_residual_plan plan_{};
    std::vector<uint8_t> modes_;
    std::vector<double> field_weight_, wavelength_weight_, u_, w_;
};

// Row layout of one variant: tuples (f, l) f-major then l, sample k = i*M + j inside a tuple,
// penalty rows after the ray rows in soft-failure mode.
class ResidualLayout {
public:
    ResidualLayout(const BatchTopology& topology, const ResidualSettings& settings);
    int64_t rays_per_variant() const { return rays_; }
    int64_t trace_rows() const;
    int64_t offset(int f, int l) const;
    int samples(int f) const { return samples_.at(f); }
    const ResidualSettings& settings() const { return settings_; }
    // the plan is heap-allocated so its internal pointers stay valid
    std::unique_ptr<ResidualPlan> plan(const SystemBatchHost& batch) const;
    // a plan with unit weights, for sizing runs of the topology (sizes ignore the weights)
    std::unique_ptr<ResidualPlan> plan_for_sizing() const;

private:
    std::unique_ptr<ResidualPlan> plan_from(const std::vector<double>& field_weight,
                                            const std::vector<double>& wavelength_weight,
                                            double reference_wavelength_nm) const;
    BatchTopology topology_;
    ResidualSettings settings_;
    std::vector<int> samples_;
    std::vector<int64_t> field_offset_;
    int64_t rays_ = 0;
};

struct Variable {
    VariableType type = VariableType::Curvature;
    int surface = 0;
    double lower = -std::numeric_limits<double>::infinity();
    double upper = std::numeric_limits<double>::infinity();
    double typical = 1.0;
    int ghost_plate = -1;  // GhostCoefficient: a_{ghost_order} of plate ghost_plate
    int ghost_order = 0;
    int glass_component = -1;  // Glass: 0 n0, 1 nu1, 2 nu2 of the medium after `surface`
};

class VariableSet {
public:
    VariableSet(const BatchTopology& topology, std::vector<Variable> variables);
    int size() const { return static_cast<int>(variables_.size()); }
    const std::vector<Variable>& variables() const { return variables_; }
    std::vector<double> extract(const SystemBatchHost& batch, int v) const;
    void apply(SystemBatchHost& batch, int v, const double* x) const;
    mkb_variables c_struct() const;

private:
    std::vector<Variable> variables_;
    std::vector<int32_t> type_, surface_, ghost_plate_, ghost_order_, glass_component_;
    std::vector<double> lower_, upper_, typical_;
};

// ExtraResiduals (include/mikroptim/optim/extra_residuals.hpp): `count` rows per variant after
// the trace rows (paraxial constraints and the like); evaluate(batch, v, out) writes variant v's
// rows. The LM differentiates them centrally on the host with the FD Jacobian's pattern and
// adds sum_e r_e^2 to every merit (extra_rows_untraced, src/optim/adjoint_jacobian.cpp:245).
struct ExtraResiduals {
    int count = 0;
    std::function<void(const SystemBatchHost& batch, int v, std::span<double> out)> evaluate;
};

// TraceExtraResiduals (include/mikroptim/optim/trace_extra_residuals.hpp): rows from the
// per-surface extrema of the same trace (semi-diameter, incidence-angle constraints);
// evaluate(batch, v, extrema [S][2], out). Every FD point and trial point is traced with its
// extrema; their sum t^2 is added to the merit after the MERIT kernel's sum.
struct TraceExtraResiduals {
    int count = 0;
    std::function<void(const SystemBatchHost& batch, int v, std::span<const double> extrema,
                       std::span<double> out)>
        evaluate;
};

// Paraxial constraints evaluated on the device as the LM's extra rows (ParaxialConstraint,
// include/mikroptim/optim/paraxial_residuals.hpp:67; mkb_paraxial_constraint): no host phase
// in a cycle. column: the wavelength column of the paraxial index; analytic: the adjoint
// Jacobian of the y-nu trace instead of the reference's central differences.
struct ParaxialConstraint {
    int type = MKB_CONSTRAINT_FOCAL_LENGTH;  // ConstraintType order
    int mode = MKB_MODE_EQUAL;
    double weight = 1.0, target = 0.0;
    int reference_surface = 0;
    double offset = 0.0, shift = 0.0;
};
struct ParaxialConstraints {
    std::vector<ParaxialConstraint> items;
    int column = 0;
    bool analytic = false;
};

struct LmOptions {
    int max_iterations = 100;
    bool reject_new_failures = true;
    double ftol = 1e-10, xtol = 1e-10, gtol = 1e-10;
    double initial_damping = 1e-3;
    double max_damping = 1e16;
    double diag_floor = 1e-12;
    JacobianMethod jacobian = JacobianMethod::Adjoint;
    bool gram_exact = true;  // false: FP64 tensor cores (with the adjoint: J never in memory)
    // outer soft-failure penalty rounds (levenberg_marquardt.hpp:120-125): runs that end with
    // failed rays restart with w_fail x fail_weight_factor while it stays <= max_fail_weight
    double fail_weight_factor = 10.0;
    double max_fail_weight = 1e14;
    ExtraResiduals extra;  // the caller's extra rows (LmOptions::jacobian.extra); count 0: none
    TraceExtraResiduals trace_extra;  // rows from the trace's extrema (::jacobian.trace_extra)
    ParaxialConstraints paraxial;     // constraints on the device (no host phase)
    // the C struct; its constraint pointer refers to `storage`, which must outlive it
    mkb_lm_options c_struct(std::vector<mkb_paraxial_constraint>* storage = nullptr) const;
};

namespace cuda {

// The extra rows of the runs x0 [runs][P] (`base` holds 1 variant or one per run):
// jacobian [runs][P][E] and residuals [runs][E], bit-identical to the reference's
// extra_rows_cpu for the same evaluate function.
void extra_rows_host(const VariableSet& variables, const SystemBatchHost& base,
                     const std::vector<double>& x0, const ExtraResiduals& extra,
                     std::vector<double>& jacobian, std::vector<double>& residuals);

class CudaError : public std::runtime_error {
public:
    using std::runtime_error::runtime_error;
};

// Throws the reference's exception class for a non-zero mkb_status.
void check(int status, const char* what);

// One device allocation, grown on demand and reused (the reference's buffer reuse).
class DeviceBuffer {
public:
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : ptr_(o.ptr_), bytes_(o.bytes_) {
        o.ptr_ = nullptr;
        o.bytes_ = 0;
    }
    ~DeviceBuffer();
    void* reserve(size_t bytes);
    void* get() const { return ptr_; }
    size_t bytes() const { return bytes_; }
    void release();

private:
    void* ptr_ = nullptr;
    size_t bytes_ = 0;
};

enum class TraceMode { Residuals, Merit };
const char* to_string(TraceMode mode);

// MemoryReserve (include/mikroptim/batch/batch_memory.hpp:119): the engine leaves
// max(min_bytes, fraction * free) of the memory it sees as free untouched.
struct MemoryReserve {
    std::size_t min_bytes = std::size_t{256} << 20;
    double fraction = 0.05;
};

// EngineOptions (include/mikroptim/cuda/trace_engine.hpp:44): memory_limit_bytes caps the
// memory the engine regards as available (tranche tests, sharing a GPU).
struct EngineOptions {
    std::optional<std::size_t> memory_limit_bytes;
    MemoryReserve reserve{};
};

// TraceSettings (trace_engine.hpp:52). opd / status / extra_residuals apply to RESIDUALS (the
// extra rows follow the ray and penalty rows and are set to 0); extra_merit (empty or one
// value per variant, valid until run returns) to MERIT, added to each variant's merit after
// its tuple sums. precision: empty = the quadrature's. pack_rays changes only the run time.
// extrema: per variant and surface the largest ray height and the smallest cos I of the valid
// rays (SurfaceExtremaResult, hard maxima; coaxial batches, else std::logic_error).
struct TraceSettings {
    TraceSettings() = default;
    TraceSettings(const ResidualSettings& q) : quadrature(q) {}  // NOLINT: implicit on purpose
    ResidualSettings quadrature{};
    bool opd = false;
    bool status = true;
    int64_t extra_residuals = 0;
    bool extrema = false;
    std::span<const double> extra_merit{};
    std::optional<Precision> precision;
    int pack_rays = 512;
    int variants_per_cta = 1;  // runtime only, like pack_rays (the autotuner's second knob)
};

// TraceRunInfo (trace_engine.hpp:93)
struct TraceRunInfo {
    int variants = 0;
    int tranches = 0;
    int tranche_variants = 0;
    std::size_t budget_bytes = 0;
    std::size_t device_bytes = 0;
};

struct ResidualResult {
    int variants = 0;
    int64_t rays_per_variant = 0, penalty_rows = 0, stride = 0;
    std::vector<double> residuals;  // [V][stride]
    std::vector<double> opd;        // [V][rays] when requested
    std::vector<uint8_t> status;    // [V][rays] when requested
    std::vector<double> extrema;    // [V][S][2] when requested (largest height, smallest cos I)
};

struct MeritResult {
    int variants = 0;
    int64_t rays_per_variant = 0;
    std::vector<double> merit;          // [V]
    std::vector<int64_t> failed;        // [V]
    std::vector<int64_t> hard_failed;   // [V]
    std::vector<double> extrema;        // [V][S][2] when requested
};

// TraceOutput (trace_engine.hpp:103): the result of the run's mode; the other is empty.
struct TraceOutput {
    TraceMode mode = TraceMode::Residuals;
    std::optional<ResidualLayout> layout;
    ResidualResult residuals;
    MeritResult merit;
    TraceRunInfo info;
};

// ---- FP32 prefilter of multistart variants (batch_prefilter.hpp) ----------------------------
struct PrefilterCriteria {  // batch_prefilter.hpp:35
    double max_failed_fraction = 0.5;
    double max_merit = std::numeric_limits<double>::infinity();
    double max_merit_factor = std::numeric_limits<double>::infinity();
};
struct PrefilterMargins {  // batch_prefilter.hpp:52
    double boundary = 0.15;
    double opl_error_factor = 32.0;
    double merit_relative = 0.01;
};
struct PrefilterOptions {
    PrefilterCriteria criteria{};
    PrefilterMargins margins{};
};
// PrefilterSettings (trace_engine.hpp:80)
struct PrefilterSettings {
    ResidualSettings quadrature{};
    PrefilterOptions options{};
    std::span<const double> extra_merit{};
};
struct PrefilterStats {  // batch_prefilter.hpp:66
    int variants = 0;
    int64_t rays_per_variant = 0;
    std::vector<double> merit, optical_length;
    std::vector<int64_t> failed, uncertain_ok, uncertain_failed;
};
enum PrefilterReason : uint8_t { kPrefilterKeep = 0, kPrefilterFailedRays = 1,
                                 kPrefilterMeritAbsolute = 2, kPrefilterMeritRelative = 4 };
struct PrefilterResult {  // batch_prefilter.hpp:94
    PrefilterStats stats;
    std::vector<double> merit_lower, merit_upper;
    std::vector<uint8_t> reject;
    double reference_merit = std::numeric_limits<double>::infinity();
    int reference_variant = -1;
    int kept = 0;
    bool keep(int v) const { return reject.at(static_cast<size_t>(v)) == kPrefilterKeep; }
};

// ---- EVAL on the dense pupil grid (include/mikroptim/eval/eval.hpp) -----------------------
enum class EvalReference : int32_t { ExitPupil = 0, Vertex = 1, Infinite = 2 };
struct EvalSettings {  // eval.hpp:27
    int grid = 64;
    bool half_pupil = false;
    EvalReference reference = EvalReference::ExitPupil;
    double field_ray_offset = 1e-3;
    int paraxial_column = 0;  // wavelength column holding the paraxial index
    Precision precision = Precision::FP64;  // FP64 or FP64_FMA
};
struct EvalResult {  // eval.hpp:96, the reference's layout
    int variants = 0, fields = 0, wavelengths = 0;
    int64_t samples = 0;
    int grid_size = 0;  // N (EvalSettings::grid)
    bool half_pupil = false;
    double field_ray_offset = 1e-3;
    std::vector<double> grid;  // [n][3] x, y, weight
    std::vector<double> reference_curvature, exit_pupil_position;
    std::vector<double> opd, spot_x, spot_y, field_rays;
    std::vector<uint8_t> status, field_status;
};

// One tranche's RESIDUALS on the device (DeviceTranche, trace_engine.hpp:117); the pointers
// are the engine's buffers and valid during the callback only.
struct DeviceTranche {
    int first = 0;
    int count = 0;
    int64_t rays_per_variant = 0;
    int64_t penalty_rows = 0;
    int64_t stride = 0;
    const double* residuals = nullptr;    // [count][stride]
    const uint8_t* status = nullptr;      // [count][rays]
    const double* opd = nullptr;          // [count][rays] with settings.opd
};
using DeviceTrancheFn = std::function<void(const DeviceTranche&)>;

// Device-resident packed batch (records and surface types).
class DeviceSystemBatch {
public:
    DeviceSystemBatch() = default;
    void upload(const SystemBatchHost& batch, void* stream);
    // variants [first, first + count) only (a tranche)
    void upload(const SystemBatchHost& batch, int first, int count, void* stream);
    mkb_device_batch c_struct() const { return batch_; }
    std::size_t capacity_bytes() const { return records_.bytes(); }
    void release() { records_.release(); }

private:
    mkb_device_batch batch_{};
    std::vector<uint8_t> type_;
    std::vector<double> wavelength_nm_;
    std::vector<double> host_records_;
    DeviceBuffer records_;
};

// TraceEngine (include/mikroptim/cuda/trace_engine.hpp:145): host batch in, host results out.
// A batch is split into tranches that fit the device memory the engine sees (free memory plus
// its own buffers, at most memory_limit_bytes, less the reserve); buffers are kept across
// calls. Every variant's results are bit-identical whatever the split.
class TraceEngine {
public:
    explicit TraceEngine(int device = 0, const EngineOptions& options = {});
    ~TraceEngine();
    TraceEngine(const TraceEngine&) = delete;
    TraceEngine& operator=(const TraceEngine&) = delete;

    void run(const SystemBatchHost& batch, TraceMode mode, const TraceSettings& settings,
             TraceOutput& out);
    TraceOutput run(const SystemBatchHost& batch, TraceMode mode,
                    const TraceSettings& settings = {});
    // RESIDUALS without the download: consume(tranche) after each tranche's kernel; the tranche
    // size is a multiple of `granularity` (only the last may be smaller).
    TraceRunInfo run_on_device(const SystemBatchHost& batch, const TraceSettings& settings,
                               int granularity, const DeviceTrancheFn& consume);
    // FP32 prefilter (TraceEngine::prefilter_variants, trace_engine.hpp:188): the float trace
    // with margins on the device, the conservative decision on the host (bit-identical to the
    // reference's prefilter_cpu).
    PrefilterResult prefilter_variants(const SystemBatchHost& batch,
                                       const PrefilterSettings& settings = {});
    // Mode EVAL (TraceEngine::evaluate, trace_engine.hpp:193), bit-identical to eval_cpu.
    EvalResult evaluate(const SystemBatchHost& batch, const EvalSettings& settings = {});
    // Largest tranche for batches of this topology; 0 when not one variant fits.
    int max_variants(const BatchTopology& topology, TraceMode mode,
                     const TraceSettings& settings = {}) const;
    int device() const { return device_; }
    const std::string& device_name() const { return device_name_; }
    const EngineOptions& options() const { return options_; }
    std::size_t device_bytes() const;
    void* stream() const { return stream_; }
    void release() noexcept;
    void synchronize();

private:
    struct TranchePlan {
        int tranche = 0;
        std::size_t usable = 0;
    };
    std::size_t available_bytes() const;
    std::size_t usable_bytes(std::size_t available) const;
    TranchePlan plan_tranches(const SystemBatchHost& batch, TraceMode mode,
                              const ResidualLayout& layout, const TraceSettings& settings,
                              int granularity);
    DeviceTranche residual_tranche(const SystemBatchHost& batch, const ResidualLayout& layout,
                                   const TraceSettings& settings, int first, int count);

    int device_;
    std::string device_name_;
    EngineOptions options_;
    void* stream_ = nullptr;
    DeviceSystemBatch batch_;
    DeviceBuffer out_, opd_, status_, merit_, failed_, hard_, workspace_, extra_, extrema_;
};

// J [runs][P][R] (column p of run i at (i*P + p)*R) and r0 [runs][R] on the host.
struct JacobianResult {
    int runs = 0, P = 0;
    int64_t rows = 0;
    std::vector<double> J, r0;
};

class DeviceFdJacobian {
public:
    void compute(TraceEngine& engine, const VariableSet& variables, const SystemBatchHost& base,
                 const std::vector<double>& x0, const ResidualSettings& settings,
                 JacobianResult& out);

private:
    DeviceSystemBatch templates_;
    DeviceBuffer x0_, J_, r0_, workspace_;
};

class DeviceAdjointJacobian {
public:
    void compute(TraceEngine& engine, const VariableSet& variables, const SystemBatchHost& base,
                 const std::vector<double>& x0, const ResidualSettings& settings,
                 JacobianResult& out);

private:
    DeviceSystemBatch templates_;
    DeviceBuffer x0_, J_, r0_, status_, workspace_;
};

class DeviceNormalEquations {
public:
    // gram of [J r0] per run; exact: FMA chain in row order (normal_equations_host bit for
    // bit), else FP64 tensor cores
    void compute(TraceEngine& engine, const JacobianResult& jac, bool exact);
    // A [runs][P][P] (column-major per run, as the reference) and g [runs][P]
    void download(std::vector<double>& a, std::vector<double>& g) const;

private:
    int runs_ = 0, P_ = 0;
    std::vector<double> gram_;
    DeviceBuffer J_, r_, dgram_;
};

struct LmResult {
    std::vector<double> x, merit, damping;
    std::vector<double> history;  // [runs][history_width], the rounds joined, NaN padded
    int history_width = 0;
    std::vector<int32_t> status, iterations, accepted, jacobians, penalty_rounds;
    std::vector<int64_t> failed, hard_failed;
    std::vector<double> fail_weight;
};

struct LmGpuStats {
    int cycles = 0;
};

// Batched LM of the runs x0 [runs][P] on `base` (1 variant for all runs or one per run); the
// whole loop runs on the device. In soft-failure mode the outer penalty rounds follow
// (optimize_lm_rounds, src/optim/levenberg_marquardt.cpp:891).
LmResult optimize_lm_gpu(TraceEngine& engine, const VariableSet& variables,
                         const SystemBatchHost& base, const std::vector<double>& x0,
                         const LmOptions& options, const ResidualSettings& settings,
                         LmGpuStats* stats = nullptr);


// ---- scalar PSF and MTF (include/mikroptim/eval/psf.hpp, include/mikroptim/cuda/psf.hpp) ----
struct PsfSettings {  // psf.hpp:33
    double padding = 4.0;
    double numerical_aperture = 0.0;  // > 0: given; 0: from the field rays
};
struct PsfPupil {  // psf.hpp:57
    int field = 0, wavelength = 0, grid = 0, full_count = 0;
    double wavelength_nm = 0.0, na_x = 0.0, na_y = 0.0;
    bool flip_x = false, flip_y = false;
    std::vector<double> opd;  // [N * N], NaN: no transmission
    double wavelength_mm() const { return wavelength_nm * 1e-6; }
};
struct PsfResult {  // psf.hpp:95
    int field = 0, wavelength = 0, grid = 0, fft_size = 0;
    double wavelength_nm = 0.0, na_x = 0.0, na_y = 0.0, dx = 0.0, dy = 0.0, airy_radius = 0.0;
    std::vector<double> psf, mtf_sagittal, mtf_tangential;
    int64_t transmitted = 0;
    double energy = 0.0, strehl_fft = 0.0, strehl_origin = 0.0, strehl = 0.0;
    double reference_x = 0.0, reference_y = 0.0, peak = 0.0, peak_x = 0.0, peak_y = 0.0;
    double psf_at(int i, int j) const {
        return psf[static_cast<size_t>(j) * static_cast<size_t>(fft_size) +
                   static_cast<size_t>(i)];
    }
};
// psf_fft_size (src/eval/psf.cpp:168); std::invalid_argument for invalid sizes
int psf_fft_size(int grid, double padding);
// eval_opd_map with piston removal and make_psf_pupil(s) (src/eval/eval.cpp:512,
// src/eval/psf.cpp:196)
std::vector<double> eval_opd_map(const EvalResult& result, int v, int f, int l);
PsfPupil make_psf_pupil(const SystemBatchHost& batch, const EvalResult& result, int v, int f,
                        int l, const PsfSettings& settings = {});
std::vector<PsfPupil> make_psf_pupils(const SystemBatchHost& batch, const EvalResult& result,
                                      int v, const PsfSettings& settings = {});

struct PsfRunInfo {  // cuda/psf.hpp:22; work_bytes: the FFT workspace
    int pupils = 0, tranche = 0, tranches = 0;
    size_t work_bytes = 0, device_bytes = 0, budget_bytes = 0;
};
// PsfEngine (include/mikroptim/cuda/psf.hpp:37): PSF, MTF and figures of pupils of one grid
// edge in tranches sized against the device memory; buffers kept across calls; the device
// work is mkb_psf_device, the figures mkb_psf_finish_host.
class PsfEngine {
public:
    explicit PsfEngine(int device = 0, const EngineOptions& options = {});
    PsfEngine(const PsfEngine&) = delete;
    PsfEngine& operator=(const PsfEngine&) = delete;
    std::vector<PsfResult> compute(std::span<const PsfPupil> pupils, int fft_size);
    std::vector<PsfResult> compute(const SystemBatchHost& batch, const EvalResult& result, int v,
                                   const PsfSettings& settings = {});
    const PsfRunInfo& last_run() const { return info_; }
    int device() const { return device_; }
    size_t device_bytes() const;
    void release();

private:
    int device_ = 0;
    EngineOptions options_;
    PsfRunInfo info_;
    DeviceBuffer maps_, params_, psf_, mtf_, work_;
};
}  // namespace cuda
}  // namespace mkb
