"""ctypes binding of the C ABI declared in include/mikroptim_b200.h.

The library ``libmikroptim_b200.so`` is built in-tree (``python -m mikroptim_b200.build``)
and loaded from this package directory. There is no fallback: if the library is missing,
``lib()`` raises, so nothing silently runs on the CPU.
"""

from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmikroptim_b200.so")

MKB_OK = 0
MKB_ERR_ARGUMENT = -1
MKB_ERR_CUDA = -2
MKB_ERR_WORKSPACE = -3
MKB_ERR_TIMEOUT = -4
MKB_ERR_UNSUPPORTED = -5
MKB_WAIT_POLLS_DEFAULT = 1 << 24

P_double = C.POINTER(C.c_double)
P_int64 = C.POINTER(C.c_int64)
P_int32 = C.POINTER(C.c_int32)
P_uint8 = C.POINTER(C.c_uint8)


class BatchView(C.Structure):
    """mkb_batch_view (SystemBatchView<double>, system_batch_view.hpp:108)."""

    _fields_ = [
        ("variants", C.c_int32), ("surfaces", C.c_int32), ("wavelengths", C.c_int32),
        ("fields", C.c_int32), ("ghost_plates", C.c_int32), ("ghost_terms", C.c_int32),
        ("reference_wavelength_nm", C.c_double),
        ("type", P_uint8),
        ("wavelength_weight", P_double),
        ("field_weight", P_double),
        ("curvature", P_double),
        ("thickness", P_double),
        ("index", P_double),
        ("pupil_radius", P_double),
        ("field_angle", P_double),
        ("field_target", P_double),
        ("decenter_tilt", P_double),
        ("ghost_coeff", P_double),
        ("ghost_norm_radius", P_double),
        ("ghost_index", P_double),
        ("buchdahl_coeff", P_double),
        ("wavelength_nm", P_double),
    ]


class DeviceBatch(C.Structure):
    """mkb_device_batch: packed per-variant records in device memory."""

    _fields_ = [
        ("variants", C.c_int32), ("surfaces", C.c_int32), ("wavelengths", C.c_int32),
        ("fields", C.c_int32), ("record_stride", C.c_int32), ("non_coaxial", C.c_int32),
        ("records", C.c_void_p),
        ("type", P_uint8),
        ("variant_surfaces", C.c_void_p),
        ("ghost_plates", C.c_int32), ("ghost_terms", C.c_int32),
        ("glass", C.c_int32),
        ("wavelength_nm", P_double),
    ]


class PsfPupilParams(C.Structure):
    """mkb_psf_pupil_params (PsfPupilParams, include/mikroptim/eval/psf_ops.hpp:48)."""

    _fields_ = [("lambda_mm", C.c_double), ("scale", C.c_double),
                ("sign_x", C.c_int32), ("sign_y", C.c_int32)]


class PsfMetrics(C.Structure):
    """mkb_psf_metrics: the figures of PsfResult (include/mikroptim/eval/psf.hpp:95)."""

    _fields_ = [("transmitted", C.c_int64)] + [
        (k, C.c_double) for k in ("energy", "strehl_fft", "strehl_origin", "strehl",
                                  "reference_x", "reference_y", "peak", "peak_x", "peak_y",
                                  "dx", "dy", "airy_radius")]


class ResidualPlan(C.Structure):
    """mkb_residual_plan (ResidualSettings + ResidualLayout, batch_residuals.hpp:24,62)."""

    _fields_ = [
        ("rings", C.c_int32), ("spokes", C.c_int32),
        ("failure", C.c_int32), ("precision", C.c_int32),
        ("fail_weight", C.c_double),
        ("reference_wavelength_nm", C.c_double),
        ("fields", C.c_int32), ("wavelengths", C.c_int32),
        ("pupil_mode", P_uint8),
        ("field_weight", P_double),
        ("wavelength_weight", P_double),
        ("quad_u", P_double),
        ("quad_w", P_double),
        ("transverse_weight", C.c_double),
    ]


class Variables(C.Structure):
    """mkb_variables (VariableSet: curvature, thickness, working distance, ghost coefficient)."""

    _fields_ = [
        ("count", C.c_int32),
        ("type", P_int32),
        ("surface", P_int32),
        ("lower", P_double),
        ("upper", P_double),
        ("typical", P_double),
        ("ghost_plate", P_int32),
        ("ghost_order", P_int32),
        ("glass_component", P_int32),
    ]


class ParaxialConstraint(C.Structure):
    """mkb_paraxial_constraint (ParaxialConstraint, optim/paraxial_residuals.hpp:67)."""

    _fields_ = [("type", C.c_int32), ("mode", C.c_int32), ("weight", C.c_double),
                ("target", C.c_double), ("reference_surface", C.c_int32),
                ("reserved", C.c_int32), ("offset", C.c_double), ("shift", C.c_double)]


class LmOptions(C.Structure):
    """mkb_lm_options (LmOptions, levenberg_marquardt.hpp:85)."""

    _fields_ = [
        ("max_iterations", C.c_int32), ("reject_new_failures", C.c_int32),
        ("ftol", C.c_double), ("xtol", C.c_double), ("gtol", C.c_double),
        ("initial_damping", C.c_double), ("max_damping", C.c_double),
        ("diag_floor", C.c_double),
        ("jacobian", C.c_int32), ("gram_exact", C.c_int32),
        ("per_run_variables", C.c_int32),
        ("paraxial_count", C.c_int32), ("paraxial", C.POINTER(ParaxialConstraint)),
        ("paraxial_column", C.c_int32), ("paraxial_derivative", C.c_int32),
    ]


MKB_PARAXIAL_FD = 0
MKB_PARAXIAL_ADJOINT = 1


class TraceOptions(C.Structure):
    """mkb_trace_options (TraceSettings::pack_rays / ::extra_merit, trace_engine.hpp:58)."""

    _fields_ = [("pack_rays", C.c_int32), ("variants_per_cta", C.c_int32),
                ("extra_merit", C.c_void_p), ("extrema", C.c_void_p)]


class PrefilterOptions(C.Structure):
    """mkb_prefilter_options (PrefilterCriteria + PrefilterMargins, batch_prefilter.hpp:35,52)."""

    _fields_ = [("max_failed_fraction", C.c_double), ("max_merit", C.c_double),
                ("max_merit_factor", C.c_double), ("boundary", C.c_double),
                ("opl_error_factor", C.c_double), ("merit_relative", C.c_double)]


MKB_PREFILTER_KEEP = 0
MKB_PREFILTER_FAILED_RAYS = 1
MKB_PREFILTER_MERIT_ABSOLUTE = 2
MKB_PREFILTER_MERIT_RELATIVE = 4

_lock = threading.Lock()
_lib = None


def _declare(lib: C.CDLL) -> None:
    c = C
    lib.mkb_last_error.restype = c.c_char_p
    lib.mkb_version.restype = c.c_char_p
    lib.mkb_launch_count.restype = c.c_int64
    lib.mkb_record_stride.restype = c.c_int32
    lib.mkb_record_stride.argtypes = [c.c_int32, c.c_int32, c.c_int32]
    lib.mkb_record_stride_ext.restype = c.c_int32
    lib.mkb_record_stride_ext.argtypes = [c.c_int32] * 7
    lib.mkb_pack_batch_host.restype = c.c_int
    lib.mkb_pack_batch_host.argtypes = [C.POINTER(BatchView), P_double]
    lib.mkb_rays_per_variant.restype = c.c_int64
    lib.mkb_rays_per_variant.argtypes = [C.POINTER(ResidualPlan)]
    lib.mkb_trace_rows.restype = c.c_int64
    lib.mkb_trace_rows.argtypes = [C.POINTER(ResidualPlan)]
    lib.mkb_residuals_device.restype = c.c_int
    lib.mkb_residuals_device.argtypes = [C.POINTER(DeviceBatch), C.POINTER(ResidualPlan),
                                         c.c_void_p, c.c_int64, c.c_void_p, c.c_void_p,
                                         c.c_void_p]
    lib.mkb_merit_workspace_bytes.restype = c.c_size_t
    lib.mkb_merit_workspace_bytes.argtypes = [c.c_int32, C.POINTER(ResidualPlan)]
    lib.mkb_merit_device.restype = c.c_int
    lib.mkb_merit_device.argtypes = [C.POINTER(DeviceBatch), C.POINTER(ResidualPlan),
                                     c.c_void_p, c.c_void_p, c.c_void_p, c.c_void_p,
                                     c.c_size_t, c.c_void_p]
    PT = C.POINTER(TraceOptions)
    lib.mkb_residuals_ex_device.restype = c.c_int
    lib.mkb_residuals_ex_device.argtypes = [C.POINTER(DeviceBatch), C.POINTER(ResidualPlan), PT,
                                            c.c_void_p, c.c_int64, c.c_void_p, c.c_void_p,
                                            c.c_void_p]
    lib.mkb_merit_ex_device.restype = c.c_int
    lib.mkb_merit_ex_device.argtypes = [C.POINTER(DeviceBatch), C.POINTER(ResidualPlan), PT,
                                        c.c_void_p, c.c_void_p, c.c_void_p, c.c_void_p,
                                        c.c_size_t, c.c_void_p]
    lib.mkb_usable_bytes.restype = c.c_int
    lib.mkb_usable_bytes.argtypes = [c.c_size_t, c.c_size_t, c.c_double,
                                     C.POINTER(c.c_size_t)]
    lib.mkb_trace_run_bytes.restype = c.c_int
    lib.mkb_trace_run_bytes.argtypes = [C.POINTER(DeviceBatch), C.POINTER(ResidualPlan),
                                        c.c_int32, c.c_int64, c.c_int32, c.c_int32,
                                        C.POINTER(c.c_size_t), C.POINTER(c.c_size_t)]
    lib.mkb_trace_tranche_variants.restype = c.c_int64
    lib.mkb_trace_tranche_variants.argtypes = [c.c_size_t, C.POINTER(DeviceBatch),
                                               C.POINTER(ResidualPlan), PT, c.c_int32,
                                               c.c_int64, c.c_int32, c.c_int32, c.c_int32]
    lib.mkb_merit_noalloc_device.restype = c.c_int
    lib.mkb_merit_noalloc_device.argtypes = [C.POINTER(DeviceBatch), C.POINTER(ResidualPlan),
                                             c.c_void_p, c.c_void_p, c.c_void_p, c.c_void_p]
    lib.mkb_device_status.restype = c.c_int
    lib.mkb_eval_grid_host.restype = c.c_int
    lib.mkb_eval_grid_host.argtypes = [c.c_int32, c.c_int32, c.c_void_p, C.POINTER(c.c_int64)]
    lib.mkb_eval_reference_host.restype = c.c_int
    lib.mkb_eval_reference_host.argtypes = [C.POINTER(BatchView), c.c_int32, c.c_int32,
                                            c.c_void_p, c.c_void_p]
    lib.mkb_eval_workspace_bytes.restype = c.c_size_t
    lib.mkb_eval_workspace_bytes.argtypes = [C.POINTER(DeviceBatch)]
    lib.mkb_eval_device.restype = c.c_int
    lib.mkb_eval_device.argtypes = [C.POINTER(DeviceBatch), c.c_int32, c.c_double, c.c_int32,
                                    c.c_void_p, c.c_int64, c.c_void_p] + [c.c_void_p] * 6 + \
        [c.c_void_p, c.c_size_t, c.c_void_p]
    lib.mkb_psf_fft_size_host.restype = c.c_int
    lib.mkb_psf_fft_size_host.argtypes = [c.c_int32, c.c_double, P_int32]
    lib.mkb_psf_workspace_bytes.restype = c.c_size_t
    lib.mkb_psf_workspace_bytes.argtypes = [c.c_int32, c.c_int32, c.c_int32]
    lib.mkb_psf_device.restype = c.c_int
    lib.mkb_psf_device.argtypes = [c.c_int32, c.c_int32, c.c_int32] + [c.c_void_p] * 5 + \
        [c.c_size_t, c.c_void_p]
    lib.mkb_psf_maps_device.restype = c.c_int
    lib.mkb_psf_maps_device.argtypes = [c.c_int32, c.c_int32, c.c_int64, c.c_int32] + \
        [c.c_void_p] * 6
    lib.mkb_psf_aperture_host.restype = c.c_int
    lib.mkb_psf_aperture_host.argtypes = [c.c_void_p, c.c_void_p, c.c_double, c.c_double,
                                          c.c_double, P_double, P_double, P_int32, P_int32]
    lib.mkb_psf_finish_host.restype = c.c_int
    lib.mkb_psf_finish_host.argtypes = [c.c_int32, c.c_int32, c.c_void_p, c.c_int32, c.c_double,
                                        c.c_double, c.c_double, c.c_int32, c.c_int32,
                                        c.c_void_p, C.POINTER(PsfMetrics)]
    lib.mkb_paraxial_rows_device.restype = c.c_int
    lib.mkb_paraxial_rows_device.argtypes = [C.POINTER(DeviceBatch), C.POINTER(ResidualPlan),
                                             C.POINTER(Variables), C.POINTER(LmOptions),
                                             c.c_void_p, c.c_int32, c.c_void_p, c.c_void_p,
                                             c.c_void_p]
    PF = C.POINTER(PrefilterOptions)
    lib.mkb_prefilter_workspace_bytes.restype = c.c_size_t
    lib.mkb_prefilter_workspace_bytes.argtypes = [c.c_int32, C.POINTER(ResidualPlan)]
    lib.mkb_prefilter_field_trig_host.restype = c.c_int
    lib.mkb_prefilter_field_trig_host.argtypes = [C.POINTER(BatchView), c.c_void_p]
    lib.mkb_prefilter_device.restype = c.c_int
    lib.mkb_prefilter_device.argtypes = [C.POINTER(DeviceBatch), C.POINTER(ResidualPlan),
                                         c.c_void_p, c.c_double] + [c.c_void_p] * 6 + \
        [c.c_size_t, c.c_void_p]
    lib.mkb_prefilter_default_options.restype = None
    lib.mkb_prefilter_default_options.argtypes = [PF]
    lib.mkb_prefilter_decide_host.restype = c.c_int
    lib.mkb_prefilter_decide_host.argtypes = [C.POINTER(ResidualPlan), PF, c.c_int32] + \
        [c.c_void_p] * 12
    lib.mkb_prefilter_decide_exact_host.restype = c.c_int
    lib.mkb_prefilter_decide_exact_host.argtypes = [PF, c.c_int32, c.c_int64] + [c.c_void_p] * 4
    lib.mkb_set_wait_limit.restype = c.c_int
    lib.mkb_set_wait_limit.argtypes = [c.c_uint32]
    PV = C.POINTER(Variables)
    PB = C.POINTER(DeviceBatch)
    PP = C.POINTER(ResidualPlan)
    lib.mkb_fd_jacobian_workspace_bytes.restype = c.c_size_t
    lib.mkb_fd_jacobian_workspace_bytes.argtypes = [PB, PP, c.c_int32, c.c_int32, c.c_int32]
    lib.mkb_fd_jacobian_device.restype = c.c_int
    lib.mkb_fd_jacobian_device.argtypes = [PB, PP, PV, c.c_void_p, c.c_int32, c.c_void_p,
                                           c.c_void_p, c.c_void_p, c.c_void_p, c.c_size_t,
                                           c.c_void_p]
    lib.mkb_adjoint_jacobian_workspace_bytes.restype = c.c_size_t
    lib.mkb_adjoint_jacobian_workspace_bytes.argtypes = [PB, c.c_int32]
    lib.mkb_adjoint_jacobian_device.restype = c.c_int
    lib.mkb_adjoint_jacobian_device.argtypes = [PB, PP, PV, c.c_void_p, c.c_int32, c.c_void_p,
                                                c.c_void_p, c.c_void_p, c.c_void_p, c.c_size_t,
                                                c.c_void_p]
    lib.mkb_adjoint_normal_equations_device.restype = c.c_int
    lib.mkb_adjoint_normal_equations_device.argtypes = [PB, PP, PV, c.c_void_p, c.c_int32,
                                                        c.c_void_p, c.c_void_p, c.c_size_t,
                                                        c.c_void_p]
    lib.mkb_adjoint_normal_equations_runs_workspace_bytes.restype = c.c_size_t
    lib.mkb_adjoint_normal_equations_runs_workspace_bytes.argtypes = [PB, PV, c.c_int32]
    lib.mkb_adjoint_normal_equations_runs_device.restype = c.c_int
    lib.mkb_adjoint_normal_equations_runs_device.argtypes = [PB, PP, PV, c.c_void_p, c.c_int32,
                                                             c.c_void_p, c.c_void_p, c.c_size_t,
                                                             c.c_void_p]
    PO = C.POINTER(LmOptions)
    lib.mkb_lm_workspace_bytes.restype = c.c_size_t
    lib.mkb_lm_workspace_bytes.argtypes = [PB, PP, PV, PO, c.c_int32]
    lib.mkb_lm_start_device.restype = c.c_int
    lib.mkb_lm_start_device.argtypes = [PB, PP, PV, PO, c.c_void_p, c.c_int32, c.c_void_p,
                                        c.c_size_t, c.c_void_p]
    lib.mkb_lm_cycle_device.restype = c.c_int
    lib.mkb_lm_cycle_device.argtypes = [PB, PP, PV, PO, c.c_int32, c.c_void_p, c.c_size_t,
                                        c.c_void_p]
    lib.mkb_lm_start_ex_device.restype = c.c_int
    lib.mkb_lm_start_ex_device.argtypes = [PB, PP, PV, PO, c.c_void_p, c.c_void_p, c.c_void_p,
                                           c.c_int32, c.c_void_p, c.c_size_t, c.c_void_p]
    lib.mkb_lm_cycle_trial_device.restype = c.c_int
    lib.mkb_lm_cycle_trial_device.argtypes = [PB, PP, PV, PO, c.c_int32, c.c_void_p,
                                              c.c_size_t, c.c_void_p, c.c_void_p, c.c_void_p]
    lib.mkb_lm_cycle_decide_device.restype = c.c_int
    lib.mkb_lm_cycle_decide_device.argtypes = [PB, PP, PV, PO, c.c_int32, c.c_void_p,
                                               c.c_size_t, c.c_void_p, c.c_void_p]
    for name in ("mkb_lm_cycle_jacobian_device", "mkb_lm_cycle_step_device"):
        getattr(lib, name).restype = c.c_int
        getattr(lib, name).argtypes = [PB, PP, PV, PO, c.c_int32, c.c_void_p, c.c_size_t,
                                       c.c_void_p]
    lib.mkb_lm_extra_rows_device.restype = c.c_int
    lib.mkb_lm_extra_rows_device.argtypes = [PB, PP, PV, PO, c.c_int32, c.c_void_p, c.c_size_t,
                                             c.c_void_p, c.c_void_p, c.c_int32, c.c_void_p]
    lib.mkb_lm_cycle_accept_device.restype = c.c_int
    lib.mkb_lm_cycle_accept_device.argtypes = [PB, PP, PV, PO, c.c_int32, c.c_void_p,
                                               c.c_size_t, c.c_void_p, c.c_void_p]
    lib.mkb_lm_points_device.restype = c.c_int
    lib.mkb_lm_points_device.argtypes = [PB, PP, PV, PO, c.c_int32, c.c_void_p, c.c_void_p,
                                         c.c_void_p, c.c_void_p, c.c_void_p, c.c_void_p]
    lib.mkb_fd_pattern_host.restype = c.c_int
    lib.mkb_fd_pattern_host.argtypes = [PV, P_double, c.c_int32, P_double, P_double, P_double,
                                        P_double, C.POINTER(c.c_int32)]
    lib.mkb_fd_derivative_host.restype = c.c_int
    lib.mkb_fd_derivative_host.argtypes = [c.c_int32, c.c_double, c.c_double, c.c_int32,
                                           P_double, P_double, P_double, P_double]
    lib.mkb_lm_results_device.restype = c.c_int
    lib.mkb_lm_results_device.argtypes = [PB, PP, PV, PO, c.c_int32, c.c_void_p] + \
        [c.c_void_p] * 11 + [c.c_void_p]
    lib.mkb_apply_variables_device.restype = c.c_int
    lib.mkb_apply_variables_device.argtypes = [PB, PV, c.c_void_p, c.c_int32, c.c_void_p,
                                               c.c_void_p]
    lib.mkb_normal_equations_device.restype = c.c_int
    lib.mkb_normal_equations_device.argtypes = [c.c_void_p, c.c_void_p, c.c_int32, c.c_int32,
                                                c.c_int64, c.c_void_p, c.c_int32, c.c_void_p]


def lib() -> C.CDLL:
    """The loaded CUDA library; raises if it has not been built."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"mikroptim_b200: CUDA library not built ({LIB_PATH}); run "
                    "`python -m mikroptim_b200.build` (there is no CPU fallback)")
            handle = C.CDLL(LIB_PATH, mode=C.RTLD_GLOBAL)
            _declare(handle)
            _lib = handle
        return _lib


def check(status: int, what: str) -> None:
    """Raise the reference-style exception for a non-zero mkb_status."""
    if status == MKB_OK:
        return
    msg = lib().mkb_last_error().decode(errors="replace")
    if status == MKB_ERR_ARGUMENT:
        raise ValueError(f"{what}: {msg}")
    if status == MKB_ERR_UNSUPPORTED:
        raise NotImplementedError(f"{what}: {msg}")
    raise RuntimeError(f"{what} (status {status}): {msg}")


def ptr(array, ctype=C.c_double):
    """ctypes pointer to a contiguous numpy array (None for None)."""
    if array is None:
        return None
    return array.ctypes.data_as(C.POINTER(ctype))
