"""Host-side batch model mirroring the reference's SystemBatch API.

Names and meaning follow the reference:
  BatchTopology      include/mikroptim/batch/system_batch.hpp:229 (non_coaxial: :45)
  SystemBatchHost    include/mikroptim/batch/system_batch.hpp:268 (FP64 SoA, variant-major)
  ResidualSettings   include/mikroptim/batch/batch_residuals.hpp:24
  ResidualLayout     include/mikroptim/batch/batch_residuals.hpp:62 (src/batch/batch_residuals.cpp:25)
  VariableSet        include/mikroptim/optim/variable_set.hpp:63 (curvature, thickness and
                     working-distance variables; Variable.batch_surface is the table surface)

Errors are raised before any device work: ValueError where the reference throws
std::invalid_argument, IndexError for std::out_of_range.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
import math

import numpy as np

from . import _capi
from .quadrature import (MAX_RINGS, PUPIL_AXIS, PUPIL_FULL, PUPIL_HALF, gauss_legendre_unit,
                         sample_count)

SURFACE_STOP, SURFACE_PLANE, SURFACE_SPHERE, SURFACE_GHOST_PLATE = 0, 1, 2, 3
# an aperture stop inside the system (no reference counterpart): a plane whose curvature slot
# holds the stop's semi-aperture; surface 0 is then the entrance pupil, placed by paraxial ray
# aiming (MKB_SURFACE_APERTURE_STOP, include/mikroptim_b200.h)
SURFACE_APERTURE_STOP = 4
FAILURE_SOFT, FAILURE_HARD = 0, 1
PRECISION_FP64, PRECISION_MIXED, PRECISION_FP64_FMA, PRECISION_DF64 = 0, 1, 2, 3
# directions and refraction in FP32, positions, intersection and optical path in FP64
# (MKB_PRECISION_FP32_BULK; coaxial batches without ghost plates)
PRECISION_FP32_BULK = 4
VAR_CURVATURE, VAR_THICKNESS, VAR_WORKING_DISTANCE, VAR_GHOST_COEFFICIENT, VAR_GLASS = 0, 1, 2, 3, 4
BUCHDAHL_LAMBDA0_UM, BUCHDAHL_ALPHA = 0.546074, 2.5  # glass/dispersion.hpp:13,15
MAX_GHOST_PLATES, MAX_GHOST_TERMS = 16, 32

MAX_SURFACES = 64
MAX_FIELDS = 16
MAX_WAVELENGTHS = 16
MAX_TUPLES = 128
MAX_VARIABLES = 64

# TraceStatus values (include/mikroptim/trace/surface_ops.hpp:24)
STATUS_OK, STATUS_MISSED, STATUS_TIR, STATUS_BACKWARD = 0, 1, 2, 3
STATUS_UNSUPPORTED, STATUS_SOFT_MISSED, STATUS_SOFT_TIR = 4, 5, 6
DEFAULT_FAIL_WEIGHT = 1e6  # kDefaultFailWeight, merit/ray_residual.hpp:175


def in_piston(status: np.ndarray) -> np.ndarray:
    """Ok or soft failure (surface_ops.hpp:66)."""
    return (status == STATUS_OK) | (status == STATUS_SOFT_MISSED) | (status == STATUS_SOFT_TIR)


@dataclass
class BatchTopology:
    """Everything all variants of one launch share (ADR-0004 of the reference)."""

    surfaces: int
    wavelengths: int
    fields: int
    type: list[int]
    pupil_mode: list[int]
    # per-surface decenter and tilt (decenter_tilt [V][S][4]); every field then uses the
    # Full pupil (check_pupil_modes, src/batch/system_batch.cpp:158)
    non_coaxial: bool = False
    # ghost plates: the surfaces of kind GhostPlate, numbered in table order, and the profile
    # terms K every plate carries (BatchTopology::ghost_plates / ghost_terms)
    ghost_terms: int = 0

    @property
    def ghost_plates(self) -> int:
        return sum(1 for t in self.type[1:] if t == SURFACE_GHOST_PLATE)

    @property
    def stop_surface(self) -> int:
        """The interior aperture stop's table surface, or 0 (the stop is surface 0)."""
        return next((s for s, t in enumerate(self.type) if s > 0 and t == SURFACE_APERTURE_STOP),
                    0)

    def ghost_surface(self, g: int) -> int:
        """Table surface of plate g."""
        return [s for s, t in enumerate(self.type) if s > 0 and t == SURFACE_GHOST_PLATE][g]

    def validate(self) -> None:
        if not 2 <= self.surfaces <= MAX_SURFACES:
            raise ValueError(f"BatchTopology: surfaces must be in [2, {MAX_SURFACES}]")
        if not 1 <= self.wavelengths <= MAX_WAVELENGTHS:
            raise ValueError(f"BatchTopology: wavelengths must be in [1, {MAX_WAVELENGTHS}]")
        if not 1 <= self.fields <= MAX_FIELDS:
            raise ValueError(f"BatchTopology: fields must be in [1, {MAX_FIELDS}]")
        if self.fields * self.wavelengths > MAX_TUPLES:
            raise ValueError(f"BatchTopology: fields * wavelengths must be <= {MAX_TUPLES}")
        if len(self.type) != self.surfaces:
            raise ValueError("BatchTopology: type needs one entry per surface")
        if self.type[0] != SURFACE_STOP:
            raise ValueError("BatchTopology: surface 0 must be the stop")
        for s, t in enumerate(self.type[1:], start=1):
            if t not in (SURFACE_PLANE, SURFACE_SPHERE, SURFACE_GHOST_PLATE,
                         SURFACE_APERTURE_STOP):
                raise ValueError(f"BatchTopology: surface {s} has unknown kind {t}")
        stops = [s for s, t in enumerate(self.type) if s > 0 and t == SURFACE_APERTURE_STOP]
        if len(stops) > 1 or (stops and not 1 <= stops[0] <= self.surfaces - 2):
            raise ValueError("BatchTopology: at most one interior aperture stop, at "
                             "1 <= s <= S - 2")
        if stops and (self.non_coaxial or self.ghost_plates > 0):
            raise NotImplementedError("BatchTopology: an interior aperture stop is traced in "
                                      "coaxial batches without ghost plates")
        if self.ghost_plates > MAX_GHOST_PLATES:
            raise NotImplementedError(f"BatchTopology: at most {MAX_GHOST_PLATES} ghost plates "
                                      "in this build")
        if not 0 <= self.ghost_terms <= MAX_GHOST_TERMS:
            raise ValueError(f"BatchTopology: ghost_terms must be in [0, {MAX_GHOST_TERMS}]")
        if self.ghost_plates > 0 and self.ghost_terms < 1:
            raise ValueError("BatchTopology: ghost plates need ghost_terms >= 1")
        if len(self.pupil_mode) != self.fields:
            raise ValueError("BatchTopology: pupil_mode needs one entry per field")
        for m in self.pupil_mode:
            if m not in (PUPIL_HALF, PUPIL_FULL, PUPIL_AXIS):
                raise ValueError("BatchTopology: unknown pupil mode")
            if self.non_coaxial and m != PUPIL_FULL:
                raise ValueError("BatchTopology: a non-coaxial batch needs the Full pupil in "
                                 "every field")


class SystemBatchHost:
    """V variants of one topology as FP64 structure of arrays (variant outermost)."""

    def __init__(self, topology: BatchTopology, variants: int):
        topology.validate()
        if variants < 0:
            raise ValueError("SystemBatchHost: variants must be >= 0")
        self.topology = topology
        S, L, F = topology.surfaces, topology.wavelengths, topology.fields
        self.reference_wavelength_nm = 0.0
        self.type = np.asarray(topology.type, dtype=np.uint8)
        self.wavelength_nm = np.zeros(L)
        self.wavelength_weight = np.zeros(L)
        self.field_weight = np.zeros(F)
        self.curvature = np.zeros((variants, S))
        self.thickness = np.zeros((variants, S))
        self.index = np.zeros((variants, S, L))
        self.pupil_radius = np.zeros(variants)
        self.field_angle = np.zeros((variants, F))
        self.field_target = np.zeros((variants, F))
        # non-coaxial batches: (dx, dy, alpha, beta) per surface, decenter in mm and tilts in
        # radians (SystemBatchHost::decenter_tilt, system_batch.hpp:156); None when coaxial
        self.decenter_tilt: np.ndarray | None = (np.zeros((variants, S, 4))
                                                 if topology.non_coaxial else None)
        # ghost plates (system_batch.hpp:102-131): profile coefficients a_1..a_K [V][G][K]
        # (mm), normalisation radius r_g [G] (mm, shared), plate glass index [V][G][L]
        G, K = topology.ghost_plates, topology.ghost_terms
        self.ghost_coeff = np.zeros((variants, G, K))
        self.ghost_norm_radius = np.ones(G)
        self.ghost_index = np.ones((variants, G, L))
        # glass variables: Buchdahl coefficients (n0, nu1, nu2, nu3) of the medium after every
        # surface [V][S][4] (SystemBatchHost::buchdahl_coeff); None when no variable is a glass
        self.buchdahl_coeff: np.ndarray | None = None
        # uneven batches: table surfaces each variant uses (2 .. S); None = all use S
        self.variant_surfaces: np.ndarray | None = None

    # ---- shape --------------------------------------------------------------------------
    @property
    def variants(self) -> int:
        return self.curvature.shape[0]

    @property
    def surfaces(self) -> int:
        return self.topology.surfaces

    @property
    def wavelengths(self) -> int:
        return self.topology.wavelengths

    @property
    def fields(self) -> int:
        return self.topology.fields

    def subset(self, first: int, count: int) -> "SystemBatchHost":
        """Variants [first, first + count) as a new batch with its own arrays (assign_variants)."""
        if first < 0 or count < 0 or first + count > self.variants:
            raise IndexError("SystemBatchHost.subset: range out of bounds")
        out = SystemBatchHost(self.topology, 0)
        out.reference_wavelength_nm = self.reference_wavelength_nm
        out.wavelength_nm = self.wavelength_nm.copy()
        out.wavelength_weight = self.wavelength_weight.copy()
        out.field_weight = self.field_weight.copy()
        sl = slice(first, first + count)
        for name in ("curvature", "thickness", "index", "pupil_radius", "field_angle",
                     "field_target"):
            setattr(out, name, np.array(getattr(self, name)[sl], copy=True))
        if self.decenter_tilt is not None:
            out.decenter_tilt = np.array(self.decenter_tilt[sl])
        if self.buchdahl_coeff is not None:
            out.buchdahl_coeff = np.array(self.buchdahl_coeff[sl])
        for name in ("ghost_coeff", "ghost_index"):
            setattr(out, name, np.array(getattr(self, name)[sl], copy=True))
        out.ghost_norm_radius = self.ghost_norm_radius.copy()
        if self.variant_surfaces is not None:
            out.variant_surfaces = np.array(self.variant_surfaces[sl])
        return out

    def take(self, variants) -> "SystemBatchHost":
        """Batch made of the listed variants (in that order)."""
        idx = np.asarray(variants, dtype=np.int64)
        out = self.subset(0, 0)
        for name in ("curvature", "thickness", "index", "pupil_radius", "field_angle",
                     "field_target"):
            setattr(out, name, np.ascontiguousarray(getattr(self, name)[idx]))
        if self.decenter_tilt is not None:
            out.decenter_tilt = np.ascontiguousarray(self.decenter_tilt[idx])
        if self.buchdahl_coeff is not None:
            out.buchdahl_coeff = np.ascontiguousarray(self.buchdahl_coeff[idx])
        for name in ("ghost_coeff", "ghost_index"):
            setattr(out, name, np.ascontiguousarray(getattr(self, name)[idx]))
        out.ghost_norm_radius = self.ghost_norm_radius.copy()
        if self.variant_surfaces is not None:
            out.variant_surfaces = np.ascontiguousarray(self.variant_surfaces[idx])
        return out

    def set_decenter_tilt(self, v: int, s: int, dx: float, dy: float, alpha: float,
                          beta: float) -> None:
        """SystemBatchHost::set_decenter_tilt (src/batch/system_batch.cpp:510)."""
        if self.decenter_tilt is None:
            raise ValueError("SystemBatchHost: decenter and tilt need a non-coaxial batch "
                             "(make_non_coaxial)")
        if not (0 <= v < self.variants and 0 <= s < self.surfaces):
            raise IndexError("SystemBatchHost.set_decenter_tilt: index out of range")
        self.decenter_tilt[v, s] = (dx, dy, alpha, beta)

    def validate_values(self) -> None:
        """validate_values (src/batch/system_batch.cpp:558) for the fields traced here."""
        names = ["curvature", "thickness", "index", "pupil_radius", "field_angle",
                 "field_target", "wavelength_weight", "field_weight"]
        if self.decenter_tilt is not None:
            names.append("decenter_tilt")
        names += ["ghost_coeff", "ghost_norm_radius", "ghost_index"]
        G, K, L = self.topology.ghost_plates, self.topology.ghost_terms, self.wavelengths
        if (self.ghost_coeff.shape != (self.variants, G, K) or
                self.ghost_norm_radius.shape != (G,) or
                self.ghost_index.shape != (self.variants, G, L)):
            raise ValueError("SystemBatchHost: ghost arrays do not match the topology")
        for name in names:
            a = getattr(self, name)
            if not np.all(np.isfinite(a)):
                bad = np.argwhere(~np.isfinite(a))[0]
                raise ValueError(f"SystemBatchHost: {name}{list(bad)} is not finite")
        if self.decenter_tilt is not None:
            if self.decenter_tilt.shape != (self.variants, self.surfaces, 4):
                raise ValueError("SystemBatchHost: decenter_tilt must be [V][S][4]")
            if not np.all(np.abs(self.decenter_tilt[:, :, 2:]) < math.pi / 2):
                raise ValueError("SystemBatchHost: tilt angles must be in (-pi/2, pi/2)")
        if np.any(self.ghost_norm_radius <= 0) or np.any(self.ghost_index <= 0):
            raise ValueError("SystemBatchHost: ghost plate radius and index must be > 0")
        if np.any(self.pupil_radius <= 0):
            raise ValueError("SystemBatchHost: pupil radius must be > 0")
        if np.any(self.index <= 0):
            raise ValueError("SystemBatchHost: refractive indices must be > 0")
        if np.any(self.wavelength_weight < 0) or np.any(self.field_weight < 0):
            raise ValueError("SystemBatchHost: weights must be >= 0")
        if not self.reference_wavelength_nm > 0:
            raise ValueError("SystemBatchHost: reference wavelength must be > 0")
        if self.variant_surfaces is not None:
            vsf = np.asarray(self.variant_surfaces)
            if vsf.shape != (self.variants,) or np.any(vsf < 2) or np.any(vsf > self.surfaces):
                raise ValueError("SystemBatchHost: variant_surfaces must hold one count in "
                                 f"[2, {self.surfaces}] per variant")
        for f, m in enumerate(self.topology.pupil_mode):
            if m == PUPIL_AXIS and np.any(self.field_angle[:, f] != 0.0):
                raise ValueError(f"SystemBatchHost: field {f} is an axis field but a variant "
                                 "has a non-zero field angle (check_pupil_modes)")

    # ---- C ABI views ----------------------------------------------------------------------
    def view(self) -> _capi.BatchView:
        """mkb_batch_view over the host arrays (valid while this batch is alive)."""
        arrays = {}
        for name in ("type", "wavelength_weight", "field_weight", "curvature", "thickness",
                     "index", "pupil_radius", "field_angle", "field_target"):
            a = getattr(self, name)
            if not a.flags.c_contiguous:
                a = np.ascontiguousarray(a)
                setattr(self, name, a)
            arrays[name] = a
        v = _capi.BatchView()
        v.variants = self.variants
        v.surfaces, v.wavelengths, v.fields = self.surfaces, self.wavelengths, self.fields
        v.ghost_plates = self.topology.ghost_plates
        v.ghost_terms = self.topology.ghost_terms
        v.reference_wavelength_nm = self.reference_wavelength_nm
        v.type = _capi.ptr(arrays["type"], C.c_uint8)
        for name in ("wavelength_weight", "field_weight", "curvature", "thickness", "index",
                     "pupil_radius", "field_angle", "field_target"):
            setattr(v, name, _capi.ptr(arrays[name]))
        if self.decenter_tilt is not None:
            dt = np.ascontiguousarray(self.decenter_tilt, dtype=np.float64)
            arrays["decenter_tilt"] = dt
            v.decenter_tilt = _capi.ptr(dt)
        if self.buchdahl_coeff is not None:
            for name in ("buchdahl_coeff", "wavelength_nm"):
                a = np.ascontiguousarray(getattr(self, name), dtype=np.float64)
                arrays[name] = a
                setattr(v, name, _capi.ptr(a))
        if self.topology.ghost_plates > 0:
            for name in ("ghost_coeff", "ghost_norm_radius", "ghost_index"):
                a = np.ascontiguousarray(getattr(self, name), dtype=np.float64)
                if a.size == 0:
                    a = np.zeros(1)
                arrays[name] = a
                setattr(v, name, _capi.ptr(a))
        v._keep = arrays  # keep the arrays alive with the struct
        return v

    @property
    def non_coaxial(self) -> bool:
        return self.decenter_tilt is not None

    def buchdahl_omega(self) -> np.ndarray:
        """Buchdahl coordinate of every wavelength, dl / (1 + 2.5 dl), dl = lambda [um] -
        0.546074 (buchdahl_omega, glass/dispersion.hpp:87)."""
        dl = self.wavelength_nm / 1000.0 - BUCHDAHL_LAMBDA0_UM
        return dl / (1.0 + BUCHDAHL_ALPHA * dl)

    def refresh_glass_index(self, v: int, s: int) -> None:
        """index[v][s][:] from the Buchdahl coefficients, n0 + w (nu1 + w (nu2 + w nu3))
        (buchdahl_index, glass/dispersion.hpp:93)."""
        n0, nu1, nu2, nu3 = self.buchdahl_coeff[v, s]
        w = self.buchdahl_omega()
        self.index[v, s, :] = n0 + w * (nu1 + w * (nu2 + w * nu3))


def make_non_coaxial(batch: SystemBatchHost) -> SystemBatchHost:
    """Copy of `batch` with a non-coaxial topology: decenter and tilt all zero, every field on
    the Full pupil (make_non_coaxial, src/batch/system_batch.cpp)."""
    t = batch.topology
    topo = BatchTopology(t.surfaces, t.wavelengths, t.fields, list(t.type),
                         [PUPIL_FULL] * t.fields, non_coaxial=True, ghost_terms=t.ghost_terms)
    out = SystemBatchHost(topo, batch.variants)
    out.reference_wavelength_nm = batch.reference_wavelength_nm
    out.wavelength_nm = batch.wavelength_nm.copy()
    out.wavelength_weight = batch.wavelength_weight.copy()
    out.field_weight = batch.field_weight.copy()
    for name in ("curvature", "thickness", "index", "pupil_radius", "field_angle",
                 "field_target", "ghost_coeff", "ghost_norm_radius", "ghost_index"):
        setattr(out, name, np.array(getattr(batch, name), copy=True))
    if batch.variant_surfaces is not None:
        out.variant_surfaces = np.array(batch.variant_surfaces, copy=True)
    return out


@dataclass
class ResidualSettings:
    """ResidualSettings (batch_residuals.hpp:24). transverse_weight (>= 0, waves^2 / mm^2; not
    in the reference, whose rows are OPD only): with a positive weight every variant's residual
    vector ends with 2 x rays transverse ray-error rows (image-plane x errors, then y errors,
    relative to the ideal image point (0, h_f); mkb_residual_plan.transverse_weight)."""

    rings: int = 10
    spokes: int = 8
    failure: int = FAILURE_SOFT
    fail_weight: float = DEFAULT_FAIL_WEIGHT
    precision: int = PRECISION_FP64
    transverse_weight: float = 0.0


class ResidualLayout:
    """Row layout of one variant's residual vector (batch_residuals.hpp:62)."""

    def __init__(self, topology: BatchTopology, settings: ResidualSettings | None = None):
        settings = settings or ResidualSettings()
        topology.validate()
        if not 1 <= settings.rings <= MAX_RINGS:
            raise ValueError(f"ResidualLayout: rings must be in [1, {MAX_RINGS}]")
        if settings.spokes < 1:
            raise ValueError("ResidualLayout: spokes must be >= 1")
        if any(m != PUPIL_AXIS for m in topology.pupil_mode) and settings.spokes > 64:
            raise ValueError("ResidualLayout: spokes must be <= 64 in this build")
        if settings.failure not in (FAILURE_SOFT, FAILURE_HARD):
            raise ValueError("ResidualLayout: unknown failure mode")
        if not (settings.fail_weight >= 0 and math.isfinite(settings.fail_weight)):
            raise ValueError("ResidualLayout: fail_weight must be finite and >= 0")
        if settings.precision not in (PRECISION_FP64, PRECISION_MIXED, PRECISION_FP64_FMA,
                                      PRECISION_DF64, PRECISION_FP32_BULK):
            raise ValueError("ResidualLayout: unknown precision")
        if not (settings.transverse_weight >= 0 and math.isfinite(settings.transverse_weight)):
            raise ValueError("ResidualLayout: transverse_weight must be finite and >= 0")
        self.topology = topology
        self.settings = settings
        self.fields = topology.fields
        self.wavelengths = topology.wavelengths
        self.samples = [sample_count(settings.rings, settings.spokes, m)
                        for m in topology.pupil_mode]
        self.field_offset = []
        off = 0
        for n in self.samples:
            self.field_offset.append(off)
            off += self.wavelengths * n
        self.rays_per_variant = off

    def offset(self, f: int, l: int) -> int:
        if not 0 <= f < self.fields:
            raise IndexError(f"ResidualLayout: field {f} does not exist")
        if not 0 <= l < self.wavelengths:
            raise IndexError(f"ResidualLayout: wavelength {l} does not exist")
        return self.field_offset[f] + l * self.samples[f]

    @property
    def soft_failure(self) -> bool:
        return self.settings.failure == FAILURE_SOFT

    @property
    def penalty_rows(self) -> int:
        return self.rays_per_variant if self.soft_failure else 0

    @property
    def transverse_rows(self) -> int:
        return 2 * self.rays_per_variant if self.settings.transverse_weight > 0 else 0

    @property
    def trace_rows(self) -> int:
        return self.rays_per_variant + self.penalty_rows + self.transverse_rows

    def plan(self, batch: SystemBatchHost) -> _capi.ResidualPlan:
        """mkb_residual_plan for this layout and the shared weights of `batch`."""
        u, w = gauss_legendre_unit(self.settings.rings)
        keep = {
            "pupil_mode": np.asarray(self.topology.pupil_mode, dtype=np.uint8),
            "field_weight": np.ascontiguousarray(batch.field_weight, dtype=np.float64),
            "wavelength_weight": np.ascontiguousarray(batch.wavelength_weight,
                                                      dtype=np.float64),
            "quad_u": np.asarray(u, dtype=np.float64),
            "quad_w": np.asarray(w, dtype=np.float64),
        }
        p = _capi.ResidualPlan()
        p.rings, p.spokes = self.settings.rings, self.settings.spokes
        p.failure, p.precision = self.settings.failure, self.settings.precision
        p.fail_weight = self.settings.fail_weight
        p.transverse_weight = self.settings.transverse_weight
        p.reference_wavelength_nm = batch.reference_wavelength_nm
        p.fields, p.wavelengths = self.fields, self.wavelengths
        p.pupil_mode = _capi.ptr(keep["pupil_mode"], C.c_uint8)
        for name in ("field_weight", "wavelength_weight", "quad_u", "quad_w"):
            setattr(p, name, _capi.ptr(keep[name]))
        p._keep = keep
        return p


@dataclass
class Variable:
    """One LM variable (variable_set.hpp:20): type, table surface, bounds, typical size."""

    type: int
    surface: int
    lower: float = -math.inf
    upper: float = math.inf
    typical: float = 1.0
    # GhostCoefficient: a_order of plate `plate` (surface is then the plate's table surface)
    plate: int = -1
    order: int = 0
    # Glass: Buchdahl component (0 n0, 1 nu1, 2 nu2) of the medium after `surface`
    component: int = -1


@dataclass
class VariableSet:
    """Fixed list of P variables for batches of one topology (variable_set.hpp:63)."""

    topology: BatchTopology
    variables: list[Variable] = field(default_factory=list)

    def __post_init__(self):
        S = self.topology.surfaces
        if len(self.variables) > MAX_VARIABLES:
            raise ValueError(f"VariableSet: at most {MAX_VARIABLES} variables")
        seen = set()
        for k, v in enumerate(self.variables):
            if v.type == VAR_CURVATURE:
                if not (1 <= v.surface < S and self.topology.type[v.surface] == SURFACE_SPHERE):
                    raise ValueError(f"VariableSet: variable {k}: curvature needs a sphere")
            elif v.type == VAR_THICKNESS:
                if not 0 <= v.surface < S - 1:
                    raise ValueError(f"VariableSet: variable {k}: thickness surface out of range")
                if v.surface == 0 and self.topology.stop_surface > 0:
                    raise ValueError(f"VariableSet: variable {k}: thickness[0] follows the "
                                     "interior stop's entrance pupil")
            elif v.type == VAR_WORKING_DISTANCE:
                v.surface = S - 1
            elif v.type == VAR_GLASS:
                if not (0 <= v.surface < S and 0 <= v.component <= 2):
                    raise ValueError(f"VariableSet: variable {k}: glass component {v.component} "
                                     f"of surface {v.surface} does not exist")
            elif v.type == VAR_GHOST_COEFFICIENT:
                if not (0 <= v.plate < self.topology.ghost_plates and
                        1 <= v.order <= self.topology.ghost_terms):
                    raise ValueError(f"VariableSet: variable {k}: ghost coefficient a_{v.order} "
                                     f"of plate {v.plate} does not exist")
                v.surface = self.topology.ghost_surface(v.plate)
            else:
                raise NotImplementedError(f"VariableSet: variable type {v.type}")
            key = ((2, v.plate, v.order) if v.type == VAR_GHOST_COEFFICIENT
                   else (3, v.surface, v.component) if v.type == VAR_GLASS
                   else (v.type == VAR_CURVATURE, v.surface))
            if key in seen:
                raise ValueError(f"VariableSet: parameter of variable {k} already used")
            seen.add(key)
            if math.isnan(v.lower) or math.isnan(v.upper) or v.lower > v.upper:
                raise ValueError(f"VariableSet: invalid bounds of variable {k}")
            if not (v.typical > 0 and math.isfinite(v.typical)):
                raise ValueError(f"VariableSet: typical size of variable {k} must be > 0")

    @property
    def size(self) -> int:
        return len(self.variables)

    def lower(self) -> np.ndarray:
        return np.array([v.lower for v in self.variables])

    def upper(self) -> np.ndarray:
        return np.array([v.upper for v in self.variables])

    def typical(self) -> np.ndarray:
        return np.array([v.typical for v in self.variables])

    def extract(self, batch: SystemBatchHost, v: int) -> np.ndarray:
        """x from variant v (VariableSet::extract, variable_set.cpp:222)."""
        x = np.empty(self.size)
        for k, var in enumerate(self.variables):
            if var.type == VAR_GHOST_COEFFICIENT:
                x[k] = batch.ghost_coeff[v, var.plate, var.order - 1]
            elif var.type == VAR_GLASS:
                x[k] = batch.buchdahl_coeff[v, var.surface, var.component]
            else:
                x[k] = (batch.curvature[v, var.surface] if var.type == VAR_CURVATURE
                        else batch.thickness[v, var.surface])
        return x

    def apply(self, batch: SystemBatchHost, v: int, x) -> None:
        """Writes x into variant v (VariableSet::apply, variable_set.cpp:237)."""
        x = np.asarray(x, dtype=np.float64)
        if x.shape != (self.size,):
            raise ValueError("VariableSet.apply: x has the wrong length")
        if not np.all(np.isfinite(x)):
            raise ValueError("VariableSet.apply: x is not finite")
        for k, var in enumerate(self.variables):
            if var.type == VAR_CURVATURE:
                batch.curvature[v, var.surface] = x[k]
            elif var.type == VAR_GHOST_COEFFICIENT:
                batch.ghost_coeff[v, var.plate, var.order - 1] = x[k]
            elif var.type == VAR_GLASS:
                batch.buchdahl_coeff[v, var.surface, var.component] = x[k]
            else:
                batch.thickness[v, var.surface] = x[k]
        for s in sorted({var.surface for var in self.variables if var.type == VAR_GLASS}):
            batch.refresh_glass_index(v, s)

    def c_struct(self) -> _capi.Variables:
        keep = {
            "type": np.array([v.type for v in self.variables], dtype=np.int32),
            "surface": np.array([v.surface for v in self.variables], dtype=np.int32),
            "lower": self.lower(), "upper": self.upper(), "typical": self.typical(),
            "ghost_plate": np.array([v.plate for v in self.variables], dtype=np.int32),
            "ghost_order": np.array([v.order for v in self.variables], dtype=np.int32),
            "glass_component": np.array([v.component for v in self.variables], dtype=np.int32),
        }
        s = _capi.Variables()
        s.count = self.size
        s.type = _capi.ptr(keep["type"], C.c_int32)
        s.surface = _capi.ptr(keep["surface"], C.c_int32)
        s.ghost_plate = _capi.ptr(keep["ghost_plate"], C.c_int32)
        s.ghost_order = _capi.ptr(keep["ghost_order"], C.c_int32)
        s.glass_component = _capi.ptr(keep["glass_component"], C.c_int32)
        s.lower, s.upper, s.typical = (_capi.ptr(keep[n]) for n in ("lower", "upper", "typical"))
        s._keep = keep
        return s
