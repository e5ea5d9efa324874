"""ctypes front end of the two CPU oracles (test infrastructure only).

``port()`` loads liboracle.so (the C restatement), ``reference()`` loads _ref/libmko_ref.so
(the reference's own sources); both expose the same calls on SystemBatchHost inputs.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from mikroptim_b200 import _capi
from mikroptim_b200.batch import ResidualLayout, SystemBatchHost, VariableSet

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libmko_ref.so")


def _reference_tree() -> str:
    """The reference source tree: $MKB_REFERENCE_TREE, else the Makefile's default REF."""
    env = os.environ.get("MKB_REFERENCE_TREE")
    if env:
        return env
    with open(os.path.join(HERE, "Makefile")) as fh:
        for line in fh:
            if line.startswith("REF ?="):
                return line.split("?=", 1)[1].strip()
    return ""


REFERENCE_TREE = _reference_tree()


def build(reference: bool = True) -> None:
    """Compile liboracle.so and, where the reference tree exists, _ref/libmko_ref.so."""
    targets = ["oracle"]
    if reference and os.path.isdir(os.path.join(REFERENCE_TREE, "src")):
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, f"-j{os.cpu_count() or 4}",
                    f"REF={REFERENCE_TREE}", *targets], check=True)


_PB = C.POINTER(_capi.BatchView)
_PP = C.POINTER(_capi.ResidualPlan)
_PV = C.POINTER(_capi.Variables)


class _Oracle:
    prefix = ""

    def __init__(self, path: str):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        p = self.prefix
        L = self.lib
        getattr(L, p + "residuals").argtypes = [_PB, _PP, C.c_void_p, C.c_void_p, C.c_void_p,
                                                C.c_int]
        getattr(L, p + "merit").argtypes = [_PB, _PP, C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.c_int]
        getattr(L, p + "normal_equations").argtypes = [C.c_void_p, C.c_void_p, C.c_int,
                                                       C.c_int64, C.c_void_p, C.c_void_p]
        for fn in ("residuals", "merit", "normal_equations", "fd_jacobian", "adjoint_jacobian"):
            getattr(L, p + fn).restype = C.c_int

    def _check(self, rc, what):
        if rc != 0:
            raise ValueError(f"{type(self).__name__}.{what} failed: {self.error()}")

    def error(self) -> str:
        return "bad argument"

    # ---- forward ------------------------------------------------------------------------
    def residuals(self, batch: SystemBatchHost, layout: ResidualLayout, threads: int = 1):
        V, rays, rows = batch.variants, layout.rays_per_variant, layout.trace_rows
        res = np.zeros((V, rows))
        opd = np.zeros((V, rays))
        st = np.zeros((V, rays), dtype=np.uint8)
        view, plan = batch.view(), layout.plan(batch)
        rc = getattr(self.lib, self.prefix + "residuals")(
            C.byref(view), C.byref(plan), res.ctypes.data, opd.ctypes.data, st.ctypes.data,
            threads)
        self._check(rc, "residuals")
        return res, opd, st

    def merit(self, batch: SystemBatchHost, layout: ResidualLayout, threads: int = 1):
        V = batch.variants
        merit = np.zeros(V)
        failed = np.zeros(V, dtype=np.int64)
        hard = np.zeros(V, dtype=np.int64)
        view, plan = batch.view(), layout.plan(batch)
        rc = getattr(self.lib, self.prefix + "merit")(
            C.byref(view), C.byref(plan), merit.ctypes.data, failed.ctypes.data,
            hard.ctypes.data, threads)
        self._check(rc, "merit")
        return merit, failed, hard

    # ---- Jacobians ----------------------------------------------------------------------
    def _jac_args(self, batch, layout, vs: VariableSet, x0):
        x0 = np.ascontiguousarray(x0, dtype=np.float64).reshape(-1, vs.size)
        runs = x0.shape[0]
        R = layout.trace_rows
        J = np.zeros((runs, vs.size, R))
        r0 = np.zeros((runs, R))
        return x0, runs, R, J, r0, batch.view(), layout.plan(batch), vs.c_struct()

    def normal_equations(self, J: np.ndarray, r: np.ndarray):
        P, R = J.shape
        J = np.ascontiguousarray(J)
        r = np.ascontiguousarray(r)
        A = np.zeros((P, P))
        g = np.zeros(P)
        rc = getattr(self.lib, self.prefix + "normal_equations")(
            J.ctypes.data, r.ctypes.data, P, R, A.ctypes.data, g.ctypes.data)
        self._check(rc, "normal_equations")
        return A, g


class Port(_Oracle):
    """liboracle.so: the plain-C restatement."""

    prefix = "mko_port_"

    def __init__(self, path: str = PORT_LIB):
        super().__init__(path)
        self.lib.mko_port_fd_jacobian.argtypes = [_PB, _PP, _PV, C.c_void_p, C.c_int,
                                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        self.lib.mko_port_adjoint_jacobian.argtypes = [_PB, _PP, _PV, C.c_void_p, C.c_int,
                                                       C.c_void_p, C.c_void_p, C.c_void_p,
                                                       C.c_int]

    def fd_jacobian(self, batch, layout, vs, x0, threads: int = 1):
        x0, runs, R, J, r0, view, plan, vars_ = self._jac_args(batch, layout, vs, x0)
        ch = np.zeros((runs, vs.size), dtype=np.int64)
        rc = self.lib.mko_port_fd_jacobian(C.byref(view), C.byref(plan), C.byref(vars_),
                                           x0.ctypes.data, runs, J.ctypes.data, r0.ctypes.data,
                                           ch.ctypes.data, threads)
        self._check(rc, "fd_jacobian")
        return J, r0, ch

    def aim(self, batch) -> tuple[np.ndarray, np.ndarray]:
        """The entrance pupil of an interior aperture stop (mko_port_aim): radius [V] and
        thickness[0] [V]."""
        self.lib.mko_port_aim.argtypes = [_PB, C.c_void_p, C.c_void_p]
        self.lib.mko_port_aim.restype = C.c_int
        view = batch.view()
        a = np.zeros(batch.variants)
        t0 = np.zeros(batch.variants)
        self._check(self.lib.mko_port_aim(C.byref(view), a.ctypes.data, t0.ctypes.data), "aim")
        return a, t0

    def aimed_equivalent(self, batch):
        """The batch the reference traces like an aimed one: the interior stop as a plane,
        surface 0 at the aimed entrance pupil."""
        from mikroptim_b200.batch import BatchTopology, SURFACE_APERTURE_STOP, SURFACE_PLANE
        import copy
        a, t0 = self.aim(batch)
        out = copy.deepcopy(batch)
        kinds = [SURFACE_PLANE if k == SURFACE_APERTURE_STOP else k for k in batch.topology.type]
        out.topology = BatchTopology(**{**batch.topology.__dict__, "type": kinds})
        out.type = np.asarray(kinds, dtype=np.uint8)
        out.pupil_radius = a
        out.thickness = batch.thickness.copy()
        out.thickness[:, 0] = t0
        out.curvature = batch.curvature.copy()
        out.curvature[:, batch.topology.stop_surface] = 0.0  # the stop's slot held R
        return out

    def adjoint_jacobian(self, batch, layout, vs, x0, threads: int = 1):
        x0, runs, R, J, r0, view, plan, vars_ = self._jac_args(batch, layout, vs, x0)
        st = np.zeros((runs, layout.rays_per_variant), dtype=np.uint8)
        rc = self.lib.mko_port_adjoint_jacobian(C.byref(view), C.byref(plan), C.byref(vars_),
                                                x0.ctypes.data, runs, J.ctypes.data,
                                                r0.ctypes.data, st.ctypes.data, threads)
        self._check(rc, "adjoint_jacobian")
        return J, r0, st


class Reference(_Oracle):
    """_ref/libmko_ref.so: the reference's own CPU sources."""

    prefix = "mko_ref_"

    def __init__(self, path: str = REF_LIB):
        super().__init__(path)
        L = self.lib
        L.mko_ref_last_error.restype = C.c_char_p
        L.mko_ref_fd_jacobian.argtypes = [_PB, _PP, _PV, C.c_void_p, C.c_int, C.c_void_p,
                                          C.c_void_p, C.c_void_p]
        L.mko_ref_adjoint_jacobian.argtypes = [_PB, _PP, _PV, C.c_void_p, C.c_int, C.c_void_p,
                                               C.c_void_p, C.c_void_p, C.c_int]
        L.mko_ref_optimize_lm.argtypes = [_PB, _PP, _PV, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                          C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p]
        L.mko_ref_optimize_lm.restype = C.c_int
        L.mko_ref_paraxial_residuals.argtypes = [_PB, _PP, C.c_int, C.c_int, C.c_void_p,
                                                 C.c_void_p, C.c_void_p, C.c_void_p,
                                                 C.c_void_p]
        L.mko_ref_paraxial_residuals.restype = C.c_int
        L.mko_ref_extra_rows.argtypes = [_PB, _PP, _PV, C.c_void_p, C.c_int, C.c_int,
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_void_p]
        L.mko_ref_extra_rows.restype = C.c_int
        L.mko_ref_surface_extrema.argtypes = [_PB, _PP, C.c_void_p]
        L.mko_ref_surface_extrema.restype = C.c_int
        _PF = C.POINTER(_capi.PrefilterOptions)
        L.mko_ref_prefilter.argtypes = [_PB, _PP, _PF] + [C.c_void_p] * 12
        L.mko_ref_prefilter.restype = C.c_int
        L.mko_ref_prefilter_decide_exact.argtypes = [_PF, C.c_int32, C.c_int64] + \
            [C.c_void_p] * 4
        L.mko_ref_prefilter_decide_exact.restype = C.c_int
        L.mko_ref_prefilter_rays.argtypes = [_PB, _PP, C.c_int, C.c_double, C.c_void_p,
                                             C.c_void_p, C.c_void_p]
        L.mko_ref_prefilter_rays.restype = C.c_int

    def error(self) -> str:
        return self.lib.mko_ref_last_error().decode(errors="replace")

    def fd_jacobian(self, batch, layout, vs, x0, threads: int = 1):
        x0, runs, R, J, r0, view, plan, vars_ = self._jac_args(batch, layout, vs, x0)
        ch = np.zeros((runs, vs.size), dtype=np.int64)
        rc = self.lib.mko_ref_fd_jacobian(C.byref(view), C.byref(plan), C.byref(vars_),
                                          x0.ctypes.data, runs, J.ctypes.data, r0.ctypes.data,
                                          ch.ctypes.data)
        self._check(rc, "fd_jacobian")
        return J, r0, ch

    def adjoint_jacobian(self, batch, layout, vs, x0, threads: int = 1):
        x0, runs, R, J, r0, view, plan, vars_ = self._jac_args(batch, layout, vs, x0)
        st = np.zeros((runs, layout.rays_per_variant), dtype=np.uint8)
        rc = self.lib.mko_ref_adjoint_jacobian(C.byref(view), C.byref(plan), C.byref(vars_),
                                               x0.ctypes.data, runs, J.ctypes.data,
                                               r0.ctypes.data, st.ctypes.data, threads)
        self._check(rc, "adjoint_jacobian")
        return J, r0, st

    @staticmethod
    def _constraints(constraints):
        """[(type, mode, weight, target)] -> the driver's flat arrays (type in ConstraintType
        order: 0 FocalLength, 1 ParfocalLength, 2 WorkingDistance, 3 ParaxialFocus, 4 Petzval;
        mode 0 Equal, 1 Min, 2 Max)."""
        c = list(constraints or [])
        return (len(c), np.array([k[0] for k in c], dtype=np.int32),
                np.array([k[1] for k in c], dtype=np.int32),
                np.array([k[2] for k in c], dtype=np.float64),
                np.array([k[3] for k in c], dtype=np.float64))

    def _ccall(self, constraints):
        n, t, m, w, g = self._constraints(constraints)
        self._keep_c = (t, m, w, g)
        return (n, t.ctypes.data, m.ctypes.data, w.ctypes.data, g.ctypes.data)

    def _tcall(self, tc):
        tc = list(tc or [])
        a = (np.array([k[0] for k in tc], dtype=np.int32),
             np.array([k[1] for k in tc], dtype=np.int32),
             np.array([k[2] for k in tc], dtype=np.float64),
             np.array([k[3] for k in tc], dtype=np.float64))
        self._keep_t = a
        return (len(tc),) + tuple(x.ctypes.data for x in a)

    def paraxial_residuals(self, batch, layout, v: int, constraints) -> np.ndarray:
        """The reference's paraxial_residuals of variant v (its ExtraResidualFn)."""
        n, t, m, w, g = self._constraints(constraints)
        out = np.zeros(n)
        view, plan = batch.view(), layout.plan(batch)
        rc = self.lib.mko_ref_paraxial_residuals(C.byref(view), C.byref(plan), v, n,
                                                 t.ctypes.data, m.ctypes.data, w.ctypes.data,
                                                 g.ctypes.data, out.ctypes.data)
        self._check(rc, "paraxial_residuals")
        return out

    def surface_extrema(self, batch, layout) -> np.ndarray:
        """The reference's surface_extrema_cpu (hard): [V][S][2] = (largest ray height,
        smallest cos I) per variant and surface over the rays with status Ok."""
        out = np.zeros((batch.variants, batch.surfaces, 2))
        view, plan = batch.view(), layout.plan(batch)
        self._check(self.lib.mko_ref_surface_extrema(C.byref(view), C.byref(plan),
                                                     out.ctypes.data), "surface_extrema")
        return out

    def extra_rows(self, batch, layout, vs, x0, constraints):
        """The reference's extra_rows_cpu with paraxial constraints: J [runs][P][E], r."""
        x0 = np.ascontiguousarray(x0, dtype=np.float64).reshape(-1, vs.size)
        runs = x0.shape[0]
        n = len(constraints)
        J = np.zeros((runs, vs.size, n))
        r = np.zeros((runs, n))
        view, plan, vars_ = batch.view(), layout.plan(batch), vs.c_struct()
        rc = self.lib.mko_ref_extra_rows(C.byref(view), C.byref(plan), C.byref(vars_),
                                         x0.ctypes.data, runs, *self._ccall(constraints),
                                         J.ctypes.data, r.ctypes.data)
        self._check(rc, "extra_rows")
        return J, r

    def eval(self, batch, layout, grid: int = 64, half: bool = False, reference: int = 0,
             delta: float = 1e-3) -> dict:
        """eval_cpu (src/eval/eval.cpp:307) in the reference's layout."""
        L = self.lib
        L.mko_ref_eval.argtypes = [_PB, _PP, C.c_int, C.c_int, C.c_int, C.c_double,
                                   C.c_void_p] + [C.c_void_p] * 8
        L.mko_ref_eval.restype = C.c_int
        view, plan = batch.view(), layout.plan(batch)
        n = C.c_int64()
        rc = L.mko_ref_eval(C.byref(view), C.byref(plan), grid, int(half), reference, delta,
                            C.addressof(n), *([None] * 8))
        self._check(rc, "eval")
        T = batch.variants * batch.fields * batch.wavelengths
        N = n.value
        out = dict(opd=np.zeros(T * N), spot_x=np.zeros(T * N), spot_y=np.zeros(T * N),
                   status=np.zeros(T * N, np.uint8), field_rays=np.zeros(T * 20),
                   field_status=np.zeros(T * 4, np.uint8),
                   kappa=np.zeros(batch.variants * batch.fields),
                   exit_pupil=np.zeros(batch.variants))
        rc = L.mko_ref_eval(C.byref(view), C.byref(plan), grid, int(half), reference, delta,
                            C.addressof(n), *[out[k].ctypes.data for k in (
                                "opd", "spot_x", "spot_y", "status", "field_rays",
                                "field_status", "kappa", "exit_pupil")])
        self._check(rc, "eval")
        return out

    PSF_METRICS = ("transmitted", "energy", "strehl_fft", "strehl_origin", "strehl",
                   "reference_x", "reference_y", "peak", "peak_x", "peak_y", "dx", "dy",
                   "airy_radius")

    def psf(self, batch, layout, v: int = 0, grid: int = 32, half: bool = False,
            reference: int = 0, delta: float = 1e-3, padding: float = 4.0,
            na: float = 0.0) -> dict:
        """eval_cpu, make_psf_pupils and psf_cpu (src/eval/psf.cpp:196,330) of variant v: the
        pupils' maps, NA and flips, PSF [T][M][M], MTF [T][2][N + 1] and the figures."""
        L = self.lib
        L.mko_ref_psf.argtypes = [_PB, _PP, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int,
                                  C.c_double, C.c_double, C.c_void_p, C.c_void_p] + \
            [C.c_void_p] * 6
        L.mko_ref_psf.restype = C.c_int
        view, plan = batch.view(), layout.plan(batch)
        lam = np.ascontiguousarray(batch.wavelength_nm, dtype=np.float64)
        view.wavelength_nm = lam.ctypes.data_as(C.POINTER(C.c_double))
        m, full = C.c_int(), C.c_int()
        rc = L.mko_ref_psf(C.byref(view), C.byref(plan), grid, int(half), reference, delta, v,
                           padding, na, C.addressof(m), C.addressof(full), *([None] * 6))
        self._check(rc, "psf")
        T, M = batch.fields * batch.wavelengths, m.value
        out = dict(fft_size=M, full_count=full.value, maps=np.zeros((T, grid * grid)),
                   na=np.zeros((T, 2)), flips=np.zeros((T, 2), np.int32),
                   psf=np.zeros((T, M * M)), mtf=np.zeros((T, 2, grid + 1)),
                   metrics=np.zeros((T, 13)))
        rc = L.mko_ref_psf(C.byref(view), C.byref(plan), grid, int(half), reference, delta, v,
                           padding, na, C.addressof(m), C.addressof(full),
                           *[out[k].ctypes.data for k in ("maps", "na", "flips", "psf", "mtf",
                                                          "metrics")])
        self._check(rc, "psf")
        return out

    def psf_pupil(self, grid: int, fft_size: int, opd_map, full_count: int,
                  wavelength_nm: float, na_x: float, na_y: float, flip_x: bool = False,
                  flip_y: bool = False) -> dict:
        """psf_cpu (src/eval/psf.cpp:330) of one given pupil map."""
        L = self.lib
        L.mko_ref_psf_pupil.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_double,
                                        C.c_double, C.c_double, C.c_int, C.c_int, C.c_void_p,
                                        C.c_void_p, C.c_void_p]
        L.mko_ref_psf_pupil.restype = C.c_int
        opd = np.ascontiguousarray(opd_map, dtype=np.float64)
        out = dict(psf=np.zeros(fft_size * fft_size), mtf=np.zeros((2, grid + 1)),
                   metrics=np.zeros(13))
        rc = L.mko_ref_psf_pupil(grid, fft_size, opd.ctypes.data, full_count, wavelength_nm,
                                 na_x, na_y, int(flip_x), int(flip_y), out["psf"].ctypes.data,
                                 out["mtf"].ctypes.data, out["metrics"].ctypes.data)
        self._check(rc, "psf_pupil")
        return out

    def psf_finish(self, grid: int, fft_size: int, opd_map, full_count: int,
                   wavelength_nm: float, na_x: float, na_y: float, flip_x: bool, flip_y: bool,
                   psf) -> np.ndarray:
        """finish_psf (src/eval/psf.cpp:290) on a given PSF: the 13 figures."""
        L = self.lib
        L.mko_ref_psf_finish.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_double,
                                         C.c_double, C.c_double, C.c_int, C.c_int, C.c_void_p,
                                         C.c_void_p]
        L.mko_ref_psf_finish.restype = C.c_int
        opd = np.ascontiguousarray(opd_map, dtype=np.float64)
        p = np.ascontiguousarray(psf, dtype=np.float64)
        out = np.zeros(13)
        rc = L.mko_ref_psf_finish(grid, fft_size, opd.ctypes.data, full_count, wavelength_nm,
                                  na_x, na_y, int(flip_x), int(flip_y), p.ctypes.data,
                                  out.ctypes.data)
        self._check(rc, "psf_finish")
        return out

    def prefilter(self, batch, layout, options, extra=None) -> dict:
        """prefilter_cpu (src/batch/batch_prefilter.cpp): raw per-variant results and the
        decision. `options` is a _capi.PrefilterOptions."""
        V = batch.variants
        out = dict(merit=np.zeros(V), optical_length=np.zeros(V),
                   failed=np.zeros(V, np.int64), uncertain_ok=np.zeros(V, np.int64),
                   uncertain_failed=np.zeros(V, np.int64), merit_lower=np.zeros(V),
                   merit_upper=np.zeros(V), reject=np.zeros(V, np.uint8))
        ref_m = C.c_double()
        ref_v = C.c_int32()
        kept = C.c_int32()
        ex = None if extra is None else np.ascontiguousarray(extra, dtype=np.float64)
        view, plan = batch.view(), layout.plan(batch)
        rc = self.lib.mko_ref_prefilter(
            C.byref(view), C.byref(plan), C.byref(options),
            ex.ctypes.data if ex is not None else None,
            *[out[k].ctypes.data for k in ("merit", "optical_length", "failed", "uncertain_ok",
                                           "uncertain_failed", "merit_lower", "merit_upper",
                                           "reject")],
            C.addressof(ref_m), C.addressof(ref_v), C.addressof(kept))
        self._check(rc, "prefilter")
        out.update(reference_merit=ref_m.value, reference_variant=ref_v.value, kept=kept.value)
        return out

    def prefilter_decide_exact(self, options, merit, failed, rays_per_variant, extra=None):
        merit = np.ascontiguousarray(merit, dtype=np.float64)
        failed = np.ascontiguousarray(failed, dtype=np.int64)
        ex = None if extra is None else np.ascontiguousarray(extra, dtype=np.float64)
        reject = np.zeros(len(merit), np.uint8)
        rc = self.lib.mko_ref_prefilter_decide_exact(
            C.byref(options), len(merit), rays_per_variant, merit.ctypes.data,
            failed.ctypes.data, ex.ctypes.data if ex is not None else None, reject.ctypes.data)
        self._check(rc, "prefilter_decide_exact")
        return reject

    def prefilter_rays(self, batch, layout, v: int, boundary: float):
        """prefilter_rays_cpu: status, margin and certain flag of variant v's rays."""
        R = layout.rays_per_variant
        status = np.zeros(R, np.uint8)
        margin = np.zeros(R)
        certain = np.zeros(R, np.uint8)
        view, plan = batch.view(), layout.plan(batch)
        rc = self.lib.mko_ref_prefilter_rays(C.byref(view), C.byref(plan), v, boundary,
                                             status.ctypes.data, margin.ctypes.data,
                                             certain.ctypes.data)
        self._check(rc, "prefilter_rays")
        return status, margin, certain

    def optimize_lm(self, batch, layout, vs, x0, max_iterations: int = 100,
                    method: str = "adjoint", penalty_rounds: int = 1, threads: int = 0,
                    constraints=None, trace_constraints=None):
        """trace_constraints: [(surface, kind, weight, limit)], rows from the extrema of the
        trace: kind 0 sqrt(w) max(0, h_s - limit), kind 1 sqrt(w) max(0, limit - cos I_s)."""
        x0 = np.ascontiguousarray(x0, dtype=np.float64).reshape(-1, vs.size)
        runs, P = x0.shape
        x = np.zeros((runs, P))
        merit = np.zeros(runs)
        status = np.zeros(runs, dtype=np.int32)
        its = np.zeros(runs, dtype=np.int32)
        acc = np.zeros(runs, dtype=np.int32)
        hist = np.zeros((runs, max_iterations + 1))
        view, plan, vars_ = batch.view(), layout.plan(batch), vs.c_struct()
        rc = self.lib.mko_ref_optimize_lm(
            C.byref(view), C.byref(plan), C.byref(vars_), x0.ctypes.data, runs, max_iterations,
            1 if method == "adjoint" else 0, penalty_rounds, threads, x.ctypes.data,
            merit.ctypes.data, status.ctypes.data, its.ctypes.data, acc.ctypes.data,
            hist.ctypes.data, *self._ccall(constraints), *self._tcall(trace_constraints))
        self._check(rc, "optimize_lm")
        return dict(x=x, merit=merit, status=status, iterations=its, accepted=acc,
                    history=hist)


_port = None
_reference = None


def port() -> Port:
    global _port
    if _port is None:
        _port = Port()
    return _port


def reference() -> Reference:
    global _reference
    if _reference is None:
        _reference = Reference()
    return _reference
