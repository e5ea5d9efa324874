"""Seeded synthetic workloads (lens systems) with the shapes of the benchmark configurations.

One generator feeds the CUDA path and the CPU oracles byte-identically. Random numbers come
from a counter-based splitmix64 stream (portable, no std:: distribution), Gaussian noise from
Box-Muller on it. Seeds: configuration k uses 20261203 + k unless given.

  singlet(...)    1024 biconvex singlets: stop plane at the first vertex, c = +1/50, -1/50,
                  t = 6 mm, image plane at the paraxial focus of each variant, 2-term Cauchy
                  n = 1.5046 + 0.00420 / lambda^2 (um) at 486.1 / 587.6 / 656.3 nm, fields
                  0, 0.7, 1.0 degree, pupil radius 5 mm, c1, c2, t perturbed by 5 % Gaussian
                  noise, quadrature 6 rings x 12 spokes.
  tolerancing(...) configuration 5: perturbed, decentered and tilted copies of one objective.
  objective(...)  4096 seven-element (14-sphere) objectives with curvatures U(-1/15, 1/15),
                  air gaps U(0.1, 5), glass thickness U(1, 8), 3-term Sellmeier glasses fitted
                  to n_d U(1.45, 1.90), V_d U(25, 95), 7 wavelengths 405..700 nm, 5 fields,
                  16 rings x 32 spokes, entrance pupil sized for image-side NA 0.95, image
                  plane at the paraxial focus, soft failure.
"""

from __future__ import annotations

import math

import numpy as np

from .batch import (BatchTopology, FAILURE_SOFT, PRECISION_FP64, ResidualSettings,
                    SURFACE_SPHERE, SURFACE_STOP, SystemBatchHost, VAR_CURVATURE,
                    VAR_THICKNESS, VAR_WORKING_DISTANCE, Variable, VariableSet)
from .quadrature import PUPIL_AXIS, PUPIL_FULL, PUPIL_HALF

_M64 = (1 << 64) - 1
_GOLDEN = 0x9E3779B97F4A7C15


def splitmix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser (Steele, Lea, Flood 2014) on uint64 arrays."""
    with np.errstate(over="ignore"):
        z = (x + np.uint64(_GOLDEN)).astype(np.uint64)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


class Stream:
    """Counter-based stream: draw n values for a named purpose, independent of call order."""

    def __init__(self, seed: int):
        self.seed = np.uint64(seed & _M64)

    def _bits(self, tag: int, n: int) -> np.ndarray:
        with np.errstate(over="ignore"):
            base = splitmix64(np.array([self.seed ^ np.uint64(tag * 0x632BE59BD9B4E019 & _M64)],
                                       dtype=np.uint64))[0]
            ctr = np.arange(n, dtype=np.uint64) * np.uint64(_GOLDEN) + base
        return splitmix64(ctr)

    def uniform(self, tag: int, n: int) -> np.ndarray:
        """U[0, 1) with 53 bits: (bits >> 11) * 2^-53."""
        return (self._bits(tag, n) >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)

    def normal(self, tag: int, n: int) -> np.ndarray:
        """N(0, 1) by Box-Muller on two uniform streams."""
        u1 = 1.0 - self.uniform(tag * 2 + 1, n)  # (0, 1]
        u2 = self.uniform(tag * 2 + 2, n)
        return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


def cauchy_index(lambda_nm, a: float = 1.5046, b: float = 0.00420) -> np.ndarray:
    lam_um = np.asarray(lambda_nm, dtype=np.float64) * 1e-3
    return a + b / (lam_um * lam_um)


def paraxial(curvature: np.ndarray, thickness: np.ndarray, index_ref: np.ndarray):
    """Paraxial y-nu trace of a collimated ray (y = 1) for [V][S] systems at one wavelength.

    index_ref[v][s] is the medium after surface s (air before surface 0). Returns (efl, bfd):
    effective focal length -1/u' and back focal distance -y/u' after the last surface.
    """
    V, S = curvature.shape
    y = np.ones(V)
    nu = np.zeros(V)  # n * u
    n_prev = index_ref[:, 0]
    for s in range(1, S):
        y = y + thickness[:, s - 1] * nu / n_prev
        n_after = index_ref[:, s]
        nu = nu - y * curvature[:, s] * (n_after - n_prev)
        n_prev = n_after
    u_last = nu / n_prev
    with np.errstate(divide="ignore", invalid="ignore"):
        efl = -1.0 / u_last
        bfd = -y / u_last
    return efl, bfd


# ---- configuration 1: biconvex singlets --------------------------------------------------

SINGLET_WAVELENGTHS = (486.1, 587.6, 656.3)


def singlet(variants: int = 1024, seed: int = 20261203 + 1, sigma: float = 0.05,
            failure: int = FAILURE_SOFT, precision: int = PRECISION_FP64):
    """Configuration 1. Returns (batch, settings, variables, x0 [V][P])."""
    topo = BatchTopology(surfaces=3, wavelengths=3, fields=3,
                         type=[SURFACE_STOP, SURFACE_SPHERE, SURFACE_SPHERE],
                         pupil_mode=[PUPIL_AXIS, PUPIL_HALF, PUPIL_HALF])
    b = SystemBatchHost(topo, variants)
    b.reference_wavelength_nm = 587.6
    b.wavelength_nm[:] = SINGLET_WAVELENGTHS
    b.wavelength_weight[:] = 1.0
    b.field_weight[:] = 1.0
    rng = Stream(seed)
    noise = rng.normal(1, 3 * variants).reshape(variants, 3)
    c1 = (1.0 / 50.0) * (1.0 + sigma * noise[:, 0])
    c2 = (-1.0 / 50.0) * (1.0 + sigma * noise[:, 1])
    t = 6.0 * (1.0 + sigma * noise[:, 2])
    b.curvature[:, 1] = c1
    b.curvature[:, 2] = c2
    b.thickness[:, 0] = 0.0  # stop plane at the first vertex
    b.thickness[:, 1] = t
    n = cauchy_index(SINGLET_WAVELENGTHS)
    b.index[:, 0, :] = 1.0
    b.index[:, 1, :] = n[None, :]
    b.index[:, 2, :] = 1.0
    n_ref = np.ones((variants, 3))
    n_ref[:, 1] = cauchy_index(587.6)
    efl, bfd = paraxial(b.curvature, b.thickness, n_ref)
    b.thickness[:, 2] = bfd
    b.pupil_radius[:] = 5.0
    angles = np.deg2rad(np.array([0.0, 0.7, 1.0]))
    b.field_angle[:, :] = angles[None, :]
    b.field_target[:, :] = efl[:, None] * np.tan(angles)[None, :]
    settings = ResidualSettings(rings=6, spokes=12, failure=failure, precision=precision)
    vs = VariableSet(topo, [
        Variable(VAR_CURVATURE, 1, -0.2, 0.2, 0.01),
        Variable(VAR_CURVATURE, 2, -0.2, 0.2, 0.01),
        Variable(VAR_THICKNESS, 1, 0.5, 20.0, 1.0),
        Variable(VAR_WORKING_DISTANCE, 2, 1.0, 500.0, 1.0),
    ])
    x0 = np.stack([vs.extract(b, v) for v in range(variants)])
    return b, settings, vs, x0


# ---- configuration 2: seven-element objectives ---------------------------------------------

OBJECTIVE_WAVELENGTHS = tuple(float(x) for x in np.linspace(405.0, 700.0, 7))
_SELLMEIER_C = (0.0060, 0.0200, 103.56)  # um^2, poles of the 3-term Sellmeier model
_SELLMEIER_B3 = 1.03


def sellmeier_index(b1, b2, lambda_nm):
    """n(lambda) of n^2 - 1 = sum_i B_i l^2 / (l^2 - C_i) with B3 and C_i fixed."""
    l2 = (np.asarray(lambda_nm, dtype=np.float64) * 1e-3) ** 2
    c1, c2, c3 = _SELLMEIER_C
    n2 = 1.0 + b1 * l2 / (l2 - c1) + b2 * l2 / (l2 - c2) + _SELLMEIER_B3 * l2 / (l2 - c3)
    return np.sqrt(n2)


def sellmeier_fit(nd, vd):
    """B1, B2 so that n(587.56) = n_d and n_F^2 - n_C^2 = 2 n_d (n_d - 1) / V_d.

    The second condition is the first-order form of n_F - n_C = (n_d - 1) / V_d; both are
    linear in (B1, B2) for fixed poles, so the fit is a 2x2 solve per glass.
    """
    nd = np.asarray(nd, dtype=np.float64)
    vd = np.asarray(vd, dtype=np.float64)
    c1, c2, c3 = _SELLMEIER_C

    def terms(lam_nm):
        l2 = (lam_nm * 1e-3) ** 2
        return l2 / (l2 - c1), l2 / (l2 - c2), _SELLMEIER_B3 * l2 / (l2 - c3)

    ad1, ad2, ad3 = terms(587.56)
    af1, af2, af3 = terms(486.13)
    ac1, ac2, ac3 = terms(656.27)
    r1 = nd * nd - 1.0 - ad3
    r2 = 2.0 * nd * (nd - 1.0) / vd - (af3 - ac3)
    m11, m12, m21, m22 = ad1, ad2, af1 - ac1, af2 - ac2
    det = m11 * m22 - m12 * m21
    b1 = (r1 * m22 - m12 * r2) / det
    b2 = (m11 * r2 - m21 * r1) / det
    return b1, b2


def objective(variants: int = 4096, seed: int = 20261203 + 2, rings: int = 16,
              spokes: int = 32, na: float = 0.95, max_field_deg: float = 1.0,
              failure: int = FAILURE_SOFT, precision: int = PRECISION_FP64,
              glass: bool = False):
    """Configuration 2. Returns (batch, settings, variables, x0 [V][P]).

    glass=True: the first element's glass becomes a Buchdahl glass (n0 = its n_d, nu1 =
    -0.12, nu2 = 0.03, nu3 = 0; index = n0 + w (nu1 + w (nu2 + w nu3)) at every wavelength)
    and its three Buchdahl coordinates join the variables (P = 32, the configuration-2 count),
    with the reference's typical sizes (1, 0.01, 0.001) and no bounds."""
    S = 15
    topo = BatchTopology(surfaces=S, wavelengths=7, fields=5,
                         type=[SURFACE_STOP] + [SURFACE_SPHERE] * 14,
                         pupil_mode=[PUPIL_AXIS] + [PUPIL_HALF] * 4)
    b = SystemBatchHost(topo, variants)
    b.reference_wavelength_nm = 587.56
    b.wavelength_nm[:] = OBJECTIVE_WAVELENGTHS
    b.wavelength_weight[:] = 1.0
    b.field_weight[:] = 1.0
    rng = Stream(seed)
    # Draw candidates in rounds; keep the first candidate of each variant whose paraxial
    # focal length and back focus are usable (5 <= f' <= 200 mm, BFD > 0.5 mm).
    todo = np.arange(variants)
    attempt = 0
    while todo.size:
        if attempt >= 64:
            raise RuntimeError("objective(): could not draw usable systems")
        n = todo.size
        tag = 100 * (attempt + 1)
        curv = (rng.uniform(tag + 1, variants * 14).reshape(variants, 14)[todo] * 2.0 - 1.0) / 15.0
        gaps = 0.1 + 4.9 * rng.uniform(tag + 2, variants * 8).reshape(variants, 8)[todo]
        glass_t = 1.0 + 7.0 * rng.uniform(tag + 3, variants * 7).reshape(variants, 7)[todo]
        nd = 1.45 + 0.45 * rng.uniform(tag + 4, variants * 7).reshape(variants, 7)[todo]
        vd = 25.0 + 70.0 * rng.uniform(tag + 5, variants * 7).reshape(variants, 7)[todo]
        c = np.zeros((n, S))
        t = np.zeros((n, S))
        c[:, 1:] = curv
        t[:, 0] = gaps[:, 0]
        for e in range(7):
            t[:, 1 + 2 * e] = glass_t[:, e]
            if e < 6:
                t[:, 2 + 2 * e] = gaps[:, e + 1]
        b1, b2 = sellmeier_fit(nd, vd)
        idx = np.ones((n, S, 7))
        n_ref = np.ones((n, S))
        for e in range(7):
            idx[:, 1 + 2 * e, :] = sellmeier_index(b1[:, e, None], b2[:, e, None],
                                                   np.array(OBJECTIVE_WAVELENGTHS)[None, :])
            n_ref[:, 1 + 2 * e] = sellmeier_index(b1[:, e], b2[:, e], 587.56)
        efl, bfd = paraxial(c, t, n_ref)
        ok = np.isfinite(efl) & (efl >= 5.0) & (efl <= 200.0) & np.isfinite(bfd) & (bfd > 0.5)
        sel = todo[ok]
        b.curvature[sel] = c[ok]
        t[ok, S - 1] = bfd[ok]
        b.thickness[sel] = t[ok]
        b.index[sel] = idx[ok]
        b.pupil_radius[sel] = na * efl[ok]
        b.field_target[sel] = efl[ok, None] * np.tan(
            np.deg2rad(max_field_deg * np.linspace(0.0, 1.0, 5)))[None, :]
        todo = todo[~ok]
        attempt += 1
    b.field_angle[:, :] = np.deg2rad(max_field_deg * np.linspace(0.0, 1.0, 5))[None, :]
    settings = ResidualSettings(rings=rings, spokes=spokes, failure=failure, precision=precision)
    variables = [Variable(VAR_CURVATURE, s, -0.2, 0.2, 0.01) for s in range(1, S)]
    variables += [Variable(VAR_THICKNESS, s, 0.05, 50.0, 1.0) for s in range(0, S - 1)]
    variables += [Variable(VAR_WORKING_DISTANCE, S - 1, 0.1, 1.0e4, 1.0)]
    if glass:
        from .batch import VAR_GLASS
        b.buchdahl_coeff = np.zeros((variants, S, 4))
        nd = sellmeier_index(*[a[:, 0] for a in sellmeier_fit(
            1.45 + 0.45 * rng.uniform(104, variants * 7).reshape(variants, 7)[:, :1],
            25.0 + 70.0 * rng.uniform(105, variants * 7).reshape(variants, 7)[:, :1])], 587.56)
        b.buchdahl_coeff[:, 1, 0] = nd
        b.buchdahl_coeff[:, 1, 1] = -0.12
        b.buchdahl_coeff[:, 1, 2] = 0.03
        for v in range(variants):
            b.refresh_glass_index(v, 1)
        variables += [Variable(VAR_GLASS, 1, -math.inf, math.inf, typ, component=c)
                      for c, typ in enumerate((1.0, 0.01, 0.001))]
    vs = VariableSet(topo, variables)
    x0 = np.stack([vs.extract(b, v) for v in range(variants)])
    return b, settings, vs, x0


def stop_heights(batch: SystemBatchHost, stop: int) -> tuple[np.ndarray, np.ndarray]:
    """y_A, y_B [V] of the aiming y-u trace (MKB_SURFACE_APERTURE_STOP): rays (y = 1, u = 0)
    and (y = 0, u = 1) at surface 1 traced to the stop at wavelength column 0."""
    V = batch.variants
    y1, u1, y2, u2 = np.ones(V), np.zeros(V), np.zeros(V), np.ones(V)
    n = batch.index[:, 0, 0].copy()
    for s in range(1, stop):
        n2 = batch.index[:, s, 0]
        c = batch.curvature[:, s] if batch.type[s] == SURFACE_SPHERE else np.zeros(V)
        phi = c * (n2 - n)
        u1 = (n * u1 - y1 * phi) / n2
        u2 = (n * u2 - y2 * phi) / n2
        y1 = y1 + batch.thickness[:, s] * u1
        y2 = y2 + batch.thickness[:, s] * u2
        n = n2
    return y1, y2


def with_aperture_stop(batch: SystemBatchHost, settings: ResidualSettings,
                       variables: VariableSet, stop: int):
    """The same systems with an aperture stop inside: a plane of kind SURFACE_APERTURE_STOP
    inserted as table surface `stop` at the vertex plane of the old surface `stop` (the old
    thickness[stop - 1] now leads to the stop, which is 0 ahead of the next surface and sits
    in the same medium). Its semi-aperture is chosen so that the aimed entrance pupil keeps the
    old pupil radius; surface 0 becomes that entrance pupil, so thickness[0] leaves the
    variables, and the stop's own gap to the next surface stays fixed (0). Returns (batch,
    settings, variables, x0). Coaxial batches of one table without ghost plates."""
    from .batch import SURFACE_APERTURE_STOP
    old = batch.topology
    if not 1 <= stop <= old.surfaces - 1:
        raise ValueError("with_aperture_stop: the stop goes between surfaces 1 and S - 1")
    S = old.surfaces + 1
    kinds = list(old.type[:stop]) + [SURFACE_APERTURE_STOP] + list(old.type[stop:])
    topo = BatchTopology(surfaces=S, wavelengths=old.wavelengths, fields=old.fields,
                         type=kinds, pupil_mode=list(old.pupil_mode))
    V = batch.variants
    b = SystemBatchHost(topo, V)
    b.reference_wavelength_nm = batch.reference_wavelength_nm
    b.wavelength_nm[:] = batch.wavelength_nm
    b.wavelength_weight[:] = batch.wavelength_weight
    b.field_weight[:] = batch.field_weight
    ins = lambda a, value: np.concatenate([a[:, :stop], value, a[:, stop:]], axis=1)
    b.curvature = ins(batch.curvature, np.zeros((V, 1)))
    b.thickness = ins(batch.thickness, np.zeros((V, 1)))
    b.index = ins(batch.index, batch.index[:, stop - 1:stop, :])
    if batch.buchdahl_coeff is not None:
        b.buchdahl_coeff = ins(batch.buchdahl_coeff, np.zeros((V, 1, 4)))
    b.pupil_radius = batch.pupil_radius.copy()
    b.field_angle = batch.field_angle.copy()
    b.field_target = batch.field_target.copy()
    ya, _ = stop_heights(b, stop)
    b.curvature[:, stop] = batch.pupil_radius * np.abs(ya)  # the stop's semi-aperture R
    moved = []
    for v in variables.variables:
        if v.type == VAR_THICKNESS and v.surface == 0:
            continue  # follows the entrance pupil now
        s_new = v.surface + (1 if v.surface >= stop else 0)
        moved.append(Variable(v.type, s_new, v.lower, v.upper, v.typical, plate=v.plate,
                              order=v.order, component=v.component))
    vs = VariableSet(topo, moved)
    x0 = np.stack([vs.extract(b, k) for k in range(V)]) if V else np.zeros((0, vs.size))
    return b, settings, vs, x0


# ---- configuration 3: uneven systems -----------------------------------------------------------

def uneven(variants: int = 8192, seed: int = 20261203 + 3, s_min: int = 6, s_max: int = 30,
           p_min: int = 8, p_max: int = 64, rings: int = 16, spokes: int = 32,
           sigma: float = 0.05, failure: int = FAILURE_SOFT, precision: int = PRECISION_FP64,
           plate: bool = True):
    """Configuration 3: variants of uneven surface and variable counts in one batch.

    Variant v has S_v ~ U{s_min .. s_max} table surfaces: the stop, then L = (S_v - 1) // 2
    biconvex elements in the style of configuration 1 (curvatures +-1/(50 L) and glass
    6/L mm, perturbed by `sigma` Gaussian noise, air gaps 0.5 mm, Cauchy glass at 7
    wavelengths 405..700 nm), and -- when S_v - 1 is odd -- a zero-power plate (curvature 0,
    air on both sides) before the image; the image plane sits at the paraxial focus. All
    variants share the 30-surface table (`variant_surfaces` holds S_v; the entries past S_v
    are unused). 5 fields 0..1 degree, all Half pupils 16 x 32, pupil radius 5 mm.
    plate=True: table surface 1 of every variant is a ghost plate of zero power (its K = 2
    Legendre coefficients 0, radius 8 mm, glass index 1.5) 0.5 mm after the stop, so every
    variant's count includes one zero-power ghost plate and the plate kernels run; the elements
    then start at surface 2 (L = (S_v - 2) // 2, the zero-curvature surface when S_v - 2 is
    odd).
    Variables of run v: the first P_v ~ U{p_min .. p_max} (at most all of them) of
    [working distance, element curvatures, glass thicknesses, air gaps].
    Returns (batch, settings, [VariableSet per run], [x0 row per run])."""
    S = s_max
    from .batch import SURFACE_GHOST_PLATE
    first = 2 if plate else 1  # table surface of the first element
    kinds = ([SURFACE_STOP, SURFACE_GHOST_PLATE] + [SURFACE_SPHERE] * (S - 2) if plate
             else [SURFACE_STOP] + [SURFACE_SPHERE] * (S - 1))
    topo = BatchTopology(surfaces=S, wavelengths=7, fields=5, type=kinds,
                         pupil_mode=[PUPIL_HALF] * 5, ghost_terms=2 if plate else 0)
    b = SystemBatchHost(topo, variants)
    if plate:
        b.ghost_coeff[:] = 0.0
        b.ghost_norm_radius[:] = 8.0
        b.ghost_index[:] = 1.5
    b.reference_wavelength_nm = 587.6
    b.wavelength_nm[:] = OBJECTIVE_WAVELENGTHS
    b.wavelength_weight[:] = 1.0
    b.field_weight[:] = 1.0
    rng = Stream(seed)
    sv = s_min + np.floor(rng.uniform(1, variants) * (s_max - s_min + 1)).astype(np.int64)
    pv = p_min + np.floor(rng.uniform(2, variants) * (p_max - p_min + 1)).astype(np.int64)
    noise = rng.normal(3, variants * 3 * S).reshape(variants, S, 3)
    n_glass = cauchy_index(OBJECTIVE_WAVELENGTHS)
    n_glass_ref = float(cauchy_index(587.6))
    angles = np.deg2rad(np.linspace(0.0, 1.0, 5))
    variable_sets, x0 = [], []
    for v in range(variants):
        n_surf = int(sv[v])
        elements = (n_surf - first) // 2
        c = np.zeros(S)
        t = np.zeros(S)
        idx = np.ones((S, 7))
        n_ref = np.ones(S)
        t[0] = 0.5 if plate else 0.0  # stop plane at the first vertex (or 0.5 mm to the plate)
        for e in range(elements):
            s1, s2 = first + 2 * e, first + 1 + 2 * e
            c[s1] = (1.0 / (50.0 * elements)) * (1.0 + sigma * noise[v, s1, 0])
            c[s2] = (-1.0 / (50.0 * elements)) * (1.0 + sigma * noise[v, s2, 0])
            t[s1] = (6.0 / elements) * (1.0 + sigma * noise[v, s1, 1])
            t[s2] = 0.5 * (1.0 + sigma * noise[v, s2, 1])
            idx[s1, :] = n_glass
            n_ref[s1] = n_glass_ref
        # surfaces past the elements (one zero-power plate when S_v - 1 is odd) stay c = 0
        _, bfd = paraxial(c[None, :n_surf], t[None, :n_surf], n_ref[None, :n_surf])
        efl, _ = paraxial(c[None, :n_surf], t[None, :n_surf], n_ref[None, :n_surf])
        t[n_surf - 1] = bfd[0]
        b.curvature[v] = c
        b.thickness[v] = t
        b.index[v] = idx
        b.pupil_radius[v] = 5.0
        b.field_angle[v] = angles
        b.field_target[v] = efl[0] * np.tan(angles)
        wd = (Variable(VAR_WORKING_DISTANCE, S - 1, 1.0, 500.0, 1.0) if n_surf == S
              else Variable(VAR_THICKNESS, n_surf - 1, 1.0, 500.0, 1.0))
        cands = [wd]
        cands += [Variable(VAR_CURVATURE, s, -0.2, 0.2, 0.01)
                  for s in range(first, first + 2 * elements)]
        cands += [Variable(VAR_THICKNESS, first + 2 * e, 0.1, 20.0, 1.0)
                  for e in range(elements)]
        cands += [Variable(VAR_THICKNESS, first + 1 + 2 * e, 0.1, 20.0, 1.0)
                  for e in range(elements - 1)]
        vs = VariableSet(topo, cands[:min(int(pv[v]), len(cands))])
        variable_sets.append(vs)
        x0.append(vs.extract(b, v))
    b.variant_surfaces = sv.astype(np.uint8)
    settings = ResidualSettings(rings=rings, spokes=spokes, failure=failure, precision=precision)
    return b, settings, variable_sets, x0


# ---- configuration 4: precision sweep -----------------------------------------------------------

def sweep(variants: int = 65536, seed: int = 20261203 + 4, surfaces: int = 20,
          wavelengths: int = 9, rings: int = 32, spokes: int = 32, sigma: float = 0.05,
          failure: int = FAILURE_SOFT, precision: int = PRECISION_FP64):
    """Configuration 4: `variants` systems of `surfaces` table surfaces in the element style of
    configuration 1 -- the stop, E = (S - 1) // 2 biconvex elements (curvatures +-1/(50 E),
    glass 6/E mm, air 0.5 mm, each perturbed by `sigma` Gaussian noise; Cauchy glass) and,
    when S - 1 is odd, a zero-power plate before the image at the paraxial focus -- at
    `wavelengths` wavelengths 405..700 nm, 5 fields 0..1 degree, Half pupils rings x spokes
    (32 x 32 = 1,024 rays per field and wavelength), pupil radius 5 mm. Variables: the working
    distance, every curvature and every glass thickness. Returns (batch, settings, variables,
    x0)."""
    S = surfaces
    E = (S - 1) // 2
    lam = np.linspace(405.0, 700.0, wavelengths)
    topo = BatchTopology(surfaces=S, wavelengths=wavelengths, fields=5,
                         type=[SURFACE_STOP] + [SURFACE_SPHERE] * (S - 1),
                         pupil_mode=[PUPIL_HALF] * 5)
    b = SystemBatchHost(topo, variants)
    b.reference_wavelength_nm = 587.6
    b.wavelength_nm[:] = lam
    b.wavelength_weight[:] = 1.0
    b.field_weight[:] = 1.0
    rng = Stream(seed)
    noise = rng.normal(1, variants * 2 * S).reshape(variants, S, 2)
    c = np.zeros((variants, S))
    t = np.zeros((variants, S))
    nr = np.ones((variants, S))
    for e in range(E):
        s1, s2 = 1 + 2 * e, 2 + 2 * e
        c[:, s1] = (1.0 / (50.0 * E)) * (1.0 + sigma * noise[:, s1, 0])
        c[:, s2] = (-1.0 / (50.0 * E)) * (1.0 + sigma * noise[:, s2, 0])
        t[:, s1] = (6.0 / E) * (1.0 + sigma * noise[:, s1, 1])
        t[:, s2] = 0.5 * (1.0 + sigma * noise[:, s2, 1])
        nr[:, s1] = float(cauchy_index(587.6))
    efl, bfd = paraxial(c, t, nr)
    t[:, S - 1] = bfd
    b.curvature[:] = c
    b.thickness[:] = t
    b.index[:] = 1.0
    n = cauchy_index(lam)
    for e in range(E):
        b.index[:, 1 + 2 * e, :] = n[None, :]
    angles = np.deg2rad(np.linspace(0.0, 1.0, 5))
    b.pupil_radius[:] = 5.0
    b.field_angle[:] = angles[None, :]
    b.field_target[:] = efl[:, None] * np.tan(angles)[None, :]
    settings = ResidualSettings(rings=rings, spokes=spokes, failure=failure, precision=precision)
    variables = [Variable(VAR_WORKING_DISTANCE, S - 1, 1.0, 500.0, 1.0)]
    variables += [Variable(VAR_CURVATURE, s, -0.2, 0.2, 0.01) for s in range(1, 1 + 2 * E)]
    variables += [Variable(VAR_THICKNESS, 1 + 2 * e, 0.1, 20.0, 1.0) for e in range(E)]
    vs = VariableSet(topo, variables)
    x0 = np.concatenate([b.thickness[:, S - 1:S], b.curvature[:, 1:1 + 2 * E],
                         b.thickness[:, 1:1 + 2 * E:2]], axis=1)
    return b, settings, vs, x0


# ---- ghost plates ------------------------------------------------------------------------------

def ghost(variants: int = 64, seed: int = 20261203 + 11, terms: int = 4,
          coeff_sigma: float = 2e-4, sigma: float = 0.05, rings: int = 6, spokes: int = 12,
          failure: int = FAILURE_SOFT, precision: int = PRECISION_FP64):
    """Two biconvex elements with a ghost plate in the air gap between them (table: stop,
    2 spheres, plate, 2 spheres): curvatures +1/60, -1/60, +1/70, -1/50 with `sigma` Gaussian
    noise, glass 5 and 4 mm (Cauchy n = 1.5046 + 0.00420/lambda^2 at 486.1 / 587.6 /
    656.3 nm), the gap 1 mm before and 1 mm after the plate, image at the paraxial focus of the
    elements. The plate: `terms` Legendre coefficients ~ N(0, coeff_sigma) mm per variant,
    normalisation radius 8 mm, glass index that of the elements. Fields 0, 0.7, 1 degree, Half
    pupils, pupil radius 5 mm. Variables: the four curvatures, both glass thicknesses, the
    working distance and the plate's coefficients. Returns (batch, settings, variables, x0)."""
    from .batch import SURFACE_GHOST_PLATE, VAR_GHOST_COEFFICIENT
    S = 6
    lam = np.array([486.1, 587.6, 656.3])
    topo = BatchTopology(surfaces=S, wavelengths=3, fields=3,
                         type=[SURFACE_STOP, SURFACE_SPHERE, SURFACE_SPHERE, SURFACE_GHOST_PLATE,
                               SURFACE_SPHERE, SURFACE_SPHERE],
                         pupil_mode=[PUPIL_HALF] * 3, ghost_terms=terms)
    b = SystemBatchHost(topo, variants)
    b.reference_wavelength_nm = 587.6
    b.wavelength_nm[:] = lam
    b.wavelength_weight[:] = 1.0
    b.field_weight[:] = 1.0
    rng = Stream(seed)
    noise = rng.normal(1, variants * 4).reshape(variants, 4)
    n = cauchy_index(lam)
    n_ref = float(cauchy_index(587.6))
    c = np.zeros((variants, S))
    c[:, 1] = (1.0 / 60.0) * (1.0 + sigma * noise[:, 0])
    c[:, 2] = (-1.0 / 60.0) * (1.0 + sigma * noise[:, 1])
    c[:, 4] = (1.0 / 70.0) * (1.0 + sigma * noise[:, 2])
    c[:, 5] = (-1.0 / 50.0) * (1.0 + sigma * noise[:, 3])
    t = np.zeros((variants, S))
    t[:, 1], t[:, 2], t[:, 3], t[:, 4] = 5.0, 1.0, 1.0, 4.0
    idx = np.ones((variants, S, 3))
    idx[:, 1, :] = n
    idx[:, 4, :] = n
    nr = np.ones((variants, S))
    nr[:, 1] = nr[:, 4] = n_ref
    efl, bfd = paraxial(c, t, nr)
    t[:, S - 1] = bfd
    b.curvature[:] = c
    b.thickness[:] = t
    b.index[:] = idx
    b.ghost_coeff[:] = coeff_sigma * rng.normal(2, variants * terms).reshape(variants, 1, terms)
    b.ghost_norm_radius[:] = 8.0
    b.ghost_index[:] = n[None, None, :]
    angles = np.deg2rad(np.array([0.0, 0.7, 1.0]))
    b.pupil_radius[:] = 5.0
    b.field_angle[:] = angles[None, :]
    b.field_target[:] = efl[:, None] * np.tan(angles)[None, :]
    settings = ResidualSettings(rings=rings, spokes=spokes, failure=failure, precision=precision)
    variables = [Variable(VAR_CURVATURE, s, -0.2, 0.2, 0.01) for s in (1, 2, 4, 5)]
    variables += [Variable(VAR_THICKNESS, s, 0.5, 20.0, 1.0) for s in (1, 4)]
    variables += [Variable(VAR_WORKING_DISTANCE, S - 1, 1.0, 500.0, 1.0)]
    variables += [Variable(VAR_GHOST_COEFFICIENT, 3, -0.1, 0.1, 1e-4, plate=0, order=k)
                  for k in range(1, terms + 1)]
    vs = VariableSet(topo, variables)
    x0 = np.stack([vs.extract(b, v) for v in range(variants)])
    return b, settings, vs, x0


# ---- configuration 5: Monte-Carlo tolerancing of a decentered / tilted objective --------------

ARCMIN = math.pi / 10800.0


def tolerancing(variants: int = 262144, seed: int = 20261203 + 5, elements: int = 10,
                rings: int = 16, spokes: int = 32, decenter_mm: float = 0.005,
                tilt_rad: float = ARCMIN, radius_rel: float = 0.001, thickness_mm: float = 0.010,
                index_delta: float = 2e-4, failure: int = FAILURE_SOFT,
                precision: int = PRECISION_FP64):
    """Configuration 5: `variants` perturbed copies of one nominal objective of `elements`
    biconvex elements (2 * elements spheres after the stop; element style of configuration 1:
    curvatures +-1/(50 E), glass 6/E mm, air 0.5 mm, Cauchy glass at 7 wavelengths, image at
    the paraxial focus), non-coaxial (every field on the Full pupil, 16 x 32), 5 fields
    0..1 degree, pupil radius 5 mm. Per variant, in the meaning of the reference's deviate
    model (tolerance/tolerance_model.hpp: c' = c/(1 + eps), t' = t + delta, n'(lambda) =
    n(lambda) + dn per glass, per-surface decenter and tilt): eps ~ U(-radius_rel, radius_rel)
    per sphere, delta ~ N(0, thickness_mm) per element thickness and air gap, dn ~
    N(0, index_delta) per glass, dx, dy ~ N(0, decenter_mm) and alpha, beta ~ N(0, tilt_rad)
    per sphere; normal draws are cut at 3 sigma. Variables: every curvature, every thickness
    between the spheres and the working distance (the design variables; the tolerances are
    not variables). Returns (batch, settings, variables, x0 [V][P])."""
    S = 1 + 2 * elements
    topo = BatchTopology(surfaces=S, wavelengths=7, fields=5,
                         type=[SURFACE_STOP] + [SURFACE_SPHERE] * (S - 1),
                         pupil_mode=[PUPIL_FULL] * 5, non_coaxial=True)
    b = SystemBatchHost(topo, variants)
    b.reference_wavelength_nm = 587.6
    b.wavelength_nm[:] = OBJECTIVE_WAVELENGTHS
    b.wavelength_weight[:] = 1.0
    b.field_weight[:] = 1.0
    rng = Stream(seed)
    # nominal design (one draw of the configuration-1 style element noise)
    nom = rng.normal(1, 3 * S).reshape(S, 3)
    c = np.zeros(S)
    t = np.zeros(S)
    idx = np.ones((S, 7))
    n_ref = np.ones(S)
    n_glass = cauchy_index(OBJECTIVE_WAVELENGTHS)
    for e in range(elements):
        s1, s2 = 1 + 2 * e, 2 + 2 * e
        c[s1] = (1.0 / (50.0 * elements)) * (1.0 + 0.05 * nom[s1, 0])
        c[s2] = (-1.0 / (50.0 * elements)) * (1.0 + 0.05 * nom[s2, 0])
        t[s1] = (6.0 / elements) * (1.0 + 0.05 * nom[s1, 1])
        t[s2] = 0.5 * (1.0 + 0.05 * nom[s2, 1])
        idx[s1, :] = n_glass
        n_ref[s1] = float(cauchy_index(587.6))
    efl, bfd = paraxial(c[None, :], t[None, :], n_ref[None, :])
    t[S - 1] = bfd[0]

    def cut_normal(tag, shape, sigma):
        z = rng.normal(tag, int(np.prod(shape))).reshape(shape)
        return sigma * np.clip(z, -3.0, 3.0)

    eps = radius_rel * (2.0 * rng.uniform(10, variants * (S - 1)).reshape(variants, S - 1) - 1.0)
    b.curvature[:, :] = c[None, :]
    b.curvature[:, 1:] = c[None, 1:] / (1.0 + eps)
    b.thickness[:, :] = t[None, :]
    b.thickness[:, 1:S - 1] += cut_normal(11, (variants, S - 2), thickness_mm)
    b.index[:, :, :] = idx[None, :, :]
    dn = cut_normal(12, (variants, elements), index_delta)
    for e in range(elements):
        b.index[:, 1 + 2 * e, :] += dn[:, e, None]
    b.decenter_tilt[:, 1:, 0] = cut_normal(13, (variants, S - 1), decenter_mm)
    b.decenter_tilt[:, 1:, 1] = cut_normal(14, (variants, S - 1), decenter_mm)
    b.decenter_tilt[:, 1:, 2] = cut_normal(15, (variants, S - 1), tilt_rad)
    b.decenter_tilt[:, 1:, 3] = cut_normal(16, (variants, S - 1), tilt_rad)
    angles = np.deg2rad(np.linspace(0.0, 1.0, 5))
    b.pupil_radius[:] = 5.0
    b.field_angle[:, :] = angles[None, :]
    b.field_target[:, :] = efl[0] * np.tan(angles)[None, :]
    settings = ResidualSettings(rings=rings, spokes=spokes, failure=failure, precision=precision)
    variables = [Variable(VAR_CURVATURE, s, -0.2, 0.2, 0.01) for s in range(1, S)]
    variables += [Variable(VAR_THICKNESS, s, 0.05, 50.0, 1.0) for s in range(1, S - 1)]
    variables += [Variable(VAR_WORKING_DISTANCE, S - 1, 0.1, 1000.0, 1.0)]
    vs = VariableSet(topo, variables)
    # the variables' values of every variant (VariableSet::extract, in the variables' order)
    x0 = np.concatenate([b.curvature[:, 1:S], b.thickness[:, 1:S - 1], b.thickness[:, S - 1:S]],
                        axis=1)
    return b, settings, vs, x0


def multistart(base: SystemBatchHost, seed: int = 20261203 + 21) -> SystemBatchHost:
    """Multistart variants of `base` for the FP32 prefilter, in the manner of the reference's
    acceptance batches (docs/numerik.md, "FP32-Vorfilterung"): every curvature scaled by
    1 + U(-0.5, 0.5), every thickness between the stop and the working distance by
    1 + U(-0.3, 0.3), the pupil radius by U(0.5, 2); every seventh variant is extreme (pupil by
    U(3, 5), curvatures by 1 + U(-1, 1)). Many rays then fail and the merits spread over orders
    of magnitude. Returns a new batch with the same topology and variant count."""
    b = base.subset(0, base.variants)
    V, S = b.variants, b.surfaces
    rng = Stream(seed)
    extreme = (np.arange(V) % 7) == 6
    cu = rng.uniform(1, V * S).reshape(V, S)
    tu = rng.uniform(2, V * S).reshape(V, S)
    pu = rng.uniform(3, V)
    cf = np.where(extreme[:, None], 1.0 + (2.0 * cu - 1.0), 1.0 + (cu - 0.5))
    b.curvature[:] = b.curvature * cf
    tf = 1.0 + 0.6 * (tu - 0.5)
    inner = np.zeros((V, S), dtype=bool)
    inner[:, 1:S - 1] = True
    b.thickness[:] = np.where(inner, b.thickness * tf, b.thickness)
    b.pupil_radius[:] = b.pupil_radius * np.where(extreme, 3.0 + 2.0 * pu, 0.5 + 1.5 * pu)
    return b


def unpad(batch: SystemBatchHost, v: int) -> SystemBatchHost:
    """Variant v of an uneven batch as a batch of its own S_v surfaces (one variant)."""
    n = int(batch.variant_surfaces[v]) if batch.variant_surfaces is not None else batch.surfaces
    kinds = list(batch.topology.type[:n])
    from .batch import SURFACE_GHOST_PLATE
    plates = sum(1 for k in kinds[1:] if k == SURFACE_GHOST_PLATE)  # the first plates of the table
    topo = BatchTopology(surfaces=n, wavelengths=batch.wavelengths, fields=batch.fields,
                         type=kinds, pupil_mode=list(batch.topology.pupil_mode),
                         ghost_terms=batch.topology.ghost_terms if plates else 0)
    out = SystemBatchHost(topo, 1)
    if plates:
        out.ghost_coeff[0] = batch.ghost_coeff[v, :plates]
        out.ghost_norm_radius[:] = batch.ghost_norm_radius[:plates]
        out.ghost_index[0] = batch.ghost_index[v, :plates]
    out.reference_wavelength_nm = batch.reference_wavelength_nm
    out.wavelength_nm = batch.wavelength_nm.copy()
    out.wavelength_weight = batch.wavelength_weight.copy()
    out.field_weight = batch.field_weight.copy()
    out.curvature[0] = batch.curvature[v, :n]
    out.thickness[0] = batch.thickness[v, :n]
    out.index[0] = batch.index[v, :n]
    out.pupil_radius[0] = batch.pupil_radius[v]
    out.field_angle[0] = batch.field_angle[v]
    out.field_target[0] = batch.field_target[v]
    return out
