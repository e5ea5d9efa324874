/*
 * Test infrastructure (the oracle), not product code.
 *
 * Plain-C restatement of the reference CPU algorithm of the batched trace-and-optimise path
 * (collimated source, stop/plane/sphere surfaces, reference sphere through the vertex of the
 * last surface, ideal image point). It is compiled like the reference (-O2,
 * -ffp-contract=off, no fast-math) and performs every floating-point operation in the
 * reference's order, so on the same inputs it agrees with the reference build bit for bit;
 * the tests check that against oracle/_ref. Each function names the reference file:line it
 * restates (paths inside the reference project).
 */
#include "mko_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---- host threads: contiguous variant ranges per thread, like the reference's
 * detail::parallel_for_variants (src/optim/parallel_variants.hpp:21); results never depend
 * on the thread count because every item writes only its own outputs. */
#include <pthread.h>

typedef void (*item_fn)(void* ctx, int i);
typedef struct { item_fn fn; void* ctx; int first, last; } chunk_t;

static void* run_chunk(void* arg) {
    chunk_t* c = (chunk_t*)arg;
    for (int i = c->first; i < c->last; ++i) c->fn(c->ctx, i);
    return NULL;
}

static void parallel_for(int count, int threads, item_fn fn, void* ctx) {
    int T = threads > 0 ? threads : 1;
    if (T > count) T = count;
    if (T <= 1) {
        for (int i = 0; i < count; ++i) fn(ctx, i);
        return;
    }
    pthread_t tid[256];
    chunk_t chunk[256];
    if (T > 256) T = 256;
    for (int c = 0; c < T; ++c) {
        chunk[c].fn = fn;
        chunk[c].ctx = ctx;
        chunk[c].first = (int)((int64_t)count * c / T);
        chunk[c].last = (int)((int64_t)count * (c + 1) / T);
    }
    for (int c = 1; c < T; ++c) pthread_create(&tid[c], NULL, run_chunk, &chunk[c]);
    run_chunk(&chunk[0]);
    for (int c = 1; c < T; ++c) pthread_join(tid[c], NULL);
}

/* ---- small vector algebra: include/mikroptim/math/vec3.hpp:9-60 ------------------------ */
typedef struct { double x, y, z; } vec3;
typedef struct { vec3 p, d; double opl; } ray_t;             /* trace/ray.hpp:9 */

static vec3 v_add(vec3 a, vec3 b) { vec3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static vec3 v_sub(vec3 a, vec3 b) { vec3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static vec3 v_scale(double s, vec3 a) { vec3 r = {s * a.x, s * a.y, s * a.z}; return r; }
static double v_dot(vec3 a, vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static double v_norm(vec3 a) { return sqrt(v_dot(a, a)); }
static vec3 v_zero(void) { vec3 r = {0.0, 0.0, 0.0}; return r; }

/* ---- status, soft failure: trace/surface_ops.hpp:24-118 --------------------------------- */
enum { ST_OK = 0, ST_MISSED = 1, ST_TIR = 2, ST_BACKWARD = 3, ST_UNSUPPORTED = 4,
       ST_SOFT_MISSED = 5, ST_SOFT_TIR = 6 };
enum { BR_REGULAR = 0, BR_SOFT_MISSED = 1, BR_SOFT_TIR = 2 };

typedef struct { double penalty; int first; } soft_t;

static int is_soft(int s) { return s == ST_SOFT_MISSED || s == ST_SOFT_TIR; }
static int in_piston(int s) { return s == ST_OK || is_soft(s); }
static int is_hard(int s) { return !in_piston(s); }
static void soft_add(soft_t* s, double amount, int kind) {       /* surface_ops.hpp:94 */
    s->penalty += amount;
    if (s->first == ST_OK) s->first = kind;
}

/* transfer_to_tangent_plane, surface_ops.hpp:122 */
static double transfer_to_tangent_plane(ray_t* r, double t) {
    r->p.z -= t;
    const double s = -r->p.z / r->d.z;
    r->p = v_add(r->p, v_scale(s, r->d));
    r->p.z = 0.0;
    return s;
}

/* intersect_sphere, surface_ops.hpp:144 */
static int intersect_sphere(ray_t* r, double c, double* s, soft_t* soft) {
    const double H = c * (r->p.x * r->p.x + r->p.y * r->p.y);
    const double B = r->d.z - c * (r->p.x * r->d.x + r->p.y * r->d.y);
    const double D = B * B - c * H;
    if (D < 0.0) {
        if (soft == NULL || (!(c > 0.0) && !(c < 0.0))) return ST_MISSED;
        soft_add(soft, -D, ST_SOFT_MISSED);
        *s = B / c;
        r->p = v_add(r->p, v_scale(*s, r->d));
        return ST_SOFT_MISSED;
    }
    const double denom = B + sqrt(D);
    if (!(denom > 0.0)) return ST_MISSED;
    *s = H / denom;
    r->p = v_add(r->p, v_scale(*s, r->d));
    return ST_OK;
}

/* refract_sphere, surface_ops.hpp:181 */
static int refract_sphere(ray_t* r, double c, double mu, soft_t* soft, int off_surface) {
    vec3 N = {-c * r->p.x, -c * r->p.y, 1.0 - c * r->p.z};
    if (off_surface) N = v_scale(1.0 / v_norm(N), N);
    const double cosI = v_dot(r->d, N);
    const double k = 1.0 - mu * mu * (1.0 - cosI * cosI);
    if (k < 0.0) {
        if (soft == NULL) return ST_TIR;
        soft_add(soft, -k, ST_SOFT_TIR);
        const vec3 t = v_sub(r->d, v_scale(cosI, N));
        r->d = v_scale(1.0 / v_norm(t), t);
        return ST_SOFT_TIR;
    }
    r->d = v_add(v_scale(mu, r->d), v_scale(sqrt(k) - mu * cosI, N));
    return ST_OK;
}

/* ---- ghost plates: trace/ghost_plate.hpp --------------------------------------------------
 * One plate at one wavelength (GhostPlateParams, ghost_plate.hpp:24). */
typedef struct {
    const double* coeff;  /* a_1 .. a_K */
    int terms;
    double norm_radius, n_glass;
} ghost_t;

/* ghost_profile, ghost_plate.hpp:67: t(u) and dt/du by the Legendre recurrences */
static void ghost_profile(const ghost_t* g, double u, double* t_out, double* dt_du) {
    const double xi = 2.0 * u - 1.0;
    double p_prev = 1.0, p_cur = xi, dp_prev = 0.0, dp_cur = 1.0, t = 0.0, dt = 0.0;
    for (int k = 1; k <= g->terms; ++k) {
        const double a = g->coeff[k - 1];
        t += a * p_cur;
        dt += a * dp_cur;
        const double p_next = ((double)(2 * k + 1) * xi * p_cur - (double)k * p_prev) /
                              (double)(k + 1);
        const double dp_next = dp_prev + (double)(2 * k + 1) * p_cur;
        p_prev = p_cur;
        p_cur = p_next;
        dp_prev = dp_cur;
        dp_cur = dp_next;
    }
    *t_out = t;
    *dt_du = 2.0 * dt;
}

/* phase_surface_step, ghost_plate.hpp:130 */
static int phase_surface_step(ray_t* ray, double phase, double grad_x, double grad_y,
                              double n_before, double n_after, soft_t* soft) {
    ray->opl += phase;
    const double dx = (n_before * ray->d.x + grad_x) / n_after;
    const double dy = (n_before * ray->d.y + grad_y) / n_after;
    const double radicand = 1.0 - dx * dx - dy * dy;
    if (radicand < 0.0) {
        if (soft == NULL) return ST_TIR;
        soft_add(soft, -radicand, ST_SOFT_TIR);
        const double inv = 1.0 / sqrt(dx * dx + dy * dy);
        vec3 d = {dx * inv, dy * inv, 0.0};
        ray->d = d;
        return ST_SOFT_TIR;
    }
    vec3 d = {dx, dy, sqrt(radicand)};
    ray->d = d;
    return ST_OK;
}

/* ghost_plate_step, ghost_plate.hpp:159 */
static int ghost_plate_step(ray_t* ray, const ghost_t* g, double n_before, double n_after,
                            soft_t* soft) {
    const double inv_r2 = 1.0 / (g->norm_radius * g->norm_radius);
    const double u = (ray->p.x * ray->p.x + ray->p.y * ray->p.y) * inv_r2;
    double t, dt_du;
    ghost_profile(g, u, &t, &dt_du);
    const double dn = g->n_glass - n_before;
    const double radial = dn * dt_du * 2.0 * inv_r2;
    return phase_surface_step(ray, dn * t, radial * ray->p.x, radial * ray->p.y, n_before,
                              n_after, soft);
}

/* propagate_surface_local, trace/trace.hpp:174 (stop, plane, sphere; ghost plate with `ghost`) */
static int propagate_surface_g(ray_t* ray, double t, int kind, double c, double n_before,
                               double n_after, soft_t* soft, unsigned char* branch,
                               const ghost_t* ghost) {
    if (kind == MKB_SURFACE_GHOST_PLATE) {
        if (ghost == NULL) return ST_UNSUPPORTED;
        if (!(ray->d.z > 0.0)) return ST_BACKWARD;
        const double s0 = transfer_to_tangent_plane(ray, t);
        ray->opl += n_before * s0;
        const int step = ghost_plate_step(ray, ghost, n_before, n_after, soft);
        if (step == ST_SOFT_TIR) {
            if (branch != NULL) *branch = BR_SOFT_TIR;
            return ST_OK;
        }
        if (branch != NULL) *branch = BR_REGULAR;
        return step;
    }
    double curv;
    if (kind == MKB_SURFACE_STOP || kind == MKB_SURFACE_PLANE) curv = 0.0;
    else if (kind == MKB_SURFACE_SPHERE) curv = c;
    else return ST_UNSUPPORTED;
    if (!(ray->d.z > 0.0)) return ST_BACKWARD;
    const double s0 = transfer_to_tangent_plane(ray, t);
    double s = 0.0;
    const int hit = intersect_sphere(ray, curv, &s, soft);
    if (hit != ST_OK && hit != ST_SOFT_MISSED) return hit;
    ray->opl += n_before * (s0 + s);
    const int refr = refract_sphere(ray, curv, n_before / n_after, soft, hit == ST_SOFT_MISSED);
    if (branch != NULL)
        *branch = (unsigned char)((hit == ST_SOFT_MISSED ? BR_SOFT_MISSED : BR_REGULAR) |
                                  (refr == ST_SOFT_TIR ? BR_SOFT_TIR : BR_REGULAR));
    return refr == ST_SOFT_TIR ? ST_OK : refr;
}

static int propagate_surface(ray_t* ray, double t, int kind, double c, double n_before,
                             double n_after, soft_t* soft, unsigned char* branch) {
    return propagate_surface_g(ray, t, kind, c, n_before, n_after, soft, branch, NULL);
}

/* reference_sphere_step, trace/reference_sphere.hpp:55 */
static int reference_sphere_step(ray_t* ray, vec3 center, double n_image, double* s_out,
                                 soft_t* soft) {
    const vec3 q = v_sub(ray->p, center);
    const double b = -v_dot(q, ray->d);
    const double g = v_dot(ray->p, v_sub(ray->p, v_scale(2.0, center)));
    const double disc = b * b - g;
    if (disc < 0.0) {
        const double radius_sq = v_dot(center, center);
        if (soft == NULL || !(radius_sq > 0.0)) return ST_MISSED;
        soft_add(soft, -disc / radius_sq, ST_SOFT_MISSED);
        ray->p = v_add(ray->p, v_scale(b, ray->d));
        ray->opl += n_image * b;
        if (s_out) *s_out = b;
        return ST_SOFT_MISSED;
    }
    const double root = sqrt(disc);
    const int real_image = center.z >= 0.0;
    const double denom = real_image ? b + root : b - root;
    if (!(real_image ? denom > 0.0 : denom < 0.0)) return ST_MISSED;
    const double s = g / denom;
    ray->p = v_add(ray->p, v_scale(s, ray->d));
    ray->opl += n_image * s;
    if (s_out) *s_out = s;
    return ST_OK;
}

/* ---- one variant's surface table (SystemBatchView::surface_table, system_batch_view.hpp:155) */
typedef struct {
    int S, L;
    const uint8_t* type;
    const double* c;  /* [S] */
    const double* t;  /* [S] */
    const double* n;  /* [S][L] */
    const double* xf; /* [S][4] dx, dy, alpha, beta, or NULL (coaxial) */
    int G, K;         /* ghost plates (GhostPlate surfaces in table order) and their terms */
    const double* gcoeff;   /* [G][K] */
    const double* gradius;  /* [G] */
    const double* gindex;   /* [G][L] */
} table_t;

/* plate data of plate g at wavelength l */
static ghost_t ghost_of(const table_t* sys, int g, int l) {
    ghost_t r = {sys->gcoeff + (size_t)g * sys->K, sys->K, sys->gradius[g],
                 sys->gindex[(size_t)g * sys->L + l]};
    return r;
}

/* ---- decenter and tilt: trace/surface_transform.hpp:27-140 ---------------------------- */
typedef struct { double dx, dy, ca, sa, cb, sb; } xform_t;

/* surface_transform_of: 0 when the table is coaxial or the surface's four values are 0 */
static int transform_of(const table_t* sys, int s, xform_t* t) {
    if (sys->xf == NULL) return 0;
    const double* v = sys->xf + (size_t)s * 4;
#define MKO_ZERO(x) (!((x) > 0.0) && !((x) < 0.0))
    if (MKO_ZERO(v[0]) && MKO_ZERO(v[1]) && MKO_ZERO(v[2]) && MKO_ZERO(v[3])) return 0;
#undef MKO_ZERO
    t->dx = v[0];
    t->dy = v[1];
    t->ca = cos(v[2]);
    t->sa = sin(v[2]);
    t->cb = cos(v[3]);
    t->sb = sin(v[3]);
    return 1;
}

static vec3 rotate_to_surface(const xform_t* t, vec3 v) {
    const double x = t->cb * v.x - t->sb * v.z;
    const double z = t->sb * v.x + t->cb * v.z;
    vec3 r = {x, t->ca * v.y + t->sa * z, t->ca * z - t->sa * v.y};
    return r;
}

static vec3 rotate_from_surface(const xform_t* t, vec3 v) {
    const double y = t->ca * v.y - t->sa * v.z;
    const double z = t->sa * v.y + t->ca * v.z;
    vec3 r = {t->cb * v.x + t->sb * z, y, t->cb * z - t->sb * v.x};
    return r;
}

static vec3 point_to_surface(const xform_t* t, vec3 p) {
    vec3 q = {p.x - t->dx, p.y - t->dy, p.z};
    return rotate_to_surface(t, q);
}

static vec3 point_from_surface(const xform_t* t, vec3 q) {
    const vec3 p = rotate_from_surface(t, q);
    vec3 r = {p.x + t->dx, p.y + t->dy, p.z};
    return r;
}

/* propagate_surface with a transform (trace/trace.hpp:233) */
static int propagate_surface_xf(ray_t* ray, double t, int kind, double c, double n_before,
                                double n_after, soft_t* soft, unsigned char* branch,
                                const xform_t* xf, const ghost_t* ghost) {
    if (xf == NULL)
        return propagate_surface_g(ray, t, kind, c, n_before, n_after, soft, branch, ghost);
    if (!(ray->d.z > 0.0)) return ST_BACKWARD;
    ray->p.z -= t;
    ray->p = point_to_surface(xf, ray->p);
    ray->d = rotate_to_surface(xf, ray->d);
    const int st = propagate_surface_g(ray, 0.0, kind, c, n_before, n_after, soft, branch,
                                       ghost);
    if (st == ST_OK) {
        ray->p = point_from_surface(xf, ray->p);
        ray->d = rotate_from_surface(xf, ray->d);
    }
    return st;
}

/* Full per-surface record of a ray (AdjointRecord, trace/adjoint_record.hpp:66). */
typedef struct {
    int count;
    vec3 p[MKB_MAX_SURFACES];
    vec3 d[MKB_MAX_SURFACES];
    unsigned char branch[MKB_MAX_SURFACES];
    unsigned char image_branch;
} record_t;

/* trace_to_reference_sphere, reference_sphere.hpp:181 (with trace_ray_recorded,
 * trace.hpp:301, and trace_segment, trace.hpp:275). */
/* img (or NULL): the intersection (x, y) with the image plane thickness[S-1] behind the last
 * vertex (transfer_to_image_plane, trace.hpp:402, on a copy), for rays in the piston: the
 * transverse ray-error rows of this build (no reference counterpart). */
static int trace_to_reference_img(const table_t* sys, int l, ray_t* ray, vec3 center,
                                  soft_t* soft, record_t* rec, double* img) {
    const int S = sys->S, L = sys->L;
    if (rec) {
        rec->count = 1;
        rec->p[0] = ray->p;
        rec->d[0] = ray->d;
        rec->branch[0] = BR_REGULAR;
        rec->image_branch = BR_REGULAR;
    }
    int st = ST_OK;
    int ghost = 0; /* ghost plates passed (TraceProgress::ghost) */
    for (int s = 1; s < S; ++s) {
        const double n_before = sys->n[(s - 1) * L + l];
        const double n_after = sys->n[s * L + l];
        unsigned char branch = BR_REGULAR;
        xform_t xf;
        const int moved = transform_of(sys, s, &xf);
        ghost_t gp;
        const int plate = sys->type[s] == MKB_SURFACE_GHOST_PLATE && ghost < sys->G;
        if (plate) gp = ghost_of(sys, ghost, l);
        st = propagate_surface_xf(ray, sys->t[s - 1], sys->type[s], sys->c[s], n_before, n_after,
                                  soft, &branch, moved ? &xf : NULL, plate ? &gp : NULL);
        if (st != ST_OK) break;
        if (sys->type[s] == MKB_SURFACE_GHOST_PLATE) ++ghost;
        if (rec) {
            rec->count = s + 1;
            rec->p[s] = ray->p;
            rec->d[s] = ray->d;
            rec->branch[s] = branch;
        }
    }
    if (st == ST_OK && soft != NULL) st = soft->first;
    if (is_hard(st)) return st;
    if (!(ray->d.z > 0.0)) return ST_BACKWARD;
    if (img) {
        ray_t copy = *ray;
        transfer_to_tangent_plane(&copy, sys->t[S - 1]);
        img[0] = copy.p.x;
        img[1] = copy.p.y;
    }
    const double n_image = sys->n[(S - 1) * L + l];
    double s_ref = 0.0;
    const int rst = reference_sphere_step(ray, center, n_image, &s_ref, soft);
    if (is_hard(rst)) return rst;
    if (rec) rec->image_branch = rst == ST_SOFT_MISSED ? BR_SOFT_MISSED : BR_REGULAR;
    if (st != ST_OK) return st;
    return rst;
}

static int trace_to_reference(const table_t* sys, int l, ray_t* ray, vec3 center, soft_t* soft,
                              record_t* rec) {
    return trace_to_reference_img(sys, l, ray, center, soft, rec, NULL);
}

/* ---- pupil samples: pupil/quadrature.hpp:71,103,112 ------------------------------------ */
typedef struct { double rho, phi, weight; } sample_t;

static int field_samples(const mkb_residual_plan* plan, int f) {
    return plan->pupil_mode[f] == MKB_PUPIL_AXIS ? plan->rings : plan->rings * plan->spokes;
}

static sample_t pupil_sample(const mkb_residual_plan* plan, int f, int index) {
    const double pi = 3.14159265358979323846264338327950288;
    const int mode = plan->pupil_mode[f];
    const int spokes = mode == MKB_PUPIL_AXIS ? 1 : plan->spokes;
    const int i = index / spokes;
    const int j = index - i * spokes;
    sample_t s;
    s.rho = sqrt(plan->quad_u[i]);
    s.weight = plan->quad_w[i] / (double)spokes;
    if (mode == MKB_PUPIL_HALF) s.phi = (double)(2 * j + 1) * pi / (double)(2 * spokes);
    else if (mode == MKB_PUPIL_FULL) s.phi = (double)(2 * j + 1) * pi / (double)spokes;
    else s.phi = 0.0;
    return s;
}

/* collimated_ray, trace/trace.hpp:109 */
static ray_t collimated_ray(double a, double theta, double rho, double phi) {
    const double r = a * rho;
    ray_t ray;
    ray.p.x = r * sin(phi);
    ray.p.y = r * cos(phi);
    ray.p.z = 0.0;
    ray.d.x = 0.0;
    ray.d.y = sin(theta);
    ray.d.z = cos(theta);
    ray.opl = v_dot(ray.p, ray.d);
    return ray;
}

/* ---- weights: merit/ray_residual.hpp:98-202 --------------------------------------------- */
static double tuple_weight(const mkb_residual_plan* plan, int f, int l) {
    const double wf = plan->field_weight[f];
    const double wl = plan->wavelength_weight[l];
    if (!(wf > 0.0) || !(wl > 0.0)) return 0.0;
    double sum_f = 0.0, sum_l = 0.0;
    for (int i = 0; i < plan->fields; ++i) sum_f += plan->field_weight[i];
    for (int i = 0; i < plan->wavelengths; ++i) sum_l += plan->wavelength_weight[i];
    return (wf / sum_f) * (wl / sum_l);
}

static double residual_scale(const mkb_residual_plan* plan, int f, int l) {
    const double w = tuple_weight(plan, f, l);
    if (!(w > 0.0)) return 0.0;
    const double lambda_ref_mm = plan->reference_wavelength_nm * 1e-6;
    return sqrt(w) / lambda_ref_mm;
}

static double penalty_scale(const mkb_residual_plan* plan, int f, int l) {
    const double w = tuple_weight(plan, f, l);
    if (!(w > 0.0)) return 0.0;
    return sqrt(plan->fail_weight * w);
}

static double failure_penalty(int st, double soft_penalty) {
    if (st == ST_OK) return 0.0;
    if (is_soft(st)) return soft_penalty;
    return soft_penalty + 1.0;  /* kHardFailurePenalty, ray_residual.hpp:170 */
}

/* ---- layout: src/batch/batch_residuals.cpp:25 ------------------------------------------- */
int mko_port_aim(const mkb_batch_view* v, double* pupil, double* thickness0) {
    if (v == NULL || pupil == NULL || thickness0 == NULL) return -1;
    const int S = v->surfaces, L = v->wavelengths;
    int stop = 0;
    for (int s = 1; s < S; ++s)
        if (v->type[s] == 4) stop = s; /* MKB_SURFACE_APERTURE_STOP */
    if (stop == 0) return -1;
    for (int i = 0; i < v->variants; ++i) {
        const double* c = v->curvature + (size_t)i * S;
        const double* t = v->thickness + (size_t)i * S;
        const double* n_of = v->index + (size_t)i * S * L; /* column 0: n_of[s * L] */
        double y1 = 1.0, u1 = 0.0, y2 = 0.0, u2 = 1.0, n = n_of[0];
        for (int s = 1; s < stop; ++s) {
            const double n2 = n_of[(size_t)s * L];
            const double cs = v->type[s] == 2 ? c[s] : 0.0; /* spheres only */
            const double phi = cs * (n2 - n);
            u1 = (n * u1 - y1 * phi) / n2;
            u2 = (n * u2 - y2 * phi) / n2;
            y1 = y1 + t[s] * u1;
            y2 = y2 + t[s] * u2;
            n = n2;
        }
        pupil[i] = c[stop] / (y1 < 0.0 ? -y1 : y1);
        thickness0[i] = -(y2 / y1);
    }
    return 0;
}

int64_t mko_port_rays_per_variant(const mkb_residual_plan* plan) {
    int64_t off = 0;
    for (int f = 0; f < plan->fields; ++f) off += (int64_t)plan->wavelengths * field_samples(plan, f);
    return off;
}

static int64_t tuple_offset(const mkb_residual_plan* plan, int f, int l) {
    int64_t off = 0;
    for (int i = 0; i < f; ++i) off += (int64_t)plan->wavelengths * field_samples(plan, i);
    return off + (int64_t)l * field_samples(plan, f);
}

static int check_plan(const mkb_batch_view* v, const mkb_residual_plan* plan) {
    if (!v || !plan || v->surfaces < 2 || v->surfaces > MKB_MAX_SURFACES || v->wavelengths < 1 ||
        v->fields < 1 || plan->fields != v->fields || plan->wavelengths != v->wavelengths ||
        plan->rings < 1 || plan->rings > MKB_MAX_RINGS || plan->spokes < 1)
        return -1;
    return 0;
}

static table_t table_of(const mkb_batch_view* v, int var) {
    table_t t;
    t.S = v->surfaces;
    t.L = v->wavelengths;
    t.type = v->type;
    t.c = v->curvature + (size_t)var * v->surfaces;
    t.t = v->thickness + (size_t)var * v->surfaces;
    t.n = v->index + (size_t)var * v->surfaces * v->wavelengths;
    t.xf = v->decenter_tilt != NULL ? v->decenter_tilt + (size_t)var * v->surfaces * 4 : NULL;
    t.G = v->ghost_plates;
    t.K = v->ghost_terms;
    t.gcoeff = t.G > 0 ? v->ghost_coeff + (size_t)var * t.G * t.K : NULL;
    t.gradius = t.G > 0 ? v->ghost_norm_radius : NULL;
    t.gindex = t.G > 0 ? v->ghost_index + (size_t)var * t.G * t.L : NULL;
    return t;
}

/* variant_residuals, src/batch/batch_residuals.cpp:177 (with opd_statistics,
 * merit/opd.hpp:37). `table` may differ from the view's variant `v` (FD variants). */
static void variant_residuals(const mkb_batch_view* view, const table_t* table, int v,
                              const mkb_residual_plan* plan, double* residuals, double* opd,
                              uint8_t* status) {
    const int soft_mode = plan->failure == MKB_FAILURE_SOFT;
    const int64_t rays = mko_port_rays_per_variant(plan);
    const int S = table->S;
    double opl[MKB_MAX_RINGS * MKB_MAX_SPOKES];
    double penalty[MKB_MAX_RINGS * MKB_MAX_SPOKES];
    double img[MKB_MAX_RINGS * MKB_MAX_SPOKES][2];
    const int transverse = plan->transverse_weight > 0.0;
    int st[MKB_MAX_RINGS * MKB_MAX_SPOKES];
    sample_t pupil[MKB_MAX_RINGS * MKB_MAX_SPOKES];
    for (int f = 0; f < plan->fields; ++f) {
        const int n = field_samples(plan, f);
        for (int k = 0; k < n; ++k) pupil[k] = pupil_sample(plan, f, k);
        const vec3 center = {0.0, view->field_target[(size_t)v * view->fields + f], table->t[S - 1]};
        const double a = view->pupil_radius[v];
        const double theta = view->field_angle[(size_t)v * view->fields + f];
        for (int l = 0; l < plan->wavelengths; ++l) {
            const int64_t o = tuple_offset(plan, f, l);
            for (int k = 0; k < n; ++k) {
                soft_t soft = {0.0, ST_OK};
                ray_t ray = collimated_ray(a, theta, pupil[k].rho, pupil[k].phi);
                img[k][0] = img[k][1] = 0.0;
                st[k] = trace_to_reference_img(table, l, &ray, center, soft_mode ? &soft : NULL,
                                               NULL, transverse ? img[k] : NULL);
                opl[k] = ray.opl;
                penalty[k] = soft.penalty;
            }
            /* opd_statistics */
            double valid = 0.0, sum = 0.0;
            for (int k = 0; k < n; ++k)
                if (in_piston(st[k])) {
                    valid += pupil[k].weight;
                    sum += pupil[k].weight * opl[k];
                }
            double* e = opd + o;
            if (!(valid > 0.0)) {
                for (int k = 0; k < n; ++k) e[k] = 0.0;
            } else {
                const double piston = sum / valid;
                for (int k = 0; k < n; ++k) e[k] = in_piston(st[k]) ? opl[k] - piston : 0.0;
            }
            const double scale = residual_scale(plan, f, l);
            for (int k = 0; k < n; ++k) {
                residuals[o + k] = scale * sqrt(pupil[k].weight) * e[k];
                status[o + k] = (uint8_t)st[k];
            }
            if (soft_mode) {
                const double pscale = penalty_scale(plan, f, l);
                for (int k = 0; k < n; ++k)
                    residuals[rays + o + k] =
                        pscale * sqrt(pupil[k].weight) * failure_penalty(st[k], penalty[k]);
            }
            if (transverse) { /* transverse ray errors after the ray and penalty rows */
                const double w = tuple_weight(plan, f, l);
                const double ts = w > 0.0 ? sqrt(plan->transverse_weight * w) : 0.0;
                const int64_t base = rays * (soft_mode ? 2 : 1);
                for (int k = 0; k < n; ++k) {
                    const int in = in_piston(st[k]);
                    const double ex = in ? img[k][0] - 0.0 : 0.0;
                    const double ey = in ? img[k][1] - center.y : 0.0;
                    residuals[base + o + k] = ts * sqrt(pupil[k].weight) * ex;
                    residuals[base + rays + o + k] = ts * sqrt(pupil[k].weight) * ey;
                }
            }
        }
    }
}

typedef struct {
    const mkb_batch_view* view;
    const mkb_residual_plan* plan;
    double* residuals;
    double* opd;
    uint8_t* status;
    int64_t rays, rows;
} res_ctx_t;

static void residuals_item(void* p, int v) {
    const res_ctx_t* c = (const res_ctx_t*)p;
    double* e = (double*)malloc(sizeof(double) * c->rays);
    uint8_t* s = (uint8_t*)malloc(c->rays);
    const table_t table = table_of(c->view, v);
    variant_residuals(c->view, &table, v, c->plan, c->residuals + v * c->rows, e, s);
    if (c->opd) memcpy(c->opd + v * c->rays, e, sizeof(double) * c->rays);
    if (c->status) memcpy(c->status + v * c->rays, s, c->rays);
    free(e);
    free(s);
}

int mko_port_residuals(const mkb_batch_view* view, const mkb_residual_plan* plan,
                       double* residuals, double* opd, uint8_t* status, int threads) {
    if (check_plan(view, plan)) return -1;
    const int64_t rays = mko_port_rays_per_variant(plan);
    const int64_t rows = rays * (1 + (plan->failure == MKB_FAILURE_SOFT) +
                                 2 * (plan->transverse_weight > 0.0));
    res_ctx_t ctx = {view, plan, residuals, opd, status, rays, rows};
    parallel_for(view->variants, threads, residuals_item, &ctx);
    return 0;
}

/* variant_merit, src/batch/batch_merit.cpp:12 */
typedef struct {
    const mkb_batch_view* view;
    const mkb_residual_plan* plan;
    double* merit;
    int64_t* failed;
    int64_t* hard_failed;
} merit_ctx_t;

static void merit_item(void* pctx, int v) {
    const merit_ctx_t* c = (const merit_ctx_t*)pctx;
    const mkb_batch_view* view = c->view;
    const mkb_residual_plan* plan = c->plan;
    double* merit = c->merit;
    int64_t* failed = c->failed;
    int64_t* hard_failed = c->hard_failed;
    const int64_t rays = mko_port_rays_per_variant(plan);
    const int soft_mode = plan->failure == MKB_FAILURE_SOFT;
    const int transverse = plan->transverse_weight > 0.0;
    const int64_t rows = rays * (1 + soft_mode + 2 * transverse);
    double* r = (double*)malloc(sizeof(double) * rows);
    double* e = (double*)malloc(sizeof(double) * rays);
    uint8_t* s = (uint8_t*)malloc(rays);
    const table_t table = table_of(view, v);
    variant_residuals(view, &table, v, plan, r, e, s);
    double sum = 0.0;
    for (int f = 0; f < plan->fields; ++f)
        for (int l = 0; l < plan->wavelengths; ++l) {
            const int64_t o = tuple_offset(plan, f, l);
            const int n = field_samples(plan, f);
            double tuple = 0.0;
            for (int k = 0; k < n; ++k) tuple += r[o + k] * r[o + k];
            if (soft_mode) {
                double pen = 0.0;
                for (int k = 0; k < n; ++k) pen += r[rays + o + k] * r[rays + o + k];
                tuple += pen;
            }
            if (transverse) { /* sum_k r_x^2, then sum_k r_y^2 */
                const int64_t base = rays * (1 + soft_mode);
                double tx = 0.0, ty = 0.0;
                for (int k = 0; k < n; ++k) tx += r[base + o + k] * r[base + o + k];
                for (int k = 0; k < n; ++k) ty += r[base + rays + o + k] * r[base + rays + o + k];
                tuple += tx;
                tuple += ty;
            }
            sum += tuple;
        }
    int64_t nf = 0, nh = 0;
    for (int64_t k = 0; k < rays; ++k) {
        nf += s[k] != ST_OK;
        nh += is_hard(s[k]);
    }
    merit[v] = sum;
    failed[v] = nf;
    hard_failed[v] = nh;
    free(r);
    free(e);
    free(s);
}

int mko_port_merit(const mkb_batch_view* view, const mkb_residual_plan* plan, double* merit,
                   int64_t* failed, int64_t* hard_failed, int threads) {
    if (check_plan(view, plan)) return -1;
    merit_ctx_t ctx = {view, plan, merit, failed, hard_failed};
    parallel_for(view->variants, threads, merit_item, &ctx);
    return 0;
}

/* ---- variables: VariableSet::apply (src/optim/variable_set.cpp:237) ---------------------- */
static int check_vars(const mkb_batch_view* v, const mkb_variables* vars) {
    if (!vars || vars->count < 1 || vars->count > MKB_MAX_VARIABLES) return -1;
    for (int k = 0; k < vars->count; ++k) {
        if (vars->type[k] == MKB_VAR_GHOST_COEFFICIENT) {
            if (!vars->ghost_plate || !vars->ghost_order || vars->ghost_plate[k] < 0 ||
                vars->ghost_plate[k] >= v->ghost_plates || vars->ghost_order[k] < 1 ||
                vars->ghost_order[k] > v->ghost_terms)
                return -1;
        } else if (vars->surface[k] < 0 || vars->surface[k] >= v->surfaces) {
            return -1;
        }
    }
    return 0;
}

/* Copy of variant `src` of the view with x applied (curvature / thickness / ghost coefficient
 * entries; VariableSet::apply, src/optim/variable_set.cpp:237). */
typedef struct {
    double c[MKB_MAX_SURFACES], t[MKB_MAX_SURFACES];
    double g[MKB_MAX_GHOST_PLATES * MKB_MAX_GHOST_TERMS];
    double n[MKB_MAX_SURFACES * MKB_MAX_WAVELENGTHS];  /* index, rewritten by glass variables */
    double b[MKB_MAX_SURFACES * 4];                      /* Buchdahl coefficients */
} params_t;

/* buchdahl_omega, glass/dispersion.hpp:87 (nm_to_um divides by 1000) */
static double buchdahl_omega_nm(double nm) {
    const double dl = nm / 1000.0 - 0.546074;
    return dl / (1.0 + 2.5 * dl);
}

static void apply_x(const mkb_batch_view* view, int src, const mkb_variables* vars,
                    const double* x, params_t* out) {
    const int S = view->surfaces, GK = view->ghost_plates * view->ghost_terms;
    memcpy(out->c, view->curvature + (size_t)src * S, sizeof(double) * S);
    memcpy(out->t, view->thickness + (size_t)src * S, sizeof(double) * S);
    if (GK > 0) memcpy(out->g, view->ghost_coeff + (size_t)src * GK, sizeof(double) * GK);
    const int L = view->wavelengths;
    memcpy(out->n, view->index + (size_t)src * S * L, sizeof(double) * S * L);
    if (view->buchdahl_coeff)
        memcpy(out->b, view->buchdahl_coeff + (size_t)src * S * 4, sizeof(double) * S * 4);
    int glass_surface[MKB_MAX_SURFACES] = {0};
    for (int k = 0; k < vars->count; ++k) {
        if (vars->type[k] == MKB_VAR_CURVATURE) out->c[vars->surface[k]] = x[k];
        else if (vars->type[k] == MKB_VAR_GHOST_COEFFICIENT)
            out->g[vars->ghost_plate[k] * view->ghost_terms + vars->ghost_order[k] - 1] = x[k];
        else if (vars->type[k] == MKB_VAR_GLASS) {
            out->b[vars->surface[k] * 4 + vars->glass_component[k]] = x[k];
            glass_surface[vars->surface[k]] = 1;
        } else out->t[vars->surface[k]] = x[k];
    }
    /* the media of the glass variables: n = n0 + w (nu1 + w (nu2 + w nu3)) (VariableSet::apply,
       src/optim/variable_set.cpp:268, buchdahl_index, glass/dispersion.hpp:93) */
    for (int s = 0; s < S; ++s) {
        if (!glass_surface[s]) continue;
        const double* b = out->b + s * 4;
        for (int l = 0; l < L; ++l) {
            const double w = buchdahl_omega_nm(view->wavelength_nm[l]);
            out->n[s * L + l] = b[0] + w * (b[1] + w * (b[2] + w * b[3]));
        }
    }
}

static table_t table_with(const mkb_batch_view* v, int var, const params_t* p) {
    table_t t = table_of(v, var);
    t.c = p->c;
    t.t = p->t;
    t.n = p->n;
    if (t.G > 0) t.gcoeff = p->g;
    return t;
}

/* ---- FD Jacobian --------------------------------------------------------------------------
 * fd_step and fd_pattern (src/optim/variant_generator.cpp:158,177), fd_derivative
 * (include/mikroptim/optim/fd_formula.hpp:40), fd_jacobian_from_residuals
 * (src/optim/fd_jacobian.cpp:80). */
static const double kFdStepFactor = 6.0554544523933395e-06;  /* variant_generator.hpp:92 */
enum { FD_CENTRAL = 0, FD_ONE_SIDED = 1, FD_TRUNCATED = 2 };

static double fd_derivative(int stencil, double r0, double ra, double rb, double da, double db) {
    if (stencil == FD_ONE_SIDED) {
        const double ga = ra - r0;
        const double gb = rb - r0;
        return (db * db * ga - da * da * gb) / (da * db * (db - da));
    }
    return (ra - rb) / (da - db);
}

static void fd_pattern(const mkb_variables* vars, const double* x0, double* xa, double* xb,
                       double* da, double* db, int* stencil) {
    for (int k = 0; k < vars->count; ++k) {
        const double x = x0[k];
        const double lo = vars->lower[k], up = vars->upper[k];
        const double ax = fabs(x);
        const double h = kFdStepFactor * (ax > vars->typical[k] ? ax : vars->typical[k]);
        const double plus = x + h, minus = x - h;
        int st = FD_CENTRAL;
        double a, b;
        if (plus <= up && minus >= lo) {
            a = plus;
            b = minus;
        } else {
            const int towards_upper = up - x >= x - lo;
            const double far = towards_upper ? x + 2.0 * h : x - 2.0 * h;
            if (towards_upper ? far <= up : far >= lo) {
                st = FD_ONE_SIDED;
                a = towards_upper ? plus : minus;
                b = far;
            } else {
                st = FD_TRUNCATED;
                a = plus <= up ? plus : up;
                b = minus >= lo ? minus : lo;
            }
        }
        stencil[k] = st;
        xa[k] = a;
        xb[k] = b;
        da[k] = a - x;
        db[k] = b - x;
    }
}

typedef struct {
    const mkb_batch_view* view;
    const mkb_residual_plan* plan;
    const mkb_variables* vars;
    const double* x0;
    double* J;
    double* r0;
    int64_t* status_changes;
    int P;
    int64_t rays;
    int64_t R;
} fd_ctx_t;

static void fd_item(void* pctx, int i) {
    const fd_ctx_t* cx = (const fd_ctx_t*)pctx;
    const mkb_batch_view* view = cx->view;
    const mkb_residual_plan* plan = cx->plan;
    const mkb_variables* vars = cx->vars;
    const double* x0 = cx->x0;
    double* J = cx->J;
    double* r0 = cx->r0;
    int64_t* status_changes = cx->status_changes;
    int P = cx->P;
    int64_t rays = cx->rays;
    int64_t R = cx->R;
    const int tmpl = view->variants == 1 ? 0 : i;
    const double* x = x0 + (size_t)i * P;
    double xa[MKB_MAX_VARIABLES], xb[MKB_MAX_VARIABLES], da[MKB_MAX_VARIABLES],
        db[MKB_MAX_VARIABLES], y[MKB_MAX_VARIABLES];
    int stencil[MKB_MAX_VARIABLES];
    fd_pattern(vars, x, xa, xb, da, db, stencil);
    double* res0 = (double*)malloc(sizeof(double) * R);
    double* resa = (double*)malloc(sizeof(double) * R);
    double* resb = (double*)malloc(sizeof(double) * R);
    double* e = (double*)malloc(sizeof(double) * rays);
    uint8_t* s0 = (uint8_t*)malloc(rays);
    uint8_t* sa = (uint8_t*)malloc(rays);
    uint8_t* sb = (uint8_t*)malloc(rays);
    params_t p;
    apply_x(view, tmpl, vars, x, &p);
    table_t t = table_with(view, tmpl, &p);
    variant_residuals(view, &t, tmpl, plan, res0, e, s0);
    memcpy(r0 + (size_t)i * R, res0, sizeof(double) * R);
    memcpy(y, x, sizeof(double) * P);
    for (int k = 0; k < P; ++k) {
        y[k] = xa[k];
        apply_x(view, tmpl, vars, y, &p);
        t = table_with(view, tmpl, &p);
        variant_residuals(view, &t, tmpl, plan, resa, e, sa);
        y[k] = xb[k];
        apply_x(view, tmpl, vars, y, &p);
        t = table_with(view, tmpl, &p);
        variant_residuals(view, &t, tmpl, plan, resb, e, sb);
        y[k] = x[k];
        double* col = J + ((size_t)i * P + k) * R;
        for (int64_t r = 0; r < R; ++r)
            col[r] = fd_derivative(stencil[k], res0[r], resa[r], resb[r], da[k], db[k]);
        if (status_changes) {
            int64_t changes = 0;
            for (int64_t r = 0; r < rays; ++r) {
                const int ok0 = s0[r] == ST_OK;
                if ((sa[r] == ST_OK) != ok0 || (sb[r] == ST_OK) != ok0) ++changes;
            }
            status_changes[(size_t)i * P + k] = changes;
        }
    }
    free(res0); free(resa); free(resb); free(e); free(s0); free(sa); free(sb);
}

int mko_port_fd_jacobian(const mkb_batch_view* view, const mkb_residual_plan* plan,
                         const mkb_variables* vars, const double* x0, int runs, double* J,
                         double* r0, int64_t* status_changes, int threads) {
    if (check_plan(view, plan) || check_vars(view, vars) || runs < 1 ||
        (view->variants != 1 && view->variants != runs))
        return -1;
    const int P = vars->count;
    const int64_t rays = mko_port_rays_per_variant(plan);
    const int64_t R = rays * (1 + (plan->failure == MKB_FAILURE_SOFT) +
                              2 * (plan->transverse_weight > 0.0));
    fd_ctx_t ctx = {view, plan, vars, x0, J, r0, status_changes, P, rays, R};
    parallel_for(runs, threads, fd_item, &ctx);
    return 0;
}

/* ---- adjoint ------------------------------------------------------------------------------
 * refracting_step_backward (trace/adjoint_backward.hpp:118), reference_step_backward
 * (adjoint_backward.hpp:376), backward_ray (adjoint_backward.hpp:495), JacobianRowWriter and
 * ray_gradient_rows (merit/ray_jacobian.hpp:50,92), projection (src/optim/adjoint_jacobian.cpp:449). */
typedef struct { vec3 p, d; } radj_t;
typedef struct { double thickness, curvature, n_before, n_after; } sadj_t;

static void refracting_step_backward(vec3 p, vec3 d, double t, double c, double n_before,
                                     double n_after, unsigned char branch, double seed_opl,
                                     double seed_pen, radj_t* adj, sadj_t* out) {
    /* forward recompute (transfer_local, adjoint_backward.hpp:78) */
    const double z = p.z - t;
    const double s0 = -z / d.z;
    const double x = p.x + s0 * d.x;
    const double y = p.y + s0 * d.y;
    const double rr = x * x + y * y;
    const double H = c * rr;
    const double xd = x * d.x + y * d.y;
    const double B = d.z - c * xd;
    const double D = B * B - c * H;
    const int missed = (branch & BR_SOFT_MISSED) != 0;
    const int tir = (branch & BR_SOFT_TIR) != 0;
    double root_d = 0.0, s;
    if (missed) s = B / c;
    else {
        root_d = sqrt(D);
        s = H / (B + root_d);
    }
    const vec3 q = {x + s * d.x, y + s * d.y, s * d.z};
    const vec3 n_raw = {-c * q.x, -c * q.y, 1.0 - c * q.z};
    double inv_norm = 1.0;
    vec3 N = n_raw;
    if (missed) {
        inv_norm = 1.0 / v_norm(n_raw);
        N = v_scale(inv_norm, n_raw);
    }
    const double mu = n_before / n_after;
    const double cos_i = v_dot(d, N);
    const double sin2 = 1.0 - cos_i * cos_i;
    const double k = 1.0 - mu * mu * sin2;
    /* reverse */
    const vec3 qb_out = adj->p;
    const vec3 d1b = adj->d;
    radj_t in = {v_zero(), v_zero()};
    vec3 nb = v_zero();
    double cosb = 0.0, kb = 0.0, mub = 0.0;
    if (tir) {
        const vec3 tau = v_sub(d, v_scale(cos_i, N));
        const double inv_tau = 1.0 / v_norm(tau);
        const vec3 d1 = v_scale(inv_tau, tau);
        const vec3 taub = v_scale(inv_tau, v_sub(d1b, v_scale(v_dot(d1, d1b), d1)));
        in.d = v_add(in.d, taub);
        cosb += -v_dot(taub, N);
        nb = v_add(nb, v_scale(-cos_i, taub));
        kb += -seed_pen;
    } else {
        const double root_k = sqrt(k);
        const double a = root_k - mu * cos_i;
        in.d = v_add(in.d, v_scale(mu, d1b));
        nb = v_add(nb, v_scale(a, d1b));
        const double ab = v_dot(d1b, N);
        mub += v_dot(d1b, d);
        kb += ab / (2.0 * root_k);
        mub += -ab * cos_i;
        cosb += -ab * mu;
    }
    mub += -kb * 2.0 * mu * sin2;
    cosb += kb * 2.0 * mu * mu * cos_i;
    in.d = v_add(in.d, v_scale(cosb, N));
    nb = v_add(nb, v_scale(cosb, d));
    out->n_before += mub / n_after;
    out->n_after += -mub * mu / n_after;
    vec3 nrb = nb;
    if (missed) nrb = v_scale(inv_norm, v_sub(nb, v_scale(v_dot(N, nb), N)));
    const vec3 qb = v_add(qb_out, v_scale(-c, nrb));
    double cb = -v_dot(q, nrb);
    double xb = qb.x, yb = qb.y;
    double sb = v_dot(qb, d);
    in.d = v_add(in.d, v_scale(s, qb));
    sb += seed_opl * n_before;
    double s0b = seed_opl * n_before;
    out->n_before += seed_opl * (s0 + s);
    double hb = 0.0, bb = 0.0;
    if (missed) {
        bb += sb / c;
        cb += -sb * s / c;
        const double db = -seed_pen;
        bb += db * 2.0 * B;
        cb += -db * H;
        hb += -db * c;
    } else {
        const double inv = 1.0 / (2.0 * root_d);
        hb += sb * inv;
        bb += -sb * s * 2.0 * inv;
        cb += sb * s * s * inv;
    }
    cb += hb * rr;
    xb += hb * 2.0 * c * x;
    yb += hb * 2.0 * c * y;
    in.d.z += bb;
    cb += -bb * xd;
    xb += -bb * c * d.x;
    yb += -bb * c * d.y;
    in.d.x += -bb * c * x;
    in.d.y += -bb * c * y;
    /* transfer_backward, adjoint_backward.hpp:91 */
    in.p.x += xb;
    in.p.y += yb;
    s0b += xb * d.x + yb * d.y;
    in.d.x += xb * s0;
    in.d.y += yb * s0;
    const double qq = s0b / d.z;
    out->thickness += qq;
    in.p.z += -qq;
    in.d.z += -qq * s0;
    out->curvature += cb;
    *adj = in;
}

static void reference_step_backward(vec3 p, vec3 d, vec3 center, double n_image,
                                    unsigned char branch, double seed_opl, double seed_pen,
                                    radj_t* adj, vec3* center_adj, double* n_image_adj) {
    const vec3 q = v_sub(p, center);
    const double b = -v_dot(q, d);
    const double g = v_dot(p, v_sub(p, v_scale(2.0, center)));
    const double disc = b * b - g;
    const int missed = (branch & BR_SOFT_MISSED) != 0;
    const double sigma = center.z >= 0.0 ? 1.0 : -1.0;
    double s, root = 0.0;
    if (missed) s = b;
    else {
        root = sqrt(disc);
        s = g / (b + sigma * root);
    }
    const double sb = seed_opl * n_image;
    *n_image_adj += seed_opl * s;
    double bb, gb;
    if (missed) {
        bb = sb;
        gb = 0.0;
        const double radius_sq = v_dot(center, center);
        const double discb = -seed_pen / radius_sq;
        bb += discb * 2.0 * b;
        gb += -discb;
        *center_adj = v_add(*center_adj,
                            v_scale(seed_pen * 2.0 * disc / (radius_sq * radius_sq), center));
    } else {
        gb = sb * sigma / (2.0 * root);
        bb = -sb * sigma * s / root;
    }
    radj_t in = {v_zero(), v_zero()};
    in.p = v_add(in.p, v_scale(-bb, d));
    in.d = v_add(in.d, v_scale(-bb, q));
    *center_adj = v_add(*center_adj, v_scale(bb, d));
    in.p = v_add(in.p, v_scale(2.0 * gb, v_sub(p, center)));
    *center_adj = v_add(*center_adj, v_scale(-2.0 * gb, p));
    *adj = in;
}

/* ghost_step_backward, trace/adjoint_backward.hpp:253: writes the adjoint of a_{k+1} of the
 * plate into w->ghost[g0 + k] (see w_write below; declared here, defined after the writer). */
typedef struct writer_s writer_t;
static void w_write(const writer_t* w, int p, double value);
static void ghost_step_backward(vec3 p, vec3 d, double t, const ghost_t* g, double n_before,
                                double n_after, unsigned char branch, double seed_opl,
                                double seed_pen, radj_t* adj, sadj_t* out, const writer_t* w,
                                const int* coeff_cols) {
    /* forward */
    const double z = p.z - t;
    const double s0 = -z / d.z;
    const double x = p.x + s0 * d.x;
    const double y = p.y + s0 * d.y;
    const double inv_r2 = 1.0 / (g->norm_radius * g->norm_radius);
    const double u = (x * x + y * y) * inv_r2;
    const double xi = 2.0 * u - 1.0;
    double prof_t = 0.0, sum_dp = 0.0, sum_ddp = 0.0;
    {
        double p_prev = 1.0, p_cur = xi, dp_prev = 0.0, dp_cur = 1.0, ddp_prev = 0.0,
               ddp_cur = 0.0;
        for (int k = 1; k <= g->terms; ++k) {
            const double a = g->coeff[k - 1];
            prof_t += a * p_cur;
            sum_dp += a * dp_cur;
            sum_ddp += a * ddp_cur;
            const double p_next = ((double)(2 * k + 1) * xi * p_cur - (double)k * p_prev) /
                                  (double)(k + 1);
            const double dp_next = dp_prev + (double)(2 * k + 1) * p_cur;
            const double ddp_next = ddp_prev + (double)(2 * k + 1) * dp_cur;
            p_prev = p_cur;
            p_cur = p_next;
            dp_prev = dp_cur;
            dp_cur = dp_next;
            ddp_prev = ddp_cur;
            ddp_cur = ddp_next;
        }
    }
    const double dt_du = 2.0 * sum_dp;
    const double d2t_du2 = 4.0 * sum_ddp;
    const double dn = g->n_glass - n_before;
    const double radial = dn * dt_du * 2.0 * inv_r2;
    const double dx = (n_before * d.x + radial * x) / n_after;
    const double dy = (n_before * d.y + radial * y) / n_after;
    const double radicand = 1.0 - dx * dx - dy * dy;
    const int tir = (branch & BR_SOFT_TIR) != 0;
    /* reverse */
    const vec3 qb = adj->p, d1b = adj->d;
    radj_t in = {v_zero(), v_zero()};
    double dxb, dyb, radb;
    if (tir) {
        const double inv_m = 1.0 / sqrt(dx * dx + dy * dy);
        const double ex = dx * inv_m, ey = dy * inv_m;
        const double proj = ex * d1b.x + ey * d1b.y;
        dxb = (d1b.x - proj * ex) * inv_m;
        dyb = (d1b.y - proj * ey) * inv_m;
        radb = -seed_pen;
    } else {
        dxb = d1b.x;
        dyb = d1b.y;
        radb = d1b.z / (2.0 * sqrt(radicand));
    }
    dxb += -2.0 * dx * radb;
    dyb += -2.0 * dy * radb;
    in.d.x += dxb * n_before / n_after;
    in.d.y += dyb * n_before / n_after;
    out->n_before += (dxb * d.x + dyb * d.y) / n_after;
    out->n_after += -(dxb * dx + dyb * dy) / n_after;
    const double gxb = dxb / n_after, gyb = dyb / n_after;
    const double radialb = gxb * x + gyb * y;
    double xb = qb.x + gxb * radial;
    double yb = qb.y + gyb * radial;
    double s0b = seed_opl * n_before;
    out->n_before += seed_opl * s0;
    const double phaseb = seed_opl;
    const double dnb = phaseb * prof_t + radialb * dt_du * 2.0 * inv_r2;
    const double tb = phaseb * dn;
    const double dtdub = radialb * dn * 2.0 * inv_r2;
    out->n_before += -dnb;
    const double ub = tb * dt_du + dtdub * d2t_du2;
    {
        double p_prev = 1.0, p_cur = xi, dp_prev = 0.0, dp_cur = 1.0;
        for (int k = 1; k <= g->terms; ++k) {
            w_write(w, coeff_cols[k - 1], tb * p_cur + dtdub * 2.0 * dp_cur);
            const double p_next = ((double)(2 * k + 1) * xi * p_cur - (double)k * p_prev) /
                                  (double)(k + 1);
            const double dp_next = dp_prev + (double)(2 * k + 1) * p_cur;
            p_prev = p_cur;
            p_cur = p_next;
            dp_prev = dp_cur;
            dp_cur = dp_next;
        }
    }
    xb += ub * 2.0 * x * inv_r2;
    yb += ub * 2.0 * y * inv_r2;
    /* transfer_backward, adjoint_backward.hpp:91 */
    in.p.x += xb;
    in.p.y += yb;
    s0b += xb * d.x + yb * d.y;
    in.d.x += xb * s0;
    in.d.y += yb * s0;
    const double q = s0b / d.z;
    out->thickness += q;
    in.p.z += -q;
    in.d.z += -q * s0;
    *adj = in;
}

/* Row writer: column map per table parameter (AdjointParameterMap, ray_jacobian.hpp:28). */
struct writer_s {
    int curvature[MKB_MAX_SURFACES];
    int thickness[MKB_MAX_SURFACES];
    int ghost[MKB_MAX_GHOST_PLATES * MKB_MAX_GHOST_TERMS];  /* ghost_coeff[g][k] */
    int glass[MKB_MAX_SURFACES * 3];                       /* (n0, nu1, nu2) of medium s */
    double slope[MKB_MAX_WAVELENGTHS * 3];                 /* (1, w_l, w_l^2) */
    int wavelength;
    double* column0;
    int64_t rows, row;
    double factor;
};

static void w_write(const writer_t* w, int p, double value) {
    if (p >= 0) w->column0[(int64_t)p * w->rows + w->row] = w->factor * value;
}

/* AdjointRowWriter::index (merit/ray_jacobian.hpp:66): the index adjoint of medium s to the
 * glass columns with dn/d(n0, nu1, nu2) = (1, w, w^2) at the ray's wavelength */
static void w_index(const writer_t* w, int s, double value) {
    for (int c = 0; c < 3; ++c)
        if (w->glass[s * 3 + c] >= 0) w_write(w, w->glass[s * 3 + c], value * w->slope[w->wavelength * 3 + c]);
}

/* backward_ray, adjoint_backward.hpp:495 (coaxial, LastSurface reference, collimated). */
static void backward_ray(const table_t* sys, int l, const record_t* rec, int reached_image,
                         vec3 center, double seed_opl, double seed_pen, const writer_t* w) {
    const int S = sys->S, L = sys->L;
    const int count = rec->count;
    radj_t adj = {v_zero(), v_zero()};
    double n_carry = 0.0;
    unsigned char next_branch = BR_REGULAR;
    int ghost = 0; /* ghost plates among the surfaces 1 .. count - 1 */
    for (int j = 1; j < count; ++j)
        if (sys->type[j] == MKB_SURFACE_GHOST_PLATE) ++ghost;
    for (int s = count - 1; s >= 0; --s) {
        const vec3 p = rec->p[s], d = rec->d[s];
        if (s == count - 1) {
            if (reached_image && count == S) {
                vec3 center_adj = v_zero();
                double n_image_adj = 0.0;
                const double n_image = sys->n[(S - 1) * L + l];
                reference_step_backward(p, d, center, n_image, rec->image_branch, seed_opl,
                                        seed_pen, &adj, &center_adj, &n_image_adj);
                w_write(w, w->thickness[S - 1], center_adj.z);
                n_carry = n_image_adj;
            }
        } else {
            const int j = s + 1;
            const int kind = sys->type[j];
            const double t = sys->t[s];
            const double n_before = sys->n[s * L + l];
            const double n_after = sys->n[j * L + l];
            sadj_t par = {0.0, 0.0, 0.0, 0.0};
            const double c = kind == MKB_SURFACE_SPHERE ? sys->c[j] : 0.0;
            /* decentered / tilted surface: the step in its tilted frame, adjoints turned in
               with R^T and back with R, t-bar = -p-bar_z (adjoint_backward.hpp:539-569) */
            xform_t xf;
            const int moved = transform_of(sys, j, &xf);
            vec3 pl = p, dl = d;
            double tl = t;
            if (moved) {
                vec3 shifted = {p.x, p.y, p.z - t};
                pl = point_to_surface(&xf, shifted);
                dl = rotate_to_surface(&xf, d);
                tl = 0.0;
                adj.p = rotate_to_surface(&xf, adj.p);
                adj.d = rotate_to_surface(&xf, adj.d);
            }
            if (kind == MKB_SURFACE_GHOST_PLATE) {
                --ghost;
                const ghost_t gp = ghost_of(sys, ghost, l);
                ghost_step_backward(pl, dl, tl, &gp, n_before, n_after, next_branch, seed_opl,
                                    seed_pen, &adj, &par, w, w->ghost + ghost * sys->K);
            } else {
                refracting_step_backward(pl, dl, tl, c, n_before, n_after, next_branch, seed_opl,
                                         seed_pen, &adj, &par);
            }
            if (moved) {
                adj.p = rotate_from_surface(&xf, adj.p);
                adj.d = rotate_from_surface(&xf, adj.d);
                par.thickness = -adj.p.z;
            }
            if (kind == MKB_SURFACE_SPHERE) w_write(w, w->curvature[j], par.curvature);
            w_write(w, w->thickness[s], par.thickness);
            w_index(w, j, par.n_after + n_carry);
            n_carry = par.n_before;
        }
        next_branch = rec->branch[s];
    }
    w_index(w, 0, n_carry);
}

typedef struct {
    const mkb_batch_view* view;
    const mkb_residual_plan* plan;
    const mkb_variables* vars;
    const double* x0;
    double* J;
    double* r0;
    uint8_t* status;
    int P;
    int S;
    int soft_mode;
    int64_t rays;
    int64_t R;
} adj_ctx_t;

static void adjoint_item(void* pctx, int i) {
    const adj_ctx_t* cx = (const adj_ctx_t*)pctx;
    const mkb_batch_view* view = cx->view;
    const mkb_residual_plan* plan = cx->plan;
    const mkb_variables* vars = cx->vars;
    const double* x0 = cx->x0;
    double* J = cx->J;
    double* r0 = cx->r0;
    uint8_t* status = cx->status;
    int P = cx->P;
    int S = cx->S;
    int soft_mode = cx->soft_mode;
    int64_t rays = cx->rays;
    int64_t R = cx->R;
    const int tmpl = view->variants == 1 ? 0 : i;
    params_t par;
    apply_x(view, tmpl, vars, x0 + (size_t)i * P, &par);
    const table_t table = table_with(view, tmpl, &par);
    double* e = (double*)malloc(sizeof(double) * rays);
    uint8_t* st_all = (uint8_t*)malloc(rays);
    variant_residuals(view, &table, tmpl, plan, r0 + (size_t)i * R, e, st_all);
    if (status) memcpy(status + (size_t)i * rays, st_all, rays);
    writer_t w;
    for (int s = 0; s < S; ++s) w.curvature[s] = w.thickness[s] = -1;
    for (int g = 0; g < MKB_MAX_GHOST_PLATES * MKB_MAX_GHOST_TERMS; ++g) w.ghost[g] = -1;
    for (int k = 0; k < P; ++k) {
        if (vars->type[k] == MKB_VAR_CURVATURE) w.curvature[vars->surface[k]] = k;
        else if (vars->type[k] == MKB_VAR_GHOST_COEFFICIENT)
            w.ghost[vars->ghost_plate[k] * view->ghost_terms + vars->ghost_order[k] - 1] = k;
        else if (vars->type[k] != MKB_VAR_GLASS) w.thickness[vars->surface[k]] = k;
    }
    w.column0 = J + (size_t)i * P * R;
    w.rows = R;
    for (int g = 0; g < MKB_MAX_SURFACES * 3; ++g) w.glass[g] = -1;
    for (int k = 0; k < P; ++k)
        if (vars->type[k] == MKB_VAR_GLASS) w.glass[vars->surface[k] * 3 + vars->glass_component[k]] = k;
    for (int l = 0; l < view->wavelengths; ++l) {
        const double om = view->wavelength_nm ? buchdahl_omega_nm(view->wavelength_nm[l]) : 0.0;
        w.slope[l * 3 + 0] = 1.0;
        w.slope[l * 3 + 1] = om;
        w.slope[l * 3 + 2] = om * om;
    }
    record_t* rec = (record_t*)malloc(sizeof(record_t));
    double weight[MKB_MAX_RINGS * MKB_MAX_SPOKES], rootw[MKB_MAX_RINGS * MKB_MAX_SPOKES];
    unsigned char piston[MKB_MAX_RINGS * MKB_MAX_SPOKES];
    for (int f = 0; f < plan->fields; ++f) {
        const int n = field_samples(plan, f);
        const vec3 center = {0.0, view->field_target[(size_t)tmpl * view->fields + f],
                             table.t[S - 1]};
        const double a = view->pupil_radius[tmpl];
        const double theta = view->field_angle[(size_t)tmpl * view->fields + f];
        for (int l = 0; l < plan->wavelengths; ++l) {
            w.wavelength = l;
            const int64_t offset = tuple_offset(plan, f, l);
            const double scale = residual_scale(plan, f, l);
            const double pscale = soft_mode ? penalty_scale(plan, f, l) : 0.0;
            for (int k = 0; k < n; ++k) {
                const sample_t smp = pupil_sample(plan, f, k);
                soft_t soft = {0.0, ST_OK};
                ray_t ray = collimated_ray(a, theta, smp.rho, smp.phi);
                const int st = trace_to_reference(&table, l, &ray, center,
                                                  soft_mode ? &soft : NULL, rec);
                weight[k] = smp.weight;
                rootw[k] = sqrt(smp.weight);
                piston[k] = (unsigned char)in_piston(st);
                const int reached = in_piston(st);
                if (reached) {
                    w.row = offset + k;
                    w.factor = 1.0;
                    backward_ray(&table, l, rec, 1, center, 1.0, 0.0, &w);
                }
                if (soft_mode && soft.first != ST_OK) {
                    w.row = rays + offset + k;
                    w.factor = pscale * rootw[k];
                    backward_ray(&table, l, rec, reached, center, 0.0, 1.0, &w);
                }
            }
            double w_ok = 0.0;
            for (int k = 0; k < n; ++k)
                if (piston[k]) w_ok += weight[k];
            for (int p = 0; p < P; ++p) {
                double* col = w.column0 + (int64_t)p * R + offset;
                if (!(w_ok > 0.0)) {
                    for (int k = 0; k < n; ++k) col[k] = 0.0;
                    continue;
                }
                double sum = 0.0;
                for (int k = 0; k < n; ++k)
                    if (piston[k]) sum += weight[k] * col[k];
                const double mean = sum / w_ok;
                for (int k = 0; k < n; ++k)
                    col[k] = piston[k] ? scale * rootw[k] * (col[k] - mean) : 0.0;
            }
        }
    }
    free(rec);
    free(e);
    free(st_all);
}

int mko_port_adjoint_jacobian(const mkb_batch_view* view, const mkb_residual_plan* plan,
                              const mkb_variables* vars, const double* x0, int runs, double* J,
                              double* r0, uint8_t* status, int threads) {
    if (plan->transverse_weight > 0.0) return -1; /* transverse rows: FD only */
    if (check_plan(view, plan) || check_vars(view, vars) || runs < 1 ||
        (view->variants != 1 && view->variants != runs))
        return -1;
    const int P = vars->count;
    const int S = view->surfaces;
    const int soft_mode = plan->failure == MKB_FAILURE_SOFT;
    const int64_t rays = mko_port_rays_per_variant(plan);
    const int64_t R = soft_mode ? 2 * rays : rays;
    memset(J, 0, sizeof(double) * (size_t)runs * P * R);
    adj_ctx_t ctx = {view, plan, vars, x0, J, r0, status, P, S, soft_mode, rays, R};
    parallel_for(runs, threads, adjoint_item, &ctx);
    return 0;
}

/* normal_equations_host with gram_dot, include/mikroptim/optim/normal_equations.hpp:19,33 */
int mko_port_normal_equations(const double* J, const double* r, int P, int64_t R, double* A,
                              double* g) {
    if (P < 1 || R < 0) return -1;
    for (int q = 0; q < P; ++q) {
        const double* cq = J + (size_t)q * R;
        for (int p = 0; p <= q; ++p) {
            const double* cp = J + (size_t)p * R;
            double acc = 0.0;
            for (int64_t k = 0; k < R; ++k) acc = fma(cp[k], cq[k], acc);
            A[q * P + p] = acc;
            A[p * P + q] = acc;
        }
        double acc = 0.0;
        for (int64_t k = 0; k < R; ++k) acc = fma(cq[k], r[k], acc);
        g[q] = acc;
    }
    return 0;
}
