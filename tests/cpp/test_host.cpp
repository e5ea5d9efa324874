// Test driver of the C++ host layer (mikroptim_b200/host): traces, differentiates and
// optimises a small singlet batch through the reference-shaped C++ classes and checks every
// result against the oracle (oracle/liboracle.so, the C restatement of the reference CPU
// path) -- bit for bit in the FP64 mode. Exit status 0 when every check passes.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cuda_runtime.h>
#include <stdexcept>
#include <vector>

#include "mikroptim_b200.hpp"
#include "mko_oracle.h"

namespace {

int failures = 0, checks = 0;

#ifdef MKB_HAVE_REF
// the reference's own CPU build (oracle/_ref): paraxial constraints as extra rows
extern "C" int mko_ref_paraxial_residuals(const mkb_batch_view*, const mkb_residual_plan*, int,
                                          int, const int32_t*, const int32_t*, const double*,
                                          const double*, double*);
extern "C" int mko_ref_surface_extrema(const mkb_batch_view*, const mkb_residual_plan*,
                                       double*);
extern "C" int mko_ref_prefilter(const mkb_batch_view*, const mkb_residual_plan*,
                                 const mkb_prefilter_options*, const double*, double*, double*,
                                 int64_t*, int64_t*, int64_t*, double*, double*, uint8_t*,
                                 double*, int32_t*, int32_t*);
extern "C" int mko_ref_eval(const mkb_batch_view*, const mkb_residual_plan*, int, int, int, double,
                            int64_t*, double*, double*, double*, uint8_t*, double*, uint8_t*,
                            double*, double*);
extern "C" int mko_ref_psf(const mkb_batch_view*, const mkb_residual_plan*, int, int, int, double,
                           int, double, double, int*, int*, double*, double*, int*, double*,
                           double*, double*);
extern "C" int mko_ref_optimize_lm(const mkb_batch_view*, const mkb_residual_plan*,
                                   const mkb_variables*, const double*, int, int, int, int, int,
                                   double*, double*, int32_t*, int32_t*, int32_t*, double*, int,
                                   const int32_t*, const int32_t*, const double*,
                                   const double*, int, const int32_t*, const int32_t*,
                                   const double*, const double*);
#endif

void expect(bool ok, const char* what) {
    ++checks;
    if (!ok) {
        ++failures;
        std::printf("FAIL: %s\n", what);
    }
}

template <class T>
bool same_bits(const std::vector<T>& a, const std::vector<T>& b) {
    return a.size() == b.size() && std::memcmp(a.data(), b.data(), a.size() * sizeof(T)) == 0;
}

// equal values, NaN where the other holds NaN (payloads aside)
bool same_values(const std::vector<double>& a, const std::vector<double>& b) {
    if (a.size() != b.size()) return false;
    for (size_t i = 0; i < a.size(); ++i)
        if (!(std::isnan(a[i]) && std::isnan(b[i])) &&
            std::memcmp(&a[i], &b[i], sizeof(double)) != 0)
            return false;
    return true;
}

mkb::SystemBatchHost singlets(int V) {
    using namespace mkb;
    BatchTopology topo;
    topo.surfaces = 3;
    topo.wavelengths = 3;
    topo.fields = 3;
    topo.type = {SurfaceKind::Stop, SurfaceKind::Sphere, SurfaceKind::Sphere};
    topo.pupil_mode = {PupilMode::Axis, PupilMode::Half, PupilMode::Half};
    SystemBatchHost b(topo, V);
    b.reference_wavelength_nm = 587.6;
    b.wavelength_nm = {486.1, 587.6, 656.3};
    const double lambda_um[3] = {0.4861, 0.5876, 0.6563};
    const double angle_deg[3] = {0.0, 0.7, 1.0};
    const double pi = 3.14159265358979323846;
    for (int v = 0; v < V; ++v) {
        b.curvature(v, 1) = (1.0 / 50.0) * (1.0 + 0.03 * v);
        b.curvature(v, 2) = (-1.0 / 50.0) * (1.0 - 0.02 * v);
        b.thickness(v, 0) = 0.0;
        b.thickness(v, 1) = 6.0 * (1.0 + 0.01 * v);
        b.thickness(v, 2) = 46.0 + 0.5 * v;
        for (int l = 0; l < 3; ++l) {
            b.index(v, 0, l) = 1.0;
            b.index(v, 1, l) = 1.5046 + 0.00420 / (lambda_um[l] * lambda_um[l]);
            b.index(v, 2, l) = 1.0;
        }
        b.pupil_radius(v) = 5.0;
        for (int f = 0; f < 3; ++f) {
            b.field_angle(v, f) = angle_deg[f] * pi / 180.0;
            b.field_target(v, f) = 48.5 * std::tan(angle_deg[f] * pi / 180.0);
        }
    }
    return b;
}

}  // namespace

int main() {
    using namespace mkb;
    const int V = 6;
    SystemBatchHost batch = singlets(V);
    ResidualSettings settings;
    settings.rings = 6;
    settings.spokes = 12;
    const ResidualLayout layout(batch.topology(), settings);
    const auto plan = layout.plan(batch);
    const mkb_batch_view view = batch.view();
    const int64_t rays = layout.rays_per_variant(), rows = layout.trace_rows();
    expect(rays == mko_port_rays_per_variant(plan->get()), "rays per variant");

    cuda::TraceEngine engine(0);
    // RESIDUALS and MERIT
    cuda::TraceOutput out;
    cuda::TraceSettings with_opd(settings);
    with_opd.opd = true;
    engine.run(batch, cuda::TraceMode::Residuals, with_opd, out);
    std::vector<double> res(V * rows), opd(V * rays);
    std::vector<uint8_t> st(V * rays);
    expect(mko_port_residuals(&view, plan->get(), res.data(), opd.data(), st.data(), 1) == 0,
           "oracle residuals");
    expect(same_bits(out.residuals.residuals, res), "RESIDUALS bit-identical to the oracle");
    expect(same_bits(out.residuals.opd, opd), "OPD bit-identical to the oracle");
    expect(same_bits(out.residuals.status, st), "status identical to the oracle");
    expect(out.info.tranches == 1 && out.merit.merit.empty(), "one tranche, no MERIT result");
    // tranches: a memory limit that holds a third of the batch gives bit-identical results
    {
        size_t per = 0, fixed = 0;
        mkb_device_batch shape{};
        std::vector<uint8_t> type;
        for (SurfaceKind k : batch.topology().type) type.push_back(static_cast<uint8_t>(k));
        shape.surfaces = batch.surfaces();
        shape.wavelengths = batch.wavelengths();
        shape.fields = batch.fields();
        shape.record_stride = mkb_record_stride(shape.surfaces, shape.wavelengths, shape.fields);
        shape.type = type.data();
        expect(mkb_trace_run_bytes(&shape, plan->get(), 0, 0, 1, 0, &per, &fixed) == 0,
               "run bytes");
        cuda::EngineOptions opts;
        opts.memory_limit_bytes = fixed + per * static_cast<size_t>((V + 2) / 3);
        opts.reserve = cuda::MemoryReserve{0, 0.0};
        cuda::TraceEngine small(0, opts);
        expect(small.max_variants(batch.topology(), cuda::TraceMode::Residuals, with_opd) ==
                   (V + 2) / 3,
               "max_variants under the memory limit");
        const cuda::TraceOutput split = small.run(batch, cuda::TraceMode::Residuals, with_opd);
        expect(split.info.tranches == 3, "three tranches");
        expect(same_bits(split.residuals.residuals, res) && same_bits(split.residuals.opd, opd) &&
                   same_bits(split.residuals.status, st),
               "tranches bit-identical to the oracle");
        std::vector<double> gathered(V * rows);
        const cuda::TraceRunInfo info = small.run_on_device(
            batch, with_opd, 2, [&](const cuda::DeviceTranche& t) {
                cudaMemcpy(gathered.data() + static_cast<size_t>(t.first) * t.stride,
                           t.residuals, sizeof(double) * t.count * t.stride,
                           cudaMemcpyDeviceToHost);
            });
        expect(info.tranches >= 3 && info.tranche_variants % 2 == 0, "run_on_device tranches");
        expect(same_bits(gathered, res), "run_on_device residuals bit-identical");
    }
    engine.run(batch, cuda::TraceMode::Merit, settings, out);
    std::vector<double> merit(V);
    std::vector<int64_t> failed(V), hard(V);
    expect(mko_port_merit(&view, plan->get(), merit.data(), failed.data(), hard.data(), 1) == 0,
           "oracle merit");
    expect(same_bits(out.merit.merit, merit), "MERIT bit-identical to the oracle");
    expect(same_bits(out.merit.failed, failed) && same_bits(out.merit.hard_failed, hard),
           "failure counts");
    {
        std::vector<double> extra(V);
        for (int v = 0; v < V; ++v) extra[v] = 0.25 * v;
        cuda::TraceSettings with_extra(settings);
        with_extra.extra_merit = extra;
        const cuda::TraceOutput m = engine.run(batch, cuda::TraceMode::Merit, with_extra);
        bool ok = true;
        for (int v = 0; v < V; ++v) ok = ok && m.merit.merit[v] == merit[v] + extra[v];
        expect(ok, "extra_merit added after the tuple sums");
    }

    {  // transverse ray-error rows beside the OPD rows
        ResidualSettings ts = settings;
        ts.transverse_weight = 0.5;
        const ResidualLayout tl(batch.topology(), ts);
        const auto tp = tl.plan(batch);
        const int64_t trows = tl.trace_rows();
        expect(trows == rows + 2 * rays, "transverse rows: two per ray");
        const cuda::TraceOutput t = engine.run(batch, cuda::TraceMode::Residuals, ts);
        std::vector<double> want(static_cast<size_t>(V) * trows), wopd(V * rays);
        std::vector<uint8_t> wst(V * rays);
        expect(mko_port_residuals(&view, tp->get(), want.data(), wopd.data(), wst.data(), 1) == 0,
               "oracle transverse residuals");
        expect(same_bits(t.residuals.residuals, want), "transverse rows bit-identical");
    }

    {  // an aperture stop inside the singlet (between its spheres): the packed entrance pupil
       // and the trace equal the oracle's aiming and its trace of the equivalent batch
        BatchTopology at = batch.topology();
        at.surfaces = 4;
        at.type = {SurfaceKind::Stop, SurfaceKind::Sphere, SurfaceKind::ApertureStop,
                   SurfaceKind::Sphere};
        SystemBatchHost ab(at, V);
        ab.reference_wavelength_nm = batch.reference_wavelength_nm;
        ab.wavelength_nm = batch.wavelength_nm;
        ab.wavelength_weight = batch.wavelength_weight;
        ab.field_weight = batch.field_weight;
        for (int v = 0; v < V; ++v) {
            const int map[4] = {0, 1, -1, 2};
            for (int s = 0; s < 4; ++s) {
                const int o = map[s] < 0 ? 1 : map[s];
                ab.curvature(v, s) = map[s] < 0 ? 4.0 : batch.curvature(v, o);  // R = 4 mm
                ab.thickness(v, s) = s == 1 ? 0.6 * batch.thickness(v, 1)
                                     : s == 2 ? 0.4 * batch.thickness(v, 1)
                                     : batch.thickness(v, o);
                for (int l = 0; l < 3; ++l) ab.index(v, s, l) = batch.view().index[
                    (static_cast<size_t>(v) * 3 + o) * 3 + l];
            }
            ab.pupil_radius(v) = 5.0;
            for (int f = 0; f < 3; ++f) {
                ab.field_angle(v, f) = batch.view().field_angle[v * 3 + f];
                ab.field_target(v, f) = batch.view().field_target[v * 3 + f];
            }
        }
        const ResidualLayout al(ab.topology(), settings);
        const cuda::TraceOutput t = engine.run(ab, cuda::TraceMode::Residuals, settings);
        // the equivalent batch: the stop as a plane, surface 0 at the oracle's pupil
        mkb_batch_view ev = ab.view();
        std::vector<double> a(V), t0(V);
        expect(mko_port_aim(&ev, a.data(), t0.data()) == 0, "oracle aiming");
        std::vector<uint8_t> etype = {MKB_SURFACE_STOP, MKB_SURFACE_SPHERE, MKB_SURFACE_PLANE,
                                      MKB_SURFACE_SPHERE};
        std::vector<double> ec(ev.curvature, ev.curvature + 4 * V), et(ev.thickness,
                                                                       ev.thickness + 4 * V);
        for (int v = 0; v < V; ++v) {
            ec[v * 4 + 2] = 0.0;
            et[v * 4] = t0[v];
        }
        ev.type = etype.data();
        ev.curvature = ec.data();
        ev.thickness = et.data();
        ev.pupil_radius = a.data();
        const auto ap = al.plan(ab);
        std::vector<double> want(static_cast<size_t>(V) * al.trace_rows());
        expect(mko_port_residuals(&ev, ap->get(), want.data(), nullptr, nullptr, 1) == 0,
               "oracle residuals of the equivalent batch");
        expect(same_bits(t.residuals.residuals, want),
               "interior stop: RESIDUALS bit-identical to the oracle on the aimed pupil");
    }

    // Jacobians and normal equations
    const VariableSet vars(batch.topology(),
                           {{VariableType::Curvature, 1, -0.2, 0.2, 0.01},
                            {VariableType::Curvature, 2, -0.2, 0.2, 0.01},
                            {VariableType::Thickness, 1, 0.5, 20.0, 1.0},
                            {VariableType::WorkingDistance, 2, 1.0, 500.0, 1.0}});
    const int P = vars.size();
    std::vector<double> x0;
    for (int v = 0; v < V; ++v) {
        const std::vector<double> x = vars.extract(batch, v);
        x0.insert(x0.end(), x.begin(), x.end());
    }
    const mkb_variables cv = vars.c_struct();
    std::vector<double> J(static_cast<size_t>(V) * P * rows), r0(static_cast<size_t>(V) * rows);
    cuda::JacobianResult jac;
    cuda::DeviceFdJacobian fd;
    fd.compute(engine, vars, batch, x0, settings, jac);
    expect(mko_port_fd_jacobian(&view, plan->get(), &cv, x0.data(), V, J.data(), r0.data(),
                                nullptr, 1) == 0,
           "oracle fd jacobian");
    expect(same_bits(jac.J, J) && same_bits(jac.r0, r0), "FD Jacobian bit-identical");
    cuda::DeviceAdjointJacobian adj;
    adj.compute(engine, vars, batch, x0, settings, jac);
    std::vector<uint8_t> jst(static_cast<size_t>(V) * rays);
    expect(mko_port_adjoint_jacobian(&view, plan->get(), &cv, x0.data(), V, J.data(), r0.data(),
                                     jst.data(), 1) == 0,
           "oracle adjoint jacobian");
    expect(same_bits(jac.J, J) && same_bits(jac.r0, r0), "adjoint Jacobian bit-identical");
    cuda::DeviceNormalEquations ne;
    ne.compute(engine, jac, true);
    std::vector<double> a, g;
    ne.download(a, g);
    bool ne_ok = true;
    for (int run = 0; run < V; ++run) {
        std::vector<double> A(P * P), gg(P);
        mko_port_normal_equations(J.data() + static_cast<size_t>(run) * P * rows,
                                  r0.data() + static_cast<size_t>(run) * rows, P, rows,
                                  A.data(), gg.data());
        ne_ok = ne_ok && std::memcmp(A.data(), a.data() + run * P * P, sizeof(double) * P * P) == 0 &&
                std::memcmp(gg.data(), g.data() + run * P, sizeof(double) * P) == 0;
    }
    expect(ne_ok, "normal equations bit-identical");

    // LM on the device
    LmOptions opt;
    opt.max_iterations = 25;
    cuda::LmGpuStats stats;
    const cuda::LmResult lm = cuda::optimize_lm_gpu(engine, vars, batch, x0, opt, settings, &stats);
    bool improved = true;
    for (int run = 0; run < V; ++run)
        improved = improved && lm.merit[run] < merit[run] && lm.iterations[run] > 0;
    expect(improved, "LM lowers every run's merit");
    expect(stats.cycles > 0, "LM ran cycles");

#ifdef MKB_HAVE_REF
    {  // per-surface extrema against the reference's surface_extrema_cpu
        cuda::TraceSettings es(settings);
        es.extrema = true;
        const cuda::TraceOutput eo = engine.run(batch, cuda::TraceMode::Merit, es);
        std::vector<double> want(static_cast<size_t>(V) * batch.surfaces() * 2);
        expect(mko_ref_surface_extrema(&view, plan->get(), want.data()) == 0,
               "reference surface extrema");
        expect(same_bits(eo.merit.extrema, want), "extrema bit-identical to the reference");
    }
    {  // extra rows: focal length, working distance, Petzval constraints (the reference's
       // paraxial_residuals as the evaluate function) against the reference LM with them
        const int32_t ctype[3] = {0, 2, 4}, cmode[3] = {0, 1, 2};
        const double cw[3] = {4.0, 1.0, 1e4}, ct[3] = {48.0, 47.5, 0.001};
        LmOptions xo;
        xo.max_iterations = 8;
        xo.fail_weight_factor = 1.0;
        xo.extra.count = 3;
        xo.extra.evaluate = [&](const SystemBatchHost& one, int v, std::span<double> out) {
            const mkb_batch_view w = one.view();
            const auto p1 = layout.plan(one);
            if (mko_ref_paraxial_residuals(&w, p1->get(), v, 3, ctype, cmode, cw, ct,
                                           out.data()) != 0)
                throw std::runtime_error("reference paraxial_residuals failed");
        };
        const cuda::LmResult g = cuda::optimize_lm_gpu(engine, vars, batch, x0, xo, settings);
        std::vector<double> rx(x0.size()), rm(V), rh(static_cast<size_t>(V) * 9);
        std::vector<int32_t> rs(V), ri(V), ra(V);
        expect(mko_ref_optimize_lm(&view, plan->get(), &cv, x0.data(), V, 8, 1, 1, 4, rx.data(),
                                   rm.data(), rs.data(), ri.data(), ra.data(), rh.data(), 3,
                                   ctype, cmode, cw, ct, 0, nullptr, nullptr, nullptr,
                                   nullptr) == 0,
               "reference LM with constraints");
        std::vector<int32_t> gs(g.status.begin(), g.status.end());
        expect(same_bits(g.x, rx) && same_bits(g.merit, rm) && same_bits(gs, rs) &&
                   same_bits(g.iterations, ri) && same_bits(g.accepted, ra),
               "LM with extra rows bit-identical to the reference");

        // plus rows from the trace's extrema (semi-diameter and incidence-angle limits)
        const int32_t tsurf[3] = {1, 2, 2}, tkind[3] = {0, 0, 1};
        const double tw[3] = {100.0, 50.0, 1e3}, tl[3] = {4.8, 4.7, 0.9995};
        xo.trace_extra.count = 3;
        xo.trace_extra.evaluate = [&](const SystemBatchHost&, int, std::span<const double> e,
                                      std::span<double> out) {
            for (int i = 0; i < 3; ++i) {
                const double q = tkind[i] == 0 ? e[2 * tsurf[i]] - tl[i]
                                               : tl[i] - e[2 * tsurf[i] + 1];
                out[i] = std::sqrt(tw[i]) * std::max(0.0, q);
            }
        };
        const cuda::LmResult g2 = cuda::optimize_lm_gpu(engine, vars, batch, x0, xo, settings);
        expect(mko_ref_optimize_lm(&view, plan->get(), &cv, x0.data(), V, 8, 1, 1, 4, rx.data(),
                                   rm.data(), rs.data(), ri.data(), ra.data(), rh.data(), 3,
                                   ctype, cmode, cw, ct, 3, tsurf, tkind, tw, tl) == 0,
               "reference LM with trace rows");
        std::vector<int32_t> gs2(g2.status.begin(), g2.status.end());
        expect(same_bits(g2.x, rx) && same_bits(g2.merit, rm) && same_bits(gs2, rs) &&
                   same_bits(g2.iterations, ri) && same_bits(g2.accepted, ra),
               "LM with trace-dependent rows bit-identical to the reference");

        // the same three constraints evaluated on the device (no host phase in the cycle)
        LmOptions po;
        po.max_iterations = 8;
        po.fail_weight_factor = 1.0;
        for (int i = 0; i < 3; ++i) {
            ParaxialConstraint c;
            c.type = ctype[i];
            c.mode = cmode[i];
            c.weight = cw[i];
            c.target = ct[i];
            po.paraxial.items.push_back(c);
        }
        const cuda::LmResult g3 = cuda::optimize_lm_gpu(engine, vars, batch, x0, po, settings);
        expect(mko_ref_optimize_lm(&view, plan->get(), &cv, x0.data(), V, 8, 1, 1, 4, rx.data(),
                                   rm.data(), rs.data(), ri.data(), ra.data(), rh.data(), 3,
                                   ctype, cmode, cw, ct, 0, nullptr, nullptr, nullptr,
                                   nullptr) == 0,
               "reference LM with constraints");
        std::vector<int32_t> gs3(g3.status.begin(), g3.status.end());
        expect(same_bits(g3.x, rx) && same_bits(g3.merit, rm) && same_bits(gs3, rs) &&
                   same_bits(g3.iterations, ri) && same_bits(g3.accepted, ra),
               "LM with device paraxial constraints bit-identical to the reference");
    }
    {  // FP32 prefilter against the reference's prefilter_cpu
        cuda::PrefilterSettings ps;
        ps.quadrature = settings;
        ps.options.criteria.max_merit_factor = 3.0;
        const cuda::PrefilterResult pr = engine.prefilter_variants(batch, ps);
        mkb_prefilter_options o{0.5, INFINITY, 3.0, 0.15, 32.0, 0.01};
        std::vector<double> m(V), opl(V), lo(V), hi(V);
        std::vector<int64_t> fl(V), uo(V), uf(V);
        std::vector<uint8_t> rej(V);
        double rmerit = 0.0;
        int32_t rv = 0, kept = 0;
        expect(mko_ref_prefilter(&view, plan->get(), &o, nullptr, m.data(), opl.data(), fl.data(),
                                 uo.data(), uf.data(), lo.data(), hi.data(), rej.data(), &rmerit,
                                 &rv, &kept) == 0,
               "reference prefilter");
        expect(same_bits(pr.stats.merit, m) && same_bits(pr.stats.optical_length, opl) &&
                   same_bits(pr.stats.failed, fl) && same_bits(pr.stats.uncertain_ok, uo) &&
                   same_bits(pr.stats.uncertain_failed, uf),
               "prefilter statistics bit-identical to the reference");
        std::vector<uint8_t> got(pr.reject.begin(), pr.reject.end());
        expect(same_bits(pr.merit_lower, lo) && same_bits(pr.merit_upper, hi) &&
                   same_bits(got, rej) && pr.kept == kept && pr.reference_variant == rv,
               "prefilter decision identical to the reference");
    }
    for (int reference = 0; reference < 3; ++reference) {  // EVAL against eval_cpu
        cuda::EvalSettings es;
        es.grid = 16;
        es.reference = static_cast<cuda::EvalReference>(reference);
        const cuda::EvalResult e = engine.evaluate(batch, es);
        int64_t n = 0;
        expect(mko_ref_eval(&view, plan->get(), 16, 0, reference, 1e-3, &n, nullptr, nullptr,
                            nullptr, nullptr, nullptr, nullptr, nullptr, nullptr) == 0 &&
                   n == e.samples,
               "reference EVAL grid");
        const size_t T = static_cast<size_t>(V) * 3 * 3, N = static_cast<size_t>(n);
        std::vector<double> opd(T * N), sx(T * N), sy(T * N), fr(T * 20), k(V * 3), zp(V);
        std::vector<uint8_t> est(T * N), fs(T * 4);
        expect(mko_ref_eval(&view, plan->get(), 16, 0, reference, 1e-3, &n, opd.data(),
                            sx.data(), sy.data(), est.data(), fr.data(), fs.data(), k.data(),
                            zp.data()) == 0,
               "reference EVAL");
        expect(same_values(e.opd, opd) && same_values(e.spot_x, sx) &&
                   same_values(e.spot_y, sy) && same_bits(e.status, est) &&
                   same_values(e.field_rays, fr) && same_bits(e.field_status, fs) &&
                   same_values(e.reference_curvature, k) &&
                   same_values(e.exit_pupil_position, zp),
               "EVAL bit-identical to the reference");
    }
    {  // scalar PSF and MTF against the reference's psf_cpu (its CPU/GPU bar: 1e-13)
        cuda::EvalSettings es;
        es.grid = 16;
        const cuda::EvalResult e = engine.evaluate(batch, es);
        cuda::PsfEngine pe(0);
        mkb_batch_view pv = view;
        pv.wavelength_nm = batch.wavelength_nm.data();
        bool ok = true;
        for (int v = 0; v < V; ++v) {
            const std::vector<cuda::PsfResult> got = pe.compute(batch, e, v);
            int M = 0, full = 0;
            expect(mko_ref_psf(&pv, plan->get(), 16, 0, 0, 1e-3, v, 4.0, 0.0, &M, &full, nullptr,
                               nullptr, nullptr, nullptr, nullptr, nullptr) == 0,
                   "reference PSF sizes");
            const size_t T = 9, m2 = size_t(M) * M;
            std::vector<double> maps(T * 256), na(2 * T), psf(T * m2), mtf(T * 34), fig(T * 13);
            std::vector<int> flips(2 * T);
            expect(mko_ref_psf(&pv, plan->get(), 16, 0, 0, 1e-3, v, 4.0, 0.0, &M, &full,
                               maps.data(), na.data(), flips.data(), psf.data(), mtf.data(),
                               fig.data()) == 0,
                   "reference PSF");
            ok = ok && got.size() == T;
            for (size_t t = 0; ok && t < T; ++t) {
                const cuda::PsfResult& r = got[t];
                for (size_t k = 0; k < m2; ++k) ok = ok && std::abs(r.psf[k] - psf[t * m2 + k]) <= 1e-13;
                for (int k = 0; k <= 16; ++k)
                    ok = ok && std::abs(r.mtf_sagittal[k] - mtf[t * 34 + k]) <= 1e-13 &&
                         std::abs(r.mtf_tangential[k] - mtf[t * 34 + 17 + k]) <= 1e-13;
                const double* q = fig.data() + t * 13;
                ok = ok && double(r.transmitted) == q[0] && std::abs(r.energy - q[1]) <= 1e-13 &&
                     std::abs(r.strehl_fft - q[2]) <= 1e-13 && r.strehl_origin == q[3] &&
                     r.strehl == q[4] && r.reference_x == q[5] && r.reference_y == q[6] &&
                     r.dx == q[10] && r.dy == q[11] && r.airy_radius == q[12];
            }
        }
        expect(ok, "PSF and MTF within 1e-13 of the reference, figures equal");
        expect(pe.last_run().pupils == 9 && pe.last_run().tranches == 1, "PSF run info");
    }
#endif

    // argument errors are thrown before any device work
    bool thrown = false;
    try {
        BatchTopology bad = batch.topology();
        bad.type[0] = SurfaceKind::Sphere;
        bad.validate();
    } catch (const std::invalid_argument&) {
        thrown = true;
    }
    expect(thrown, "invalid topology -> std::invalid_argument");
    thrown = false;
    try {
        std::vector<double> short_x(P + 1, 0.0);
        cuda::optimize_lm_gpu(engine, vars, batch, short_x, opt, settings);
    } catch (const std::invalid_argument&) {
        thrown = true;
    }
    expect(thrown, "x0 of the wrong size -> std::invalid_argument");

    std::printf("host API: %d of %d checks passed\n", checks - failures, checks);
    return failures == 0 ? 0 : 1;
}
