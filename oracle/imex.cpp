// imex.cpp — restatement of TimeIntegrationIMEX.jl (integrate_step!,
// make_velocity_compatible!) and the oracle's C entry points.
// TEST INFRASTRUCTURE ONLY (the oracle); see oracle.hpp.  The entry points carry
// the `oracle_` prefix and otherwise mirror include/efsi.h so that tests can
// drive the oracle and the CUDA library with the same host code.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <string>

#include "oracle.hpp"

namespace ora {
using OpFn = std::function<void(const std::vector<double>&, std::vector<double>&)>;
template <class Op>
int bicgstab(const Op&, const std::vector<double>&, std::vector<double>&, double, int);

// Tableaux (TimeIntegrationIMEX.jl:74-90).
static const double AE[4][4] = {{0, 0, 0, 0}, {8.0 / 15, 0, 0, 0}, {1.0 / 4, 5.0 / 12, 0, 0}, {1.0 / 4, 0, 3.0 / 4, 0}};
static const double AI[4][4] = {{0, 0, 0, 0}, {4.0 / 15, 4.0 / 15, 0, 0}, {4.0 / 15, 1.0 / 3, 1.0 / 15, 0},
                                {4.0 / 15, 1.0 / 3, 7.0 / 30, 1.0 / 6}};
static const double CS[4] = {0.0, 8.0 / 15, 2.0 / 3, 1.0};

struct Ctx {
    efsi_models md;
    efsi_numerics nu;
    Mesh m;
    BCS bu, bv, bq, bphi, bc, bsig[3];
    std::unique_ptr<Projector, void (*)(Projector*)> proj{nullptr, free_projector};
    F2 U, V, phi, c, sxx, syy, sxy, correction;
    std::string err;
    efsi_stats stats{};
};

static bool visc_active(const efsi_models& md) { return md.viscosity != EFSI_VISC_NONE; }
static bool diff_active(const efsi_models& md) { return md.diffusivity != EFSI_DIFF_NONE; }

static void compact(const F2& U, const F2& V, int Nx, int Ny, std::vector<double>& out) {  // :531-541
    const size_t N = (size_t)Nx * Ny;
    out.resize(2 * N);
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            out[(size_t)i + (size_t)j * Nx] = U(i, j);
            out[N + (size_t)i + (size_t)j * Nx] = V(i, j);
        }
}

static void inject(F2& U, F2& V, const std::vector<double>& x, const Ctx& C) {  // :543-579
    const int Nx = C.m.Nx, Ny = C.m.Ny;
    const size_t N = (size_t)Nx * Ny;
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            U(i, j) = x[(size_t)i + (size_t)j * Nx];
            V(i, j) = x[N + (size_t)i + (size_t)j * Nx];
        }
    if (C.m.px) {
        for (int j = 0; j < Ny; ++j) U(Nx, j) = U(0, j);
    } else if (C.bu.right().type == EFSI_BC_DIRICHLET) {
        for (int j = 0; j < Ny; ++j) U(Nx, j) = C.bu.right().val(j);
    } else {
        arg_error("The compact predictor currently requires a Dirichlet or Periodic U-right boundary.");
    }
    if (C.m.py) {
        for (int i = 0; i < Nx; ++i) V(i, Ny) = V(i, 0);
    } else if (C.bv.top().type == EFSI_BC_DIRICHLET) {
        for (int i = 0; i < Nx; ++i) V(i, Ny) = C.bv.top().val(i);
    } else {
        arg_error("The compact predictor currently requires a Dirichlet or Periodic V-top boundary.");
    }
}

static void validate_state(const Ctx& C, const F2& U, const F2& V, const F2& phi, const F2& c,
                           const F2& sxx, const F2& syy, const F2& sxy) {  // :495-523
    const F2* cells[5] = {&phi, &c, &sxx, &syy, &sxy};
    const char* names[5] = {"state.phi", "state.resource", "state.sigma_xx", "state.sigma_yy", "state.sigma_xy"};
    for (int k = 0; k < 5; ++k)
        for (double v : cells[k]->a)
            if (!std::isfinite(v)) arg_error(std::string(names[k]) + " contains non-finite values.");
    for (double v : U.a) if (!std::isfinite(v)) arg_error("state.U contains non-finite values.");
    for (double v : V.a) if (!std::isfinite(v)) arg_error("state.V contains non-finite values.");
    (void)C;
}

// _solve_linear_system! (TimeIntegrationIMEX.jl:602-641) with BiCGStab standing in for
// both methods: :direct is a 1e-13 solve; :gmres runs to reltol within maxiter and
// is judged by |A x - b| / max(|b|, eps): non-finite or above fallback_reltol falls
// back to the 1e-13 solve when direct_fallback is set and throws otherwise (:637).
static int judged_solve(const OpFn& op, const std::vector<double>& b, std::vector<double>& x, int method,
                        const efsi_numerics& nu, const std::string& name) {
    if (method != EFSI_LINEAR_GMRES) return bicgstab(op, b, x, 1e-13, EFSI_LINEAR_HARD_CAP);
    int it = bicgstab(op, b, x, nu.linear_reltol, std::max(nu.linear_maxiter, 1));
    std::vector<double> ax;
    op(x, ax);
    double rn = 0.0, bn = 0.0;
    for (size_t k = 0; k < b.size(); ++k) {
        rn += (ax[k] - b[k]) * (ax[k] - b[k]);
        bn += b[k] * b[k];
    }
    const double rr = std::sqrt(rn) / std::max(std::sqrt(bn), 2.220446049250313e-16);
    if (!std::isfinite(rr) || rr > nu.fallback_reltol) {
        if (!nu.direct_fallback) {
            char buf[64];
            snprintf(buf, sizeof buf, "%.17g", rr);
            solve_error(name + " GMRES residual is too large: " + buf);
        }
        it += bicgstab(op, b, x, 1e-13, EFSI_LINEAR_HARD_CAP);
    }
    return it;
}

// Solve (I - alpha*A) x = rhs with the reference's row Dirichlet elimination (:643-672, :786-812).
static void velocity_solve(const Ctx& C, const F2& mu, double alpha, std::vector<double>& rhs,
                           std::vector<double>& x, int& iters, int stage) {
    std::vector<int> idx;
    std::vector<double> val;
    velocity_dirichlet_data(C.m, C.bu, C.bv, idx, val);
    std::vector<uint8_t> fixed(rhs.size(), 0);
    for (size_t k = 0; k < idx.size(); ++k) { fixed[idx[k]] = 1; rhs[idx[k]] = val[k]; }
    OpFn op = [&](const std::vector<double>& in, std::vector<double>& out) {
        std::vector<double> ax;
        viscous_apply(in, mu, C.m, C.bu, C.bv, false, ax);
        out.resize(in.size());
        for (size_t k = 0; k < in.size(); ++k) out[k] = fixed[k] ? in[k] : in[k] - alpha * ax[k];
    };
    iters = judged_solve(op, rhs, x, C.nu.velocity_method, C.nu, "velocity stage " + std::to_string(stage + 1));
}

static void resource_solve(const Ctx& C, const F2& D, double alpha, const std::vector<double>& rhs,
                           std::vector<double>& x, int& iters, int stage) {
    OpFn op = [&](const std::vector<double>& in, std::vector<double>& out) {
        F2 f(C.m.Nx, C.m.Ny);
        f.a = in;
        F2 Lf;
        diffusion_matrix_apply(f, D, C.m, C.bc, Lf);
        out.resize(in.size());
        for (size_t k = 0; k < in.size(); ++k) out[k] = in[k] - alpha * Lf.a[k];
    };
    iters = judged_solve(op, rhs, x, C.nu.resource_method, C.nu, "resource stage " + std::to_string(stage + 1));
}

struct Tend {
    std::vector<double> Euv, Iuv, Ec, Ic;
    F2 Ephi, Exx, Eyy, Exy;
};

// Explicit momentum forcing (TimeIntegrationIMEX.jl:959-985) on the full MAC faces.
static void momentum_forcing(const Ctx& C, double t_stage, const F2& U, const F2& V, const F2& phi,
                             const F2& sxx, const F2& syy, const F2& sxy, const F2& G,
                             const F2& Kxx, const F2& Kxy, const F2& Kyx, const F2& Kyy,
                             const F2& mu, F2& Fx, F2& Fy) {
    const Mesh& m = C.m;
    const int Nx = m.Nx, Ny = m.Ny;
    F2 Cu, Cv;
    material_convection(U, V, G, m, C.bu, C.bv, Cu, Cv);
    Fx = Cu; Fy = Cv;
    for (double& v : Fx.a) v = -v;
    for (double& v : Fy.a) v = -v;
    F2 bx, by;
    body_force(C.md, t_stage, m, bx, by);
    for (size_t k = 0; k < Fx.size(); ++k) Fx.a[k] += bx.a[k];
    for (size_t k = 0; k < Fy.size(); ++k) Fy.a[k] += by.a[k];
    F2 cx, cy;
    capillary_force(C.md, phi, m, C.bphi, cx, cy);
    for (size_t k = 0; k < Fx.size(); ++k) Fx.a[k] += cx.a[k];
    for (size_t k = 0; k < Fy.size(); ++k) Fy.a[k] += cy.a[k];
    {  // _accumulate_elastic_force! (:903-924)
        F2 txx(Nx, Ny), tyy(Nx, Ny), txy(Nx, Ny);
        if (C.md.elastic_stress == EFSI_ELASTIC_LINEAR) {
            double g = C.md.elastic_coefficient;
            for (size_t k = 0; k < txx.size(); ++k) {
                txx.a[k] = phi.a[k] * (g * (sxx.a[k] - 1.0));
                tyy.a[k] = phi.a[k] * (g * (syy.a[k] - 1.0));
                txy.a[k] = phi.a[k] * (g * sxy.a[k]);
            }
        }
        F2 ex, ey;
        symmetric_stress_divergence(txx, tyy, txy, m, ex, ey);
        for (size_t k = 0; k < Fx.size(); ++k) Fx.a[k] += ex.a[k];
        for (size_t k = 0; k < Fy.size(); ++k) Fy.a[k] += ey.a[k];
    }
    if (visc_active(C.md)) {  // _accumulate_growth_viscous_force! (:926-942)
        F2 txx(Nx, Ny), tyy(Nx, Ny), txy(Nx, Ny);
        for (size_t k = 0; k < txx.size(); ++k) {
            txx.a[k] = -2.0 * mu.a[k] * Kxx.a[k];
            tyy.a[k] = -2.0 * mu.a[k] * Kyy.a[k];
            txy.a[k] = -mu.a[k] * (Kxy.a[k] + Kyx.a[k]);
        }
        F2 ex, ey;
        symmetric_stress_divergence(txx, tyy, txy, m, ex, ey);
        for (size_t k = 0; k < Fx.size(); ++k) Fx.a[k] += ex.a[k];
        for (size_t k = 0; k < Fy.size(); ++k) Fy.a[k] += ey.a[k];
    }
}

static void stage_tendencies(Ctx& C, double t_stage, const F2& U, const F2& V, const F2& phi,
                             const F2& c, const F2& sxx, const F2& syy, const F2& sxy, const F2& G,
                             const F2& Kxx, const F2& Kxy, const F2& Kyx, const F2& Kyy, const F2& mu,
                             const F2& D, Tend& T) {  // :944-1071
    const Mesh& m = C.m;
    const int Nx = m.Nx, Ny = m.Ny;
    F2 Fx, Fy;
    momentum_forcing(C, t_stage, U, V, phi, sxx, syy, sxy, G, Kxx, Kxy, Kyx, Kyy, mu, Fx, Fy);
    compact(Fx, Fy, Nx, Ny, T.Euv);
    T.Ephi = phase_field_rhs(C.md, U, V, phi, G, m, C.bphi);
    const size_t N = (size_t)Nx * Ny;
    if (C.md.growth_source == EFSI_GROWTH_NONE && C.md.diffusivity == EFSI_DIFF_NONE &&
        C.md.resource_consumption == EFSI_CONSUMPTION_NONE) {
        T.Ec.assign(N, 0.0);
    } else {
        F2 sink;
        resource_sink(C.md, phi, c, sink);
        F2 e = resource_explicit_rhs(U, V, c, sink, m, C.bc);
        T.Ec = e.a;
    }
    structure_tensor_rhs(sxx, syy, sxy, U, V, Kxx, Kxy, Kyx, Kyy, C.md, C.nu, m, C.bsig, C.bu, C.bv,
                         phi, T.Exx, T.Eyy, T.Exy);
    std::vector<double> uv;
    compact(U, V, Nx, Ny, uv);
    if (visc_active(C.md)) viscous_apply(uv, mu, m, C.bu, C.bv, true, T.Iuv);
    else T.Iuv.assign(2 * N, 0.0);
    if (diff_active(C.md)) T.Ic = diffusion_apply(c, D, m, C.bc).a;
    else T.Ic.assign(N, 0.0);
}

static void integrate_step(Ctx& C, double t, double dt, efsi_step_report* rep) {  // :1152-1256
    validate_state(C, C.U, C.V, C.phi, C.c, C.sxx, C.syy, C.sxy);
    if (!std::isfinite(t)) arg_error("t must be finite.");
    if (!std::isfinite(dt)) arg_error("dt must be finite.");
    if (!(dt > 0)) arg_error("dt must be strictly positive.");
    const Mesh& m = C.m;
    const int Nx = m.Nx, Ny = m.Ny;
    const size_t N = (size_t)Nx * Ny;
    std::vector<double> uvn;
    compact(C.U, C.V, Nx, Ny, uvn);
    F2 cn = C.c, phin = C.phi, sxn = C.sxx, syn = C.syy, sxyn = C.sxy;
    apply_structure_extension(C.nu, sxn, syn, sxyn, phin);
    double max_c = 0.0, max_tr = 0.0;
    Tend T[3];
    F2 Us = C.U, Vs = C.V, phis, cs, sxs, sys, sxys;
    std::vector<double> uvs;
    for (int s = 0; s < 4; ++s) {
        if (s == 0) {
            Us = C.U; Vs = C.V; phis = phin; cs = cn; sxs = sxn; sys = syn; sxys = sxyn; uvs = uvn;
        } else {  // _build_explicit_stage! (:716-740)
            phis = phin; sxs = sxn; sys = syn; sxys = sxyn;
            for (int j = 0; j < s; ++j) {
                double a = AE[s][j];
                if (a == 0.0) continue;
                for (size_t k = 0; k < N; ++k) {
                    phis.a[k] += dt * a * T[j].Ephi.a[k];
                    sxs.a[k] += dt * a * T[j].Exx.a[k];
                    sys.a[k] += dt * a * T[j].Eyy.a[k];
                    sxys.a[k] += dt * a * T[j].Exy.a[k];
                }
            }
            apply_structure_extension(C.nu, sxs, sys, sxys, phis);
        }
        F2 D;
        diffusivity_field(C.md, phis, D);
        if (s > 0) {  // _build_resource_stage! (:742-774)
            std::vector<double> rc = cn.a;
            for (int j = 0; j < s; ++j) {
                double ae = AE[s][j], ai = AI[s][j];
                if (ae != 0.0 || ai != 0.0)
                    for (size_t k = 0; k < N; ++k) rc[k] += dt * (ae * T[j].Ec[k] + ai * T[j].Ic[k]);
            }
            cs = F2(Nx, Ny);
            if (!diff_active(C.md)) {
                cs.a = rc;
            } else {
                double alpha = dt * AI[s][s];
                F2 zero(Nx, Ny);
                F2 bD = diffusion_apply(zero, D, m, C.bc);
                for (size_t k = 0; k < N; ++k) rc[k] += alpha * bD.a[k];
                std::vector<double> x = cn.a;
                int it = 0;
                resource_solve(C, D, alpha, rc, x, it, s);
                C.stats.resource_iterations[s] = it;
                cs.a = x;
            }
        }
        F2 G, Kxx, Kxy, Kyx, Kyy;  // _evaluate_growth! (:842-865)
        growth_source(C.md, phis, cs, G);
        growth_tensor(C.md, G, Kxx, Kxy, Kyx, Kyy);
        max_tr = std::max(max_tr, growth_trace_error(G, Kxx, Kyy));
        F2 mu;
        viscosity_field(C.md, phis, mu);
        if (s == 0) {  // :1194-1201, :1111-1127
            compact(Us, Vs, Nx, Ny, uvs);
            F2 d = divergence(Us, Vs, m);
            double linf = 0.0, gmax = 0.0;
            for (size_t k = 0; k < N; ++k) {
                linf = std::max(linf, std::fabs(d.a[k] - G.a[k]));
                gmax = std::max(gmax, std::fabs(G.a[k]));
            }
            if (C.nu.check_stage1_constraint) {
                double tol = C.nu.stage1_constraint_atol + C.nu.stage1_constraint_rtol * std::max(gmax, 1.0);
                if (!(linf <= tol))
                    arg_error("The velocity entering stage 1 does not satisfy the prescribed divergence constraint.");
            }
            max_c = std::max(max_c, linf);
        } else {  // _build_velocity_stage! (:776-836)
            std::vector<double> rhs = uvn;
            for (int j = 0; j < s; ++j) {
                double ae = AE[s][j], ai = AI[s][j];
                if (ae != 0.0 || ai != 0.0)
                    for (size_t k = 0; k < 2 * N; ++k) rhs[k] += dt * (ae * T[j].Euv[k] + ai * T[j].Iuv[k]);
            }
            std::vector<double> pred;
            if (!visc_active(C.md)) {
                pred = rhs;
                std::vector<int> idx;
                std::vector<double> val;
                velocity_dirichlet_data(m, C.bu, C.bv, idx, val);
                for (size_t k = 0; k < idx.size(); ++k) pred[idx[k]] = val[k];
            } else {
                double alpha = dt * AI[s][s];
                std::vector<double> zero(2 * N, 0.0), bvis;
                viscous_apply(zero, mu, m, C.bu, C.bv, true, bvis);
                for (size_t k = 0; k < 2 * N; ++k) rhs[k] += alpha * bvis[k];
                pred = uvn;
                int it = 0;
                velocity_solve(C, mu, alpha, rhs, pred, it, s);
                C.stats.velocity_iterations[s] = it;
            }
            inject(Us, Vs, pred, C);
            ProjOut po = project(C.proj.get(), Us, Vs, G, C.correction, C.nu.projection_reltol,
                                 C.nu.projection_maxiter);
            C.stats.projection_iterations[s] = po.iters;
            max_c = std::max(max_c, po.constraint_linf);
            compact(Us, Vs, Nx, Ny, uvs);
        }
        if (s < 3)
            stage_tendencies(C, t + CS[s] * dt, Us, Vs, phis, cs, sxs, sys, sxys, G, Kxx, Kxy, Kyx,
                             Kyy, mu, D, T[s]);
    }
    C.U = Us; C.V = Vs; C.phi = phis; C.c = cs; C.sxx = sxs; C.syy = sys; C.sxy = sxys;
    SigmaDiag sd = structure_tensor_diagnostics(C.sxx, C.syy, C.sxy);
    if (rep) {
        rep->maximum_projection_constraint_linf = max_c;
        rep->maximum_growth_trace_error = max_tr;
        rep->minimum_phi = *std::min_element(C.phi.a.begin(), C.phi.a.end());
        rep->maximum_phi = *std::max_element(C.phi.a.begin(), C.phi.a.end());
        rep->minimum_resource = *std::min_element(C.c.a.begin(), C.c.a.end());
        rep->minimum_sigma_eigenvalue = sd.min_eig;
        rep->maximum_abs_sigma_determinant_error = sd.max_abs_det_err;
        rep->non_spd_cells = sd.non_spd;
    }
}

}  // namespace ora

// ============================================================================
// C entry points
// ============================================================================
using namespace ora;

static thread_local std::string g_create_err;

template <class F>
static int guarded(Ctx* h, F&& f) {
    try {
        f();
        return EFSI_OK;
    } catch (const Err& e) {
        if (h) h->err = e.what();
        else g_create_err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        if (h) h->err = e.what();
        else g_create_err = e.what();
        return EFSI_ARG;
    }
}

static F2 wrap(const double* p, int nx, int ny) {
    F2 f(nx, ny);
    if (p) std::memcpy(f.a.data(), p, sizeof(double) * f.a.size());
    return f;
}
static void unwrap(const F2& f, double* p) {
    if (p) std::memcpy(p, f.a.data(), sizeof(double) * f.a.size());
}

extern "C" {

int oracle_create(const efsi_config* cfg, Ctx** out) {
    *out = nullptr;
    auto c = std::make_unique<Ctx>();
    int st = guarded(nullptr, [&] {
        if (!cfg) arg_error("config is NULL");
        if (cfg->abi_version != EFSI_ABI_VERSION) arg_error("config ABI version mismatch");
        c->md = cfg->models;
        c->nu = cfg->numerics;
        c->m = make_mesh(cfg->mesh);
        const int Nx = c->m.Nx, Ny = c->m.Ny;
        c->bu = make_bcs(cfg->bc_U, Ny, Nx + 1, "U");
        c->bv = make_bcs(cfg->bc_V, Ny + 1, Nx, "V");
        c->bq = make_bcs(cfg->bc_correction, Ny, Nx, "correction");
        c->bphi = make_bcs(cfg->bc_phi, Ny, Nx, "phi");
        c->bc = make_bcs(cfg->bc_resource, Ny, Nx, "resource");
        c->bsig[0] = make_bcs(cfg->bc_sigma_xx, Ny, Nx, "sigma_xx");
        c->bsig[1] = make_bcs(cfg->bc_sigma_yy, Ny, Nx, "sigma_yy");
        c->bsig[2] = make_bcs(cfg->bc_sigma_xy, Ny, Nx, "sigma_xy");
        const BCS* all[8] = {&c->bu, &c->bv, &c->bq, &c->bphi, &c->bc, &c->bsig[0], &c->bsig[1], &c->bsig[2]};
        for (const BCS* b : all)  // :447-466
            if (b->periodic_x() != c->m.px || b->periodic_y() != c->m.py)
                arg_error("boundary conditions do not match MeshMetrics periodicity.");
        if (c->md.viscosity != EFSI_VISC_NONE)  // Operators.jl:89-105
            for (const BCS* b : {&c->bu, &c->bv})
                for (const Side& sd : b->s)
                    if (sd.type != EFSI_BC_DIRICHLET && sd.type != EFSI_BC_PERIODIC)
                        arg_error("The current compact viscous operator supports Dirichlet or Periodic velocity boundaries.");
        c->proj.reset(make_projector(c->m, c->bq));
        c->U = F2(Nx + 1, Ny); c->V = F2(Nx, Ny + 1);
        c->phi = F2(Nx, Ny); c->c = F2(Nx, Ny);
        c->sxx = F2(Nx, Ny, 1.0); c->syy = F2(Nx, Ny, 1.0); c->sxy = F2(Nx, Ny);
        c->correction = F2(Nx, Ny);
    });
    if (st == EFSI_OK) *out = c.release();
    return st;
}

void oracle_destroy(Ctx* h) { delete h; }

const char* oracle_last_error(const Ctx* h) { return h ? h->err.c_str() : g_create_err.c_str(); }

int oracle_upload_state(Ctx* h, const double* U, const double* V, const double* phi, const double* c,
                        const double* sxx, const double* syy, const double* sxy) {
    return guarded(h, [&] {
        const int Nx = h->m.Nx, Ny = h->m.Ny;
        h->U = wrap(U, Nx + 1, Ny); h->V = wrap(V, Nx, Ny + 1);
        h->phi = wrap(phi, Nx, Ny);
        h->c = c ? wrap(c, Nx, Ny) : F2(Nx, Ny);  // legacy 6-array state (:116-118)
        h->sxx = wrap(sxx, Nx, Ny); h->syy = wrap(syy, Nx, Ny); h->sxy = wrap(sxy, Nx, Ny);
    });
}

int oracle_download_state(Ctx* h, double* U, double* V, double* phi, double* c, double* sxx,
                          double* syy, double* sxy) {
    return guarded(h, [&] {
        unwrap(h->U, U); unwrap(h->V, V); unwrap(h->phi, phi); unwrap(h->c, c);
        unwrap(h->sxx, sxx); unwrap(h->syy, syy); unwrap(h->sxy, sxy);
    });
}

int oracle_set_correction(Ctx* h, const double* q) {
    return guarded(h, [&] { h->correction = wrap(q, h->m.Nx, h->m.Ny); });
}
int oracle_get_correction(Ctx* h, double* q) {
    return guarded(h, [&] { unwrap(h->correction, q); });
}

int oracle_make_velocity_compatible(Ctx* h, efsi_projection_result* r) {  // :1088-1109
    return guarded(h, [&] {
        validate_state(*h, h->U, h->V, h->phi, h->c, h->sxx, h->syy, h->sxy);
        F2 G;
        growth_source(h->md, h->phi, h->c, G);
        ProjOut po = project(h->proj.get(), h->U, h->V, G, h->correction, h->nu.projection_reltol,
                             h->nu.projection_maxiter);
        h->stats.projection_iterations[0] = po.iters;
        if (r) {
            r->linear_relative_residual = po.linear_relative_residual;
            r->constraint_linf = po.constraint_linf;
            r->constraint_l2 = po.constraint_l2;
            r->compatibility_defect = po.compatibility_defect;
        }
    });
}

int oracle_integrate_step(Ctx* h, double t, double dt, efsi_step_report* rep) {
    return guarded(h, [&] {
        F2 U = h->U, V = h->V, phi = h->phi, c = h->c, sxx = h->sxx, syy = h->syy, sxy = h->sxy;
        F2 q = h->correction;
        try {
            integrate_step(*h, t, dt, rep);
        } catch (...) {  // a throwing step leaves the state untouched, as in Julia
            h->U = U; h->V = V; h->phi = phi; h->c = c; h->sxx = sxx; h->syy = syy; h->sxy = sxy;
            h->correction = q;
            throw;
        }
    });
}

int oracle_project(Ctx* h, double* U, double* V, const double* target, efsi_projection_result* r) {
    return guarded(h, [&] {
        const int Nx = h->m.Nx, Ny = h->m.Ny;
        F2 u = wrap(U, Nx + 1, Ny), v = wrap(V, Nx, Ny + 1), g = wrap(target, Nx, Ny);
        ProjOut po = project(h->proj.get(), u, v, g, h->correction, h->nu.projection_reltol,
                             h->nu.projection_maxiter);
        unwrap(u, U); unwrap(v, V);
        h->stats.projection_iterations[0] = po.iters;
        if (r) {
            r->linear_relative_residual = po.linear_relative_residual;
            r->constraint_linf = po.constraint_linf;
            r->constraint_l2 = po.constraint_l2;
            r->compatibility_defect = po.compatibility_defect;
        }
    });
}

int oracle_phase_field_rhs(Ctx* h, const double* U, const double* V, const double* phi,
                           const double* G, double* out) {
    return guarded(h, [&] {
        const int Nx = h->m.Nx, Ny = h->m.Ny;
        F2 r = phase_field_rhs(h->md, wrap(U, Nx + 1, Ny), wrap(V, Nx, Ny + 1), wrap(phi, Nx, Ny),
                               wrap(G, Nx, Ny), h->m, h->bphi);
        unwrap(r, out);
    });
}

int oracle_structure_tensor_rhs(Ctx* h, const double* sxx, const double* syy, const double* sxy,
                                const double* U, const double* V, const double* phi,
                                const double* G, double* rxx, double* ryy, double* rxy) {
    return guarded(h, [&] {
        const int Nx = h->m.Nx, Ny = h->m.Ny;
        F2 g = wrap(G, Nx, Ny), Kxx, Kxy, Kyx, Kyy;
        growth_tensor(h->md, g, Kxx, Kxy, Kyx, Kyy);
        F2 a, b, c;
        structure_tensor_rhs(wrap(sxx, Nx, Ny), wrap(syy, Nx, Ny), wrap(sxy, Nx, Ny),
                             wrap(U, Nx + 1, Ny), wrap(V, Nx, Ny + 1), Kxx, Kxy, Kyx, Kyy, h->md,
                             h->nu, h->m, h->bsig, h->bu, h->bv, wrap(phi, Nx, Ny), a, b, c);
        unwrap(a, rxx); unwrap(b, ryy); unwrap(c, rxy);
    });
}

int oracle_momentum_explicit_rhs(Ctx* h, double t, const double* U, const double* V,
                                 const double* phi, const double* sxx, const double* syy,
                                 const double* sxy, const double* G, double* Fx_out,
                                 double* Fy_out) {
    return guarded(h, [&] {
        const int Nx = h->m.Nx, Ny = h->m.Ny;
        F2 p = wrap(phi, Nx, Ny), g = wrap(G, Nx, Ny), Kxx, Kxy, Kyx, Kyy, mu, Fx, Fy;
        growth_tensor(h->md, g, Kxx, Kxy, Kyx, Kyy);
        viscosity_field(h->md, p, mu);
        momentum_forcing(*h, t, wrap(U, Nx + 1, Ny), wrap(V, Nx, Ny + 1), p, wrap(sxx, Nx, Ny),
                         wrap(syy, Nx, Ny), wrap(sxy, Nx, Ny), g, Kxx, Kxy, Kyx, Kyy, mu, Fx, Fy);
        unwrap(Fx, Fx_out);
        unwrap(Fy, Fy_out);
    });
}

int oracle_apply_viscous_operator(Ctx* h, const double* phi, const double* uv, double* out) {
    return guarded(h, [&] {
        const int Nx = h->m.Nx, Ny = h->m.Ny;
        const size_t N = (size_t)Nx * Ny;
        F2 mu;
        viscosity_field(h->md, wrap(phi, Nx, Ny), mu);
        if (h->md.viscosity == EFSI_VISC_NONE) arg_error("viscosity model is inactive");
        std::vector<double> x(uv, uv + 2 * N), y;
        viscous_apply(x, mu, h->m, h->bu, h->bv, true, y);
        std::memcpy(out, y.data(), sizeof(double) * 2 * N);
    });
}

int oracle_get_stats(const Ctx* h, efsi_stats* s) {
    if (s) *s = h->stats;
    return EFSI_OK;
}

// ---- primitives for the reference's known-answer tests -------------------------------
int oracle_structure_extension_rhs(double rate, double exponent, int n, const double* sxx,
                                   const double* syy, const double* sxy, const double* phi,
                                   double* rxx, double* ryy, double* rxy, char* msg, int msglen) {
    try {
        efsi_numerics nu{};
        nu.structure_extension = EFSI_EXT_GEOMETRIC;
        nu.extension_rate = rate;
        nu.extension_exponent = exponent;
        F2 a(n, 1), b(n, 1), c(n, 1), p(n, 1), o1, o2, o3;
        std::memcpy(a.a.data(), sxx, sizeof(double) * n);
        std::memcpy(b.a.data(), syy, sizeof(double) * n);
        std::memcpy(c.a.data(), sxy, sizeof(double) * n);
        std::memcpy(p.a.data(), phi, sizeof(double) * n);
        structure_extension_rhs(nu, a, b, c, p, o1, o2, o3);
        std::memcpy(rxx, o1.a.data(), sizeof(double) * n);
        std::memcpy(ryy, o2.a.data(), sizeof(double) * n);
        std::memcpy(rxy, o3.a.data(), sizeof(double) * n);
        return EFSI_OK;
    } catch (const Err& e) {
        if (msg && msglen > 0) { std::strncpy(msg, e.what(), msglen - 1); msg[msglen - 1] = 0; }
        return e.code;
    }
}

int oracle_apply_structure_extension(int kind, double cutoff, int n, double* sxx, double* syy,
                                     double* sxy, const double* phi) {
    efsi_numerics nu{};
    nu.structure_extension = kind;
    nu.extension_cutoff = cutoff;
    F2 a(n, 1), b(n, 1), c(n, 1), p(n, 1);
    std::memcpy(a.a.data(), sxx, sizeof(double) * n);
    std::memcpy(b.a.data(), syy, sizeof(double) * n);
    std::memcpy(c.a.data(), sxy, sizeof(double) * n);
    std::memcpy(p.a.data(), phi, sizeof(double) * n);
    int cnt = apply_structure_extension(nu, a, b, c, p);
    std::memcpy(sxx, a.a.data(), sizeof(double) * n);
    std::memcpy(syy, b.a.data(), sizeof(double) * n);
    std::memcpy(sxy, c.a.data(), sizeof(double) * n);
    return cnt;
}

void oracle_relaxation_rhs(double rate, int n, const double* sxx, const double* syy,
                           const double* sxy, double* rxx, double* ryy, double* rxy) {
    efsi_models md{};
    md.tensor_relaxation = EFSI_RELAX_MAXWELL;
    md.relaxation_rate = rate;
    for (int k = 0; k < n; ++k) relaxation_rhs(md, sxx[k], syy[k], sxy[k], rxx[k], ryy[k], rxy[k]);
}

void oracle_structure_tensor_diagnostics(int n, const double* sxx, const double* syy,
                                         const double* sxy, double* out4) {
    F2 a(n, 1), b(n, 1), c(n, 1);
    std::memcpy(a.a.data(), sxx, sizeof(double) * n);
    std::memcpy(b.a.data(), syy, sizeof(double) * n);
    std::memcpy(c.a.data(), sxy, sizeof(double) * n);
    SigmaDiag d = structure_tensor_diagnostics(a, b, c);
    out4[0] = d.min_det; out4[1] = d.max_abs_det_err; out4[2] = d.min_eig; out4[3] = (double)d.non_spd;
}

int oracle_body_force(Ctx* h, double t, double* Fx, double* Fy) {
    return guarded(h, [&] {
        F2 a, b;
        body_force(h->md, t, h->m, a, b);
        unwrap(a, Fx); unwrap(b, Fy);
    });
}

int oracle_uwcdi_strang_step(Ctx* h, const double* U, const double* V, const double* phi,
                             double dt, int x_first, double* out) {
    return guarded(h, [&] {
        const int Nx = h->m.Nx, Ny = h->m.Ny;
        if (h->md.phase_field_method != EFSI_PF_UWCDI) arg_error("context method is not UWCDI");
        F2 r = uwcdi_strang_step(h->md, wrap(U, Nx + 1, Ny), wrap(V, Nx, Ny + 1), wrap(phi, Nx, Ny),
                                 dt, h->m, h->bphi, x_first != 0);
        unwrap(r, out);
    });
}

int oracle_resource_explicit_rhs(Ctx* h, const double* U, const double* V, const double* c,
                                 const double* sink, double* out) {
    return guarded(h, [&] {
        const int Nx = h->m.Nx, Ny = h->m.Ny;
        F2 r = resource_explicit_rhs(wrap(U, Nx + 1, Ny), wrap(V, Nx, Ny + 1), wrap(c, Nx, Ny),
                                     wrap(sink, Nx, Ny), h->m, h->bc);
        unwrap(r, out);
    });
}

int oracle_constitutive_fields(Ctx* h, const double* phi, const double* c, double* G, double* Kxx,
                               double* Kxy, double* Kyx, double* Kyy, double* mu, double* D,
                               double* sink, double* trace_error) {
    return guarded(h, [&] {
        const int Nx = h->m.Nx, Ny = h->m.Ny;
        F2 p = wrap(phi, Nx, Ny), cc = wrap(c, Nx, Ny), g, a, b, e, d, m_, dd, s;
        growth_source(h->md, p, cc, g);
        growth_tensor(h->md, g, a, b, e, d);
        viscosity_field(h->md, p, m_);
        diffusivity_field(h->md, p, dd);
        resource_sink(h->md, p, cc, s);
        unwrap(g, G); unwrap(a, Kxx); unwrap(b, Kxy); unwrap(e, Kyx); unwrap(d, Kyy);
        unwrap(m_, mu); unwrap(dd, D); unwrap(s, sink);
        if (trace_error) *trace_error = growth_trace_error(g, a, d);
    });
}

int oracle_state_diagnostics(Ctx* h, const efsi_diag_config* cfg, efsi_diagnostics* out) {
    return guarded(h, [&] {
        if (!cfg || !out) arg_error("config and out must not be NULL");
        state_diagnostics(h->m, h->bphi, h->U, h->V, h->phi, h->sxx, h->syy, h->sxy, *cfg, *out);
    });
}

int oracle_tensor_cell_diagnostics(double sxx, double syy, double sxy, double phi, double modulus, double* out) {
    tensor_cell_diagnostics(sxx, syy, sxy, phi, modulus, out);
    return 0;
}

int oracle_divergence(Ctx* h, const double* U, const double* V, double* out) {
    return guarded(h, [&] {
        const int Nx = h->m.Nx, Ny = h->m.Ny;
        unwrap(divergence(wrap(U, Nx + 1, Ny), wrap(V, Nx, Ny + 1), h->m), out);
    });
}

}  // extern "C"
