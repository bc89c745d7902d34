// ccall_mirror.cpp — calls libefsi.so the way the Julia binding of INTEGRATION.md does:
// symbols looked up by name at run time (ccall((:name, LIBEFSI), ...)), argument lists
// spelled out from the ccall lines rather than taken from the header, and the 8-field
// StepReport and 4-field ProjectionResult read as the Julia isbits structs lay them out.
// The same sequence runs through the FP64 CPU oracle (liboracle_efsi.so, same ABI with
// the oracle_ prefix, used here as the checker), and the two must agree.
//
//   ccall_mirror <libefsi.so> <liboracle_efsi.so>      exit 0 on agreement
//
// Workload: the lid-driven cavity with one ACDI disk at N = 24 (the cavity configuration
// at a small size), make_velocity_compatible! and three integrate_step! calls.
#include <dlfcn.h>

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/efsi.h"

// Julia-side mirrors of the result structs (field order of TimeIntegrationIMEX.jl:318-327
// and Projection.jl:31-37); the header's layout must match them.
struct JlStepReport {
    double maximum_projection_constraint_linf, maximum_growth_trace_error, minimum_phi, maximum_phi,
        minimum_resource, minimum_sigma_eigenvalue, maximum_abs_sigma_determinant_error;
    int64_t non_spd_cells;
};
struct JlProjectionResult {
    double linear_relative_residual, constraint_linf, constraint_l2, compatibility_defect;
};
static_assert(sizeof(JlStepReport) == sizeof(efsi_step_report), "StepReport layout");
static_assert(offsetof(JlStepReport, non_spd_cells) == offsetof(efsi_step_report, non_spd_cells), "StepReport");
static_assert(sizeof(JlProjectionResult) == sizeof(efsi_projection_result), "ProjectionResult layout");

// The ccall signatures of INTEGRATION.md section 2.
using create_t = int (*)(const efsi_config*, void**);
using destroy_t = void (*)(void*);
using last_error_t = const char* (*)(void*);
using state7_t = int (*)(void*, double*, double*, double*, double*, double*, double*, double*);
using correction_t = int (*)(void*, double*);
using compatible_t = int (*)(void*, JlProjectionResult*);
using step_host_t = int (*)(void*, double*, double*, double*, double*, double*, double*, double*, double*, double,
                            double, JlStepReport*);
using step_t = int (*)(void*, double, double, JlStepReport*);

struct Lib {
    void* so = nullptr;
    const char* prefix = "";
    template <class F>
    F sym(const char* name) const {
        char buf[128];
        snprintf(buf, sizeof buf, "%s%s", prefix, name);
        void* p = dlsym(so, buf);
        if (!p) {
            fprintf(stderr, "missing symbol %s\n", buf);
            std::exit(2);
        }
        return reinterpret_cast<F>(p);
    }
};

int main(int argc, char** argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: ccall_mirror libefsi.so liboracle_efsi.so\n");
        return 2;
    }
    Lib gpu{dlopen(argv[1], RTLD_NOW | RTLD_LOCAL), "efsi_"};
    Lib ora{dlopen(argv[2], RTLD_NOW | RTLD_LOCAL), "oracle_"};
    if (!gpu.so || !ora.so) {
        fprintf(stderr, "dlopen: %s\n", dlerror());
        return 2;
    }

    const int N = 24;
    const double L = 1.0, h = L / N;
    // MeshMetrics of a uniform grid (MeshGeneration.jl:237-335)
    std::vector<double> dxf(N + 1, h), dxc(N, h), half_f(N + 1, 0.5), half_c(N, 0.5), corner(N + 1, 0.5 * h);
    efsi_config cfg;
    std::memset(&cfg, 0, sizeof cfg);
    cfg.abi_version = EFSI_ABI_VERSION;
    efsi_mesh& m = cfg.mesh;
    m.Nx = m.Ny = N;
    m.Lx = m.Ly = L;
    m.dx_f = m.dy_f = dxf.data();
    m.dx_c = m.dy_c = dxc.data();
    m.wL_c2fx = m.wR_c2fx = m.wB_c2fy = m.wT_c2fy = half_f.data();
    m.wL_f2cx = m.wR_f2cx = m.wB_f2cy = m.wT_f2cy = half_c.data();
    m.dx_west_corner = m.dx_east_corner = m.dy_south_corner = m.dy_north_corner = corner.data();
    // boundary data flattened on the host (BoundaryConditions.jl:103-136)
    std::vector<double> zeros(N + 1, 0.0), ones(N + 1, 1.0);
    auto side = [&](int type, const std::vector<double>& v) {
        efsi_bc_side s{};
        s.type = type;
        s.n = (int32_t)v.size();
        s.value = v.data();
        return s;
    };
    auto setup = [&](efsi_bc_side a, efsi_bc_side b, efsi_bc_side c, efsi_bc_side d) {
        efsi_bc_setup s;
        s.left = a;
        s.right = b;
        s.bottom = c;
        s.top = d;
        return s;
    };
    const efsi_bc_side wall = side(EFSI_BC_DIRICHLET, zeros), lid = side(EFSI_BC_DIRICHLET, ones),
                       noflux = side(EFSI_BC_NEUMANN, zeros);
    cfg.bc_U = setup(wall, wall, wall, lid);
    cfg.bc_V = setup(wall, wall, wall, wall);
    cfg.bc_correction = cfg.bc_phi = cfg.bc_resource = setup(noflux, noflux, noflux, noflux);
    cfg.bc_sigma_xx = cfg.bc_sigma_yy = cfg.bc_sigma_xy = cfg.bc_phi;
    // FSIModels of the cavity driver (run_sugiyama_lid_driven_cavity.jl:387-447)
    efsi_models& md = cfg.models;
    md.viscosity = EFSI_VISC_CONSTANT;
    md.viscosity_fluid = 0.01;
    md.elastic_stress = EFSI_ELASTIC_LINEAR;
    md.elastic_coefficient = 0.1;
    md.phase_field_method = EFSI_PF_ACDI;
    md.pf_param[0] = 1.0;
    md.pf_param[1] = 0.51 * h;
    md.pf_param[2] = 1e-100;
    md.pf_param[3] = 1e-14;
    md.pf_option = 0;
    efsi_numerics& nu = cfg.numerics;
    nu.structure_extension = EFSI_EXT_GEOMETRIC;
    nu.extension_rate = 20.0;
    nu.extension_exponent = 4.0;
    nu.extension_cutoff = 1e-6;
    nu.projection_reltol = 1e-13;
    nu.projection_maxiter = 3000;
    nu.stage1_constraint_atol = 5e-8;
    nu.stage1_constraint_rtol = 1e-8;
    nu.check_stage1_constraint = 1;
    nu.velocity_method = EFSI_LINEAR_DIRECT;
    nu.resource_method = EFSI_LINEAR_DIRECT;
    nu.linear_reltol = 1e-8;
    nu.linear_maxiter = 800;
    nu.direct_fallback = 1;
    nu.fallback_reltol = 1e-6;
    nu.precision = EFSI_PRECISION_FP64;

    // FSIState: rest, sigma = I, a tanh disk of radius 0.2 at (0.6, 0.5), width 1.5 h
    const size_t nc = (size_t)N * N, nf = (size_t)(N + 1) * N;
    struct State {
        std::vector<double> U, V, phi, c, sxx, syy, sxy, q;
    };
    auto initial = [&] {
        State s{std::vector<double>(nf, 0.0), std::vector<double>(nf, 0.0), std::vector<double>(nc),
                std::vector<double>(nc, 0.0), std::vector<double>(nc, 1.0), std::vector<double>(nc, 1.0),
                std::vector<double>(nc, 0.0), std::vector<double>(nc, 0.0)};
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < N; ++i) {
                const double x = (i + 0.5) * h, y = (j + 0.5) * h;
                const double d = std::hypot(x - 0.6, y - 0.5) - 0.2;
                s.phi[i + (size_t)j * N] = 0.5 * (1.0 - std::tanh(d / (1.5 * h)));
            }
        return s;
    };
    State sg = initial(), so = initial();
    const double dt = 0.2 * h;
    int fails = 0;

    // the CUDA library, exactly as the ccall lines of INTEGRATION.md section 2
    void* hg = nullptr;
    if (int st = gpu.sym<create_t>("create")(&cfg, &hg)) {
        fprintf(stderr, "efsi_create: %d %s\n", st, gpu.sym<last_error_t>("last_error")(nullptr));
        return 1;
    }
    auto check_g = [&](int st, const char* what) {
        if (st) {
            fprintf(stderr, "%s: %d %s\n", what, st, gpu.sym<last_error_t>("last_error")(hg));
            std::exit(1);
        }
    };
    JlProjectionResult pr{};
    check_g(gpu.sym<state7_t>("upload_state")(hg, sg.U.data(), sg.V.data(), sg.phi.data(), sg.c.data(),
                                                 sg.sxx.data(), sg.syy.data(), sg.sxy.data()),
            "upload");
    check_g(gpu.sym<correction_t>("set_correction")(hg, sg.q.data()), "set_correction");
    check_g(gpu.sym<compatible_t>("make_velocity_compatible")(hg, &pr), "make_velocity_compatible");
    check_g(gpu.sym<state7_t>("download_state")(hg, sg.U.data(), sg.V.data(), sg.phi.data(), sg.c.data(),
                                                   sg.sxx.data(), sg.syy.data(), sg.sxy.data()),
            "download");
    check_g(gpu.sym<correction_t>("get_correction")(hg, sg.q.data()), "get_correction");
    JlStepReport rg[3];
    for (int k = 0; k < 3; ++k)
        check_g(gpu.sym<step_host_t>("integrate_step_host")(hg, sg.U.data(), sg.V.data(), sg.phi.data(),
                                                            sg.c.data(), sg.sxx.data(), sg.syy.data(),
                                                            sg.sxy.data(), sg.q.data(), k * dt, dt, &rg[k]),
                "integrate_step_host");
    gpu.sym<destroy_t>("destroy")(hg);

    // the oracle (device-resident style entry points of the same ABI)
    void* ho = nullptr;
    if (ora.sym<create_t>("create")(&cfg, &ho)) {
        fprintf(stderr, "oracle_create failed\n");
        return 1;
    }
    JlProjectionResult po{};
    ora.sym<state7_t>("upload_state")(ho, so.U.data(), so.V.data(), so.phi.data(), so.c.data(), so.sxx.data(),
                                      so.syy.data(), so.sxy.data());
    ora.sym<correction_t>("set_correction")(ho, so.q.data());
    if (ora.sym<compatible_t>("make_velocity_compatible")(ho, &po)) {
        fprintf(stderr, "oracle projection failed\n");
        return 1;
    }
    JlStepReport ro[3];
    for (int k = 0; k < 3; ++k)
        if (ora.sym<step_t>("integrate_step")(ho, k * dt, dt, &ro[k])) {
            fprintf(stderr, "oracle step failed\n");
            return 1;
        }
    ora.sym<state7_t>("download_state")(ho, so.U.data(), so.V.data(), so.phi.data(), so.c.data(), so.sxx.data(),
                                        so.syy.data(), so.sxy.data());
    ora.sym<destroy_t>("destroy")(ho);

    auto rel = [](const std::vector<double>& a, const std::vector<double>& b) {
        double n = 0.0, d = 0.0;
        for (size_t k = 0; k < a.size(); ++k) {
            n += (a[k] - b[k]) * (a[k] - b[k]);
            d += b[k] * b[k];
        }
        return d > 0.0 ? std::sqrt(n / d) : std::sqrt(n);
    };
    const char* names[6] = {"U", "V", "phi", "sigma_xx", "sigma_yy", "sigma_xy"};
    const std::vector<double>* a[6] = {&sg.U, &sg.V, &sg.phi, &sg.sxx, &sg.syy, &sg.sxy};
    const std::vector<double>* b[6] = {&so.U, &so.V, &so.phi, &so.sxx, &so.syy, &so.sxy};
    for (int f = 0; f < 6; ++f) {
        const double e = rel(*a[f], *b[f]);
        printf("%-9s rel L2 %.3e\n", names[f], e);
        if (!(e <= 1e-10)) ++fails;
    }
    for (int k = 0; k < 3; ++k) {
        const double d[5] = {rg[k].minimum_phi - ro[k].minimum_phi, rg[k].maximum_phi - ro[k].maximum_phi,
                             rg[k].minimum_resource - ro[k].minimum_resource,
                             rg[k].minimum_sigma_eigenvalue - ro[k].minimum_sigma_eigenvalue,
                             rg[k].maximum_abs_sigma_determinant_error - ro[k].maximum_abs_sigma_determinant_error};
        for (double x : d)
            if (!(std::fabs(x) <= 1e-10)) ++fails;
        if (rg[k].non_spd_cells != ro[k].non_spd_cells) ++fails;
        if (!(rg[k].maximum_projection_constraint_linf <= 1e-9)) ++fails;
    }
    if (!(std::fabs(pr.constraint_linf) <= 1e-9 && std::fabs(po.constraint_linf) <= 1e-9)) ++fails;
    printf(fails ? "ccall mirror FAILED (%d)\n" : "ccall mirror ok\n", fails);
    return fails ? 1 : 0;
}
