// diagnostics.cpp — restatement of the cavity drivers' diagnostics
// (scripts/benchmarks/run_sugiyama_lid_driven_cavity.jl:484-828 and
// scripts/benchmarks/BenchmarkUtilities.jl:62-87).
// TEST INFRASTRUCTURE ONLY (the oracle); see oracle.hpp.  Loops run j outer,
// i inner, as the reference's `for j in 1:Ny, i in 1:Nx`.
#include <algorithm>
#include <cmath>
#include <limits>

#include "oracle.hpp"

namespace ora {

namespace {
const double kPi = 3.14159265358979323846;
const double kEps = 2.220446049250313e-16;

struct CellTensor {  // tensor_cell_diagnostics_2d, BenchmarkUtilities.jl:62-87
    double det, det_err, lmin, lmax, stress;
};
CellTensor cell_tensor(double xx, double yy, double xy, double phi, double modulus) {
    CellTensor t;
    t.det = xx * yy - xy * xy;
    const double tr = xx + yy;
    const double gap = std::hypot(xx - yy, 2.0 * xy);
    t.lmin = 0.5 * (tr - gap);
    t.lmax = 0.5 * (tr + gap);
    t.det_err = t.det - 1.0;
    t.stress = std::fabs(phi * modulus) * std::sqrt((xx - 1.0) * (xx - 1.0) + (yy - 1.0) * (yy - 1.0) + 2.0 * xy * xy);
    return t;
}
}  // namespace

void tensor_cell_diagnostics(double sxx, double syy, double sxy, double phi, double modulus, double out[5]) {
    CellTensor t = cell_tensor(sxx, syy, sxy, phi, modulus);
    out[0] = t.det; out[1] = t.det_err; out[2] = t.lmin; out[3] = t.lmax; out[4] = t.stress;
}

void state_diagnostics(const Mesh& m, const BCS& bphi, const F2& U, const F2& V, const F2& phi, const F2& sxx,
                       const F2& syy, const F2& sxy, const efsi_diag_config& cfg, efsi_diagnostics& out) {
    const int Nx = m.Nx, Ny = m.Ny;
    if (cfg.nmax < 0 || cfg.nmax > EFSI_DIAG_MAX_MODES) arg_error("nmax must lie in 0..8");
    out = efsi_diagnostics{};
    std::vector<double> xp(Nx), yp(Ny);  // cell centres of the grid
    for (int i = 0; i < Nx; ++i) xp[i] = (i + 0.5) * (m.Lx / Nx);
    for (int j = 0; j < Ny; ++j) yp[j] = (j + 0.5) * (m.Ly / Ny);
    auto area = [&](int i, int j) { return m.dx_c[i] * m.dy_c[j]; };
    // phase_centroid (:488-507)
    double mass = 0.0;
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) mass += phi(i, j) * area(i, j);
    if (!(mass > kEps)) arg_error("Phase integral is too small to define a centroid.");
    double xm = 0.0, ym = 0.0;
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            double w = phi(i, j) * area(i, j);
            xm += xp[i] * w;
            ym += yp[j] * w;
        }
    const double xc = xm / mass, yc = ym / mass;
    // phase_center_gradient (:600-613)
    F2 gxf, gyf;
    scalar_gradient(phi, m, bphi, gxf, gyf);
    // phase_geometry_diagnostics (:615-707)
    double perim = 0.0, mixed = 0.0, cxx = 0.0, cyy = 0.0, cxy = 0.0;
    double rc[EFSI_DIAG_MAX_MODES] = {}, rs[EFSI_DIAG_MAX_MODES] = {};
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            const double a = area(i, j), p = phi(i, j);
            const double pb = std::min(std::max(p, 0.0), 1.0);
            const double gx = m.wL_f2cx[i] * gxf(i, j) + m.wR_f2cx[i] * gxf(i + 1, j);
            const double gy = m.wB_f2cy[j] * gyf(i, j) + m.wT_f2cy[j] * gyf(i, j + 1);
            const double iw = a * std::hypot(gx, gy);
            perim += iw;
            mixed += a * 4.0 * pb * (1.0 - pb);
            const double dx = xp[i] - xc, dy = yp[j] - yc, mw = a * p;
            cxx += mw * dx * dx;
            cyy += mw * dy * dy;
            cxy += mw * dx * dy;
            const double th = std::atan2(dy, dx);
            for (int n = 1; n <= cfg.nmax; ++n) {
                rc[n - 1] += iw * std::cos(n * th) / kPi;
                rs[n - 1] += iw * std::sin(n * th) / kPi;
            }
        }
    cxx /= mass; cyy /= mass; cxy /= mass;
    const double gap = std::hypot(cxx - cyy, 2.0 * cxy);
    out.x_centroid = xc;
    out.y_centroid = yc;
    out.phase_integral = mass;
    out.perimeter_proxy = perim;
    out.mixed_layer_measure = mixed;
    out.effective_interface_width = perim > kEps ? mixed / perim : std::nan("");
    out.effective_interface_cells = out.effective_interface_width / cfg.h_interface;
    out.covariance_major = 0.5 * (cxx + cyy + gap);
    out.covariance_minor = 0.5 * (cxx + cyy - gap);
    out.aspect_ratio = out.covariance_minor > 0.0 ? std::sqrt(out.covariance_major / out.covariance_minor)
                                                  : std::numeric_limits<double>::infinity();
    out.orientation_radians = gap > 100.0 * kEps ? 0.5 * std::atan2(2.0 * cxy, cxx - cyy) : 0.0;
    out.R0 = perim / (2.0 * kPi);
    for (int n = 0; n < cfg.nmax; ++n) {
        out.Rc[n] = rc[n];
        out.Rs[n] = rs[n];
        out.amplitudes[n] = std::hypot(rc[n], rs[n]);
    }
    // phase_bound_diagnostics (:709-722)
    double pmin = std::numeric_limits<double>::infinity(), pmax = -pmin;
    long long oob = 0;
    for (double v : phi.a) {
        pmin = std::min(pmin, v);
        pmax = std::max(pmax, v);
        if (v < 0.0 || v > 1.0) ++oob;
    }
    out.phi_minimum = pmin;
    out.phi_maximum = pmax;
    out.lower_violation = std::max(0.0, -pmin);
    out.upper_violation = std::max(0.0, pmax - 1.0);
    out.out_of_bounds_cells = oob;
    // flow_diagnostics (:724-749)
    double ke = 0.0, vmax = 0.0, dl2 = 0.0, vol = 0.0, dinf = 0.0;
    F2 div = divergence(U, V, m);
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            const double u = 0.5 * (U(i, j) + U(i + 1, j)), v = 0.5 * (V(i, j) + V(i, j + 1));
            const double s2 = u * u + v * v;
            vmax = std::max(vmax, std::sqrt(s2));
            ke += 0.5 * cfg.density * s2 * area(i, j);
        }
    for (double d : div.a) dinf = std::max(dinf, std::fabs(d));
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            dl2 += area(i, j) * div(i, j) * div(i, j);
            vol += area(i, j);
        }
    out.maximum_speed = vmax;
    out.kinetic_energy = ke;
    out.divergence_linf = dinf;
    out.divergence_l2 = std::sqrt(dl2 / vol);
    // comparison_timestep_bounds inputs (:852-934)
    double mu = 0.0, mv = 0.0;
    for (double v : U.a) mu = std::max(mu, std::fabs(v));
    for (double v : V.a) mv = std::max(mv, std::fabs(v));
    out.max_abs_U = mu;
    out.max_abs_V = mv;
    // tensor_diagnostics_detailed (:739-828)
    for (int r = 0; r < 4; ++r) {
        auto sel = [&](double p) {
            switch (r) {
                case 0: return true;
                case 1: return p >= cfg.sigma_core_cutoff;
                case 2: return cfg.sigma_interface_cutoff < p && p < cfg.sigma_core_cutoff;
                default: return cfg.sigma_safety_cutoff < p && p <= cfg.sigma_interface_cutoff;
            }
        };
        efsi_tensor_region& g = out.tensor[r];
        double at = 0.0, dmin = std::numeric_limits<double>::infinity(), dmax = -dmin, mx_err = 0.0, mean_err = 0.0;
        double lmin = dmin, lmax = -dmin, mx_s = 0.0, mean_s = 0.0;
        long long cells = 0, nonspd = 0;
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                const double p = phi(i, j);
                if (!sel(p)) continue;
                const double a = area(i, j);
                CellTensor t = cell_tensor(sxx(i, j), syy(i, j), sxy(i, j), p, cfg.elastic_modulus);
                at += a;
                ++cells;
                dmin = std::min(dmin, t.det);
                dmax = std::max(dmax, t.det);
                const double de = std::fabs(t.det_err);
                mx_err = std::max(mx_err, de);
                mean_err += a * de;
                lmin = std::min(lmin, t.lmin);
                lmax = std::max(lmax, t.lmax);
                if (!(std::isfinite(t.lmin) && t.lmin > 0.0)) ++nonspd;
                mx_s = std::max(mx_s, t.stress);
                mean_s += a * t.stress;
            }
        const double nan = std::nan("");
        if (cells == 0 || at == 0.0) {
            g = efsi_tensor_region{0, 0.0, nan, nan, nan, nan, nan, nan, 0, nan, nan};
        } else {
            g = efsi_tensor_region{cells, at, dmin, dmax, mx_err, mean_err / at, lmin, lmax, nonspd, mx_s,
                                   mean_s / at};
        }
    }
}

}  // namespace ora
