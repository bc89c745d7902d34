// physics.cpp — restatement of MomentumTransport.jl, InterfaceTransport.jl,
// InterfaceRegularization.jl, PhaseFieldMethods.jl, StructureTensor.jl,
// StructuralConstitutive.jl, Capillarity.jl, TransportConstitutive.jl,
// GrowthModels.jl and ResourceTransport.jl.
// TEST INFRASTRUCTURE ONLY (the oracle); see oracle.hpp.
#include <algorithm>
#include <cmath>

#include "oracle.hpp"

namespace ora {

static inline double clamp01(double x) { return std::min(std::max(x, 0.0), 1.0); }

// ---- MomentumTransport.jl ----------------------------------------------------------
static double tangential_u(const F2& U, int ii, bool top, const Mesh& m, const BCS& bu) {  // :68-103
    const Side& s = top ? bu.top() : bu.bottom();
    double adjacent = top ? U(ii, m.Ny - 1) : U(ii, 0);
    double dist = top ? m.dy_f[m.Ny] / 2.0 : m.dy_f[0] / 2.0;
    if (s.type == EFSI_BC_DIRICHLET) return s.val(ii);
    if (s.type == EFSI_BC_NEUMANN) return adjacent + s.val(ii) * dist;
    if (s.type == EFSI_BC_PERIODIC)
        arg_error("Periodic transverse U values must be handled through periodic interpolation.");
    arg_error("Unsupported U boundary condition.");
}
static double tangential_v(const F2& V, int jj, bool right, const Mesh& m, const BCS& bv) {  // :105-137
    const Side& s = right ? bv.right() : bv.left();
    double adjacent = right ? V(m.Nx - 1, jj) : V(0, jj);
    double dist = right ? m.dx_f[m.Nx] / 2.0 : m.dx_f[0] / 2.0;
    if (s.type == EFSI_BC_DIRICHLET) return s.val(jj);
    if (s.type == EFSI_BC_NEUMANN) return adjacent + s.val(jj) * dist;
    if (s.type == EFSI_BC_PERIODIC)
        arg_error("Periodic transverse V values must be handled through periodic interpolation.");
    arg_error("Unsupported V boundary condition.");
}

void material_convection(const F2& U, const F2& V, const F2& S, const Mesh& m, const BCS& bu,
                         const BCS& bv, F2& Cu, F2& Cv) {
    const int Nx = m.Nx, Ny = m.Ny;
    if (m.px != bu.periodic_x() || m.py != bu.periodic_y() || m.px != bv.periodic_x() ||
        m.py != bv.periodic_y())
        arg_error("U/V boundary conditions do not match MeshMetrics periodicity.");
    F2 u2(Nx, Ny), v2(Nx, Ny);  // :141-159
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            double ur = (m.px && i == Nx - 1) ? U(0, j) : U(i + 1, j);
            double uc = m.wL_f2cx[i] * U(i, j) + m.wR_f2cx[i] * ur;
            u2(i, j) = uc * uc;
            double vt = (m.py && j == Ny - 1) ? V(i, 0) : V(i, j + 1);
            double vc = m.wB_f2cy[j] * V(i, j) + m.wT_f2cy[j] * vt;
            v2(i, j) = vc * vc;
        }
    F2 uv(Nx + 1, Ny + 1);  // :221-247
    for (int j = 0; j <= Ny; ++j)
        for (int i = 0; i <= Nx; ++i) {
            int ii = (m.px && i == Nx) ? 0 : i;
            double uc;
            if (m.py) {
                if (j == 0 || j == Ny) uc = m.wB_c2fy[0] * U(ii, Ny - 1) + m.wT_c2fy[0] * U(ii, 0);
                else uc = m.wB_c2fy[j] * U(ii, j - 1) + m.wT_c2fy[j] * U(ii, j);
            } else if (j == 0) uc = tangential_u(U, ii, false, m, bu);
            else if (j == Ny) uc = tangential_u(U, ii, true, m, bu);
            else uc = m.wB_c2fy[j] * U(ii, j - 1) + m.wT_c2fy[j] * U(ii, j);
            int jj = (m.py && j == Ny) ? 0 : j;
            double vc;
            if (m.px) {
                if (i == 0 || i == Nx) vc = m.wL_c2fx[0] * V(Nx - 1, jj) + m.wR_c2fx[0] * V(0, jj);
                else vc = m.wL_c2fx[i] * V(i - 1, jj) + m.wR_c2fx[i] * V(i, jj);
            } else if (i == 0) vc = tangential_v(V, jj, false, m, bv);
            else if (i == Nx) vc = tangential_v(V, jj, true, m, bv);
            else vc = m.wL_c2fx[i] * V(i - 1, jj) + m.wR_c2fx[i] * V(i, jj);
            uv(i, j) = uc * vc;
        }
    if (m.px)
        for (int j = 0; j <= Ny; ++j) uv(Nx, j) = uv(0, j);
    if (m.py)
        for (int i = 0; i <= Nx; ++i) uv(i, Ny) = uv(i, 0);
    Cu = F2(Nx + 1, Ny);  // :266-297
    Cv = F2(Nx, Ny + 1);
    for (int j = 0; j < Ny; ++j) {
        if (m.px) {
            Cu(0, j) = (u2(0, j) - u2(Nx - 1, j)) / m.dx_f[0] + (uv(0, j + 1) - uv(0, j)) / m.dy_c[j];
            Cu(Nx, j) = Cu(0, j);
        }
        for (int i = 1; i < Nx; ++i)
            Cu(i, j) = (u2(i, j) - u2(i - 1, j)) / m.dx_f[i] + (uv(i, j + 1) - uv(i, j)) / m.dy_c[j];
    }
    for (int i = 0; i < Nx; ++i) {
        if (m.py) {
            Cv(i, 0) = (uv(i + 1, 0) - uv(i, 0)) / m.dx_c[i] + (v2(i, 0) - v2(i, Ny - 1)) / m.dy_f[0];
            Cv(i, Ny) = Cv(i, 0);
        }
        for (int j = 1; j < Ny; ++j)
            Cv(i, j) = (uv(i + 1, j) - uv(i, j)) / m.dx_c[i] + (v2(i, j) - v2(i, j - 1)) / m.dy_f[j];
    }
    F2 Sx = interp_c2fx(S, m), Sy = interp_c2fy(S, m);  // :311-336
    for (size_t k = 0; k < Cu.size(); ++k) Cu.a[k] -= Sx.a[k] * U.a[k];
    for (size_t k = 0; k < Cv.size(); ++k) Cv.a[k] -= Sy.a[k] * V.a[k];
    if (m.px) {
        for (int j = 0; j < Ny; ++j) Cu(Nx, j) = Cu(0, j);
    } else {
        for (int j = 0; j < Ny; ++j) { Cu(0, j) = 0.0; Cu(Nx, j) = 0.0; }
    }
    if (m.py) {
        for (int i = 0; i < Nx; ++i) Cv(i, Ny) = Cv(i, 0);
    } else {
        for (int i = 0; i < Nx; ++i) { Cv(i, 0) = 0.0; Cv(i, Ny) = 0.0; }
    }
}

// ---- first-order upwind conservative advection --------------------------------------
// Shared by InterfaceTransport.jl:83-233, StructureTensor.jl:191-343 and
// ResourceTransport.jl:103-271; `allow_outflow` selects the resource rule that
// AdvectiveOutflow supplies its backflow value.
static double inflow_state(const Side& s, int k, double interior, double vel, bool low_side,
                           bool allow_outflow, const char* what) {
    if (vel == 0.0) return interior;
    bool inflow = low_side ? vel > 0.0 : vel < 0.0;
    if (!inflow) return interior;
    if (s.type == EFSI_BC_DIRICHLET) return s.val(k);
    if (allow_outflow && s.type == EFSI_BC_ADVECTIVE_OUTFLOW) return s.val(k);
    if (s.type == EFSI_BC_NEUMANN)
        arg_error(std::string("A Neumann ") + what +
                  " condition does not define the incoming advected state. Prescribe Dirichlet data for inflow.");
    if (s.type == EFSI_BC_PERIODIC) arg_error("Periodic boundary states must be handled by wrapping.");
    arg_error(std::string("Unsupported ") + what + " boundary condition.");
}

static F2 upwind_advection(const F2& U, const F2& V, const F2& q, const Mesh& m, const BCS& bc,
                           bool allow_outflow, const char* what) {
    const int Nx = m.Nx, Ny = m.Ny;
    F2 fx(Nx + 1, Ny), fy(Nx, Ny + 1);
    for (int j = 0; j < Ny; ++j) {
        double u = U(0, j);
        if (m.px) {
            fx(0, j) = u * (u >= 0.0 ? q(Nx - 1, j) : q(0, j));
        } else {
            double b = inflow_state(bc.left(), j, q(0, j), u, true, allow_outflow, what);
            fx(0, j) = u * (u >= 0.0 ? b : q(0, j));
        }
        for (int i = 1; i < Nx; ++i) {
            u = U(i, j);
            fx(i, j) = u * (u >= 0.0 ? q(i - 1, j) : q(i, j));
        }
        if (m.px) {
            fx(Nx, j) = fx(0, j);
        } else {
            u = U(Nx, j);
            double b = inflow_state(bc.right(), j, q(Nx - 1, j), u, false, allow_outflow, what);
            fx(Nx, j) = u * (u >= 0.0 ? q(Nx - 1, j) : b);
        }
    }
    for (int i = 0; i < Nx; ++i) {
        double v = V(i, 0);
        if (m.py) {
            fy(i, 0) = v * (v >= 0.0 ? q(i, Ny - 1) : q(i, 0));
        } else {
            double b = inflow_state(bc.bottom(), i, q(i, 0), v, true, allow_outflow, what);
            fy(i, 0) = v * (v >= 0.0 ? b : q(i, 0));
        }
        for (int j = 1; j < Ny; ++j) {
            v = V(i, j);
            fy(i, j) = v * (v >= 0.0 ? q(i, j - 1) : q(i, j));
        }
        if (m.py) {
            fy(i, Ny) = fy(i, 0);
        } else {
            v = V(i, Ny);
            double b = inflow_state(bc.top(), i, q(i, Ny - 1), v, false, allow_outflow, what);
            fy(i, Ny) = v * (v >= 0.0 ? q(i, Ny - 1) : b);
        }
    }
    F2 r(Nx, Ny);
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i)
            r(i, j) = -((fx(i + 1, j) - fx(i, j)) / m.dx_c[i] + (fy(i, j + 1) - fy(i, j)) / m.dy_c[j]);
    return r;
}

// ---- phase-field helpers (PhaseFieldMethods.jl:174-404) -----------------------------
static double phase_boundary_value(const Side& s, int k, double interior) {  // :174-196
    const double tiny = 100 * 2.220446049250313e-16;
    switch (s.type) {
        case EFSI_BC_DIRICHLET: return s.val(k);
        case EFSI_BC_NEUMANN:
            if (std::fabs(s.val(k)) > tiny)
                arg_error("Only homogeneous Neumann phase boundaries are supported by the ACDI/UWCDI operators.");
            return interior;
        case EFSI_BC_ADVECTIVE_OUTFLOW: return interior;
        case EFSI_BC_MIXED:
            if (s.is_dir(k)) return s.val(k);
            if (std::fabs(s.neu(k)) > tiny)
                arg_error("Only homogeneous-Neumann mixed phase faces are supported here.");
            return interior;
    }
    arg_error("Unsupported phase boundary condition.");
}

// Cell-centred gradient from face gradients (:219-231, InterfaceRegularization.jl:99-121).
static void center_gradient(const F2& f, const Mesh& m, const BCS& bc, F2& gx, F2& gy, F2& gxf,
                            F2& gyf) {
    scalar_gradient(f, m, bc, gxf, gyf);
    gx = F2(m.Nx, m.Ny); gy = F2(m.Nx, m.Ny);
    for (int j = 0; j < m.Ny; ++j)
        for (int i = 0; i < m.Nx; ++i) {
            gx(i, j) = m.wL_f2cx[i] * gxf(i, j) + m.wR_f2cx[i] * gxf(i + 1, j);
            gy(i, j) = m.wB_f2cy[j] * gyf(i, j) + m.wT_f2cy[j] * gyf(i, j + 1);
        }
}

static void center_normals(const F2& f, const Mesh& m, const BCS& bc, double delta, F2& nx,
                           F2& ny) {  // :233-244
    F2 gx, gy, gxf, gyf;
    center_gradient(f, m, bc, gx, gy, gxf, gyf);
    nx = F2(m.Nx, m.Ny); ny = F2(m.Nx, m.Ny);
    double d2 = delta * delta;
    for (size_t k = 0; k < gx.size(); ++k) {
        double mag = std::sqrt(gx.a[k] * gx.a[k] + gy.a[k] * gy.a[k] + d2);
        nx.a[k] = gx.a[k] / mag;
        ny.a[k] = gy.a[k] / mag;
    }
}

static void face_normals_from_centers(const F2& nxc, const F2& nyc, const Mesh& m, double delta,
                                      F2& nxf, F2& nyf) {  // :246-273
    nxf = interp_c2fx(nxc, m);
    nyf = interp_c2fy(nyc, m);
    F2 ny_on_x = interp_c2fx(nyc, m), nx_on_y = interp_c2fy(nxc, m);
    double d2 = delta * delta;
    for (int j = 0; j < m.Ny; ++j)
        for (int i = 0; i <= m.Nx; ++i)
            nxf(i, j) /= std::sqrt(nxf(i, j) * nxf(i, j) + ny_on_x(i, j) * ny_on_x(i, j) + d2);
    for (int j = 0; j <= m.Ny; ++j)
        for (int i = 0; i < m.Nx; ++i)
            nyf(i, j) /= std::sqrt(nx_on_y(i, j) * nx_on_y(i, j) + nyf(i, j) * nyf(i, j) + d2);
    if (m.px)
        for (int j = 0; j < m.Ny; ++j) nxf(m.Nx, j) = nxf(0, j);
    if (m.py)
        for (int i = 0; i < m.Nx; ++i) nyf(i, m.Ny) = nyf(i, 0);
}

static void youngs_center_normals(const F2& f, const Mesh& m, const BCS& bc, double delta, F2& nx,
                                  F2& ny) {  // :285-337
    double hx = m.dx_c[0], hy = m.dy_c[0];
    double tolx = 100 * 2.220446049250313e-16 * std::max(1.0, std::fabs(hx));
    double toly = 100 * 2.220446049250313e-16 * std::max(1.0, std::fabs(hy));
    for (double d : m.dx_c)
        if (std::fabs(d - hx) > tolx) arg_error("Youngs normal reconstruction currently requires a uniform x grid.");
    for (double d : m.dy_c)
        if (std::fabs(d - hy) > toly) arg_error("Youngs normal reconstruction currently requires a uniform y grid.");
    center_normals(f, m, bc, delta, nx, ny);
    const int Nx = m.Nx, Ny = m.Ny;
    double d2 = delta * delta;
    auto wrap = [](int k, int n, bool p) { return p ? ((k % n) + n) % n : k; };
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            if ((!m.px && (i == 0 || i == Nx - 1)) || (!m.py && (j == 0 || j == Ny - 1))) continue;
            int im = wrap(i - 1, Nx, m.px), ip = wrap(i + 1, Nx, m.px);
            int jm = wrap(j - 1, Ny, m.py), jp = wrap(j + 1, Ny, m.py);
            double gx = (f(ip, jm) + 2.0 * f(ip, j) + f(ip, jp) - f(im, jm) - 2.0 * f(im, j) - f(im, jp)) / (8.0 * hx);
            double gy = (f(im, jp) + 2.0 * f(i, jp) + f(ip, jp) - f(im, jm) - 2.0 * f(i, jm) - f(ip, jm)) / (8.0 * hy);
            double mag = std::sqrt(gx * gx + gy * gy + d2);
            nx(i, j) = gx / mag;
            ny(i, j) = gy / mag;
        }
}

static F2 smoothed9(const F2& f, const Mesh& m, const BCS& bc) {  // :347-397
    for (int k = 0; k < 4; ++k) {
        const Side& s = bc.s[k];
        if (s.type == EFSI_BC_PERIODIC) continue;
        if (s.type == EFSI_BC_NEUMANN) {
            if (std::fabs(s.val(0)) > 100 * 2.220446049250313e-16)
                arg_error("smoothed9 normal reconstruction requires homogeneous Neumann or periodic phase boundaries.");
        } else {
            arg_error("smoothed9 normal reconstruction requires homogeneous Neumann or periodic phase boundaries.");
        }
    }
    const int Nx = m.Nx, Ny = m.Ny;
    auto ix = [&](int k, int n, bool p) { return p ? ((k % n) + n) % n : std::min(std::max(k, 0), n - 1); };
    F2 s(Nx, Ny);
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            int im = ix(i - 1, Nx, m.px), ip = ix(i + 1, Nx, m.px);
            int jm = ix(j - 1, Ny, m.py), jp = ix(j + 1, Ny, m.py);
            s(i, j) = 0.25 * f(i, j) + 0.125 * (f(ip, j) + f(im, j) + f(i, jp) + f(i, jm)) +
                      0.0625 * (f(ip, jp) + f(im, jp) + f(ip, jm) + f(im, jm));
        }
    return s;
}

// ---- CDI (InterfaceRegularization.jl:123-228) and the legacy split path -----------
static void cdi_flux(double ip, double eps, double delta, const F2& phi, const Mesh& m,
                     const BCS& bphi, F2& jx, F2& jy) {
    F2 gx, gy, gxf, gyf;
    center_gradient(phi, m, bphi, gx, gy, gxf, gyf);
    F2 sx(m.Nx, m.Ny), sy(m.Nx, m.Ny);
    double d2 = delta * delta;
    for (size_t k = 0; k < phi.size(); ++k) {
        double mag = std::sqrt(gx.a[k] * gx.a[k] + gy.a[k] * gy.a[k] + d2);
        double amp = phi.a[k] * (1.0 - phi.a[k]);
        sx.a[k] = amp * gx.a[k] / mag;
        sy.a[k] = amp * gy.a[k] / mag;
    }
    F2 sxf = interp_c2fx(sx, m), syf = interp_c2fy(sy, m);
    double ell = 0.5 * eps;
    jx = F2(m.Nx + 1, m.Ny); jy = F2(m.Nx, m.Ny + 1);
    for (size_t k = 0; k < jx.size(); ++k) jx.a[k] = ip * (sxf.a[k] - ell * gxf.a[k]);
    for (size_t k = 0; k < jy.size(); ++k) jy.a[k] = ip * (syf.a[k] - ell * gyf.a[k]);
    for (int j = 0; j < m.Ny; ++j) {  // :147-167
        if (m.px) jx(m.Nx, j) = jx(0, j);
        else { jx(0, j) = 0.0; jx(m.Nx, j) = 0.0; }
    }
    for (int i = 0; i < m.Nx; ++i) {
        if (m.py) jy(i, m.Ny) = jy(i, 0);
        else { jy(i, 0) = 0.0; jy(i, m.Ny) = 0.0; }
    }
}

// ---- ACDI (PhaseFieldMethods.jl:479-671) -----------------------------------------
static double psi_value(double phi, double eps, double floor_) {  // :479-483
    double p = clamp01(phi);
    return eps * std::log((p + floor_) / (1.0 - p + floor_));
}

static BCS psi_bcs(const BCS& b, double eps, double floor_) {  // :493-529
    BCS r = b;
    for (int k = 0; k < 4; ++k) {
        Side& s = r.s[k];
        if (s.type == EFSI_BC_PERIODIC) continue;
        if (s.type == EFSI_BC_NEUMANN) {
            if (std::fabs(b.s[k].val(0)) > 100 * 2.220446049250313e-16)
                arg_error("ACDI currently supports only homogeneous Neumann phase gradients.");
            std::fill(s.value.begin(), s.value.end(), 0.0);
        } else if (s.type == EFSI_BC_DIRICHLET) {
            double v0 = b.s[k].val(0);
            for (double v : b.s[k].value)
                if (v != v0) arg_error("ACDI psi transformation currently requires scalar Dirichlet phase data.");
            std::fill(s.value.begin(), s.value.end(), psi_value(v0, eps, floor_));
        } else {
            arg_error("ACDI psi geometry supports Periodic, homogeneous Neumann, or scalar Dirichlet phase boundaries.");
        }
    }
    return r;
}

static F2 acdi_rhs(const efsi_models& md, const F2& U, const F2& V, const F2& phi, const F2& S,
                   const Mesh& m, const BCS& bphi) {
    const int Nx = m.Nx, Ny = m.Ny;
    const double gamma = md.pf_param[0], eps = md.pf_param[1], floor_ = md.pf_param[2],
                 delta = md.pf_param[3];
    // Central convective fluxes (:531-574).
    F2 fx(Nx + 1, Ny), fy(Nx, Ny + 1);
    for (int j = 0; j < Ny; ++j) {
        if (m.px) {
            double pf = m.wL_c2fx[0] * phi(Nx - 1, j) + m.wR_c2fx[0] * phi(0, j);
            fx(0, j) = U(0, j) * pf;
            fx(Nx, j) = fx(0, j);
        } else {
            fx(0, j) = U(0, j) * phase_boundary_value(bphi.left(), j, phi(0, j));
            fx(Nx, j) = U(Nx, j) * phase_boundary_value(bphi.right(), j, phi(Nx - 1, j));
        }
        for (int i = 1; i < Nx; ++i)
            fx(i, j) = U(i, j) * (m.wL_c2fx[i] * phi(i - 1, j) + m.wR_c2fx[i] * phi(i, j));
    }
    for (int i = 0; i < Nx; ++i) {
        if (m.py) {
            double pf = m.wB_c2fy[0] * phi(i, Ny - 1) + m.wT_c2fy[0] * phi(i, 0);
            fy(i, 0) = V(i, 0) * pf;
            fy(i, Ny) = fy(i, 0);
        } else {
            fy(i, 0) = V(i, 0) * phase_boundary_value(bphi.bottom(), i, phi(i, 0));
            fy(i, Ny) = V(i, Ny) * phase_boundary_value(bphi.top(), i, phi(i, Ny - 1));
        }
        for (int j = 1; j < Ny; ++j)
            fy(i, j) = V(i, j) * (m.wB_c2fy[j] * phi(i, j - 1) + m.wT_c2fy[j] * phi(i, j));
    }
    // Regularisation fluxes (:598-650).
    F2 psi(Nx, Ny);
    for (size_t k = 0; k < psi.size(); ++k) psi.a[k] = psi_value(phi.a[k], eps, floor_);
    BCS bpsi = psi_bcs(bphi, eps, floor_);
    F2 gx, gy, gpx, gpy;
    center_gradient(phi, m, bphi, gx, gy, gpx, gpy);
    F2 nxc, nyc;
    center_normals(psi, m, bpsi, delta, nxc, nyc);
    F2 nxf = interp_c2fx(nxc, m), nyf = interp_c2fy(nyc, m);
    F2 psx = interp_c2fx(psi, m), psy = interp_c2fy(psi, m);
    double geff = gamma;  // :576-596
    if (md.pf_option) {
        double umax = 0.0;
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                double uc = m.wL_f2cx[i] * U(i, j) + m.wR_f2cx[i] * U(i + 1, j);
                double vc = m.wB_f2cy[j] * V(i, j) + m.wT_f2cy[j] * V(i, j + 1);
                umax = std::max(umax, std::hypot(uc, vc));
            }
        geff = gamma * umax;
    }
    F2 Ax(Nx + 1, Ny), Ay(Nx, Ny + 1);
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i <= Nx; ++i) {
            double t = std::tanh(psx(i, j) / (2.0 * eps));
            double amp = 0.25 * (1.0 - t * t);
            Ax(i, j) = geff * (eps * gpx(i, j) - amp * nxf(i, j));
        }
    for (int j = 0; j <= Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            double t = std::tanh(psy(i, j) / (2.0 * eps));
            double amp = 0.25 * (1.0 - t * t);
            Ay(i, j) = geff * (eps * gpy(i, j) - amp * nyf(i, j));
        }
    for (int j = 0; j < Ny; ++j) {
        if (m.px) Ax(Nx, j) = Ax(0, j);
        else { Ax(0, j) = 0.0; Ax(Nx, j) = 0.0; }
    }
    for (int i = 0; i < Nx; ++i) {
        if (m.py) Ay(i, Ny) = Ay(i, 0);
        else { Ay(i, 0) = 0.0; Ay(i, Ny) = 0.0; }
    }
    F2 df = divergence(fx, fy, m), dA = divergence(Ax, Ay, m);  // :668-670
    F2 r(Nx, Ny);
    for (size_t k = 0; k < r.size(); ++k) r.a[k] = -df.a[k] + dA.a[k] + phi.a[k] * S.a[k];
    return r;
}

// ---- UWCDI (PhaseFieldMethods.jl:675-867) ----------------------------------------
static void uwcdi_fluxes(const efsi_models& md, const F2& U, const F2& V, const F2& phi,
                         const Mesh& m, const BCS& bphi, F2& fx, F2& fy) {
    const int Nx = m.Nx, Ny = m.Ny;
    const double alpha = md.pf_param[0], delta = md.pf_param[1];
    F2 nxf, nyf;
    if (md.pf_option == EFSI_NORMALS_STANDARD) {
        F2 nxc, nyc;
        center_normals(phi, m, bphi, delta, nxc, nyc);
        face_normals_from_centers(nxc, nyc, m, delta, nxf, nyf);
    } else if (md.pf_option == EFSI_NORMALS_YOUNGS) {
        F2 nxc, nyc;
        youngs_center_normals(phi, m, bphi, delta, nxc, nyc);
        face_normals_from_centers(nxc, nyc, m, delta, nxf, nyf);
    } else if (md.pf_option == EFSI_NORMALS_SMOOTHED9) {
        F2 sm = smoothed9(phi, m, bphi);
        F2 nxc, nyc;
        center_normals(sm, m, bphi, delta, nxc, nyc);
        face_normals_from_centers(nxc, nyc, m, delta, nxf, nyf);
    } else {
        arg_error("Unsupported UWCDI normal reconstruction.");
    }
    fx = F2(Nx + 1, Ny); fy = F2(Nx, Ny + 1);
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i <= Nx; ++i) {
            double u = U(i, j), up;
            if (!m.px && i == 0) {
                double b = phase_boundary_value(bphi.left(), j, phi(0, j));
                up = u >= 0.0 ? b : phi(0, j);
            } else if (!m.px && i == Nx) {
                double b = phase_boundary_value(bphi.right(), j, phi(Nx - 1, j));
                up = u >= 0.0 ? phi(Nx - 1, j) : b;
            } else {
                int iL = i == 0 ? Nx - 1 : (i == Nx ? Nx - 1 : i - 1);
                int iR = i == 0 ? 0 : (i == Nx ? 0 : i);
                up = u >= 0.0 ? phi(iL, j) : phi(iR, j);
            }
            double ax = alpha * std::max(1.0, m.dy_c[j] / m.dx_f[i]);
            double bx = std::fabs(u) / ax;
            fx(i, j) = up * (u + bx * nxf(i, j) * (1.0 - up));
        }
    for (int j = 0; j <= Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            double v = V(i, j), up;
            if (!m.py && j == 0) {
                double b = phase_boundary_value(bphi.bottom(), i, phi(i, 0));
                up = v >= 0.0 ? b : phi(i, 0);
            } else if (!m.py && j == Ny) {
                double b = phase_boundary_value(bphi.top(), i, phi(i, Ny - 1));
                up = v >= 0.0 ? phi(i, Ny - 1) : b;
            } else {
                int jB = j == 0 ? Ny - 1 : (j == Ny ? Ny - 1 : j - 1);
                int jT = j == 0 ? 0 : (j == Ny ? 0 : j);
                up = v >= 0.0 ? phi(i, jB) : phi(i, jT);
            }
            double ay = alpha * std::max(1.0, m.dx_c[i] / m.dy_f[j]);
            double by = std::fabs(v) / ay;
            fy(i, j) = up * (v + by * nyf(i, j) * (1.0 - up));
        }
    if (m.px)
        for (int j = 0; j < Ny; ++j) fx(Nx, j) = fx(0, j);
    if (m.py)
        for (int i = 0; i < Nx; ++i) fy(i, Ny) = fy(i, 0);
}

F2 uwcdi_strang_step(const efsi_models& md, const F2& U, const F2& V, const F2& phi, double dt,
                     const Mesh& m, const BCS& bphi, bool x_first) {
    auto sweep = [&](bool dir_x, const F2& q, double h) {
        if (h == 0.0) return q;
        F2 fx, fy;
        uwcdi_fluxes(md, U, V, q, m, bphi, fx, fy);
        if (dir_x) std::fill(fy.a.begin(), fy.a.end(), 0.0);
        else std::fill(fx.a.begin(), fx.a.end(), 0.0);
        F2 d = divergence(fx, fy, m);
        F2 out = q;
        for (size_t k = 0; k < out.size(); ++k) out.a[k] = q.a[k] + h * (-d.a[k]);
        return out;
    };
    F2 q1 = sweep(x_first, phi, 0.5 * dt);
    F2 q2 = sweep(!x_first, q1, dt);
    return sweep(x_first, q2, 0.5 * dt);
}

F2 phase_field_rhs(const efsi_models& md, const F2& U, const F2& V, const F2& phi, const F2& S,
                   const Mesh& m, const BCS& bphi) {
    if (m.px != bphi.periodic_x() || m.py != bphi.periodic_y())
        arg_error("phi boundary conditions do not match MeshMetrics periodicity.");
    for (double v : phi.a)
        if (!std::isfinite(v)) arg_error("phi contains non-finite values.");
    switch (md.phase_field_method) {
        case EFSI_PF_UPWIND:
        case EFSI_PF_CDI: {  // PhaseFieldMethods.jl:408-475 -> InterfaceTransport.jl:260-276
            F2 adv = upwind_advection(U, V, phi, m, bphi, false, "phi");
            F2 r(m.Nx, m.Ny);
            F2 dj(m.Nx, m.Ny);
            if (md.phase_field_method == EFSI_PF_CDI) {
                F2 jx, jy;
                cdi_flux(md.pf_param[0], md.pf_param[1], md.pf_param[2], phi, m, bphi, jx, jy);
                dj = divergence(jx, jy, m);
            }
            for (size_t k = 0; k < r.size(); ++k) r.a[k] = adv.a[k] - dj.a[k] + phi.a[k] * S.a[k];
            return r;
        }
        case EFSI_PF_ACDI:
            return acdi_rhs(md, U, V, phi, S, m, bphi);
        case EFSI_PF_UWCDI: {
            F2 fx, fy;
            uwcdi_fluxes(md, U, V, phi, m, bphi, fx, fy);
            F2 d = divergence(fx, fy, m);
            F2 r(m.Nx, m.Ny);
            for (size_t k = 0; k < r.size(); ++k) r.a[k] = -d.a[k] + phi.a[k] * S.a[k];
            return r;
        }
    }
    arg_error("phase_field_method must be an AbstractPhaseFieldMethod.");
}

// ---- StructuralConstitutive.jl --------------------------------------------------
void relaxation_rhs(const efsi_models& md, double sxx, double syy, double sxy, double& rxx,
                    double& ryy, double& rxy) {
    if (md.tensor_relaxation == EFSI_RELAX_MAXWELL) {
        double r = md.relaxation_rate;
        rxx = -r * (sxx - 1.0);
        ryy = -r * (syy - 1.0);
        rxy = -r * sxy;
    } else {
        rxx = ryy = rxy = 0.0;
    }
}

// ---- StructureTensor.jl -----------------------------------------------------------
void sigma_log_product_2d(double a, double d, double b, double& oxx, double& oyy, double& oxy) {
    double mm = 0.5 * (a + d);  // :482-515
    double delta = 0.5 * (a - d);
    double r = std::hypot(delta, b);
    double lhi = mm + r, llo = mm - r;
    if (!(std::isfinite(llo) && std::isfinite(lhi) && llo > 0.0))
        domain_error("GeometricStructureExtension requires an SPD tensor; encountered a non-positive or non-finite eigenvalue.");
    double ghi = lhi * std::log(lhi), glo = llo * std::log(llo);
    double scale = std::max(1.0, std::fabs(mm));
    double alpha, beta;
    if (r <= 1.0e-12 * scale) {
        alpha = std::log(mm) + 1.0;
        beta = -mm;
    } else {
        double den = lhi - llo;
        alpha = (ghi - glo) / den;
        beta = (lhi * glo - llo * ghi) / den;
    }
    oxx = alpha * a + beta;
    oyy = alpha * d + beta;
    oxy = alpha * b;
}

void structure_extension_rhs(const efsi_numerics& nu, const F2& sxx, const F2& syy, const F2& sxy,
                             const F2& phi, F2& rxx, F2& ryy, F2& rxy) {
    rxx = F2(sxx.nx, sxx.ny); ryy = F2(sxx.nx, sxx.ny); rxy = F2(sxx.nx, sxx.ny);
    if (nu.structure_extension != EFSI_EXT_GEOMETRIC) return;
    for (size_t k = 0; k < phi.size(); ++k) {
        double kappa = nu.extension_rate * std::pow(1.0 - clamp01(phi.a[k]), nu.extension_exponent);
        if (kappa == 0.0) continue;
        double gx, gy, gxy;
        sigma_log_product_2d(sxx.a[k], syy.a[k], sxy.a[k], gx, gy, gxy);
        rxx.a[k] = -kappa * gx;
        ryy.a[k] = -kappa * gy;
        rxy.a[k] = -kappa * gxy;
    }
}

int apply_structure_extension(const efsi_numerics& nu, F2& sxx, F2& syy, F2& sxy, const F2& phi) {
    double cutoff;  // :553-613
    if (nu.structure_extension == EFSI_EXT_IDENTITY_OUTSIDE) cutoff = nu.extension_cutoff;
    else if (nu.structure_extension == EFSI_EXT_GEOMETRIC) {
        cutoff = nu.extension_cutoff;
        if (cutoff <= 0.0) return 0;
    } else return 0;
    int n = 0;
    for (size_t k = 0; k < phi.size(); ++k)
        if (phi.a[k] < cutoff) { sxx.a[k] = 1.0; syy.a[k] = 1.0; sxy.a[k] = 0.0; ++n; }
    return n;
}

void structure_tensor_rhs(const F2& sxx, const F2& syy, const F2& sxy, const F2& U, const F2& V,
                          const F2& Kxx, const F2& Kxy, const F2& Kyx, const F2& Kyy,
                          const efsi_models& md, const efsi_numerics& nu, const Mesh& m,
                          const BCS* bsig, const BCS& bu, const BCS& bv, const F2& phi,
                          F2& rxx, F2& ryy, F2& rxy) {
    for (int c = 0; c < 3; ++c)
        if (m.px != bsig[c].periodic_x() || m.py != bsig[c].periodic_y())
            arg_error("bc_sigma does not match MeshMetrics periodicity.");
    F2 axx = upwind_advection(U, V, sxx, m, bsig[0], false, "structural-tensor");
    F2 ayy = upwind_advection(U, V, syy, m, bsig[1], false, "structural-tensor");
    F2 axy = upwind_advection(U, V, sxy, m, bsig[2], false, "structural-tensor");
    F2 dv = divergence(U, V, m);
    F2 dudx, dudy, dvdx, dvdy;
    velocity_gradient(U, V, m, bu, bv, dudx, dudy, dvdx, dvdy);
    F2 exx, eyy, exy;
    structure_extension_rhs(nu, sxx, syy, sxy, phi, exx, eyy, exy);
    rxx = F2(m.Nx, m.Ny); ryy = F2(m.Nx, m.Ny); rxy = F2(m.Nx, m.Ny);
    for (size_t k = 0; k < rxx.size(); ++k) {
        double a11 = dudx.a[k] - Kxx.a[k], a12 = dudy.a[k] - Kxy.a[k];
        double a21 = dvdx.a[k] - Kyx.a[k], a22 = dvdy.a[k] - Kyy.a[k];
        double sx = sxx.a[k], sy = syy.a[k], sc = sxy.a[k];
        double dxx = 2.0 * (a11 * sx + a12 * sc);
        double dyy = 2.0 * (a21 * sc + a22 * sy);
        double dxy = a21 * sx + a12 * sy + (a11 + a22) * sc;
        double qx, qy, qc;
        relaxation_rhs(md, sx, sy, sc, qx, qy, qc);
        rxx.a[k] = (axx.a[k] + sx * dv.a[k]) + dxx + qx + exx.a[k];
        ryy.a[k] = (ayy.a[k] + sy * dv.a[k]) + dyy + qy + eyy.a[k];
        rxy.a[k] = (axy.a[k] + sc * dv.a[k]) + dxy + qc + exy.a[k];
    }
}

SigmaDiag structure_tensor_diagnostics(const F2& sxx, const F2& syy, const F2& sxy) {
    SigmaDiag d{INFINITY, 0.0, INFINITY, 0};
    for (size_t k = 0; k < sxx.size(); ++k) {
        double a = sxx.a[k], dd = syy.a[k], b = sxy.a[k];
        double det = a * dd - b * b;
        double lmin = 0.5 * (a + dd - std::hypot(a - dd, 2.0 * b));
        d.min_det = std::min(d.min_det, det);
        d.max_abs_det_err = std::max(d.max_abs_det_err, std::fabs(det - 1.0));
        d.min_eig = std::min(d.min_eig, lmin);
        if (!(std::isfinite(lmin) && lmin > 0.0)) d.non_spd += 1;
    }
    return d;
}

// ---- Capillarity.jl ------------------------------------------------------------------
void capillary_force(const efsi_models& md, const F2& phi, const Mesh& m, const BCS& bphi, F2& Fx,
                     F2& Fy) {
    const int Nx = m.Nx, Ny = m.Ny;
    Fx = F2(Nx + 1, Ny); Fy = F2(Nx, Ny + 1);
    if (md.capillarity != EFSI_CAP_DIFFUSE_AREA) return;
    F2 geo = phi;  // :96-118
    auto cv = [&](const F2& f, int i, int j) {
        int ii = m.px ? ((i % Nx) + Nx) % Nx : std::min(std::max(i, 0), Nx - 1);
        int jj = m.py ? ((j % Ny) + Ny) % Ny : std::min(std::max(j, 0), Ny - 1);
        return f(ii, jj);
    };
    for (int p = 0; p < md.capillary_smoothing_passes; ++p) {
        F2 nx(Nx, Ny);
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i)
                nx(i, j) = 0.25 * cv(geo, i, j) +
                           0.125 * (cv(geo, i + 1, j) + cv(geo, i - 1, j) + cv(geo, i, j + 1) + cv(geo, i, j - 1)) +
                           0.0625 * (cv(geo, i + 1, j + 1) + cv(geo, i - 1, j + 1) + cv(geo, i + 1, j - 1) + cv(geo, i - 1, j - 1));
        geo = nx;
    }
    F2 ggx, ggy, gx, gy;
    scalar_gradient(geo, m, bphi, ggx, ggy);
    scalar_gradient(phi, m, bphi, gx, gy);
    F2 nxc(Nx, Ny), nyc(Nx, Ny);
    double d2 = md.capillary_delta_normal * md.capillary_delta_normal;
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            double cx = m.wL_f2cx[i] * ggx(i, j) + m.wR_f2cx[i] * ggx(i + 1, j);
            double cy = m.wB_f2cy[j] * ggy(i, j) + m.wT_f2cy[j] * ggy(i, j + 1);
            double den = std::sqrt(cx * cx + cy * cy + d2);
            nxc(i, j) = cx / den;
            nyc(i, j) = cy / den;
        }
    F2 nxf = interp_c2fx(nxc, m), nyf = interp_c2fy(nyc, m);
    F2 kap = divergence(nxf, nyf, m);
    for (double& v : kap.a) v = -v;
    F2 kx = interp_c2fx(kap, m), ky = interp_c2fy(kap, m);
    for (size_t k = 0; k < Fx.size(); ++k) Fx.a[k] = md.capillary_coefficient * kx.a[k] * gx.a[k];
    for (size_t k = 0; k < Fy.size(); ++k) Fy.a[k] = md.capillary_coefficient * ky.a[k] * gy.a[k];
}

// ---- TransportConstitutive.jl --------------------------------------------------------
void body_force(const efsi_models& md, double t, const Mesh& m, F2& Fx, F2& Fy) {
    Fx = F2(m.Nx + 1, m.Ny); Fy = F2(m.Nx, m.Ny + 1);
    if (md.body_force == EFSI_FORCE_NONE) return;
    if (!std::isfinite(t)) arg_error("Body-force evaluation time must be finite.");
    if (md.body_force == EFSI_FORCE_CONSTANT) {
        std::fill(Fx.a.begin(), Fx.a.end(), md.body_force_param[0]);
        std::fill(Fy.a.begin(), Fy.a.end(), md.body_force_param[1]);
        return;
    }
    double y = 0.0;  // :385-397
    for (int j = 0; j < m.Ny; ++j) {
        y += 0.5 * m.dy_c[j];
        double f = md.body_force_param[0] * std::sin(md.body_force_param[1] * y + md.body_force_param[2]);
        for (int i = 0; i <= m.Nx; ++i) Fx(i, j) = f;
        y += 0.5 * m.dy_c[j];
    }
}

void viscosity_field(const efsi_models& md, const F2& phi, F2& out) {
    out = F2(phi.nx, phi.ny);
    if (md.viscosity == EFSI_VISC_CONSTANT) std::fill(out.a.begin(), out.a.end(), md.viscosity_fluid);
    else if (md.viscosity == EFSI_VISC_HARMONIC) {
        for (size_t k = 0; k < phi.size(); ++k) {
            double p = clamp01(phi.a[k]);
            out.a[k] = 1.0 / ((1.0 - p) / md.viscosity_fluid + p / md.viscosity_structure);
        }
        for (double v : out.a)
            if (!(std::isfinite(v) && v > 0.0)) arg_error("evaluated viscosity must be strictly positive everywhere.");
    }
}

void diffusivity_field(const efsi_models& md, const F2& phi, F2& out) {
    out = F2(phi.nx, phi.ny);
    if (md.diffusivity == EFSI_DIFF_CONSTANT) std::fill(out.a.begin(), out.a.end(), md.diffusivity_fluid);
    else if (md.diffusivity == EFSI_DIFF_HARMONIC) {
        for (size_t k = 0; k < phi.size(); ++k)
            out.a[k] = 1.0 / ((1.0 - phi.a[k]) / md.diffusivity_fluid + phi.a[k] / md.diffusivity_structure);
        for (double v : out.a)
            if (!(std::isfinite(v) && v > 0.0)) arg_error("evaluated diffusivity must be strictly positive everywhere.");
    }
}

void resource_sink(const efsi_models& md, const F2& phi, const F2& c, F2& out) {
    out = F2(phi.nx, phi.ny);
    if (md.resource_consumption != EFSI_CONSUMPTION_SATURATING) return;
    for (size_t k = 0; k < phi.size(); ++k)
        out.a[k] = md.consumption_rate * phi.a[k] * c.a[k] / (md.consumption_half_saturation + c.a[k]);
    for (double v : out.a)
        if (!std::isfinite(v)) arg_error("Evaluated resource sink contains non-finite values.");
}

void growth_source(const efsi_models& md, const F2& phi, const F2& c, F2& G) {
    G = F2(phi.nx, phi.ny);
    if (md.growth_source == EFSI_GROWTH_CONSTANT)
        for (size_t k = 0; k < phi.size(); ++k) G.a[k] = md.growth_rate * phi.a[k];
    else if (md.growth_source == EFSI_GROWTH_SATURATING)
        for (size_t k = 0; k < phi.size(); ++k)
            G.a[k] = md.growth_rate * phi.a[k] * c.a[k] / (md.growth_half_saturation + c.a[k]);
}

void growth_tensor(const efsi_models& md, const F2& G, F2& Kxx, F2& Kxy, F2& Kyx, F2& Kyy) {
    Kxx = F2(G.nx, G.ny); Kxy = F2(G.nx, G.ny); Kyx = F2(G.nx, G.ny); Kyy = F2(G.nx, G.ny);
    if (md.growth_tensor == EFSI_GTENSOR_DIRECTIONAL) {
        double tx = md.growth_direction_x, ty = md.growth_direction_y;
        double mag = std::hypot(tx, ty);
        tx /= mag; ty /= mag;
        for (size_t k = 0; k < G.size(); ++k) {
            Kxx.a[k] = tx * tx * G.a[k];
            Kxy.a[k] = tx * ty * G.a[k];
            Kyx.a[k] = tx * ty * G.a[k];
            Kyy.a[k] = ty * ty * G.a[k];
        }
    } else {
        for (size_t k = 0; k < G.size(); ++k) {
            Kxx.a[k] = 0.5 * G.a[k];
            Kyy.a[k] = 0.5 * G.a[k];
        }
    }
}

double growth_trace_error(const F2& G, const F2& Kxx, const F2& Kyy) {
    double e = 0.0;
    for (size_t k = 0; k < G.size(); ++k) e = std::max(e, std::fabs(Kxx.a[k] + Kyy.a[k] - G.a[k]));
    return e;
}

// ---- ResourceTransport.jl --------------------------------------------------------------
F2 resource_explicit_rhs(const F2& U, const F2& V, const F2& c, const F2& sink, const Mesh& m,
                         const BCS& bc) {
    if (m.px != bc.periodic_x() || m.py != bc.periodic_y())
        arg_error("Resource boundary conditions do not match MeshMetrics periodicity.");
    F2 r = upwind_advection(U, V, c, m, bc, true, "resource");
    for (size_t k = 0; k < r.size(); ++k) r.a[k] -= sink.a[k];
    return r;
}

}  // namespace ora
