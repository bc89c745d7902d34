// ops.cpp — restatement of Operators.jl and the boundary-data helpers.
// TEST INFRASTRUCTURE ONLY (the oracle); see oracle.hpp.
#include <algorithm>
#include <cstring>

#include "oracle.hpp"

namespace ora {

// ---- boundary data (BoundaryConditions.jl:100-136) ---------------------------
double Side::val(int k) const {
    if (k < 0 || k >= (int)value.size()) dim_error("boundary data index out of range");
    return value[k];
}
double Side::neu(int k) const {
    if (k < 0 || k >= (int)neumann.size()) dim_error("mixed Neumann data index out of range");
    return neumann[k];
}
bool Side::is_dir(int k) const {
    if (k < 0 || k >= (int)mask.size()) dim_error("mixed mask index out of range");
    return mask[k] != 0;
}
bool BCS::has_dirichlet() const {  // BoundaryConditions.jl:92-98
    for (const Side& sd : s) {
        if (sd.type == EFSI_BC_DIRICHLET) return true;
        if (sd.type == EFSI_BC_MIXED)
            for (uint8_t q : sd.mask)
                if (q) return true;
    }
    return false;
}

static std::vector<double> copy_arr(const double* p, int n) {
    return p ? std::vector<double>(p, p + n) : std::vector<double>((size_t)std::max(n, 0), 0.0);
}

BCS make_bcs(const efsi_bc_setup& b, int n_lr, int n_bt, const char* name) {
    BCS r;
    const efsi_bc_side* in[4] = {&b.left, &b.right, &b.bottom, &b.top};
    for (int k = 0; k < 4; ++k) {
        const efsi_bc_side& s = *in[k];
        Side& o = r.s[k];
        o.type = s.type;
        if (s.type < EFSI_BC_PERIODIC || s.type > EFSI_BC_ADVECTIVE_OUTFLOW)
            arg_error(std::string(name) + ": unknown boundary type");
        int need = k < 2 ? n_lr : n_bt;
        if (s.type != EFSI_BC_PERIODIC) {
            if (s.n < need) dim_error(std::string(name) + ": boundary data shorter than the side");
            o.value = copy_arr(s.value, s.n);
            if (s.type == EFSI_BC_MIXED) {
                o.neumann = copy_arr(s.neumann, s.n);
                o.mask.assign(s.n, 0);
                if (s.mask) std::memcpy(o.mask.data(), s.mask, (size_t)s.n);
            }
        }
    }
    // BoundaryConditionSetup requires opposing periodic pairs (BoundaryConditions.jl:74-83).
    if ((r.s[0].type == EFSI_BC_PERIODIC) != (r.s[1].type == EFSI_BC_PERIODIC))
        arg_error(std::string(name) + ": periodic boundaries in the x-direction must be specified as an opposing pair.");
    if ((r.s[2].type == EFSI_BC_PERIODIC) != (r.s[3].type == EFSI_BC_PERIODIC))
        arg_error(std::string(name) + ": periodic boundaries in the y-direction must be specified as an opposing pair.");
    return r;
}

Mesh make_mesh(const efsi_mesh& m) {
    Mesh r;
    r.Nx = m.Nx; r.Ny = m.Ny; r.Lx = m.Lx; r.Ly = m.Ly;
    r.px = m.periodic_x != 0; r.py = m.periodic_y != 0;
    if (m.Nx < 2 || m.Ny < 2) arg_error("Nx and Ny must be at least 2.");
    auto cp = [](const double* p, int n, const char* nm) {
        if (!p) arg_error(std::string("mesh metric ") + nm + " missing");
        return std::vector<double>(p, p + n);
    };
    int Nx = m.Nx, Ny = m.Ny;
    r.dx_f = cp(m.dx_f, Nx + 1, "dx_f"); r.dx_c = cp(m.dx_c, Nx, "dx_c");
    r.dy_f = cp(m.dy_f, Ny + 1, "dy_f"); r.dy_c = cp(m.dy_c, Ny, "dy_c");
    r.wL_c2fx = cp(m.wL_c2fx, Nx + 1, "wL_c2fx"); r.wR_c2fx = cp(m.wR_c2fx, Nx + 1, "wR_c2fx");
    r.wB_c2fy = cp(m.wB_c2fy, Ny + 1, "wB_c2fy"); r.wT_c2fy = cp(m.wT_c2fy, Ny + 1, "wT_c2fy");
    r.wL_f2cx = cp(m.wL_f2cx, Nx, "wL_f2cx"); r.wR_f2cx = cp(m.wR_f2cx, Nx, "wR_f2cx");
    r.wB_f2cy = cp(m.wB_f2cy, Ny, "wB_f2cy"); r.wT_f2cy = cp(m.wT_f2cy, Ny, "wT_f2cy");
    r.dxw = cp(m.dx_west_corner, Nx + 1, "dx_west_corner");
    r.dxe = cp(m.dx_east_corner, Nx + 1, "dx_east_corner");
    r.dys = cp(m.dy_south_corner, Ny + 1, "dy_south_corner");
    r.dyn = cp(m.dy_north_corner, Ny + 1, "dy_north_corner");
    return r;
}

// ---- interpolation (Operators.jl:109-185) -------------------------------------
F2 interp_c2fx(const F2& f, const Mesh& m) {
    const int Nx = m.Nx, Ny = m.Ny;
    F2 face(Nx + 1, Ny);
    for (int j = 0; j < Ny; ++j) {
        if (m.px) {
            double v = m.wL_c2fx[0] * f(Nx - 1, j) + m.wR_c2fx[0] * f(0, j);
            face(0, j) = v;
            face(Nx, j) = v;
        } else {
            face(0, j) = f(0, j);
            face(Nx, j) = f(Nx - 1, j);
        }
        for (int i = 1; i < Nx; ++i) face(i, j) = m.wL_c2fx[i] * f(i - 1, j) + m.wR_c2fx[i] * f(i, j);
    }
    return face;
}

F2 interp_c2fy(const F2& f, const Mesh& m) {
    const int Nx = m.Nx, Ny = m.Ny;
    F2 face(Nx, Ny + 1);
    for (int i = 0; i < Nx; ++i) {
        if (m.py) {
            double v = m.wB_c2fy[0] * f(i, Ny - 1) + m.wT_c2fy[0] * f(i, 0);
            face(i, 0) = v;
            face(i, Ny) = v;
        } else {
            face(i, 0) = f(i, 0);
            face(i, Ny) = f(i, Ny - 1);
        }
        for (int j = 1; j < Ny; ++j) face(i, j) = m.wB_c2fy[j] * f(i, j - 1) + m.wT_c2fy[j] * f(i, j);
    }
    return face;
}

F2 interp_c2corners(const F2& f, const Mesh& m) {
    const int Nx = m.Nx, Ny = m.Ny;
    F2 xf = interp_c2fx(f, m);
    F2 c(Nx + 1, Ny + 1);
    for (int i = 0; i <= Nx; ++i) {
        if (m.py) {
            double v = m.wB_c2fy[0] * xf(i, Ny - 1) + m.wT_c2fy[0] * xf(i, 0);
            c(i, 0) = v;
            c(i, Ny) = v;
        } else {
            c(i, 0) = xf(i, 0);
            c(i, Ny) = xf(i, Ny - 1);
        }
        for (int j = 1; j < Ny; ++j) c(i, j) = m.wB_c2fy[j] * xf(i, j - 1) + m.wT_c2fy[j] * xf(i, j);
    }
    return c;
}

// ---- scalar gradient (Operators.jl:189-356 assembled, :395-404 applied) ------
// Boundary face value for one side.  `interior` is the adjacent cell value,
// `dist` the half-width h/2, `sgn` = -1 on the low side and +1 on the high side
// (the reference's gx_bc sign convention: -value/dist on left, +value/dist on
// right; -g on left Neumann, +g on right Neumann).
static double boundary_gradient(const Side& s, int k, double interior, double dist, double sgn) {
    switch (s.type) {
        case EFSI_BC_DIRICHLET:
            return sgn < 0 ? interior / dist - s.val(k) / dist : s.val(k) / dist - interior / dist;
        case EFSI_BC_NEUMANN:
            return sgn * s.val(k);
        case EFSI_BC_MIXED:
            if (s.is_dir(k))
                return sgn < 0 ? interior / dist - s.val(k) / dist : s.val(k) / dist - interior / dist;
            return sgn * s.neu(k);
        case EFSI_BC_ADVECTIVE_OUTFLOW:
            return 0.0;
    }
    arg_error("Unsupported scalar boundary condition.");
}

void scalar_gradient(const F2& f, const Mesh& m, const BCS& bc, F2& gx, F2& gy) {
    const int Nx = m.Nx, Ny = m.Ny;
    if (m.px != bc.periodic_x() || m.py != bc.periodic_y())
        arg_error("The periodicity encoded in MeshMetrics does not match the boundary conditions.");
    gx = F2(Nx + 1, Ny);
    gy = F2(Nx, Ny + 1);
    for (int j = 0; j < Ny; ++j) {
        if (m.px) {
            double w = (f(0, j) - f(Nx - 1, j)) / m.dx_f[0];
            double wr = (f(0, j) - f(Nx - 1, j)) / m.dx_f[Nx];
            gx(0, j) = w;
            gx(Nx, j) = wr;
        } else {
            gx(0, j) = boundary_gradient(bc.left(), j, f(0, j), m.dx_f[0] / 2.0, -1.0);
            gx(Nx, j) = boundary_gradient(bc.right(), j, f(Nx - 1, j), m.dx_f[Nx] / 2.0, +1.0);
        }
        for (int i = 1; i < Nx; ++i) gx(i, j) = (f(i, j) - f(i - 1, j)) / m.dx_f[i];
    }
    for (int i = 0; i < Nx; ++i) {
        if (m.py) {
            gy(i, 0) = (f(i, 0) - f(i, Ny - 1)) / m.dy_f[0];
            gy(i, Ny) = (f(i, 0) - f(i, Ny - 1)) / m.dy_f[Ny];
        } else {
            gy(i, 0) = boundary_gradient(bc.bottom(), i, f(i, 0), m.dy_f[0] / 2.0, -1.0);
            gy(i, Ny) = boundary_gradient(bc.top(), i, f(i, Ny - 1), m.dy_f[Ny] / 2.0, +1.0);
        }
        for (int j = 1; j < Ny; ++j) gy(i, j) = (f(i, j) - f(i, j - 1)) / m.dy_f[j];
    }
}

F2 divergence(const F2& U, const F2& V, const Mesh& m) {
    const int Nx = m.Nx, Ny = m.Ny;
    if (U.nx != Nx + 1 || U.ny != Ny || V.nx != Nx || V.ny != Ny + 1)
        dim_error("divergence: U/V have the wrong size.");
    F2 d(Nx, Ny);
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i)
            d(i, j) = (U(i + 1, j) - U(i, j)) / m.dx_c[i] + (V(i, j + 1) - V(i, j)) / m.dy_c[j];
    return d;
}

// ---- diffusion operator (Operators.jl:361-384) ----------------------------------
// apply_operator(op, c) = Div(D_face .* scalar_gradient(c)) including the boundary vector.
F2 diffusion_apply(const F2& c, const F2& D, const Mesh& m, const BCS& bc) {
    F2 gx, gy;
    scalar_gradient(c, m, bc, gx, gy);
    F2 Dx = interp_c2fx(D, m), Dy = interp_c2fy(D, m);
    for (size_t k = 0; k < gx.size(); ++k) gx.a[k] *= Dx.a[k];
    for (size_t k = 0; k < gy.size(); ++k) gy.a[k] *= Dy.a[k];
    return divergence(gx, gy, m);
}

// Matrix part only (boundary data set to zero): used inside the implicit solves.
void diffusion_matrix_apply(const F2& c, const F2& D, const Mesh& m, const BCS& bc, F2& out) {
    BCS hom = bc;
    for (Side& s : hom.s) {
        std::fill(s.value.begin(), s.value.end(), 0.0);
        std::fill(s.neumann.begin(), s.neumann.end(), 0.0);
    }
    out = diffusion_apply(c, D, m, hom);
}

// ---- velocity gradient at cell centres (Operators.jl:431-616) -------------------
static double wall_value_at_x_center(const Side& s, int i, const Mesh& m) {  // :590-601
    return m.wL_f2cx[i] * s.val(i) + m.wR_f2cx[i] * s.val(i + 1);
}
static double wall_value_at_y_center(const Side& s, int j, const Mesh& m) {  // :605-616
    return m.wB_f2cy[j] * s.val(j) + m.wT_f2cy[j] * s.val(j + 1);
}

void velocity_gradient(const F2& U, const F2& V, const Mesh& m, const BCS& bu, const BCS& bv,
                       F2& dudx, F2& dudy, F2& dvdx, F2& dvdy) {
    const int Nx = m.Nx, Ny = m.Ny;
    dudx = F2(Nx, Ny); dudy = F2(Nx, Ny); dvdx = F2(Nx, Ny); dvdy = F2(Nx, Ny);
    F2 Uc(Nx, Ny), Vc(Nx, Ny);
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            dudx(i, j) = (U(i + 1, j) - U(i, j)) / m.dx_c[i];
            dvdy(i, j) = (V(i, j + 1) - V(i, j)) / m.dy_c[j];
            Uc(i, j) = m.wL_f2cx[i] * U(i, j) + m.wR_f2cx[i] * U(i + 1, j);
            Vc(i, j) = m.wB_f2cy[j] * V(i, j) + m.wT_f2cy[j] * V(i, j + 1);
        }
    for (int i = 0; i < Nx; ++i) {
        if (m.py) {
            for (int j = 0; j < Ny; ++j) {
                int jm = j == 0 ? Ny - 1 : j - 1, jp = j == Ny - 1 ? 0 : j + 1;
                dudy(i, j) = (Uc(i, jp) - Uc(i, jm)) / (m.dy_f[j] + m.dy_f[j + 1]);
            }
        } else {
            const Side& b = bu.bottom();
            const Side& t = bu.top();
            if (b.type == EFSI_BC_DIRICHLET)
                dudy(i, 0) = (Uc(i, 0) - wall_value_at_x_center(b, i, m)) / m.dyn[0];
            else if (b.type == EFSI_BC_NEUMANN)
                dudy(i, 0) = -wall_value_at_x_center(b, i, m);
            else
                arg_error("Unsupported U-bottom boundary for du/dy.");
            for (int j = 1; j < Ny - 1; ++j)
                dudy(i, j) = (Uc(i, j + 1) - Uc(i, j - 1)) / (m.dy_f[j] + m.dy_f[j + 1]);
            if (t.type == EFSI_BC_DIRICHLET)
                dudy(i, Ny - 1) = (wall_value_at_x_center(t, i, m) - Uc(i, Ny - 1)) / m.dys[Ny];
            else if (t.type == EFSI_BC_NEUMANN)
                dudy(i, Ny - 1) = wall_value_at_x_center(t, i, m);
            else
                arg_error("Unsupported U-top boundary for du/dy.");
        }
    }
    for (int j = 0; j < Ny; ++j) {
        if (m.px) {
            for (int i = 0; i < Nx; ++i) {
                int im = i == 0 ? Nx - 1 : i - 1, ip = i == Nx - 1 ? 0 : i + 1;
                dvdx(i, j) = (Vc(ip, j) - Vc(im, j)) / (m.dx_f[i] + m.dx_f[i + 1]);
            }
        } else {
            const Side& l = bv.left();
            const Side& r = bv.right();
            if (l.type == EFSI_BC_DIRICHLET)
                dvdx(0, j) = (Vc(0, j) - wall_value_at_y_center(l, j, m)) / m.dxe[0];
            else if (l.type == EFSI_BC_NEUMANN)
                dvdx(0, j) = -wall_value_at_y_center(l, j, m);
            else
                arg_error("Unsupported V-left boundary for dv/dx.");
            for (int i = 1; i < Nx - 1; ++i)
                dvdx(i, j) = (Vc(i + 1, j) - Vc(i - 1, j)) / (m.dx_f[i] + m.dx_f[i + 1]);
            if (r.type == EFSI_BC_DIRICHLET)
                dvdx(Nx - 1, j) = (wall_value_at_y_center(r, j, m) - Vc(Nx - 1, j)) / m.dxw[Nx];
            else if (r.type == EFSI_BC_NEUMANN)
                dvdx(Nx - 1, j) = wall_value_at_y_center(r, j, m);
            else
                arg_error("Unsupported V-right boundary for dv/dx.");
        }
    }
}

// ---- symmetric stress divergence (Operators.jl:620-842) -----------------------
static double lin_left(const F2& f, int j, const Mesh& m) {  // :738-744
    double d = m.dxe[0];
    return f(0, j) - (f(1, j) - f(0, j)) * d / m.dx_f[1];
}
static double lin_right(const F2& f, int j, const Mesh& m) {  // :746-752
    int Nx = m.Nx;
    double d = m.dxw[Nx];
    return f(Nx - 1, j) + (f(Nx - 1, j) - f(Nx - 2, j)) * d / m.dx_f[Nx - 1];
}
static double lin_bottom(const F2& f, int i, const Mesh& m) {  // :754-760 and :813-818
    double d = m.dyn[0];
    return f(i, 0) - (f(i, 1) - f(i, 0)) * d / m.dy_f[1];
}
static double lin_top(const F2& f, int i, const Mesh& m) {  // :762-768 and :820-826
    int Ny = m.Ny;
    double d = m.dys[Ny];
    return f(i, Ny - 1) + (f(i, Ny - 1) - f(i, Ny - 2)) * d / m.dy_f[Ny - 1];
}

void symmetric_stress_divergence(const F2& Txx, const F2& Tyy, const F2& Txy, const Mesh& m,
                                 F2& Fx, F2& Fy) {
    const int Nx = m.Nx, Ny = m.Ny;
    // Txy on x-faces and y-faces with linear boundary extrapolation (:770-810).
    F2 Tx(Nx + 1, Ny), Ty(Nx, Ny + 1);
    for (int j = 0; j < Ny; ++j) {
        if (m.px) {
            double v = m.wL_c2fx[0] * Txy(Nx - 1, j) + m.wR_c2fx[0] * Txy(0, j);
            Tx(0, j) = v; Tx(Nx, j) = v;
        } else {
            Tx(0, j) = lin_left(Txy, j, m);
            Tx(Nx, j) = lin_right(Txy, j, m);
        }
        for (int i = 1; i < Nx; ++i) Tx(i, j) = m.wL_c2fx[i] * Txy(i - 1, j) + m.wR_c2fx[i] * Txy(i, j);
    }
    for (int i = 0; i < Nx; ++i) {
        if (m.py) {
            double v = m.wB_c2fy[0] * Txy(i, Ny - 1) + m.wT_c2fy[0] * Txy(i, 0);
            Ty(i, 0) = v; Ty(i, Ny) = v;
        } else {
            Ty(i, 0) = lin_bottom(Txy, i, m);
            Ty(i, Ny) = lin_top(Txy, i, m);
        }
        for (int j = 1; j < Ny; ++j) Ty(i, j) = m.wB_c2fy[j] * Txy(i, j - 1) + m.wT_c2fy[j] * Txy(i, j);
    }
    Fx = F2(Nx + 1, Ny);
    Fy = F2(Nx, Ny + 1);
    for (int j = 0; j < Ny; ++j) {
        if (m.px) {
            double w = (Txx(0, j) - Txx(Nx - 1, j)) / m.dx_f[0];
            Fx(0, j) = w; Fx(Nx, j) = w;
        } else {
            Fx(0, j) = (Txx(0, j) - lin_left(Txx, j, m)) / m.dxe[0];
            Fx(Nx, j) = (lin_right(Txx, j, m) - Txx(Nx - 1, j)) / m.dxw[Nx];
        }
        for (int i = 1; i < Nx; ++i) Fx(i, j) = (Txx(i, j) - Txx(i - 1, j)) / m.dx_f[i];
    }
    for (int i = 0; i <= Nx; ++i) {
        if (m.py) {
            for (int j = 0; j < Ny; ++j) {
                int jm = j == 0 ? Ny - 1 : j - 1, jp = j == Ny - 1 ? 0 : j + 1;
                Fx(i, j) += (Tx(i, jp) - Tx(i, jm)) / (m.dy_f[j] + m.dy_f[j + 1]);
            }
        } else {
            // Tx is already on x-faces; _linear_extrapolate_{bottom,top}_row (:813-826).
            double bw = Tx(i, 0) - (Tx(i, 1) - Tx(i, 0)) * m.dyn[0] / m.dy_f[1];
            double tw = Tx(i, Ny - 1) + (Tx(i, Ny - 1) - Tx(i, Ny - 2)) * m.dys[Ny] / m.dy_f[Ny - 1];
            Fx(i, 0) += (Tx(i, 0) - bw) / m.dyn[0];
            for (int j = 1; j < Ny - 1; ++j)
                Fx(i, j) += (Tx(i, j + 1) - Tx(i, j - 1)) / (m.dy_f[j] + m.dy_f[j + 1]);
            Fx(i, Ny - 1) += (tw - Tx(i, Ny - 1)) / m.dys[Ny];
        }
    }
    for (int i = 0; i < Nx; ++i) {
        if (m.py) {
            double w = (Tyy(i, 0) - Tyy(i, Ny - 1)) / m.dy_f[0];
            Fy(i, 0) = w; Fy(i, Ny) = w;
        } else {
            Fy(i, 0) = (Tyy(i, 0) - lin_bottom(Tyy, i, m)) / m.dyn[0];
            Fy(i, Ny) = (lin_top(Tyy, i, m) - Tyy(i, Ny - 1)) / m.dys[Ny];
        }
        for (int j = 1; j < Ny; ++j) Fy(i, j) = (Tyy(i, j) - Tyy(i, j - 1)) / m.dy_f[j];
    }
    for (int j = 0; j <= Ny; ++j) {
        if (m.px) {
            for (int i = 0; i < Nx; ++i) {
                int im = i == 0 ? Nx - 1 : i - 1, ip = i == Nx - 1 ? 0 : i + 1;
                Fy(i, j) += (Ty(ip, j) - Ty(im, j)) / (m.dx_f[i] + m.dx_f[i + 1]);
            }
        } else {
            double lw = Ty(0, j) - (Ty(1, j) - Ty(0, j)) * m.dxe[0] / m.dx_f[1];
            double rw = Ty(Nx - 1, j) + (Ty(Nx - 1, j) - Ty(Nx - 2, j)) * m.dxw[Nx] / m.dx_f[Nx - 1];
            Fy(0, j) += (Ty(0, j) - lw) / m.dxe[0];
            for (int i = 1; i < Nx - 1; ++i)
                Fy(i, j) += (Ty(i + 1, j) - Ty(i - 1, j)) / (m.dx_f[i] + m.dx_f[i + 1]);
            Fy(Nx - 1, j) += (rw - Ty(Nx - 1, j)) / m.dxw[Nx];
        }
    }
    if (m.px)
        for (int j = 0; j < Ny; ++j) Fx(Nx, j) = Fx(0, j);
    if (m.py)
        for (int i = 0; i < Nx; ++i) Fy(i, Ny) = Fy(i, 0);
}

// ---- compact viscous operator (Operators.jl:848-1083) ----------------------------
// x and out hold [u; v] with u(i,j) = U[i,j] (i < Nx) and v(i,j) = V[i,j] (j < Ny).
// The assembled matrix is Dstress * diag(2 mu) * E plus the wall-shear lifting on
// the diagonal; the boundary vector is Dstress * (w .* E_bc) plus lifting data.
void viscous_apply(const std::vector<double>& x, const F2& mu, const Mesh& m, const BCS& bu,
                   const BCS& bv, bool with_boundary, std::vector<double>& out) {
    const int Nx = m.Nx, Ny = m.Ny;
    const size_t N = (size_t)Nx * Ny;
    auto u = [&](int i, int j) { return x[(size_t)i + (size_t)j * Nx]; };
    auto v = [&](int i, int j) { return x[N + (size_t)i + (size_t)j * Nx]; };
    F2 muc = interp_c2corners(mu, m);
    F2 txx(Nx, Ny), tyy(Nx, Ny), txy(Nx, Ny);
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            double exx = -u(i, j) / m.dx_c[i];
            if (i < Nx - 1) exx += u(i + 1, j) / m.dx_c[i];
            else if (m.px) exx += u(0, j) / m.dx_c[i];
            else if (with_boundary) exx += bu.right().val(j) / m.dx_c[i];
            double eyy = -v(i, j) / m.dy_c[j];
            if (j < Ny - 1) eyy += v(i, j + 1) / m.dy_c[j];
            else if (m.py) eyy += v(i, 0) / m.dy_c[j];
            else if (with_boundary) eyy += bv.top().val(i) / m.dy_c[j];
            double duy = 0.0, dvx = 0.0;
            if (j > 0) duy = (u(i, j) - u(i, j - 1)) / m.dy_f[j];
            else if (m.py) duy = (u(i, 0) - u(i, Ny - 1)) / m.dy_f[0];
            if (i > 0) dvx = (v(i, j) - v(i - 1, j)) / m.dx_f[i];
            else if (m.px) dvx = (v(0, j) - v(Nx - 1, j)) / m.dx_f[0];
            txx(i, j) = 2.0 * mu(i, j) * exx;
            tyy(i, j) = 2.0 * mu(i, j) * eyy;
            txy(i, j) = 2.0 * muc(i, j) * (0.5 * duy + 0.5 * dvx);
        }
    out.assign(2 * N, 0.0);
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            double axx = txx(i, j);
            if (i > 0) axx -= txx(i - 1, j);
            else if (m.px) axx -= txx(Nx - 1, j);
            double axy = -txy(i, j);
            if (j < Ny - 1) axy += txy(i, j + 1);
            else if (m.py) axy += txy(i, 0);
            out[(size_t)i + (size_t)j * Nx] = axx / m.dx_f[i] + axy / m.dy_c[j];
            double ayx = -txy(i, j);
            if (i < Nx - 1) ayx += txy(i + 1, j);
            else if (m.px) ayx += txy(0, j);
            double ayy = tyy(i, j);
            if (j > 0) ayy -= tyy(i, j - 1);
            else if (m.py) ayy -= tyy(i, Ny - 1);
            out[N + (size_t)i + (size_t)j * Nx] = ayx / m.dx_c[i] + ayy / m.dy_f[j];
        }
    // Tangential Dirichlet wall shear (Operators.jl:1036-1080).
    if (!m.py) {
        double db = m.dy_f[0] / 2.0, dt = m.dy_f[Ny] / 2.0;
        for (int i = 0; i < Nx; ++i) {
            if (bu.bottom().type == EFSI_BC_DIRICHLET) {
                size_t row = (size_t)i;
                double w = muc(i, 0) / (m.dy_c[0] * db);
                out[row] -= w * u(i, 0);
                if (with_boundary) out[row] += w * bu.bottom().val(i);
            }
            if (bu.top().type == EFSI_BC_DIRICHLET) {
                size_t row = (size_t)i + (size_t)(Ny - 1) * Nx;
                double w = muc(i, Ny) / (m.dy_c[Ny - 1] * dt);
                out[row] -= w * u(i, Ny - 1);
                if (with_boundary) out[row] += w * bu.top().val(i);
            }
        }
    }
    if (!m.px) {
        double dl = m.dx_f[0] / 2.0, dr = m.dx_f[Nx] / 2.0;
        for (int j = 0; j < Ny; ++j) {
            if (bv.left().type == EFSI_BC_DIRICHLET) {
                size_t row = N + (size_t)j * Nx;
                double w = muc(0, j) / (m.dx_c[0] * dl);
                out[row] -= w * v(0, j);
                if (with_boundary) out[row] += w * bv.left().val(j);
            }
            if (bv.right().type == EFSI_BC_DIRICHLET) {
                size_t row = N + (size_t)(Nx - 1) + (size_t)j * Nx;
                double w = muc(Nx, j) / (m.dx_c[Nx - 1] * dr);
                out[row] -= w * v(Nx - 1, j);
                if (with_boundary) out[row] += w * bv.right().val(j);
            }
        }
    }
}

void velocity_dirichlet_data(const Mesh& m, const BCS& bu, const BCS& bv, std::vector<int>& idx,
                             std::vector<double>& val) {
    const int Nx = m.Nx, Ny = m.Ny;
    idx.clear(); val.clear();
    if (bu.left().type == EFSI_BC_DIRICHLET)
        for (int j = 0; j < Ny; ++j) { idx.push_back(j * Nx); val.push_back(bu.left().val(j)); }
    if (bv.bottom().type == EFSI_BC_DIRICHLET)
        for (int i = 0; i < Nx; ++i) { idx.push_back(Nx * Ny + i); val.push_back(bv.bottom().val(i)); }
}

}  // namespace ora
