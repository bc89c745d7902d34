// solvers.cpp — linear solves of the oracle: the projection Poisson problem
// (Projection.jl:149-307) and a BiCGSTAB for the implicit velocity/resource
// systems (TimeIntegrationIMEX.jl:602-672).
// TEST INFRASTRUCTURE ONLY (the oracle); see oracle.hpp.
//
// The reference solves the Poisson problem with GMRES(50)+Ruge-Stueben AMG on the
// gauge-pinned matrix (Projection.jl:106-113, :232-251) and the velocity system
// with UMFPACK or GMRES.  These are third-party algorithms (AlgebraicMultigrid.jl
// 2.0.1, IterativeSolvers.jl 0.9.4, SuiteSparse 7.8.3); what is pinned is the
// discrete solution, so the oracle converges its own solvers far below the
// reference tolerances:
//  * Poisson: CG on the cell-area weighted operator W(-L), which is symmetric for
//    any tensor-product mesh, preconditioned by a cell-centred geometric multigrid
//    V-cycle (red-black Gauss-Seidel, bilinear prolongation, restriction = its
//    transpose, dense Cholesky on the coarsest grid).  With a constant nullspace
//    the weighted right-hand side is made consistent (its defect is the reference's
//    compatibility_defect) and the zero-mean representative is selected.
//  * implicit velocity/resource systems: BiCGSTAB on the exact row-eliminated
//    affine systems of the reference, no symmetry assumed.
#include <algorithm>
#include <cmath>
#include <memory>

#include "oracle.hpp"

namespace ora {

static double dot(const std::vector<double>& a, const std::vector<double>& b) {
    double s = 0.0;
    for (size_t k = 0; k < a.size(); ++k) s += a[k] * b[k];
    return s;
}

template <class Op>
int bicgstab(const Op& A, const std::vector<double>& b, std::vector<double>& x, double tol, int maxiter) {
    const size_t n = b.size();
    std::vector<double> r(n), rh(n), p(n, 0.0), v(n, 0.0), s(n), t(n), ax(n);
    A(x, ax);
    for (size_t k = 0; k < n; ++k) r[k] = b[k] - ax[k];
    rh = r;
    double bn = std::sqrt(dot(b, b));
    if (bn == 0.0) bn = 1.0;
    double rho = 1.0, alpha = 1.0, omega = 1.0;
    if (std::sqrt(dot(r, r)) <= tol * bn) return 0;
    for (int it = 1; it <= maxiter; ++it) {
        double rho_new = dot(rh, r);
        if (rho_new == 0.0) {  // breakdown: restart from the current iterate
            A(x, ax);
            for (size_t k = 0; k < n; ++k) r[k] = b[k] - ax[k];
            rh = r;
            std::fill(p.begin(), p.end(), 0.0);
            std::fill(v.begin(), v.end(), 0.0);
            rho = alpha = omega = 1.0;
            continue;
        }
        double beta = (rho_new / rho) * (alpha / omega);
        rho = rho_new;
        for (size_t k = 0; k < n; ++k) p[k] = r[k] + beta * (p[k] - omega * v[k]);
        A(p, v);
        alpha = rho / dot(rh, v);
        for (size_t k = 0; k < n; ++k) s[k] = r[k] - alpha * v[k];
        if (std::sqrt(dot(s, s)) <= tol * bn) {
            for (size_t k = 0; k < n; ++k) x[k] += alpha * p[k];
            return it;
        }
        A(s, t);
        double tt = dot(t, t);
        omega = tt > 0.0 ? dot(t, s) / tt : 0.0;
        for (size_t k = 0; k < n; ++k) {
            x[k] += alpha * p[k] + omega * s[k];
            r[k] = s[k] - omega * t[k];
        }
        if (std::sqrt(dot(r, r)) <= tol * bn) {
            // confirm with the true residual
            A(x, ax);
            double rr = 0.0;
            for (size_t k = 0; k < n; ++k) { double d = b[k] - ax[k]; rr += d * d; r[k] = d; }
            if (std::sqrt(rr) <= tol * bn) return it;
        }
    }
    return maxiter;
}

// Explicit instantiation for the std::function operator used by imex.cpp.
}  // namespace ora

#include <functional>
namespace ora {
using OpFn = std::function<void(const std::vector<double>&, std::vector<double>&)>;
template int bicgstab<OpFn>(const OpFn&, const std::vector<double>&, std::vector<double>&, double, int);

// ---- Poisson projector -----------------------------------------------------------------
struct Level {
    int nx, ny;
    double hx, hy;
    // Boundary coefficient factors per boundary cell: 0 (Neumann), 2 (Dirichlet),
    // fractional on coarse levels where the fine sides mix.
    std::vector<double> cl, cr, cb, ct;
    std::vector<double> x, b, r;
};

struct Projector {
    Mesh m;
    BCS bq;
    bool nullspace;
    std::vector<Level> lv;
    std::vector<double> chol;  // dense Cholesky factor of the coarsest (shifted) operator
    int nc = 0;
};

static double side_coef(const Side& s, int k) {
    if (s.type == EFSI_BC_DIRICHLET) return 2.0;
    if (s.type == EFSI_BC_MIXED) return s.is_dir(k) ? 2.0 : 0.0;
    return 0.0;
}

// Weighted operator K = hx*hy*(-L) on a uniform level (matrix part).
static void level_apply(const Level& L, bool px, bool py, const std::vector<double>& x,
                        std::vector<double>& y) {
    const int nx = L.nx, ny = L.ny;
    const double ax = L.hy / L.hx, ay = L.hx / L.hy;
    y.assign((size_t)nx * ny, 0.0);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            size_t k = (size_t)i + (size_t)j * nx;
            double c = x[k], s = 0.0;
            if (i > 0) s += ax * (c - x[k - 1]);
            else if (px) s += ax * (c - x[k + nx - 1]);
            else s += ax * L.cl[j] * c;
            if (i < nx - 1) s += ax * (c - x[k + 1]);
            else if (px) s += ax * (c - x[k - (nx - 1)]);
            else s += ax * L.cr[j] * c;
            if (j > 0) s += ay * (c - x[k - nx]);
            else if (py) s += ay * (c - x[k + (size_t)(ny - 1) * nx]);
            else s += ay * L.cb[i] * c;
            if (j < ny - 1) s += ay * (c - x[k + nx]);
            else if (py) s += ay * (c - x[k - (size_t)(ny - 1) * nx]);
            else s += ay * L.ct[i] * c;
            y[k] = s;
        }
}

static void level_diag_offsum(const Level& L, bool px, bool py, int i, int j,
                              const std::vector<double>& x, double& diag, double& off) {
    const int nx = L.nx, ny = L.ny;
    const double ax = L.hy / L.hx, ay = L.hx / L.hy;
    size_t k = (size_t)i + (size_t)j * nx;
    diag = 0.0; off = 0.0;
    if (i > 0) { diag += ax; off += ax * x[k - 1]; }
    else if (px) { diag += ax; off += ax * x[k + nx - 1]; }
    else diag += ax * L.cl[j];
    if (i < nx - 1) { diag += ax; off += ax * x[k + 1]; }
    else if (px) { diag += ax; off += ax * x[k - (nx - 1)]; }
    else diag += ax * L.cr[j];
    if (j > 0) { diag += ay; off += ay * x[k - nx]; }
    else if (py) { diag += ay; off += ay * x[k + (size_t)(ny - 1) * nx]; }
    else diag += ay * L.cb[i];
    if (j < ny - 1) { diag += ay; off += ay * x[k + nx]; }
    else if (py) { diag += ay; off += ay * x[k - (size_t)(ny - 1) * nx]; }
    else diag += ay * L.ct[i];
}

static void gs_color(const Level& L, bool px, bool py, std::vector<double>& x,
                     const std::vector<double>& b, int color) {
    for (int j = 0; j < L.ny; ++j)
        for (int i = 0; i < L.nx; ++i) {
            if (((i + j) & 1) != color) continue;
            double d, o;
            level_diag_offsum(L, px, py, i, j, x, d, o);
            if (d > 0.0) x[(size_t)i + (size_t)j * L.nx] = (b[(size_t)i + (size_t)j * L.nx] + o) / d;
        }
}

// 1-D bilinear weights of fine cell f onto coarse cell I (cell-centred, factor 2).
static void interp_pair(int f, int nc, bool periodic, int& I0, double& w0, int& I1, double& w1) {
    int I = f / 2;
    int J = (f & 1) ? I + 1 : I - 1;
    if (J < 0) J = periodic ? nc - 1 : I;
    if (J >= nc) J = periodic ? 0 : I;
    I0 = I; w0 = 0.75; I1 = J; w1 = 0.25;
}

static void prolong_add(const Level& F, const Level& C, bool px, bool py, const std::vector<double>& e,
                        std::vector<double>& x) {
    for (int j = 0; j < F.ny; ++j) {
        int J0, J1; double v0, v1;
        interp_pair(j, C.ny, py, J0, v0, J1, v1);
        for (int i = 0; i < F.nx; ++i) {
            int I0, I1; double u0, u1;
            interp_pair(i, C.nx, px, I0, u0, I1, u1);
            auto E = [&](int a, int b) { return e[(size_t)a + (size_t)b * C.nx]; };
            x[(size_t)i + (size_t)j * F.nx] += v0 * (u0 * E(I0, J0) + u1 * E(I1, J0)) +
                                               v1 * (u0 * E(I0, J1) + u1 * E(I1, J1));
        }
    }
}

static void restrict_T(const Level& F, const Level& C, bool px, bool py, const std::vector<double>& r,
                       std::vector<double>& rc) {
    rc.assign((size_t)C.nx * C.ny, 0.0);
    for (int j = 0; j < F.ny; ++j) {
        int J0, J1; double v0, v1;
        interp_pair(j, C.ny, py, J0, v0, J1, v1);
        for (int i = 0; i < F.nx; ++i) {
            int I0, I1; double u0, u1;
            interp_pair(i, C.nx, px, I0, u0, I1, u1);
            double q = r[(size_t)i + (size_t)j * F.nx];
            rc[(size_t)I0 + (size_t)J0 * C.nx] += v0 * u0 * q;
            rc[(size_t)I1 + (size_t)J0 * C.nx] += v0 * u1 * q;
            rc[(size_t)I0 + (size_t)J1 * C.nx] += v1 * u0 * q;
            rc[(size_t)I1 + (size_t)J1 * C.nx] += v1 * u1 * q;
        }
    }
}

Projector* make_projector(const Mesh& m, const BCS& bq) {
    auto P = std::make_unique<Projector>();
    P->m = m;
    P->bq = bq;
    P->nullspace = !bq.has_dirichlet();
    Level L0;
    L0.nx = m.Nx; L0.ny = m.Ny;
    L0.hx = m.Lx / m.Nx; L0.hy = m.Ly / m.Ny;
    L0.cl.resize(m.Ny); L0.cr.resize(m.Ny); L0.cb.resize(m.Nx); L0.ct.resize(m.Nx);
    for (int j = 0; j < m.Ny; ++j) {
        L0.cl[j] = m.px ? 0.0 : side_coef(bq.left(), j);
        L0.cr[j] = m.px ? 0.0 : side_coef(bq.right(), j);
    }
    for (int i = 0; i < m.Nx; ++i) {
        L0.cb[i] = m.py ? 0.0 : side_coef(bq.bottom(), i);
        L0.ct[i] = m.py ? 0.0 : side_coef(bq.top(), i);
    }
    P->lv.push_back(L0);
    while (true) {
        const Level& F = P->lv.back();
        if ((long)F.nx * F.ny <= 1024 || (F.nx & 1) || (F.ny & 1) || F.nx < 4 || F.ny < 4) break;
        Level C;
        C.nx = F.nx / 2; C.ny = F.ny / 2; C.hx = 2 * F.hx; C.hy = 2 * F.hy;
        C.cl.resize(C.ny); C.cr.resize(C.ny); C.cb.resize(C.nx); C.ct.resize(C.nx);
        for (int j = 0; j < C.ny; ++j) {
            C.cl[j] = 0.5 * (F.cl[2 * j] + F.cl[2 * j + 1]);
            C.cr[j] = 0.5 * (F.cr[2 * j] + F.cr[2 * j + 1]);
        }
        for (int i = 0; i < C.nx; ++i) {
            C.cb[i] = 0.5 * (F.cb[2 * i] + F.cb[2 * i + 1]);
            C.ct[i] = 0.5 * (F.ct[2 * i] + F.ct[2 * i + 1]);
        }
        P->lv.push_back(C);
    }
    for (Level& L : P->lv) {
        L.x.assign((size_t)L.nx * L.ny, 0.0);
        L.b = L.x; L.r = L.x;
    }
    // Dense Cholesky of the coarsest operator, shifted by s*11^T when singular.
    Level& C = P->lv.back();
    int n = C.nx * C.ny;
    P->nc = n;
    std::vector<double> A((size_t)n * n, 0.0), e(n, 0.0), col;
    for (int k = 0; k < n; ++k) {
        e[k] = 1.0;
        level_apply(C, m.px, m.py, e, col);
        for (int r = 0; r < n; ++r) A[(size_t)r * n + k] = col[r];
        e[k] = 0.0;
    }
    if (P->nullspace) {
        double s = 0.0;
        for (int k = 0; k < n; ++k) s += A[(size_t)k * n + k];
        s /= (double)n * n;
        for (size_t k = 0; k < A.size(); ++k) A[k] += s;
    }
    for (int j = 0; j < n; ++j) {  // in-place lower Cholesky
        double d = A[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) d -= A[(size_t)j * n + k] * A[(size_t)j * n + k];
        if (!(d > 0.0)) solve_error("coarse projection operator is not positive definite");
        d = std::sqrt(d);
        A[(size_t)j * n + j] = d;
        for (int i = j + 1; i < n; ++i) {
            double v = A[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) v -= A[(size_t)i * n + k] * A[(size_t)j * n + k];
            A[(size_t)i * n + j] = v / d;
        }
    }
    P->chol = std::move(A);
    return P.release();
}

void free_projector(Projector* p) { delete p; }

static void coarse_solve(const Projector& P, const std::vector<double>& b, std::vector<double>& x) {
    int n = P.nc;
    const std::vector<double>& A = P.chol;
    x = b;
    for (int i = 0; i < n; ++i) {
        double v = x[i];
        for (int k = 0; k < i; ++k) v -= A[(size_t)i * n + k] * x[k];
        x[i] = v / A[(size_t)i * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
        double v = x[i];
        for (int k = i + 1; k < n; ++k) v -= A[(size_t)k * n + i] * x[k];
        x[i] = v / A[(size_t)i * n + i];
    }
}

static void vcycle(Projector& P, int l) {
    Level& L = P.lv[l];
    bool px = P.m.px, py = P.m.py;
    if (l + 1 == (int)P.lv.size()) {
        coarse_solve(P, L.b, L.x);
        return;
    }
    std::fill(L.x.begin(), L.x.end(), 0.0);
    gs_color(L, px, py, L.x, L.b, 0);
    gs_color(L, px, py, L.x, L.b, 1);
    std::vector<double> ax;
    level_apply(L, px, py, L.x, ax);
    for (size_t k = 0; k < ax.size(); ++k) L.r[k] = L.b[k] - ax[k];
    Level& C = P.lv[l + 1];
    restrict_T(L, C, px, py, L.r, C.b);
    vcycle(P, l + 1);
    prolong_add(L, C, px, py, C.x, L.x);
    gs_color(L, px, py, L.x, L.b, 1);
    gs_color(L, px, py, L.x, L.b, 0);
}

// Exact weighted operator K q = W * (-(Div Grad) q) on the actual metrics.
static void exact_weighted_apply(const Projector& P, const std::vector<double>& q, std::vector<double>& y) {
    const Mesh& m = P.m;
    F2 f(m.Nx, m.Ny);
    f.a = q;
    F2 ones(m.Nx, m.Ny, 1.0);
    F2 out;
    diffusion_matrix_apply(f, ones, m, P.bq, out);
    y.resize(q.size());
    for (int j = 0; j < m.Ny; ++j)
        for (int i = 0; i < m.Nx; ++i) {
            size_t k = (size_t)i + (size_t)j * m.Nx;
            y[k] = -out.a[k] * m.dx_c[i] * m.dy_c[j];
        }
}

ProjOut project(Projector* Pp, F2& U, F2& V, const F2& target, F2& correction, double reltol, int maxiter) {
    Projector& P = *Pp;
    const Mesh& m = P.m;
    const int Nx = m.Nx, Ny = m.Ny;
    const size_t N = (size_t)Nx * Ny;
    if (U.nx != Nx + 1 || U.ny != Ny) dim_error("U has the wrong size.");
    if (V.nx != Nx || V.ny != Ny + 1) dim_error("V has the wrong size.");
    for (double v : U.a) if (!std::isfinite(v)) arg_error("U contains non-finite values.");
    for (double v : V.a) if (!std::isfinite(v)) arg_error("V contains non-finite values.");
    for (double v : target.a) if (!std::isfinite(v)) arg_error("target_divergence contains non-finite values.");
    if (!(reltol > 0)) arg_error("reltol must be positive.");
    if (!(maxiter > 0)) arg_error("maxiter must be positive.");
    F2 pdiv = divergence(U, V, m);
    // Poisson boundary vector: the affine operator applied to q = 0 (Operators.jl:380-383).
    F2 zero(Nx, Ny);
    F2 ones(Nx, Ny, 1.0);
    F2 bbc = diffusion_apply(zero, ones, m, P.bq);
    std::vector<double> rhs(N);
    for (size_t k = 0; k < N; ++k) rhs[k] = (pdiv.a[k] - target.a[k]) - bbc.a[k];
    ProjOut out{};
    out.compatibility_defect = 0.0;
    if (P.nullspace) {  // Projection.jl:206-221
        double defect = 0.0, scale = 0.0;
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                double a = m.dx_c[i] * m.dy_c[j];
                defect += rhs[(size_t)i + (size_t)j * Nx] * a;
                scale += std::fabs(rhs[(size_t)i + (size_t)j * Nx]) * a;
            }
        double tol = 1e-12 + 1e-10 * std::max(scale, 2.220446049250313e-16);
        out.compatibility_defect = defect;
        if (!(std::fabs(defect) <= tol))
            arg_error("The prescribed divergence constraint is incompatible with the Neumann/periodic correction boundaries.");
    }
    // Weighted system K q = b, b = -W rhs.
    std::vector<double> b(N);
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i)
            b[(size_t)i + (size_t)j * Nx] = -rhs[(size_t)i + (size_t)j * Nx] * m.dx_c[i] * m.dy_c[j];
    if (P.nullspace) {
        double mb = 0.0;
        for (double v : b) mb += v;
        mb /= (double)N;
        for (double& v : b) v -= mb;
    }
    std::vector<double> x = correction.a;
    if (x.size() != N) x.assign(N, 0.0);
    for (double v : x) if (!std::isfinite(v)) arg_error("correction_guess contains non-finite values.");
    std::vector<double> r(N), z(N), p(N), Ap(N), Kx;
    exact_weighted_apply(P, x, Kx);
    for (size_t k = 0; k < N; ++k) r[k] = b[k] - Kx[k];
    double bn = std::sqrt(dot(b, b));
    int it = 0;
    if (bn > 0.0 && std::sqrt(dot(r, r)) > reltol * bn) {
        auto precond = [&](const std::vector<double>& rr, std::vector<double>& zz) {
            P.lv[0].b = rr;
            vcycle(P, 0);
            zz = P.lv[0].x;
        };
        precond(r, z);
        p = z;
        double rz = dot(r, z);
        for (it = 1; it <= maxiter; ++it) {
            exact_weighted_apply(P, p, Ap);
            double alpha = rz / dot(p, Ap);
            for (size_t k = 0; k < N; ++k) { x[k] += alpha * p[k]; r[k] -= alpha * Ap[k]; }
            if (std::sqrt(dot(r, r)) <= reltol * bn) break;
            precond(r, z);
            double rz_new = dot(r, z);
            double beta = rz_new / rz;
            rz = rz_new;
            for (size_t k = 0; k < N; ++k) p[k] = z[k] + beta * p[k];
        }
        if (it > maxiter) it = maxiter;
    }
    out.iters = it;
    correction = F2(Nx, Ny);
    correction.a = x;
    if (P.nullspace) {  // Projection.jl:255-259
        double s = 0.0;
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) s += correction(i, j) * m.dx_c[i] * m.dy_c[j];
        double mean = s / (m.Lx * m.Ly);
        for (double& v : correction.a) v -= mean;
    }
    // True residual of the unpinned system (Projection.jl:261-264).
    F2 Lq;
    diffusion_matrix_apply(correction, ones, m, P.bq, Lq);
    double rr = 0.0, rn = 0.0;
    for (size_t k = 0; k < N; ++k) { double d = Lq.a[k] - rhs[k]; rr += d * d; rn += rhs[k] * rhs[k]; }
    out.linear_relative_residual = std::sqrt(rr) / std::max(std::sqrt(rn), 2.220446049250313e-16);
    F2 gx, gy;  // :266-273
    scalar_gradient(correction, m, P.bq, gx, gy);
    for (size_t k = 0; k < U.size(); ++k) U.a[k] -= gx.a[k];
    for (size_t k = 0; k < V.size(); ++k) V.a[k] -= gy.a[k];
    F2 cres = divergence(U, V, m);  // :275-277
    double linf = 0.0, l2 = 0.0;
    auto wl2 = [&](const F2& f) {
        double t = 0.0;
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) t += f(i, j) * f(i, j) * m.dx_c[i] * m.dy_c[j];
        return std::sqrt(t / (m.Lx * m.Ly));
    };
    for (size_t k = 0; k < N; ++k) {
        cres.a[k] -= target.a[k];
        linf = std::max(linf, std::fabs(cres.a[k]));
    }
    l2 = wl2(cres);
    out.constraint_linf = linf;
    out.constraint_l2 = l2;
    if (!(out.linear_relative_residual <= 1e-8))  // :279-298
        solve_error("Projection Poisson solve did not reach the required true-residual accuracy.");
    double cscale = std::max(std::max(wl2(pdiv), wl2(target)), 1.0);
    if (!(l2 <= 1e-12 + 1e-8 * cscale))
        solve_error("Projection did not satisfy the prescribed divergence constraint.");
    return out;
}

}  // namespace ora
