// efsi_solvers.cu — the implicit parts of the IMEX step on sm_100a.
//
// * Viscous predictor (TimeIntegrationIMEX.jl:776-812, Operators.jl:929-1083):
//   (I - alpha*A) u = rhs.  On a uniform mesh the compact viscous operator is
//   symmetric, and eliminating the Dirichlet rows (U-left, V-bottom) symmetrically
//   leaves an SPD system for the free unknowns with the same solution as the
//   reference's row elimination; it is solved by Jacobi-preconditioned CG.
// * Resource diffusion (TimeIntegrationIMEX.jl:742-774): (I - alpha*L_D) c = rhs,
//   SPD, Jacobi-preconditioned CG.
// * Projection (Projection.jl:170-307): the cell-area weighted Poisson operator
//   K = hx*hy*(-L) is SPD (semi-definite with constant nullspace for Neumann /
//   periodic correction boundaries); it is solved by CG preconditioned with one
//   geometric multigrid V(1,1)-cycle (red-black Gauss-Seidel smoothing, bilinear
//   prolongation P, restriction P^T, dense inverse on the coarsest grid).  The
//   reference pins q[1]=0 and later subtracts the mean; here the consistent
//   right-hand side is solved directly and the zero-mean representative is taken,
//   which is the same correction potential.
//
// Every CG keeps its scalars (alpha, beta, residual norms) in device memory; one
// iteration is a fixed sequence of kernels that return immediately once `done`
// is set, so iterations can be enqueued without host round trips.
#include <algorithm>
#include <cmath>

#include "efsi_device.cuh"
#include "efsi_solvers.cuh"

namespace efsi {

static constexpr int BX = 32, BY = 8;
static inline dim3 grid2(int nx, int ny) { return dim3((nx + BX - 1) / BX, (ny + BY - 1) / BY); }

// =====================================================================================
// Viscous operator pieces
// =====================================================================================
struct CompactUV {
    const double* u;
    const double* v;
    int Nx;
    __device__ __forceinline__ double U(int i, int j) const { return u[cidx(i, j, Nx)]; }
    __device__ __forceinline__ double V(int i, int j) const { return v[cidx(i, j, Nx)]; }
};

// Matrix part of the viscous operator (no boundary data), rows u(i,j) and v(i,j).
template <class X>
__device__ void visc_A(const Params& P, const MuField& mu, const X& x, int i, int j, double& au, double& av) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const double ihx = P.g.ihx, ihy = P.g.ihy;
    const bool px = P.g.px, py = P.g.py;
    auto txx = [&](int c, int r) {
        double nxt = c < Nx - 1 ? x.U(c + 1, r) : (px ? x.U(0, r) : 0.0);
        return 2.0 * mu.c(c, r) * ((nxt - x.U(c, r)) * ihx);
    };
    auto tyy = [&](int c, int r) {
        double nxt = r < Ny - 1 ? x.V(c, r + 1) : (py ? x.V(c, 0) : 0.0);
        return 2.0 * mu.c(c, r) * ((nxt - x.V(c, r)) * ihy);
    };
    auto txy = [&](int c, int r) {
        double duy = r > 0 ? (x.U(c, r) - x.U(c, r - 1)) * ihy : (py ? (x.U(c, 0) - x.U(c, Ny - 1)) * ihy : 0.0);
        double dvx = c > 0 ? (x.V(c, r) - x.V(c - 1, r)) * ihx : (px ? (x.V(0, r) - x.V(Nx - 1, r)) * ihx : 0.0);
        return 2.0 * mu.k(c, r) * (0.5 * duy + 0.5 * dvx);
    };
    double axx = txx(i, j) - (i > 0 ? txx(i - 1, j) : (px ? txx(Nx - 1, j) : 0.0));
    double axy = -txy(i, j) + (j < Ny - 1 ? txy(i, j + 1) : (py ? txy(i, 0) : 0.0));
    au = axx * ihx + axy * ihy;
    double ayx = -txy(i, j) + (i < Nx - 1 ? txy(i + 1, j) : (px ? txy(0, j) : 0.0));
    double ayy = tyy(i, j) - (j > 0 ? tyy(i, j - 1) : (py ? tyy(i, Ny - 1) : 0.0));
    av = ayx * ihx + ayy * ihy;
    if (!py) {
        if (j == 0 && P.bu.s[BOTTOM].type == EFSI_BC_DIRICHLET) au -= mu.k(i, 0) / (P.g.hy * (0.5 * P.g.hy)) * x.U(i, 0);
        if (j == Ny - 1 && P.bu.s[TOP].type == EFSI_BC_DIRICHLET)
            au -= mu.k(i, Ny) / (P.g.hy * (0.5 * P.g.hy)) * x.U(i, Ny - 1);
    }
    if (!px) {
        if (i == 0 && P.bv.s[LEFT].type == EFSI_BC_DIRICHLET) av -= mu.k(0, j) / (P.g.hx * (0.5 * P.g.hx)) * x.V(0, j);
        if (i == Nx - 1 && P.bv.s[RIGHT].type == EFSI_BC_DIRICHLET)
            av -= mu.k(Nx, j) / (P.g.hx * (0.5 * P.g.hx)) * x.V(Nx - 1, j);
    }
}

// Diagonal of the viscous operator A at rows u(i,j), v(i,j).
__device__ void visc_diag(const Params& P, const MuField& mu, int i, int j, double& du, double& dv) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const bool px = P.g.px, py = P.g.py;
    const double ihx2 = P.g.ihx * P.g.ihx, ihy2 = P.g.ihy * P.g.ihy;
    double a = 2.0 * mu.c(i, j) + ((i > 0 || px) ? 2.0 * mu.c(wrapi(i - 1, Nx), j) : 0.0);
    double b = ((j > 0 || py) ? mu.k(i, j) : 0.0) + ((j < Ny - 1 || py) ? mu.k(i, j + 1) : 0.0);
    du = -a * ihx2 - b * ihy2;
    double c = ((i > 0 || px) ? mu.k(i, j) : 0.0) + ((i < Nx - 1 || px) ? mu.k(i + 1, j) : 0.0);
    double d = 2.0 * mu.c(i, j) + ((j > 0 || py) ? 2.0 * mu.c(i, wrapi(j - 1, Ny)) : 0.0);
    dv = -c * ihx2 - d * ihy2;
    if (!py) {
        if (j == 0 && P.bu.s[BOTTOM].type == EFSI_BC_DIRICHLET) du -= mu.k(i, 0) / (P.g.hy * (0.5 * P.g.hy));
        if (j == Ny - 1 && P.bu.s[TOP].type == EFSI_BC_DIRICHLET) du -= mu.k(i, Ny) / (P.g.hy * (0.5 * P.g.hy));
    }
    if (!px) {
        if (i == 0 && P.bv.s[LEFT].type == EFSI_BC_DIRICHLET) dv -= mu.k(0, j) / (P.g.hx * (0.5 * P.g.hx));
        if (i == Nx - 1 && P.bv.s[RIGHT].type == EFSI_BC_DIRICHLET) dv -= mu.k(Nx, j) / (P.g.hx * (0.5 * P.g.hx));
    }
}

// Dirichlet rows of the compact system (velocity_dirichlet_data, Operators.jl:1085-1110).
__device__ __forceinline__ bool u_fixed(const Params& P, int i) {
    return !P.g.px && i == 0 && P.bu.s[LEFT].type == EFSI_BC_DIRICHLET;
}
__device__ __forceinline__ bool v_fixed(const Params& P, int j) {
    return !P.g.py && j == 0 && P.bv.s[BOTTOM].type == EFSI_BC_DIRICHLET;
}

// x0 = uv_n with the Dirichlet rows set to their data (the reference's GMRES start,
// TimeIntegrationIMEX.jl:807, after _impose_row_dirichlet).
__global__ void k_visc_x0(Params P, const double* __restrict__ Un, const double* __restrict__ Vn, double* xu,
                          double* xv) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx;
    if (i >= Nx || j >= P.g.Ny) return;
    size_t k = cidx(i, j, Nx);
    xu[k] = u_fixed(P, i) ? bval(P.bu.s[LEFT], j) : Un[uidx(i, j, Nx)];
    xv[k] = v_fixed(P, j) ? bval(P.bv.s[BOTTOM], i) : Vn[vidx(i, j, Nx)];
}

__global__ void k_visc_init(Params P, DtCoef ac, double reltol, int maxiter, const double* __restrict__ xu,
                            const double* __restrict__ xv, const double* __restrict__ rhs_u,
                            const double* __restrict__ rhs_v, const double* __restrict__ phi, double* ru, double* rv,
                            double* dinv_u, double* dinv_v, CGScal* cg, RedSlot rs, int* iters_out,
                            cudaGraphConditionalHandle cond) {
    __shared__ double sh[64];
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx;
    const double alpha = ac.value();
    double acc[2] = {0.0, 0.0};
    if (i < Nx && j < P.g.Ny) {
        MuField mu = make_mu(P, phi);
        CompactUV x{xu, xv, Nx};
        double au, av, du, dv;
        visc_A(P, mu, x, i, j, au, av);
        visc_diag(P, mu, i, j, du, dv);
        size_t k = cidx(i, j, Nx);
        double r1 = u_fixed(P, i) ? 0.0 : rhs_u[k] - (xu[k] - alpha * au);
        double r2 = v_fixed(P, j) ? 0.0 : rhs_v[k] - (xv[k] - alpha * av);
        double d1 = u_fixed(P, i) ? 0.0 : 1.0 / (1.0 - alpha * du);
        double d2 = v_fixed(P, j) ? 0.0 : 1.0 / (1.0 - alpha * dv);
        ru[k] = r1;
        rv[k] = r2;
        dinv_u[k] = d1;
        dinv_v[k] = d2;
        acc[0] = r1 * r1 + r2 * r2;
        acc[1] = r1 * r1 * d1 + r2 * r2 * d2;
    }
    double tot[2];
    if (grid_reduce<2>(acc, rs, tot, sh) && threadIdx.x == 0 && threadIdx.y == 0) {
        cg->rr0 = tot[0];
        cg->rr = tot[0];
        cg->rz = tot[1];
        cg->tol2 = reltol * reltol * tot[0];
        cg->iter = 0;
        cg->maxiter = maxiter;
        cg->beta = 0.0;
        cg->conv = tot[0] == 0.0 ? 1 : 0;
        cg->done = (cg->conv || !isfinite(tot[0])) ? 1 : 0;  // a non-finite start ends at once
        if (iters_out) *iters_out = 0;
        set_loop(cond, !cg->done);
    }
}

// p = D^-1 r + beta*p (Jacobi-preconditioned search direction; zero on Dirichlet rows).
__global__ void k_visc_pupdate(int n, const double* __restrict__ ru, const double* __restrict__ rv,
                               const double* __restrict__ dinv_u, const double* __restrict__ dinv_v, double* pu,
                               double* pv, const CGScal* cg) {
    if (cg->done) return;
    const int first = cg->iter == 0;
    const double beta = first ? 0.0 : cg->beta;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        double a = ru[k] * dinv_u[k], b = rv[k] * dinv_v[k];
        pu[k] = first ? a : a + beta * pu[k];
        pv[k] = first ? b : b + beta * pv[k];
    }
}

// Ap = (I - alpha*A) p on the free rows (0 on Dirichlet rows), partial p.Ap -> alpha_cg.
__global__ void k_visc_matvec(Params P, DtCoef ac, const double* __restrict__ phi, const double* __restrict__ pu,
                              const double* __restrict__ pv, double* Apu, double* Apv, CGScal* cg, RedSlot rs) {
    __shared__ double sh[32];
    if (cg->done) return;
    const double alpha = ac.value();
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    double acc[1] = {0.0};
    if (i < Nx && j < Ny) {
        MuField mu = make_mu(P, phi);
        CompactUV x{pu, pv, Nx};
        size_t k = cidx(i, j, Nx);
        double au, av;
        visc_A(P, mu, x, i, j, au, av);
        double a = pu[k], b = pv[k];
        double qa = u_fixed(P, i) ? 0.0 : a - alpha * au;
        double qb = v_fixed(P, j) ? 0.0 : b - alpha * av;
        Apu[k] = qa; Apv[k] = qb;
        acc[0] = a * qa + b * qb;
    }
    double tot[1];
    if (grid_reduce<1>(acc, rs, tot, sh) && threadIdx.x == 0 && threadIdx.y == 0) {
        cg->pAp = tot[0];
        cg->alpha = tot[0] != 0.0 ? cg->rz / tot[0] : 0.0;
    }
}

// x += a p, r -= a Ap, partial |r|^2 and r.z  ->  convergence and beta.
__global__ void k_visc_update(Params P, const double* __restrict__ dinv_u, const double* __restrict__ dinv_v,
                              double* xu, double* xv, double* ru, double* rv, const double* __restrict__ pu,
                              const double* __restrict__ pv, const double* __restrict__ Apu,
                              const double* __restrict__ Apv, CGScal* cg, RedSlot rs, int* iters_out,
                              cudaGraphConditionalHandle cond) {
    __shared__ double sh[64];
    if (cg->done) return;
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx;
    const double a = cg->alpha;
    double acc[2] = {0.0, 0.0};
    if (i < Nx && j < P.g.Ny) {
        size_t k = cidx(i, j, Nx);
        xu[k] += a * pu[k];
        xv[k] += a * pv[k];
        double r1 = ru[k] - a * Apu[k], r2 = rv[k] - a * Apv[k];
        ru[k] = r1; rv[k] = r2;
        acc[0] = r1 * r1 + r2 * r2;
        acc[1] = r1 * r1 * dinv_u[k] + r2 * r2 * dinv_v[k];
    }
    double tot[2];
    if (grid_reduce<2>(acc, rs, tot, sh) && threadIdx.x == 0 && threadIdx.y == 0) {
        cg->iter += 1;
        cg->rr = tot[0];
        cg->beta = cg->rz != 0.0 ? tot[1] / cg->rz : 0.0;
        cg->rz = tot[1];
        if (tot[0] <= cg->tol2) { cg->conv = 1; cg->done = 1; }
        else if (cg->iter >= cg->maxiter || !isfinite(tot[0])) cg->done = 1;
        if (iters_out) *iters_out = cg->iter;
        set_loop(cond, !cg->done);
    }
}

void visc_init(const Params& P, DtCoef alpha, double reltol, int maxiter, const double* Un, const double* Vn,
               const double* rhs_u, const double* rhs_v, const double* phi, const ViscSolve& w, CGScal* cg,
               const RedSlot& rs, int* iters_out, cudaGraphConditionalHandle cond, cudaStream_t s) {
    dim3 g = grid2(P.g.Nx, P.g.Ny), b(BX, BY);
    k_visc_x0<<<g, b, 0, s>>>(P, Un, Vn, w.x_u, w.x_v);
    k_visc_init<<<g, b, 0, s>>>(P, alpha, reltol, maxiter, w.x_u, w.x_v, rhs_u, rhs_v, phi, w.r_u, w.r_v, w.dinv_u,
                                w.dinv_v, cg, rs, iters_out, cond);
}

void visc_matvec(const Params& P, DtCoef alpha, const double* phi, const ViscSolve& w, CGScal* cg, const RedSlot& rs,
                 cudaStream_t s) {
    const int n = P.g.Nx * P.g.Ny;
    k_visc_pupdate<<<std::min((n + 255) / 256, 148 * 8), 256, 0, s>>>(n, w.r_u, w.r_v, w.dinv_u, w.dinv_v, w.p_u[0],
                                                                     w.p_v[0], cg);
    k_visc_matvec<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, alpha, phi, w.p_u[0], w.p_v[0], w.Ap_u, w.Ap_v,
                                                              cg, rs);
}
void visc_update(const Params& P, const ViscSolve& w, CGScal* cg, const RedSlot& rs, int* iters_out,
                 cudaGraphConditionalHandle cond, cudaStream_t s) {
    k_visc_update<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, w.dinv_u, w.dinv_v, w.x_u, w.x_v, w.r_u, w.r_v,
                                                              w.p_u[0], w.p_v[0], w.Ap_u, w.Ap_v, cg, rs, iters_out,
                                                              cond);
}

// NoViscosity: predictor = rhs with the Dirichlet rows enforced (:786-788).
__global__ void k_visc_enforce(Params P, const double* __restrict__ ru, const double* __restrict__ rv, double* xu,
                               double* xv) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx;
    if (i >= Nx || j >= P.g.Ny) return;
    size_t k = cidx(i, j, Nx);
    xu[k] = u_fixed(P, i) ? bval(P.bu.s[LEFT], j) : ru[k];
    xv[k] = v_fixed(P, j) ? bval(P.bv.s[BOTTOM], i) : rv[k];
}
void visc_enforce_dirichlet(const Params& P, const double* rhs_u, const double* rhs_v, double* x_u, double* x_v,
                            cudaStream_t s) {
    k_visc_enforce<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, rhs_u, rhs_v, x_u, x_v);
}

// =====================================================================================
// Resource diffusion (I - alpha*L_D) c = rhs
// =====================================================================================
// Face diffusivity (interpolate_center_to_{x,y}_faces of D, constant copy at walls).
__device__ __forceinline__ double Dcell(const Params& P, const double* phi, int i, int j) {
    return diffusivity(P.md, phi[cidx(i, j, P.g.Nx)]);
}
// Matrix part of L_D at (i,j) applied through accessor f, and its diagonal.
template <class F>
__device__ void diff_L(const Params& P, const double* phi, const F& f, int i, int j, double& Lc, double& diag) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const bool px = P.g.px, py = P.g.py;
    const double ihx = P.g.ihx, ihy = P.g.ihy;
    const double c = f(i, j);
    double D = Dcell(P, phi, i, j);
    double flux_x[2], flux_y[2], dx[2], dy[2];
    for (int s = 0; s < 2; ++s) {
        // x face i+s
        int fi = i + s;
        if (px || (fi > 0 && fi < Nx)) {
            int nb = s == 0 ? wrapi(i - 1, Nx) : wrapi(i + 1, Nx);
            double Df = 0.5 * D + 0.5 * Dcell(P, phi, nb, j);
            double g = s == 0 ? (c - f(nb, j)) * ihx : (f(nb, j) - c) * ihx;
            flux_x[s] = Df * g;
            dx[s] = Df * ihx;
        } else {
            const SideD& sd = P.bc.s[s == 0 ? LEFT : RIGHT];
            if (bdir(sd, j)) {  // homogeneous Dirichlet part: (c - 0)/(h/2)
                double g = s == 0 ? c / (0.5 * P.g.hx) : -c / (0.5 * P.g.hx);
                flux_x[s] = D * g;
                dx[s] = D / (0.5 * P.g.hx);
            } else {
                flux_x[s] = 0.0;
                dx[s] = 0.0;
            }
        }
        int fj = j + s;
        if (py || (fj > 0 && fj < Ny)) {
            int nb = s == 0 ? wrapi(j - 1, Ny) : wrapi(j + 1, Ny);
            double Df = 0.5 * D + 0.5 * Dcell(P, phi, i, nb);
            double g = s == 0 ? (c - f(i, nb)) * ihy : (f(i, nb) - c) * ihy;
            flux_y[s] = Df * g;
            dy[s] = Df * ihy;
        } else {
            const SideD& sd = P.bc.s[s == 0 ? BOTTOM : TOP];
            if (bdir(sd, i)) {
                double g = s == 0 ? c / (0.5 * P.g.hy) : -c / (0.5 * P.g.hy);
                flux_y[s] = D * g;
                dy[s] = D / (0.5 * P.g.hy);
            } else {
                flux_y[s] = 0.0;
                dy[s] = 0.0;
            }
        }
    }
    Lc = (flux_x[1] - flux_x[0]) * ihx + (flux_y[1] - flux_y[0]) * ihy;
    diag = -(dx[0] + dx[1]) * ihx - (dy[0] + dy[1]) * ihy;
}

__global__ void k_diff_init(Params P, DtCoef ac, double reltol, int maxiter, const double* __restrict__ c0,
                            const double* __restrict__ rhs, const double* __restrict__ phi, double* x, double* r,
                            double* dinv, CGScal* cg, RedSlot rs, int* iters_out, cudaGraphConditionalHandle cond) {
    __shared__ double sh[64];
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx;
    const double alpha = ac.value();
    double acc[2] = {0.0, 0.0};
    if (i < Nx && j < P.g.Ny) {
        auto f = [&](int a, int b) { return c0[cidx(a, b, Nx)]; };
        double L, d;
        diff_L(P, phi, f, i, j, L, d);
        size_t k = cidx(i, j, Nx);
        double rr = rhs[k] - (c0[k] - alpha * L);
        double di = 1.0 / (1.0 - alpha * d);
        x[k] = c0[k];
        r[k] = rr;
        dinv[k] = di;
        acc[0] = rr * rr;
        acc[1] = rr * rr * di;
    }
    double tot[2];
    if (grid_reduce<2>(acc, rs, tot, sh) && threadIdx.x == 0 && threadIdx.y == 0) {
        cg->rr0 = tot[0]; cg->rr = tot[0]; cg->rz = tot[1];
        cg->tol2 = reltol * reltol * tot[0];
        cg->iter = 0; cg->maxiter = maxiter; cg->beta = 0.0;
        cg->conv = tot[0] == 0.0 ? 1 : 0;
        cg->done = (cg->conv || !isfinite(tot[0])) ? 1 : 0;  // a non-finite start ends at once
        if (iters_out) *iters_out = 0;
        set_loop(cond, !cg->done);
    }
}

__global__ void k_diff_pupdate(int n, const double* __restrict__ r, const double* __restrict__ dinv, double* p,
                               const CGScal* cg) {
    if (cg->done) return;
    const int first = cg->iter == 0;
    const double beta = first ? 0.0 : cg->beta;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        double z = r[k] * dinv[k];
        p[k] = first ? z : z + beta * p[k];
    }
}

__global__ void k_diff_matvec(Params P, DtCoef ac, const double* __restrict__ phi, const double* __restrict__ p,
                              double* Ap, CGScal* cg, RedSlot rs) {
    __shared__ double sh[32];
    if (cg->done) return;
    const double alpha = ac.value();
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx;
    double acc[1] = {0.0};
    if (i < Nx && j < P.g.Ny) {
        auto f = [&](int a, int b) { return p[cidx(a, b, Nx)]; };
        double L, d;
        diff_L(P, phi, f, i, j, L, d);
        size_t k = cidx(i, j, Nx);
        double q = p[k] - alpha * L;
        Ap[k] = q;
        acc[0] = p[k] * q;
    }
    double tot[1];
    if (grid_reduce<1>(acc, rs, tot, sh) && threadIdx.x == 0 && threadIdx.y == 0) {
        cg->pAp = tot[0];
        cg->alpha = tot[0] != 0.0 ? cg->rz / tot[0] : 0.0;
    }
}

__global__ void k_diff_update(Params P, const double* __restrict__ dinv, double* x, double* r,
                              const double* __restrict__ p, const double* __restrict__ Ap, CGScal* cg, RedSlot rs,
                              int* iters_out, cudaGraphConditionalHandle cond) {
    __shared__ double sh[64];
    if (cg->done) return;
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx;
    const double a = cg->alpha;
    double acc[2] = {0.0, 0.0};
    if (i < Nx && j < P.g.Ny) {
        size_t k = cidx(i, j, Nx);
        x[k] += a * p[k];
        double rr = r[k] - a * Ap[k];
        r[k] = rr;
        acc[0] = rr * rr;
        acc[1] = rr * rr * dinv[k];
    }
    double tot[2];
    if (grid_reduce<2>(acc, rs, tot, sh) && threadIdx.x == 0 && threadIdx.y == 0) {
        cg->iter += 1;
        cg->rr = tot[0];
        cg->beta = cg->rz != 0.0 ? tot[1] / cg->rz : 0.0;
        cg->rz = tot[1];
        if (tot[0] <= cg->tol2) { cg->conv = 1; cg->done = 1; }
        else if (cg->iter >= cg->maxiter || !isfinite(tot[0])) cg->done = 1;
        if (iters_out) *iters_out = cg->iter;
        set_loop(cond, !cg->done);
    }
}

void diff_init(const Params& P, DtCoef alpha, double reltol, int maxiter, const double* c0, const double* rhs,
               const double* phi, const ScalarSolve& w, CGScal* cg, const RedSlot& rs, int* iters_out,
               cudaGraphConditionalHandle cond, cudaStream_t s) {
    k_diff_init<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, alpha, reltol, maxiter, c0, rhs, phi, w.x, w.r,
                                                              w.dinv, cg, rs, iters_out, cond);
}
void diff_iter(const Params& P, DtCoef alpha, const double* phi, const ScalarSolve& w, CGScal* cg, const RedSlot& rs1,
               const RedSlot& rs2, int* iters_out, cudaGraphConditionalHandle cond, cudaStream_t s) {
    dim3 g = grid2(P.g.Nx, P.g.Ny), b(BX, BY);
    const int n = P.g.Nx * P.g.Ny;
    k_diff_pupdate<<<std::min((n + 255) / 256, 148 * 8), 256, 0, s>>>(n, w.r, w.dinv, w.p[0], cg);
    k_diff_matvec<<<g, b, 0, s>>>(P, alpha, phi, w.p[0], w.Ap, cg, rs1);
    k_diff_update<<<g, b, 0, s>>>(P, w.dinv, w.x, w.r, w.p[0], w.Ap, cg, rs2, iters_out, cond);
}

// =====================================================================================
// Projection: weighted Poisson operator, multigrid V-cycle, CG
// =====================================================================================
// K x at one cell of a level: diag*x - off, off = sum of neighbour couplings.
__device__ __forceinline__ void lev_diag(const MGLevel& L, int px, int py, int i, int j, double& diag) {
    diag = 0.0;
    diag += (i > 0 || px) ? L.ax : L.ax * L.cl[j];
    diag += (i < L.nx - 1 || px) ? L.ax : L.ax * L.cr[j];
    diag += (j > 0 || py) ? L.ay : L.ay * L.cb[i];
    diag += (j < L.ny - 1 || py) ? L.ay : L.ay * L.ct[i];
}
template <class F>
__device__ __forceinline__ double lev_off(const MGLevel& L, int px, int py, int i, int j, const F& x) {
    double off = 0.0;
    if (i > 0) off += L.ax * x(i - 1, j); else if (px) off += L.ax * x(L.nx - 1, j);
    if (i < L.nx - 1) off += L.ax * x(i + 1, j); else if (px) off += L.ax * x(0, j);
    if (j > 0) off += L.ay * x(i, j - 1); else if (py) off += L.ay * x(i, L.ny - 1);
    if (j < L.ny - 1) off += L.ay * x(i, j + 1); else if (py) off += L.ay * x(i, 0);
    return off;
}
__device__ __forceinline__ bool lev_rb(const MGLevel& L, int px, int py) {
    return !((px && (L.nx & 1)) || (py && (L.ny & 1)));  // valid red-black colouring
}
static constexpr double JACOBI_W = 0.8;

// Pre-smoothing from x = 0: red cells x = b/D, black cells one GS update
// (or one damped-Jacobi sweep when the periodic colouring is not bipartite).
__global__ void k_mg_pre(MGLevel L, int px, int py, const double* __restrict__ b, double* x, const CGScal* cg) {
    if (cg && cg->done) return;
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    if (i >= L.nx || j >= L.ny) return;
    const int nx = L.nx;
    double d;
    lev_diag(L, px, py, i, j, d);
    double bc = b[cidx(i, j, nx)];
    double out;
    if (!lev_rb(L, px, py)) out = JACOBI_W * bc / d;
    else if (((i + j) & 1) == 0) out = bc / d;
    else {
        auto red = [&](int a, int c) {
            double dd;
            lev_diag(L, px, py, a, c, dd);
            return b[cidx(a, c, nx)] / dd;
        };
        out = (bc + lev_off(L, px, py, i, j, red)) / d;
    }
    x[cidx(i, j, nx)] = out;
}

__global__ void k_mg_resid(MGLevel L, int px, int py, const double* __restrict__ b, const double* __restrict__ x,
                           double* r, const CGScal* cg) {
    if (cg && cg->done) return;
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    if (i >= L.nx || j >= L.ny) return;
    const int nx = L.nx;
    double d;
    lev_diag(L, px, py, i, j, d);
    auto xf = [&](int a, int c) { return x[cidx(a, c, nx)]; };
    r[cidx(i, j, nx)] = b[cidx(i, j, nx)] - (d * x[cidx(i, j, nx)] - lev_off(L, px, py, i, j, xf));
}

// Restriction b_c = P^T r (bilinear weights, reflection at walls, wrap when periodic).
__device__ __forceinline__ void rweights(int I, int nc, bool per, int (&f)[4], double (&w)[4]) {
    f[0] = 2 * I - 1; w[0] = 0.25;
    f[1] = 2 * I;     w[1] = 0.75 + ((I == 0 && !per) ? 0.25 : 0.0);
    f[2] = 2 * I + 1; w[2] = 0.75 + ((I == nc - 1 && !per) ? 0.25 : 0.0);
    f[3] = 2 * I + 2; w[3] = 0.25;
    const int nf = 2 * nc;
    if (f[0] < 0) { if (per) f[0] += nf; else w[0] = 0.0; }
    if (f[3] >= nf) { if (per) f[3] -= nf; else w[3] = 0.0; }
}
__global__ void k_mg_restrict(MGLevel F, MGLevel C, int px, int py, const double* __restrict__ r, double* bc,
                              const CGScal* cg) {
    if (cg && cg->done) return;
    const int I = blockIdx.x * BX + threadIdx.x, J = blockIdx.y * BY + threadIdx.y;
    if (I >= C.nx || J >= C.ny) return;
    int fx[4], fy[4];
    double wx[4], wy[4];
    rweights(I, C.nx, px, fx, wx);
    rweights(J, C.ny, py, fy, wy);
    double s = 0.0;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        if (wy[b] == 0.0) continue;
        double row = 0.0;
#pragma unroll
        for (int a = 0; a < 4; ++a)
            if (wx[a] != 0.0) row += wx[a] * r[cidx(fx[a], fy[b], F.nx)];
        s += wy[b] * row;
    }
    bc[cidx(I, J, C.nx)] = s;
}

// Bilinear prolongation value (P e) at fine cell (i,j).
__device__ __forceinline__ double prolong(const MGLevel& C, int px, int py, const double* e, int i, int j) {
    auto pair = [](int f, int nc, bool per, int& I0, int& I1) {
        I0 = f / 2;
        I1 = (f & 1) ? I0 + 1 : I0 - 1;
        if (I1 < 0) I1 = per ? nc - 1 : I0;
        if (I1 >= nc) I1 = per ? 0 : I0;
    };
    int I0, I1, J0, J1;
    pair(i, C.nx, px, I0, I1);
    pair(j, C.ny, py, J0, J1);
    auto E = [&](int a, int b) { return e[cidx(a, b, C.nx)]; };
    return 0.75 * (0.75 * E(I0, J0) + 0.25 * E(I1, J0)) + 0.25 * (0.75 * E(I0, J1) + 0.25 * E(I1, J1));
}

// x_out = x + P e on red cells; black cells are smoothed against the corrected red
// neighbours (the first half of the post-smoothing black-then-red sweep).
__global__ void k_mg_prolong_black(MGLevel F, MGLevel C, int px, int py, const double* __restrict__ x,
                                   const double* __restrict__ e, const double* __restrict__ b, double* xo,
                                   const CGScal* cg) {
    if (cg && cg->done) return;
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    if (i >= F.nx || j >= F.ny) return;
    const int nx = F.nx;
    auto xc = [&](int a, int c) { return x[cidx(a, c, nx)] + prolong(C, px, py, e, a, c); };
    double out;
    double d;
    lev_diag(F, px, py, i, j, d);
    if (!lev_rb(F, px, py)) {
        double xx = xc(i, j);
        out = xx + JACOBI_W * (b[cidx(i, j, nx)] - (d * xx - lev_off(F, px, py, i, j, xc))) / d;
    } else if (((i + j) & 1) == 0) {
        out = xc(i, j);
    } else {
        out = (b[cidx(i, j, nx)] + lev_off(F, px, py, i, j, xc)) / d;
    }
    xo[cidx(i, j, nx)] = out;
}

// Red half of the post-smoothing; on the fine level it also forms r.z for CG.
__global__ void k_mg_red(MGLevel L, int px, int py, const double* __restrict__ b, double* xo, CGScal* cg,
                         RedSlot rs, int dot) {
    __shared__ double sh[32];
    if (cg && cg->done) return;
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int nx = L.nx;
    double acc[1] = {0.0};
    const bool inside = i < L.nx && j < L.ny;
    if (inside) {
        double val = xo[cidx(i, j, nx)];
        if (lev_rb(L, px, py) && ((i + j) & 1) == 0) {
            double d;
            lev_diag(L, px, py, i, j, d);
            auto xf = [&](int a, int c) { return xo[cidx(a, c, nx)]; };
            val = (b[cidx(i, j, nx)] + lev_off(L, px, py, i, j, xf)) / d;
            xo[cidx(i, j, nx)] = val;
        }
        acc[0] = b[cidx(i, j, nx)] * val;
    }
    if (!dot) return;
    double tot[1];
    if (grid_reduce<1>(acc, rs, tot, sh) && threadIdx.x == 0 && threadIdx.y == 0) {
        cg->beta = cg->rz != 0.0 ? tot[0] / cg->rz : 0.0;
        cg->rz = tot[0];
    }
}

// Coarsest level: x = Minv b with the dense (shifted) inverse; 8 rows per block.
__global__ void k_mg_dense(int n, const double* __restrict__ Minv, const double* __restrict__ b, double* x,
                           const CGScal* cg) {
    if (cg && cg->done) return;
    __shared__ double sb[1024];
    for (int k = threadIdx.x; k < n; k += blockDim.x) sb[k] = b[k];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row = blockIdx.x * 8 + warp;
    if (row < n) {
        double s = 0.0;
        for (int k = lane; k < n; k += 32) s += Minv[(size_t)row * n + k] * sb[k];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) x[row] = s;
    }
}

// r.z for CG when the whole problem is the dense coarse level.
__global__ void k_dot_rz(int n, const double* __restrict__ r, const double* __restrict__ z, CGScal* cg, RedSlot rs) {
    __shared__ double sh[32];
    if (cg->done) return;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[1] = {k < n ? r[k] * z[k] : 0.0};
    double tot[1];
    if (grid_reduce<1>(acc, rs, tot, sh) && threadIdx.x == 0) {
        cg->beta = cg->rz != 0.0 ? tot[0] / cg->rz : 0.0;
        cg->rz = tot[0];
    }
}

static void vcycle(const Projection& pj, int l, const double* b, double* out, CGScal* cg, const RedSlot& rs,
                   int px, int py, cudaStream_t s) {
    const MGLevel& L = pj.lev[l];
    if (l == pj.nlev - 1) {
        k_mg_dense<<<(pj.nc + 7) / 8, 256, 0, s>>>(pj.nc, pj.coarse_inv, b, out, cg);
        if (l == 0) k_dot_rz<<<(pj.nc + 255) / 256, 256, 0, s>>>(pj.nc, b, out, cg, rs);
        return;
    }
    const MGLevel& C = pj.lev[l + 1];
    dim3 g = grid2(L.nx, L.ny), gc = grid2(C.nx, C.ny), bk(BX, BY);
    k_mg_pre<<<g, bk, 0, s>>>(L, px, py, b, L.x, cg);
    k_mg_resid<<<g, bk, 0, s>>>(L, px, py, b, L.x, L.r, cg);
    k_mg_restrict<<<gc, bk, 0, s>>>(L, C, px, py, L.r, C.b, cg);
    vcycle(pj, l + 1, C.b, C.xo, cg, rs, px, py, s);
    k_mg_prolong_black<<<g, bk, 0, s>>>(L, C, px, py, L.x, C.xo, b, out, cg);
    k_mg_red<<<g, bk, 0, s>>>(L, px, py, b, out, cg, rs, l == 0 ? 1 : 0);
}

int proj_kernels_per_iter(const Projection& pj) { return 2 + 6 * (pj.nlev - 1) + 1; }

// ---- right-hand side (Projection.jl:198-221) -----------------------------------------------
__device__ __forceinline__ double q_boundary_vec(const Params& P, int i, int j) {
    // Poisson boundary vector b_bc = Div(gradient_bc) at cell (i,j) (Operators.jl:380-383).
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    double s = 0.0;
    auto side = [&](const SideD& sd, int k, double h) {
        if (bdir(sd, k)) return bval(sd, k) / ((0.5 * h) * h);
        if (sd.type == EFSI_BC_NEUMANN) return bval(sd, k) / h;
        if (sd.type == EFSI_BC_MIXED) return bneu(sd, k) / h;
        return 0.0;
    };
    if (!P.g.px) {
        if (i == 0) s += side(P.bq.s[LEFT], j, P.g.hx);
        if (i == Nx - 1) s += side(P.bq.s[RIGHT], j, P.g.hx);
    }
    if (!P.g.py) {
        if (j == 0) s += side(P.bq.s[BOTTOM], i, P.g.hy);
        if (j == Ny - 1) s += side(P.bq.s[TOP], i, P.g.hy);
    }
    return s;
}

// Predictor face velocity from a compact vector (_inject_compact_predictor!, :543-579)
// or from full MAC arrays.
struct PredIn {
    const double *u, *v;
    int compact;
    __device__ __forceinline__ double U(const Params& P, int i, int j) const {
        const int Nx = P.g.Nx;
        if (!compact) return u[uidx(i, j, Nx)];
        if (i < Nx) return u[cidx(i, j, Nx)];
        return P.g.px ? u[cidx(0, j, Nx)] : bval(P.bu.s[RIGHT], j);
    }
    __device__ __forceinline__ double V(const Params& P, int i, int j) const {
        const int Nx = P.g.Nx, Ny = P.g.Ny;
        if (!compact) return v[vidx(i, j, Nx)];
        if (j < Ny) return v[cidx(i, j, Nx)];
        return P.g.py ? v[cidx(i, 0, Nx)] : bval(P.bv.s[TOP], i);
    }
};

__global__ void k_proj_rhs(Params P, PredIn in, const double* __restrict__ G, double* Up, double* Vp, double* rhs,
                           double* bw, int nullspace, ProjScal* ps, RedSlot rs, DevStatus* st) {
    __shared__ double sh[32 * 6];
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const double area = P.g.hx * P.g.hy;
    if (j < Ny && i <= Nx) Up[uidx(i, j, Nx)] = in.U(P, i, j);
    if (i < Nx && j <= Ny) Vp[vidx(i, j, Nx)] = in.V(P, i, j);
    double acc[6] = {0, 0, 0, 0, 0, 0};
    if (i < Nx && j < Ny) {
        double div = (in.U(P, i + 1, j) - in.U(P, i, j)) * P.g.ihx + (in.V(P, i, j + 1) - in.V(P, i, j)) * P.g.ihy;
        double g = G ? G[cidx(i, j, Nx)] : 0.0;
        double rr = (div - g) - q_boundary_vec(P, i, j);
        size_t k = cidx(i, j, Nx);
        rhs[k] = rr;
        double b = -rr * area;
        bw[k] = b;
        acc[0] = rr * area;
        acc[1] = fabs(rr) * area;
        acc[2] = b;
        acc[3] = rr * rr;
        acc[4] = div * div * area;
        acc[5] = g * g * area;
    }
    double tot[6];
    if (grid_reduce<6>(acc, rs, tot, sh) && threadIdx.x == 0 && threadIdx.y == 0) {
        for (int k = 0; k < 6; ++k) ps->v[k] = tot[k];
        ps->v[10] = nullspace ? tot[2] / ((double)Nx * Ny) : 0.0;
        if (nullspace) {
            double tol = 1e-12 + 1e-10 * fmax(tot[1], 2.220446049250313e-16);
            if (!(fabs(tot[0]) <= tol)) raise_err(st, DE_INCOMPATIBLE, 0, -1, -1, tot[0]);
        }
    }
}

void proj_rhs(const Params& P, const Projection& pj, bool compact_in, const double* u_in, const double* v_in,
              const double* G, ProjScal* ps, const RedSlot& rs, DevStatus* st, cudaStream_t s) {
    PredIn in{u_in, v_in, compact_in ? 1 : 0};
    k_proj_rhs<<<grid2(P.g.Nx + 1, P.g.Ny + 1), dim3(BX, BY), 0, s>>>(P, in, G, pj.Up, pj.Vp, pj.rhs, pj.b,
                                                                     pj.nullspace ? 1 : 0, ps, rs, st);
}

// ---- CG on the fine level --------------------------------------------------------------------
__global__ void k_pcg_init(MGLevel L, int px, int py, double reltol, int maxiter, const double* __restrict__ q0,
                           const double* __restrict__ b, double* x, double* r, const ProjScal* ps, CGScal* cg,
                           RedSlot rs, const DevStatus* st, int* iters_out, cudaGraphConditionalHandle cond) {
    __shared__ double sh[32];
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int nx = L.nx;
    const double bmean = ps->v[10];
    double acc[1] = {0.0};
    if (i < L.nx && j < L.ny) {
        double d;
        lev_diag(L, px, py, i, j, d);
        auto xf = [&](int a, int c) { return q0[cidx(a, c, nx)]; };
        size_t k = cidx(i, j, nx);
        double rr = (b[k] - bmean) - (d * q0[k] - lev_off(L, px, py, i, j, xf));
        x[k] = q0[k];
        r[k] = rr;
        acc[0] = rr * rr;
    }
    double tot[1];
    if (grid_reduce<1>(acc, rs, tot, sh) && threadIdx.x == 0 && threadIdx.y == 0) {
        cg->rr0 = tot[0]; cg->rr = tot[0];
        cg->tol2 = reltol * reltol * tot[0];
        cg->iter = 0; cg->maxiter = maxiter; cg->beta = 0.0; cg->rz = 1.0;
        cg->conv = tot[0] == 0.0 ? 1 : 0;
        // a flagged step skips its solves (the state is not committed)
        cg->done = (cg->conv || st->code != 0) ? 1 : 0;
        if (iters_out) *iters_out = 0;
        set_loop(cond, !cg->done);
    }
}

__global__ void k_pcg_matvec(MGLevel L, int px, int py, const double* __restrict__ z,
                             const double* __restrict__ p_old, double* p, double* Ap, CGScal* cg, RedSlot rs) {
    __shared__ double sh[32];
    if (cg->done) return;
    const int first = cg->iter == 0;
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int nx = L.nx;
    const double beta = first ? 0.0 : cg->beta;
    auto pn = [&](int a, int c) {
        size_t k = cidx(a, c, nx);
        return first ? z[k] : z[k] + beta * p_old[k];
    };
    double acc[1] = {0.0};
    if (i < L.nx && j < L.ny) {
        double d;
        lev_diag(L, px, py, i, j, d);
        double pc = pn(i, j);
        double q = d * pc - lev_off(L, px, py, i, j, pn);
        size_t k = cidx(i, j, nx);
        p[k] = pc;
        Ap[k] = q;
        acc[0] = pc * q;
    }
    double tot[1];
    if (grid_reduce<1>(acc, rs, tot, sh) && threadIdx.x == 0 && threadIdx.y == 0) {
        cg->pAp = tot[0];
        cg->alpha = tot[0] != 0.0 ? cg->rz / tot[0] : 0.0;
    }
}

__global__ void k_pcg_update(MGLevel L, double* x, double* r, const double* __restrict__ p,
                             const double* __restrict__ Ap, CGScal* cg, RedSlot rs, int* iters_out,
                             cudaGraphConditionalHandle cond) {
    __shared__ double sh[32];
    if (cg->done) return;
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const double a = cg->alpha;
    double acc[1] = {0.0};
    if (i < L.nx && j < L.ny) {
        size_t k = cidx(i, j, L.nx);
        x[k] += a * p[k];
        double rr = r[k] - a * Ap[k];
        r[k] = rr;
        acc[0] = rr * rr;
    }
    double tot[1];
    if (grid_reduce<1>(acc, rs, tot, sh) && threadIdx.x == 0 && threadIdx.y == 0) {
        cg->iter += 1;
        cg->rr = tot[0];
        if (tot[0] <= cg->tol2) { cg->conv = 1; cg->done = 1; }
        else if (cg->iter >= cg->maxiter || !isfinite(tot[0])) cg->done = 1;
        if (iters_out) *iters_out = cg->iter;
        set_loop(cond, !cg->done);
    }
}

void proj_cg_init(const Params& P, const Projection& pj, double reltol, int maxiter, const double* q0, CGScal* cg,
                  const ProjScal* ps, const RedSlot& rs, const RedSlot& rs2, const DevStatus* st, int* iters_out,
                  cudaGraphConditionalHandle cond, cudaStream_t s) {
    const MGLevel& L = pj.lev[0];
    k_pcg_init<<<grid2(L.nx, L.ny), dim3(BX, BY), 0, s>>>(L, P.g.px, P.g.py, reltol, maxiter, q0, pj.b, pj.x, pj.r,
                                                          ps, cg, rs, st, iters_out, cond);
    vcycle(pj, 0, pj.r, pj.z, cg, rs2, P.g.px, P.g.py, s);
}

// One CG iteration; `parity` selects the search-direction buffers (p[parity] is written).
void proj_matvec(const Params& P, const Projection& pj, int parity, CGScal* cg, const RedSlot& rs, cudaStream_t s) {
    const MGLevel& L = pj.lev[0];
    const int cur = parity & 1, old = cur ^ 1;
    k_pcg_matvec<<<grid2(L.nx, L.ny), dim3(BX, BY), 0, s>>>(L, P.g.px, P.g.py, pj.z, pj.p[old], pj.p[cur], pj.Ap, cg,
                                                            rs);
}
void proj_update(const Params& P, const Projection& pj, int parity, CGScal* cg, const RedSlot& rs, int* iters_out,
                 cudaGraphConditionalHandle cond, cudaStream_t s) {
    const MGLevel& L = pj.lev[0];
    const int cur = parity & 1;
    k_pcg_update<<<grid2(L.nx, L.ny), dim3(BX, BY), 0, s>>>(L, pj.x, pj.r, pj.p[cur], pj.Ap, cg, rs, iters_out, cond);
}
void proj_vcycle(const Params& P, const Projection& pj, CGScal* cg, const RedSlot& rs, cudaStream_t s) {
    vcycle(pj, 0, pj.r, pj.z, cg, rs, P.g.px, P.g.py, s);
}

// ---- correction and diagnostics (Projection.jl:253-306) ---------------------------------------
__global__ void k_proj_mean(MGLevel L, const double* __restrict__ x, ProjScal* ps, RedSlot rs, int nullspace) {
    __shared__ double sh[32];
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    double acc[1] = {0.0};
    if (i < L.nx && j < L.ny) acc[0] = x[cidx(i, j, L.nx)];
    double tot[1];
    if (grid_reduce<1>(acc, rs, tot, sh) && threadIdx.x == 0 && threadIdx.y == 0)
        ps->v[6] = nullspace ? tot[0] / ((double)L.nx * L.ny) : 0.0;
}

__device__ __forceinline__ double q_grad_x(const Params& P, const double* x, double mean, int i, int j) {
    const int Nx = P.g.Nx;
    auto q = [&](int a) { return x[cidx(a, j, Nx)] - mean; };
    if (P.g.px) {
        int ic = (i == Nx) ? 0 : i;
        return (q(ic) - q(wrapi(ic - 1, Nx))) * P.g.ihx;
    }
    if (i == 0 || i == Nx) {
        const SideD& s = P.bq.s[i == 0 ? LEFT : RIGHT];
        double in = q(i == 0 ? 0 : Nx - 1), dist = 0.5 * P.g.hx;
        if (bdir(s, j)) return i == 0 ? in / dist - bval(s, j) / dist : bval(s, j) / dist - in / dist;
        if (s.type == EFSI_BC_NEUMANN) return (i == 0 ? -1.0 : 1.0) * bval(s, j);
        if (s.type == EFSI_BC_MIXED) return (i == 0 ? -1.0 : 1.0) * bneu(s, j);
        return 0.0;
    }
    return (q(i) - q(i - 1)) * P.g.ihx;
}
__device__ __forceinline__ double q_grad_y(const Params& P, const double* x, double mean, int i, int j) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    auto q = [&](int b) { return x[cidx(i, b, Nx)] - mean; };
    if (P.g.py) {
        int jc = (j == Ny) ? 0 : j;
        return (q(jc) - q(wrapi(jc - 1, Ny))) * P.g.ihy;
    }
    if (j == 0 || j == Ny) {
        const SideD& s = P.bq.s[j == 0 ? BOTTOM : TOP];
        double in = q(j == 0 ? 0 : Ny - 1), dist = 0.5 * P.g.hy;
        if (bdir(s, i)) return j == 0 ? in / dist - bval(s, i) / dist : bval(s, i) / dist - in / dist;
        if (s.type == EFSI_BC_NEUMANN) return (j == 0 ? -1.0 : 1.0) * bval(s, i);
        if (s.type == EFSI_BC_MIXED) return (j == 0 ? -1.0 : 1.0) * bneu(s, i);
        return 0.0;
    }
    return (q(j) - q(j - 1)) * P.g.ihy;
}

__global__ void k_proj_correct(Params P, MGLevel L, const double* __restrict__ x, const double* __restrict__ Up,
                               const double* __restrict__ Vp, const double* __restrict__ G,
                               const double* __restrict__ rhs, double* q_out, double* U_out, double* V_out,
                               ProjScal* ps, double* stage_linf, RedSlot rmax, RedSlot rsum, DevStatus* st) {
    __shared__ double sh[64];
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const double mean = ps->v[6];
    const double area = P.g.hx * P.g.hy;
    double mx[1] = {0.0}, sm[2] = {0.0, 0.0};
    if (i < Nx && j < Ny) {
        size_t k = cidx(i, j, Nx);
        double uL = Up[uidx(i, j, Nx)] - q_grad_x(P, x, mean, i, j);
        double uR = Up[uidx(i + 1, j, Nx)] - q_grad_x(P, x, mean, i + 1, j);
        double vB = Vp[vidx(i, j, Nx)] - q_grad_y(P, x, mean, i, j);
        double vT = Vp[vidx(i, j + 1, Nx)] - q_grad_y(P, x, mean, i, j + 1);
        U_out[uidx(i, j, Nx)] = uL;
        if (i == Nx - 1) U_out[uidx(Nx, j, Nx)] = uR;
        V_out[vidx(i, j, Nx)] = vB;
        if (j == Ny - 1) V_out[vidx(i, Ny, Nx)] = vT;
        q_out[k] = x[k] - mean;
        double g = G ? G[k] : 0.0;
        double c = ((uR - uL) * P.g.ihx + (vT - vB) * P.g.ihy) - g;
        mx[0] = fabs(c);
        sm[0] = c * c * area;
        // linear residual of the unpinned operator: L q - rhs, L q = -(K x)/area
        double d;
        lev_diag(L, P.g.px, P.g.py, i, j, d);
        auto xf = [&](int a, int b) { return x[cidx(a, b, Nx)] - mean; };
        double Lq = -(d * (x[k] - mean) - lev_off(L, P.g.px, P.g.py, i, j, xf)) / area;
        double lr = Lq - rhs[k];
        sm[1] = lr * lr;
    }
    double t1[1], t2[2];
    bool last1 = grid_reduce<1, true>(mx, rmax, t1, sh);
    if (last1 && threadIdx.x == 0 && threadIdx.y == 0) {
        ps->v[8] = t1[0];
        *stage_linf = fmax(*stage_linf, t1[0]);
    }
    if (grid_reduce<2>(sm, rsum, t2, sh) && threadIdx.x == 0 && threadIdx.y == 0) {
        double LxLy = P.g.Lx * P.g.Ly;
        double l2 = sqrt(t2[0] / LxLy);
        double lin = sqrt(t2[1]) / fmax(sqrt(ps->v[3]), 2.220446049250313e-16);
        ps->v[7] = lin;
        ps->v[9] = l2;
        if (!(lin <= 1e-8)) raise_err(st, DE_PROJ_RESIDUAL, 0, -1, -1, lin);
        double scale = fmax(fmax(sqrt(ps->v[4] / LxLy), sqrt(ps->v[5] / LxLy)), 1.0);
        if (!(l2 <= 1e-12 + 1e-8 * scale)) raise_err(st, DE_PROJ_CONSTRAINT, 0, -1, -1, l2);
    }
}

void proj_finish(const Params& P, const Projection& pj, const double* G, double* q_out, double* U_out, double* V_out,
                 ProjScal* ps, double* stage_linf, const RedSlot& rs1, const RedSlot& rs2, DevStatus* st,
                 cudaStream_t s) {
    const MGLevel& L = pj.lev[0];
    dim3 g = grid2(L.nx, L.ny), b(BX, BY);
    k_proj_mean<<<g, b, 0, s>>>(L, pj.x, ps, rs1, pj.nullspace ? 1 : 0);
    k_proj_correct<<<g, b, 0, s>>>(P, L, pj.x, pj.Up, pj.Vp, G, pj.rhs, q_out, U_out, V_out, ps, stage_linf, rs1,
                                   rs2, st);
}

}  // namespace efsi
