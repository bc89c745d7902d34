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
#include <type_traits>

#include "efsi_device.cuh"
#include "efsi_solvers.cuh"

namespace efsi {

static constexpr int BX = 32, BY = 8;
static inline dim3 grid2(int nx, int ny) { return dim3((nx + BX - 1) / BX, (ny + BY - 1) / BY); }

// Persistent loop over the BX x BY tiles of an nx x ny index space (1-D grid of
// BX x BY blocks); f(i, j) runs for the points inside it.  A kernel that ends in a
// grid reduction accumulates over all its tiles and reduces once per block.
template <class F>
__device__ __forceinline__ void for_tiles(int nx, int ny, F&& f) {
    const int ntx = (nx + BX - 1) / BX, nt = ntx * ((ny + BY - 1) / BY);
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int i = (t % ntx) * BX + threadIdx.x, j = (t / ntx) * BY + threadIdx.y;
        if (i < nx && j < ny) f(i, j);
    }
}
static inline int tiles2(int nx, int ny) { return ((nx + BX - 1) / BX) * ((ny + BY - 1) / BY); }

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

template <class X>
__device__ __forceinline__ void visc_A_any(const Params& P, const MuField& mu, const X& x, int i, int j, double& au,
                                           double& av) {
    if (i >= 1 && i <= P.g.Nx - 2 && j >= 1 && j <= P.g.Ny - 2) visc_A<true>(P, mu, x, i, j, au, av);
    else visc_A<false>(P, mu, x, i, j, au, av);
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

// Start-of-solve scalars of a velocity / resource CG from the squared initial residual
// rr0 and |b|^2; a non-finite start fails at once.
__device__ __forceinline__ void cg_begin(CGScal* cg, const SolveOpts& o, double rr0, double bnorm2) {
    cg->tol2 = o.reltol * o.reltol * rr0;
    cg->iter = 0;
    cg->maxiter = o.maxiter;
    cg->alpha = 0.0;
    cg->beta = 0.0;
    cg->bnorm2 = bnorm2;
    cg->fb_tol = o.fb_tol;
    cg->fallback = o.fallback;
    cg->in_fallback = 0;
    cg->fail_rel = 0.0;
    cg->conv = rr0 == 0.0 ? 1 : 0;
    cg->fail = isfinite(rr0) && isfinite(bnorm2) ? 0 : 1;
    if (cg->fail) cg->fail_rel = NAN;
    cg->done = (cg->conv || cg->fail) ? 1 : 0;
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

__global__ void k_visc_init(Params P, DtCoef ac, SolveOpts o, const double* __restrict__ xu,
                            const double* __restrict__ xv, const double* __restrict__ rhs_u,
                            const double* __restrict__ rhs_v, const double* __restrict__ phi, double* ru, double* rv,
                            double* dinv_u, double* dinv_v, CGScal* cg, RedSlot rs, int* iters_out,
                            cudaGraphConditionalHandle cond) {
    __shared__ double sh[96];
    const int Nx = P.g.Nx;
    const double alpha = ac.value();
    double acc[3] = {0.0, 0.0, 0.0};
    for_tiles(Nx, P.g.Ny, [&](int i, int j) {
        MuField mu = make_mu(P, phi);
        CompactUV x{xu, xv, Nx};
        double au, av, du, dv;
        visc_A_any(P, mu, x, i, j, au, av);
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
        acc[0] += r1 * r1 + r2 * r2;
        acc[1] += r1 * r1 * d1 + r2 * r2 * d2;
        // |b|^2 of the reference's row-eliminated system: Dirichlet rows carry their data
        const double b1 = u_fixed(P, i) ? xu[k] : rhs_u[k], b2 = v_fixed(P, j) ? xv[k] : rhs_v[k];
        acc[2] += b1 * b1 + b2 * b2;
    });
    double tot[3];
    if (grid_reduce<3>(acc, rs, tot, sh) && threadIdx.x == 0 && threadIdx.y == 0) {
        cg->rr0 = tot[0];
        cg->rr = tot[0];
        cg->rz = tot[1];  // gamma_0 = r.M r
        cg_begin(cg, o, tot[0], tot[2]);
        if (iters_out) *iters_out = 0;
        set_loop(cond, !cg->done);
    }
}

// ---- Chronopoulos-Gear CG, one kernel per iteration ------------------------------------
// With u = M r (Jacobi) and w = A u, one iteration i -> i+1 is
//   p_i = u_i + b_i p_{i-1},  s_i = w_i + b_i s_{i-1},  x += a_i p_i,  r_{i+1} = r_i - a_i s_i,
//   u_{i+1} = M r_{i+1},  w_{i+1} = A u_{i+1},
//   g = r_{i+1}.u_{i+1},  d = u_{i+1}.w_{i+1},  b_{i+1} = g / g_i,  a_{i+1} = g / (d - b_{i+1} g / a_i),
// so the three dot products (g, d, |r|^2) share one grid reduction.  In exact
// arithmetic this is the Jacobi-PCG of the reference's SPD system; u_{i+1} is
// staged in shared memory over the block's tile plus a one-cell halo.
constexpr int VTX = 32, VTY = 8, VSX = VTX + 2, VSY = VTY + 2;

// Shared-memory view of a compact (u, v) pair over one tile with a one-cell halo.
// Slots hold the values at wrapped global indices (periodic) or zero outside walls;
// requests use global indices, wrapped requests are mapped back into the halo.
struct TileUV {
    const double* su;
    const double* sv;
    int i0, j0, Nx, Ny;
    __device__ __forceinline__ int slot(int c, int r) const {
        int lc = c - i0 + 1, lr = r - j0 + 1;
        if (lc < 0) lc += Nx; else if (lc >= VSX) lc -= Nx;
        if (lr < 0) lr += Ny; else if (lr >= VSY) lr -= Ny;
        return lr * VSX + lc;
    }
    __device__ __forceinline__ double U(int c, int r) const { return su[slot(c, r)]; }
    __device__ __forceinline__ double V(int c, int r) const { return sv[slot(c, r)]; }
};

struct ViscIterArgs {
    const double *r_u, *r_v, *w_u, *w_v, *s_u, *s_v;  // iteration i (read)
    double *rn_u, *rn_v, *wn_u, *wn_v, *sn_u, *sn_v;  // iteration i+1 (written)
    double *x_u, *x_v, *p_u, *p_v;
    const double *dinv_u, *dinv_v;
};

// Global index of halo slot h (0 <= h < 2*VSX + 2*VTY) of a tile.
__device__ __forceinline__ void visc_halo_slot(int h, int& lx, int& ly) {
    if (h < VSX) { lx = h; ly = 0; }
    else if (h < 2 * VSX) { lx = h - VSX; ly = VSY - 1; }
    else { int t = h - 2 * VSX; lx = t < VTY ? 0 : VSX - 1; ly = 1 + (t % VTY); }
}

// Shared-memory view of a tile that lies with its halo inside the grid: every
// request is within one cell of the tile, so no request wraps.
struct TileIn {
    const double* su;
    const double* sv;
    int i0, j0;
    __device__ __forceinline__ int slot(int c, int r) const { return (r - j0 + 1) * VSX + (c - i0 + 1); }
    __device__ __forceinline__ double U(int c, int r) const { return su[slot(c, r)]; }
    __device__ __forceinline__ double V(int c, int r) const { return sv[slot(c, r)]; }
};

// A tile (i0, j0) whose points and halo all lie at least one cell inside the edges:
// no wrapped index, no Dirichlet row, no boundary term in its stencils.
__device__ __forceinline__ bool visc_tile_inside(int i0, int j0, int Nx, int Ny) {
    return i0 >= 1 && j0 >= 1 && i0 + VTX <= Nx - 1 && j0 + VTY <= Ny - 1;
}

// A u at an interior point of an inside tile (the interior form of visc_A_tile).
__device__ __forceinline__ void visc_A_inside(const Params& P, const double* phi, const TileIn& t, int i, int j,
                                              double& au, double& av) {
    if (P.md.viscosity == EFSI_VISC_CONSTANT)
        visc_A<true>(P, MuConst{P.md.viscosity_fluid}, t, i, j, au, av);
    else
        visc_A<true>(P, make_mu(P, phi), t, i, j, au, av);
}

// A u at (i,j) from a staged tile; interior points of a constant-viscosity model take
// the specialised form (same arithmetic, viscosity known to the compiler).
__device__ __forceinline__ void visc_A_tile(const Params& P, const double* phi, const TileUV& t, int i, int j,
                                            double& au, double& av) {
    if (P.md.viscosity == EFSI_VISC_CONSTANT && i >= 1 && i <= P.g.Nx - 2 && j >= 1 && j <= P.g.Ny - 2)
        visc_A<true>(P, MuConst{P.md.viscosity_fluid}, t, i, j, au, av);
    else
        visc_A_any(P, make_mu(P, phi), t, i, j, au, av);
}

// w = u - alpha*A u at the thread's own point from the staged tile (0 on Dirichlet rows).
__device__ __forceinline__ void visc_apply_tile(const Params& P, double alpha, const double* phi, const TileUV& t,
                                                int i, int j, double un, double vn, double& w1, double& w2) {
    double au, av;
    visc_A_tile(P, phi, t, i, j, au, av);
    w1 = u_fixed(P, i) ? 0.0 : un - alpha * au;
    w2 = v_fixed(P, j) ? 0.0 : vn - alpha * av;
}

// Staged value u = M r (INIT) or u_{i+1} = M (r_i - a (w_i + b s_{i-1})) at (gi, gj);
// zero outside walls, wrapped when periodic.
template <bool INIT>
__device__ __forceinline__ void visc_stage_value(const Params& P, const ViscIterArgs& v, bool first, double a,
                                                 double b, int gi, int gj, double& hu, double& hv) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const bool inx = gi >= 0 && gi < Nx, iny = gj >= 0 && gj < Ny;
    hu = 0.0;
    hv = 0.0;
    if (!((inx || P.g.px) && (iny || P.g.py))) return;
    const size_t k = cidx(inx ? gi : wrapm(gi, Nx), iny ? gj : wrapm(gj, Ny), Nx);
    if (INIT) {
        hu = __ldg(v.dinv_u + k) * __ldg(v.r_u + k);
        hv = __ldg(v.dinv_v + k) * __ldg(v.r_v + k);
    } else {
        const double d1 = __ldg(v.dinv_u + k), d2 = __ldg(v.dinv_v + k);
        const double r1 = __ldg(v.r_u + k), r2 = __ldg(v.r_v + k);
        const double w1 = __ldg(v.w_u + k), w2 = __ldg(v.w_v + k);
        const double s1 = first ? w1 : w1 + b * __ldg(v.s_u + k);
        const double s2 = first ? w2 : w2 + b * __ldg(v.s_v + k);
        hu = d1 * (r1 - a * s1);
        hv = d2 * (r2 - a * s2);
    }
}

// visc_stage_value<false> at a slot of an inside tile (no wrap, no wall).
__device__ __forceinline__ void visc_stage_inside(const ViscIterArgs& v, bool first, double a, double b, size_t k,
                                                  double& hu, double& hv) {
    const double d1 = __ldg(v.dinv_u + k), d2 = __ldg(v.dinv_v + k);
    const double r1 = __ldg(v.r_u + k), r2 = __ldg(v.r_v + k);
    const double w1 = __ldg(v.w_u + k), w2 = __ldg(v.w_v + k);
    const double s1 = first ? w1 : w1 + b * __ldg(v.s_u + k);
    const double s2 = first ? w2 : w2 + b * __ldg(v.s_v + k);
    hu = d1 * (r1 - a * s1);
    hv = d2 * (r2 - a * s2);
}

// w_0 = A M r_0 and d_0 = u_0.w_0 -> a_0 = g_0 / d_0.
__global__ void __launch_bounds__(VTX * VTY, 4) k_visc_w0(Params P, DtCoef ac, const double* __restrict__ phi,
                                                          ViscIterArgs v, CGScal* cg, RedSlot rs) {
    __shared__ double su[VSX * VSY], sv[VSX * VSY];
    __shared__ double sh[32];
    if (cg->done) return;
    const double alpha = ac.value();
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + ty * VTX;
    const int ntx = (P.g.Nx + VTX - 1) / VTX, nt = ntx * ((P.g.Ny + VTY - 1) / VTY);
    double acc[1] = {0.0};
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int i0 = (t % ntx) * VTX, j0 = (t / ntx) * VTY;
        const int i = i0 + tx, j = j0 + ty;
        double un, vn;
        visc_stage_value<true>(P, v, true, 0.0, 0.0, i, j, un, vn);
        su[(ty + 1) * VSX + tx + 1] = un;
        sv[(ty + 1) * VSX + tx + 1] = vn;
        if (tid < 2 * VSX + 2 * VTY) {
            int lx, ly;
            visc_halo_slot(tid, lx, ly);
            double hu, hv;
            visc_stage_value<true>(P, v, true, 0.0, 0.0, i0 + lx - 1, j0 + ly - 1, hu, hv);
            su[ly * VSX + lx] = hu;
            sv[ly * VSX + lx] = hv;
        }
        __syncthreads();
        if (i < P.g.Nx && j < P.g.Ny) {
            TileUV tl{su, sv, i0, j0, P.g.Nx, P.g.Ny};
            double w1, w2;
            visc_apply_tile(P, alpha, phi, tl, i, j, un, vn, w1, w2);
            size_t k = cidx(i, j, P.g.Nx);
            v.wn_u[k] = w1;
            v.wn_v[k] = w2;
            acc[0] += un * w1 + vn * w2;
        }
        __syncthreads();
    }
    double tot[1];
    if (grid_reduce<1>(acc, rs, tot, sh) && tid == 0) {
        cg->pAp = tot[0];
        cg->alpha = tot[0] != 0.0 ? cg->rz / tot[0] : 0.0;
    }
}

__global__ void __launch_bounds__(VTX * VTY, 4) k_visc_cg(Params P, DtCoef ac, const double* __restrict__ phi,
                                                          ViscIterArgs v, CGScal* cg, RedSlot rs, int* iters_out,
                                                          cudaGraphConditionalHandle cond) {
    __shared__ double su[VSX * VSY], sv[VSX * VSY];
    __shared__ double sh[3 * 32];
    if (cg->done) return;
    const double alpha = ac.value();
    const bool first = cg->iter == 0;
    const double a = cg->alpha, b = first ? 0.0 : cg->beta;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + ty * VTX;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const int ntx = (Nx + VTX - 1) / VTX, nt = ntx * ((Ny + VTY - 1) / VTY);
    double acc[3] = {0.0, 0.0, 0.0};  // g = r.u, d = u.w, |r|^2
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int i0 = (t % ntx) * VTX, j0 = (t / ntx) * VTY;
        const int i = i0 + tx, j = j0 + ty;
        const bool own = i < Nx && j < Ny;
        // every global load of the tile is issued before the first store
        double d1 = 0.0, d2 = 0.0, r1 = 0.0, r2 = 0.0, w1 = 0.0, w2 = 0.0, s1 = 0.0, s2 = 0.0;
        double p1 = 0.0, p2 = 0.0, x1 = 0.0, x2 = 0.0;
        size_t k = 0;
        if (own) {
            k = cidx(i, j, Nx);
            d1 = __ldg(v.dinv_u + k); d2 = __ldg(v.dinv_v + k);
            r1 = __ldg(v.r_u + k); r2 = __ldg(v.r_v + k);
            w1 = __ldg(v.w_u + k); w2 = __ldg(v.w_v + k);
            if (!first) {
                s1 = __ldg(v.s_u + k); s2 = __ldg(v.s_v + k);
                p1 = v.p_u[k]; p2 = v.p_v[k];
            }
            x1 = v.x_u[k]; x2 = v.x_v[k];
        }
        const bool inside = visc_tile_inside(i0, j0, Nx, Ny);
        const bool halo = tid < 2 * VSX + 2 * VTY;
        int hx = 0, hy = 0;
        double hu = 0.0, hv = 0.0;
        if (halo) {
            visc_halo_slot(tid, hx, hy);
            if (inside) visc_stage_inside(v, first, a, b, cidx(i0 + hx - 1, j0 + hy - 1, Nx), hu, hv);
            else visc_stage_value<false>(P, v, first, a, b, i0 + hx - 1, j0 + hy - 1, hu, hv);
        }
        double un = 0.0, vn = 0.0;
        if (own) {
            s1 = first ? w1 : w1 + b * s1;
            s2 = first ? w2 : w2 + b * s2;
            p1 = first ? d1 * r1 : d1 * r1 + b * p1;
            p2 = first ? d2 * r2 : d2 * r2 + b * p2;
            const double q1 = r1 - a * s1, q2 = r2 - a * s2;
            v.p_u[k] = p1;
            v.p_v[k] = p2;
            v.x_u[k] = x1 + a * p1;
            v.x_v[k] = x2 + a * p2;
            v.sn_u[k] = s1;
            v.sn_v[k] = s2;
            v.rn_u[k] = q1;
            v.rn_v[k] = q2;
            un = d1 * q1;
            vn = d2 * q2;
            acc[0] += q1 * un + q2 * vn;
            acc[2] += q1 * q1 + q2 * q2;
        } else {
            visc_stage_value<false>(P, v, first, a, b, i, j, un, vn);
        }
        su[(ty + 1) * VSX + tx + 1] = un;
        sv[(ty + 1) * VSX + tx + 1] = vn;
        if (halo) {
            su[hy * VSX + hx] = hu;
            sv[hy * VSX + hx] = hv;
        }
        __syncthreads();
        if (own) {
            double w1, w2;
            if (inside) {
                double au, av;
                visc_A_inside(P, phi, TileIn{su, sv, i0, j0}, i, j, au, av);
                w1 = un - alpha * au;
                w2 = vn - alpha * av;
            } else {
                visc_apply_tile(P, alpha, phi, TileUV{su, sv, i0, j0, Nx, Ny}, i, j, un, vn, w1, w2);
            }
            const size_t k = cidx(i, j, Nx);
            v.wn_u[k] = w1;
            v.wn_v[k] = w2;
            acc[1] += un * w1 + vn * w2;
        }
        __syncthreads();
    }
    double tot[3];
    if (grid_reduce<3>(acc, rs, tot, sh) && tid == 0) {
        const double g = tot[0], d = tot[1];
        cg->iter += 1;
        cg->rr = tot[2];
        const double bn = cg->rz != 0.0 ? g / cg->rz : 0.0;
        const double den = d - (cg->alpha != 0.0 ? bn * g / cg->alpha : 0.0);
        cg->beta = bn;
        cg->alpha = den != 0.0 ? g / den : 0.0;
        cg->rz = g;
        cg->pAp = d;
        if (tot[2] <= cg->tol2) { cg->conv = 1; cg->done = 1; }
        else if (cg->iter >= cg->maxiter || !isfinite(tot[2])) cg_unconverged(cg, tot[2]);
        if (iters_out) *iters_out = cg->iter;
        set_loop(cond, !cg->done);
    }
}

static ViscIterArgs visc_args(const ViscSolve& w, int parity) {
    const int c = parity & 1, n = c ^ 1;
    return ViscIterArgs{w.r_u[c], w.r_v[c], w.w_u[c], w.w_v[c], w.s_u[c], w.s_v[c],
                        w.r_u[n], w.r_v[n], w.w_u[n], w.w_v[n], w.s_u[n], w.s_v[n],
                        w.x_u, w.x_v, w.p_u, w.p_v, w.dinv_u, w.dinv_v};
}

void visc_init(const Params& P, DtCoef alpha, const SolveOpts& o, const double* Un, const double* Vn,
               const double* rhs_u, const double* rhs_v, const double* phi, const ViscSolve& w, CGScal* cg,
               const RedSlot& rs, const RedSlot& rs2, int* iters_out, cudaGraphConditionalHandle cond,
               cudaStream_t s) {
    dim3 g = grid2(P.g.Nx, P.g.Ny), b(BX, BY);
    k_visc_x0<<<g, b, 0, s>>>(P, Un, Vn, w.x_u, w.x_v);
    k_visc_init<<<persistent_grid(tiles2(P.g.Nx, P.g.Ny), P.nsm, 2), b, 0, s>>>(P, alpha, o, w.x_u, w.x_v, rhs_u, rhs_v, phi, w.r_u[0], w.r_v[0],
                                w.dinv_u, w.dinv_v, cg, rs, iters_out, cond);
    // w_0 goes to the parity-0 "read" slot: the first iteration reads (r, w)[0].
    ViscIterArgs v = visc_args(w, 1);
    v.r_u = w.r_u[0];
    v.r_v = w.r_v[0];
    v.wn_u = w.w_u[0];
    v.wn_v = w.w_v[0];
    const int nt = ((P.g.Nx + VTX - 1) / VTX) * ((P.g.Ny + VTY - 1) / VTY);
    k_visc_w0<<<persistent_grid(nt, P.nsm, 4), dim3(VTX, VTY), 0, s>>>(P, alpha, phi, v, cg, rs2);
}

void visc_iter(const Params& P, DtCoef alpha, const double* phi, const ViscSolve& w, int parity, CGScal* cg,
               const RedSlot& rs, int* iters_out, cudaGraphConditionalHandle cond, cudaStream_t s) {
    const int nt = ((P.g.Nx + VTX - 1) / VTX) * ((P.g.Ny + VTY - 1) / VTY);
    k_visc_cg<<<persistent_grid(nt, P.nsm, 4), dim3(VTX, VTY), 0, s>>>(P, alpha, phi, visc_args(w, parity), cg, rs,
                                                                        iters_out, cond);
}

// ---- precision form of the viscous solve -------------------------------------------------
enum { MX_ITER = 0, MX_REFINE = 1, MX_RESTART = 2 };
// The FP32 recurrence runs until its residual has dropped by this factor (squared:
// 1e-4 in norm) below the residual of its restart, or below the solve's target.
constexpr double kMxInnerDrop2 = 1e-8;

struct ViscMxArgs {
    const float *r_u, *r_v, *w_u, *w_v, *s_u, *s_v;  // iteration i (read)
    float *rn_u, *rn_v, *wn_u, *wn_v, *sn_u, *sn_v;  // iteration i+1 (written)
    float *p_u, *p_v, *dinv_u, *dinv_v, *rR_u, *rR_v;
    double *x_u, *x_v;
    const double *rhs_u, *rhs_v;
};

// FP64 value staged at tile slot (gi, gj): x (REFINE/START), M rR (RESTART) or
// M (r_i - a (w_i + b s_{i-1})) (ITER); zero outside walls, wrapped when periodic.
// `inside`: the slot is known to lie in the grid (a halo slot of an inside tile).
__device__ __forceinline__ void visc_mx_slot(const Params& P, const ViscMxArgs& v, int phase, bool first, double a,
                                             double b, int gi, int gj, double& hu, double& hv,
                                             bool inside = false) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    size_t k;
    if (inside) {
        k = cidx(gi, gj, Nx);
    } else {
        const bool inx = gi >= 0 && gi < Nx, iny = gj >= 0 && gj < Ny;
        hu = 0.0;
        hv = 0.0;
        if (!((inx || P.g.px) && (iny || P.g.py))) return;
        k = cidx(inx ? gi : wrapm(gi, Nx), iny ? gj : wrapm(gj, Ny), Nx);
    }
    if (phase == MX_REFINE) {
        hu = v.x_u[k];
        hv = v.x_v[k];
    } else if (phase == MX_RESTART) {
        hu = (double)v.dinv_u[k] * (double)v.rR_u[k];
        hv = (double)v.dinv_v[k] * (double)v.rR_v[k];
    } else {
        const double w1 = __ldg(v.w_u + k), w2 = __ldg(v.w_v + k);
        const double s1 = first ? w1 : w1 + b * (double)__ldg(v.s_u + k);
        const double s2 = first ? w2 : w2 + b * (double)__ldg(v.s_v + k);
        hu = (double)__ldg(v.dinv_u + k) * ((double)__ldg(v.r_u + k) - a * s1);
        hv = (double)__ldg(v.dinv_v + k) * ((double)__ldg(v.r_v + k) - a * s2);
    }
}

// One launch of the refined solve.  START: first launch of a solve (x = x0 given):
// Jacobi diagonal, FP64 residual, tolerance.  Otherwise the phase stored in `cg`:
//   ITER     one FP32 Chronopoulos-Gear iteration (x accumulates in FP64)
//   REFINE   r = rhs - (I - alpha A) x in FP64; stop, or restart from it
//   RESTART  w = A M r, r.Mr, Mr.w, from the refined residual
template <bool START>
__global__ void __launch_bounds__(VTX * VTY, 3) k_visc_mx(Params P, DtCoef ac, SolveOpts o,
                                                          const double* __restrict__ phi, ViscMxArgs v, CGScal* cg,
                                                          RedSlot rs, int* iters_out,
                                                          cudaGraphConditionalHandle cond) {
    __shared__ double su[VSX * VSY], sv[VSX * VSY];
    __shared__ double sh[3 * 32];
    if (!START && cg->done) return;
    const int phase = START ? MX_REFINE : cg->phase;
    const double alpha = ac.value();
    const bool first = START ? true : cg->inner == 0;
    const double a = START ? 0.0 : cg->alpha, b = first ? 0.0 : cg->beta;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + ty * VTX;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const int ntx = (Nx + VTX - 1) / VTX, nt = ntx * ((Ny + VTY - 1) / VTY);
    double acc[3] = {0.0, 0.0, 0.0};
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int i0 = (t % ntx) * VTX, j0 = (t / ntx) * VTY;
        const int i = i0 + tx, j = j0 + ty;
        const bool own = i < Nx && j < Ny;
        const size_t k = own ? cidx(i, j, Nx) : 0;
        double un = 0.0, vn = 0.0;
        if (own && phase == MX_ITER) {
            const double d1 = v.dinv_u[k], d2 = v.dinv_v[k];
            const double r1 = v.r_u[k], r2 = v.r_v[k];
            const double w1 = v.w_u[k], w2 = v.w_v[k];
            double s1 = 0.0, s2 = 0.0, p1 = 0.0, p2 = 0.0;
            if (!first) { s1 = v.s_u[k]; s2 = v.s_v[k]; p1 = v.p_u[k]; p2 = v.p_v[k]; }
            const double x1 = v.x_u[k], x2 = v.x_v[k];
            s1 = first ? w1 : w1 + b * s1;
            s2 = first ? w2 : w2 + b * s2;
            p1 = first ? d1 * r1 : d1 * r1 + b * p1;
            p2 = first ? d2 * r2 : d2 * r2 + b * p2;
            const double q1 = r1 - a * s1, q2 = r2 - a * s2;
            v.p_u[k] = (float)p1;
            v.p_v[k] = (float)p2;
            v.x_u[k] = x1 + a * p1;
            v.x_v[k] = x2 + a * p2;
            v.sn_u[k] = (float)s1;
            v.sn_v[k] = (float)s2;
            v.rn_u[k] = (float)q1;
            v.rn_v[k] = (float)q2;
            un = d1 * q1;
            vn = d2 * q2;
            acc[0] += q1 * un + q2 * vn;
            acc[2] += q1 * q1 + q2 * q2;
        } else {
            visc_mx_slot(P, v, phase, first, a, b, i, j, un, vn);
        }
        su[(ty + 1) * VSX + tx + 1] = un;
        sv[(ty + 1) * VSX + tx + 1] = vn;
        const bool inside = !START && visc_tile_inside(i0, j0, Nx, Ny);
        if (tid < 2 * VSX + 2 * VTY) {
            int lx, ly;
            visc_halo_slot(tid, lx, ly);
            double hu, hv;
            visc_mx_slot(P, v, phase, first, a, b, i0 + lx - 1, j0 + ly - 1, hu, hv, inside);
            su[ly * VSX + lx] = hu;
            sv[ly * VSX + lx] = hv;
        }
        __syncthreads();
        if (own && inside) {  // no Dirichlet row, no wrap (START never takes this path)
            double au, av;
            visc_A_inside(P, phi, TileIn{su, sv, i0, j0}, i, j, au, av);
            if (phase == MX_REFINE) {
                const double r1 = v.rhs_u[k] - (un - alpha * au);
                const double r2 = v.rhs_v[k] - (vn - alpha * av);
                v.rR_u[k] = (float)r1;
                v.rR_v[k] = (float)r2;
                acc[0] += r1 * r1 + r2 * r2;
            } else {
                const double w1 = un - alpha * au, w2 = vn - alpha * av;
                v.wn_u[k] = (float)w1;
                v.wn_v[k] = (float)w2;
                acc[1] += un * w1 + vn * w2;
                if (phase == MX_RESTART) {
                    const double r1 = v.rR_u[k], r2 = v.rR_v[k];
                    v.rn_u[k] = (float)r1;
                    v.rn_v[k] = (float)r2;
                    acc[0] += r1 * un + r2 * vn;
                }
            }
        } else if (own) {
            TileUV tl{su, sv, i0, j0, Nx, Ny};
            MuField mu = make_mu(P, phi);
            double au, av;
            visc_A_tile(P, phi, tl, i, j, au, av);
            if (phase == MX_REFINE) {
                if (START) {
                    double du, dv;
                    visc_diag(P, mu, i, j, du, dv);
                    v.dinv_u[k] = u_fixed(P, i) ? 0.0f : (float)(1.0 / (1.0 - alpha * du));
                    v.dinv_v[k] = v_fixed(P, j) ? 0.0f : (float)(1.0 / (1.0 - alpha * dv));
                }
                const double r1 = u_fixed(P, i) ? 0.0 : v.rhs_u[k] - (un - alpha * au);
                const double r2 = v_fixed(P, j) ? 0.0 : v.rhs_v[k] - (vn - alpha * av);
                v.rR_u[k] = (float)r1;
                v.rR_v[k] = (float)r2;
                acc[0] += r1 * r1 + r2 * r2;
                if (START) {  // |b|^2 of the row-eliminated system (acc[1] is free at START)
                    const double b1 = u_fixed(P, i) ? un : v.rhs_u[k], b2 = v_fixed(P, j) ? vn : v.rhs_v[k];
                    acc[1] += b1 * b1 + b2 * b2;
                }
            } else {
                const double w1 = u_fixed(P, i) ? 0.0 : un - alpha * au;
                const double w2 = v_fixed(P, j) ? 0.0 : vn - alpha * av;
                v.wn_u[k] = (float)w1;
                v.wn_v[k] = (float)w2;
                acc[1] += un * w1 + vn * w2;
                if (phase == MX_RESTART) {
                    const double r1 = v.rR_u[k], r2 = v.rR_v[k];
                    v.rn_u[k] = (float)r1;
                    v.rn_v[k] = (float)r2;
                    acc[0] += r1 * un + r2 * vn;
                }
            }
        }
        __syncthreads();
    }
    double tot[3];
    if (grid_reduce<3>(acc, rs, tot, sh) && tid == 0) {
        if (START) {
            cg->rr0 = tot[0];
            cg->rr = tot[0];
            cg_begin(cg, o, tot[0], tot[1]);
            cg->inner = 0;
            cg->rr_restart = tot[0];
            cg->phase = MX_RESTART;
            if (iters_out) *iters_out = 0;
            set_loop(cond, !cg->done);
            return;
        }
        cg->iter += 1;
        if (phase == MX_ITER) {
            const double g = tot[0], d = tot[1];
            const double bn = cg->rz != 0.0 ? g / cg->rz : 0.0;
            const double den = d - (cg->alpha != 0.0 ? bn * g / cg->alpha : 0.0);
            cg->beta = bn;
            cg->alpha = den != 0.0 ? g / den : 0.0;
            cg->rz = g;
            cg->pAp = d;
            cg->inner += 1;
            cg->rr = tot[2];
            if (!isfinite(tot[2])) cg_unconverged(cg, tot[2]);
            else if (tot[2] <= cg->tol2 || tot[2] <= kMxInnerDrop2 * cg->rr_restart) cg->phase = MX_REFINE;
        } else if (phase == MX_REFINE) {
            cg->rr = tot[0];
            if (tot[0] <= cg->tol2) { cg->conv = 1; cg->done = 1; }
            else if (!isfinite(tot[0])) cg_unconverged(cg, tot[0]);
            else { cg->phase = MX_RESTART; cg->rr_restart = tot[0]; }
        } else {  // restart: r.Mr and Mr.w of the refined residual
            cg->rz = tot[0];
            cg->pAp = tot[1];
            cg->alpha = tot[1] != 0.0 ? tot[0] / tot[1] : 0.0;
            cg->beta = 0.0;
            cg->inner = 0;
            cg->phase = MX_ITER;
        }
        if (!cg->done && cg->iter >= cg->maxiter) cg_unconverged(cg, cg->rr);
        if (iters_out) *iters_out = cg->iter;
        set_loop(cond, !cg->done);
    }
}

static ViscMxArgs visc_mx_args(const ViscSolve& w, const ViscMixed& m, const double* rhs_u, const double* rhs_v,
                               int parity) {
    const int c = parity & 1, n = c ^ 1;
    return ViscMxArgs{m.r_u[c], m.r_v[c], m.w_u[c], m.w_v[c], m.s_u[c], m.s_v[c],
                      m.r_u[n], m.r_v[n], m.w_u[n], m.w_v[n], m.s_u[n], m.s_v[n],
                      m.p_u, m.p_v, m.dinv_u, m.dinv_v, m.rR_u, m.rR_v, w.x_u, w.x_v, rhs_u, rhs_v};
}

void visc_mx_init(const Params& P, DtCoef alpha, const SolveOpts& o, const double* Un, const double* Vn,
                  const double* rhs_u, const double* rhs_v, const double* phi, const ViscSolve& w,
                  const ViscMixed& m, CGScal* cg, const RedSlot& rs, int* iters_out,
                  cudaGraphConditionalHandle cond, cudaStream_t s) {
    k_visc_x0<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, Un, Vn, w.x_u, w.x_v);
    const int nt = ((P.g.Nx + VTX - 1) / VTX) * ((P.g.Ny + VTY - 1) / VTY);
    k_visc_mx<true><<<persistent_grid(nt, P.nsm, 3), dim3(VTX, VTY), 0, s>>>(
        P, alpha, o, phi, visc_mx_args(w, m, rhs_u, rhs_v, 0), cg, rs, iters_out, cond);
}

void visc_mx_iter(const Params& P, DtCoef alpha, const double* phi, const double* rhs_u, const double* rhs_v,
                  const ViscSolve& w, const ViscMixed& m, int parity, CGScal* cg, const RedSlot& rs,
                  int* iters_out, cudaGraphConditionalHandle cond, cudaStream_t s) {
    const int nt = ((P.g.Nx + VTX - 1) / VTX) * ((P.g.Ny + VTY - 1) / VTY);
    k_visc_mx<false><<<persistent_grid(nt, P.nsm, 3), dim3(VTX, VTY), 0, s>>>(
        P, alpha, SolveOpts{}, phi, visc_mx_args(w, m, rhs_u, rhs_v, parity), cg, rs, iters_out, cond);
}

// ---- precision form with a constant viscosity: FP32 Chebyshev inner solver -----------
// Phases of the body launches: ITER (kChebSteps FP32 Chebyshev steps on the correction
// equation; the last launch of an inner cycle adds e to x in FP64), REFINE (r = rhs -
// (I - alpha A) x in FP64; stop or start the next inner cycle from it).  Chebyshev recurrence for M e = r with
// spec(M) in [1, 1 + 2 delta] (Saad, Iterative Methods for Sparse Linear Systems,
// Algorithm 12.1): theta = 1 + delta, sigma = theta / delta, rho_0 = 1 / sigma,
// d_0 = r_0 / theta; per step e += d, r -= M d, rho' = 1 / (2 sigma - rho),
// d = rho' rho d + (2 rho' / delta) r.
enum { CH_ITER = 0, CH_REFINE = 2 };
constexpr int CK = kChebSteps, CTX = 32, CTY = 32, CWX = CTX + 2 * CK, CWY = CTY + 2 * CK;
// Block of the body launches: CWX x CBY threads; in ITER thread (lx, ly0) owns the CNR
// consecutive cells (lx, CNR ly0 + m) of one region column, so that the north and south
// neighbours of all but its end cells are its own registers.
constexpr int CBY = 8, CNR = CWY / CBY, CNT = CWX * CBY, kChebBlocksPerSM = 2;
static_assert(CWY % CBY == 0, "region rows must split evenly over the block rows");
// Residual drop one FP32 inner cycle aims for (FP32 resolves about 1e-7; 1e-4 measured
// 1.3% faster per step than 1e-5 and 2.4% faster than 1e-6 at 1024^2).
constexpr double kChebDrop = 1e-4;

struct ChebArgs {
    const float *r_u, *r_v, *d_u, *d_v, *e_u, *e_v;  // set read by this launch
    float *rn_u, *rn_v, *dn_u, *dn_v, *en_u, *en_v;  // set written by this launch
    double *x_u, *x_v;
    const double *rhs_u, *rhs_v;
    const float* ring_w;  // A at the outer-ring cells (visc_ring_weights)
};

// Index of ring cell (i, j) in the weight table: bottom row, top row, left column,
// right column (a corner belongs to its row).
__device__ __forceinline__ int ring_index(const GridD& g, int i, int j) {
    if (!g.py && j == 0) return i;
    if (!g.py && j == g.Ny - 1) return g.Nx + i;
    if (!g.px && i == 0) return 2 * g.Nx + j;
    return 2 * g.Nx + g.Ny + j;
}
// Unit vector: 1 at component q of cell (ti, tj), 0 elsewhere.
struct ProbeTile {
    int q, ti, tj;
    __device__ __forceinline__ double U(int c, int r) const { return (q == 0 && c == ti && r == tj) ? 1.0 : 0.0; }
    __device__ __forceinline__ double V(int c, int r) const { return (q == 1 && c == ti && r == tj) ? 1.0 : 0.0; }
};
// One thread per (ring cell, column component, offset).
__global__ void k_ring_weights(Params P, float* ring_w) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const int n = (int)visc_ring_cells(Nx, Ny) * 18;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int c = t / 18, rem = t % 18, q = rem / 9, dy = (rem % 9) / 3 - 1, dx = rem % 3 - 1;
    int i, j;
    if (c < Nx) { i = c; j = 0; }
    else if (c < 2 * Nx) { i = c - Nx; j = Ny - 1; }
    else if (c < 2 * Nx + Ny) { i = 0; j = c - 2 * Nx; }
    else { i = Nx - 1; j = c - 2 * Nx - Ny; }
    const int ti = wrapm(i + dx, Nx), tj = wrapm(j + dy, Ny);
    double a1, a2;
    visc_A<false>(P, MuConst{P.md.viscosity_fluid}, ProbeTile{q, ti, tj}, i, j, a1, a2);
    float* w = ring_w + (size_t)kRingWeights * c;
    w[9 * q + 3 * (dy + 1) + dx + 1] = (float)a1;
    w[18 + 9 * q + 3 * (dy + 1) + dx + 1] = (float)a2;
}

// theta and delta of the free block of I - alpha A for a constant viscosity mu:
// spec in [1, 1 + alpha g] with g = mu (max(8/hx^2 + 4/hy^2, 4/hx^2 + 8/hy^2) +
// 4/(hx hy)), the Gershgorin bound of the rows of -A (wall rows sum to less).
__device__ __forceinline__ void cheb_bounds(const Params& P, double alpha, double& theta, double& delta) {
    const double ix2 = P.g.ihx * P.g.ihx, iy2 = P.g.ihy * P.g.ihy;
    const double g = P.md.viscosity_fluid * (fmax(8.0 * ix2 + 4.0 * iy2, 4.0 * ix2 + 8.0 * iy2) + 4.0 * P.g.ihx * P.g.ihy);
    delta = 0.5 * alpha * g;
    theta = 1.0 + delta;
}
// Chebyshev steps of one inner cycle for the residual drop `drop` (|r_n| <= |r_0| /
// T_n(sigma)), rounded up to whole launches.
__device__ __forceinline__ int cheb_steps(double theta, double delta, double drop) {
    if (!(delta > 1e-300)) return CK;
    const double n = acosh(1.0 / drop) / acosh(theta / delta);
    const int k = max(1, (int)ceil(n));
    return ((k + CK - 1) / CK) * CK;
}

// Shared-memory view (doubles converted from the FP32 region) for the general stencil
// at cells next to an edge; requests use global indices, wrapped ones map back.
struct ChebTile {
    const float* su;
    const float* sv;
    int i0, j0, Nx, Ny;
    __device__ __forceinline__ int slot(int c, int r) const {
        int lc = c - i0 + CK, lr = r - j0 + CK;
        if (lc < 0) lc += Nx; else if (lc >= CWX) lc -= Nx;
        if (lr < 0) lr += Ny; else if (lr >= CWY) lr -= Ny;
        return lr * CWX + lc;
    }
    __device__ __forceinline__ double U(int c, int r) const { return su[slot(c, r)]; }
    __device__ __forceinline__ double V(int c, int r) const { return sv[slot(c, r)]; }
};

// REFINE (and the START of a solve): stage x (the last ITER of the cycle has added the
// correction) over a CTX x CTY tile and its one-cell ring, r = rhs - (x - alpha A x) in
// FP64 at the tile, |r|^2 and |b|^2; the next inner cycle starts from r: r_set = r,
// d_set = r / theta, e_set = 0.  Every thread of the block takes up to kRefCells cells of
// the tile, whose right-hand sides it loads together with its share of the ring, so a
// tile is one round of independent loads and two barriers (the launch keeps the ITER
// launches' block shape and occupancy).
constexpr int RSX = CTX + 2, RSY = CTY + 2, kRefCells = (CTX * CTY + CNT - 1) / CNT;
struct RefTileUV {  // the refinement tile: global requests, wrapped ones mapped back
    const double* su;
    const double* sv;
    int i0, j0, Nx, Ny;
    __device__ __forceinline__ int slot(int c, int r) const {
        int lc = c - i0 + 1, lr = r - j0 + 1;
        if (lc < 0) lc += Nx; else if (lc >= RSX) lc -= Nx;
        if (lr < 0) lr += Ny; else if (lr >= RSY) lr -= Ny;
        return lr * RSX + lc;
    }
    __device__ __forceinline__ double U(int c, int r) const { return su[slot(c, r)]; }
    __device__ __forceinline__ double V(int c, int r) const { return sv[slot(c, r)]; }
};
template <bool START>
__device__ void cheb_refine(const Params& P, double alpha, double theta, const ChebArgs& v, double* sm, double (&acc)[2]) {
    double* su = sm;
    double* sv = sm + RSX * RSY;
    const int tid = threadIdx.x + threadIdx.y * blockDim.x, nthr = blockDim.x * blockDim.y;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const double mu = P.md.viscosity_fluid, ix2 = P.g.ihx * P.g.ihx, iy2 = P.g.ihy * P.g.ihy;
    const double cxx = 2.0 * mu * ix2, cyy = mu * iy2, cxx2 = mu * ix2, cyy2 = 2.0 * mu * iy2;
    const double cxy = mu * P.g.ihx * P.g.ihy;
    const int ntx = (Nx + CTX - 1) / CTX, nt = ntx * ((Ny + CTY - 1) / CTY);
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int i0 = (t % ntx) * CTX, j0 = (t / ntx) * CTY;
        double bu[kRefCells], bv[kRefCells];
#pragma unroll
        for (int m = 0; m < kRefCells; ++m) {
            const int q = tid + m * nthr, i = i0 + q % CTX, j = j0 + q / CTX;
            bu[m] = bv[m] = 0.0;
            if (q < CTX * CTY && i < Nx && j < Ny) {
                const size_t k = cidx(i, j, Nx);
                bu[m] = v.rhs_u[k];
                bv[m] = v.rhs_v[k];
            }
        }
        for (int q = tid; q < RSX * RSY; q += nthr) {
            const int gi = i0 + q % RSX - 1, gj = j0 + q / RSX - 1;
            const bool inx = gi >= 0 && gi < Nx, iny = gj >= 0 && gj < Ny;
            double hu = 0.0, hv = 0.0;
            if ((inx || P.g.px) && (iny || P.g.py)) {
                const size_t k = cidx(inx ? gi : wrapm(gi, Nx), iny ? gj : wrapm(gj, Ny), Nx);
                hu = v.x_u[k];
                hv = v.x_v[k];
            }
            su[q] = hu;
            sv[q] = hv;
        }
        __syncthreads();
#pragma unroll
        for (int m = 0; m < kRefCells; ++m) {
            const int q = tid + m * nthr, tx = q % CTX, ty = q / CTX, i = i0 + tx, j = j0 + ty;
            if (q >= CTX * CTY || i >= Nx || j >= Ny) continue;
            const size_t k = cidx(i, j, Nx);
            const int sl = (ty + 1) * RSX + tx + 1;
            const double un = su[sl], vn = sv[sl];
            double au, av;
            if ((P.g.px || (i >= 1 && i <= Nx - 2)) && (P.g.py || (j >= 1 && j <= Ny - 2))) {
                // free interior, constant viscosity: the compact stencil read from the tile
                au = cxx * (su[sl + 1] - 2.0 * un + su[sl - 1]) + cyy * (su[sl + RSX] - 2.0 * un + su[sl - RSX]) +
                     cxy * (sv[sl + RSX] - sv[sl + RSX - 1] - vn + sv[sl - 1]);
                av = cxx2 * (sv[sl + 1] - 2.0 * vn + sv[sl - 1]) + cyy2 * (sv[sl + RSX] - 2.0 * vn + sv[sl - RSX]) +
                     cxy * (su[sl + 1] - su[sl + 1 - RSX] - un + su[sl - RSX]);
            } else {
                visc_A<false>(P, MuConst{mu}, RefTileUV{su, sv, i0, j0, Nx, Ny}, i, j, au, av);
            }
            const bool uf = u_fixed(P, i), vf = v_fixed(P, j);
            const double r1 = uf ? 0.0 : bu[m] - (un - alpha * au);
            const double r2 = vf ? 0.0 : bv[m] - (vn - alpha * av);
            if (START) {  // |b|^2 of the row-eliminated system: Dirichlet rows hold their data
                const double b1 = uf ? un : bu[m], b2 = vf ? vn : bv[m];
                acc[1] += b1 * b1 + b2 * b2;
            }
            acc[0] += r1 * r1 + r2 * r2;
            v.rn_u[k] = (float)r1;
            v.rn_v[k] = (float)r2;
            v.dn_u[k] = (float)(r1 / theta);
            v.dn_v[k] = (float)(r2 / theta);
            v.en_u[k] = 0.0f;
            v.en_v[k] = 0.0f;
        }
        __syncthreads();
    }
}

// ITER: CK Chebyshev steps of e, r, d on a CTX x CTY tile with a CK-cell halo (FP32
// storage and arithmetic).  Each thread keeps e, r and d of its CNR cells in registers
// (e and r are pointwise); d, read at neighbours, is double-buffered in shared memory,
// so a step is one barrier.  Free interior cells form M d = d - alpha A d directly with
// alpha folded into the stencil weights (six shared loads per cell).  Cells next to a
// wall or on a Dirichlet row are "special": they are listed per tile, keep e and r in
// shared memory and are shared out over the whole block each step, so a wall tile costs
// about as much as an interior one.  Every step updates the whole region but its outer
// ring; a value next to the ring goes stale one cell per step, so after CK steps the
// tile itself is exact.
__device__ void cheb_iter(const Params& P, double alpha, double theta, double delta, double rho0, bool last,
                          const ChebArgs& v, float* sm, double (&acc)[2]) {
    float* const dbu[2] = {sm, sm + 2 * CWX * CWY};
    float* const dbv[2] = {sm + CWX * CWY, sm + 3 * CWX * CWY};
    float* const seu = sm + 4 * CWX * CWY;  // e, r of special cells
    float* const sev = seu + CWX * CWY;
    float* const sru = sev + CWX * CWY;
    float* const srv = sru + CWX * CWY;
    short* const slist = reinterpret_cast<short*>(srv + CWX * CWY);  // special slots of the tile
    float* const scoef = reinterpret_cast<float*>(slist + CWX * CWY);  // a_s, b_s per step
    __shared__ int nspec;
    const int tid = threadIdx.x + threadIdx.y * blockDim.x, nthr = blockDim.x * blockDim.y;
    const int lx = threadIdx.x, lyb = CNR * threadIdx.y;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const bool px = P.g.px, py = P.g.py;
    const double mu = P.md.viscosity_fluid;
    const float fa = (float)alpha;
    // M d on the free interior: kcu uC - (kx (uE + uW) + ky (uN + uS) + kxy (vN - vNW + vW - vC))
    // and its mirror for v (2 mu u_xx + mu u_yy + mu v_xy; mu v_xx + 2 mu v_yy + mu u_xy)
    const double ix2 = P.g.ihx * P.g.ihx, iy2 = P.g.ihy * P.g.ihy;
    const float kx = (float)(alpha * mu * 2.0 * ix2), ky = (float)(alpha * mu * iy2);
    const float kx2 = (float)(alpha * mu * ix2), ky2 = (float)(alpha * mu * 2.0 * iy2);
    const float kxy = (float)(alpha * mu * P.g.ihx * P.g.ihy);
    const float kcu = (float)(1.0 + 2.0 * alpha * mu * (2.0 * ix2 + iy2));
    const float kcv = (float)(1.0 + 2.0 * alpha * mu * (ix2 + 2.0 * iy2));
    if (tid == 0) {  // per-step coefficients a_s = rho' rho, b_s = 2 rho' / delta
        const double s1 = theta / delta;
        double rho = rho0;
        for (int q = 0; q < CK; ++q) {
            const double rn = 1.0 / (2.0 * s1 - rho);
            scoef[2 * q] = (float)(rn * rho);
            scoef[2 * q + 1] = (float)(2.0 * rn / delta);
            rho = rn;
        }
    }
    const bool xring = lx == 0 || lx == CWX - 1;
    const int ntx = (Nx + CTX - 1) / CTX, nt = ntx * ((Ny + CTY - 1) / CTY);
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int i0 = (t % ntx) * CTX, j0 = (t / ntx) * CTY;
        if (tid == 0) nspec = 0;
        __syncthreads();  // also orders this tile's loads after the last tile's write-out
        const int gi = i0 + lx - CK;
        const bool inx = gi >= 0 && gi < Nx;
        const int wi = inx ? gi : (px ? wrapm(gi, Nx) : 0);
        float eu[CNR], ev[CNR], ru[CNR], rv[CNR], du[CNR], dv[CNR];
        unsigned skip = 0;  // bit m: cell m is outside the grid, on the ring or special
        // load the region: slots outside the grid (walls) hold 0 and are never updated
#pragma unroll
        for (int m = 0; m < CNR; ++m) {
            const int ly = lyb + m, sl = ly * CWX + lx, gj = j0 + ly - CK;
            const bool iny = gj >= 0 && gj < Ny;
            const bool valid = (inx || px) && (iny || py);
            eu[m] = ev[m] = ru[m] = rv[m] = du[m] = dv[m] = 0.f;
            if (valid) {
                const int wj = iny ? gj : wrapm(gj, Ny);
                const size_t k = cidx(wi, wj, Nx);
                eu[m] = v.e_u[k]; ev[m] = v.e_v[k]; ru[m] = v.r_u[k]; rv[m] = v.r_v[k]; du[m] = v.d_u[k]; dv[m] = v.d_v[k];
                const bool ring = xring || ly == 0 || ly == CWY - 1;
                const bool free_cell = (px || (wi >= 1 && wi <= Nx - 2)) && (py || (wj >= 1 && wj <= Ny - 2)) &&
                                       !u_fixed(P, wi) && !v_fixed(P, wj);
                if (ring) {
                    skip |= 1u << m;
                } else if (!free_cell) {
                    skip |= 1u << m;
                    slist[atomicAdd(&nspec, 1)] = (short)sl;
                    seu[sl] = eu[m]; sev[sl] = ev[m]; sru[sl] = ru[m]; srv[sl] = rv[m];
                }
            } else {
                skip |= 1u << m;
            }
            dbu[0][sl] = du[m]; dbv[0][sl] = dv[m];
            dbu[1][sl] = du[m]; dbv[1][sl] = dv[m];
        }
        __syncthreads();
        const int ns = nspec;
#pragma unroll 1
        for (int st = 0; st < CK; ++st) {
            const float* cu = dbu[st & 1];
            const float* cv = dbv[st & 1];
            float* nu = dbu[(st & 1) ^ 1];
            float* nv = dbv[(st & 1) ^ 1];
            const float a_s = scoef[2 * st], b_s = scoef[2 * st + 1];
            // e += d; r -= M d; d = a_s d + b_s r
            float pu = 0.f, pv = 0.f;  // d of cell m - 1 before this step
#pragma unroll
            for (int m = 0; m < CNR; ++m) {
                const int sl = (lyb + m) * CWX + lx;
                if (skip & (1u << m)) {  // special cells move in shared memory; refresh d
                    du[m] = cu[sl];
                    dv[m] = cv[sl];
                }
            }
#pragma unroll
            for (int m = 0; m < CNR; ++m) {
                const int sl = (lyb + m) * CWX + lx;
                const float uC = du[m], vC = dv[m];
                if (!(skip & (1u << m))) {
                    const float uS = m > 0 ? pu : cu[sl - CWX], vS = m > 0 ? pv : cv[sl - CWX];
                    const float uN = m < CNR - 1 ? du[m + 1] : cu[sl + CWX];
                    const float vN = m < CNR - 1 ? dv[m + 1] : cv[sl + CWX];
                    const float uE = cu[sl + 1], uW = cu[sl - 1], vE = cv[sl + 1], vW = cv[sl - 1];
                    const float vNW = cv[sl + CWX - 1], uSE = cu[sl + 1 - CWX];
                    const float mdu = kcu * uC - (kx * (uE + uW) + ky * (uN + uS) + kxy * ((vN - vNW) + (vW - vC)));
                    const float mdv = kcv * vC - (kx2 * (vE + vW) + ky2 * (vN + vS) + kxy * ((uE - uSE) + (uS - uC)));
                    eu[m] += uC;
                    ru[m] -= mdu;
                    du[m] = a_s * uC + b_s * ru[m];
                    nu[sl] = du[m];
                    ev[m] += vC;
                    rv[m] -= mdv;
                    dv[m] = a_s * vC + b_s * rv[m];
                    nv[sl] = dv[m];
                }
                pu = uC;
                pv = vC;
            }
            // special cells, shared out over the block: the general stencil
            for (int q = tid; q < ns; q += nthr) {
                const int sl = slist[q], sx = sl % CWX, sy = sl / CWX;
                const int ci = i0 + sx - CK, cj = j0 + sy - CK;
                const int qi = (ci >= 0 && ci < Nx) ? ci : wrapm(ci, Nx), qj = (cj >= 0 && cj < Ny) ? cj : wrapm(cj, Ny);
                const bool uf = u_fixed(P, qi), vf = v_fixed(P, qj);
                const float dcu = cu[sl], dcv = cv[sl];
                const float* w = v.ring_w + (size_t)kRingWeights * ring_index(P.g, qi, qj);
                float a1 = 0.f, a2 = 0.f;
#pragma unroll
                for (int oy = 0; oy < 3; ++oy)
#pragma unroll
                    for (int ox = 0; ox < 3; ++ox) {
                        const int o = sl + (oy - 1) * CWX + ox - 1, k = 3 * oy + ox;
                        const float nu_ = cu[o], nv_ = cv[o];
                        a1 += __ldg(w + k) * nu_ + __ldg(w + 9 + k) * nv_;
                        a2 += __ldg(w + 18 + k) * nu_ + __ldg(w + 27 + k) * nv_;
                    }
                if (!uf) {
                    const float r = sru[sl] - (dcu - fa * a1);
                    seu[sl] += dcu;
                    sru[sl] = r;
                    nu[sl] = a_s * dcu + b_s * r;
                }
                if (!vf) {
                    const float r = srv[sl] - (dcv - fa * a2);
                    sev[sl] += dcv;
                    srv[sl] = r;
                    nv[sl] = a_s * dcv + b_s * r;
                }
            }
            __syncthreads();
        }
        if (last) {
            // end of the inner cycle: x += e (REFINE then restarts r, d, e).  e of the
            // tile goes to the d buffer the last step read (free after its barrier), then
            // the block adds it to x cell by cell, every thread's x loads issued together
            // before its stores.
            float* const fu = dbu[(CK & 1) ^ 1];
            float* const fv = dbv[(CK & 1) ^ 1];
#pragma unroll
            for (int m = 0; m < CNR; ++m) {
                const int ly = lyb + m, sl = ly * CWX + lx, gj = j0 + ly - CK;
                if (lx < CK || lx >= CK + CTX || ly < CK || ly >= CK + CTY || gi >= Nx || gj >= Ny) continue;
                float e1 = eu[m], e2 = ev[m], r1 = ru[m], r2 = rv[m];
                if (skip & (1u << m)) { e1 = seu[sl]; e2 = sev[sl]; r1 = sru[sl]; r2 = srv[sl]; }
                fu[sl] = e1;
                fv[sl] = e2;
                acc[0] += (double)r1 * r1 + (double)r2 * r2;
            }
            __syncthreads();
            double xu[kRefCells], xv[kRefCells];
#pragma unroll
            for (int m = 0; m < kRefCells; ++m) {
                const int q = tid + m * nthr, i = i0 + q % CTX, j = j0 + q / CTX;
                xu[m] = xv[m] = 0.0;
                if (q < CTX * CTY && i < Nx && j < Ny) {
                    const size_t k = cidx(i, j, Nx);
                    xu[m] = v.x_u[k];
                    xv[m] = v.x_v[k];
                }
            }
#pragma unroll
            for (int m = 0; m < kRefCells; ++m) {
                const int q = tid + m * nthr, tx = q % CTX, ty = q / CTX, i = i0 + tx, j = j0 + ty;
                if (q >= CTX * CTY || i >= Nx || j >= Ny) continue;
                const int sl = (ty + CK) * CWX + tx + CK;
                const size_t k = cidx(i, j, Nx);
                v.x_u[k] = xu[m] + (double)fu[sl];
                v.x_v[k] = xv[m] + (double)fv[sl];
            }
            continue;  // the next tile starts with a barrier
        }
        // write the tile (special cells from shared memory; the latest d is in buffer CK & 1)
#pragma unroll
        for (int m = 0; m < CNR; ++m) {
            const int ly = lyb + m, sl = ly * CWX + lx, gj = j0 + ly - CK;
            if (lx < CK || lx >= CK + CTX || ly < CK || ly >= CK + CTY || gi >= Nx || gj >= Ny) continue;
            float e1 = eu[m], e2 = ev[m], r1 = ru[m], r2 = rv[m], d1 = du[m], d2 = dv[m];
            if (skip & (1u << m)) {
                e1 = seu[sl]; e2 = sev[sl]; r1 = sru[sl]; r2 = srv[sl];
                d1 = dbu[CK & 1][sl]; d2 = dbv[CK & 1][sl];
            }
            const size_t k = cidx(gi, gj, Nx);
            v.en_u[k] = e1; v.en_v[k] = e2;
            v.rn_u[k] = r1; v.rn_v[k] = r2;
            v.dn_u[k] = d1; v.dn_v[k] = d2;
            acc[0] += (double)r1 * r1 + (double)r2 * r2;
        }
    }
}

// The FP32 region of cheb_iter or the FP64 tile of cheb_refine.
// (dynamic shared memory: d double-buffered, e and r of special cells, the special-slot
// list and the step coefficients)
constexpr int kChebSmemBytes = 8 * CWX * CWY * 4 + CWX * CWY * 2 + 2 * CK * 4;
static_assert(kChebSmemBytes >= 2 * RSX * RSY * 8, "the refinement tile shares the buffer");
static_assert(CWX * CWY <= 32767, "special slots are stored as short");

template <bool START>
__global__ void __launch_bounds__(CNT, kChebBlocksPerSM) k_vcheb(Params P, DtCoef ac, SolveOpts o, ChebArgs v, CGScal* cg,
                                                     RedSlot rs, int* iters_out, cudaGraphConditionalHandle cond) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double sh[64];
    if (!START && cg->done) return;
    const int phase = START ? CH_REFINE : cg->phase;
    const double alpha = ac.value();
    double theta, delta;
    cheb_bounds(P, alpha, theta, delta);
    double acc[2] = {0.0, 0.0};
    if (phase == CH_ITER) {
        cheb_iter(P, alpha, theta, delta, cg->rho, cg->inner + CK >= cg->nin, v, reinterpret_cast<float*>(smem), acc);
    } else {
        cheb_refine<START>(P, alpha, theta, v, reinterpret_cast<double*>(smem), acc);
    }
    double tot[2];
    if (grid_reduce<2>(acc, rs, tot, sh) && threadIdx.x == 0 && threadIdx.y == 0) {
        auto next_cycle = [&](double rr) {  // start an inner cycle from a refined residual rr
            const double drop = fmax(kChebDrop, sqrt(cg->tol2 / rr));
            cg->nin = cheb_steps(theta, delta, drop);
            cg->inner = 0;
            cg->rho = delta / theta;
            cg->phase = CH_ITER;
        };
        if (START) {
            cg->rr0 = tot[0];
            cg->rr = tot[0];
            cg_begin(cg, o, tot[0], tot[1]);
            if (!cg->done) next_cycle(tot[0]);
            if (iters_out) *iters_out = 0;
            set_loop(cond, !cg->done);
            return;
        }
        cg->iter += 1;
        if (phase == CH_ITER) {
            double rho = cg->rho;
            for (int q = 0; q < CK; ++q) rho = 1.0 / (2.0 * (theta / delta) - rho);
            cg->rho = rho;
            cg->inner += CK;
            if (!isfinite(tot[0])) cg_unconverged(cg, tot[0]);
            else if (cg->inner >= cg->nin) cg->phase = CH_REFINE;
        } else {
            cg->rr = tot[0];
            if (tot[0] <= cg->tol2) { cg->conv = 1; cg->done = 1; }
            else if (!isfinite(tot[0])) cg_unconverged(cg, tot[0]);
            else next_cycle(tot[0]);
        }
        if (!cg->done && cg->iter >= cg->maxiter) cg_unconverged(cg, cg->rr);
        if (iters_out) *iters_out = cg->iter;
        set_loop(cond, !cg->done);
    }
}

static ChebArgs cheb_args(const ViscSolve& w, const ViscMixed& m, const double* rhs_u, const double* rhs_v,
                          int parity) {
    const int c = parity & 1, n = c ^ 1;
    return ChebArgs{m.r_u[c], m.r_v[c], m.w_u[c], m.w_v[c], m.s_u[c], m.s_v[c],
                    m.r_u[n], m.r_v[n], m.w_u[n], m.w_v[n], m.s_u[n], m.s_v[n], w.x_u, w.x_v, rhs_u, rhs_v, m.ring_w};
}

void visc_ring_weights(const Params& P, float* ring_w, cudaStream_t s) {
    const int n = (int)visc_ring_cells(P.g.Nx, P.g.Ny) * 18;
    k_ring_weights<<<(n + 255) / 256, 256, 0, s>>>(P, ring_w);
}

cudaError_t solvers_configure() {
    cudaError_t e = cudaFuncSetAttribute(k_vcheb<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kChebSmemBytes);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_vcheb<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kChebSmemBytes);
}

bool visc_cheb_applies(const Params& P) {
    return P.md.viscosity == EFSI_VISC_CONSTANT && (!P.g.px || P.g.Nx >= CWX) && (!P.g.py || P.g.Ny >= CWY);
}

// One grid for every phase: a block per refinement tile (the smaller tile), at most
// kChebBlocksPerSM per SM, which all stay resident (the launch bounds).
static int cheb_grid(const Params& P) {
    return persistent_grid(((P.g.Nx + VTX - 1) / VTX) * ((P.g.Ny + VTY - 1) / VTY), P.nsm, kChebBlocksPerSM);
}

void visc_cheb_init(const Params& P, DtCoef alpha, const SolveOpts& o, const double* Un, const double* Vn,
                    const double* rhs_u, const double* rhs_v, const ViscSolve& w, const ViscMixed& m, CGScal* cg,
                    const RedSlot& rs, int* iters_out, cudaGraphConditionalHandle cond, cudaStream_t s) {
    k_visc_x0<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, Un, Vn, w.x_u, w.x_v);
    // the first body launch has parity 0 and reads set 0, which START writes (its "next")
    k_vcheb<true><<<cheb_grid(P), dim3(CWX, CBY), kChebSmemBytes, s>>>(P, alpha, o, cheb_args(w, m, rhs_u, rhs_v, 1), cg, rs,
                                                         iters_out, cond);
}

void visc_cheb_iter(const Params& P, DtCoef alpha, const double* rhs_u, const double* rhs_v, const ViscSolve& w,
                    const ViscMixed& m, int parity, CGScal* cg, const RedSlot& rs, int* iters_out,
                    cudaGraphConditionalHandle cond, cudaStream_t s) {
    k_vcheb<false><<<cheb_grid(P), dim3(CWX, CBY), kChebSmemBytes, s>>>(P, alpha, SolveOpts{}, cheb_args(w, m, rhs_u, rhs_v, parity),
                                                          cg, rs, iters_out, cond);
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

__global__ void k_diff_init(Params P, DtCoef ac, SolveOpts o, const double* __restrict__ c0,
                            const double* __restrict__ rhs, const double* __restrict__ phi, double* x, double* r,
                            double* dinv, CGScal* cg, RedSlot rs, int* iters_out, cudaGraphConditionalHandle cond) {
    __shared__ double sh[96];
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx;
    const double alpha = ac.value();
    double acc[3] = {0.0, 0.0, 0.0};
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
        acc[2] = rhs[k] * rhs[k];
    }
    double tot[3];
    if (grid_reduce<3>(acc, rs, tot, sh) && threadIdx.x == 0 && threadIdx.y == 0) {
        cg->rr0 = tot[0]; cg->rr = tot[0]; cg->rz = tot[1];
        cg_begin(cg, o, tot[0], tot[2]);
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
        else if (cg->iter >= cg->maxiter || !isfinite(tot[0])) cg_unconverged(cg, tot[0]);
        if (iters_out) *iters_out = cg->iter;
        set_loop(cond, !cg->done);
    }
}

void diff_init(const Params& P, DtCoef alpha, const SolveOpts& o, const double* c0, const double* rhs,
               const double* phi, const ScalarSolve& w, CGScal* cg, const RedSlot& rs, int* iters_out,
               cudaGraphConditionalHandle cond, cudaStream_t s) {
    k_diff_init<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, alpha, o, c0, rhs, phi, w.x, w.r,
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

// ---- judgement of a finished velocity / resource solve ----------------------------------
SolveOpts solve_opts(const efsi_numerics& nu, int method) {
    SolveOpts o;
    const bool direct = method != EFSI_LINEAR_GMRES;
    o.reltol = direct ? kDirectReltol : nu.linear_reltol;
    o.maxiter = direct ? EFSI_LINEAR_HARD_CAP : std::max(1, nu.linear_maxiter);
    o.fallback = (!direct && nu.direct_fallback) ? 1 : 0;  // DIRECT has nothing to fall back to
    o.fb_tol = nu.fallback_reltol;
    return o;
}

__global__ void k_solve_status(const CGScal* cg, DevStatus* st, int which, int stage) {
    if (cg->fail) raise_err(st, DE_LINEAR_NOCONV, which, stage, cg->iter, cg->fail_rel);
}
void solve_status(const CGScal* cg, DevStatus* st, int which, int stage, cudaStream_t s) {
    k_solve_status<<<1, 1, 0, s>>>(cg, st, which, stage);
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

// Restriction weights of coarse cell I (bilinear P^T, reflection at walls, wrap when periodic).
__device__ __forceinline__ void rweights(int I, int nc, bool per, int (&f)[4], double (&w)[4]) {
    f[0] = 2 * I - 1; w[0] = 0.25;
    f[1] = 2 * I;     w[1] = 0.75 + ((I == 0 && !per) ? 0.25 : 0.0);
    f[2] = 2 * I + 1; w[2] = 0.75 + ((I == nc - 1 && !per) ? 0.25 : 0.0);
    f[3] = 2 * I + 2; w[3] = 0.25;
    const int nf = 2 * nc;
    if (f[0] < 0) { if (per) f[0] += nf; else w[0] = 0.0; }
    if (f[3] >= nf) { if (per) f[3] -= nf; else w[3] = 0.0; }
}

// Bilinear prolongation value (P e) at fine cell (i,j).
template <class E>
__device__ __forceinline__ double prolong(const MGLevel& C, int px, int py, const E* e, int i, int j) {
    auto pair = [](int f, int nc, bool per, int& I0, int& I1) {
        I0 = f / 2;
        I1 = (f & 1) ? I0 + 1 : I0 - 1;
        if (I1 < 0) I1 = per ? nc - 1 : I0;
        if (I1 >= nc) I1 = per ? 0 : I0;
    };
    int I0, I1, J0, J1;
    pair(i, C.nx, px, I0, I1);
    pair(j, C.ny, py, J0, J1);
    auto Ev = [&](int a, int b) { return (double)__ldg(e + cidx(a, b, C.nx)); };
    return 0.75 * (0.75 * Ev(I0, J0) + 0.25 * Ev(I1, J0)) + 0.25 * (0.75 * Ev(I0, J1) + 0.25 * Ev(I1, J1));
}

// ---- fused multigrid kernels ----------------------------------------------------------------
// Each block owns T x T fine cells ((T/2)^2 coarse cells) per tile and loops over tiles
// (persistent grid).  Shared-memory slots hold values at wrapped global indices when
// periodic and zero outside walls, so a neighbour that exists (lev_off's tests) is the
// adjacent slot.  The slot's diagonal (0 = no cell) is computed once per tile.  Red
// cells are (i+j) even; tile origins are even, so the colour of a slot is the parity of
// its local coordinates.  A tile whose loaded region is at least one cell away from
// every edge is "inner": constant diagonal, all four couplings present.
struct SlotPos {
    int wi, wj;    // wrapped global cell
    bool valid;    // a cell of the level (possibly through periodic wrap)
};
__device__ __forceinline__ SlotPos slot_pos(const MGLevel& L, int px, int py, int gi, int gj) {
    const bool inx = gi >= 0 && gi < L.nx, iny = gj >= 0 && gj < L.ny;
    SlotPos p;
    p.valid = (inx || px) && (iny || py);
    p.wi = inx ? gi : (p.valid ? wrapm(gi, L.nx) : 0);
    p.wj = iny ? gj : (p.valid ? wrapm(gj, L.ny) : 0);
    return p;
}
// lev_off over neighbour slots (W, E, S, N order); (gi, gj) unwrapped: a wrapped slot
// lies in a periodic direction, where every coupling exists.
__device__ __forceinline__ double slot_off(const MGLevel& L, int px, int py, int gi, int gj, const double* s, int k,
                                           int row) {
    double off = 0.0;
    off += ((gi > 0 || px) ? L.ax : 0.0) * s[k - 1];
    off += ((gi < L.nx - 1 || px) ? L.ax : 0.0) * s[k + 1];
    off += ((gj > 0 || py) ? L.ay : 0.0) * s[k - row];
    off += ((gj < L.ny - 1 || py) ? L.ay : 0.0) * s[k + row];
    return off;
}
__device__ __forceinline__ double inner_off(const MGLevel& L, const double* s, int k, int row) {
    double off = 0.0;
    off += L.ax * s[k - 1];
    off += L.ax * s[k + 1];
    off += L.ay * s[k - row];
    off += L.ay * s[k + row];
    return off;
}
__device__ __forceinline__ double inner_diag(const MGLevel& L) {
    double d = 0.0;
    d += L.ax; d += L.ax; d += L.ay; d += L.ay;
    return d;
}
__device__ __forceinline__ bool inner_tile(const MGLevel& L, int i0, int j0, int T, int H) {
    return i0 - H >= 1 && i0 + T + H <= L.nx - 1 && j0 - H >= 1 && j0 + T + H <= L.ny - 1;
}

// Chronopoulos-Gear CG update fused into the finest pre-smoothing (z = M r and w = K z
// of the previous V-cycle):  p = z + b p_old, s = w + b s_old, x += a p,
// r_new = r_old - a s  (first iteration: p = z, s = w).
struct CGFuse {
    const double* r_old;
    const double* w;
    const double* s_old;
    const double* z;
    const double* p_old;
    double* x;
    double* r_new;
    double* s_new;
    double* p_new;
};

// Down leg of one level: pre-smoothing from x = 0 (red x = b/D, then one black GS
// update), residual r = b - K x, restriction b_c = P^T r (bilinear weights, reflection
// at walls, wrap when periodic).  Writes L.x (needed by the up leg) and C.b.
// FUSE: b is r_new of the CG update, formed on the fly over the halo; the owned cells
// of r_new and x are written and |r_new|^2 decides convergence.
// IN: element type of b (the finest level reads the FP64 CG residual); S: storage of
// the level arrays (FP64, or FP32 in the precision form).  Arithmetic is FP64.
template <int T, bool FUSE, class IN, class S>
__global__ void __launch_bounds__(256, 4) k_mg_down(MGLevel L, MGLevel C, int px, int py,
                                                    const IN* __restrict__ b, S* x_out, S* cb_out, CGFuse f,
                                                    CGScal* cg, RedSlot rs, int* iters_out,
                                                    cudaGraphConditionalHandle cond) {
    constexpr int H = 3, W = T + 2 * H;
    __shared__ double sb[W * W];  // b, then the residual (halo 1)
    __shared__ double sx[W * W];  // pre-smoothed x (valid within halo 2)
    __shared__ double sd[W * W];  // diagonal, 0 where there is no cell
    __shared__ double sh[32];
    if (cg && cg->done) return;
    const int tid = threadIdx.x;
    const int nx = L.nx;
    const double a = FUSE ? cg->alpha : 0.0;
    const bool first = FUSE && cg->iter == 0;
    const double bt = FUSE && !first ? cg->beta : 0.0;
    const double d0 = inner_diag(L);
    double acc[1] = {0.0};
    const int ntx = (nx + T - 1) / T, nt = ntx * ((L.ny + T - 1) / T);
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int bx = t % ntx, by = t / ntx;
        const int i0 = bx * T, j0 = by * T;
        const bool inner = inner_tile(L, i0, j0, T, H);
        // load b (FUSE: r_old - a Kp) over the region; loads are batched per thread
        constexpr int NS = (W * W + 255) / 256;
        double vb[NS], vd[NS];
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            const int s = tid + q * 256;
            vb[q] = 0.0;
            vd[q] = 0.0;
            if (s >= W * W) continue;
            const int gi = i0 + s % W - H, gj = j0 + s / W - H;
            size_t k;
            if (inner) {
                k = cidx(gi, gj, nx);
                vd[q] = d0;
            } else {
                const SlotPos sp = slot_pos(L, px, py, gi, gj);
                if (!sp.valid) continue;
                k = cidx(sp.wi, sp.wj, nx);
                lev_diag(L, px, py, sp.wi, sp.wj, vd[q]);
            }
            if (FUSE) {
                const double sv = first ? __ldg(f.w + k) : __ldg(f.w + k) + bt * __ldg(f.s_old + k);
                vb[q] = __ldg(f.r_old + k) - a * sv;
            } else {
                vb[q] = (double)__ldg(b + k);
            }
        }
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            const int s = tid + q * 256;
            if (s >= W * W) continue;
            const int lx = s % W, ly = s / W;
            sb[s] = vb[q];
            sd[s] = vd[q];
            sx[s] = (vd[q] != 0.0 && ((lx + ly) & 1) == 0) ? vb[q] / vd[q] : 0.0;
        }
        __syncthreads();
        if (FUSE) {  // owned cells: p, s, x += a p, r_new, |r_new|^2
            constexpr int NO = T * T / 256;
            double pv[NO], sv[NO], xv[NO];
            size_t kk[NO];
            bool in[NO];
#pragma unroll
            for (int q = 0; q < NO; ++q) {
                const int s = tid + q * 256, lx = s % T, ly = s / T;
                in[q] = i0 + lx < nx && j0 + ly < L.ny;
                kk[q] = cidx(i0 + lx, j0 + ly, nx);
                pv[q] = 0.0;
                sv[q] = 0.0;
                xv[q] = 0.0;
                if (!in[q]) continue;
                pv[q] = first ? f.z[kk[q]] : f.z[kk[q]] + bt * f.p_old[kk[q]];
                sv[q] = first ? f.w[kk[q]] : f.w[kk[q]] + bt * f.s_old[kk[q]];
                xv[q] = f.x[kk[q]];
            }
#pragma unroll
            for (int q = 0; q < NO; ++q) {
                if (!in[q]) continue;
                const int s = tid + q * 256, lx = s % T, ly = s / T;
                const double v = sb[(ly + H) * W + lx + H];
                f.p_new[kk[q]] = pv[q];
                f.s_new[kk[q]] = sv[q];
                f.r_new[kk[q]] = v;
                f.x[kk[q]] = xv[q] + a * pv[q];
                acc[0] += v * v;
            }
        }
        // black cells within halo 2
        constexpr int B = T + 4;
        for (int s = tid; s < B * B / 2; s += 256) {
            const int ry = s / (B / 2), rx = 2 * (s % (B / 2)) + ((ry + 1) & 1);
            const int lx = rx + 1, ly = ry + 1, k = ly * W + lx;
            const double d = sd[k];
            if (d == 0.0) continue;
            const double off = inner ? inner_off(L, sx, k, W)
                                     : slot_off(L, px, py, i0 + lx - H, j0 + ly - H, sx, k, W);
            sx[k] = (sb[k] + off) / d;
        }
        __syncthreads();
        // residual within halo 1 (in place of b)
        constexpr int R = T + 2;
        for (int s = tid; s < R * R; s += 256) {
            const int lx = s % R + 2, ly = s / R + 2, k = ly * W + lx;
            const double d = sd[k];
            if (d == 0.0) continue;
            const double off = inner ? inner_off(L, sx, k, W)
                                     : slot_off(L, px, py, i0 + lx - H, j0 + ly - H, sx, k, W);
            sb[k] = sb[k] - (d * sx[k] - off);
        }
        __syncthreads();
        if (tid < (T / 2) * (T / 2)) {
            // restriction: fine cells 2I-1 .. 2I+2 are slots 2(I-I0)+2 .. +5 (wrapped values
            // already sit in the halo)
            const int cx = tid % (T / 2), cy = tid / (T / 2);
            const int I = bx * (T / 2) + cx, J = by * (T / 2) + cy;
            if (I < C.nx && J < C.ny) {
                int fx[4], fy[4];
                double wx[4], wy[4];
                rweights(I, C.nx, px, fx, wx);
                rweights(J, C.ny, py, fy, wy);
                double sum = 0.0;
#pragma unroll
                for (int bb = 0; bb < 4; ++bb) {
                    if (wy[bb] == 0.0) continue;
                    double row = 0.0;
#pragma unroll
                    for (int aa = 0; aa < 4; ++aa)
                        if (wx[aa] != 0.0) row += wx[aa] * sb[(2 * cy + bb + 2) * W + 2 * cx + aa + 2];
                    sum += wy[bb] * row;
                }
                cb_out[cidx(I, J, C.nx)] = (S)sum;
            }
        }
        for (int s = tid; s < T * T; s += 256) {
            const int lx = s % T, ly = s / T;
            const int gi = i0 + lx, gj = j0 + ly;
            if (gi < nx && gj < L.ny) x_out[cidx(gi, gj, nx)] = (S)sx[(ly + H) * W + lx + H];
        }
        __syncthreads();
    }
    if (!FUSE) return;
    double tot[1];
    if (grid_reduce<1>(acc, rs, tot, sh) && tid == 0) {
        cg->iter += 1;
        cg->rr = tot[0];
        if (tot[0] <= cg->tol2) { cg->conv = 1; cg->done = 1; }
        else if (cg->iter >= cg->maxiter || !isfinite(tot[0])) cg->done = 1;
        if (iters_out) *iters_out = cg->iter;
        set_loop(cond, !cg->done);
    }
}

// Up leg of one level: x + P e (bilinear prolongation), then the post-smoothing
// black-then-red Gauss-Seidel sweep.  DOT (finest level, the CG preconditioner):
// z is completed over the tile and a one-cell ring, w = K z is formed on the tile,
// and the Chronopoulos-Gear scalars follow from g = r.z and d = z.w:
//   first V-cycle of a solve: a = g / d;  otherwise b = g / g_old, a = g / (d - b g / a_old).
template <int T, bool DOT, class S, class IN, class OUT>
__global__ void __launch_bounds__(256, 4) k_mg_up(MGLevel L, MGLevel C, int px, int py, const S* __restrict__ x,
                                                  const S* __restrict__ e, const IN* __restrict__ b, OUT* xo,
                                                  double* wo, CGScal* cg, RedSlot rs) {
    constexpr int H = DOT ? 3 : 2, W = T + 2 * H;
    __shared__ double sx[W * W];
    __shared__ double sb[W * W];
    __shared__ double sd[W * W];
    __shared__ double sh[2 * 32];  // block sums of r.z and z.w
    if (cg && cg->done) return;
    const int tid = threadIdx.x;
    const int nx = L.nx;
    const double d0 = inner_diag(L);
    double acc[2] = {0.0, 0.0};
    const int ntx = (nx + T - 1) / T, nt = ntx * ((L.ny + T - 1) / T);
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int i0 = (t % ntx) * T, j0 = (t / ntx) * T;
        const bool inner = inner_tile(L, i0, j0, T, H);
        constexpr int NS = (W * W + 255) / 256;
        double xv[NS], bv[NS], dv[NS];
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            const int s = tid + q * 256;
            xv[q] = 0.0;
            bv[q] = 0.0;
            dv[q] = 0.0;
            if (s >= W * W) continue;
            int wi = i0 + s % W - H, wj = j0 + s / W - H;
            if (inner) {
                dv[q] = d0;
            } else {
                const SlotPos sp = slot_pos(L, px, py, wi, wj);
                if (!sp.valid) continue;
                wi = sp.wi;
                wj = sp.wj;
                lev_diag(L, px, py, wi, wj, dv[q]);
            }
            const size_t k = cidx(wi, wj, nx);
            xv[q] = (double)__ldg(x + k) + prolong(C, px, py, e, wi, wj);
            bv[q] = (double)__ldg(b + k);
        }
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            const int s = tid + q * 256;
            if (s >= W * W) continue;
            sx[s] = xv[q];
            sb[s] = bv[q];
            sd[s] = dv[q];
        }
        __syncthreads();
        // black cells within halo H - 1 (a slot's colour is the parity of lx + ly: tile
        // origins are even, so it does not depend on H)
        constexpr int B = T + 2 * (H - 1);
        for (int s = tid; s < B * B / 2; s += 256) {
            const int ry = s / (B / 2), rx = 2 * (s % (B / 2)) + ((ry + 1) & 1);  // lx + ly odd
            const int lx = rx + 1, ly = ry + 1, k = ly * W + lx;
            const double d = sd[k];
            if (d == 0.0) continue;
            const double off = inner ? inner_off(L, sx, k, W)
                                     : slot_off(L, px, py, i0 + lx - H, j0 + ly - H, sx, k, W);
            sx[k] = (sb[k] + off) / d;
        }
        __syncthreads();
        if (DOT) {
            // red cells of the tile and its one-cell ring (their black neighbours are final)
            constexpr int R = T + 2;
            for (int s = tid; s < R * R / 2; s += 256) {
                // lx + ly even; lx = rx + H - 1 and ly = ry + H - 1 with H - 1 = 2 even
                const int ry = s / (R / 2), rx = 2 * (s % (R / 2)) + (ry & 1);
                const int lx = rx + H - 1, ly = ry + H - 1, k = ly * W + lx;
                const double d = sd[k];
                if (d == 0.0) continue;
                const double off = inner ? inner_off(L, sx, k, W)
                                         : slot_off(L, px, py, i0 + lx - H, j0 + ly - H, sx, k, W);
                sx[k] = (sb[k] + off) / d;
            }
            __syncthreads();
            // z on the tile, w = K z, r.z and z.w
            for (int s = tid; s < T * T; s += 256) {
                const int lx = s % T, ly = s / T;
                const int gi = i0 + lx, gj = j0 + ly;
                if (gi >= nx || gj >= L.ny) continue;
                const int k = (ly + H) * W + lx + H;
                const double zc = sx[k];
                const double off = inner ? inner_off(L, sx, k, W) : slot_off(L, px, py, gi, gj, sx, k, W);
                const double wc = sd[k] * zc - off;
                xo[cidx(gi, gj, nx)] = (OUT)zc;
                wo[cidx(gi, gj, nx)] = wc;
                acc[0] += sb[k] * zc;
                acc[1] += zc * wc;
            }
            __syncthreads();
            continue;
        }
        // red cells of the tile (their black neighbours are final); write the tile
        for (int s = tid; s < T * T; s += 256) {
            const int lx = s % T, ly = s / T;
            const int gi = i0 + lx, gj = j0 + ly;
            if (gi >= nx || gj >= L.ny) continue;
            const int k = (ly + H) * W + lx + H;
            const double bc = sb[k];
            double val = sx[k];
            if (((lx + ly) & 1) == 0) {
                const double off = inner ? inner_off(L, sx, k, W) : slot_off(L, px, py, gi, gj, sx, k, W);
                val = (bc + off) / sd[k];
            }
            xo[cidx(gi, gj, nx)] = (OUT)val;
        }
        __syncthreads();
    }
    if (!DOT) return;
    double tot[2];
    if (grid_reduce<2>(acc, rs, tot, sh) && tid == 0) {
        const double g = tot[0], d = tot[1];
        if (cg->iter == 0) {
            cg->beta = 0.0;
            cg->alpha = d != 0.0 ? g / d : 0.0;
        } else {
            const double bn = cg->rz != 0.0 ? g / cg->rz : 0.0;
            const double den = d - (cg->alpha != 0.0 ? bn * g / cg->alpha : 0.0);
            cg->beta = bn;
            cg->alpha = den != 0.0 ? g / den : 0.0;
        }
        cg->rz = g;
        cg->pAp = d;
    }
}

// Coarsest level: x = Minv b with the dense (shifted) inverse; 8 rows per block.
template <class S>
__global__ void k_mg_dense(int n, const S* __restrict__ Minv, const S* __restrict__ b, S* x, const CGScal* cg) {
    if (cg && cg->done) return;
    __shared__ double sb[1024];
    for (int k = threadIdx.x; k < n; k += blockDim.x) sb[k] = b[k];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row = blockIdx.x * 8 + warp;
    if (row < n) {
        // 16-byte loads, eight per lane in flight before the adds (two accumulators);
        // the row start is 16-byte aligned when n is a multiple of the vector width
        const S* m = Minv + (size_t)row * n;
        constexpr int VW = 16 / (int)sizeof(S);
        double s0 = 0.0, s1 = 0.0;
        if (n % VW == 0) {
            using Vec = typename std::conditional<sizeof(S) == 4, float4, double2>::type;
            const Vec* mv = reinterpret_cast<const Vec*>(m);
            const int nv = n / VW;
#pragma unroll 8
            for (int q = lane; q < nv; q += 32) {
                const Vec w = __ldg(mv + q);
                const double* bb = sb + q * VW;
                if constexpr (sizeof(S) == 4) {
                    s0 += (double)w.x * bb[0] + (double)w.y * bb[1];
                    s1 += (double)w.z * bb[2] + (double)w.w * bb[3];
                } else {
                    s0 += w.x * bb[0];
                    s1 += w.y * bb[1];
                }
            }
        } else {
#pragma unroll 8
            for (int k = lane; k < n; k += 32) s0 += (double)__ldg(m + k) * sb[k];
        }
        double s = s0 + s1;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) x[row] = (S)s;
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

// Level arrays of storage type S (FP64, or FP32 in the precision form).
template <class S> struct LevelArrays;
template <> struct LevelArrays<double> {
    static double* x(const MGLevel& L) { return L.x; }
    static double* xo(const MGLevel& L) { return L.xo; }
    static double* b(const MGLevel& L) { return L.b; }
    static const double* inv(const Projection& p) { return p.coarse_inv; }
};
template <> struct LevelArrays<float> {
    static float* x(const MGLevel& L) { return L.xf; }
    static float* xo(const MGLevel& L) { return L.xof; }
    static float* b(const MGLevel& L) { return L.bf; }
    static const float* inv(const Projection& p) { return p.coarse_inv_f; }
};

template <int T, class S>
static void mg_down(const MGLevel& L, const MGLevel& C, int l, const double* r_fine, const CGFuse* fuse, int grid,
                    CGScal* cg, const RedSlot& rs, int* iters_out, cudaGraphConditionalHandle cond, int px, int py,
                    cudaStream_t s) {
    using A = LevelArrays<S>;
    if (l == 0) {
        if (fuse)
            k_mg_down<T, true, double, S><<<grid, 256, 0, s>>>(L, C, px, py, r_fine, A::x(L), A::b(C), *fuse, cg, rs,
                                                              iters_out, cond);
        else
            k_mg_down<T, false, double, S><<<grid, 256, 0, s>>>(L, C, px, py, r_fine, A::x(L), A::b(C), CGFuse{},
                                                               cg, rs, nullptr, 0);
    } else {
        k_mg_down<T, false, S, S><<<grid, 256, 0, s>>>(L, C, px, py, A::b(L), A::x(L), A::b(C), CGFuse{}, cg, rs,
                                                       nullptr, 0);
    }
}

template <int T, class S>
static void mg_up(const Projection& pj, const MGLevel& L, const MGLevel& C, int l, const double* r_fine, int grid,
                  CGScal* cg, const RedSlot& rs2, int px, int py, cudaStream_t s) {
    using A = LevelArrays<S>;
    if (l == 0)
        k_mg_up<T, true, S, double, double><<<grid, 256, 0, s>>>(L, C, px, py, A::x(L), A::xo(C), r_fine, pj.z,
                                                                pj.w, cg, rs2);
    else
        k_mg_up<T, false, S, S, S><<<grid, 256, 0, s>>>(L, C, px, py, A::x(L), A::xo(C), A::b(L), A::xo(L),
                                                        nullptr, cg, rs2);
}

template <class S>
static void vcycle_levels(const Projection& pj, const double* r_fine, const CGFuse* fuse, CGScal* cg,
                          const RedSlot& rs, const RedSlot& rs2, int* iters_out, cudaGraphConditionalHandle cond,
                          int px, int py, cudaStream_t s) {
    const int n = pj.nlev;
    // 32x32 tiles while they give every SM its 4 resident blocks, 16x16 below (more
    // blocks and shorter dependent chains; at 512^2 this measured 3 us faster per cycle)
    auto wide = [&](const MGLevel& L) { return ((L.nx + 31) / 32) * ((L.ny + 31) / 32) >= 4 * pj.nsm; };
    auto grid = [&](const MGLevel& L, int T) {
        return persistent_grid(((L.nx + T - 1) / T) * ((L.ny + T - 1) / T), pj.nsm, 4);
    };
    for (int l = 0; l + 1 < n; ++l) {
        const MGLevel &L = pj.lev[l], &C = pj.lev[l + 1];
        if (wide(L)) mg_down<32, S>(L, C, l, r_fine, fuse, grid(L, 32), cg, rs, iters_out, cond, px, py, s);
        else mg_down<16, S>(L, C, l, r_fine, fuse, grid(L, 16), cg, rs, iters_out, cond, px, py, s);
    }
    const MGLevel& B = pj.lev[n - 1];
    using A = LevelArrays<S>;
    k_mg_dense<S><<<(pj.nc + 7) / 8, 256, 0, s>>>(pj.nc, A::inv(pj), A::b(B), A::xo(B), cg);
    for (int l = n - 2; l >= 0; --l) {
        const MGLevel &L = pj.lev[l], &C = pj.lev[l + 1];
        if (wide(L)) mg_up<32, S>(pj, L, C, l, r_fine, grid(L, 32), cg, rs2, px, py, s);
        else mg_up<16, S>(pj, L, C, l, r_fine, grid(L, 16), cg, rs2, px, py, s);
    }
}

// z = M r_fine with one V(1,1)-cycle; the finest down leg optionally carries the CG update.
static void vcycle(const Projection& pj, const double* r_fine, const CGFuse* fuse, CGScal* cg, const RedSlot& rs,
                   const RedSlot& rs2, int* iters_out, cudaGraphConditionalHandle cond, int px, int py,
                   cudaStream_t s) {
    if (pj.nlev == 1) {
        k_mg_dense<double><<<(pj.nc + 7) / 8, 256, 0, s>>>(pj.nc, pj.coarse_inv, r_fine, pj.z, cg);
        k_dot_rz<<<(pj.nc + 255) / 256, 256, 0, s>>>(pj.nc, r_fine, pj.z, cg, rs2);
        return;
    }
    if (pj.mixed) vcycle_levels<float>(pj, r_fine, fuse, cg, rs, rs2, iters_out, cond, px, py, s);
    else vcycle_levels<double>(pj, r_fine, fuse, cg, rs, rs2, iters_out, cond, px, py, s);
}

int proj_update_vcycle_kernels(const Projection& pj) { return pj.nlev == 1 ? 3 : 2 * (pj.nlev - 1) + 1; }
int proj_matvec_kernels(const Projection& pj) { return pj.nlev == 1 ? 1 : 0; }
int proj_init_kernels(const Projection& pj) { return 1 + (pj.nlev == 1 ? 2 : 2 * (pj.nlev - 1) + 1); }
double proj_update_vcycle_bytes(const Projection& pj) {
    const double n0 = (double)pj.lev[0].nx * pj.lev[0].ny;
    if (pj.nlev == 1) return 8.0 * (6.0 * n0 + (double)pj.nc * pj.nc + 4.0 * pj.nc);
    const double e = pj.mixed ? 4.0 : 8.0;  // bytes of a multigrid level element
    // finest down: r_old, w, s_old, z, p_old, x read and p, s, x, r_new written (FP64);
    // L.x and C.b written; up: L.x, e read, r_new read, z and w written (FP64)
    double b = 8.0 * 13.0 * n0 + e * (2.25 * n0 + 0.25 * n0 + 1.0 * n0);
    for (int l = 1; l + 1 < pj.nlev; ++l) b += e * 5.5 * (double)pj.lev[l].nx * pj.lev[l].ny;
    b += e * ((double)pj.nc * pj.nc + 2.0 * pj.nc);
    return b;
}

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

// 64 registers at most: four blocks per SM
__global__ void __launch_bounds__(256, 4) k_proj_rhs(Params P, PredIn in, const double* __restrict__ G, double* Up, double* Vp, double* rhs,
                           double* bw, int nullspace, ProjScal* ps, RedSlot rs, DevStatus* st) {
    __shared__ double sh[32 * 6];
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const double area = P.g.hx * P.g.hy;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for_tiles(Nx + 1, Ny + 1, [&](int i, int j) {
        if (j < Ny) Up[uidx(i, j, Nx)] = in.U(P, i, j);
        if (i < Nx) Vp[vidx(i, j, Nx)] = in.V(P, i, j);
        if (i >= Nx || j >= Ny) return;
        double div = (in.U(P, i + 1, j) - in.U(P, i, j)) * P.g.ihx + (in.V(P, i, j + 1) - in.V(P, i, j)) * P.g.ihy;
        double g = G ? G[cidx(i, j, Nx)] : 0.0;
        double rr = (div - g) - q_boundary_vec(P, i, j);
        size_t k = cidx(i, j, Nx);
        rhs[k] = rr;
        double b = -rr * area;
        bw[k] = b;
        acc[0] += rr * area;
        acc[1] += fabs(rr) * area;
        acc[2] += b;
        acc[3] += rr * rr;
        acc[4] += div * div * area;
        acc[5] += g * g * area;
    });
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
    k_proj_rhs<<<persistent_grid(tiles2(P.g.Nx + 1, P.g.Ny + 1), P.nsm, 4), dim3(BX, BY), 0, s>>>(P, in, G, pj.Up, pj.Vp, pj.rhs, pj.b,
                                                                     pj.nullspace ? 1 : 0, ps, rs, st);
}

// ---- CG on the fine level --------------------------------------------------------------------
__global__ void k_pcg_init(MGLevel L, int px, int py, double reltol, int maxiter, const double* __restrict__ q0,
                           const double* __restrict__ b, double* x, double* r, const ProjScal* ps, CGScal* cg,
                           RedSlot rs, const DevStatus* st, int* iters_out, cudaGraphConditionalHandle cond) {
    __shared__ double sh[32];
    const int nx = L.nx;
    const double bmean = ps->v[10];
    double acc[1] = {0.0};
    for_tiles(L.nx, L.ny, [&](int i, int j) {
        double d;
        lev_diag(L, px, py, i, j, d);
        auto xf = [&](int a, int c) { return q0[cidx(a, c, nx)]; };
        size_t k = cidx(i, j, nx);
        double rr = (b[k] - bmean) - (d * q0[k] - lev_off(L, px, py, i, j, xf));
        x[k] = q0[k];
        r[k] = rr;
        acc[0] += rr * rr;
    });
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

// Shared-memory view of p over one 32x8 tile with a one-cell halo: every slot holds
// p at its wrapped global cell (zero outside walls), so the wrapped requests of
// lev_off map back into the tile.
struct TileP {
    const double* sp;
    int i0, j0, nx, ny;
    __device__ __forceinline__ double operator()(int c, int r) const {
        int lc = c - i0 + 1, lr = r - j0 + 1;
        if (lc < 0) lc += nx; else if (lc >= VSX) lc -= nx;
        if (lr < 0) lr += ny; else if (lr >= VSY) lr -= ny;
        return sp[lr * VSX + lc];
    }
};

// p = z + beta p_old, Kp, p.Kp -> alpha.  Persistent over 32x8 tiles; p is formed
// once per cell of the tile and its halo in shared memory.  Cells away from the edges
// take the branch-free form of lev_diag/lev_off (same terms, same order).
__global__ void __launch_bounds__(BX * BY, 6) k_pcg_matvec(MGLevel L, int px, int py, const double* __restrict__ z,
                                                           const double* __restrict__ p_old, double* p, double* Ap,
                                                           CGScal* cg, RedSlot rs) {
    static_assert(BX == VTX && BY == VTY, "the matvec tile is the viscous tile");
    __shared__ double sp[VSX * VSY];
    __shared__ double sh[32];
    if (cg->done) return;
    const int first = cg->iter == 0;
    const int nx = L.nx, ny = L.ny;
    const double beta = first ? 0.0 : cg->beta;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + ty * BX;
    auto pn = [&](size_t k) { return first ? z[k] : z[k] + beta * p_old[k]; };
    auto stage = [&](int gi, int gj) -> double {
        const bool inx = gi >= 0 && gi < nx, iny = gj >= 0 && gj < ny;
        if (!((inx || px) && (iny || py))) return 0.0;
        return pn(cidx(inx ? gi : wrapm(gi, nx), iny ? gj : wrapm(gj, ny), nx));
    };
    const int ntx = (nx + BX - 1) / BX, nt = ntx * ((ny + BY - 1) / BY);
    double acc[1] = {0.0};
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int i0 = (t % ntx) * BX, j0 = (t / ntx) * BY;
        const int i = i0 + tx, j = j0 + ty;
        const bool own = i < nx && j < ny;
        const int s = (ty + 1) * VSX + tx + 1;
        const double pc = own ? pn(cidx(i, j, nx)) : stage(i, j);
        sp[s] = pc;
        if (tid < 2 * VSX + 2 * VTY) {
            int lx, ly;
            visc_halo_slot(tid, lx, ly);
            sp[ly * VSX + lx] = stage(i0 + lx - 1, j0 + ly - 1);
        }
        __syncthreads();
        if (own) {
            const size_t k = cidx(i, j, nx);
            double q;
            if (i > 0 && i < nx - 1 && j > 0 && j < ny - 1) {
                double d = 0.0;
                d += L.ax; d += L.ax; d += L.ay; d += L.ay;
                double off = 0.0;
                off += L.ax * sp[s - 1];
                off += L.ax * sp[s + 1];
                off += L.ay * sp[s - VSX];
                off += L.ay * sp[s + VSX];
                q = d * pc - off;
            } else {
                double d;
                lev_diag(L, px, py, i, j, d);
                q = d * pc - lev_off(L, px, py, i, j, TileP{sp, i0, j0, nx, ny});
            }
            p[k] = pc;
            Ap[k] = q;
            acc[0] += pc * q;
        }
        __syncthreads();
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
    k_pcg_init<<<persistent_grid(tiles2(L.nx, L.ny), P.nsm, 6), dim3(BX, BY), 0, s>>>(L, P.g.px, P.g.py, reltol, maxiter, q0, pj.b, pj.x,
                                                          pj.r[0], ps, cg, rs, st, iters_out, cond);
    vcycle(pj, pj.r[0], nullptr, cg, rs, rs2, nullptr, 0, P.g.px, P.g.py, s);
}

void proj_spectral_init(const Params& P, const Projection& pj, double reltol, int maxiter, const double* q0,
                        CGScal* cg, const ProjScal* ps, const RedSlot& rs, const DevStatus* st, int* iters_out,
                        cudaGraphConditionalHandle cond, cudaStream_t s) {
    const MGLevel& L = pj.lev[0];
    k_pcg_init<<<persistent_grid(tiles2(L.nx, L.ny), P.nsm, 6), dim3(BX, BY), 0, s>>>(
        L, P.g.px, P.g.py, reltol, maxiter, q0, pj.b, pj.x, pj.r[0], ps, cg, rs, st, iters_out, cond);
}

// One CG iteration is proj_matvec then proj_update_vcycle with the same parity:
// p[parity] is written, r[parity] is read and r[parity^1] written (multigrid case).
void proj_matvec(const Params& P, const Projection& pj, int parity, CGScal* cg, const RedSlot& rs, cudaStream_t s) {
    if (pj.nlev > 1) return;  // the multigrid V-cycle forms w = K z itself (Chronopoulos-Gear)
    const MGLevel& L = pj.lev[0];
    const int cur = parity & 1, old = cur ^ 1;
    const int nt = ((L.nx + BX - 1) / BX) * ((L.ny + BY - 1) / BY);
    k_pcg_matvec<<<persistent_grid(nt, pj.nsm, 6), dim3(BX, BY), 0, s>>>(L, P.g.px, P.g.py, pj.z, pj.p[old],
                                                                          pj.p[cur], pj.Ap, cg, rs);
}
void proj_update_vcycle(const Params& P, const Projection& pj, int parity, CGScal* cg, const RedSlot& rs,
                        const RedSlot& rs2, int* iters_out, cudaGraphConditionalHandle cond, cudaStream_t s) {
    const MGLevel& L = pj.lev[0];
    const int cur = parity & 1;
    if (pj.nlev == 1) {
        k_pcg_update<<<grid2(L.nx, L.ny), dim3(BX, BY), 0, s>>>(L, pj.x, pj.r[0], pj.p[cur], pj.Ap, cg, rs,
                                                                iters_out, cond);
        vcycle(pj, pj.r[0], nullptr, cg, rs, rs2, nullptr, 0, P.g.px, P.g.py, s);
        return;
    }
    const int old = cur ^ 1;
    const CGFuse f{pj.r[cur], pj.w, pj.s[old], pj.z, pj.p[old], pj.x, pj.r[old], pj.s[cur], pj.p[cur]};
    vcycle(pj, pj.r[old], &f, cg, rs, rs2, iters_out, cond, P.g.px, P.g.py, s);
}

// ---- correction and diagnostics (Projection.jl:253-306) ---------------------------------------
__global__ void k_proj_mean(MGLevel L, const double* __restrict__ x, ProjScal* ps, RedSlot rs, int nullspace) {
    __shared__ double sh[32];
    double acc[1] = {0.0};
    for_tiles(L.nx, L.ny, [&](int i, int j) { acc[0] += x[cidx(i, j, L.nx)]; });
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

// 64 registers at most: four blocks per SM
__global__ void __launch_bounds__(256, 4) k_proj_correct(Params P, MGLevel L, const double* __restrict__ x, const double* __restrict__ Up,
                               const double* __restrict__ Vp, const double* __restrict__ G,
                               const double* __restrict__ rhs, double* q_out, double* U_out, double* V_out,
                               ProjScal* ps, double* stage_linf, RedSlot rmax, RedSlot rsum, DevStatus* st) {
    __shared__ double sh[64];
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const double mean = ps->v[6];
    const double area = P.g.hx * P.g.hy;
    double mx[1] = {0.0}, sm[2] = {0.0, 0.0};
    for_tiles(Nx, Ny, [&](int i, int j) {
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
        mx[0] = fmax(mx[0], fabs(c));
        sm[0] += c * c * area;
        // linear residual of the unpinned operator: L q - rhs, L q = -(K x)/area
        double d;
        lev_diag(L, P.g.px, P.g.py, i, j, d);
        auto xf = [&](int a, int b) { return x[cidx(a, b, Nx)] - mean; };
        double Lq = -(d * (x[k] - mean) - lev_off(L, P.g.px, P.g.py, i, j, xf)) / area;
        double lr = Lq - rhs[k];
        sm[1] += lr * lr;
    });
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

void proj_mean(const Params& P, const Projection& pj, ProjScal* ps, const RedSlot& rs, cudaStream_t s) {
    const MGLevel& L = pj.lev[0];
    k_proj_mean<<<persistent_grid(tiles2(L.nx, L.ny), P.nsm, 8), dim3(BX, BY), 0, s>>>(L, pj.x, ps, rs,
                                                                                     pj.nullspace ? 1 : 0);
}

void proj_finish(const Params& P, const Projection& pj, const double* G, double* q_out, double* U_out, double* V_out,
                 ProjScal* ps, double* stage_linf, const RedSlot& rs1, const RedSlot& rs2, DevStatus* st,
                 cudaStream_t s) {
    const MGLevel& L = pj.lev[0];
    const int nt = tiles2(L.nx, L.ny);
    dim3 b(BX, BY);
    k_proj_mean<<<persistent_grid(nt, P.nsm, 8), b, 0, s>>>(L, pj.x, ps, rs1, pj.nullspace ? 1 : 0);
    k_proj_correct<<<persistent_grid(nt, P.nsm, 4), b, 0, s>>>(P, L, pj.x, pj.Up, pj.Vp, G, pj.rhs, q_out, U_out, V_out, ps, stage_linf, rs1,
                                   rs2, st);
}

}  // namespace efsi
