// efsi_solvers.cuh — device-resident Krylov solvers of the IMEX step (host-side API).
#pragma once

#include "efsi_common.cuh"

namespace efsi {

// Scalars of one preconditioned-CG solve, kept in device memory so that the
// iteration runs without host round trips; `done` stops every later kernel.
struct CGScal {
    double rz, pAp, alpha, beta, rr, rr0, tol2;
    int iter, done, maxiter, conv;
};

// ---- viscous predictor (I - alpha*A) u = rhs with Dirichlet rows eliminated --------
struct ViscSolve {
    double *x_u, *x_v, *r_u, *r_v, *p_u[2], *p_v[2], *Ap_u, *Ap_v, *dinv_u, *dinv_v;
};
void visc_init(const Params& P, DtCoef alpha, double reltol, int maxiter, const double* Un, const double* Vn,
               const double* rhs_u, const double* rhs_v, const double* phi, const ViscSolve& w, CGScal* cg,
               const RedSlot& rs, int* iters_out, cudaGraphConditionalHandle cond, cudaStream_t s);
void visc_matvec(const Params& P, DtCoef alpha, const double* phi, const ViscSolve& w, CGScal* cg, const RedSlot& rs,
                 cudaStream_t s);
void visc_update(const Params& P, const ViscSolve& w, CGScal* cg, const RedSlot& rs, int* iters_out,
                 cudaGraphConditionalHandle cond, cudaStream_t s);
void visc_enforce_dirichlet(const Params& P, const double* rhs_u, const double* rhs_v, double* x_u, double* x_v,
                            cudaStream_t s);

// ---- resource implicit diffusion (I - alpha*L_D) c = rhs -----------------------------
struct ScalarSolve {
    double *x, *r, *p[2], *Ap, *dinv;
};
void diff_init(const Params& P, DtCoef alpha, double reltol, int maxiter, const double* c0, const double* rhs,
               const double* phi, const ScalarSolve& w, CGScal* cg, const RedSlot& rs, int* iters_out,
               cudaGraphConditionalHandle cond, cudaStream_t s);
void diff_iter(const Params& P, DtCoef alpha, const double* phi, const ScalarSolve& w, CGScal* cg, const RedSlot& rs1,
               const RedSlot& rs2, int* iters_out, cudaGraphConditionalHandle cond, cudaStream_t s);

// ---- projection ------------------------------------------------------------------------
struct MGLevel {
    int nx, ny;
    double ax, ay;                      // hy/hx, hx/hy (same on every level)
    double *cl, *cr, *cb, *ct;          // boundary coefficient factor per boundary cell (device)
    double *x, *xo, *b, *r;             // level vectors (x/xo ping-pong)
};
struct Projection {
    int nlev;
    MGLevel lev[16];
    double* coarse_inv;   // dense inverse of the coarsest operator (shifted when singular)
    int nc;
    bool nullspace;
    // fine-level CG vectors
    double *x, *r, *z, *p[2], *Ap, *b, *rhs;
    double *Up, *Vp;      // predictor velocity (full MAC arrays)
};
// Per-projection scalars: [0] defect, [1] scale, [2] sum b, [3] |rhs|^2, [4] wl2(div)^2,
// [5] wl2(target)^2, [6] mean of x, [7] linear relative residual, [8] constraint linf,
// [9] constraint l2, [10] b mean
struct ProjScal {
    double v[12];
};
void proj_rhs(const Params& P, const Projection& pj, bool compact_in, const double* u_in, const double* v_in,
              const double* G, ProjScal* ps, const RedSlot& rs, DevStatus* st, cudaStream_t s);
void proj_cg_init(const Params& P, const Projection& pj, double reltol, int maxiter, const double* q0, CGScal* cg,
                  const ProjScal* ps, const RedSlot& rs, const RedSlot& rs2, const DevStatus* st, int* iters_out,
                  cudaGraphConditionalHandle cond, cudaStream_t s);
void proj_matvec(const Params& P, const Projection& pj, int parity, CGScal* cg, const RedSlot& rs, cudaStream_t s);
void proj_update(const Params& P, const Projection& pj, int parity, CGScal* cg, const RedSlot& rs, int* iters_out,
                 cudaGraphConditionalHandle cond, cudaStream_t s);
void proj_vcycle(const Params& P, const Projection& pj, CGScal* cg, const RedSlot& rs, cudaStream_t s);
void proj_finish(const Params& P, const Projection& pj, const double* G, double* q_out, double* U_out,
                 double* V_out, ProjScal* ps, double* stage_linf, const RedSlot& rs1, const RedSlot& rs2,
                 DevStatus* st, cudaStream_t s);
// Number of kernel launches of one projection CG iteration (statistics).
int proj_kernels_per_iter(const Projection& pj);

}  // namespace efsi
