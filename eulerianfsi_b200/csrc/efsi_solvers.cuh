// efsi_solvers.cuh — device-resident Krylov solvers of the IMEX step (host-side API).
#pragma once

#include "efsi_common.cuh"

namespace efsi {

// Scalars of one preconditioned-CG solve, kept in device memory so that the
// iteration runs without host round trips; `done` stops every later kernel.
struct CGScal {
    double rz, pAp, alpha, beta, rr, rr0, tol2;
    int iter, done, maxiter, conv;
    // precision form: phase of the refined solve, inner iterations since the last
    // restart, squared residual at that restart
    int phase, inner;
    double rr_restart;
    // judgement of a solve that stops short of its tolerance, as _solve_linear_system!
    // judges a GMRES result (TimeIntegrationIMEX.jl:602-641): |b|^2 of the whole system
    // (Dirichlet rows hold their data), fallback_reltol, whether the DIRECT continuation
    // is allowed / running, and the outcome (fail: relative residual fail_rel too large)
    double bnorm2, fb_tol, fail_rel;
    int fallback, in_fallback, fail;
    // precision form with the polynomial inner solver: Chebyshev steps of the current
    // inner cycle (nin) and the recurrence coefficient rho of its next step
    int nin;
    double rho;
};

// Tolerance and iteration limit of one velocity or resource solve, from its method
// (EFSI_LINEAR_DIRECT: 1e-13 and EFSI_LINEAR_HARD_CAP; EFSI_LINEAR_GMRES: reltol and
// maxiter) and the fallback options.
struct SolveOpts {
    double reltol;
    int maxiter;
    int fallback;
    double fb_tol;
};
SolveOpts solve_opts(const efsi_numerics& nu, int method);

// Squared relative residual of the DIRECT stand-in (1e-13 against the initial residual).
constexpr double kDirectReltol = 1e-13;

// The deciding thread of a velocity or resource CG calls this when the iteration
// stops without meeting its tolerance (iteration limit or a non-finite residual;
// rr = squared residual of the current iterate).  A relative residual within
// fallback_reltol is accepted, as the reference accepts such a GMRES result;
// otherwise the DIRECT continuation starts when allowed, or the solve fails.
__device__ __forceinline__ void cg_unconverged(CGScal* cg, double rr) {
    const double rel = sqrt(rr) / fmax(sqrt(cg->bnorm2), 2.220446049250313e-16);
    if (isfinite(rel) && rel <= cg->fb_tol) { cg->done = 1; return; }
    if (cg->fallback && !cg->in_fallback && isfinite(rel)) {
        cg->in_fallback = 1;
        cg->tol2 = kDirectReltol * kDirectReltol * cg->rr0;
        cg->maxiter = cg->iter + EFSI_LINEAR_HARD_CAP;
        return;
    }
    cg->done = 1;
    cg->fail = 1;
    cg->fail_rel = rel;
}

// Raise DE_LINEAR_NOCONV (EFSI_SOLVE) when the solve just finished failed its
// judgement; `which` 0 = velocity, 1 = resource; `stage` the 0-based stage.
void solve_status(const CGScal* cg, DevStatus* st, int which, int stage, cudaStream_t s);

// ---- viscous predictor (I - alpha*A) u = rhs with Dirichlet rows eliminated --------
// Chronopoulos-Gear (single-reduction) Jacobi-PCG: one kernel per iteration.  r, w
// (= A M r) and s (= A p) are ping-ponged between iterations (parity), so that the
// neighbours read by one launch are never the values it writes.
struct ViscSolve {
    double *x_u, *x_v, *p_u, *p_v, *dinv_u, *dinv_v;
    double *r_u[2], *r_v[2], *w_u[2], *w_v[2], *s_u[2], *s_v[2];
};
void visc_init(const Params& P, DtCoef alpha, const SolveOpts& o, const double* Un, const double* Vn,
               const double* rhs_u, const double* rhs_v, const double* phi, const ViscSolve& w, CGScal* cg,
               const RedSlot& rs, const RedSlot& rs2, int* iters_out, cudaGraphConditionalHandle cond,
               cudaStream_t s);
void visc_iter(const Params& P, DtCoef alpha, const double* phi, const ViscSolve& w, int parity, CGScal* cg,
               const RedSlot& rs, int* iters_out, cudaGraphConditionalHandle cond, cudaStream_t s);
// Precision form (EFSI_PRECISION_MIXED): the same Chronopoulos-Gear CG with FP32
// vectors and FP64 x, inner products and scalars; when the FP32 recurrence has reduced
// the residual by 1e-4, the true residual is recomputed in FP64 from x (iterative
// refinement) and the recurrence restarts from it.  Both calls launch the same kernel;
// device-side phases (iterate, refine, restart) decide what each launch does.
struct ViscMixed {
    float *r_u[2], *r_v[2], *w_u[2], *w_v[2], *s_u[2], *s_v[2];
    float *p_u, *p_v, *dinv_u, *dinv_v, *rR_u, *rR_v;
    // Constant viscosity: the viscous operator A at the cells of the grid's outer ring
    // (walled directions) as 36 weights per cell, kRingWeights (see visc_ring_weights).
    float* ring_w;
};
constexpr int kRingWeights = 36;
// Ring cells (bottom row, top row, left column, right column): 2 Nx + 2 Ny.
__host__ __device__ inline size_t visc_ring_cells(int Nx, int Ny) { return 2 * (size_t)Nx + 2 * (size_t)Ny; }
// Weights of A (rows u and v at a ring cell (i, j), columns u and v at (i + dx, j + dy),
// |dx|, |dy| <= 1) for a constant viscosity, from the general stencil probed with unit
// vectors: ring_w[36 c + 18 o + 9 q + 3 (dy + 1) + dx + 1], o = row, q = column component.
void visc_ring_weights(const Params& P, float* ring_w, cudaStream_t s);
void visc_mx_init(const Params& P, DtCoef alpha, const SolveOpts& o, const double* Un, const double* Vn,
                  const double* rhs_u, const double* rhs_v, const double* phi, const ViscSolve& w,
                  const ViscMixed& m, CGScal* cg, const RedSlot& rs, int* iters_out,
                  cudaGraphConditionalHandle cond, cudaStream_t s);
void visc_mx_iter(const Params& P, DtCoef alpha, const double* phi, const double* rhs_u, const double* rhs_v,
                  const ViscSolve& w, const ViscMixed& m, int parity, CGScal* cg, const RedSlot& rs,
                  int* iters_out, cudaGraphConditionalHandle cond, cudaStream_t s);
// Precision form for a constant viscosity: FP64 iterative refinement around an FP32
// Chebyshev inner solver of the correction equation (I - alpha A) e = r.  The spectrum of
// the free block lies in [1, 1 + alpha g], g the Gershgorin bound of -A, so the inner
// iteration needs no inner products; each inner launch advances four Chebyshev steps on
// a shared-memory tile with a four-cell halo (temporal blocking), and the refinement
// launch applies x += e and recomputes the true FP64 residual, which alone decides
// convergence.  Uses the FP32 arrays of ViscMixed: r and w as the ping-ponged residual
// and direction, s as the ping-ponged correction.
void visc_cheb_init(const Params& P, DtCoef alpha, const SolveOpts& o, const double* Un, const double* Vn,
                    const double* rhs_u, const double* rhs_v, const ViscSolve& w, const ViscMixed& m, CGScal* cg,
                    const RedSlot& rs, int* iters_out, cudaGraphConditionalHandle cond, cudaStream_t s);
void visc_cheb_iter(const Params& P, DtCoef alpha, const double* rhs_u, const double* rhs_v, const ViscSolve& w,
                    const ViscMixed& m, int parity, CGScal* cg, const RedSlot& rs, int* iters_out,
                    cudaGraphConditionalHandle cond, cudaStream_t s);
// Chebyshev steps per inner launch.
constexpr int kChebSteps = 4;
// The polynomial inner solver serves a constant viscosity on grids whose periodic
// extents cover its shared-memory region (40 x 24 cells); other precision-form
// configurations keep the FP32 CG of visc_mx_*.
bool visc_cheb_applies(const Params& P);
// Function attributes of the solver kernels (dynamic shared memory); once per handle,
// before any launch or capture.
cudaError_t solvers_configure();
void visc_enforce_dirichlet(const Params& P, const double* rhs_u, const double* rhs_v, double* x_u, double* x_v,
                            cudaStream_t s);

// ---- resource implicit diffusion (I - alpha*L_D) c = rhs -----------------------------
struct ScalarSolve {
    double *x, *r, *p[2], *Ap, *dinv;
};
void diff_init(const Params& P, DtCoef alpha, const SolveOpts& o, const double* c0, const double* rhs,
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
    float *xf, *xof, *bf;               // the same in FP32 (precision form)
};
// Fast diagonalisation of the level-0 operator K = ax (Tx (x) I) + ay (I (x) Ty) when
// both 1-D operators have one boundary kind per side and power-of-two sizes: Tx, Ty are
// diagonalised by a cosine, sine or Hartley transform computed with a complex FFT.
enum SpecKind : int { SPEC_NN = 0, SPEC_DD = 1, SPEC_ND = 2, SPEC_DN = 3, SPEC_P = 4 };
struct SpecDir {
    int n, logn;        // cells along the direction (a power of two)
    int L, logL;        // complex FFT length (n, or 2n for the odd extension of ND / DN)
    double inv_n, inv_L;  // 1 / n, 1 / L (exact)
    int kind;           // SpecKind
    const double2* w;   // exp(-2 pi i t / L), t < L / 2
    const double2* mk;  // exp(-i pi k / (2 L)), k < L (cosine-transform twiddles)
    const double* mu;   // eigenvalues of the 1-D operator, n
};
struct Spectral {
    bool on;
    SpecDir dx, dy;
    int rows_a, rows_b, rows_c;  // rows (x passes) and modes (y pass) transformed per block (powers of two)
    int lg_a, lg_b, lg_c;        // their base-2 logarithms
    size_t smem_a, smem_b, smem_c;
};
// Padded complex elements of one FFT row of length L in shared memory (one spare per 32).
__host__ __device__ inline int spectral_row(int L) { return L + (L >> 5); }
struct Projection {
    int nlev;
    MGLevel lev[16];
    Spectral sp;          // direct solve of level 0 (used instead of multigrid CG when on)
    double* coarse_inv;   // dense inverse of the coarsest operator (shifted when singular)
    float* coarse_inv_f;  // its FP32 copy (precision form)
    int nc;
    bool nullspace;
    bool mixed;           // precision form: multigrid levels stored and applied in FP32
    int nsm;              // multiprocessors (persistent launch grids)
    // fine-level CG vectors (r, p and s ping-pong between iterations when multigrid
    // levels exist; w = K z, s = w + beta s_old in the Chronopoulos-Gear recurrence)
    double *x, *r[2], *z, *p[2], *Ap, *b, *rhs, *w, *s[2];
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
// Standard PCG p and Kp on a single-level (dense) hierarchy; nothing with multigrid levels.
void proj_matvec(const Params& P, const Projection& pj, int parity, CGScal* cg, const RedSlot& rs, cudaStream_t s);
int proj_matvec_kernels(const Projection& pj);
// CG update fused with the multigrid V-cycle z = M r: Chronopoulos-Gear with levels (p, s,
// x, r updated in the finest down leg; w = K z and both inner products in the finest up
// leg), standard PCG (x += a p, r -= a Kp) on a single dense level.
void proj_update_vcycle(const Params& P, const Projection& pj, int parity, CGScal* cg, const RedSlot& rs,
                        const RedSlot& rs2, int* iters_out, cudaGraphConditionalHandle cond, cudaStream_t s);
void proj_finish(const Params& P, const Projection& pj, const double* G, double* q_out, double* U_out,
                 double* V_out, ProjScal* ps, double* stage_linf, const RedSlot& rs1, const RedSlot& rs2,
                 DevStatus* st, cudaStream_t s);
// Richardson iteration with the exact spectral inverse, x += K^-1 (b - K x), from the
// initial guess and tolerance that proj_cg_init set (no V-cycle is run): one body is
// three kernels (residual and x transform; y transform, eigenvalue division and inverse;
// inverse x transform and update).  Configuring the kernels' shared memory happens in
// spectral_configure (before any capture).
void proj_spectral_init(const Params& P, const Projection& pj, double reltol, int maxiter, const double* q0,
                        CGScal* cg, const ProjScal* ps, const RedSlot& rs, const DevStatus* st, int* iters_out,
                        cudaGraphConditionalHandle cond, cudaStream_t s);
void proj_spectral_iter(const Params& P, const Projection& pj, CGScal* cg, const ProjScal* ps, const RedSlot& rs,
                        int* iters_out, cudaGraphConditionalHandle cond, cudaStream_t s);
cudaError_t spectral_configure(const Spectral& sp);
// ps->v[6] = mean of the solution pj.x with a constant nullspace (0 otherwise).
void proj_mean(const Params& P, const Projection& pj, ProjScal* ps, const RedSlot& rs, cudaStream_t s);
// Kernel launches of proj_update_vcycle and of proj_cg_init (statistics).
int proj_update_vcycle_kernels(const Projection& pj);
int proj_init_kernels(const Projection& pj);
// Algorithmic bytes of one proj_update_vcycle (unique FP64 words read + written once).
double proj_update_vcycle_bytes(const Projection& pj);

}  // namespace efsi
