// efsi_adjoint.cuh — reverse-mode (discrete adjoint) pieces of the IMEX step, host side.
//
// The adjoint sweeps one step backwards (TimeIntegrationIMEX.jl:1152-1256 in reverse):
// for each stage the transposed Jacobian of the explicit tendencies (momentum forcing,
// phase field, structure tensor, viscous operator), the transposed projection and
// viscous solves, and the transposed stage combinations.  Every array named lam_* holds
// the derivative of the objective with respect to the same-named forward quantity.
#pragma once

#include "efsi_common.cuh"
#include "efsi_solvers.cuh"

namespace efsi {

// Forward fields of one stage (full MAC U, V; cell fields).
struct AdjIn {
    const double *U, *V, *phi, *sxx, *syy, *sxy;
};
// Adjoints of one stage's fields (accumulated into, never overwritten).
struct AdjOut {
    double *U, *V, *phi, *sxx, *syy, *sxy;
};
// Adjoints of one stage's tendencies: E_uv and I_uv on the compact rows
// (U(0:Nx-1, :), V(:, 0:Ny-1)), E_phi and E_sigma on cells.
struct AdjTend {
    const double *Eu, *Ev, *Iu, *Iv, *Ephi, *Exx, *Eyy, *Exy;
};
// Adjoints of parameters: tangential wall velocity data (the moving-wall data of
// U bottom/top, Nx+1 entries, and of V left/right, Ny+1 entries) and the elastic
// coefficient G of LinearInternalTensorStress.
struct AdjParam {
    double *bu_bottom, *bu_top, *bv_left, *bv_right;
    double* G;
};
// Scratch of the layered phase-field reverse (psi, cell normals and their adjoints).
struct AdjScratch {
    double *psi, *nx, *ny, *lpsi, *lnx, *lny, *ltxx, *ltyy, *ltxy;
};

// Models the adjoint differentiates; an empty string means supported.
const char* adjoint_unsupported(const Params& P, bool resource, bool growth);

// lam_in += T^T lam_tend at the stage fields `f` (T = the explicit tendencies of
// TimeIntegrationIMEX.jl:944-1071).  `scratch` is overwritten.
void adj_tendencies(const Params& P, const AdjIn& f, const AdjTend& lt, const AdjOut& out, const AdjParam& par,
                    const AdjScratch& scratch, DevStatus* st, cudaStream_t s);

// Transposed projection (Projection.jl:170-307) in two halves around the Poisson
// solve K y = omega:  omega = P0(-Gq^T lam_U) into pj.b (+ its mean into ps->v[10]),
// then lam_pred (compact, 2 x N cells) = lam_U - area D^T (y - mean y) after the solve.
void adj_proj_rhs(const Params& P, const Projection& pj, const double* lamU, const double* lamV, ProjScal* ps,
                  const RedSlot& rs, cudaStream_t s);
void adj_proj_finish(const Params& P, const Projection& pj, const double* lamU, const double* lamV,
                     const ProjScal* ps, double* lam_pu, double* lam_pv, cudaStream_t s);
// The same for full MAC input arrays (efsi_project's input): lam of every face.
void adj_proj_finish_full(const Params& P, const Projection& pj, const double* lamU, const double* lamV,
                          const ProjScal* ps, double* lam_U_in, double* lam_V_in, cudaStream_t s);

// Stage s >= 1 of the velocity path: distribute lam_rhs (compact) over lam_uvn, the
// E/I histories of stages j < s and the viscous boundary data.
void adj_velocity_rhs(const Params& P, int stage, double dt, const double* lr_u, const double* lr_v,
                      double* luvn_u, double* luvn_v, double* const* lEu, double* const* lEv, double* const* lIu,
                      double* const* lIv, const AdjParam& par, cudaStream_t s);
// Stage s >= 1 of the scalar path: the extension reset at phi_s, then the stage
// combination of phi and sigma (TimeIntegrationIMEX.jl:716-740).
void adj_combine(const Params& P, int stage, double dt, const double* phis, const double* lphi,
                 const double* lsxx, const double* lsyy, const double* lsxy, double* lphin, double* lsxn,
                 double* lsyn, double* lsxyn, double* const* lEphi, double* const* lExx, double* const* lEyy,
                 double* const* lExy, cudaStream_t s);
// Start of the step: lam of (U_n, V_n) from the stage-0 field adjoints plus lam_uvn,
// lam of phi_n, and lam of sigma_n through the time-n extension reset.
void adj_step_start(const Params& P, const double* phin, const double* lU0, const double* lV0,
                    const double* luvn_u, const double* luvn_v, const double* lphi0, const double* lphin,
                    const double* lsx0, const double* lsy0, const double* lsxy0, const double* lsxn,
                    const double* lsyn, const double* lsxyn, double* oU, double* oV, double* ophi, double* osxx,
                    double* osyy, double* osxy, cudaStream_t s);
// sigma_n' = the time-n extension reset of sigma_n (k_prepare's reset).
void adj_reset_sigma(const Params& P, const double* phi, const double* sxx, const double* syy, const double* sxy,
                     double* oxx, double* oyy, double* oxy, cudaStream_t s);
// Copy of a stage's fields into the tape slot d_counter (one slot per recorded step).
void adj_record(const Params& P, const int* counter, size_t slot_stride, size_t offset, const double* U,
                const double* V, const double* phi, const double* sxx, const double* syy, const double* sxy,
                double* tape, cudaStream_t s);
// Zero-homogeneous copy of P: every boundary datum reads as 0 (the adjoint solves).
Params homogeneous(const Params& P);

}  // namespace efsi
